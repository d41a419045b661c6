"""Checkpoint records in the reference world simulator's layout.

CPU: the record layout and the layout hash equal the reference build's
(src/main.cu:164-177, src/checkpoint_impl.cuh:20-32), read from the reference
compiled here when oracle/_ref is present, and from the recorded values
otherwise.
GPU: export -> import into a fresh batch of the same genomes -> both batches
continue bit-identically; exported states equal the oracle's; records whose
genes do not describe the batch are refused.
"""
import ctypes as ct

import numpy as np
import pytest

from oracle.pyoracle import OracleBrain, ref_world_lib

LAYOUT_HASH = 0x2B1CD1C766EEBF82
# offsetof(CheckpointNeuron, gene/state/pending_exc/pending_inh/mod_event_tick/spike_history),
# offsetof(CheckpointSynapse, gene/state)
OFFSETS = [16, 140, 260, 276, 280, 328, 12, 56]


def test_layout_hash_matches_reference(nsb):
    lib = nsb.native.library()
    assert lib.nsb_checkpoint_layout() == LAYOUT_HASH
    ref = ref_world_lib()
    if ref is None:
        pytest.skip("reference world build (oracle/_ref) absent; recorded values checked above")
    v = (ct.c_uint64 * 20)()
    h = ct.c_uint64()
    o = (ct.c_uint64 * 8)()
    ref.ref_world_layout(v, ct.byref(h), o)
    assert h.value == LAYOUT_HASH
    assert list(o) == OFFSETS
    assert v[15] == nsb.native.CHECKPOINT_NEURON_BYTES and v[16] == nsb.native.CHECKPOINT_SYNAPSE_BYTES


def _state_fields(rec):
    """NeuronState bytes of a CheckpointNeuron record (offset 140, 120 bytes)."""
    return rec[:, 140:260]


@pytest.mark.gpu
def test_checkpoint_round_trip(nsb, oracle_built):
    batch = nsb.workloads.parity_mix(brains=10)
    a = nsb.GpuBatch.from_rows(batch)
    seeds = np.arange(10, dtype=np.uint32) + 40
    a.reset(seeds)
    for _ in range(3):
        a.step(batch.inputs, None, 16, batch.gain)
    nr, sr, ticks = a.checkpoint_export()
    assert nr.shape == (len(batch.neuron_rows), 344) and sr.shape == (len(batch.synapse_rows), 136)
    assert (ticks == 48).all()
    slots = nr[:, 0:4].copy().view(np.int32).ravel()
    assert (slots == np.arange(len(nr))).all()
    b = nsb.GpuBatch.from_rows(batch)
    b.reset(seeds + 1000)                      # different state, replaced by the import
    b.checkpoint_import(nr, sr, ticks)
    nr2, sr2, ticks2 = b.checkpoint_export()
    np.testing.assert_array_equal(nr, nr2)
    np.testing.assert_array_equal(sr, sr2)
    for _ in range(3):
        oa, sa = a.step(batch.inputs, None, 16, batch.gain)
        ob, sb = b.step(batch.inputs, None, 16, batch.gain)
        np.testing.assert_array_equal(oa, ob)
        np.testing.assert_array_equal(sa, sb)
    for i in range(batch.brains):
        np.testing.assert_array_equal(a.dump(i)[0], b.dump(i)[0])
        np.testing.assert_array_equal(a.dump(i)[1], b.dump(i)[1])
    # the exported membrane voltages equal the oracle's after the same 3 calls
    ng, sg, mo = batch.brain(0)
    o = OracleBrain(ng, sg, mo, batch.channels, batch.max_delay)
    o.reset(int(seeds[0]))
    for _ in range(3):
        o.step(batch.inputs[0], 16, batch.gain, stop_on_nonfinite=False)
    v = nr[: len(ng), 140:144].copy().view(np.float32).ravel()
    np.testing.assert_array_equal(v.view(np.uint32), o.dump()[0][:, 0])
    # records that do not describe the batch are refused
    bad = nr.copy()
    bad[0, 16:20] = np.frombuffer(np.float32(999.0).tobytes(), np.uint8)   # gene.cap
    with pytest.raises(RuntimeError, match="genes differ"):
        b.checkpoint_import(bad, sr, ticks)
    with pytest.raises(RuntimeError, match="counts differ"):
        b.checkpoint_import(nr[:-1], sr, ticks)
    a.close(); b.close()
