"""CPU checks of the world neural stage's oracle and layouts.

- The record layouts the world stage reads (Animal, PlasticityCohort and the
  neural records) agree between the library, the oracle, the Python dtypes and
  the reference simulator as built from its sources.
- The oracle's world restatement (or_world_step: the reference world loop's
  tick-major order, src/main.cu:659-801, with per-branch sums in each animal's
  synapse list order) equals the Gym-ordered oracle (pinned bit for bit to the
  reference host executor) on a population where the two semantics coincide:
  contiguous lists in row order, receptor cells only on channels 0-5, one
  neuron per motor port, no frozen cohort, age = step. Every state word,
  history slot and motor count is compared.
"""
import ctypes as ct

import numpy as np
import pytest

from oracle.pyoracle import OracleBrain, oracle_lib, oracle_records, ref_world_lib, world_homeostasis, world_step


def _fields_equal(a, b, dtype, label):
    for name in dtype.names:
        x, y = a[name], b[name]
        if x.dtype.kind == "f":
            same = np.array_equal(x.view(np.uint32 if x.dtype.itemsize == 4 else np.uint64),
                                  y.view(np.uint32 if y.dtype.itemsize == 4 else np.uint64))
        else:
            same = np.array_equal(x, y)
        if not same:
            bad = np.nonzero(~np.all((x == y).reshape(len(x), -1), axis=1))[0]
            raise AssertionError(f"{label}.{name} differs at {bad[:10]}")


def test_world_layouts(nsb, oracle_built):
    lib = nsb.native.library()
    got = (ct.c_uint64 * 10)()
    assert lib.nsb_world_layout(got) == 10
    o = (ct.c_uint64 * 14)()
    assert oracle_lib().or_world_layout(o) == 14
    got, o = list(got), list(o)
    assert got[:2] == [472, 80] and o[:2] == [472, 80]
    assert o[2:6] == [124, 120, 40, 80]
    assert got[2:] == o[6:]
    W = nsb.world
    assert W.ANIMAL.itemsize == 472 and W.COHORT.itemsize == 80
    assert [W.ANIMAL.fields[f][1] for f in ("id", "age", "alive", "neuron_head", "synapse_head", "neuron_count",
                                            "synapse_count")] == got[2:9]
    assert W.COHORT.fields["frozen"][1] == got[9]
    assert (W.NEURON_GENE.itemsize, W.NEURON_STATE.itemsize, W.SYNAPSE_GENE.itemsize,
            W.SYNAPSE_STATE.itemsize) == (124, 120, 40, 80)
    ref = ref_world_lib()
    if ref is not None and hasattr(ref, "ref_world_animal_layout"):
        r = (ct.c_uint64 * 10)()
        ref.ref_world_animal_layout.argtypes = [ct.POINTER(ct.c_uint64)]
        assert ref.ref_world_animal_layout(r) == 10
        assert list(r) == got


@pytest.mark.parametrize("heavy", [False, True])
def test_world_restatement_equals_gym_oracle(nsb, oracle_built, heavy):
    batch = nsb.workloads.world_founders(seed=3, founders=5, heavy_types=heavy)
    B = batch.brains
    seeds = (np.arange(B) * 17 + 5).astype(np.uint32)
    gym = []
    for b in range(B):
        o = OracleBrain(*batch.brain(b), batch.channels, batch.max_delay)
        o.reset(int(seeds[b]))
        gym.append(o)
    pools = nsb.world.place_population(batch, *oracle_records(batch, seeds), receptor_baseline=0.0)
    steps = 12
    outs = np.zeros((B, 5), np.float32)
    for k in range(1, steps + 1):
        for b, o in enumerate(gym):
            rc, out, _ = o.step(batch.inputs[b], 16, 230.0, stop_on_nonfinite=False)
            outs[b] += out
        world_step(pools, k)
        pools.animals["age"][:B] = k
        world_homeostasis(pools)
    W = nsb.world
    assert np.array_equal(pools.motors[:B].astype(np.float32), outs)
    assert outs.sum() > 0
    no, so = batch.neuron_offsets, batch.synapse_offsets
    for b, o in enumerate(gym):
        ng, ns, sg, ss = o.records()
        _fields_equal(pools.neuron_state[no[b]:no[b + 1]], ns.view(W.NEURON_STATE).reshape(-1), W.NEURON_STATE,
                      f"brain {b} neuron")
        _fields_equal(pools.synapse_state[so[b]:so[b + 1]], ss.view(W.SYNAPSE_STATE).reshape(-1), W.SYNAPSE_STATE,
                      f"brain {b} synapse")
    # accumulators consumed, history holds the last 9 ticks' spikes
    assert not pools.pending_exc.any() and not pools.pending_inh.any()
    assert pools.spike_history.any()


def test_world_oracle_rejects_bad_delay(nsb, oracle_built):
    batch = nsb.workloads.world_founders(seed=4, founders=2)
    pools = nsb.world.place_population(batch, *oracle_records(batch, np.array([1, 2], np.uint32)))
    pools.synapses["delay"][3] = 9
    with pytest.raises(ValueError):
        world_step(pools, 1)
