"""GPU parity: the CUDA engine, called through the C ABI (libns_b200.so),
against the C oracle with correctly rounded exp/log — bit-exact in every state
word, motor output and status, over multi-call runs with masks and resets.
The oracle itself is pinned bit-exactly to the reference's own host executor
(tests/test_oracle.py, tests/test_golden.py)."""
import numpy as np
import pytest

from oracle.pyoracle import OracleBrain

pytestmark = pytest.mark.gpu


def _oracles(batch, delay):
    out = []
    for i in range(batch.brains):
        ng, sg, mo = batch.brain(i)
        out.append(OracleBrain(ng, sg, mo, batch.channels, delay))
    return out


# Integer words of the canonical neuron dump (total spikes, spike, receptor
# RNG, history); every other word is binary32.
_INT_WORDS = [26, 27, 29, 30, 31]


def _nan_equivalent(a, b, int_words=()):
    """Bitwise equality, except that two NaNs compare equal: IEEE 754 leaves
    NaN payloads unspecified and the GPU returns one canonical NaN."""
    fa, fb = a.view(np.float32), b.view(np.float32)
    both_nan = np.isnan(fa) & np.isnan(fb)
    if len(int_words):
        both_nan[:, int_words] = False
    return (a == b) | both_nan


def _assert_brain_equal(gpu, ora, i, what):
    gn, gs, gt = gpu.dump(i)
    on, os_, ot = ora.dump()
    assert gt == ot, f"{what}: brain {i} tick {gt} != {ot}"
    bad = np.argwhere(~_nan_equivalent(gn, on, _INT_WORDS))
    assert bad.size == 0, f"{what}: brain {i} neuron words differ at {bad[:6].tolist()}"
    bad = np.argwhere(gs != os_)
    assert bad.size == 0, f"{what}: brain {i} synapse words differ at {bad[:6].tolist()}"


def run_parity(nsb, batch, calls, ticks=16, mask_fn=None, reset_at=(), seeds=None, check_every=1, block=0,
               gain=None, delivery=None, autotune_at=(), pulse=None):
    delay = batch.max_delay
    gain = batch.gain if gain is None else gain
    gpu = nsb.GpuBatch.from_rows(batch, block=block)
    if delivery is not None:
        gpu.set_delivery(delivery)
    ora = _oracles(batch, delay)
    if pulse is not None:
        gpu.set_modulation(*pulse)
        for o in ora:
            o.set_pulse(*pulse)
    seeds = np.arange(batch.brains, dtype=np.uint32) * 17 + 20 if seeds is None else seeds
    gpu.reset(seeds)
    for i, o in enumerate(ora):
        o.reset(int(seeds[i]))
    inputs = batch.inputs
    for c in range(calls):
        mask = np.ones(batch.brains, np.uint8) if mask_fn is None else mask_fn(c)
        if c in reset_at:
            rmask = (np.arange(batch.brains) % 3 == c % 3).astype(np.uint8)
            gpu.reset(seeds + c, rmask)
            for i, o in enumerate(ora):
                if rmask[i]:
                    o.reset(int(seeds[i] + c))
        if c in autotune_at:
            gpu.upload(inputs, mask)
            gpu.autotune(ticks, gain)      # times both modes; must leave the state untouched
        out, status = gpu.step(inputs, mask, ticks, gain)
        for i, o in enumerate(ora):
            if mask[i]:
                rc, oo, _ = o.step(inputs[i], ticks, gain, stop_on_nonfinite=False)
                assert status[i] == rc, f"call {c} brain {i} status {status[i]} != {rc}"
                np.testing.assert_array_equal(out[i], oo, err_msg=f"call {c} brain {i} outputs")
            else:
                assert not out[i].any() and status[i] == 0
        if (c + 1) % check_every == 0 or c == calls - 1:
            for i, o in enumerate(ora):
                _assert_brain_equal(gpu, o, i, f"call {c}")
    return gpu, ora


@pytest.mark.parametrize("delivery", [False, True])
def test_parity_mix_every_profile_and_cell_type(nsb, delivery):
    batch = nsb.workloads.parity_mix(brains=16)
    gpu, _ = run_parity(nsb, batch, calls=8, mask_fn=lambda c: np.array(
        [1 if (i + c) % 4 else 0 for i in range(batch.brains)], np.uint8), reset_at=(3, 6), delivery=delivery)
    gpu.close()


@pytest.mark.parametrize("warp_cells", ["0", "4", "32"])
def test_lp_and_prinz_cells_in_every_form(nsb, monkeypatch, warp_cells):
    """A heavy unit's pooled LP and Prinz cells stepped each on its own lane
    (0), and on whole warps, a share of the pool each (4, 32): every form
    gives the oracle's bits."""
    monkeypatch.setenv("NSB_WARP_CELLS", warp_cells)
    batch = nsb.workloads.parity_mix(seed=7, brains=12, heavy_types=True)
    gpu, _ = run_parity(nsb, batch, calls=4)
    gpu.close()


@pytest.mark.parametrize("delivery", [False, True])
def test_plasticity_heavy_triplet_dopamine(nsb, delivery):
    """Every synapse on profile 6 (triplet STDP into a dopamine eligibility
    trace), 30% of hidden neurons driven to ~60 Hz, a global dopamine pulse
    every 50 ms; 10 calls = 160 ticks, so pulses fall inside calls."""
    batch = nsb.workloads.plasticity_heavy(brains=32, total_neurons=32 * 96, total_synapses=32 * 192)
    gpu, ora = run_parity(nsb, batch, calls=10, check_every=5, delivery=delivery,
                          pulse=(batch.meta["pulse_period"], batch.meta["pulse_mod"]))
    changed = 0
    for i, o in enumerate(ora):
        w = o.dump()[1][:, 0].view(np.float32)
        changed += int((w != batch.brain(i)[1][:, 2]).sum())
    assert changed > 0
    gpu.close()


def test_autotune_leaves_state_untouched(nsb):
    batch = nsb.workloads.plain_small(brains=12)
    gpu, _ = run_parity(nsb, batch, calls=6, autotune_at=(2, 4))
    gpu.close()


def test_plain_small_config_bitexact(nsb):
    """The plain-small configuration as specified: 64 brains x 48 neurons, 600
    synapses each, 200 world steps x 16 ticks = 3,200 ticks; outputs and
    status every step, full state every 50 steps."""
    batch = nsb.workloads.plain_small()
    gpu, ora = run_parity(nsb, batch, calls=200, check_every=50)
    gpu.close()


def test_plain_small_2000_ticks_bitexact(nsb):
    batch = nsb.workloads.plain_small(brains=16)
    gpu, ora = run_parity(nsb, batch, calls=125, check_every=25)
    assert sum(o.dump()[0][:, 26].astype(np.int64).sum() for o in ora) > 0


@pytest.mark.parametrize("delivery", [False, True])
def test_extended_delays_and_large_brains(nsb, delivery):
    """Delays up to 16 ms (ring of 17 in the oracle) and brains above the CTA
    size, which take the multi-neuron-per-thread path."""
    batch = nsb.workloads.batched_uneven(brains=48, total_neurons=48 * 160, total_synapses=48 * 320)
    assert max(n for n, _ in zip(np.diff(batch.neuron_offsets), range(99))) > 256
    gpu, _ = run_parity(nsb, batch, calls=6, check_every=2, delivery=delivery)
    st = gpu.stats()
    assert st["big_units"] >= 1


def test_block_128_matches(nsb):
    batch = nsb.workloads.parity_mix(brains=10, heavy_types=False)
    run_parity(nsb, batch, calls=5, block=128)


def test_single_brain_ns_step(nsb):
    batch = nsb.workloads.parity_mix(brains=4)
    for i in range(4):
        ng, sg, mo = batch.brain(i)
        b = nsb.Brain(ng, sg, mo, batch.channels)
        o = OracleBrain(ng, sg, mo, batch.channels, 8)
        on = np.arange(len(ng), dtype=np.uint32) * 3 + 1
        os_ = np.arange(len(sg), dtype=np.uint32) * 5 + 2
        b.original_indices(on, os_); o.original_indices(on, os_)
        b.reset(2 ** 31 + 47); o.reset(2 ** 31 + 47)
        for c in range(6):
            out = b.step(batch.inputs[i], 1 + 3 * c, 150.0)
            rc, oo, _ = o.step(batch.inputs[i], 1 + 3 * c, 150.0)
            assert rc == 0
            np.testing.assert_array_equal(out, oo)
        gn, gs, gt = b.dump()
        on_, os2, ot = o.dump()
        np.testing.assert_array_equal(gn, on_)
        np.testing.assert_array_equal(gs, os2)
        assert gt == ot
        b.close()


def test_nonfinite_voltage_reports_status(nsb):
    """An LP cell (type 2) driven by an enormous tonic current integrates to a
    non-finite voltage; the batch reports status -1 for that brain only and
    keeps stepping the others (gym_adapter/gpu.cu:49)."""
    W = nsb.workloads
    ng = np.array([[2, 0, 1, 0, 0, 1, 1, -42, 0, 0], [0, -1, 1, 0, 0, 1, 1, -52, 0, 0]], np.float32)
    sg = np.array([[0, 1, 3.0, 1, 2, 0, .5, 100, 0, 1, 0]], np.float32)
    rows_n = np.concatenate([ng, ng]); rows_s = np.concatenate([sg, sg])
    batch = W.Batch(rows_n, rows_s, np.array([0, 2, 4]), np.array([0, 1, 2]), np.array([[1], [1]], np.int32), 1, 8,
                    "nonfinite", np.array([[1.0], [0.0]], np.float32), 3.0e38)
    gpu = nsb.GpuBatch.from_rows(batch)
    ora = _oracles(batch, 8)
    gpu.reset(np.array([3, 4], np.uint32))
    ora[0].reset(3); ora[1].reset(4)
    out, status = gpu.step(batch.inputs, None, 4, 3.0e38)
    for i, o in enumerate(ora):
        rc, oo, _ = o.step(batch.inputs[i], 4, 3.0e38, stop_on_nonfinite=False)
        assert status[i] == rc
        np.testing.assert_array_equal(out[i], oo)
    assert status.tolist() == [-1, 0]
    for i, o in enumerate(ora):
        _assert_brain_equal(gpu, o, i, "nonfinite")


def test_validation_messages(nsb):
    batch = nsb.workloads.parity_mix(brains=2, heavy_types=False)
    gpu = nsb.GpuBatch.from_rows(batch)
    gpu.reset(np.zeros(2, np.uint32))
    with pytest.raises(RuntimeError, match="Invalid neural integration interval"):
        gpu.step(batch.inputs, None, 0)
    bad = batch.inputs.copy(); bad[0, 0] = 1.5
    with pytest.raises(RuntimeError, match="Invalid encoded observation"):
        gpu.step(bad, None, 4)
    # a masked-out brain's observation is not validated (gym_adapter/gpu.cu:118)
    gpu.step(bad, np.array([0, 1], np.uint8), 4)


def test_graph_replay_matches_host_step(nsb):
    batch = nsb.workloads.plain_small(brains=8)
    a = nsb.GpuBatch.from_rows(batch)
    b = nsb.GpuBatch.from_rows(batch)
    seeds = np.arange(8, dtype=np.uint32)
    a.reset(seeds); b.reset(seeds)
    b.upload(batch.inputs, np.ones(8, np.uint8))
    for _ in range(5):
        out_a, st_a = a.step(batch.inputs, None, 16, 230.0)
        b.step_graph(16, 230.0)
        out_b, st_b = b.download()
        np.testing.assert_array_equal(out_a, out_b)
        np.testing.assert_array_equal(st_a, st_b)
    for i in range(8):
        np.testing.assert_array_equal(a.dump(i)[0], b.dump(i)[0])
        np.testing.assert_array_equal(a.dump(i)[1], b.dump(i)[1])


def test_maze_brain_step_matches_gpu_step(nsb):
    """ns_maze_brain_step (gym_adapter/maze_gpu.cu:85-90) steps the batch on a
    device maze batch's encoded observations; the reference's MazeBatch is
    mirrored here by its leading fields. Same results as ns_gpu_step on the
    same observations."""
    import ctypes as ct
    import torch
    batch = nsb.workloads.parity_mix(brains=6, channels=294, heavy_types=False)
    a = nsb.GpuBatch.from_rows(batch)
    b = nsb.GpuBatch.from_rows(batch)
    seeds = np.arange(6, dtype=np.uint32) + 3
    a.reset(seeds); b.reset(seeds)
    rng = np.random.default_rng(1)

    class Maze(ct.Structure):
        _fields_ = [("count", ct.c_int), ("grid", ct.c_void_p), ("objects", ct.c_void_p), ("agents", ct.c_void_p),
                    ("observations", ct.c_void_p), ("encoded", ct.c_void_p), ("lookup", ct.c_void_p)]
    lib = nsb.native.library()
    for c in range(4):
        x = rng.uniform(0, 1, (6, 294)).astype(np.float32)
        mask = np.array([1, 1, 0, 1, 1, 1], np.uint8)
        enc = torch.from_numpy(x).cuda()
        torch.cuda.synchronize()
        maze = Maze(6, None, None, None, None, enc.data_ptr(), None)
        out = np.zeros((6, batch.outputs), np.float32)
        status = np.zeros(6, np.int32)
        rc = lib.ns_maze_brain_step(ct.byref(maze), a.ptr, mask.ctypes.data_as(ct.POINTER(ct.c_uint8)), 16, 230.0,
                                    out.ctypes.data_as(ct.POINTER(ct.c_float)),
                                    status.ctypes.data_as(ct.POINTER(ct.c_int32)))
        assert rc == 0, lib.ns_error().decode()
        ob, sb = b.step(x, mask, 16, 230.0)
        np.testing.assert_array_equal(out, ob)
        np.testing.assert_array_equal(status, sb)
    for i in range(6):
        np.testing.assert_array_equal(a.dump(i)[0], b.dump(i)[0])
    bad = Maze(5, None, None, None, None, enc.data_ptr(), None)
    assert lib.ns_maze_brain_step(ct.byref(bad), a.ptr, mask.ctypes.data_as(ct.POINTER(ct.c_uint8)), 16, 230.0,
                                  out.ctypes.data_as(ct.POINTER(ct.c_float)),
                                  status.ctypes.data_as(ct.POINTER(ct.c_int32))) == -1
    assert lib.ns_error().decode() == "Maze/brain dimensions differ"
    a.close(); b.close()


def test_handles_from_the_reference_library(nsb):
    """ns_gpu_create accepts Brain handles made by the reference's own host
    library (gym_adapter/native.cpp built from its sources, exp/log correctly
    rounded): the batch then steps bit-identically to those brains stepped on
    the reference host executor."""
    import ctypes as ct
    from oracle.pyoracle import RefBrain, ref_lib
    if ref_lib(cr=True) is None:
        pytest.skip("reference host build (oracle/_ref) absent")
    batch = nsb.workloads.parity_mix(brains=6, heavy_types=True)
    makers = [RefBrain(*batch.brain(i), batch.channels, cr=True) for i in range(6)]
    lib = nsb.native.library()
    arr = (ct.c_void_p * 6)(*[m.ptr for m in makers])
    ptr = lib.ns_gpu_create(arr, 6)
    assert ptr, lib.ns_error().decode()
    gpu = nsb.GpuBatch(ptr, 6, batch.channels, batch.outputs,
                       [(len(batch.brain(i)[0]), len(batch.brain(i)[1])) for i in range(6)])
    for m in makers:                     # the batch deep-copied the genomes
        m.close()
    seeds = np.arange(6, dtype=np.uint32) + 11
    gpu.reset(seeds)
    refs = [RefBrain(*batch.brain(i), batch.channels, cr=True) for i in range(6)]
    for i, r in enumerate(refs):
        r.reset(int(seeds[i]))
    for c in range(5):
        out, status = gpu.step(batch.inputs, None, 16, batch.gain)
        for i, r in enumerate(refs):
            rc, ro, _ = r.step(batch.inputs[i], 16, batch.gain)
            assert status[i] == rc
            np.testing.assert_array_equal(out[i], ro)
    for i, r in enumerate(refs):
        gn, gs, gt = gpu.dump(i)
        rn, rs, rt = r.dump()
        assert gt == rt
        assert (_nan_equivalent(gn, rn, _INT_WORDS)).all()
        np.testing.assert_array_equal(gs, rs)
    gpu.close()


def test_edge_sizes(nsb):
    """A one-neuron brain without synapses, a brain without synapses, and a
    brain at the maximum size (16,384 neurons), in one batch."""
    W = nsb.workloads
    big = W.batched_uneven(seed=9, brains=1, total_neurons=16384, total_synapses=32768, lo=16, hi=16384)
    tiny_n = np.array([[5, 0, 1, 0, 0, 1, 1, -40, 30, 2]], np.float32)
    lone_n = np.array([[0, -1, 1, 0, 0, 1, 1, -52, 0, 0], [5, 1, 1, 0, 0, 1, 1, -40, 20, 2],
                       [1, -1, 1, 1, 0, 1, 1, -42, 0, 0]], np.float32)
    ch = big.channels
    rows_n = np.concatenate([tiny_n, lone_n, big.neuron_rows])
    rows_s = big.synapse_rows
    no = np.array([0, 1, 4, 4 + len(big.neuron_rows)])
    so = np.array([0, 0, 0, len(rows_s)])
    motors = np.array([[0] * big.outputs, [0] * big.outputs, list(big.motors[0])], np.int32)
    inputs = np.ones((3, ch), np.float32)
    batch = W.Batch(rows_n, rows_s, no, so, motors, ch, big.max_delay, "edge_sizes", inputs, 230.0, {})
    gpu, _ = run_parity(nsb, batch, calls=3)
    assert gpu.stats()["max_unit_neurons"] == 16384
    gpu.close()


def _concat(batches, name):
    """One Batch of all brains of `batches`, in order."""
    rows_n = np.concatenate([b.neuron_rows for b in batches])
    rows_s = np.concatenate([b.synapse_rows for b in batches])
    no, so = [0], [0]
    for b in batches:
        no.extend((no[-1] + np.asarray(b.neuron_offsets[1:]) - b.neuron_offsets[0]).tolist())
        so.extend((so[-1] + np.asarray(b.synapse_offsets[1:]) - b.synapse_offsets[0]).tolist())
    no, so = np.asarray(no, np.int64), np.asarray(so, np.int64)
    motors = np.concatenate([b.motors for b in batches]).astype(np.int32)
    inputs = np.concatenate([b.inputs for b in batches]).astype(np.float32)
    b0 = batches[0]
    return type(b0)(rows_n, rows_s, no, so, motors, b0.channels, b0.max_delay, name, inputs, b0.gain, {})


@pytest.mark.parametrize("delivery,cluster", [(False, "1"), (True, "1"), (True, "0")])
def test_big_brains_on_thread_block_clusters(nsb, monkeypatch, delivery, cluster):
    """Brains above the 768-neuron unit are stepped by clusters of 2, 4 and 8
    CTAs exchanging spikes through distributed shared memory (and, with
    NSB_CLUSTER=0, by one CTA each): sizes 1,000
    (2 CTAs), 2,000 (4), 3,500 and 6,500 (8, with 832 neurons per CTA), with
    pair STDP on every excitatory pair, next to small brains, under masks and
    partial resets."""
    W = nsb.workloads
    parts = [W.batched_uneven(seed=20 + k, brains=1, total_neurons=n, total_synapses=3 * n, lo=16, hi=16384,
                              plastic_all=True) for k, n in enumerate([1000, 2000, 3500, 6500])]
    parts.append(W.batched_uneven(seed=30, brains=6, total_neurons=6 * 120, total_synapses=6 * 300, plastic_all=True))
    batch = _concat(parts, "big_brains")
    monkeypatch.setenv("NSB_CLUSTER", cluster)     # "0": the same brains on one CTA each
    monkeypatch.setenv("NSB_UNIT_SLOTS", "3")      # 768-neuron units, as in full batches
    gpu, _ = run_parity(nsb, batch, calls=6, check_every=2, delivery=delivery, reset_at=(3,),
                        mask_fn=lambda c: np.array([1 if (i + c) % 5 else 0 for i in range(batch.brains)], np.uint8))
    assert gpu.stats()["big_units"] == 4
    gpu.close()
