import numpy as np


def test_philox4x32_10_known_answers(nsb):
    """Known-answer vectors of Philox4x32-10 (Salmon et al., SC'11)."""
    P = nsb.workloads.philox4x32
    def h(x):
        return [int(v) for v in x]
    assert h(P(np.zeros(4, np.uint32), (0, 0))) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert h(P(np.full(4, 0xffffffff, np.uint32), (0xffffffff, 0xffffffff))) == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert h(P(np.array([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], np.uint32),
               (0xa4093822, 0x299f31d0))) == [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def test_plain_small_shape(nsb):
    b = nsb.workloads.plain_small()
    assert b.brains == 64 and len(b.neuron_rows) == 64 * 48 and len(b.synapse_rows) == 64 * 600
    pre, post = b.synapse_rows[:, 0], b.synapse_rows[:, 1]
    assert (pre != post).all()
    d = b.synapse_rows[:, 4]
    assert d.min() == 1 and d.max() == 8
    assert b.outputs == 5 and b.channels == 12


def test_uneven_sizes_fill_the_pools(nsb):
    s = nsb.workloads.uneven_sizes(2, 32768, 4194304, 96.0, 1.0, 16, 4096)
    assert s.sum() == 4194304 and s.min() >= 16 and s.max() <= 4096 and len(s) == 32768


def test_uneven_small_is_deterministic(nsb):
    a = nsb.workloads.batched_uneven(brains=64, total_neurons=8192, total_synapses=16384)
    b = nsb.workloads.batched_uneven(brains=64, total_neurons=8192, total_synapses=16384)
    assert np.array_equal(a.synapse_rows, b.synapse_rows)
    assert len(a.synapse_rows) == 16384 and a.synapse_rows[:, 4].max() == 16


def test_lp_prinz_bench_batches(nsb):
    """The LP/Prinz batches the benchmark times (bench.py --workload
    heavy_smoke / heavy_founders): their sizes and cell counts, and, in the
    founders, warps of list order that own several LP cells (the case the
    heavy kernels' per-CTA pool balances)."""
    W = nsb.workloads
    smoke = W.parity_mix(seed=3, brains=4)
    t = smoke.neuron_rows[:, 0].astype(int)
    assert smoke.brains == 4 and len(t) == 182
    assert int(((t == 2) | (t == 3)).sum()) == 43
    founders = W.world_founders(seed=2, founders=256, heavy_types=True)
    t = founders.neuron_rows[:, 0].astype(int)
    assert founders.brains == 256 and len(t) == 16310
    assert 200 < (t == 2).sum() < 330 and 200 < (t == 3).sum() < 330 and (t == 6).sum() > 150
    lp_per_warp = [int((t[w:w + 32] == 2).sum()) for w in range(0, len(t), 32)]
    assert max(lp_per_warp) >= 4
