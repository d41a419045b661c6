"""The per-bucket launch configurations and their autotuner, on the GPU.

A batch with work units in every bucket (brains of 3,500, 2,000 and 1,200
neurons above the 768-neuron unit, packed small brains, and brains with LP,
Prinz and LFS cells) is stepped under many bucket configurations: 128 or
256 threads per CTA, serial or warp-cooperative delivery, one CTA or a
thread-block cluster per big brain, synapse meta words staged in shared
memory or read from global memory, and list or per-thread integration. Every configuration gives the oracle's
results bit for bit, and the autotuner leaves the brains' state untouched.
"""
import numpy as np
import pytest

from oracle.pyoracle import OracleBrain

pytestmark = pytest.mark.gpu

CALLS = 3


def _batch(nsb):
    W = nsb.workloads
    parts = [W.batched_uneven(seed=40 + k, brains=1, total_neurons=n, total_synapses=3 * n, lo=16, hi=16384,
                              plastic_all=True) for k, n in enumerate([3500, 2000, 1200])]
    parts.append(W.batched_uneven(seed=44, brains=10, total_neurons=10 * 120, total_synapses=10 * 400,
                                  plastic_all=True))
    parts.append(W.parity_mix(seed=45, brains=6, channels=8, outputs=5))   # LP, Prinz and LFS cells
    return W.concat(parts, "buckets")


def _oracle_run(batch, seeds):
    outs, dumps = [], []
    ora = []
    for i in range(batch.brains):
        o = OracleBrain(*batch.brain(i), batch.channels, batch.max_delay)
        o.reset(int(seeds[i]))
        ora.append(o)
    for _ in range(CALLS):
        outs.append(np.stack([o.step(batch.inputs[i], 16, batch.gain, stop_on_nonfinite=False)[1]
                              for i, o in enumerate(ora)]))
    dumps = [o.dump() for o in ora]
    return outs, dumps


def _check(gpu, batch, seeds, want, label, tune_after=None):
    """Reset, step CALLS calls (running the autotuner after call tune_after,
    if given) and compare every output and the final state with the oracle."""
    gpu.reset(seeds)
    for c in range(CALLS):
        out, status = gpu.step(batch.inputs, None, 16, batch.gain)
        np.testing.assert_array_equal(out, want[0][c], err_msg=f"{label}: call {c} outputs")
        if c == tune_after:
            gpu.upload(batch.inputs, np.ones(batch.brains, np.uint8))
            gpu.autotune(16, batch.gain)
    for i in range(batch.brains):
        gn, gs, gt = gpu.dump(i)
        on, os_, ot = want[1][i]
        assert gt == ot
        fa, fb = gn.view(np.float32), on.view(np.float32)
        assert ((gn == on) | (np.isnan(fa) & np.isnan(fb))).all(), f"{label}: brain {i} neuron words differ"
        assert np.array_equal(gs, os_), f"{label}: brain {i} synapse words differ"


def test_every_bucket_configuration_matches_the_oracle(nsb, monkeypatch):
    monkeypatch.setenv("NSB_UNIT_SLOTS", "3")       # 768-neuron units, as in full batches
    batch = _batch(nsb)
    seeds = np.arange(batch.brains, dtype=np.uint32) * 7 + 3
    want = _oracle_run(batch, seeds)
    gpu = nsb.GpuBatch.from_rows(batch)
    try:
        bk = gpu.buckets()
        assert [b["units"] > 0 for b in bk] == [True] * 5, bk
        assert [b["max_neurons"] for b in bk[:3]] == [3500, 2000, 1200]
        _check(gpu, batch, seeds, want, "default")
        configs = [(256, 0, False, 6144, 1), (128, 1, True, 6144, 1), (128, 0, True, 0, 1), (256, 1, False, 0, 0),
                   (128, 1, False, 32768, 1), (256, 0, True, 32768, 1), (128, 0, False, 64, 0),
                   (256, 1, True, 6144, 1), (256, 0, False, 6144, 0), (128, 1, False, 6144, 0)]
        for block, coop, clustered, cap, lst in configs:
            for b in range(4):
                gpu.set_bucket(b, block, coop, (8, 4, 2, 1)[b] if clustered else 1, cap, lst)
            got = gpu.buckets()
            label = f"block {block} coop {coop} clustered {clustered} meta {cap} list {lst}"
            assert all(g["block"] == block for g in got[:4]), label
            _check(gpu, batch, seeds, want, label)
        # heavy units on 128-thread CTAs: four warps share the LP/Prinz pool
        gpu.set_bucket(4, 128, 0, 1, 6144, 1)
        assert gpu.buckets()[4]["block"] == 128
        _check(gpu, batch, seeds, want, "heavy block 128")
        gpu.set_bucket(4, 256, 0, 1, 6144, 1)
        with pytest.raises(RuntimeError):
            gpu.set_bucket(3, 256, 0, 2, 6144)          # packed units have no cluster form
        with pytest.raises(RuntimeError):
            gpu.set_bucket(0, 192, 0, 1, 6144)          # 128 or 256 threads only
        # the autotuner picks per bucket, between calls, leaving the state untouched
        _check(gpu, batch, seeds, want, "tuned", tune_after=0)
        _check(gpu, batch, seeds, want, "after tuning")
    finally:
        gpu.close()
