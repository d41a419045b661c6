"""Parity at the full sizes of the measured workloads, over 2,000 ticks.

- Batched uneven brains at full pools: 32,768 brains, 4,194,304 neurons,
  8,388,608 synapses, delays 1-16 (the benchmark's batch, seed 2), stepped
  for 125 calls of 16 ticks, in both delivery modes and with big brains on
  thread-block clusters.
- Plasticity-heavy full pools: the same pool sizes, every synapse on triplet
  STDP with dopamine eligibility, 30 % of neurons bursting, a dopamine pulse
  every 50 ms.
- The world's founding population: 2,048 founders, 125 world steps (2,000
  ticks) of the world neural stage with fresh senses every step.

The whole batch runs on the GPU. Brains never interact within a step, so a
sample of them is stepped by the oracle (correctly rounded exp/log, pinned to
the reference's host executor) in worker processes while the GPU runs: every
64th brain by size plus the largest brains. Every call's motor outputs and
status, and the final state words of every sampled brain, must be equal bit
for bit. The world gate splits the living animals into disjoint subsets, one
oracle process each, and compares every step's motor counts of every animal
and every pool word at the end.
"""
import numpy as np
import pytest

from oracle.pyoracle import SampledOracle, SubsetWorldOracle

pytestmark = pytest.mark.gpu

CALLS = 125          # 125 calls x 16 ticks = 2,000 ticks
INT_WORDS = [26, 27, 29, 30, 31]


def _sample(batch, stride=64, largest=6):
    sizes = np.diff(batch.neuron_offsets)
    order = np.argsort(sizes, kind="stable")
    return np.unique(np.concatenate([order[::stride], order[-largest:]]))


def _nan_equivalent(a, b):
    fa, fb = a.view(np.float32), b.view(np.float32)
    both = np.isnan(fa) & np.isnan(fb)
    both[:, INT_WORDS] = False
    return (a == b) | both


def _gpu_run(nsb, batch, seeds, idx, delivery=None, pulse=None):
    """Steps the whole batch for CALLS calls; returns the sampled brains'
    outputs (calls x sample x outputs), status (calls x sample), final dumps,
    the engine's stats and the batch's total motor spikes."""
    gpu = nsb.GpuBatch.from_rows(batch)
    try:
        if delivery is not None:
            gpu.set_delivery(delivery)
        if pulse is not None:
            gpu.set_modulation(*pulse)
        gpu.reset(seeds)
        outs = np.zeros((CALLS, len(idx), batch.outputs), np.float32)
        status = np.zeros((CALLS, len(idx)), np.int32)
        spikes = 0.0
        for c in range(CALLS):
            out, st = gpu.step(batch.inputs, None, 16, batch.gain)
            outs[c] = out[idx]
            status[c] = st[idx]
            spikes += float(out.sum())
        dumps = [gpu.dump(int(i)) for i in idx]
        return outs, status, dumps, gpu.stats(), spikes
    finally:
        gpu.close()


def _compare(idx, run, want):
    outs, status, dumps = run[:3]
    for k, i in enumerate(idx):
        w_out, w_st, w_n, w_s, w_t = want[int(i)]
        assert np.array_equal(status[:, k], w_st), f"brain {i}: status differs"
        bad = np.nonzero(~np.all(outs[:, k] == w_out, axis=1))[0]
        assert bad.size == 0, f"brain {i}: motor outputs differ first at call {bad[0]}"
        gn, gs, gt = dumps[k]
        assert gt == w_t == 16 * CALLS
        badn = np.argwhere(~_nan_equivalent(gn, w_n))
        assert badn.size == 0, f"brain {i}: neuron words differ at {badn[:6].tolist()}"
        bads = np.argwhere(gs != w_s)
        assert bads.size == 0, f"brain {i}: synapse words differ at {bads[:6].tolist()}"


def _assert_same(x, y, name):
    """Bitwise equality of every field (record padding is not compared)."""
    if x.dtype.names:
        for fld in x.dtype.names:
            _assert_same(x[fld], y[fld], f"{name}.{fld}")
        return
    bx = np.ascontiguousarray(x).view(np.uint8).reshape(len(x), -1)
    by = np.ascontiguousarray(y).view(np.uint8).reshape(len(y), -1)
    bad = np.nonzero(~np.all(bx == by, axis=1))[0]
    assert bad.size == 0, f"{name} differs at {bad.size} slots (first {bad[:4].tolist()})"


class _Expected:
    """The oracle's results for a sample, computed once in the background."""

    def __init__(self, oracle):
        self.oracle, self.value = oracle, None

    def get(self):
        if self.value is None:
            self.value = self.oracle.result()
        return self.value


@pytest.fixture(scope="module")
def uneven(nsb):
    batch = nsb.workloads.batched_uneven(seed=2)
    assert (batch.brains, len(batch.neuron_rows), len(batch.synapse_rows)) == (32768, 4194304, 8388608)
    seeds = np.arange(batch.brains, dtype=np.uint32) * 17 + 20
    idx = _sample(batch)
    want = _Expected(SampledOracle(batch, idx, seeds, CALLS))
    yield batch, seeds, idx, want
    want.oracle.pool.shutdown(cancel_futures=True)


@pytest.mark.parametrize("delivery,cluster", [(False, None), (True, None), (True, "1")])
def test_full_pools_2000_ticks(nsb, uneven, monkeypatch, delivery, cluster):
    """The benchmark's batch for 2,000 ticks: serial and warp-cooperative
    delivery on the default plan, and brains above the unit size on
    thread-block clusters. Every sampled brain's outputs every call and its
    whole state at the end equal the oracle's."""
    batch, seeds, idx, want = uneven
    if cluster is not None:
        monkeypatch.setenv("NSB_CLUSTER", cluster)
    run = _gpu_run(nsb, batch, seeds, idx, delivery=delivery)
    _compare(idx, run, want.get())
    stats, spikes = run[3], run[4]
    assert stats["neurons"] == 4194304 and stats["synapses"] == 8388608
    if cluster == "1":
        assert stats["big_units"] > 0
    assert spikes > 0
    sizes = np.diff(batch.neuron_offsets)
    assert sizes[idx].max() == sizes.max()                   # the largest brains are in the sample


def test_plasticity_heavy_full_pools_2000_ticks(nsb):
    """Config 4 at full pools for 2,000 ticks with pulses inside the calls:
    sampled brains equal the oracle, and their weights have moved."""
    batch = nsb.workloads.plasticity_heavy(seed=4)
    assert (len(batch.neuron_rows), len(batch.synapse_rows)) == (4194304, 8388608)
    pulse = (batch.meta["pulse_period"], batch.meta["pulse_mod"])
    seeds = np.arange(batch.brains, dtype=np.uint32) * 13 + 5
    idx = _sample(batch, stride=128, largest=3)
    oracle = SampledOracle(batch, idx, seeds, CALLS, pulse=pulse)
    try:
        run = _gpu_run(nsb, batch, seeds, idx, pulse=pulse)
    except BaseException:
        oracle.pool.shutdown(cancel_futures=True)
        raise
    want = oracle.result()
    _compare(idx, run, want)
    moved = sum(int((want[int(i)][3][:, 0].view(np.float32) != batch.brain(int(i))[1][:, 2]).sum())
                for i in idx)
    assert moved > 0


def test_world_founders_2048_open_loop_2000_ticks(nsb):
    """Config 2's raster gate at its specified size: 2,048 founders (about
    132,000 neurons and 1.06 M synapses), 125 world steps with fresh senses
    every step. Motor counts of every animal equal the oracle's every step;
    every pool word of every animal equals it at the end."""
    W = nsb.world
    batch = nsb.workloads.world_founders(seed=2, founders=2048)
    seeds = np.arange(batch.brains, dtype=np.uint32) + 1
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds), scatter_seed=3)
    oracle = SubsetWorldOracle(pools.copy(), CALLS, senses_seed=4)
    world = W.World(pools)
    try:
        animals = pools.animals.copy()
        rng = np.random.default_rng(4)
        motors = np.zeros((CALLS,) + pools.motors.shape, np.int32)
        for step in range(1, CALLS + 1):
            world.upload("senses", rng.random(pools.senses.shape).astype(np.float32))
            world.upload("motors", np.zeros_like(pools.motors))
            world.neural_step(step)
            motors[step - 1] = world.dev["motors"].cpu().numpy().view(np.int32).reshape(pools.motors.shape)
            animals["age"][animals["alive"] == 1] += 1
            world.upload("animals", animals.copy())
            world.homeostasis()
        got = world.download()
    finally:
        world.close()
    res = oracle.result()
    covered = np.zeros(len(pools.animals), bool)
    for subset, want_motors, f in res:
        covered[subset] = True
        bad = np.nonzero(~np.all(motors[:, subset] == want_motors[:, subset], axis=(1, 2)))[0]
        assert bad.size == 0, f"motor counts differ first at step {bad[0] + 1}"
        nmask = np.isin(got.neuron_owner, subset)
        smask = np.isin(got.synapse_owner, subset)
        for name, mask in (("neuron_state", nmask), ("synapse_state", smask), ("pending_exc", nmask),
                           ("pending_inh", nmask), ("mod_event_tick", nmask)):
            _assert_same(getattr(got, name)[mask], f[name][mask], name)
        _assert_same(got.spike_history[:, nmask].T, f["spike_history"][:, nmask].T, "spike_history")
        _assert_same(got.animals[subset], f["animals"][subset], "animals")
    assert covered[pools.animals["alive"] == 1].all()
    assert motors.sum() > 0 and got.neuron_state["total"].sum() > 0
