"""Host logic of multi-GPU placement, on CPU: shard ranges, the timing /
gather collectives run by world_size-2 gloo process groups (the NCCL path of
bench.py uses the same helpers with CUDA tensors), and sharded stepping: two
ranks each stepping their own brain range give the same motor outputs and
states as one process stepping every brain."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def test_shard_ranges_cover_and_balance(nsb):
    b = nsb.workloads.batched_uneven(brains=512, total_neurons=512 * 128, total_synapses=512 * 256)
    for world in (1, 2, 3, 4, 8):
        r = nsb.sharding.shard_ranges(b.neuron_offsets, b.synapse_offsets, world)
        assert r[0][0] == 0 and r[-1][1] == b.brains
        assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
        work = np.diff(b.neuron_offsets) + np.diff(b.synapse_offsets)
        per = np.array([work[x:y].sum() for x, y in r])
        assert per.max() - per.min() <= 2 * work.max()
    # fewer brains than ranks: empty ranges, still a partition
    r = nsb.sharding.shard_ranges([0, 5, 9], [0, 3, 4], 4)
    assert r[0][0] == 0 and r[-1][1] == 2 and sum(y - x for x, y in r) == 2


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, q):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from conftest import load_package
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    nsb = load_package()
    b = nsb.workloads.batched_uneven(brains=64, total_neurons=64 * 64, total_synapses=64 * 128)
    ranges = nsb.sharding.shard_ranges(b.neuron_offsets, b.synapse_offsets, world)
    lo, hi = ranges[rank]
    # per-rank "timing" and per-brain results (brain index, neurons)
    t = nsb.sharding.max_over_ranks(1.5 + rank, dist)
    local = np.stack([np.arange(lo, hi), np.diff(b.neuron_offsets)[lo:hi]], axis=1).astype(np.int64)
    allres = nsb.sharding.gather_results(local, dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, t, allres.tolist(), ranges))


@pytest.mark.timeout(120)
def test_gloo_world_size_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=90) for _ in procs]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    out.sort()
    assert out[0][1] == out[1][1] == 2.5            # max over ranks
    assert out[0][2] == out[1][2]                   # same gathered results on both ranks
    rows = np.array(out[0][2])
    assert rows[:, 0].tolist() == list(range(64))   # every brain exactly once, in order
    assert out[0][3] == out[1][3]


def _digest(nw, sw):
    import hashlib
    h = hashlib.blake2b(np.ascontiguousarray(nw).tobytes() + np.ascontiguousarray(sw).tobytes(), digest_size=8)
    return int(np.frombuffer(h.digest(), np.int64)[0])


def _step_range(nsb, batch, lo, hi, calls):
    """Rows (brain, outputs of every call, state digest) of brains [lo, hi)
    stepped by the oracle (the stand-in for a rank's device)."""
    from oracle.pyoracle import OracleBrain
    rows = []
    for b in range(lo, hi):
        o = OracleBrain(*batch.brain(b), batch.channels, batch.max_delay)
        o.reset(b * 13 + 1)
        outs = []
        for _ in range(calls):
            rc, out, _ = o.step(batch.inputs[b], 16, batch.gain, stop_on_nonfinite=False)
            outs.extend(out.astype(np.int64).tolist() + [rc])
        nw, sw, t = o.dump()
        rows.append([b, *outs, t, _digest(nw, sw)])
        o.close()
    return np.array(rows, np.int64).reshape(-1, 3 + calls * (batch.outputs + 1))


def _shard_main(rank, world, port, q):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root.parent))
    from conftest import load_package
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    nsb = load_package()
    b = nsb.workloads.parity_mix(seed=5, brains=24)
    lo, hi = nsb.sharding.shard_ranges(b.neuron_offsets, b.synapse_offsets, world)[rank]
    rows = _step_range(nsb, b, lo, hi, 2)
    allrows = nsb.sharding.gather_results(rows, dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, allrows.tolist(), (lo, hi)))


@pytest.mark.timeout(180)
def test_sharded_stepping_equals_one_process(nsb):
    """A population of 24 brains of every cell type and plasticity profile
    stepped 32 ticks as two gloo ranks, each on its shard_ranges slice, then
    gathered: every brain's motor outputs per call, status, tick and state
    digest equal those of one process stepping all 24 brains. Brains have no cross-brain term in the neural stage, so a
    sharded run needs no data-path collective."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=150) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert out[0][1] == out[1][1]
    assert out[0][2][1] == out[1][2][0] and out[0][2][1] > 0       # two non-empty contiguous shards
    b = nsb.workloads.parity_mix(seed=5, brains=24)
    whole = _step_range(nsb, b, 0, b.brains, 2)
    sharded = np.array(out[0][1], np.int64)
    assert sharded.shape == whole.shape
    np.testing.assert_array_equal(sharded, whole)
    assert whole[:, 1:-2].sum() > 0                                  # some motor spikes
