"""Host logic of multi-GPU placement, on CPU: shard ranges, and the timing /
gather collectives run by world_size-2 gloo process groups (the NCCL path of
bench.py uses the same helpers with CUDA tensors)."""
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
