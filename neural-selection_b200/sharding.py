"""Multi-GPU placement of independent brains.

Brains never interact within a world step (no cross-brain term in the
reference's neural stage, src/main.cu:659-801), so a population shards across
GPUs with no data-path collective: each rank steps a contiguous range of
brains, balanced by neurons + synapses, on its own device. Collectives are
used only for timing (the max over ranks) and, optionally, for gathering
per-brain results to one rank.
"""
from __future__ import annotations

import numpy as np


def shard_ranges(neuron_offsets, synapse_offsets, world):
    """Contiguous brain ranges [(b0, b1), ...], one per rank, splitting the
    cumulative work N + E as evenly as whole brains allow. Every brain is in
    exactly one range; a range may be empty when there are fewer brains than
    ranks."""
    no = np.asarray(neuron_offsets, np.int64)
    so = np.asarray(synapse_offsets, np.int64)
    brains = len(no) - 1
    if world < 1:
        raise ValueError("world size must be positive")
    work = np.diff(no) + np.diff(so)
    cum = np.concatenate([[0], np.cumsum(work)])
    total = cum[-1]
    cuts = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cum, target, side="left"))
        # take the nearer of the two brain boundaries around the target
        if b > 0 and abs(cum[b - 1] - target) <= abs(cum[min(b, brains)] - target):
            b -= 1
        cuts.append(min(max(b, cuts[-1]), brains))
    cuts.append(brains)
    return [(cuts[r], cuts[r + 1]) for r in range(world)]


def max_over_ranks(value, dist=None, device=None):
    """The maximum of a per-rank float over all ranks (the timing rule for
    multi-GPU numbers). Uses the process group's backend: a CUDA tensor for
    NCCL, a CPU tensor for gloo."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value, dist=None, device=None):
    """The sum of a per-rank number over all ranks (event counts)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def gather_results(local, dist=None, device=None):
    """Concatenate per-rank 2-D result arrays (rows in rank order) on every
    rank. Rows may differ in count between ranks."""
    local = np.ascontiguousarray(local)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return local
    import torch
    world = dist.get_world_size()
    n = torch.tensor([local.shape[0]], dtype=torch.int64, device=device or "cpu")
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    counts = [int(c.item()) for c in counts]
    width = local.shape[1] if local.ndim > 1 else 1
    pad = max(counts)
    buf = np.zeros((pad, width), local.dtype)
    buf[: local.shape[0]] = local.reshape(local.shape[0], width)
    t = torch.from_numpy(buf).to(device or "cpu")
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    out = [p.cpu().numpy()[:c] for p, c in zip(parts, counts)]
    return np.concatenate(out).reshape(-1, *local.shape[1:]) if local.ndim > 1 else np.concatenate(out).ravel()
