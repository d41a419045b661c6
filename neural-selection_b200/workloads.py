"""Seeded synthetic workloads for the neural tick, drawn from Philox4x32-10.

Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
as 1, 2, 3", SC'11) is a counter-based generator: output = bijection(counter,
key). Every random field here is addressed by a counter
(brain, entity, field, 0) under key (seed, stream), so any subset of a
workload can be regenerated without generating the rest, on the host or the
device, and the stream does not depend on generation order.

Genomes use the reference's Gym ABI rows (gym_adapter/adapter.py:45-66):
  neuron  [profile, channel, active, inhibitory, modulator, C x, gL x,
           V_threshold, receptor Hz gain, receptor event nS]
  synapse [pre, post, weight nS, active, delay, branch, U, recovery ms,
           facilitation ms, plasticity profile, modulator receptor mask]
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
W0, W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32(counter, key, rounds=10):
    """Vectorised Philox4x32. counter: (..., 4) uint32, key: (2,) uint32.
    Returns (..., 4) uint32."""
    c = np.asarray(counter, dtype=np.uint32)
    c0, c1, c2, c3 = (c[..., i].astype(np.uint64) for i in range(4))
    k0 = np.uint64(np.uint32(key[0]))
    k1 = np.uint64(np.uint32(key[1]))
    for r in range(rounds):
        p0 = M0 * c0
        p1 = M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & MASK32
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0), lo1, (hi0 ^ c3 ^ k1), lo0
        if r + 1 < rounds:
            k0 = (k0 + np.uint64(W0)) & MASK32
            k1 = (k1 + np.uint64(W1)) & MASK32
    return np.stack([c0, c1, c2, c3], axis=-1).astype(np.uint32)


class Stream:
    """Philox draws addressed by (brain, entity, field)."""

    def __init__(self, seed, stream=0x6E735F62):
        self.key = (np.uint32(seed & 0xFFFFFFFF), np.uint32(stream & 0xFFFFFFFF))

    def bits(self, brain, entity, fld):
        brain, entity = np.broadcast_arrays(np.asarray(brain, np.uint32), np.asarray(entity, np.uint32))
        ctr = np.stack([brain, entity, np.full(brain.shape, fld, np.uint32),
                        np.zeros(brain.shape, np.uint32)], axis=-1)
        return philox4x32(ctr, self.key)

    def uniform(self, brain, entity, fld):
        """Uniform in [0, 1) with 24-bit resolution (exact in binary32)."""
        return (self.bits(brain, entity, fld)[..., 0] >> np.uint32(8)).astype(np.float64) / 16777216.0

    def normal(self, brain, entity, fld):
        """Standard normal by Box-Muller on two 32-bit words."""
        w = self.bits(brain, entity, fld)
        u1 = (w[..., 0].astype(np.float64) + 1.0) / 4294967296.0
        u2 = w[..., 1].astype(np.float64) / 4294967296.0
        return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * np.pi * u2)

    def integers(self, brain, entity, fld, low, high):
        """Integer in [low, high) (multiply-shift, bias < 2^-32 * span)."""
        w = self.bits(brain, entity, fld)[..., 0].astype(np.uint64)
        span = np.asarray(high, np.int64) - np.asarray(low, np.int64)
        return (np.asarray(low, np.int64) + ((w * span.astype(np.uint64)) >> np.uint64(32)).astype(np.int64))


@dataclass
class Batch:
    """A population of Gym-ABI genomes stored as concatenated rows."""
    neuron_rows: np.ndarray            # (sum N, 10) float32
    synapse_rows: np.ndarray           # (sum E, 11) float32, pre/post brain-local
    neuron_offsets: np.ndarray         # (B+1,) int64
    synapse_offsets: np.ndarray        # (B+1,) int64
    motors: np.ndarray                 # (B, outputs) int32, brain-local
    channels: int
    max_delay: int
    name: str = ""
    inputs: np.ndarray | None = None   # (B, channels) float32 encoded observation
    gain: float = 230.0
    meta: dict = field(default_factory=dict)

    @property
    def brains(self):
        return len(self.neuron_offsets) - 1

    @property
    def outputs(self):
        return self.motors.shape[1]

    def brain(self, i):
        n0, n1 = self.neuron_offsets[i], self.neuron_offsets[i + 1]
        e0, e1 = self.synapse_offsets[i], self.synapse_offsets[i + 1]
        return (self.neuron_rows[n0:n1], self.synapse_rows[e0:e1], self.motors[i])

    def subset(self, index):
        index = list(index)
        nr, sr, no, so = [], [], [0], [0]
        for i in index:
            a, b_, _ = self.brain(i)
            nr.append(a); sr.append(b_)
            no.append(no[-1] + len(a)); so.append(so[-1] + len(b_))
        return Batch(np.concatenate(nr), np.concatenate(sr) if sr else np.zeros((0, 11), np.float32),
                     np.asarray(no, np.int64), np.asarray(so, np.int64), self.motors[index].copy(),
                     self.channels, self.max_delay, self.name + "[subset]",
                     None if self.inputs is None else self.inputs[index].copy(), self.gain, dict(self.meta))


THRESHOLD = {0: -52.0, 1: -42.0, 2: -42.0, 3: -42.0, 4: -40.0, 5: -40.0, 6: -51.8}


def _assemble(name, sizes, edges, channels, max_delay, neuron_fn, synapse_fn, motors, inputs, gain, meta):
    no = np.zeros(len(sizes) + 1, np.int64); no[1:] = np.cumsum(sizes)
    so = np.zeros(len(edges) + 1, np.int64); so[1:] = np.cumsum(edges)
    nr = neuron_fn(no)
    sr = synapse_fn(no, so)
    return Batch(nr.astype(np.float32), sr.astype(np.float32), no, so, motors.astype(np.int32),
                 channels, max_delay, name, inputs.astype(np.float32), gain, meta)


def _brain_of(offsets):
    counts = np.diff(offsets)
    return np.repeat(np.arange(len(counts), dtype=np.int64), counts), \
        np.arange(offsets[-1], dtype=np.int64) - np.repeat(offsets[:-1], counts)


def plain_small(seed=2, brains=64, neurons=48, synapses=600, sensory=12, outputs=5):
    """Plain method, small: 64 brains x 48 AdEx neurons, 600 synapses each,
    no self-loops, delays 1-8 ms, weights lognormal(-1, 0.5) nS, STP split
    50/50 facilitating (U .1, tau_rec 30, tau_fac 1700; src/main.cu:512-517) /
    depressing (U .55, tau_rec 450; src/main.cu:498-500), pair STDP (profile
    1) on excitatory->excitatory synapses, 12 sensory receptor neurons per
    brain driven at 20 Hz Poisson (type 5, receptor gain 20 Hz at input 1),
    5 motor neurons read out. 80% of non-sensory neurons excitatory (type 0),
    20% inhibitory (type 1 with inhibitory transmitter)."""
    st = Stream(seed)
    sizes = np.full(brains, neurons, np.int64)
    edges = np.full(brains, synapses, np.int64)

    def nfn(no):
        b, i = _brain_of(no)
        rows = np.zeros((len(b), 10))
        inhib = (st.uniform(b, i, 1) < 0.2) & (i >= sensory)
        prof = np.where(i < sensory, 5, np.where(inhib, 1, 0))
        rows[:, 0] = prof
        rows[:, 1] = np.where(i < sensory, i, -1)
        rows[:, 2] = 1
        rows[:, 3] = inhib
        rows[:, 5] = 1.0
        rows[:, 6] = 1.0
        rows[:, 7] = [THRESHOLD[int(p)] for p in prof]
        rows[:, 8] = np.where(i < sensory, 20.0, 0.0)
        rows[:, 9] = np.where(i < sensory, 2.0, 0.0)
        return rows

    def sfn(no, so):
        b, e = _brain_of(so)
        n = (no[b + 1] - no[b])
        pre = st.integers(b, e, 10, 0, n)
        post = st.integers(b, e, 11, 0, n - 1)
        post = np.where(post >= pre, post + 1, post)
        rows = np.zeros((len(b), 11))
        rows[:, 0] = pre
        rows[:, 1] = post
        rows[:, 2] = np.exp(-1.0 + 0.5 * st.normal(b, e, 12))
        rows[:, 3] = 1
        rows[:, 4] = st.integers(b, e, 13, 1, 9)
        rows[:, 5] = st.integers(b, e, 14, 0, 4)
        fac = st.uniform(b, e, 15) < 0.5
        rows[:, 6] = np.where(fac, 0.1, 0.55)
        rows[:, 7] = np.where(fac, 30.0, 450.0)
        rows[:, 8] = np.where(fac, 1700.0, 0.0)
        # excitatory -> excitatory pairs are plastic (pair STDP)
        nb = no[b]
        inhib = (st.uniform(b, pre, 1) < 0.2) & (pre >= sensory)
        inhib_post = (st.uniform(b, post, 1) < 0.2) & (post >= sensory)
        rows[:, 9] = np.where(~inhib & ~inhib_post, 1, 0)
        rows[:, 10] = 0
        return rows

    motors = np.tile(np.arange(sensory, sensory + outputs), (brains, 1))
    inputs = np.ones((brains, sensory), np.float32)
    return _assemble("plain_small", sizes, edges, sensory, 8, nfn, sfn, motors, inputs, 230.0,
                     {"ticks_per_step": 16, "steps": 200})


def uneven_sizes(seed, brains, total, median, sigma, lo, hi):
    """Lognormal(median, sigma) brain sizes clipped to [lo, hi] and rescaled so
    they sum exactly to `total` (largest-remainder rounding)."""
    st = Stream(seed, 0x73697a65)
    raw = np.clip(median * np.exp(sigma * st.normal(np.arange(brains), 0, 0)), lo, hi)
    for _ in range(50):
        scaled = np.clip(raw * (total / raw.sum()), lo, hi)
        if abs(scaled.sum() - total) < 0.5:
            break
        raw = scaled
    base = np.floor(scaled).astype(np.int64)
    short = int(total - base.sum())
    order = np.argsort(-(scaled - base), kind="stable")
    room = base < hi
    k = 0
    for j in order:
        if k >= short:
            break
        if room[j]:
            base[j] += 1
            k += 1
    assert base.sum() == total and base.min() >= lo and base.max() <= hi
    return base


def batched_uneven(seed=2, brains=32768, total_neurons=4194304, total_synapses=8388608,
                   sensory=8, outputs=5, max_delay=16, plastic_all=False, median=96.0, sigma=1.0, lo=16, hi=4096):
    """Batched uneven brains at full pools: sizes lognormal(median 96,
    sigma 1) clipped to [16, 4096] and rescaled to fill 4,194,304 neuron slots;
    8,388,608 synapses in proportion to size (2 per neuron); delays 1-16 ms;
    8 sensory receptor neurons per brain at a Poisson rate uniform in 10-40 Hz;
    5 motor neurons. Hidden neurons: 80% excitatory type 0, 20% inhibitory
    type 1. Synapse phenotypes follow the reference world's founders
    (src/main.cu:462-528): weight 0.5 + 3.5 U nS, 14 sites, depressing
    (U .55, tau_rec 450) except facilitating onto inhibitory targets (U .1,
    tau_rec 30, tau_fac 1700); pair STDP (profile 1) on excitatory pairs."""
    st = Stream(seed)
    sizes = uneven_sizes(seed, brains, total_neurons, median, sigma, lo, hi)
    per = total_synapses // total_neurons
    edges = sizes * per
    rem = total_synapses - edges.sum()
    edges[:rem] += 1

    def kinds(b, i):
        inhib = (st.uniform(b, i, 1) < 0.2) & (i >= sensory)
        return inhib

    def nfn(no):
        b, i = _brain_of(no)
        rows = np.zeros((len(b), 10))
        inhib = kinds(b, i)
        prof = np.where(i < sensory, 5, np.where(inhib, 1, 0))
        rows[:, 0] = prof
        rows[:, 1] = np.where(i < sensory, i, -1)
        rows[:, 2] = 1
        rows[:, 3] = inhib
        rows[:, 5] = 1.0
        rows[:, 6] = 1.0
        rows[:, 7] = np.where(prof == 5, -40.0, np.where(prof == 1, -42.0, -52.0))
        rows[:, 8] = np.where(i < sensory, 10.0 + 30.0 * st.uniform(b, i, 2), 0.0)
        rows[:, 9] = np.where(i < sensory, 2.0, 0.0)
        return rows

    def sfn(no, so):
        b, e = _brain_of(so)
        n = no[b + 1] - no[b]
        pre = st.integers(b, e, 10, 0, n)
        post = st.integers(b, e, 11, 0, n - 1)
        post = np.where(post >= pre, post + 1, post)
        rows = np.zeros((len(b), 11))
        rows[:, 0] = pre
        rows[:, 1] = post
        rows[:, 2] = 0.5 + 3.5 * st.uniform(b, e, 12)
        rows[:, 3] = 1
        rows[:, 4] = st.integers(b, e, 13, 1, max_delay + 1)
        rows[:, 5] = st.integers(b, e, 14, 0, 4)
        inh_pre = kinds(b, pre)
        inh_post = kinds(b, post)
        fac = inh_post & ~inh_pre
        rows[:, 6] = np.where(fac, 0.1, 0.55)
        rows[:, 7] = np.where(fac, 30.0, 450.0)
        rows[:, 8] = np.where(fac, 1700.0, 0.0)
        rows[:, 9] = np.where(plastic_all | (~inh_pre & ~inh_post), 1, 0)
        return rows

    motors = np.tile(np.arange(sensory, sensory + outputs), (brains, 1))
    inputs = np.ones((brains, sensory), np.float32)
    return _assemble("batched_uneven", sizes, edges, sensory, max_delay, nfn, sfn, motors, inputs, 230.0,
                     {"ticks_per_step": 16, "steps": 500})


def plasticity_heavy(seed=4, brains=32768, total_neurons=4194304, total_synapses=8388608, sensory=8, outputs=5,
                     max_delay=16, burst_frac=0.3, burst_level=0.65, median=96.0, sigma=1.0, lo=16, hi=4096):
    """Plasticity-heavy full pools: the batched-uneven population with every
    synapse on profile 6 (triplet STDP into a dopamine eligibility trace,
    tau 200 ms) and a dopamine receptor, 30% of the hidden neurons driven
    tonically to about 60 Hz (type 0 on an extra input channel at level 0.65,
    i.e. 150 pA at the default gain of 230), and a global dopamine pulse every
    50 ms (meta pulse_period / pulse_mod, applied with set_modulation)."""
    base = batched_uneven(seed=seed, brains=brains, total_neurons=total_neurons, total_synapses=total_synapses,
                          sensory=sensory, outputs=outputs, max_delay=max_delay, median=median, sigma=sigma, lo=lo,
                          hi=hi)
    st = Stream(seed, 0x62757273)
    nr = base.neuron_rows.copy()
    b, i = _brain_of(base.neuron_offsets)
    hidden = i >= sensory + outputs
    burst = hidden & (st.uniform(b, i, 20) < burst_frac)
    nr[burst, 0] = 0                       # excitatory AdEx with afterdepolarisation
    nr[burst, 1] = sensory                 # the drive channel
    nr[burst, 3] = 0
    nr[burst, 7] = -52.0
    sr = base.synapse_rows.copy()
    sr[:, 9] = 6                           # triplet STDP + dopamine eligibility on every synapse
    sr[:, 10] = 4                          # dopamine receptor
    inputs = np.concatenate([np.ones((base.brains, sensory), np.float32),
                             np.full((base.brains, 1), burst_level, np.float32)], axis=1)
    return Batch(nr, sr, base.neuron_offsets, base.synapse_offsets, base.motors, sensory + 1, max_delay,
                 "plasticity_heavy", inputs, 230.0, {"ticks_per_step": 16, "steps": 1000, "pulse_period": 50,
                                                     "pulse_mod": 4, "burst_fraction": burst_frac})


def parity_mix(seed=7, brains=24, min_n=8, max_n=160, fanin=8, channels=6, outputs=4, max_delay=8,
               heavy_types=True):
    """Parity workload: every neuron profile (0-6, LP and Prinz cells
    included when heavy_types), inhibitory and all three modulator kinds, every
    plasticity profile 0-5 and receptor mask 0-7, inactive neurons and
    synapses, recurrent and parallel edges, tonic sensory current and receptor
    drive, strong weights so neurons fire."""
    st = Stream(seed, 0x70617269)
    sizes = st.integers(np.arange(brains), 0, 0, min_n, max_n + 1)
    sizes = np.maximum(sizes, outputs + 1)
    edges = sizes * fanin

    def nfn(no):
        b, i = _brain_of(no)
        u = st.uniform(b, i, 1)
        choices = np.array([0, 0, 0, 1, 1, 4, 5, 6, 2, 3] if heavy_types else [0, 0, 0, 1, 1, 4, 5])
        prof = choices[(u * len(choices)).astype(int)]
        rows = np.zeros((len(b), 10))
        rows[:, 0] = prof
        has_ch = st.uniform(b, i, 2) < 0.35
        rows[:, 1] = np.where(has_ch, st.integers(b, i, 3, 0, channels), -1)
        rows[:, 2] = (st.uniform(b, i, 4) > 0.07).astype(float)
        rows[:, 3] = ((prof == 1) | (st.uniform(b, i, 5) < 0.1)).astype(float)
        mod_draw = st.uniform(b, i, 6)
        rows[:, 4] = np.where(mod_draw < 0.04, 1, np.where(mod_draw < 0.08, 2, np.where(mod_draw < 0.12, 3, 0)))
        rows[:, 5] = 0.6 + 0.8 * st.uniform(b, i, 7)
        rows[:, 6] = 0.6 + 0.8 * st.uniform(b, i, 8)
        rows[:, 7] = np.array([THRESHOLD[int(p)] for p in prof]) + 4.0 * (st.uniform(b, i, 9) - 0.5)
        rows[:, 8] = np.where(prof == 5, 5.0 + 60.0 * st.uniform(b, i, 10), 43.0)
        rows[:, 9] = np.where(st.uniform(b, i, 11) < 0.05, 0.0, 2.0)
        return rows

    def sfn(no, so):
        b, e = _brain_of(so)
        n = no[b + 1] - no[b]
        rows = np.zeros((len(b), 11))
        rows[:, 0] = st.integers(b, e, 20, 0, n)
        rows[:, 1] = st.integers(b, e, 21, 0, n)
        rows[:, 2] = 1.0 + 17.0 * st.uniform(b, e, 22)
        rows[:, 3] = (st.uniform(b, e, 23) > 0.06).astype(float)
        rows[:, 4] = st.integers(b, e, 24, 1, max_delay + 1)
        rows[:, 5] = st.integers(b, e, 25, 0, 4)
        rows[:, 6] = 0.05 + 0.95 * st.uniform(b, e, 26)
        rows[:, 7] = 10.0 + 500.0 * st.uniform(b, e, 27)
        rows[:, 8] = np.where(st.uniform(b, e, 28) < 0.5, 0.0, 50.0 + 1500.0 * st.uniform(b, e, 29))
        rows[:, 9] = st.integers(b, e, 30, 0, 6)
        rows[:, 10] = st.integers(b, e, 31, 0, 8)
        return rows

    bi = np.arange(brains)
    motors = np.stack([st.integers(bi, 1000 + k, 40, 0, sizes) for k in range(outputs)], axis=1)
    inputs = st.uniform(np.repeat(bi, channels), np.tile(np.arange(channels), brains), 50).reshape(brains, channels)
    return _assemble("parity_mix", sizes, edges, channels, max_delay, nfn, sfn, motors, inputs, 230.0, {})


def serving_library(seed=5, genomes=512, lo=32, hi=4096, per_neuron=8, channels=8, outputs=2, max_delay=8):
    """Genomes of the serving workload (config 5): N log-uniform in [lo, hi],
    per_neuron*N synapses. Ports follow the reference's random_genome
    (gym_adapter/adapter.py:74-88): `channels` sensory neurons (profile 4,
    channel i), `outputs` motor neurons (profile 4), hidden neurons of profile
    0, 1 or 4 with 20% inhibitory transmitter; synapses as its synapse()
    (weight U(1, 18) nS, branch 0-3, U .8, recovery 60 ms, facilitation 50 ms,
    no plasticity) with pre uniform over all neurons, post uniform over
    non-sensory neurons and delays 1-max_delay ms. Returns a Batch (inputs
    zero: the server encodes observations itself)."""
    st = Stream(seed, 0x73657276)
    u = st.uniform(np.arange(genomes), 0, 0)
    sizes = np.floor(np.exp(np.log(lo) + u * (np.log(hi + 1) - np.log(lo)))).astype(np.int64)
    sizes = np.clip(sizes, max(lo, channels + outputs), hi)
    edges = sizes * per_neuron

    def nfn(no):
        b, i = _brain_of(no)
        rows = np.zeros((len(b), 10))
        hidden = i >= channels + outputs
        prof = np.where(hidden, np.array([0, 1, 4])[st.integers(b, i, 1, 0, 3)], 4)
        inhib = hidden & (st.uniform(b, i, 2) < 0.2)
        rows[:, 0] = prof
        rows[:, 1] = np.where(i < channels, i, -1)
        rows[:, 2] = 1
        rows[:, 3] = inhib
        rows[:, 5] = 1.0
        rows[:, 6] = 1.0
        rows[:, 7] = [THRESHOLD[int(p)] for p in prof]
        rows[:, 8] = 43.0
        rows[:, 9] = 2.0
        return rows

    def sfn(no, so):
        b, e = _brain_of(so)
        n = no[b + 1] - no[b]
        rows = np.zeros((len(b), 11))
        rows[:, 0] = st.integers(b, e, 10, 0, n)
        rows[:, 1] = st.integers(b, e, 11, channels, n)
        rows[:, 2] = 1.0 + 17.0 * st.uniform(b, e, 12)
        rows[:, 3] = 1
        rows[:, 4] = st.integers(b, e, 13, 1, max_delay + 1)
        rows[:, 5] = st.integers(b, e, 14, 0, 4)
        rows[:, 6] = 0.8
        rows[:, 7] = 60.0
        rows[:, 8] = 50.0
        return rows

    motors = np.tile(np.arange(channels, channels + outputs), (genomes, 1))
    inputs = np.zeros((genomes, channels), np.float32)
    return _assemble("serving_library", sizes, edges, channels, max_delay, nfn, sfn, motors, inputs, 230.0,
                     {"per_neuron": per_neuron})


def serving_schedule(seed, rate, seconds, genomes, lo_steps=200, hi_steps=2000, start=0.0):
    """Poisson arrivals at `rate` per second over [start, start + seconds):
    returns dict of arrays arrival (s), genome (uniform over the library), seed,
    steps (uniform integer in [lo_steps, hi_steps]) and tag (request index)."""
    st = Stream(seed, 0x61727276)
    n_max = int(rate * seconds + 10 * np.sqrt(rate * seconds + 1) + 16)
    idx = np.arange(n_max)
    gaps = -np.log(1.0 - st.uniform(idx, 0, 0)) / rate
    arrival = start + np.cumsum(gaps)
    keep = arrival < start + seconds
    idx = idx[keep]
    return {"arrival": arrival[keep], "genome": st.integers(idx, 0, 1, 0, genomes).astype(np.int32),
            "seed": st.bits(idx, 0, 2)[:, 0].astype(np.uint32),
            "steps": st.integers(idx, 0, 3, lo_steps, hi_steps + 1).astype(np.int32),
            "tag": idx.astype(np.uint64)}


def world_founders(seed=2, founders=2048, lo=32, hi=96, epn_lo=4, epn_hi=12, heavy_types=False):
    """Founder brains of the world workload (config 2): `founders` animals of
    N ~ U{lo..hi} neurons and N x U{epn_lo..epn_hi} synapses. Ports follow the
    world simulator's layout (src/main.cu:36-42, 544-591): neurons 0-18 are
    sensory on world channels 0-18 (type 5 receptor cells on the chemical
    channels 0-5, type 4 relays on 6-18), neurons 19-23 the five motor
    neurons (type 0), the rest hidden: type 0, 20% type 1 inhibitory, 5%
    modulatory (NE / 5-HT / DA), and with heavy_types some LP, Prinz and LFS
    cells. Synapses: pre uniform over all neurons, post uniform over
    non-sensory neurons, weight U(1, 18) nS, delay 1-8 ms, branch 0-3,
    facilitating or depressing release (src/main.cu:498-517), plasticity
    profile 0-5 and modulator receptor mask 0-7 uniform. inputs: the world
    senses, U(0, 1) per animal and channel."""
    st = Stream(seed, 0x776f726c)
    fi = np.arange(founders)
    sizes = st.integers(fi, 0, 0, lo, hi + 1)
    sizes = np.maximum(sizes, 25)
    edges = sizes * st.integers(fi, 0, 1, epn_lo, epn_hi + 1)
    channels, outputs = 19, 5

    def nfn(no):
        b, i = _brain_of(no)
        rows = np.zeros((len(b), 10))
        u = st.uniform(b, i, 1)
        hidden = i >= channels + outputs
        prof = np.where(i < 6, 5, np.where(i < channels, 4, 0))
        inhib = hidden & (u < 0.2)
        prof = np.where(inhib, 1, prof)
        if heavy_types:
            h = st.uniform(b, i, 2)
            prof = np.where(hidden & ~inhib & (h < 0.03), 2, prof)
            prof = np.where(hidden & ~inhib & (h >= 0.03) & (h < 0.06), 3, prof)
            prof = np.where(hidden & ~inhib & (h >= 0.06) & (h < 0.09), 6, prof)
        mod = np.where(hidden & ~inhib & (u >= 0.2) & (u < 0.25), st.integers(b, i, 3, 1, 4), 0)
        rows[:, 0] = prof
        rows[:, 1] = np.where(i < channels, i, -1)
        rows[:, 2] = 1
        rows[:, 3] = inhib
        rows[:, 4] = mod
        rows[:, 5] = 0.8 + 0.4 * st.uniform(b, i, 4)
        rows[:, 6] = 0.8 + 0.4 * st.uniform(b, i, 5)
        rows[:, 7] = [THRESHOLD[int(p)] for p in prof]
        rows[:, 8] = np.where(prof == 5, 40.0 + 40.0 * st.uniform(b, i, 6), 0.0)
        rows[:, 9] = np.where(prof == 5, 2.0, 0.0)
        return rows

    def sfn(no, so):
        b, e = _brain_of(so)
        n = no[b + 1] - no[b]
        rows = np.zeros((len(b), 11))
        rows[:, 0] = st.integers(b, e, 10, 0, n)
        rows[:, 1] = st.integers(b, e, 11, channels, n)
        rows[:, 2] = 1.0 + 17.0 * st.uniform(b, e, 12)
        rows[:, 3] = 1
        rows[:, 4] = st.integers(b, e, 13, 1, 9)
        rows[:, 5] = st.integers(b, e, 14, 0, 4)
        fac = st.uniform(b, e, 15) < 0.5
        rows[:, 6] = np.where(fac, 0.1, 0.55)
        rows[:, 7] = np.where(fac, 30.0, 450.0)
        rows[:, 8] = np.where(fac, 1700.0, 0.0)
        rows[:, 9] = st.integers(b, e, 16, 0, 6)
        rows[:, 10] = st.integers(b, e, 17, 0, 8)
        return rows

    motors = np.tile(np.arange(channels, channels + outputs), (founders, 1))
    inputs = st.uniform(np.repeat(fi, channels), np.tile(np.arange(channels), founders), 50).reshape(founders,
                                                                                                      channels)
    return _assemble("world_founders", sizes, edges, channels, 8, nfn, sfn, motors, inputs, 230.0,
                     {"ticks_per_step": 16})


def concat(batches, name="concat"):
    """One Batch holding every brain of `batches`, in order (same channels,
    outputs and delay ring)."""
    no, so = [0], [0]
    for b in batches:
        no.extend((no[-1] + np.asarray(b.neuron_offsets[1:]) - b.neuron_offsets[0]).tolist())
        so.extend((so[-1] + np.asarray(b.synapse_offsets[1:]) - b.synapse_offsets[0]).tolist())
    b0 = batches[0]
    inputs = None if b0.inputs is None else np.concatenate([b.inputs for b in batches]).astype(np.float32)
    return Batch(np.concatenate([b.neuron_rows for b in batches]), np.concatenate([b.synapse_rows for b in batches]),
                 np.asarray(no, np.int64), np.asarray(so, np.int64),
                 np.concatenate([b.motors for b in batches]).astype(np.int32), b0.channels, b0.max_delay, name, inputs,
                 b0.gain, {})
