"""World neural stage (nsb_world_* in libns_b200.so) and world pools.

The reference world simulator keeps its population in device pools
(struct Device, mixic/neural-selection src/main.cu:105-140): Animal records,
NeuronGene / NeuronState / SynapseGene / SynapseState records indexed by pool
slot, per-slot owner / next / port arrays, the 9-tick spike history, the
per-animal senses and motor counts. `WorldPools` holds such pools on the host
in exactly those layouts; `World` uploads them and runs the library's world
stage on them in place (the replacement for src/main.cu:2634-2728 and its
homeostasis launches 2751-2758).

    pools = world.pools_from_batch(batch, records)        # or build by hand
    w = world.World(pools)
    for step in range(1, n + 1):
        w.neural_step(step); w.homeostasis()
    out = w.download()
"""
from __future__ import annotations

import ctypes as ct
from dataclasses import dataclass, field, fields

import numpy as np

from . import native

S, M, HIST, CONTACT = 19, 5, 9, 16

NEURON_GENE = np.dtype({"names": ["cap", "gl", "el", "vt", "slope", "a", "tau_w", "b", "vr", "adp_b", "adp_tau",
                                  "type", "active", "modulator", "inh_tx", "lp", "prinz_g", "prinz_leak",
                                  "sensory_channel", "rec_base", "rec_gain", "rec_event", "rec_decay", "affinity"],
                        "formats": ["<f4"] * 11 + ["u1"] * 4 + [("<f4", 4), ("<f4", 8), "<f4", "i1"] + ["<f4"] * 5,
                        "offsets": [0, 4, 8, 12, 16, 20, 24, 28, 32, 36, 40, 44, 45, 46, 47, 48, 64, 96, 100, 104,
                                    108, 112, 116, 120],
                        "itemsize": 124})
NEURON_STATE = np.dtype({"names": ["v", "w", "adp", "inh", "depol", "log_ampa", "dend", "cell", "total", "spike",
                                   "rec_ns", "rec_rng"],
                         "formats": ["<f4"] * 6 + [("<f4", 4), ("<f4", 16), "<i4", "u1", "<f4", "<u4"],
                         "offsets": [0, 4, 8, 12, 16, 20, 24, 40, 104, 108, 112, 116], "itemsize": 120})
SYNAPSE_GENE = np.dtype({"names": ["w0", "U", "trec", "tfac", "pre", "post", "delay", "active", "plasticity",
                                   "branch", "sites", "receptors", "slow_rec", "slow_depl"],
                         "formats": ["<f4"] * 4 + ["<i4"] * 2 + ["u1"] * 6 + ["<f4"] * 2,
                         "offsets": [0, 4, 8, 12, 16, 20, 24, 25, 26, 27, 28, 29, 32, 36], "itemsize": 40})
SYNAPSE_STATE = np.dtype({"names": ["w", "ru", "pre_tr", "post_tr", "eltp", "eltd", "da_age", "spine", "st_age",
                                    "pre_age", "post_age", "last", "ready", "rng", "arrived", "slow"],
                          "formats": ["<f4"] * 11 + ["<i8", "<u8", "<u4", "u1", "<f4"],
                          "offsets": [0, 4, 8, 12, 16, 20, 24, 28, 32, 36, 40, 48, 56, 64, 68, 72], "itemsize": 80})
ANIMAL = np.dtype({"names": ["x", "y", "heading", "energy", "health", "fullness", "pain", "taste", "muscle", "rng",
                             "id", "parent_id", "generation", "age", "alive", "neuron_head", "synapse_head",
                             "neuron_count", "synapse_count", "ports", "behavior"],
                   "formats": ["<f4"] * 7 + [("<f4", 4), ("<f4", 3), "<u8"] + ["<i4"] * 9 + [("<i4", 24),
                                                                                          ("<i4", 69)],
                   "offsets": [0, 4, 8, 12, 16, 20, 24, 28, 44, 56, 64, 68, 72, 76, 80, 84, 88, 92, 96, 100, 196],
                   "itemsize": 472})
COHORT = np.dtype({"names": ["id", "assigned", "frozen", "initial_age", "initial_offspring", "final_age",
                             "final_offspring", "alive", "death_cause", "neurons", "synapses", "generation",
                             "initial_energy", "initial_health", "start_step", "observed_step", "death_step"],
                   "formats": ["<i4"] * 12 + ["<f4"] * 2 + ["<i8"] * 3,
                   "offsets": [0, 4, 8, 12, 16, 20, 24, 28, 32, 36, 40, 44, 48, 52, 56, 64, 72], "itemsize": 80})


BEHAVIOR = np.dtype({"names": ["opportunities", "accepted", "empty_steps", "empty_eat", "approach_progress",
                               "approach_travel", "first_b_age", "offspring", "death_cause"],
                     "formats": [("<i4", (3, 2, 3)), ("<i4", (3, 2, 3)), ("<i4", (3, 2)), ("<i4", (3, 2)),
                                 ("<f4", (3, 3)), ("<f4", (3, 3)), "<i4", "<i4", "<i4"],
                     "offsets": [0, 72, 144, 168, 192, 228, 264, 268, 272], "itemsize": 276})
LIFE_RECORD = np.dtype({"names": ["body", "death_step", "active_neurons", "active_synapses", "modulatory_neurons",
                                  "plastic_synapses", "mean_abs_weight_change"],
                        "formats": [ANIMAL, "<i8", "<i4", "<i4", "<i4", "<i4", "<f4"],
                        "offsets": [0, 472, 480, 484, 488, 492, 496], "itemsize": 504})
BITE_EVENT = np.dtype({"names": ["step", "attacker_id", "prey_id", "x", "y"],
                       "formats": ["<i8", "<i4", "<i4", "<f4", "<f4"], "offsets": [0, 8, 12, 16, 20],
                       "itemsize": 24})
GRID = 128
CELLS = GRID * GRID


def behavior(animals):
    """The Behavior counters of Animal records, as a structured view."""
    return animals["behavior"].view(np.uint8).reshape(len(animals), -1).view(BEHAVIOR).reshape(-1)


class NsbWorldPools(ct.Structure):
    """include/ns_b200.h NsbWorldPools (pointers: device for the library,
    host for the oracle's or_world_pools, which has the same layout)."""
    _fields_ = [(n, ct.c_void_p) for n in (
        "animals", "plasticity_cohort", "neurons", "synapses", "neuron_state", "synapse_state", "pending_exc",
        "pending_inh", "senses", "mod_event_tick", "spike_history", "neuron_owner", "synapse_owner", "neuron_next",
        "synapse_next", "neuron_port", "motors", "trace_exc_arrivals", "trace_exc_releases", "trace_inh_arrivals",
        "trace_exc_ns", "trace_inh_ns", "trace_peak_mv")] + [(n, ct.c_int) for n in (
        "trace_animal", "silence_senses", "silence_contact", "animal_capacity", "neuron_capacity",
        "synapse_capacity")]


ARRAYS = ("animals", "plasticity_cohort", "neurons", "synapses", "neuron_state", "synapse_state", "pending_exc",
          "pending_inh", "senses", "mod_event_tick", "spike_history", "neuron_owner", "synapse_owner", "neuron_next",
          "synapse_next", "neuron_port", "motors", "trace_exc_arrivals", "trace_exc_releases", "trace_inh_arrivals",
          "trace_exc_ns", "trace_inh_ns", "trace_peak_mv")


@dataclass
class WorldPools:
    """Host copy of the world's neural pools in the reference layouts."""
    animals: np.ndarray
    plasticity_cohort: np.ndarray | None
    neurons: np.ndarray
    synapses: np.ndarray
    neuron_state: np.ndarray
    synapse_state: np.ndarray
    pending_exc: np.ndarray          # (neuron_capacity, 4) f32
    pending_inh: np.ndarray          # (neuron_capacity,) f32
    senses: np.ndarray               # (animal_capacity, 19) f32
    mod_event_tick: np.ndarray       # (neuron_capacity, 6) u64
    spike_history: np.ndarray        # (9, neuron_capacity) u8
    neuron_owner: np.ndarray
    synapse_owner: np.ndarray
    neuron_next: np.ndarray
    synapse_next: np.ndarray
    neuron_port: np.ndarray
    motors: np.ndarray               # (animal_capacity, 5) i32
    trace_exc_arrivals: np.ndarray = field(default_factory=lambda: np.zeros(M, np.int32))
    trace_exc_releases: np.ndarray = field(default_factory=lambda: np.zeros(M, np.int32))
    trace_inh_arrivals: np.ndarray = field(default_factory=lambda: np.zeros(M, np.int32))
    trace_exc_ns: np.ndarray = field(default_factory=lambda: np.zeros(M, np.float32))
    trace_inh_ns: np.ndarray = field(default_factory=lambda: np.zeros(M, np.float32))
    trace_peak_mv: np.ndarray = field(default_factory=lambda: np.full(M, -1000.0, np.float32))
    trace_animal: int = -1
    silence_senses: int = 0
    silence_contact: int = 0

    @property
    def capacities(self):
        return len(self.animals), len(self.neurons), len(self.synapses)

    def copy(self):
        kw = {}
        for f in fields(self):
            v = getattr(self, f.name)
            kw[f.name] = v.copy() if isinstance(v, np.ndarray) else v
        return WorldPools(**kw)

    def struct(self):
        """NsbWorldPools over these host arrays (for the oracle)."""
        s = NsbWorldPools()
        for n in ARRAYS:
            a = getattr(self, n)
            setattr(s, n, None if a is None else a.ctypes.data)
        s.trace_animal, s.silence_senses, s.silence_contact = self.trace_animal, self.silence_senses, \
            self.silence_contact
        s.animal_capacity, s.neuron_capacity, s.synapse_capacity = self.capacities
        return s


class NsbWorldEcology(ct.Structure):
    """include/ns_b200.h NsbWorldEcology (device pointers for the library,
    host pointers for the oracle's or_world_eco, which has the same layout)."""
    _fields_ = [(n, ct.c_void_p) for n in (
        "food", "kind", "cell_head", "cell_next", "bite_intent", "neuron_used", "synapse_used",
        "founder_motor_steps", "founder_observed_steps", "deaths", "predation_deaths", "bites", "life_records",
        "life_count", "bite_events", "bite_event_count")] + [(n, ct.c_int) for n in (
        "initial_count", "instant_motors", "life_capacity")] + [(n, ct.c_void_p) for n in (
        "neuron_clone", "births", "next_id")]


ECO_ARRAYS = ("food", "kind", "cell_head", "cell_next", "bite_intent", "neuron_used", "synapse_used",
              "founder_motor_steps", "founder_observed_steps", "deaths", "predation_deaths", "bites", "life_records",
              "life_count", "bite_events", "bite_event_count", "neuron_clone", "births", "next_id")


@dataclass
class Ecology:
    """Host copy of the world's ecology state beside the neural pools (the
    food grid, spatial index, slot bitmaps, counters and appended records of
    the simulator's struct Device, src/main.cu:105-140)."""
    food: np.ndarray                 # (128 * 128,) i32
    kind: np.ndarray                 # (128 * 128,) i32
    cell_head: np.ndarray            # (128 * 128,) i32
    cell_next: np.ndarray            # (animal_capacity,) i32
    bite_intent: np.ndarray          # (animal_capacity,) u8
    neuron_used: np.ndarray          # (ceil(neuron_capacity / 32),) u32
    synapse_used: np.ndarray
    founder_motor_steps: np.ndarray  # (5,) i32
    founder_observed_steps: np.ndarray   # (1,) i32 each
    deaths: np.ndarray
    predation_deaths: np.ndarray
    bites: np.ndarray
    life_records: np.ndarray | None  # LIFE_RECORD
    life_count: np.ndarray
    bite_events: np.ndarray | None   # BITE_EVENT, 2 * animal_capacity
    bite_event_count: np.ndarray
    neuron_clone: np.ndarray         # (neuron_capacity,) i32, reproduction scratch
    births: np.ndarray
    next_id: np.ndarray
    initial_count: int = 0
    instant_motors: int = 0

    def copy(self):
        kw = {}
        for f in fields(self):
            v = getattr(self, f.name)
            kw[f.name] = v.copy() if isinstance(v, np.ndarray) else v
        return Ecology(**kw)

    def struct(self):
        """NsbWorldEcology over these host arrays (for the oracle)."""
        s = NsbWorldEcology()
        for n in ECO_ARRAYS:
            a = getattr(self, n)
            setattr(s, n, None if a is None else a.ctypes.data)
        s.initial_count, s.instant_motors = self.initial_count, self.instant_motors
        s.life_capacity = 0 if self.life_records is None else len(self.life_records)
        return s


def _seed_for(seed, i):
    """src/main.cu:341-346 over numpy uint64 arrays."""
    with np.errstate(over="ignore"):
        x = np.uint64(seed) + np.uint64(0x9e3779b97f4a7c15) * (np.asarray(i, np.uint64) + np.uint64(1))
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xbf58476d1ce4e5b9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94d049bb133111eb)
        return (x ^ (x >> np.uint64(31))) | np.uint64(1)


def _uniform(s):
    """xorshift64* step and uniform draw (src/main.cu:331-337); returns (u, s)."""
    with np.errstate(over="ignore"):
        s = s ^ (s >> np.uint64(12))
        s = s ^ (s << np.uint64(25))
        s = s ^ (s >> np.uint64(27))
        r = s * np.uint64(2685821657736338717)
    return ((r >> np.uint64(40)).astype(np.float64) * (1.0 / 16777216.0)).astype(np.float32), s


def make_ecology(pools, seed, initial_count=None, life_capacity=None, bite_events=True, instant_motors=0):
    """Ecology state for `pools`: the food grid of init_world
    (src/main.cu:456-462, seed `seed`), slot bitmaps from the pool owners,
    an empty spatial index and zero counters."""
    P, NC, EC = pools.capacities
    c = np.arange(CELLS, dtype=np.uint64)
    s = _seed_for(seed, c + np.uint64(P))
    u, s = _uniform(s)
    kind = (u * np.float32(3)).astype(np.int32)
    u, s = _uniform(s)
    food = (u < np.float32(0.28)).astype(np.int32)

    def bitmap(owner):
        words = np.zeros((len(owner) + 31) // 32, np.uint32)
        used = np.nonzero(owner >= 0)[0]
        np.bitwise_or.at(words, used // 32, (np.uint32(1) << (used % 32).astype(np.uint32)))
        return words

    one = lambda: np.zeros(1, np.int32)
    return Ecology(food=food, kind=kind, cell_head=np.full(CELLS, -1, np.int32), cell_next=np.full(P, -1, np.int32),
                   bite_intent=np.zeros(P, np.uint8), neuron_used=bitmap(pools.neuron_owner),
                   synapse_used=bitmap(pools.synapse_owner), founder_motor_steps=np.zeros(M, np.int32),
                   founder_observed_steps=one(), deaths=one(), predation_deaths=one(), bites=one(),
                   life_records=np.zeros(life_capacity if life_capacity is not None else 16 * P, LIFE_RECORD),
                   life_count=one(), bite_events=np.zeros(2 * P, BITE_EVENT) if bite_events else None,
                   bite_event_count=one(), neuron_clone=np.zeros(NC, np.int32), births=one(),
                   next_id=np.array([int(pools.animals["id"].max()) + 1], np.int32),
                   initial_count=P if initial_count is None else int(initial_count), instant_motors=instant_motors)


def place_bodies(pools, seed, energy=14.0, health=10.0):
    """Bodies for the living animals as init_animals gives founders
    (src/main.cu:527-541): uniform position and heading, energy 14, health 10."""
    rng = np.random.default_rng(seed)
    A = pools.animals
    live = np.nonzero(A["alive"] == 1)[0]
    A["x"][live] = rng.uniform(0, GRID - 1, len(live)).astype(np.float32)
    A["y"][live] = rng.uniform(0, GRID - 1, len(live)).astype(np.float32)
    A["heading"][live] = rng.uniform(0, 2 * np.pi, len(live)).astype(np.float32)
    A["energy"][live] = energy
    A["health"][live] = health
    return pools


def empty_pools(animal_capacity, neuron_capacity, synapse_capacity, cohort=False):
    a = np.zeros(animal_capacity, ANIMAL)
    a["neuron_head"] = -1
    a["synapse_head"] = -1
    a["ports"] = -1
    return WorldPools(
        animals=a, plasticity_cohort=np.zeros(animal_capacity, COHORT) if cohort else None,
        neurons=np.zeros(neuron_capacity, NEURON_GENE), synapses=np.zeros(synapse_capacity, SYNAPSE_GENE),
        neuron_state=np.zeros(neuron_capacity, NEURON_STATE), synapse_state=np.zeros(synapse_capacity, SYNAPSE_STATE),
        pending_exc=np.zeros((neuron_capacity, 4), np.float32), pending_inh=np.zeros(neuron_capacity, np.float32),
        senses=np.zeros((animal_capacity, S), np.float32),
        mod_event_tick=np.zeros((neuron_capacity, 6), np.uint64),
        spike_history=np.zeros((HIST, neuron_capacity), np.uint8),
        neuron_owner=np.full(neuron_capacity, -1, np.int32), synapse_owner=np.full(synapse_capacity, -1, np.int32),
        neuron_next=np.full(neuron_capacity, -1, np.int32), synapse_next=np.full(synapse_capacity, -1, np.int32),
        neuron_port=np.full(neuron_capacity, -1, np.int32), motors=np.zeros((animal_capacity, M), np.int32))


def _records(a, dtype):
    """Records as a 1-D array of `dtype` (from uint8 rows or the dtype itself)."""
    a = np.ascontiguousarray(a)
    if a.dtype == dtype:
        return a.reshape(-1)
    return a.view(np.uint8).reshape(-1, dtype.itemsize).view(dtype).reshape(-1)


def place_population(batch, neuron_genes, neuron_states, synapse_genes, synapse_states, *, animal_capacity=None,
                     neuron_capacity=None, synapse_capacity=None, scatter_seed=None, animal_slots=None,
                     receptor_baseline=7.0, cohort=False):
    """Lay out a population of Gym-ABI genomes (a workloads.Batch with 19
    world channels and 5 motor outputs) as world pools.

    neuron_genes/states, synapse_genes/states: the brains' records in the
    reference layouts, concatenated in batch order (synapse pre/post
    brain-local). Animal b goes to slot animal_slots[b] (default b), with id
    1000 + b, alive, age 1. With scatter_seed the neuron and synapse slots of
    all animals are a random permutation of the pools (lists interleaved),
    and each animal's lists run in a random order; otherwise slots are
    contiguous and lists run in row order. Sensory neurons keep their world
    channel in the gene (receptor baseline `receptor_baseline` Hz for type 5
    on channels below 6) and take port = channel; motor k takes port 19 + k.
    """
    B = batch.brains
    no, so = batch.neuron_offsets, batch.synapse_offsets
    N, E = int(no[-1]), int(so[-1])
    P = animal_capacity or B
    NC = neuron_capacity or N
    EC = synapse_capacity or E
    pools = empty_pools(P, NC, EC, cohort)
    slots_a = np.arange(B) if animal_slots is None else np.asarray(animal_slots)
    if scatter_seed is None:
        nslot = np.arange(N)
        eslot = np.arange(E)
        rng = None
    else:
        rng = np.random.default_rng(scatter_seed)
        nslot = rng.permutation(NC)[:N]
        eslot = rng.permutation(EC)[:E]
    ng = _records(neuron_genes, NEURON_GENE).copy()
    sg = _records(synapse_genes, SYNAPSE_GENE).copy()
    ch = batch.neuron_rows[:, 1].astype(np.int32)
    ng["sensory_channel"] = np.where((ch >= 0) & (ch < S), ch, -1).astype(np.int8)
    ng["rec_base"] = np.where((ng["type"] == 5) & (ch >= 0) & (ch < 6), receptor_baseline, 0.0)
    pools.neurons[nslot] = ng
    pools.neuron_state[nslot] = _records(neuron_states, NEURON_STATE)
    nb = np.repeat(np.arange(B), np.diff(no))
    sb = np.repeat(np.arange(B), np.diff(so))
    sg["pre"] = nslot[no[sb] + sg["pre"]]
    sg["post"] = nslot[no[sb] + sg["post"]]
    pools.synapses[eslot] = sg
    pools.synapse_state[eslot] = _records(synapse_states, SYNAPSE_STATE)
    pools.neuron_owner[nslot] = slots_a[nb]
    pools.synapse_owner[eslot] = slots_a[sb]
    port = np.where((ch >= 0) & (ch < S), ch, -1)
    mo = batch.motors
    for k in range(min(M, mo.shape[1])):
        port[no[:-1] + mo[:, k]] = S + k
    pools.neuron_port[nslot] = port
    A = pools.animals
    for b in range(B):
        a = int(slots_a[b])
        ln = nslot[no[b]:no[b + 1]]
        le = eslot[so[b]:so[b + 1]]
        if rng is not None:
            ln = ln[rng.permutation(len(ln))]
            le = le[rng.permutation(len(le))]
        if len(ln):
            pools.neuron_next[ln[:-1]] = ln[1:]
            A["neuron_head"][a] = ln[0]
        if len(le):
            pools.synapse_next[le[:-1]] = le[1:]
            A["synapse_head"][a] = le[0]
        A["neuron_count"][a] = len(ln)
        A["synapse_count"][a] = len(le)
        A["alive"][a] = 1
        A["id"][a] = 1000 + b
        A["age"][a] = 1
        pt = port[no[b]:no[b + 1]]
        for p in range(S + M):
            hit = np.nonzero(pt == p)[0]
            A["ports"][a, p] = nslot[no[b] + hit[0]] if len(hit) else -1
    if batch.inputs is not None and batch.inputs.shape[1] == S:
        pools.senses[slots_a] = batch.inputs
    return pools


def records_from_gpu(batch, seeds):
    """Reset states of the batch's brains (one seed per brain), as reference
    records, computed by the library's batch engine: (neuron genes, neuron
    states, synapse genes, synapse states), concatenated in batch order."""
    g = native.GpuBatch.from_rows(batch)
    try:
        g.reset(np.asarray(seeds, np.uint32))
        nrec, srec, _ = g.checkpoint_export()
    finally:
        g.close()
    ng = nrec[:, 16:140].copy().view(NEURON_GENE).reshape(-1)
    ns = nrec[:, 140:260].copy().view(NEURON_STATE).reshape(-1)
    sg = srec[:, 12:52].copy().view(SYNAPSE_GENE).reshape(-1)
    ss = srec[:, 56:136].copy().view(SYNAPSE_STATE).reshape(-1)
    return ng, ns, sg, ss


class World:
    """The library's world stage over device copies of `pools` (torch CUDA
    tensors; the pools stay resident between steps)."""

    def __init__(self, pools: WorldPools, max_brain_neurons=0, max_brain_synapses=0, device="cuda"):
        import torch
        self.torch = torch
        self.lib = native.library()
        self.host = pools
        self.dev = {}
        for n in ARRAYS:
            a = getattr(pools, n)
            if a is None:
                self.dev[n] = None
                continue
            raw = np.ascontiguousarray(a).view(np.uint8).reshape(-1)
            self.dev[n] = torch.from_numpy(raw.copy()).to(device)
        s = NsbWorldPools()
        for n in ARRAYS:
            t = self.dev[n]
            setattr(s, n, None if t is None else t.data_ptr())
        s.trace_animal, s.silence_senses, s.silence_contact = pools.trace_animal, pools.silence_senses, \
            pools.silence_contact
        s.animal_capacity, s.neuron_capacity, s.synapse_capacity = pools.capacities
        self.struct = s
        self.ptr = self.lib.nsb_world_create(ct.byref(s), int(max_brain_neurons), int(max_brain_synapses))
        if not self.ptr:
            raise RuntimeError(self.lib.ns_error().decode())

    def neural_step(self, step):
        if self.lib.nsb_world_neural_step(self.ptr, int(step)) != 0:
            raise RuntimeError(self.lib.ns_error().decode())

    def homeostasis(self):
        if self.lib.nsb_world_homeostasis(self.ptr) != 0:
            raise RuntimeError(self.lib.ns_error().decode())

    def stats(self):
        out = (ct.c_longlong * 4)()
        self.lib.nsb_world_stats(self.ptr, out)
        return dict(zip(("animals", "neurons", "synapses", "events"), list(out)))

    def upload(self, name, array):
        """Replace one pool on the device (e.g. senses or animals between steps)."""
        raw = np.ascontiguousarray(array).view(np.uint8).reshape(-1)
        self.dev[name].copy_(self.torch.from_numpy(raw))
        setattr(self.host, name, array)

    def download(self) -> WorldPools:
        out = self.host.copy()
        for n in ARRAYS:
            t = self.dev[n]
            if t is None:
                continue
            a = getattr(out, n)
            a.view(np.uint8).reshape(-1)[:] = t.cpu().numpy()
        return out

    def close(self):
        if getattr(self, "eco", None):
            self.lib.nsb_world_ecology_destroy(self.eco)
            self.eco = None
        if getattr(self, "ptr", None):
            self.lib.nsb_world_destroy(self.ptr)
            self.ptr = None

    __del__ = close

    # ---- ecology (the rest of the world step) ----
    def attach_ecology(self, ecology: Ecology):
        """Upload `ecology` and bind the library's ecology stage to it and to
        this world's pools."""
        torch = self.torch
        dev = next(t for t in self.dev.values() if t is not None).device
        self.eco_host = ecology
        self.eco_dev = {}
        for n in ECO_ARRAYS:
            a = getattr(ecology, n)
            self.eco_dev[n] = None if a is None else torch.from_numpy(
                np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).to(dev)
        s = NsbWorldEcology()
        for n in ECO_ARRAYS:
            t = self.eco_dev[n]
            setattr(s, n, None if t is None else t.data_ptr())
        s.initial_count, s.instant_motors = ecology.initial_count, ecology.instant_motors
        s.life_capacity = 0 if ecology.life_records is None else len(ecology.life_records)
        self.eco_struct = s
        self.eco = self.lib.nsb_world_ecology_create(ct.byref(self.struct), ct.byref(s))
        if not self.eco:
            raise RuntimeError(self.lib.ns_error().decode())

    def _eco_call(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ns_error().decode())

    def body_step(self, step):
        self._eco_call(self.lib.nsb_world_body_step(self.eco, int(step)))

    def reclaim(self, step):
        self._eco_call(self.lib.nsb_world_reclaim(self.eco, int(step)))

    def reproduce(self):
        self._eco_call(self.lib.nsb_world_reproduce(self.eco))

    def regrow_and_sense(self, step, seed, renewal_probability):
        self._eco_call(self.lib.nsb_world_regrow_and_sense(self.eco, int(step), int(seed),
                                                            float(renewal_probability)))

    def upload_ecology(self, name, array):
        raw = np.ascontiguousarray(array).view(np.uint8).reshape(-1)
        self.eco_dev[name].copy_(self.torch.from_numpy(raw))
        setattr(self.eco_host, name, array)

    def download_ecology(self) -> Ecology:
        out = self.eco_host.copy()
        for n in ECO_ARRAYS:
            t = self.eco_dev[n]
            if t is None:
                continue
            getattr(out, n).view(np.uint8).reshape(-1)[:] = t.cpu().numpy()
        return out
