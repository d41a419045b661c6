"""GPU tests of the world ecology stage (nsb_world_body_step, nsb_world_reclaim,
nsb_world_regrow_and_sense through the C ABI).

A closed world loop: the neural stage, the body step, homeostasis, genome
reclamation, reproduction with mutation (where a test asks for births),
regrowth and senses, with the senses of each step feeding the next step's
neural stage (src/main.cu:2634-2770). Every
pool and every ecology array must equal the oracle's (the reference kernels
restated as loops in ascending slot order) after each step. The populations
crowd animals into a few cells so that harvests of one food unit, bites, kills
and the spatial lists are contended, and give some animals low health and
energy so that deaths, predation deaths and genome reclamation happen.

The last test pins the stage to the reference simulator's own ecology kernels
(src/main.cu built from its sources with IEEE arithmetic and correctly rounded
cos/sin/hypot/exp/log, oracle/ref_world_harness.cu), replayed one animal at a
time in ascending slot order, on full-capacity pools.
"""
import ctypes as ct

import numpy as np
import pytest

from oracle.pyoracle import (HERE, world_body_step, world_homeostasis, world_reclaim, world_regrow_and_sense,
                             world_reproduce, world_step)

pytestmark = pytest.mark.gpu

POOLS = ("neurons", "synapses", "neuron_state", "synapse_state", "pending_exc", "pending_inh", "mod_event_tick",
         "spike_history", "motors", "senses", "animals", "neuron_owner", "synapse_owner", "neuron_next",
         "synapse_next", "neuron_port")
ECO = ("food", "cell_head", "cell_next", "bite_intent", "neuron_used", "synapse_used", "founder_motor_steps",
       "founder_observed_steps", "deaths", "predation_deaths", "bites", "life_records", "life_count", "bite_events",
       "bite_event_count", "neuron_clone", "births", "next_id")


def _bits(a):
    a = np.ascontiguousarray(a)
    if a.dtype.names:
        return a.view(np.uint8).reshape(len(a), -1)
    if a.dtype.kind == "f":
        return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)
    return a


def _same(x, y):
    """Records compared field by field (padding bytes are not state)."""
    if x.dtype.names:
        return all(_same(x[f], y[f]) for f in x.dtype.names)
    return np.array_equal(_bits(x), _bits(y))


def _compare(got_pools, want_pools, got_eco, want_eco, label):
    for name in POOLS:
        assert _same(getattr(got_pools, name), getattr(want_pools, name)), f"{label}: pool {name} differs"
    for name in ECO:
        x, y = getattr(got_eco, name), getattr(want_eco, name)
        if x is None:
            continue
        if name == "life_records":
            n = min(int(want_eco.life_count[0]), len(y))
            x, y = x[:n], y[:n]
        if name == "bite_events":
            n = min(int(want_eco.bite_event_count[0]), len(y))
            x, y = x[:n], y[:n]
        assert _same(x, y), f"{label}: ecology {name} differs"


def _crowd(pools, seed, cells=6):
    """Move most living animals into a few cells (two to a dozen per cell)
    and spread health and energy so that bites kill and animals starve."""
    rng = np.random.default_rng(seed)
    A = pools.animals
    live = np.nonzero(A["alive"] == 1)[0]
    crowd = live[: (len(live) * 2) // 3]
    centres = rng.uniform(8, 120, (cells, 2)).astype(np.float32)
    which = rng.integers(0, cells, len(crowd))
    A["x"][crowd] = np.floor(centres[which, 0]) + rng.uniform(0.05, 0.95, len(crowd)).astype(np.float32)
    A["y"][crowd] = np.floor(centres[which, 1]) + rng.uniform(0.05, 0.95, len(crowd)).astype(np.float32)
    A["health"][live] = rng.choice(np.float32([1.5, 2.0, 3.0, 10.0]), len(live))
    A["energy"][live] = rng.choice(np.float32([0.01, 5.0, 14.0, 25.0]), len(live))
    A["age"][live] = rng.integers(1, 400, len(live))
    A["muscle"][live] = rng.uniform(0, 1, (len(live), 3)).astype(np.float32)


def _population(nsb, seed, founders, animal_capacity, neuron_capacity=None, synapse_capacity=None, cohort=False):
    W = nsb.world
    batch = nsb.workloads.world_founders(seed=seed, founders=founders)
    seeds = np.arange(batch.brains, dtype=np.uint32) * 5 + 1
    N, E = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1])
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds), animal_capacity=animal_capacity,
                               neuron_capacity=neuron_capacity or N + 500, synapse_capacity=synapse_capacity or E + 900,
                               scatter_seed=seed + 1, cohort=cohort)
    W.place_bodies(pools, seed + 2)
    _crowd(pools, seed + 3)
    # the first ids are founders (motor statistics)
    pools.animals["id"][pools.animals["alive"] == 1] = np.arange(batch.brains)
    return pools


def _closed_loop(nsb, pools, eco, steps, seed, renewal, label, births=False):
    W = nsb.world
    world = W.World(pools)
    world.attach_ecology(eco)
    ref, ref_eco = pools.copy(), eco.copy()
    # initial senses (the host loop senses before its first step)
    world.regrow_and_sense(0, seed, 0.0)
    world_regrow_and_sense(ref, ref_eco, 0, seed, 0.0)
    try:
        for step in range(1, steps + 1):
            world.neural_step(step)
            world_step(ref, step)
            world.body_step(step)
            world_body_step(ref, ref_eco, step)
            world.homeostasis()
            world_homeostasis(ref)
            world.reclaim(step)
            world_reclaim(ref, ref_eco, step)
            if births:
                world.reproduce()
                world_reproduce(ref, ref_eco)
            world.regrow_and_sense(step, seed, renewal)
            world_regrow_and_sense(ref, ref_eco, step, seed, renewal)
            _compare(world.download(), ref, world.download_ecology(), ref_eco, f"{label} step {step}")
    finally:
        world.close()
    return ref, ref_eco


@pytest.mark.parametrize("instant", [0, 1])
def test_ecology_closed_loop_matches_oracle(nsb, oracle_built, instant):
    W = nsb.world
    pools = _population(nsb, 21 + instant, founders=160, animal_capacity=224)
    eco = W.make_ecology(pools, seed=2, initial_count=120, life_capacity=64, instant_motors=instant)
    ref, ref_eco = _closed_loop(nsb, pools, eco, 12, seed=2, renewal=0.02, label=f"instant={instant}")
    # the population exercised the contended paths
    assert ref_eco.bites[0] > 0 and ref_eco.predation_deaths[0] > 0
    assert ref_eco.deaths[0] > ref_eco.predation_deaths[0]
    assert ref_eco.life_count[0] > 0 and ref_eco.founder_observed_steps[0] > 0
    assert W.behavior(ref.animals)["accepted"].sum() > 0
    assert W.behavior(ref.animals)["empty_eat"].sum() > 0


def test_ecology_life_records_past_capacity_and_no_bite_events(nsb, oracle_built):
    """More reclaimed genomes than life records (the count still advances) and
    no bite-event buffer (the event counter stays)."""
    W = nsb.world
    pools = _population(nsb, 31, founders=96, animal_capacity=128)
    pools.animals["health"][pools.animals["alive"] == 1] = 0.0
    eco = W.make_ecology(pools, seed=5, initial_count=0, life_capacity=3, bite_events=False)
    ref, ref_eco = _closed_loop(nsb, pools, eco, 3, seed=5, renewal=0.0, label="capacity")
    assert ref_eco.life_count[0] > 3 and ref_eco.bite_event_count[0] == 0
    assert not (ref.neuron_owner >= 0).any()


def test_ecology_reclaims_long_and_short_lists(nsb, oracle_built):
    """Every animal dies in the first body step: lists from a few synapses to
    more than the 4,096 that are ranked in shared memory (those are walked),
    all recorded and released."""
    W, wl = nsb.world, nsb.workloads
    batch = wl.concat([wl.world_founders(seed=61, founders=20, lo=4, hi=40, epn_lo=1, epn_hi=6),
                       wl.world_founders(seed=62, founders=3, lo=380, hi=420, epn_lo=12, epn_hi=13)], "reclaim")
    seeds = np.arange(batch.brains, dtype=np.uint32) + 9
    N, E = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1])
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds), animal_capacity=40,
                               neuron_capacity=N + 100, synapse_capacity=E + 300, scatter_seed=63)
    assert pools.animals["synapse_count"].max() > 4096
    W.place_bodies(pools, 64)
    pools.animals["health"][pools.animals["alive"] == 1] = 0.0
    eco = W.make_ecology(pools, seed=3, life_capacity=64)
    ref, ref_eco = _closed_loop(nsb, pools, eco, 1, seed=3, renewal=0.0, label="reclaim")
    assert ref_eco.life_count[0] == batch.brains
    assert ref_eco.life_records["active_synapses"][:batch.brains].max() > 4096
    assert not (ref.synapse_owner >= 0).any() and not ref_eco.synapse_used.any()


def test_reproduction_closed_loop_matches_oracle(nsb, oracle_built):
    """Births with mutation in the closed loop: 30 of 120 founders well fed
    (energy 100) reproduce every step, some in crowded cells and some of them
    dying, so the births reuse reclaimed animal and pool slots. About 240
    births over 8 steps draw every mutation choice."""
    W = nsb.world
    pools2 = _population(nsb, 71, founders=120, animal_capacity=400, neuron_capacity=60000,
                         synapse_capacity=600000)
    pools2.animals["energy"][np.nonzero(pools2.animals["alive"] == 1)[0][::4]] = 100.0
    eco = W.make_ecology(pools2, seed=9, initial_count=60, life_capacity=256)
    ref, ref_eco = _closed_loop(nsb, pools2, eco, 8, seed=9, renewal=0.01, label="births", births=True)
    assert ref_eco.births[0] > 150
    assert ref_eco.next_id[0] == eco.next_id[0] + ref_eco.births[0]
    assert (ref.animals["generation"] > 0).sum() > 100
    counts = ref.animals["neuron_count"][ref.animals["generation"] > 0]
    assert len(np.unique(counts)) > 10                  # mutation changed brain sizes


def test_reproduction_with_full_pools_undoes_births(nsb, oracle_built):
    """Pools with little room: births that run out of neuron or synapse slots
    midway are released again (src/main.cu:1712-1717)."""
    W = nsb.world
    pools = _population(nsb, 81, founders=40, animal_capacity=60)
    pools.animals["energy"][pools.animals["alive"] == 1] = 60.0
    eco = W.make_ecology(pools, seed=4, initial_count=0, life_capacity=64)
    ref, ref_eco = _closed_loop(nsb, pools, eco, 2, seed=4, renewal=0.0, label="full", births=True)
    assert 0 < ref_eco.births[0] < 80
    # a parent left without offspring while animal slots were free: its birth was undone
    A = ref.animals
    assert (A["alive"] == 0).any() and ((A["alive"] == 1) & (A["energy"] > 55) & (A["generation"] == 0)).any()


def _words_for_long_scans(full_words, hints, min_run=300):
    """A bitmap size in words, above full_words, for which at least three of
    `hints` (taken modulo the size) start more than min_run full words before
    the end of the packed run [0, full_words)."""
    for words in range(full_words + 64, full_words + 4000):
        if sum((h % words) < full_words - min_run for h in hints) >= 3:
            return words
    raise AssertionError("no bitmap size found")


def test_births_search_past_the_first_256_candidates(nsb, oracle_built):
    """Birth searches that need more than one round of 256 candidates (the
    loops whose exits are decided by __syncthreads_or): 590 living animals in
    600 slots with only the last ten free, so most parents' drawn starts lie
    more than 256 live slots before a free one; neuron and synapse slots
    packed, with pool sizes chosen so that several children's hint words
    (child*131, child*257) start more than 300 full bitmap words before a
    free bit. Twelve parents for ten free slots: the last two find no slot.
    Every pool, bitmap and counter equals the oracle's after each step."""
    W = nsb.world
    batch = nsb.workloads.world_founders(seed=91, founders=590, lo=32, hi=40, epn_lo=4, epn_hi=5)
    seeds = np.arange(batch.brains, dtype=np.uint32) * 3 + 7
    N, E = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1])
    children = range(590, 596)
    nwords = _words_for_long_scans(N // 32, [c * 131 for c in children])
    swords = _words_for_long_scans(E // 32, [c * 257 for c in children])
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds), animal_capacity=600,
                               neuron_capacity=32 * nwords, synapse_capacity=32 * swords)
    W.place_bodies(pools, 93)
    alive = np.nonzero(pools.animals["alive"] == 1)[0]
    assert len(alive) == 590 and alive.max() == 589
    pools.animals["id"][alive] = np.arange(len(alive))
    pools.animals["energy"][alive[::49][:12]] = 100.0
    eco = W.make_ecology(pools, seed=5, initial_count=0, life_capacity=64)
    ref, ref_eco = _closed_loop(nsb, pools, eco, 2, seed=5, renewal=0.0, label="long searches", births=True)
    assert ref_eco.births[0] == 10                         # every free slot filled, two parents without one
    assert (ref.animals["alive"] == 1).sum() == 600


def test_ecology_reports_bad_lists(nsb):
    """A dead animal whose neuron list is shorter than its count: reclamation
    walks the list (at most count + 1 entries) and reports it."""
    W = nsb.world
    pools = _population(nsb, 41, founders=8, animal_capacity=16)
    A = pools.animals
    A["alive"][3] = 0
    A["neuron_count"][3] += 2
    eco = W.make_ecology(pools, seed=1)
    world = W.World(pools)
    world.attach_ecology(eco)
    with pytest.raises(RuntimeError, match="lists disagree"):
        world.reclaim(1)
    world.close()


def _ref_eco_lib():
    path = HERE / "_ref" / "libns_ref_world_cr.so"
    if not path.exists():
        return None
    lib = ct.CDLL(str(path))
    lib.ref_world_eco_create.restype = ct.c_void_p
    lib.ref_world_eco_create.argtypes = [ct.c_void_p, ct.c_void_p]
    lib.ref_world_eco_body.argtypes = [ct.c_void_p, ct.c_longlong, ct.c_int]
    lib.ref_world_eco_reclaim.argtypes = [ct.c_void_p, ct.c_longlong, ct.c_int]
    lib.ref_world_eco_regrow_and_sense.argtypes = [ct.c_void_p, ct.c_longlong, ct.c_ulonglong, ct.c_float,
                                                   ct.c_int]
    for f in ("ref_world_eco_body", "ref_world_eco_reclaim", "ref_world_eco_regrow_and_sense"):
        getattr(lib, f).restype = ct.c_int
    lib.ref_world_eco_destroy.argtypes = [ct.c_void_p]
    lib.ref_world_eco_reproduce.argtypes = [ct.c_void_p, ct.c_int]
    lib.ref_world_eco_reproduce.restype = ct.c_int
    return lib


@pytest.mark.parametrize("births", [False, True])
def test_ecology_matches_reference_kernels(nsb, births):
    """Both sides run this library's neural stage (pinned separately); the
    ecology kernels are this stage's on one copy of the pools and the
    reference's own, replayed in slot order, on the other. With births,
    a third of the animals are well fed and reproduce every step (the
    reference's reproduce with mutate, one parent at a time)."""
    ref = _ref_eco_lib()
    if ref is None:
        pytest.skip("oracle/_ref/libns_ref_world_cr.so not built")
    W = nsb.world
    pools = _population(nsb, 51, founders=72, animal_capacity=32768, neuron_capacity=4194304,
                        synapse_capacity=8388608)
    if births:
        live = np.nonzero(pools.animals["alive"] == 1)[0]
        pools.animals["energy"][live[::3]] = 100.0
    eco = W.make_ecology(pools, seed=7, initial_count=40, life_capacity=32768 * 16)
    ours = W.World(pools)
    ours.attach_ecology(eco)
    theirs = W.World(pools)
    theirs.attach_ecology(eco)
    h = ref.ref_world_eco_create(ct.byref(theirs.struct), ct.byref(theirs.eco_struct))
    assert h, "reference ecology setup failed"
    try:
        ours.regrow_and_sense(0, 7, 0.0)
        assert ref.ref_world_eco_regrow_and_sense(h, 0, 7, 0.0, 1) == 0
        for step in range(1, 7):
            ours.neural_step(step)
            theirs.neural_step(step)
            ours.body_step(step)
            assert ref.ref_world_eco_body(h, step, 1) == 0
            ours.homeostasis()
            theirs.homeostasis()
            ours.reclaim(step)
            assert ref.ref_world_eco_reclaim(h, step, 1) == 0
            if births:
                ours.reproduce()
                assert ref.ref_world_eco_reproduce(h, 1) == 0
            ours.regrow_and_sense(step, 7, 0.05)
            assert ref.ref_world_eco_regrow_and_sense(h, step, 7, 0.05, 1) == 0
            want_eco = theirs.download_ecology()
            _compare(ours.download(), theirs.download(), ours.download_ecology(), want_eco, f"step {step}")
        assert want_eco.bites[0] > 0 and want_eco.deaths[0] > 0 and want_eco.life_count[0] > 0
        assert want_eco.births[0] > (100 if births else -1)
    finally:
        ref.ref_world_eco_destroy(h)
        ours.close()
        theirs.close()
