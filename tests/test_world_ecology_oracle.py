"""CPU checks of the oracle's world ecology restatement (or_world_body_step,
or_world_reclaim, or_world_reproduce, or_world_regrow_and_sense) on small
hand-built situations with known outcomes. These pin the slot-order rule by
which contended steps resolve (src/main.cu:612-657, 1138-1737 run as loops in
ascending animal slot order), and invariants the world keeps.
"""
import numpy as np
import pytest

from oracle.pyoracle import (oracle_records, world_body_step, world_reclaim, world_regrow_and_sense,
                             world_reproduce)


def _pools(nsb, founders=12, capacity=32, seed=5):
    W = nsb.world
    batch = nsb.workloads.world_founders(seed=seed, founders=founders)
    seeds = np.arange(batch.brains, dtype=np.uint32) + 1
    N, E = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1])
    # capacities in whole bitmap words (a claim that finds its first free bit
    # past the capacity fails, src/main.cu:376-379)
    pools = W.place_population(batch, *oracle_records(batch, seeds), animal_capacity=capacity,
                               neuron_capacity=(N + 3000) // 32 * 32, synapse_capacity=(E + 30000) // 32 * 32,
                               scatter_seed=seed)
    W.place_bodies(pools, seed)
    A = pools.animals
    A["id"][:founders] = np.arange(founders)
    # everyone far apart and idle unless a test says otherwise
    A["x"][:founders] = 3.5 + 9.0 * np.arange(founders)
    A["y"][:founders] = 100.5
    A["heading"][:founders] = 0.0
    A["muscle"][:founders] = 0.0
    return pools


def _together(pools, slots, x=40.5, y=40.5):
    pools.animals["x"][slots] = x
    pools.animals["y"][slots] = y


def test_one_food_unit_goes_to_the_lowest_eating_slot(nsb, oracle_built):
    W = nsb.world
    pools = _pools(nsb)
    _together(pools, [2, 5, 9])
    eco = W.make_ecology(pools, seed=1)
    c = 40 * 128 + 40
    eco.food[:] = 0
    eco.food[c] = 1
    eco.kind[c] = 0
    pools.motors[[2, 5, 9], 3] = 1                   # all three eat
    world_body_step(pools, eco, 1)
    B = W.behavior(pools.animals)
    assert eco.food[c] == 0
    assert B["accepted"][2].sum() == 1 and B["accepted"][5].sum() == 0 and B["accepted"][9].sum() == 0
    assert B["empty_eat"][5].sum() == 1 and B["empty_eat"][9].sum() == 1
    assert pools.animals["taste"][2, 0] == np.float32(1.0)


def test_bites_run_in_slot_order_and_the_second_bite_kills(nsb, oracle_built):
    """Three animals in one cell, all biting. The cell list runs 9, 5, 2, so
    attacker 2 bites 9 (health 3 -> 1), attacker 5 bites 9 again and kills it
    (its previous health 1 <= 2), attacker 9 is dead by its turn."""
    W = nsb.world
    pools = _pools(nsb)
    _together(pools, [2, 5, 9])
    A = pools.animals
    A["health"][[2, 5, 9]] = [10.0, 10.0, 3.0]
    A["energy"][[2, 5, 9]] = [10.0, 10.0, 12.0]
    eco = W.make_ecology(pools, seed=1)
    eco.food[:] = 0
    pools.motors[[2, 5, 9], 4] = 1
    world_body_step(pools, eco, 7)
    c = 40 * 128 + 40
    # indexed before the bites, 9 still alive: the list runs 9, 5, 2
    assert eco.cell_head[c] == 9 and eco.cell_next[9] == 5 and eco.cell_next[5] == 2 and eco.cell_next[2] == -1
    assert eco.bites[0] == 2 and eco.bite_event_count[0] == 2
    ev = eco.bite_events[:2]
    assert list(ev["attacker_id"]) == [2, 5] and list(ev["prey_id"]) == [9, 9] and list(ev["step"]) == [7, 7]
    assert A["alive"][9] == 0 and W.behavior(A)["death_cause"][9] == 1
    assert eco.predation_deaths[0] == 1
    assert A["taste"][5, 3] == np.float32(1.0) and A["taste"][2, 3] != np.float32(1.0)
    # meat: 45 % of the prey's energy after its own body step
    assert A["energy"][5] > A["energy"][2]


def test_spatial_lists_run_from_the_highest_slot(nsb, oracle_built):
    W = nsb.world
    pools = _pools(nsb)
    _together(pools, [1, 4, 7, 11], x=60.2, y=20.7)
    _together(pools, [3], x=62.2, y=20.7)             # two cells ahead along heading 0
    eco = W.make_ecology(pools, seed=1)
    world_regrow_and_sense(pools, eco, 0, 1, 0.0)
    c = 20 * 128 + 60
    order, q = [], eco.cell_head[c]
    while q >= 0:
        order.append(int(q))
        q = eco.cell_next[q]
    assert order == [11, 7, 4, 1]
    # the straight-ahead ray (ranges 1-4 cells) finds animal 3 once: 0.25
    assert all(pools.senses[a, 13] == np.float32(0.25) for a in (1, 4, 7, 11))


def test_reclaim_records_in_slot_order_and_releases_slots(nsb, oracle_built):
    W = nsb.world
    pools = _pools(nsb)
    A = pools.animals
    A["alive"][[8, 3, 6]] = 0
    eco = W.make_ecology(pools, seed=1, life_capacity=2)
    counts = A["neuron_count"][[3, 6, 8]].copy()
    world_reclaim(pools, eco, 11)
    assert eco.life_count[0] == 3                     # counted past the 2 records
    rec = eco.life_records[:2]
    assert list(rec["body"]["id"]) == [3, 6] and list(rec["death_step"]) == [11, 11]
    for a in (3, 6, 8):
        assert A["neuron_head"][a] == -1 and A["neuron_count"][a] == 0 and (A["ports"][a] == -1).all()
    assert not np.isin(pools.neuron_owner, [3, 6, 8]).any()
    used = np.unpackbits(eco.neuron_used.view(np.uint8), bitorder="little")[:len(pools.neuron_owner)]
    assert np.array_equal(used.astype(bool), pools.neuron_owner >= 0)
    assert rec["active_neurons"][0] <= counts[0]


def test_food_grid_matches_a_scalar_restatement_of_init_world(nsb):
    """make_ecology's vectorised init_world (src/main.cu:456-462) against the
    same seed hash and xorshift64* draws written as scalar Python."""
    W = nsb.world
    pools = _pools(nsb)
    eco = W.make_ecology(pools, seed=2)
    P = pools.capacities[0]
    M = (1 << 64) - 1

    def seed_for(seed, i):
        x = (seed + 0x9e3779b97f4a7c15 * (i + 1)) & M
        x = ((x ^ (x >> 30)) * 0xbf58476d1ce4e5b9) & M
        x = ((x ^ (x >> 27)) * 0x94d049bb133111eb) & M
        return (x ^ (x >> 31)) | 1

    def uniform(s):
        s ^= s >> 12
        s ^= (s << 25) & M
        s ^= s >> 27
        r = (s * 2685821657736338717) & M
        return np.float32((r >> 40) * (1.0 / 16777216.0)), s

    for c in list(range(0, 16384, 997)) + [16383]:
        s = seed_for(2, c + P)
        u, s = uniform(s)
        kind = int(u * np.float32(3))
        u, s = uniform(s)
        assert eco.kind[c] == kind and eco.food[c] == int(u < np.float32(0.28)), c


def _walk(nxt, head, limit):
    out, q = [], head
    while q >= 0 and len(out) <= limit:
        out.append(int(q))
        q = nxt[q]
    return out


def test_reproduction_keeps_the_pools_consistent(nsb, oracle_built):
    W = nsb.world
    pools = _pools(nsb, founders=12, capacity=40)
    A = pools.animals
    A["energy"][[0, 4, 7]] = 30.0
    eco = W.make_ecology(pools, seed=1)
    next_id = int(eco.next_id[0])
    world_reproduce(pools, eco)
    assert eco.births[0] == 3 and eco.next_id[0] == next_id + 3
    kids = np.nonzero(A["generation"] == 1)[0]
    assert len(kids) == 3 and (A["alive"][kids] == 1).all()
    assert sorted(A["parent_id"][kids]) == [0, 4, 7]
    assert np.allclose(A["energy"][[0, 4, 7]], 20.0)
    assert (W.behavior(A)["offspring"][[0, 4, 7]] == 1).all()
    for a in np.nonzero(A["alive"] == 1)[0]:
        ns = _walk(pools.neuron_next, A["neuron_head"][a], A["neuron_count"][a])
        es = _walk(pools.synapse_next, A["synapse_head"][a], A["synapse_count"][a])
        assert len(ns) == A["neuron_count"][a] and len(es) == A["synapse_count"][a]
        assert (pools.neuron_owner[ns] == a).all() and (pools.synapse_owner[es] == a).all()
        # synapses stay inside the animal
        assert np.isin(pools.synapses["pre"][es], ns).all() and np.isin(pools.synapses["post"][es], ns).all()
    for owner, words in ((pools.neuron_owner, eco.neuron_used), (pools.synapse_owner, eco.synapse_used)):
        used = np.unpackbits(words.view(np.uint8), bitorder="little")[:len(owner)].astype(bool)
        assert np.array_equal(used, owner >= 0)
    # a second run from the same state gives the same world
    pools2, eco2 = pools.copy(), eco.copy()
    A["energy"][kids] = 40.0
    pools2.animals["energy"][kids] = 40.0
    world_reproduce(pools, eco)
    world_reproduce(pools2, eco2)
    assert np.array_equal(pools.animals.view(np.uint8), pools2.animals.view(np.uint8))
    assert np.array_equal(eco.neuron_used, eco2.neuron_used)


def test_body_step_death_causes_and_food_kind_one(nsb, oracle_built):
    """Known answers of body_step (src/main.cu:1146-1249) in binary32:
    starvation (cause 2), old age (cause 4), and a meal of food kind 1
    (energy +2, health and pain 1.4, first_b_age)."""
    W = nsb.world
    pools = _pools(nsb)
    A = pools.animals
    f32 = np.float32
    A["energy"][1], A["health"][1] = 0.001, 0.1          # starves
    A["age"][2] = 9999                                   # dies of age
    A["energy"][3], A["health"][3], A["age"][3] = 12.0, 10.0, 150
    eco = W.make_ecology(pools, seed=1)
    eco.food[:] = 0
    c3 = int(A["y"][3]) * 128 + int(A["x"][3])
    eco.food[c3], eco.kind[c3] = 1, 1
    pools.motors[3, 3] = 2                               # eats
    before = A[[1, 2, 3]].copy()
    world_body_step(pools, eco, 1)
    B = W.behavior(A)
    assert A["alive"][1] == 0 and B["death_cause"][1] == 2 and A["energy"][1] == 0
    assert A["health"][1] == f32(f32(0.1) - f32(0.15))
    assert A["alive"][2] == 0 and B["death_cause"][2] == 4 and A["age"][2] == 10000
    assert eco.deaths[0] == 2
    # animal 3: upkeep first, then the meal (energy capped at 30)
    active = int(pools.neurons["active"][pools.neuron_owner == 3].sum())
    e = f32(12.0) - (f32(f32(0.003) + f32(active) * f32(0.00002)) + f32(0.0) * f32(0.02) + f32(0.0))
    assert A["energy"][3] == min(f32(30), f32(e + f32(2)))
    assert A["health"][3] == f32(f32(10.0) - f32(1.4)) and A["pain"][3] == f32(f32(before["pain"][2] * f32(0.8)) + f32(1.4))
    assert B["first_b_age"][3] == 151 and B["accepted"][3, 1, 0, 1] == 1 and eco.food[c3] == 0
    assert A["age"][3] == 151 and A["alive"][3] == 1


def test_muscle_twitch_moves_along_the_heading(nsb, oracle_built):
    """Thrust from three spikes on the thrust motor: muscle = min(1, 0.9231
    m + 0.3 spikes) (src/main.cu:1152-1160); heading 0 moves along +x by
    thrust x 1.5 (cos 0 = 1 exactly, sin 0 = 0)."""
    W = nsb.world
    pools = _pools(nsb)
    A = pools.animals
    f32 = np.float32
    A["muscle"][4] = [0.5, 0.0, 0.0]
    x0, y0 = A["x"][4], A["y"][4]
    eco = W.make_ecology(pools, seed=1)
    pools.motors[4, 0] = 3
    world_body_step(pools, eco, 1)
    m = min(f32(1.0), f32(f32(f32(0.5) * f32(0.92311635)) + f32(f32(3) * f32(0.30))))
    assert A["muscle"][4, 0] == m
    assert A["x"][4] == f32(x0 + f32(m * f32(1.5))) and A["y"][4] == y0
    assert (pools.motors[4] == 0).all()


def test_place_population_and_make_ecology_are_consistent(nsb):
    """Host helpers (world.py): scattered pools give each animal lists of its
    own slots with ports on its sensory and motor neurons; the ecology's slot
    bitmaps mark exactly the owned slots; record layouts match the reference
    sizes (LifeRecord 504 B, BiteEvent 24 B, Behavior 276 B)."""
    W = nsb.world
    assert (W.LIFE_RECORD.itemsize, W.BITE_EVENT.itemsize, W.BEHAVIOR.itemsize) == (504, 24, 276)
    assert W.LIFE_RECORD.fields["death_step"][1] == 472
    pools = _pools(nsb, founders=10, capacity=16)
    A = pools.animals
    for a in range(10):
        ns = _walk(pools.neuron_next, A["neuron_head"][a], A["neuron_count"][a])
        es = _walk(pools.synapse_next, A["synapse_head"][a], A["synapse_count"][a])
        assert len(ns) == A["neuron_count"][a] and len(es) == A["synapse_count"][a]
        assert (pools.neuron_owner[ns] == a).all() and (pools.synapse_owner[es] == a).all()
        ports = A["ports"][a]
        assert (ports >= 0).all()                       # 19 channels and 5 motors in every founder
        assert all(pools.neuron_port[ports[p]] == p for p in range(24))
    assert (A["alive"][10:] == 0).all() and (A["neuron_head"][10:] == -1).all()
    eco = W.make_ecology(pools, seed=3)
    for owner, words in ((pools.neuron_owner, eco.neuron_used), (pools.synapse_owner, eco.synapse_used)):
        used = np.unpackbits(words.view(np.uint8), bitorder="little")[:len(owner)].astype(bool)
        assert np.array_equal(used, owner >= 0)
    assert eco.next_id[0] == A["id"].max() + 1
    assert (eco.cell_head == -1).all() and eco.food.sum() > 0.2 * 16384
