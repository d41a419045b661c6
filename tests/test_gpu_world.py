"""GPU tests of the world neural stage (nsb_world_* through the C ABI).

The world stage steps the world simulator's own pools (reference record
layouts) in place. After several world steps with homeostasis in between,
every pool must be bit-identical to the oracle's world restatement
(or_world_step) run on a host copy. The population exercises every rule of the
world tick (src/main.cu:659-801):
- dead and dying animals (untouched);
- frozen plasticity cohorts, and a stale cohort record that does not freeze;
- the traced animal's counters;
- silenced contact channels;
- a type-5 cell on a non-receptor channel;
- two neurons on one motor port;
- inactive neurons and synapses, and a synapse whose source belongs to another animal;
- input left pending from before the step;
- spike history and modulatory timestamps from earlier ticks;
- scattered, interleaved pool slots and list orders;
- animals large enough for the one-animal-per-CTA path (by neurons and by synapses),
  and animals exactly at the small path's capacity.

A population that changes between steps (deaths, births, slots taken over
by new animals) checks the compiled-brain cache, its arena reset included.

test_world_stage_matches_reference_kernels pins the stage to the reference
simulator's own world kernels
(src/main.cu built from its sources with IEEE arithmetic and correctly rounded
exp/log, oracle/ref_world_harness.cu) on a population whose float sums are
order-independent: at most two live synapses per (post-synaptic neuron,
branch) for excitation and per neuron for inhibition, so the reference's float
atomics are deterministic.
"""
import ctypes as ct

import numpy as np
import pytest

from oracle.pyoracle import HERE, oracle_records, world_homeostasis, world_step

pytestmark = pytest.mark.gpu

POOLS = ("neurons", "synapses", "neuron_state", "synapse_state", "pending_exc", "pending_inh", "mod_event_tick",
         "spike_history", "motors", "trace_exc_arrivals", "trace_exc_releases", "trace_inh_arrivals", "trace_exc_ns",
         "trace_inh_ns", "trace_peak_mv", "animals")


def _bits(a):
    a = np.ascontiguousarray(a)
    if a.dtype.names:
        return {n: _bits(a[n]) for n in a.dtype.names}
    if a.dtype.kind == "f":
        return a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)
    return a


def _compare(got, want, label=""):
    for name in POOLS:
        x, y = getattr(got, name), getattr(want, name)
        if x.dtype.names:
            for f in x.dtype.names:
                bx, by = _bits(x[f]), _bits(y[f])
                if not np.array_equal(bx, by):
                    bad = np.nonzero(~np.all((bx == by).reshape(len(bx), -1), axis=1))[0]
                    raise AssertionError(f"{label}{name}.{f} differs at slots {bad[:8]} ({len(bad)} slots)")
        else:
            if not np.array_equal(_bits(x), _bits(y)):
                raise AssertionError(f"{label}{name} differs")


def _population(nsb, seed=6):
    W, wl = nsb.world, nsb.workloads
    batch = wl.concat([wl.world_founders(seed=seed, founders=40, heavy_types=True),
                       wl.world_founders(seed=seed + 1, founders=3, lo=300, hi=700),
                       wl.world_founders(seed=seed + 2, founders=2, lo=190, hi=220, epn_lo=11, epn_hi=12),
                       # exactly the small path's capacity: 256 neurons, 8 synapses each (2,048)
                       wl.world_founders(seed=seed + 3, founders=2, lo=256, hi=256, epn_lo=8, epn_hi=8)],
                      "world_mix")
    B = batch.brains
    N, E = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1])
    seeds = np.arange(B, dtype=np.uint32) * 7 + 3
    recs = W.records_from_gpu(batch, seeds)
    for got, want, dt in zip(recs, oracle_records(batch, seeds),
                             (W.NEURON_GENE, W.NEURON_STATE, W.SYNAPSE_GENE, W.SYNAPSE_STATE)):
        want = np.ascontiguousarray(want).view(dt).reshape(-1)
        for f in dt.names:                       # field by field: padding bytes are not state
            assert np.array_equal(_bits(got[f]), _bits(want[f])), f
    P = B + 7
    slots = np.random.default_rng(1).permutation(P)[:B]
    pools = W.place_population(batch, *recs, animal_capacity=P, neuron_capacity=N + 777, synapse_capacity=E + 999,
                               scatter_seed=11, animal_slots=slots, cohort=True)
    rng = np.random.default_rng(2)
    A, C = pools.animals, pools.plasticity_cohort
    A["alive"][slots[5]] = 0
    A["alive"][slots[9]] = -2
    for b in (1, 2, 3):
        C["assigned"][slots[b]] = 1
        C["frozen"][slots[b]] = 1
        C["id"][slots[b]] = A["id"][slots[b]]
    C["id"][slots[3]] += 1                       # record of an earlier occupant: not frozen
    pools.trace_animal = int(slots[4])
    pools.silence_contact = 1
    A["age"][slots] = rng.integers(1, 500, B)
    owned_n = np.nonzero(pools.neuron_owner >= 0)[0]
    owned_e = np.nonzero(pools.synapse_owner >= 0)[0]
    pools.neurons["active"][rng.choice(owned_n, len(owned_n) // 25, replace=False)] = 0
    pools.synapses["active"][rng.choice(owned_e, len(owned_e) // 20, replace=False)] = 0
    # a second neuron on motor port 21 (traced animal and another)
    for b in (4, 6):
        a = slots[b]
        mine = owned_n[pools.neuron_owner[owned_n] == a]
        hidden = mine[pools.neuron_port[mine] < 0]
        pools.neuron_port[hidden[0]] = 21
    # a type-5 cell on channel 7: channel level x 230 pA, no receptor events
    mine = owned_n[pools.neuron_owner[owned_n] == slots[0]]
    ch7 = mine[pools.neuron_port[mine] == 7][0]
    pools.neurons["type"][ch7] = 5
    pools.neurons["rec_event"][ch7] = 2.0
    pools.neurons["rec_gain"][ch7] = 40.0
    # a synapse of animal 0 whose source neuron belongs to animal 7
    e0 = owned_e[pools.synapse_owner[owned_e] == slots[0]][0]
    pools.synapses["pre"][e0] = owned_n[pools.neuron_owner[owned_n] == slots[7]][0]
    # leftovers from before the step, history and modulatory timestamps
    pick = rng.choice(owned_n, 12, replace=False)
    pools.pending_exc[pick] = rng.uniform(0, 2, (12, 4)).astype(np.float32)
    pools.pending_inh[pick] = rng.uniform(0, 1, 12).astype(np.float32)
    pools.spike_history[:, owned_n] = (rng.random((9, len(owned_n))) < 0.08).astype(np.uint8)
    pools.mod_event_tick[owned_n] = rng.integers(0, 64, (len(owned_n), 6)).astype(np.uint64)
    return pools, slots


def _run_both(nsb, pools, first_step, steps):
    world = nsb.world.World(pools)
    ref = pools.copy()
    for step in range(first_step, first_step + steps):
        world.neural_step(step)
        world_step(ref, step)
        ref.animals["age"][ref.animals["alive"] == 1] += 1
        world.upload("animals", ref.animals.copy())
        world.homeostasis()
        world_homeostasis(ref)
    got = world.download()
    st = world.stats()
    world.close()
    return got, ref, st


@pytest.mark.parametrize("warp_cells", [None, "0"])
def test_world_stage_matches_oracle(nsb, oracle_built, monkeypatch, warp_cells):
    """The world stage on a mixed population against the oracle; LP and Prinz
    cells on the whole warp (the default) and each on its own lane (0)."""
    if warp_cells is not None:
        monkeypatch.setenv("NSB_WORLD_WARP_CELLS", warp_cells)
    pools, slots = _population(nsb)
    before = pools.copy()
    got, ref, st = _run_both(nsb, pools, 5, 6)
    _compare(got, ref)
    alive = int((pools.animals["alive"] == 1).sum())
    assert st["animals"] == alive and st["events"] > 0
    # the stage did something, the dead animals kept their state
    assert not np.array_equal(_bits(got.neuron_state["v"]), _bits(before.neuron_state["v"]))
    dead = np.isin(pools.neuron_owner, [slots[5], slots[9]])
    assert np.array_equal(_bits(got.neuron_state["v"][dead]), _bits(before.neuron_state["v"][dead]))
    assert got.motors.sum() > 0 and got.trace_exc_arrivals.sum() > 0


@pytest.mark.parametrize("warp_cells", [None, "0"])
def test_world_stage_big_animals_with_lp_and_prinz_cells(nsb, oracle_built, monkeypatch, warp_cells):
    """Animals above the small units' 256 neurons with LP, Prinz and LFS cells
    (the big-animal kernel's heavy build, whose CTA pools the cells of each
    256-neuron slot) beside small heavy founders, against the oracle: whole
    warps (the default) and each cell on its own lane (0)."""
    if warp_cells is not None:
        monkeypatch.setenv("NSB_WORLD_WARP_CELLS", warp_cells)
    W, wl = nsb.world, nsb.workloads
    batch = wl.concat([wl.world_founders(seed=21, founders=3, lo=300, hi=700, heavy_types=True),
                       wl.world_founders(seed=22, founders=5, heavy_types=True)], "world_big_heavy")
    t = batch.neuron_rows[:, 0].astype(int)
    assert ((t == 2) | (t == 3)).sum() > 20 and np.diff(batch.neuron_offsets).max() > 256
    seeds = np.arange(batch.brains, dtype=np.uint32) * 5 + 1
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds), scatter_seed=7)
    got, ref, st = _run_both(nsb, pools, 3, 4)
    _compare(got, ref)
    assert st["animals"] == batch.brains
    assert got.motors.sum() > 0 or got.neuron_state["total"].sum() > 0


def test_world_stage_steady_population(nsb, oracle_built):
    """Config-2 founders (32-96 neurons, 4-12 synapses per neuron), packed
    slots: the compiled brains are reused across steps."""
    W = nsb.world
    batch = nsb.workloads.world_founders(seed=2, founders=300)
    seeds = np.arange(batch.brains, dtype=np.uint32) + 1
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds))
    got, ref, st = _run_both(nsb, pools, 1, 8)
    _compare(got, ref)
    assert st["animals"] == 300 and st["neurons"] == int(batch.neuron_offsets[-1])


def test_world_stage_reports_bad_pools(nsb):
    W = nsb.world
    batch = nsb.workloads.world_founders(seed=8, founders=4)
    pools = W.place_population(batch, *W.records_from_gpu(batch, np.arange(4, dtype=np.uint32)))
    bad = pools.copy()
    bad.animals["neuron_count"][2] += 1
    w = W.World(bad)
    with pytest.raises(RuntimeError, match="lists disagree"):
        w.neural_step(1)
    w.close()
    w = W.World(pools.copy(), max_brain_neurons=30)
    with pytest.raises(RuntimeError, match="larger than"):
        w.neural_step(1)
    w.close()
    bad = pools.copy()
    bad.synapses["branch"][bad.synapse_owner >= 0] = 4
    w = W.World(bad)
    with pytest.raises(RuntimeError, match="Invalid synapse gene"):
        w.neural_step(1)
    w.close()


def _limit_fanin(pools):
    """Deactivate synapses so that no (post-synaptic neuron, branch) receives
    more than two live excitatory synapses and no neuron more than two live
    inhibitory ones."""
    g = pools.synapses
    e = np.nonzero(pools.synapse_owner >= 0)[0]
    pre, post = g["pre"][e], g["post"][e]
    mod = pools.neurons["modulator"][pre] > 0
    inh = (pools.neurons["inh_tx"][pre] > 0) & ~mod
    key = np.where(inh, 4 * post.astype(np.int64) + (1 << 40), 4 * post.astype(np.int64) + g["branch"][e])
    key = np.where(mod, -1 - np.arange(len(e)), key)
    order = np.argsort(key, kind="stable")
    ks = key[order]
    first = np.r_[0, np.nonzero(np.diff(ks))[0] + 1]
    rank = np.arange(len(ks)) - np.repeat(first, np.diff(np.r_[first, len(ks)]))
    g["active"][e[order[rank >= 2]]] = 0


def _ref_world_cr():
    path = HERE / "_ref" / "libns_ref_world_cr.so"
    if not path.exists():
        return None
    lib = ct.CDLL(str(path))
    lib.ref_world_pools_create.restype = ct.c_void_p
    lib.ref_world_pools_create.argtypes = [ct.c_void_p, ct.c_int]
    lib.ref_world_pools_step.argtypes = [ct.c_void_p, ct.c_longlong]
    lib.ref_world_pools_step.restype = ct.c_int
    lib.ref_world_pools_homeostasis.argtypes = [ct.c_void_p]
    lib.ref_world_pools_homeostasis.restype = ct.c_int
    lib.ref_world_pools_destroy.argtypes = [ct.c_void_p]
    return lib


@pytest.mark.parametrize("block_mode", [0, 1])
def test_world_stage_matches_reference_kernels(nsb, block_mode):
    ref = _ref_world_cr()
    if ref is None:
        pytest.skip("oracle/_ref/libns_ref_world_cr.so not built")
    import torch
    W = nsb.world
    batch = nsb.workloads.world_founders(seed=12, founders=96, heavy_types=True)
    seeds = np.arange(batch.brains, dtype=np.uint32) * 3 + 1
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds), animal_capacity=32768,
                               neuron_capacity=4194304, synapse_capacity=8388608, scatter_seed=5, cohort=True)
    _limit_fanin(pools)
    A, C = pools.animals, pools.plasticity_cohort
    C["assigned"][3] = C["frozen"][3] = 1
    C["id"][3] = A["id"][3]
    A["alive"][7] = 0
    A["age"][:batch.brains] = np.arange(batch.brains) % 40 + 1
    pools.silence_contact = 1
    world = W.World(pools)
    dev = {n: (None if t is None else t.clone()) for n, t in world.dev.items()}
    st = W.NsbWorldPools()
    for n, t in dev.items():
        setattr(st, n, None if t is None else t.data_ptr())
    st.trace_animal, st.silence_senses, st.silence_contact = -1, 0, 1
    st.animal_capacity, st.neuron_capacity, st.synapse_capacity = pools.capacities
    h = ref.ref_world_pools_create(ct.byref(st), block_mode)
    assert h, "reference pools setup failed"
    try:
        for step in range(1, 9):
            world.neural_step(step)
            assert ref.ref_world_pools_step(h, step) == 0
            ages = world.dev["animals"].view(torch.int32).view(-1, 118)
            ages[:, 19] += (ages[:, 20] == 1).to(torch.int32)
            rages = dev["animals"].view(torch.int32).view(-1, 118)
            rages[:, 19] += (rages[:, 20] == 1).to(torch.int32)
            world.homeostasis()
            assert ref.ref_world_pools_homeostasis(h) == 0
        got = world.download()
        want = pools.copy()
        for n in W.ARRAYS:
            t = dev[n]
            if t is not None:
                getattr(want, n).view(np.uint8).reshape(-1)[:] = t.cpu().numpy()
    finally:
        ref.ref_world_pools_destroy(h)
        world.close()
    names = POOLS if block_mode == 0 else tuple(p for p in POOLS if p != "mod_event_tick")
    for name in names:
        x, y = getattr(got, name), getattr(want, name)
        if x.dtype.names:
            for f in x.dtype.names:
                assert np.array_equal(_bits(x[f]), _bits(y[f])), f"{name}.{f} differs from the reference kernels"
        else:
            assert np.array_equal(_bits(x), _bits(y)), f"{name} differs from the reference kernels"
    assert got.motors.sum() > 0


def test_world_stage_open_loop_2000_ticks(nsb, oracle_built):
    """Config 2's gate: 125 world steps (2,000 ticks) of founders with new
    world senses every step (open loop: the same senses fed to both sides),
    motor counts compared every step and every pool at the end."""
    W = nsb.world
    batch = nsb.workloads.world_founders(seed=2, founders=128)
    seeds = np.arange(batch.brains, dtype=np.uint32) + 1
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds), scatter_seed=3)
    world = W.World(pools)
    ref = pools.copy()
    rng = np.random.default_rng(4)
    for step in range(1, 126):
        senses = rng.random(ref.senses.shape).astype(np.float32)
        ref.senses[:] = senses
        world.upload("senses", senses.copy())
        ref.motors[:] = 0
        world.upload("motors", np.zeros_like(ref.motors))
        world.neural_step(step)
        world_step(ref, step)
        got_motors = world.dev["motors"].cpu().numpy().view(np.int32).reshape(ref.motors.shape)
        assert np.array_equal(got_motors, ref.motors), f"motor counts differ at step {step}"
        ref.animals["age"][ref.animals["alive"] == 1] += 1
        world.upload("animals", ref.animals.copy())
        world.homeostasis()
        world_homeostasis(ref)
    got = world.download()
    world.close()
    _compare(got, ref)
    assert got.neuron_state["total"].sum() > 0



def _genome_slots(pools, a):
    """Pool slots of animal slot a's neuron and synapse lists, in list order."""
    A = pools.animals[a]
    n, q = [], int(A["neuron_head"])
    while q >= 0:
        n.append(q)
        q = int(pools.neuron_next[q])
    e, q = [], int(A["synapse_head"])
    while q >= 0:
        e.append(q)
        q = int(pools.synapse_next[q])
    return np.array(n), np.array(e)


def _occupy(pools, a, genome, record, new_id):
    """Animal slot a takes over a brain (its pool lists and state) as a new
    animal: new id, age 1, owners rewritten, as a birth into a reused slot
    does in the simulator (src/main.cu:1662-1732, which fills the lists from
    freed pool slots)."""
    nslots, eslots = genome
    A = pools.animals
    for f in ("neuron_head", "synapse_head", "neuron_count", "synapse_count", "ports"):
        A[f][a] = record[f]
    A["alive"][a] = 1
    A["id"][a] = new_id
    A["age"][a] = 1
    pools.neuron_owner[nslots] = a
    pools.synapse_owner[eslots] = a


def test_world_stage_births_deaths_and_slot_reuse(nsb, oracle_built):
    """Animals die and are born between steps, with every path of the
    compiled-brain cache taken: a birth into a never-used animal slot, a
    smaller brain taking over a dead animal's slot (its region rewritten in
    place), a larger one (a new region), a brain moving through several slots
    until the arena passes half full and the cache is reset, and the steps
    after the reset that compile every living animal again. Every pool must
    equal the oracle's after each phase."""
    W, wl = nsb.world, nsb.workloads
    batch = wl.concat([wl.world_founders(seed=9, founders=24),
                       wl.world_founders(seed=10, founders=1, lo=230, hi=250, epn_lo=7, epn_hi=8),
                       wl.world_founders(seed=11, founders=1, lo=20, hi=24)], "births")
    seeds = np.arange(batch.brains, dtype=np.uint32) + 5
    N, E = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1])
    pools = W.place_population(batch, *W.records_from_gpu(batch, seeds), animal_capacity=32,
                               neuron_capacity=N, synapse_capacity=E, scatter_seed=8)
    big, small = 24, 25
    genomes = {g: _genome_slots(pools, g) for g in range(batch.brains)}
    records = {g: pools.animals[g].copy() for g in range(batch.brains)}
    pools.animals["alive"][[big, small]] = 0          # not born yet
    world = W.World(pools)
    ref = pools.copy()
    step = 0

    def run(k):
        nonlocal step
        for _ in range(k):
            step += 1
            world.neural_step(step)
            world_step(ref, step)
            ref.animals["age"][ref.animals["alive"] == 1] += 1
            world.upload("animals", ref.animals.copy())
            world.homeostasis()
            world_homeostasis(ref)
        _compare(world.download(), ref, f"after step {step}: ")
        assert world.stats()["animals"] == int((ref.animals["alive"] == 1).sum())

    def publish():
        for name in ("animals", "neuron_owner", "synapse_owner", "senses"):
            world.upload(name, getattr(ref, name).copy())

    run(2)
    ref.animals["alive"][5] = 0                                   # a death
    _occupy(ref, big, genomes[big], records[big], 5001)           # a birth into an unused slot
    ref.senses[big] = batch.inputs[big]
    publish()
    run(2)
    _occupy(ref, 5, genomes[small], records[small], 5002)         # smaller brain in a dead animal's slot
    ref.senses[5] = batch.inputs[small]
    ref.animals["alive"][big] = 0
    _occupy(ref, 26, genomes[big], records[big], 5003)            # larger brain: a new region
    ref.senses[26] = batch.inputs[big]
    publish()
    run(2)
    next_id = 5004
    for a in (27, 28, 29, 30):                                    # the arena passes half full
        ref.animals["alive"][a - 1] = 0
        _occupy(ref, a, genomes[big], records[big], next_id)
        ref.senses[a] = batch.inputs[big]
        next_id += 1
        publish()
        run(1)
    run(2)                                                        # every living animal compiled again
    world.close()
    assert ref.motors.sum() > 0
