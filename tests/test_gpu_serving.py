"""GPU tests of the serving loop (nsb_serve_* through the C ABI).

An episode's result (steps, reward, falls, per-step action/motor-count trace,
status) must be bit-identical to the CPU oracle's episode (oracle/or_episode.c
driving the oracle brain), and identical whether the episode runs alone or
admitted into a mix of other episodes of different sizes and lengths
(packed into shared work units, admitted mid-flight).
"""
import time

import numpy as np
import pytest

from oracle.pyoracle import OracleBrain

pytestmark = pytest.mark.gpu

FIELDS = ("steps", "reward", "failures", "trace", "status")


def _library(nsb):
    # sizes across the range, including brains above the 768-neuron unit
    return nsb.workloads.serving_library(seed=5, genomes=40)


def _result_dict(r):
    return {k: int(r[k]) for k in FIELDS}


def _server(nsb, **kw):
    kw.setdefault("max_inflight_neurons", 262144)
    kw.setdefault("max_slots", 4096)
    return nsb.Server(**kw)


def test_served_episodes_match_oracle(nsb, oracle_built):
    lib = _library(nsb)
    sizes = np.diff(lib.neuron_offsets)
    pick = [int(i) for i in np.argsort(sizes)[::4]]          # 10 genomes, smallest to largest
    srv = _server(nsb)
    ids = srv.register_batch(lib)
    seeds = np.arange(len(pick), dtype=np.uint32) * 101 + 7
    steps = 30 + (np.arange(len(pick)) * 7) % 25
    srv.submit([ids[g] for g in pick], seeds, steps, tag=np.arange(len(pick)), arrival=0.0)
    srv.run()
    res = srv.poll_all()
    srv.close()
    assert len(res) == len(pick)
    by_tag = {int(r["tag"]): r for r in res}
    for k, g in enumerate(pick):
        ng, sg, mo = lib.brain(g)
        o = OracleBrain(ng, sg, mo, lib.channels, lib.max_delay)
        want = o.episode(int(seeds[k]), int(steps[k]))
        got = _result_dict(by_tag[k])
        assert got == want, f"genome {g} ({sizes[g]} neurons): {got} != {want}"


def test_episode_alone_equals_in_mix(nsb, oracle_built):
    lib = _library(nsb)
    sizes = np.diff(lib.neuron_offsets)
    x_genome = int(np.argsort(sizes)[len(sizes) // 2])
    x_seed, x_steps = 424242, 60
    # alone
    srv = _server(nsb)
    ids = srv.register_batch(lib)
    srv.submit([ids[x_genome]], x_seed, x_steps, tag=0, arrival=0.0)
    srv.run()
    alone = srv.poll_all()
    srv.close()
    assert len(alone) == 1
    # in one admission round with 150 others (packed into shared units)
    rng = np.random.default_rng(9)
    others = rng.integers(0, len(sizes), 150)
    srv = _server(nsb)
    ids = srv.register_batch(lib)
    srv.submit([ids[g] for g in others], rng.integers(1, 2**31, 150).astype(np.uint32),
               rng.integers(20, 120, 150).astype(np.int32), tag=np.arange(1, 151), arrival=0.0)
    srv.submit([ids[x_genome]], x_seed, x_steps, tag=0, arrival=0.0)
    srv.run()
    packed = srv.poll_all()
    srv.close()
    assert len(packed) == 151
    # admitted mid-flight by the background loop
    srv = _server(nsb)
    ids = srv.register_batch(lib)
    srv.submit([ids[g] for g in others], rng.integers(1, 2**31, 150).astype(np.uint32),
               rng.integers(20, 120, 150).astype(np.int32), tag=np.arange(1, 151), arrival=0.0)
    srv.start()
    time.sleep(0.05)
    srv.submit([ids[x_genome]], x_seed, x_steps, tag=0)
    got = []
    deadline = time.time() + 120
    while sum(len(g) for g in got) < 151 and time.time() < deadline:
        got.append(srv.poll())
        time.sleep(0.01)
    srv.stop()
    st = srv.stats()
    srv.close()
    mixed = np.concatenate(got)
    assert len(mixed) == 151 and st["inflight"] == 0
    ref = _result_dict(alone[0])
    for res, label in ((packed, "packed"), (mixed, "mid-flight")):
        x = res[res["tag"] == 0][0]
        assert _result_dict(x) == ref, f"{label}: {_result_dict(x)} != {ref}"
        assert x["admit_s"] >= x["arrival_s"] and x["done_s"] >= x["admit_s"]


def test_admission_respects_inflight_cap(nsb, oracle_built):
    lib = _library(nsb)
    sizes = np.diff(lib.neuron_offsets)
    small = [int(i) for i in np.argsort(sizes)[:20]]
    biggest = int(sizes[small].max())
    cap = max(int(sizes[small].sum() // 3), biggest)
    srv = _server(nsb, max_inflight_neurons=cap, max_slots=64, max_brain_neurons=biggest)
    ids = [srv.register(*lib.brain(g)) for g in small]
    srv.submit(ids * 3, np.arange(60, dtype=np.uint32), 25, tag=np.arange(60), arrival=0.0)
    srv.start()
    seen = 0
    peak = 0
    deadline = time.time() + 120
    while seen < 60 and time.time() < deadline:
        st = srv.stats()
        peak = max(peak, st["inflight_neurons"])
        seen += len(srv.poll())
        time.sleep(0.002)
    srv.stop()
    srv.close()
    assert seen == 60
    assert 0 < peak <= cap


def test_serving_rejects_bad_input(nsb):
    srv = _server(nsb)
    lib = _library(nsb)
    ng, sg, mo = lib.brain(0)
    bad = ng.copy()
    bad[0, 1] = 8          # channel outside the 8 observation channels
    with pytest.raises(RuntimeError, match="Invalid neuron gene"):
        srv.register(bad, sg, mo)
    lp = ng.copy()
    lp[-1, 0] = 2
    with pytest.raises(RuntimeError, match="AdEx-family"):
        srv.register(lp, sg, mo)
    g = srv.register(ng, sg, mo)
    with pytest.raises(RuntimeError, match="Unknown genome id"):
        srv.submit([g + 5], 1, 10)
    with pytest.raises(RuntimeError, match="Invalid episode length"):
        srv.submit([g], 1, 0)
    srv.close()


def test_request_that_can_never_fit_is_reported(nsb):
    """A request larger than the server's synapse pool can never be admitted:
    with nothing in flight the loop reports it instead of waiting forever."""
    lib = _library(nsb)
    sizes = np.diff(lib.neuron_offsets)
    g = int(np.argmax(sizes))                      # ~4,000 neurons, ~32,000 synapses
    srv = nsb.Server(max_inflight_neurons=int(sizes[g]), synapses_per_neuron=1.0, max_slots=16,
                     max_brain_neurons=int(sizes[g]))
    gid = srv.register(*lib.brain(g))
    srv.submit([gid], 1, 10, tag=0, arrival=0.0)
    with pytest.raises(RuntimeError, match="does not fit"):
        srv.run()
    srv.close()
