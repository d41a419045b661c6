"""CPU checks of the serving loop's host-side pieces.

- The environment arithmetic of the library (csrc/ns_env.h, compiled here for
  the host) equals the oracle's restatement (oracle/or_episode.c) bit for bit,
  and its exp/tanh/sin/cos are accurate to a few binary64 ulps.
- The pool range allocator never overlaps ranges, refuses only when no free
  run is long enough, and coalesces back to one range.
- The oracle's episode runner is deterministic per seed.
- The request schedule has the configured rate and length distribution.
"""
import ctypes as ct
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import OracleBrain, oracle_lib

ROOT = Path(__file__).resolve().parents[1]
CSRC = ROOT / "neural-selection_b200" / "csrc"
CPP = Path(__file__).resolve().parent / "cpp"


def _compile(tmp_path, name):
    exe = tmp_path / name
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", str(CSRC), str(CPP / f"{name}.cpp"),
                    "-o", str(exe)], check=True)
    return exe


def _bits(x):
    return int(np.float64(x).view(np.uint64))


def test_env_functions_match_oracle_bitwise(tmp_path, oracle_built):
    exe = _compile(tmp_path, "env_check")
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(-1, 1, 300), rng.uniform(-30, 30, 300), rng.uniform(-0.3, 0.3, 300),
                         [0.0, 1e-9, -1e-9, 0.5, -0.5, 20.0, 25.0, -25.0, 3.14159, 1.5707963267948966]])
    out = subprocess.run([str(exe)], input="\n".join(repr(float(x)) for x in xs), capture_output=True, text=True,
                         check=True).stdout.split("\n")
    lib = oracle_lib()
    s, c = ct.c_double(), ct.c_double()
    for x, line in zip(xs, out):
        e, t, si, co = (int(v, 16) for v in line.split())
        lib.or_env_sincos(float(x), ct.byref(s), ct.byref(c))
        assert e == _bits(lib.or_env_exp(float(x))), x
        assert t == _bits(lib.or_env_tanh(float(x))), x
        assert si == _bits(s.value) and co == _bits(c.value), x
    seq = (ct.c_uint64 * 4)()
    lib.or_env_sequence(seq)
    fields = out[len(xs)].split()
    assert fields[0] == "episode"
    assert [int(v, 16) for v in fields[1:]] == list(seq)


def test_env_functions_accuracy(oracle_built):
    lib = oracle_lib()
    xs = np.linspace(-20, 20, 4001)
    e = np.array([lib.or_env_exp(float(x)) for x in xs])
    np.testing.assert_allclose(e, np.exp(xs), rtol=4e-16)
    t = np.array([lib.or_env_tanh(float(x)) for x in xs])
    np.testing.assert_allclose(t, np.tanh(xs), rtol=0, atol=5e-16)
    s, c = ct.c_double(), ct.c_double()
    ys = np.linspace(-10, 10, 2001)
    sc = []
    for y in ys:
        lib.or_env_sincos(float(y), ct.byref(s), ct.byref(c))
        sc.append((s.value, c.value))
    sc = np.array(sc)
    np.testing.assert_allclose(sc[:, 0], np.sin(ys), rtol=0, atol=2e-15)
    np.testing.assert_allclose(sc[:, 1], np.cos(ys), rtol=0, atol=2e-15)


@pytest.mark.parametrize("seed", [1, 7, 123])
def test_range_allocator(tmp_path, seed):
    exe = _compile(tmp_path, "alloc_check")
    r = subprocess.run([str(exe), str(seed)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout


def test_oracle_episode_deterministic(nsb, oracle_built):
    lib = nsb.workloads.serving_library(genomes=4)
    ng, sg, mo = lib.brain(1)
    a = OracleBrain(ng, sg, mo, lib.channels, lib.max_delay)
    r1 = a.episode(11, 40)
    r2 = a.episode(11, 40)
    assert r1 == r2
    assert r1["steps"] == 40 and r1["reward"] + r1["failures"] == 40 and r1["status"] == 0
    r3 = a.episode(12, 40)
    assert r3["trace"] != r1["trace"] or r3["reward"] != r1["reward"]


def test_serving_schedule(nsb):
    s = nsb.workloads.serving_schedule(1, 2000.0, 5.0, 512)
    n = len(s["arrival"])
    assert abs(n - 10000) < 400
    assert np.all(np.diff(s["arrival"]) >= 0) and s["arrival"][-1] < 5.0
    assert s["steps"].min() >= 200 and s["steps"].max() <= 2000
    assert abs(s["steps"].mean() - 1100) < 20
    lib = nsb.workloads.serving_library(genomes=512)
    sizes = np.diff(lib.neuron_offsets)
    assert sizes.min() >= 32 and sizes.max() <= 4096
    # log-uniform on [32, 4096]: mean (4096 - 32) / ln 128 = 838
    assert 700 < sizes.mean() < 980
    assert len(lib.synapse_rows) == 8 * sizes.sum()
