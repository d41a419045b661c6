"""Pins the C oracle to the reference.

1. Bit-exact: the oracle built against glibc reproduces the reference host
   executor (gym_adapter/native.cpp compiled from the reference sources into
   oracle/_ref) in every state word, spike raster and output; the oracle with
   correctly rounded exp/log reproduces the same reference sources compiled
   with exp/log correctly rounded. Skipped where oracle/_ref is absent; the
   committed golden fixtures (test_golden.py) carry the pin to such machines.
2. Windows: the reference's own protocol checks (tests/physiology.cpp,
   tests/event_synapses.cpp, tests/cuda_relay_parity.cu) on the oracle.
"""
import numpy as np
import pytest

from oracle.pyoracle import OracleBrain, RefBrain, ref_lib, protocols


def _compare(batch, brains, calls, ticks, libm, seeds_base=100, delay=8):
    for i in brains:
        ng, sg, mo = batch.brain(i)
        o = OracleBrain(ng, sg, mo, batch.channels, delay, libm=libm)
        r = RefBrain(ng, sg, mo, batch.channels, cr=not libm)
        o.reset(seeds_base + i); r.reset(seeds_base + i)
        for c in range(calls):
            x = batch.inputs[i]
            a = o.step(x, ticks, batch.gain, raster=True)
            b = r.step(x, ticks, batch.gain, raster=True)
            assert a[0] == b[0]
            np.testing.assert_array_equal(a[1], b[1])
            np.testing.assert_array_equal(a[2], b[2])
            da, db = o.dump(), r.dump()
            np.testing.assert_array_equal(da[0], db[0], err_msg=f"brain {i} call {c} neurons")
            np.testing.assert_array_equal(da[1], db[1], err_msg=f"brain {i} call {c} synapses")
            assert da[2] == db[2]


needs_ref = pytest.mark.skipif(ref_lib() is None and ref_lib(cr=True) is None,
                               reason="reference build (oracle/_ref) absent")


@needs_ref
@pytest.mark.parametrize("libm", [True, False])
def test_oracle_bitexact_vs_reference_parity_mix(oracle_built, nsb, libm):
    batch = nsb.workloads.parity_mix(brains=10)
    _compare(batch, range(batch.brains), calls=12, ticks=16, libm=libm)


@needs_ref
@pytest.mark.parametrize("libm", [True, False])
def test_oracle_bitexact_vs_reference_plain_small(oracle_built, nsb, libm):
    batch = nsb.workloads.plain_small(brains=4)
    _compare(batch, range(4), calls=125, ticks=16, libm=libm)   # 2,000 ticks


@needs_ref
def test_oracle_bitexact_reset_with_original_indices(oracle_built, nsb):
    batch = nsb.workloads.parity_mix(brains=3, heavy_types=False)
    for i in range(3):
        ng, sg, mo = batch.brain(i)
        o = OracleBrain(ng, sg, mo, batch.channels, 8, libm=True)
        r = RefBrain(ng, sg, mo, batch.channels)
        on = np.arange(len(ng), dtype=np.uint32) * 3 + 5
        os_ = np.arange(len(sg), dtype=np.uint32) * 7 + 1
        o.original_indices(on, os_); r.original_indices(on, os_)
        o.reset(2 ** 31 + 47); r.reset(2 ** 31 + 47)
        for _ in range(5):
            a = o.step(batch.inputs[i], 7, 150.0, raster=True)
            b = r.step(batch.inputs[i], 7, 150.0, raster=True)
            np.testing.assert_array_equal(a[2], b[2])
        np.testing.assert_array_equal(o.dump()[0], r.dump()[0])
        np.testing.assert_array_equal(o.dump()[1], r.dump()[1])


def test_oracle_rejects_what_the_abi_rejects(oracle_built):
    good_n = np.array([[0, -1, 1, 0, 0, 1, 1, -52, 0, 0]] * 3, np.float32)
    good_s = np.array([[0, 1, 2.0, 1, 3, 0, .5, 100, 0, 1, 0]], np.float32)
    OracleBrain(good_n, good_s, [2], 4)
    bad_n = good_n.copy(); bad_n[0, 0] = 7
    with pytest.raises(ValueError, match="Invalid neuron gene"):
        OracleBrain(bad_n, good_s, [2], 4)
    bad_m = good_n.copy(); bad_m[0, 7] = -10
    with pytest.raises(ValueError, match="Invalid membrane parameters"):
        OracleBrain(bad_m, good_s, [2], 4)
    bad_s = good_s.copy(); bad_s[0, 4] = 9
    with pytest.raises(ValueError, match="Invalid synapse gene"):
        OracleBrain(good_n, bad_s, [2], 4)
    OracleBrain(good_n, bad_s, [2], 4, max_delay=16)          # extended ring accepts it
    with pytest.raises(ValueError, match="Invalid motor index"):
        OracleBrain(good_n, good_s, [3], 4)
    with pytest.raises(ValueError, match="Invalid brain dimensions"):
        OracleBrain(good_n, good_s, [2], 0)


def test_reference_protocol_windows(oracle_built):
    r = protocols()
    # tests/physiology.cpp:124-145 step currents
    assert r[0] > 4 and r[3] > 4 and r[6] == 0
    assert r[2] > r[1]                       # RS adapts
    assert abs(r[5] - r[4]) < 10             # cNA nearly non-adapting
    # 177-192 release means at U = 0.55
    assert abs(r[7] - 0.55) < 0.02 and 0.45 * r[7] < r[8] < 0.7 * r[7] and r[9] > 0.95 * r[7]
    # 226-239 STDP pairs
    assert 1.3 < r[10] < 1.6 and 0.75 < r[11] < 0.9
    assert abs(r[12] - 1) < 1e-5 and abs(r[13] - 1) < 1e-5 and abs(r[14] - 1) < 1e-5
    assert abs(r[15] - 1) < 1e-5 and r[16] > 1.2
    # 288-315 homeostasis
    assert abs(r[17] - 1.92) < 0.02 and abs(r[18] - 1) < 1e-5 and abs(r[19] - 0.70) < 0.02
    # event_synapses.cpp:9-11 quiet jumps within 2e-4
    assert r[20] <= 2e-4
    # cuda_relay_parity.cu / EXPERIMENTS.md:190: 15 arrivals, 5.91 nS released,
    # -64.23 mV peak, no postsynaptic spike
    assert r[21] == 15 and abs(r[22] - 5.91) < 0.01 and abs(r[23] - (-64.23)) < 0.01 and r[25] == 0
