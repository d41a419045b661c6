"""Correctly rounded exp, log, sin, cos and hypot: the product implementation
(csrc/ns_crmath.h, built into oracle/_build/exhaustive_math) against the
oracle's independent long-double/binary128 implementation, over a strided
sample of all binary32 inputs (the full 2^32 sweep is
`oracle/_build/exhaustive_math exp 8 1`; hypot pairs each input with four
partners, Pythagorean ratios among them)."""
import json
import subprocess

import numpy as np
import pytest

from oracle.pyoracle import oracle_lib


@pytest.mark.parametrize("fn", ["exp", "log", "sin", "cos", "hypot"])
def test_sampled_sweep_matches_independent_cr(oracle_built, fn):
    from oracle.build import BUILD
    out = subprocess.run([str(BUILD / "exhaustive_math"), fn, "4", "1009"], capture_output=True, text=True)
    res = json.loads(out.stdout)
    assert res["checked"] > 2_000_000
    assert res["mismatches"] == 0, res


# Arguments the reference passes to expf/logf as compile-time constants
# (src/physiology.cuh:228,266,271,309-310,371-372,514-515,537-538;
# src/prinz_cell.cuh:75) and the gene-constant ones every ABI genome uses
# (receptor decay 3 ms, L5 afterdepolarisation 45 ms).
CONST_EXP_ARGS = [-1.0 / 3.0, -0.1, -1.0 / 40.0, -1.0 / 750.0, -0.25 / 3.0, -0.25 / 10.0,
                  -0.25 / 45.0, 10.0, -1.0 / 7200.0, -1.0 / 3600.0, -1.0 / 17.0, -1.0 / 34.0,
                  -0.025 / 200.0]


def test_constant_arguments_agree_with_glibc(oracle_built):
    """If glibc rounds these constant-argument exponentials correctly, the
    reference's results do not depend on whether the compiler folds them."""
    lib = oracle_lib()
    import ctypes
    libm = ctypes.CDLL("libm.so.6")
    libm.expf.argtypes = [ctypes.c_float]; libm.expf.restype = ctypes.c_float
    libm.logf.argtypes = [ctypes.c_float]; libm.logf.restype = ctypes.c_float
    for a in CONST_EXP_ARGS:
        x = float(np.float32(a))
        assert np.float32(libm.expf(x)).tobytes() == np.float32(lib.or_cr_expf(x)).tobytes(), a
    for a in (1.92, 0.70):
        x = float(np.float32(a))
        assert np.float32(libm.logf(x)).tobytes() == np.float32(lib.or_cr_logf(x)).tobytes(), a


def test_cr_exp_special_values(oracle_built):
    lib = oracle_lib()
    assert lib.or_cr_expf(0.0) == 1.0
    assert lib.or_cr_expf(-200.0) == 0.0
    assert np.isinf(lib.or_cr_expf(100.0))
    assert np.isnan(lib.or_cr_expf(float("nan")))


def test_trig_special_values(oracle_built):
    lib = oracle_lib()
    import ctypes
    for name in ("or_cr_sinf", "or_cr_cosf"):
        getattr(lib, name).argtypes = [ctypes.c_float]
        getattr(lib, name).restype = ctypes.c_float
    lib.or_cr_hypotf.argtypes = [ctypes.c_float, ctypes.c_float]
    lib.or_cr_hypotf.restype = ctypes.c_float
    assert np.float32(lib.or_cr_sinf(-0.0)).tobytes() == np.float32(-0.0).tobytes()
    assert lib.or_cr_cosf(0.0) == 1.0
    assert np.isnan(lib.or_cr_sinf(float("inf"))) and np.isnan(lib.or_cr_cosf(float("nan")))
    assert lib.or_cr_hypotf(3.0, 4.0) == 5.0
    assert np.isinf(lib.or_cr_hypotf(float("nan"), float("-inf")))
    assert np.isnan(lib.or_cr_hypotf(float("nan"), 1.0))
    # headings far from the origin (the reference's headings grow without bound)
    import mpmath
    mpmath.mp.prec = 200
    for x in (12007.25, -3.0e4, 1.0e30, 3.4e38, 7.853981e-1, 1.5707964):
        xf = float(np.float32(x))
        assert np.float32(lib.or_cr_sinf(xf)) == np.float32(float(mpmath.sin(xf))), x
        assert np.float32(lib.or_cr_cosf(xf)) == np.float32(float(mpmath.cos(xf))), x
