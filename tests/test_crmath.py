"""Correctly rounded exp/log: the product implementation (csrc/ns_crmath.h,
built into oracle/_build/exhaustive_math) against the oracle's independent
long-double/binary128 implementation, over a strided sample of all binary32
inputs (the full 2^32 sweep is `oracle/_build/exhaustive_math exp 8 1`)."""
import json
import subprocess

import numpy as np
import pytest

from oracle.pyoracle import oracle_lib


@pytest.mark.parametrize("fn", ["exp", "log"])
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
