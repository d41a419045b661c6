"""Committed golden runs of the reference host executor
(tests/golden/reference_runs.npz, made by tests/golden/make_golden.py from the
reference sources): per 16-tick call, motor outputs, spike raster and digests
of the full canonical state. The oracle must reproduce the glibc runs and the
correctly rounded runs (CPU); the CUDA engine must reproduce the correctly
rounded runs (GPU). No reference tree is needed at test time."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import OracleBrain

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_runs.npz"
CASES = {"parity_mix": dict(fn="parity_mix", kw=dict(seed=11, brains=6), calls=10),
         "plain_small": dict(fn="plain_small", kw=dict(brains=2), calls=40)}


def digest(a):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


@pytest.mark.parametrize("binding", ["libm", "cr"])
@pytest.mark.parametrize("case", list(CASES))
def test_oracle_reproduces_reference_golden(oracle_built, nsb, golden, binding, case):
    c = CASES[case]
    batch = getattr(nsb.workloads, c["fn"])(**c["kw"])
    for i in range(batch.brains):
        key = f"{binding}/{case}/{i}"
        ng, sg, mo = batch.brain(i)
        o = OracleBrain(ng, sg, mo, batch.channels, 8, libm=(binding == "libm"))
        o.reset(1000 + i)
        for call in range(c["calls"]):
            rc, out, ras = o.step(batch.inputs[i], 16, batch.gain, raster=True)
            assert rc == 0
            np.testing.assert_array_equal(out, golden[key + "/outputs"][call])
            np.testing.assert_array_equal(np.packbits(ras), golden[key + "/raster"][call])
            nw, sw, _ = o.dump()
            assert (digest(nw) == golden[key + "/neuron_sha"][call]).all(), (key, call)
            assert (digest(sw) == golden[key + "/synapse_sha"][call]).all(), (key, call)


@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES))
def test_engine_reproduces_reference_golden_cr(nsb, golden, case):
    c = CASES[case]
    batch = getattr(nsb.workloads, c["fn"])(**c["kw"])
    gpu = nsb.GpuBatch.from_rows(batch)
    gpu.reset(np.arange(batch.brains, dtype=np.uint32) + 1000)
    for call in range(c["calls"]):
        out, status = gpu.step(batch.inputs, None, 16, batch.gain)
        assert not status.any()
        for i in range(batch.brains):
            key = f"cr/{case}/{i}"
            np.testing.assert_array_equal(out[i], golden[key + "/outputs"][call])
            nw, sw, _ = gpu.dump(i)
            assert (digest(nw) == golden[key + "/neuron_sha"][call]).all(), (key, call)
            assert (digest(sw) == golden[key + "/synapse_sha"][call]).all(), (key, call)
