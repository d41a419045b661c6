"""Generate tests/golden/reference_runs.npz from the reference host executor
(gym_adapter/native.cpp compiled from the reference sources into oracle/_ref,
both with glibc expf/logf and with correctly rounded exp/log).

For each workload and binding the fixture stores, per 16-tick call: the motor
outputs, the bit-packed spike raster and SHA-256 digests of the canonical
neuron and synapse state dumps. Run from the repository root:
    python tests/golden/make_golden.py
"""
import hashlib
import importlib.util
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import build, pyoracle  # noqa: E402


def load_workloads():
    spec = importlib.util.spec_from_file_location("nsb_workloads", ROOT / "neural-selection_b200" / "workloads.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["nsb_workloads"] = mod
    spec.loader.exec_module(mod)
    return mod


def digest(a):
    return np.frombuffer(hashlib.sha256(np.ascontiguousarray(a).tobytes()).digest(), np.uint8)


CASES = {"parity_mix": dict(fn="parity_mix", kw=dict(seed=11, brains=6), calls=10),
         "plain_small": dict(fn="plain_small", kw=dict(brains=2), calls=40)}


def run(W, binding):
    out = {}
    for name, c in CASES.items():
        batch = getattr(W, c["fn"])(**c["kw"])
        for i in range(batch.brains):
            ng, sg, mo = batch.brain(i)
            r = pyoracle.RefBrain(ng, sg, mo, batch.channels, cr=(binding == "cr"))
            r.reset(1000 + i)
            outs, rasters, nd, sd = [], [], [], []
            for _ in range(c["calls"]):
                rc, o, ras = r.step(batch.inputs[i], 16, batch.gain, raster=True)
                assert rc == 0
                nw, sw, _ = r.dump()
                outs.append(o); rasters.append(np.packbits(ras)); nd.append(digest(nw)); sd.append(digest(sw))
            key = f"{binding}/{name}/{i}"
            out[key + "/outputs"] = np.stack(outs)
            out[key + "/raster"] = np.stack(rasters)
            out[key + "/neuron_sha"] = np.stack(nd)
            out[key + "/synapse_sha"] = np.stack(sd)
            r.close()
    return out


if __name__ == "__main__":
    build.build_oracle()
    if build.build_ref(gpu=False) is None:
        sys.exit("reference tree absent")
    W = load_workloads()
    data = {}
    for binding in ("libm", "cr"):
        data.update(run(W, binding))
    np.savez_compressed(Path(__file__).with_name("reference_runs.npz"), **data)
    print("wrote", len(data), "arrays")
