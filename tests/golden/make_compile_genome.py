"""Golden vectors of the genome compiler (tests/test_compile_genome.py).

Runs the reference's own compile_genome (gym_adapter/compile_graph.py of
mixic/neural-selection, read from REFERENCE_ROOT, default: a directory named
"reference" beside this repository) on seeded genomes and writes inputs and
outputs to compile_genome.npz. The reference module imports Genome from its
adapter, which needs gymnasium; a stub package supplies a Genome with the same
fields (neurons, synapses, motors, channels), which is all compile_genome uses.

    python tests/golden/make_compile_genome.py
"""
import importlib.util
import os
import sys
import types
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
REFERENCE = Path(os.environ.get("REFERENCE_ROOT", ROOT.parent / "reference"))


def reference_compiler():
    pkg = types.ModuleType("refgym")
    pkg.__path__ = []
    adapter = types.ModuleType("refgym.adapter")

    @dataclass
    class Genome:
        neurons: list
        synapses: list
        motors: list
        channels: int
    adapter.Genome = Genome
    sys.modules["refgym"] = pkg
    sys.modules["refgym.adapter"] = adapter
    spec = importlib.util.spec_from_file_location("refgym.compile_graph",
                                                  REFERENCE / "gym_adapter" / "compile_graph.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return Genome, mod.compile_genome


def cases():
    sys.path.insert(0, str(ROOT / "tests"))
    from conftest import load_package
    nsb = load_package()
    rng = np.random.default_rng(17)
    out = []
    mix = nsb.workloads.parity_mix(seed=23, brains=6)
    for b in range(mix.brains):
        ng, sg, mo = mix.brain(b)
        out.append((ng.copy(), sg.copy(), mo.copy(), mix.channels))
    # sparse genomes with dead subgraphs: few edges, some inactive genes
    for k in range(6):
        n = int(rng.integers(12, 60))
        e = int(rng.integers(0, 2 * n))
        ng = np.zeros((n, 10), np.float32)
        ng[:, 0] = rng.integers(0, 2, n)
        ng[:, 1] = np.where(np.arange(n) < 3, np.arange(n), -1)
        ng[:, 2] = (rng.random(n) > 0.1).astype(np.float32)
        ng[:, 5] = ng[:, 6] = 1.0
        ng[:, 7] = -50.0
        sg = np.zeros((e, 11), np.float32)
        sg[:, 0] = rng.integers(0, n, e)
        sg[:, 1] = rng.integers(0, n, e)
        sg[:, 2] = 5.0
        sg[:, 3] = (rng.random(e) > 0.15).astype(np.float32)
        sg[:, 4] = rng.integers(1, 9, e)
        sg[:, 5] = rng.integers(0, 4, e)
        sg[:, 6] = 0.5
        sg[:, 7] = 100.0
        mo = rng.integers(0, n, 2).astype(np.int32)
        if k == 0:
            mo[1] = mo[0]                      # the same neuron on two ports
        out.append((ng, sg, mo, 3))
    return out


def main():
    Genome, compile_genome = reference_compiler()
    arrays = {}
    for i, (ng, sg, mo, ch) in enumerate(cases()):
        g = Genome([list(map(float, r)) for r in ng], [list(map(float, r)) for r in sg], [int(m) for m in mo], ch)
        c = compile_genome(g)
        arrays[f"in_neurons_{i}"] = ng
        arrays[f"in_synapses_{i}"] = sg.reshape(-1, 11)
        arrays[f"in_motors_{i}"] = mo
        arrays[f"out_neurons_{i}"] = np.asarray(c.neurons, np.float32).reshape(-1, 10)
        arrays[f"out_synapses_{i}"] = np.asarray(c.synapses, np.float32).reshape(-1, 11)
        arrays[f"out_motors_{i}"] = np.asarray(c.motors, np.int32)
        arrays[f"orig_neurons_{i}"] = np.asarray(c._original_neurons, np.uint32)
        arrays[f"orig_synapses_{i}"] = np.asarray(c._original_synapses, np.uint32)
    arrays["cases"] = np.asarray(len(arrays) // 8)
    np.savez_compressed(HERE / "compile_genome.npz", **arrays)
    print("wrote", HERE / "compile_genome.npz", int(arrays["cases"]), "cases")


if __name__ == "__main__":
    main()
