"""The genome compiler (nsb_compile_genome) against the reference's own
compile_genome (gym_adapter/compile_graph.py:10-28; golden vectors made by
tests/golden/make_compile_genome.py), and the property it exists for: a
compiled genome, reset with its original indices, produces the same motor
outputs as the full genome, step after step (oracle on the CPU, the library's
single-brain path on the GPU)."""
from pathlib import Path

import numpy as np
import pytest

from oracle.pyoracle import OracleBrain

GOLDEN = Path(__file__).resolve().parent / "golden" / "compile_genome.npz"


def _golden():
    z = np.load(GOLDEN)
    for i in range(int(z["cases"])):
        yield {k: z[f"{k}_{i}"] for k in ("in_neurons", "in_synapses", "in_motors", "out_neurons", "out_synapses",
                                          "out_motors", "orig_neurons", "orig_synapses")}


def test_compiler_matches_reference_golden(nsb):
    n_cases = 0
    for c in _golden():
        ng, sg, mo, on, osn = nsb.native.compile_genome(c["in_neurons"], c["in_synapses"], c["in_motors"])
        assert np.array_equal(ng.view(np.uint32), c["out_neurons"].view(np.uint32))
        assert np.array_equal(sg.view(np.uint32), c["out_synapses"].view(np.uint32))
        assert np.array_equal(mo, c["out_motors"])
        assert np.array_equal(on, c["orig_neurons"]) and np.array_equal(osn, c["orig_synapses"])
        n_cases += 1
    assert n_cases == 12


def test_compiler_rejects_bad_genomes(nsb):
    ng = np.zeros((4, 10), np.float32)
    ng[:, 2] = 1
    sg = np.zeros((1, 11), np.float32)
    sg[0, :4] = [0, 9, 1, 1]
    with pytest.raises(ValueError, match="Invalid synapse gene"):
        nsb.native.compile_genome(ng, sg, [1])
    with pytest.raises(ValueError, match="Invalid motor neuron"):
        nsb.native.compile_genome(ng, np.zeros((0, 11), np.float32), [7])
    ng2, sg2, mo2, on, osn = nsb.native.compile_genome(ng, np.zeros((0, 11), np.float32), [2, 2])
    assert len(ng2) == 1 and list(mo2) == [0, 0] and list(on) == [2] and len(sg2) == 0


def _full_and_compiled(nsb):
    batch = nsb.workloads.parity_mix(seed=31, brains=4, heavy_types=False)
    out = []
    for b in range(batch.brains):
        ng, sg, mo = batch.brain(b)
        sg = sg.copy()
        sg[::3, 3] = 0                        # sparser graphs: real pruning
        out.append((ng, sg, mo, batch.channels, batch.inputs[b], nsb.native.compile_genome(ng, sg, mo)))
    return out


def test_compiled_genome_same_outputs_oracle(nsb, oracle_built):
    pruned = 0
    for ng, sg, mo, ch, x, (cng, csg, cmo, on, osn) in _full_and_compiled(nsb):
        full = OracleBrain(ng, sg, mo, ch)
        comp = OracleBrain(cng, csg, cmo, ch)
        comp.original_indices(on, osn)
        full.reset(5)
        comp.reset(5)
        pruned += len(ng) - len(cng)
        for _ in range(60):
            r1, o1, _ = full.step(x, 16, 230.0, stop_on_nonfinite=False)
            r2, o2, _ = comp.step(x, 16, 230.0, stop_on_nonfinite=False)
            assert r1 == r2 and np.array_equal(o1, o2)
    assert pruned > 0


@pytest.mark.gpu
def test_compiled_genome_same_outputs_gpu(nsb):
    for ng, sg, mo, ch, x, (cng, csg, cmo, on, osn) in _full_and_compiled(nsb):
        full = nsb.Brain(ng, sg, mo, ch)
        comp = nsb.Brain(cng, csg, cmo, ch)
        comp.original_indices(on, osn)
        full.reset(5)
        comp.reset(5)
        for _ in range(30):
            o1 = full.step(x, 16, 230.0)
            o2 = comp.step(x, 16, 230.0)
            assert np.array_equal(np.asarray(o1), np.asarray(o2))
        full.close()
        comp.close()
