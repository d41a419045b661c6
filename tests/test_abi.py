"""CPU checks of the C-ABI library: it loads, and exports every symbol that
include/ns_b200.h declares (no compute calls: there is no GPU here)."""
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    text = (ROOT / "include" / "ns_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ns_\w+|nsb_\w+)\s*\(", text)))


def test_header_declares_reference_entry_points():
    names = declared_symbols()
    for ref in ["ns_error", "ns_create", "ns_original_indices", "ns_destroy", "ns_reset", "ns_step",
                "ns_gpu_create", "ns_gpu_destroy", "ns_gpu_reset", "ns_gpu_step"]:
        assert ref in names


def test_library_loads_and_exports_every_declared_symbol(nsb):
    from neural_selection_b200 import build
    try:
        build.build()
    except RuntimeError as e:  # pragma: no cover - toolkit missing
        pytest.skip(str(e))
    lib = nsb.native.library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert set(nsb.native.SIGNATURES) == set(declared_symbols())


def test_errors_surface_without_a_gpu(nsb):
    """Creation validates rows on the host before touching the device."""
    import numpy as np
    lib = nsb.native.library()
    with pytest.raises(ValueError, match="Invalid neuron gene"):
        nsb.Brain(np.array([[9, -1, 1, 0, 0, 1, 1, -52, 0, 0]], np.float32), np.zeros((0, 11)), [0], 1)
    with pytest.raises(ValueError, match="Invalid brain dimensions"):
        nsb.Brain(np.array([[0, -1, 1, 0, 0, 1, 1, -52, 0, 0]], np.float32), np.zeros((0, 11)), [0], 0)
    assert lib.ns_error().decode() == "Invalid brain dimensions"
