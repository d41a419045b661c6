"""B200-native neural tick of Neural Selection.

libns_b200.so (csrc/, built by build.py) runs the reference's neural tick —
AdEx/conductance neurons, delayed stochastic spike delivery with short-term
plasticity, STDP and modulatory eligibility — as one persistent CUDA kernel per
call on sm_100a, behind the reference's own C ABI (include/ns_b200.h).
`native` binds that ABI; `serve` runs genome-evaluation episodes with
continuous batching; `workloads` builds seeded synthetic populations.
"""
from . import sharding, workloads, world  # noqa: F401
from .native import Brain, GpuBatch, library  # noqa: F401
from .serve import Server  # noqa: F401
