"""ctypes bindings of libns_b200.so (include/ns_b200.h).

`Brain` mirrors the host-executor entry points the reference's Gym adapter
binds (gym_adapter/adapter.py:28-41: ns_create/ns_reset/ns_step/...), and
`GpuBatch` the batched ones (gym_adapter/gpu.py:35-38: ns_gpu_*), with the same
argument meaning and error behaviour (RuntimeError carrying ns_error()). All
stepping runs on the GPU; there is no CPU fallback: if the library or a GPU is
missing the calls raise.
"""
from __future__ import annotations

import ctypes as ct
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libns_b200.so"

_f = ct.POINTER(ct.c_float)
_u8 = ct.POINTER(ct.c_uint8)
_u32 = ct.POINTER(ct.c_uint32)
_i32 = ct.POINTER(ct.c_int)
_i64 = ct.POINTER(ct.c_int64)
_vp = ct.c_void_p

_lib = None

# Every symbol include/ns_b200.h declares, with (restype, argtypes).
SIGNATURES = {
    "ns_error": (ct.c_char_p, []),
    "ns_create": (_vp, [ct.c_int] * 4 + [_f, _f, _i32]),
    "ns_original_indices": (None, [_vp, _u32, _u32]),
    "ns_destroy": (None, [_vp]),
    "ns_reset": (None, [_vp, ct.c_uint32]),
    "ns_step": (ct.c_int, [_vp, _f, ct.c_int, ct.c_float, _f]),
    "ns_gpu_create": (_vp, [ct.POINTER(_vp), ct.c_int]),
    "ns_gpu_destroy": (None, [_vp]),
    "ns_gpu_reset": (ct.c_int, [_vp, _u8, _u32]),
    "ns_gpu_step": (ct.c_int, [_vp, _f, _u8, ct.c_int, ct.c_float, _f, _i32]),
    "ns_maze_brain_step": (ct.c_int, [_vp, _vp, _u8, ct.c_int, ct.c_float, _f, _i32]),
    "nsb_create_ext": (_vp, [ct.c_int] * 4 + [_f, _f, _i32, ct.c_int]),
    "nsb_gpu_create_ext": (_vp, [ct.POINTER(_vp), ct.c_int, ct.c_int, ct.c_int]),
    "nsb_gpu_create_rows": (_vp, [ct.c_int, _i64, _i64, _f, _f, _i32, ct.c_int, ct.c_int, ct.c_int, ct.c_int]),
    "nsb_gpu_step_device": (ct.c_int, [_vp, _vp, _vp, ct.c_int, ct.c_float, _vp, _vp, _vp]),
    "nsb_gpu_step_graph": (ct.c_int, [_vp, ct.c_int, ct.c_float, _vp]),
    "nsb_gpu_step_noalloc": (ct.c_int, [_vp, _vp, _vp, ct.c_int, ct.c_float, _vp, _vp, _vp]),
    "nsb_gpu_buffer": (_vp, [_vp, ct.c_int]),
    "nsb_gpu_upload": (ct.c_int, [_vp, _f, _u8]),
    "nsb_gpu_download": (ct.c_int, [_vp, _f, _i32]),
    "nsb_gpu_dump": (ct.c_int, [_vp, ct.c_int, _u32, _u32, _i64]),
    "nsb_dump": (ct.c_int, [_vp, _u32, _u32, _i64]),
    "nsb_gpu_load_state": (ct.c_int, [_vp, ct.c_int, _vp]),
    "nsb_gpu_stats": (ct.c_int, [_vp, _i32]),
    "nsb_gpu_take_events": (ct.c_longlong, [_vp]),
    "nsb_gpu_set_delivery": (ct.c_int, [_vp, ct.c_int]),
    "nsb_gpu_set_modulation": (ct.c_int, [_vp, ct.c_int, ct.c_int]),
    "nsb_pool_claim": (ct.c_int, [_vp, ct.c_int, _i32, ct.c_int, _i32]),
    "nsb_pool_release": (ct.c_int, [_vp, _i32, ct.c_int]),
    "nsb_checkpoint_layout": (ct.c_ulonglong, []),
    "nsb_gpu_checkpoint_export": (ct.c_int, [_vp, _vp, _vp, _i64]),
    "nsb_gpu_checkpoint_import": (ct.c_int, [_vp, _vp, ct.c_longlong, _vp, ct.c_longlong, _i64]),
    "nsb_gpu_autotune": (ct.c_int, [_vp, ct.c_int, ct.c_float, _vp]),
    "nsb_gpu_buckets": (ct.c_int, [_vp, _i32]),
    "nsb_gpu_set_bucket": (ct.c_int, [_vp, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int, ct.c_int]),
    "nsb_compile_genome": (ct.c_int, [ct.c_int, ct.c_int, _f, _f, ct.c_int, _i32, _f, _f, _i32, _u32, _u32, _i32,
                                      _i32]),
    "nsb_world_create": (_vp, [_vp, ct.c_int, ct.c_int]),
    "nsb_world_destroy": (None, [_vp]),
    "nsb_world_neural_step": (ct.c_int, [_vp, ct.c_int64]),
    "nsb_world_homeostasis": (ct.c_int, [_vp]),
    "nsb_world_stats": (ct.c_int, [_vp, ct.POINTER(ct.c_longlong)]),
    "nsb_world_ecology_create": (_vp, [_vp, _vp]),
    "nsb_world_ecology_destroy": (None, [_vp]),
    "nsb_world_body_step": (ct.c_int, [_vp, ct.c_int64]),
    "nsb_world_reclaim": (ct.c_int, [_vp, ct.c_int64]),
    "nsb_world_reproduce": (ct.c_int, [_vp]),
    "nsb_world_regrow_and_sense": (ct.c_int, [_vp, ct.c_int64, ct.c_ulonglong, ct.c_float]),
    "nsb_world_layout": (ct.c_int, [ct.POINTER(ct.c_uint64)]),
    "nsb_serve_create": (_vp, [ct.c_longlong, ct.c_double, ct.c_double, ct.c_int, ct.c_int, ct.c_int, ct.c_float,
                               ct.c_double]),
    "nsb_serve_destroy": (None, [_vp]),
    "nsb_serve_register": (ct.c_int, [_vp, ct.c_int, ct.c_int, _f, _f, _i32]),
    "nsb_serve_submit": (ct.c_int, [_vp, ct.c_int, _i32, _u32, _i32, ct.POINTER(ct.c_uint64),
                                    ct.POINTER(ct.c_double)]),
    "nsb_serve_start": (ct.c_int, [_vp]),
    "nsb_serve_stop": (ct.c_int, [_vp]),
    "nsb_serve_run": (ct.c_int, [_vp, ct.c_longlong]),
    "nsb_serve_poll": (ct.c_int, [_vp, _vp, ct.c_int]),
    "nsb_serve_now": (ct.c_double, [_vp]),
    "nsb_serve_stats": (ct.c_int, [_vp, ct.POINTER(ct.c_double)]),
}


def library(path=None):
    """Load libns_b200.so (built by neural-selection_b200/build.py)."""
    global _lib
    if _lib is None or path is not None:
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            raise RuntimeError(f"{p.name} is not built; run neural-selection_b200/build.py (needs nvcc)")
        lib = ct.CDLL(str(p))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


def _err(lib):
    return lib.ns_error().decode()


def compile_genome(neuron_rows, synapse_rows, motors):
    """The genome without neurons that have no causal path to a motor
    (gym_adapter/compile_graph.py:10-28 of the reference, nsb_compile_genome):
    (neuron rows, synapse rows, motors, original neuron indices, original
    synapse indices). Pass the indices to Brain.original_indices so the reset
    streams stay those of the full genome."""
    lib = library()
    ng = np.ascontiguousarray(neuron_rows, np.float32).reshape(-1, 10)
    sg = np.ascontiguousarray(synapse_rows, np.float32).reshape(-1, 11)
    mo = np.ascontiguousarray(motors, np.int32)
    on = np.zeros((max(len(ng), 1), 10), np.float32)
    os_ = np.zeros((max(len(sg), 1), 11), np.float32)
    om = np.zeros(max(len(mo), 1), np.int32)
    idn = np.zeros(max(len(ng), 1), np.uint32)
    ids = np.zeros(max(len(sg), 1), np.uint32)
    n, e = ct.c_int(0), ct.c_int(0)
    sgp = sg if len(sg) else np.zeros((1, 11), np.float32)
    ngp = ng if len(ng) else np.zeros((1, 10), np.float32)
    mop = mo if len(mo) else np.zeros(1, np.int32)
    if lib.nsb_compile_genome(len(ng), len(sg), _p(ngp, _f), _p(sgp, _f), len(mo), _p(mop, _i32), _p(on, _f),
                              _p(os_, _f), _p(om, _i32), _p(idn, _u32), _p(ids, _u32), ct.byref(n), ct.byref(e)):
        raise ValueError(_err(lib))
    return on[:n.value], os_[:e.value], om[:len(mo)], idn[:n.value], ids[:e.value]


NW, SW = 32, 20
CHECKPOINT_NEURON_BYTES, CHECKPOINT_SYNAPSE_BYTES = 344, 136
STATS = ("brains", "units", "big_units", "neurons", "synapses", "heavy", "max_unit_neurons", "grid", "block",
         "smem_bytes", "ctas_per_sm")


class Brain:
    """One brain behind ns_create/ns_reset/ns_step (stepped on the GPU)."""

    def __init__(self, neuron_rows, synapse_rows, motors, channels, max_delay=8):
        self.lib = library()
        ng = np.ascontiguousarray(neuron_rows, np.float32)
        sg = np.ascontiguousarray(synapse_rows, np.float32).reshape(-1, 11)
        mo = np.ascontiguousarray(motors, np.int32)
        self.count, self.edges, self.outputs, self.channels = len(ng), len(sg), len(mo), channels
        sgp = sg if len(sg) else np.zeros((1, 11), np.float32)
        if max_delay == 8:
            self.ptr = self.lib.ns_create(self.count, self.edges, channels, self.outputs, _p(ng, _f), _p(sgp, _f),
                                          _p(mo, _i32))
        else:
            self.ptr = self.lib.nsb_create_ext(self.count, self.edges, channels, self.outputs, _p(ng, _f),
                                               _p(sgp, _f), _p(mo, _i32), max_delay)
        if not self.ptr:
            raise ValueError(_err(self.lib))

    def original_indices(self, neurons, synapses):
        n = np.ascontiguousarray(neurons, np.uint32)
        s = np.ascontiguousarray(synapses, np.uint32) if len(synapses) else np.zeros(1, np.uint32)
        self.lib.ns_original_indices(self.ptr, _p(n, _u32), _p(s, _u32))

    def reset(self, seed):
        self.lib.ns_reset(self.ptr, ct.c_uint32(int(seed) & 0xFFFFFFFF))

    def step(self, inputs, ticks=16, gain=230.0):
        x = np.ascontiguousarray(inputs, np.float32)
        out = np.zeros(self.outputs, np.float32)
        if self.lib.ns_step(self.ptr, _p(x, _f), int(ticks), float(gain), _p(out, _f)):
            raise RuntimeError(_err(self.lib))
        return out

    def dump(self):
        nw = np.zeros((self.count, NW), np.uint32)
        sw = np.zeros((max(self.edges, 1), SW), np.uint32)
        t = ct.c_int64(0)
        if self.lib.nsb_dump(self.ptr, _p(nw, _u32), _p(sw, _u32), ct.byref(t)):
            raise RuntimeError(_err(self.lib))
        return nw, sw[: self.edges], t.value

    def close(self):
        if getattr(self, "ptr", None):
            self.lib.ns_destroy(self.ptr)
            self.ptr = None

    __del__ = close


class GpuBatch:
    """A device batch behind ns_gpu_create/ns_gpu_reset/ns_gpu_step."""

    def __init__(self, ptr, brains, channels, outputs, sizes=None):
        self.lib = library()
        self.ptr = ptr
        self.count, self.channels, self.outputs = brains, channels, outputs
        self.sizes = sizes
        self._keep = None

    @classmethod
    def from_brains(cls, brains, max_delay=8, block=0):
        lib = library()
        arr = (ct.c_void_p * len(brains))(*[b.ptr for b in brains])
        if max_delay == 8 and block == 0:
            ptr = lib.ns_gpu_create(arr, len(brains))
        else:
            ptr = lib.nsb_gpu_create_ext(arr, len(brains), max_delay, block)
        if not ptr:
            raise RuntimeError(_err(lib))
        sizes = [(b.count, b.edges) for b in brains]
        return cls(ptr, len(brains), brains[0].channels, brains[0].outputs, sizes)

    @classmethod
    def from_rows(cls, batch, block=0):
        """From a workloads.Batch of concatenated ABI rows."""
        lib = library()
        no = np.ascontiguousarray(batch.neuron_offsets, np.int64)
        so = np.ascontiguousarray(batch.synapse_offsets, np.int64)
        ng = np.ascontiguousarray(batch.neuron_rows, np.float32)
        sg = np.ascontiguousarray(batch.synapse_rows, np.float32)
        if len(sg) == 0:
            sg = np.zeros((1, 11), np.float32)
        mo = np.ascontiguousarray(batch.motors, np.int32)
        ptr = lib.nsb_gpu_create_rows(batch.brains, _p(no, _i64), _p(so, _i64), _p(ng, _f), _p(sg, _f),
                                      _p(mo, _i32), batch.channels, batch.outputs, batch.max_delay, block)
        if not ptr:
            raise RuntimeError(_err(lib))
        sizes = list(zip(np.diff(no).tolist(), np.diff(so).tolist()))
        return cls(ptr, batch.brains, batch.channels, batch.outputs, sizes)

    def reset(self, seeds, mask=None):
        seeds = np.ascontiguousarray(seeds, np.uint32)
        mask = np.ones(self.count, np.uint8) if mask is None else np.ascontiguousarray(mask, np.uint8)
        if seeds.shape != (self.count,) or mask.shape != (self.count,):
            raise ValueError("Reset dimensions differ")
        if self.lib.ns_gpu_reset(self.ptr, _p(mask, _u8), _p(seeds, _u32)):
            raise RuntimeError(_err(self.lib))

    def step(self, inputs, mask=None, ticks=16, gain=230.0):
        x = np.ascontiguousarray(inputs, np.float32)
        mask = np.ones(self.count, np.uint8) if mask is None else np.ascontiguousarray(mask, np.uint8)
        if x.shape != (self.count, self.channels) or mask.shape != (self.count,):
            raise ValueError("Batch dimensions differ")
        out = np.zeros((self.count, self.outputs), np.float32)
        status = np.zeros(self.count, np.int32)
        if self.lib.ns_gpu_step(self.ptr, _p(x, _f), _p(mask, _u8), int(ticks), float(gain), _p(out, _f),
                                _p(status, _i32)):
            raise RuntimeError(_err(self.lib))
        return out, status

    def step_device(self, d_input, d_mask, ticks, gain, d_output, d_status, stream=0):
        if self.lib.nsb_gpu_step_device(self.ptr, d_input, d_mask, int(ticks), float(gain), d_output, d_status,
                                        stream):
            raise RuntimeError(_err(self.lib))

    def step_noalloc(self, d_input, d_mask, ticks, gain, d_output, d_status, stream=0):
        """Allocation-free step on caller device buffers (see nsb_gpu_step_noalloc)."""
        if self.lib.nsb_gpu_step_noalloc(self.ptr, d_input, d_mask, int(ticks), float(gain), d_output, d_status,
                                         stream):
            raise RuntimeError(_err(self.lib))

    def step_graph(self, ticks=16, gain=230.0, stream=0):
        if self.lib.nsb_gpu_step_graph(self.ptr, int(ticks), float(gain), stream):
            raise RuntimeError(_err(self.lib))

    def upload(self, inputs=None, mask=None):
        x = None if inputs is None else np.ascontiguousarray(inputs, np.float32)
        m = None if mask is None else np.ascontiguousarray(mask, np.uint8)
        if self.lib.nsb_gpu_upload(self.ptr, None if x is None else _p(x, _f), None if m is None else _p(m, _u8)):
            raise RuntimeError(_err(self.lib))

    def download(self):
        out = np.zeros((self.count, self.outputs), np.float32)
        status = np.zeros(self.count, np.int32)
        if self.lib.nsb_gpu_download(self.ptr, _p(out, _f), _p(status, _i32)):
            raise RuntimeError(_err(self.lib))
        return out, status

    def buffer(self, which):
        return self.lib.nsb_gpu_buffer(self.ptr, {"input": 0, "mask": 1, "output": 2, "status": 3}[which])

    def dump(self, brain):
        n, e = self.sizes[brain]
        nw = np.zeros((n, NW), np.uint32)
        sw = np.zeros((max(e, 1), SW), np.uint32)
        t = ct.c_int64(0)
        if self.lib.nsb_gpu_dump(self.ptr, brain, _p(nw, _u32), _p(sw, _u32), ct.byref(t)):
            raise RuntimeError(_err(self.lib))
        return nw, sw[:e], t.value

    def load_state(self, brain, handle):
        if self.lib.nsb_gpu_load_state(self.ptr, brain, handle):
            raise RuntimeError(_err(self.lib))

    def stats(self):
        out = np.zeros(16, np.int32)
        n = self.lib.nsb_gpu_stats(self.ptr, _p(out, _i32))
        return dict(zip(STATS, out[:n].tolist()))

    def take_events(self):
        v = self.lib.nsb_gpu_take_events(self.ptr)
        if v < 0:
            raise RuntimeError(_err(self.lib))
        return int(v)

    def checkpoint_export(self):
        """Reference checkpoint records of every brain: (neuron records as a
        uint8 array of N x 344, synapse records E x 136, ticks per brain)."""
        n = sum(c for c, _ in self.sizes)
        e = sum(m for _, m in self.sizes)
        nr = np.zeros((max(n, 1), CHECKPOINT_NEURON_BYTES), np.uint8)
        sr = np.zeros((max(e, 1), CHECKPOINT_SYNAPSE_BYTES), np.uint8)
        ticks = np.zeros(self.count, np.int64)
        if self.lib.nsb_gpu_checkpoint_export(self.ptr, nr.ctypes.data_as(ct.c_void_p), sr.ctypes.data_as(ct.c_void_p),
                                              _p(ticks, _i64)):
            raise RuntimeError(_err(self.lib))
        return nr[:n], sr[:e], ticks

    def checkpoint_import(self, neuron_records, synapse_records, ticks):
        nr = np.ascontiguousarray(neuron_records, np.uint8).reshape(-1, CHECKPOINT_NEURON_BYTES)
        sr = np.ascontiguousarray(synapse_records, np.uint8).reshape(-1, CHECKPOINT_SYNAPSE_BYTES)
        t = np.ascontiguousarray(ticks, np.int64)
        nrp = nr if len(nr) else np.zeros((1, CHECKPOINT_NEURON_BYTES), np.uint8)
        srp = sr if len(sr) else np.zeros((1, CHECKPOINT_SYNAPSE_BYTES), np.uint8)
        if self.lib.nsb_gpu_checkpoint_import(self.ptr, nrp.ctypes.data_as(ct.c_void_p), len(nr),
                                              srp.ctypes.data_as(ct.c_void_p), len(sr), _p(t, _i64)):
            raise RuntimeError(_err(self.lib))

    def set_modulation(self, period, mod=4):
        """Global modulator pulse every `period` ticks (0: off) with bits `mod` (4 = dopamine)."""
        if self.lib.nsb_gpu_set_modulation(self.ptr, int(period), int(mod)):
            raise RuntimeError(_err(self.lib))

    def set_delivery(self, cooperative):
        """Tick-kernel delivery mode (True: warp-cooperative release). Returns the previous mode."""
        v = self.lib.nsb_gpu_set_delivery(self.ptr, 1 if cooperative else 0)
        if v < 0:
            raise RuntimeError(_err(self.lib))
        return bool(v)

    def autotune(self, ticks=16, gain=230.0, stream=0):
        """Per-bucket autotuner: time candidate configurations of every
        work-unit bucket on the batch's own buffers (state restored) and keep
        the fastest. Returns the packed bucket's delivery mode."""
        v = self.lib.nsb_gpu_autotune(self.ptr, int(ticks), float(gain), ct.c_void_p(stream))
        if v < 0:
            raise RuntimeError(_err(self.lib))
        return bool(v)

    BUCKETS = ("huge", "large", "big", "packed", "heavy")
    BUCKET_FIELDS = ("first_unit", "units", "max_neurons", "max_synapses", "block", "cooperative", "cluster",
                     "meta_cap", "list", "smem_bytes", "grid")

    def buckets(self):
        """The five work-unit buckets and their launch configurations, as dicts."""
        out = np.zeros(55, np.int32)
        n = self.lib.nsb_gpu_buckets(self.ptr, _p(out, _i32))
        rows = out[:n].reshape(-1, 11)
        return [dict(name=name, **{f: int(v) for f, v in zip(self.BUCKET_FIELDS, row)})
                for name, row in zip(self.BUCKETS, rows)]

    def set_bucket(self, bucket, block=256, cooperative=False, cluster=1, meta_cap=6144, list_=True):
        """Set one bucket's configuration (RuntimeError when it cannot run)."""
        if self.lib.nsb_gpu_set_bucket(self.ptr, int(bucket), int(block), 1 if cooperative else 0, int(cluster),
                                       int(meta_cap), 1 if list_ else 0):
            raise RuntimeError(_err(self.lib))

    def close(self):
        if getattr(self, "ptr", None):
            self.lib.ns_gpu_destroy(self.ptr)
            self.ptr = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    __del__ = close
