"""ORACLE — test infrastructure only. ctypes drivers for the C oracle
(oracle/_build) and for the reference host executor compiled from the
reference's own sources (oracle/_ref). Used by tests/, the smoke check and the
CPU-baseline leg of bench.py; never by the product library."""
from __future__ import annotations

import ctypes as ct
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
NW, SW = 32, 20

_f = ct.POINTER(ct.c_float)
_u8 = ct.POINTER(ct.c_uint8)
_u32 = ct.POINTER(ct.c_uint32)
_i32 = ct.POINTER(ct.c_int)
_i64 = ct.POINTER(ct.c_int64)


def _ptr(a, t):
    return a.ctypes.data_as(t)


_libs = {}


def oracle_lib(libm=False):
    """The C restatement: correctly rounded exp/log (default) or glibc."""
    name = "libns_oracle_libm.so" if libm else "libns_oracle.so"
    if name not in _libs:
        path = HERE / "_build" / name
        if not path.exists():
            from . import build as _b  # noqa
        lib = ct.CDLL(str(path))
        lib.or_create.restype = ct.c_void_p
        lib.or_create.argtypes = [ct.c_int] * 4 + [_f, _f, _i32, ct.c_int, ct.c_char_p, ct.c_int]
        lib.or_original_indices.argtypes = [ct.c_void_p, _u32, _u32]
        lib.or_destroy.argtypes = [ct.c_void_p]
        lib.or_set_pulse.argtypes = [ct.c_void_p, ct.c_int, ct.c_int]
        lib.or_reset.argtypes = [ct.c_void_p, ct.c_uint32]
        lib.or_step.argtypes = [ct.c_void_p, _f, ct.c_int, ct.c_float, _f, _u8, ct.c_int]
        lib.or_step.restype = ct.c_int
        lib.or_dump.argtypes = [ct.c_void_p, _u32, _u32, _i64]
        lib.or_count.argtypes = [ct.c_void_p]
        lib.or_edges.argtypes = [ct.c_void_p]
        lib.or_last_events.argtypes = [ct.c_void_p]
        lib.or_last_events.restype = ct.c_int64
        lib.or_cr_expf.argtypes = [ct.c_float]; lib.or_cr_expf.restype = ct.c_float
        lib.or_cr_logf.argtypes = [ct.c_float]; lib.or_cr_logf.restype = ct.c_float
        lib.or_bound_expf.argtypes = [ct.c_float]; lib.or_bound_expf.restype = ct.c_float
        lib.or_protocols.argtypes = [_f, ct.c_int]; lib.or_protocols.restype = ct.c_int
        lib.or_shadow_enable.argtypes = [ct.c_void_p]; lib.or_shadow_enable.restype = ct.c_int
        _d = ct.POINTER(ct.c_double)
        lib.or_shadow_stats.argtypes = [ct.c_void_p, _d, _d]; lib.or_shadow_stats.restype = ct.c_int64
        lib.or_shadow_field.argtypes = [ct.c_int]; lib.or_shadow_field.restype = ct.c_char_p
        lib.or_shadow_dump.argtypes = [ct.c_void_p, _d, _d]
        lib.or_episode.argtypes = [ct.c_void_p, ct.c_uint32, ct.c_int, ct.c_int, ct.c_float, ct.c_double, _i32]
        lib.or_episode.restype = ct.c_int
        lib.or_env_exp.argtypes = [ct.c_double]; lib.or_env_exp.restype = ct.c_double
        lib.or_env_tanh.argtypes = [ct.c_double]; lib.or_env_tanh.restype = ct.c_double
        lib.or_env_sincos.argtypes = [ct.c_double, _d, _d]
        lib.or_env_sequence.argtypes = [ct.POINTER(ct.c_uint64)]
        lib.or_world_step.argtypes = [ct.c_void_p, ct.c_int64]
        lib.or_world_step.restype = ct.c_int
        lib.or_world_homeostasis.argtypes = [ct.c_void_p]
        lib.or_world_body_step.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int64]
        lib.or_world_reclaim.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int64]
        lib.or_world_reproduce.argtypes = [ct.c_void_p, ct.c_void_p]
        lib.or_world_regrow_and_sense.argtypes = [ct.c_void_p, ct.c_void_p, ct.c_int64, ct.c_ulonglong,
                                                  ct.c_float]
        for fn in ("or_cr_sinf", "or_cr_cosf"):
            getattr(lib, fn).argtypes = [ct.c_float]; getattr(lib, fn).restype = ct.c_float
        lib.or_cr_hypotf.argtypes = [ct.c_float, ct.c_float]; lib.or_cr_hypotf.restype = ct.c_float
        lib.or_records.argtypes = [ct.c_void_p] * 5
        lib.or_world_layout.argtypes = [ct.POINTER(ct.c_uint64)]
        lib.or_world_layout.restype = ct.c_int
        _libs[name] = lib
    return _libs[name]


def ref_lib(cr=False):
    """The reference host executor built from its own sources, or None."""
    name = "libns_ref_cr.so" if cr else "libns_ref.so"
    path = HERE / "_ref" / name
    if not path.exists():
        return None
    if name not in _libs:
        lib = ct.CDLL(str(path))
        lib.ns_create.restype = ct.c_void_p
        lib.ns_create.argtypes = [ct.c_int] * 4 + [_f, _f, _i32]
        lib.ns_destroy.argtypes = [ct.c_void_p]
        lib.ns_reset.argtypes = [ct.c_void_p, ct.c_uint32]
        lib.ns_step.argtypes = [ct.c_void_p, _f, ct.c_int, ct.c_float, _f]
        lib.ns_step.restype = ct.c_int
        lib.ns_error.restype = ct.c_char_p
        lib.ns_original_indices.argtypes = [ct.c_void_p, _u32, _u32]
        lib.ref_dump.argtypes = [ct.c_void_p, _u32, _u32, _i64]
        lib.ref_step_raster.argtypes = [ct.c_void_p, _f, ct.c_int, ct.c_float, _f, _u8]
        lib.ref_step_raster.restype = ct.c_int
        _libs[name] = lib
    return _libs[name]


def ref_gpu_lib():
    """The reference CUDA batch (gym_adapter/gpu.cu built from its sources
    with its own flags for sm_100a), or None."""
    path = HERE / "_ref" / "libns_ref_gpu.so"
    if not path.exists():
        return None
    name = "libns_ref_gpu.so"
    if name not in _libs:
        lib = ct.CDLL(str(path))
        lib.ns_create.restype = ct.c_void_p
        lib.ns_create.argtypes = [ct.c_int] * 4 + [_f, _f, _i32]
        lib.ns_destroy.argtypes = [ct.c_void_p]
        lib.ns_error.restype = ct.c_char_p
        lib.ns_gpu_create.restype = ct.c_void_p
        lib.ns_gpu_create.argtypes = [ct.POINTER(ct.c_void_p), ct.c_int]
        lib.ns_gpu_destroy.argtypes = [ct.c_void_p]
        lib.ns_gpu_reset.argtypes = [ct.c_void_p, _u8, _u32]
        lib.ns_gpu_reset.restype = ct.c_int
        lib.ns_gpu_step.argtypes = [ct.c_void_p, _f, _u8, ct.c_int, ct.c_float, _f, _i32]
        lib.ns_gpu_step.restype = ct.c_int
        _libs[name] = lib
    return _libs[name]


def ref_world_lib():
    """The reference world simulator's neural kernels (src/main.cu) behind the
    timing harness oracle/ref_world_harness.cu, or None."""
    path = HERE / "_ref" / "libns_ref_world.so"
    if not path.exists():
        return None
    name = "libns_ref_world.so"
    if name not in _libs:
        lib = ct.CDLL(str(path))
        lib.ref_world_create.restype = ct.c_void_p
        lib.ref_world_create.argtypes = [ct.c_int, _i64, _i64, _f, _f, _i32, ct.c_int, ct.c_uint32, ct.c_int]
        lib.ref_world_step.argtypes = [ct.c_void_p]
        lib.ref_world_step.restype = ct.c_int
        lib.ref_world_sync.restype = ct.c_int
        lib.ref_world_total_spikes.argtypes = [ct.c_void_p, ct.c_int]
        lib.ref_world_total_spikes.restype = ct.c_longlong
        lib.ref_world_destroy.argtypes = [ct.c_void_p]
        lib.ref_world_layout.argtypes = [ct.POINTER(ct.c_uint64), ct.POINTER(ct.c_uint64), ct.POINTER(ct.c_uint64)]
        lib.ref_world_layout.restype = ct.c_int
        lib.ref_world_claim_sequential.argtypes = [ct.c_void_p, ct.c_int, ct.c_void_p, ct.c_int, ct.c_void_p]
        lib.ref_world_claim_sequential.restype = ct.c_int
        _libs[name] = lib
    return _libs[name]


def world_step(pools, step):
    """The oracle's world stage (or_world_step) on host WorldPools, in place."""
    lib = oracle_lib()
    st = pools.struct()
    if lib.or_world_step(ct.byref(st), int(step)) != 0:
        raise ValueError("oracle: invalid live synapse gene")


def world_homeostasis(pools):
    lib = oracle_lib()
    st = pools.struct()
    lib.or_world_homeostasis(ct.byref(st))


def world_body_step(pools, eco, step):
    """The oracle's body step, spatial index, bites and predation deaths
    (or_world_body_step) on host WorldPools and Ecology, in place."""
    oracle_lib().or_world_body_step(ct.byref(pools.struct()), ct.byref(eco.struct()), int(step))


def world_reclaim(pools, eco, step):
    """The oracle's reclaim_dead_genomes (or_world_reclaim), in place."""
    oracle_lib().or_world_reclaim(ct.byref(pools.struct()), ct.byref(eco.struct()), int(step))


def world_reproduce(pools, eco):
    """The oracle's reproduce with mutate (or_world_reproduce), in place."""
    oracle_lib().or_world_reproduce(ct.byref(pools.struct()), ct.byref(eco.struct()))


def world_regrow_and_sense(pools, eco, step, seed, renewal_probability):
    """The oracle's regrow, spatial index and update_senses, in place."""
    oracle_lib().or_world_regrow_and_sense(ct.byref(pools.struct()), ct.byref(eco.struct()), int(step), int(seed),
                                           float(renewal_probability))


def oracle_records(batch, seeds):
    """Reset records of every brain of a workloads.Batch from the oracle, in
    the reference layouts (neuron genes 124 B, states 120 B, synapse genes
    40 B, states 80 B), concatenated in batch order."""
    lib = oracle_lib()
    N, E = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1])
    ng = np.zeros((N, 124), np.uint8)
    ns = np.zeros((N, 120), np.uint8)
    sg = np.zeros((max(E, 1), 40), np.uint8)
    ss = np.zeros((max(E, 1), 80), np.uint8)
    for b in range(batch.brains):
        n0, n1 = batch.neuron_offsets[b], batch.neuron_offsets[b + 1]
        e0, e1 = batch.synapse_offsets[b], batch.synapse_offsets[b + 1]
        o = OracleBrain(*batch.brain(b), batch.channels, batch.max_delay)
        o.reset(int(seeds[b]))
        lib.or_records(ct.c_void_p(o.ptr), ng[n0:].ctypes.data, ns[n0:].ctypes.data, sg[e0:].ctypes.data,
                       ss[e0:].ctypes.data)
    return ng, ns, sg[:E], ss[:E]


class OracleBrain:
    """One brain in the C oracle."""

    def __init__(self, neuron_rows, synapse_rows, motors, channels, max_delay=8, libm=False):
        self.lib = oracle_lib(libm)
        ng = np.ascontiguousarray(neuron_rows, np.float32)
        sg = np.ascontiguousarray(synapse_rows, np.float32).reshape(-1, 11)
        mo = np.ascontiguousarray(motors, np.int32)
        err = ct.create_string_buffer(128)
        self.count, self.edges, self.outputs, self.channels = len(ng), len(sg), len(mo), channels
        sgp = sg if len(sg) else np.zeros((1, 11), np.float32)
        self.ptr = self.lib.or_create(self.count, self.edges, channels, self.outputs, _ptr(ng, _f),
                                      _ptr(sgp, _f), _ptr(mo, _i32), max_delay, err, 128)
        if not self.ptr:
            raise ValueError(err.value.decode())

    def reset(self, seed):
        self.lib.or_reset(self.ptr, ct.c_uint32(seed))

    def records(self):
        """(neuron genes, neuron states, synapse genes, synapse states) as
        uint8 rows of the reference layouts (124, 120, 40, 80 bytes)."""
        ng = np.zeros((self.count, 124), np.uint8)
        ns = np.zeros((self.count, 120), np.uint8)
        sg = np.zeros((max(self.edges, 1), 40), np.uint8)
        ss = np.zeros((max(self.edges, 1), 80), np.uint8)
        self.lib.or_records(ct.c_void_p(self.ptr), ng.ctypes.data, ns.ctypes.data, sg.ctypes.data, ss.ctypes.data)
        return ng, ns, sg[:self.edges], ss[:self.edges]

    def set_pulse(self, period, mod=4):
        """Global modulator pulse every `period` ticks with bits `mod` (4 = dopamine)."""
        self.lib.or_set_pulse(self.ptr, int(period), int(mod))

    def original_indices(self, neurons, synapses):
        n = np.ascontiguousarray(neurons, np.uint32)
        s = np.ascontiguousarray(synapses, np.uint32) if len(synapses) else np.zeros(1, np.uint32)
        self.lib.or_original_indices(self.ptr, _ptr(n, _u32), _ptr(s, _u32))

    def step(self, inputs, ticks, gain=230.0, raster=False, stop_on_nonfinite=True):
        x = np.ascontiguousarray(inputs, np.float32)
        out = np.zeros(self.outputs, np.float32)
        r = np.zeros((ticks, self.count), np.uint8) if raster else None
        rc = self.lib.or_step(self.ptr, _ptr(x, _f), ticks, gain, _ptr(out, _f),
                              _ptr(r, _u8) if raster else None, 1 if stop_on_nonfinite else 0)
        return rc, out, r

    def events(self):
        return self.lib.or_last_events(self.ptr)

    SHADOW_FIELDS = 15

    def enable_shadow(self):
        """Start the FP64 shadow from the current state (ValueError for LP/Prinz cells)."""
        if self.lib.or_shadow_enable(self.ptr):
            raise ValueError("FP64 shadow: brain has LP/Prinz cells")

    def shadow_stats(self):
        """{field: (max abs error, max rel error)} of the binary32 state against
        the FP64 shadow over every tick since enable_shadow, and the tick count."""
        a = np.zeros(self.SHADOW_FIELDS, np.float64)
        r = np.zeros(self.SHADOW_FIELDS, np.float64)
        d = ct.POINTER(ct.c_double)
        ticks = self.lib.or_shadow_stats(self.ptr, a.ctypes.data_as(d), r.ctypes.data_as(d))
        names = [self.lib.or_shadow_field(i).decode() for i in range(self.SHADOW_FIELDS)]
        return {n: (float(x), float(y)) for n, x, y in zip(names, a, r)}, int(ticks)

    def episode(self, seed, steps, ticks=16, gain=230.0, smoothing=0.4):
        """One pole-on-cart episode from a reset with `seed` (or_episode.c)."""
        out = np.zeros(5, np.int32)
        if self.lib.or_episode(self.ptr, ct.c_uint32(seed), int(steps), int(ticks), float(gain), float(smoothing),
                               _ptr(out, _i32)):
            raise ValueError("or_episode: invalid arguments")
        return {"steps": int(out[0]), "reward": int(out[1]), "failures": int(out[2]),
                "trace": int(np.uint32(out[3].view(np.uint32))), "status": int(out[4])}

    def shadow_dump(self):
        """FP64 shadow voltages (count,) and synaptic weights (edges,)."""
        v = np.zeros(self.count, np.float64)
        w = np.zeros(max(self.edges, 1), np.float64)
        d = ct.POINTER(ct.c_double)
        self.lib.or_shadow_dump(self.ptr, v.ctypes.data_as(d), w.ctypes.data_as(d))
        return v, w[: self.edges]

    def dump(self):
        nw = np.zeros((self.count, NW), np.uint32)
        sw = np.zeros((max(self.edges, 1), SW), np.uint32)
        t = ct.c_int64(0)
        self.lib.or_dump(self.ptr, _ptr(nw, _u32), _ptr(sw, _u32), ct.byref(t))
        return nw, sw[: self.edges], t.value

    def close(self):
        if self.ptr:
            self.lib.or_destroy(self.ptr)
            self.ptr = None

    __del__ = close


class RefBrain:
    """One brain in the reference host executor (gym_adapter/native.cpp)."""

    def __init__(self, neuron_rows, synapse_rows, motors, channels, cr=False):
        self.lib = ref_lib(cr)
        if self.lib is None:
            raise FileNotFoundError("reference build absent (oracle/_ref)")
        ng = np.ascontiguousarray(neuron_rows, np.float32)
        sg = np.ascontiguousarray(synapse_rows, np.float32).reshape(-1, 11)
        mo = np.ascontiguousarray(motors, np.int32)
        self.count, self.edges, self.outputs = len(ng), len(sg), len(mo)
        sgp = sg if len(sg) else np.zeros((1, 11), np.float32)
        self.ptr = self.lib.ns_create(self.count, self.edges, channels, self.outputs,
                                      _ptr(ng, _f), _ptr(sgp, _f), _ptr(mo, _i32))
        if not self.ptr:
            raise ValueError(self.lib.ns_error().decode())

    def reset(self, seed):
        self.lib.ns_reset(self.ptr, ct.c_uint32(seed))

    def original_indices(self, neurons, synapses):
        n = np.ascontiguousarray(neurons, np.uint32)
        s = np.ascontiguousarray(synapses, np.uint32) if len(synapses) else np.zeros(1, np.uint32)
        self.lib.ns_original_indices(self.ptr, _ptr(n, _u32), _ptr(s, _u32))

    def step(self, inputs, ticks, gain=230.0, raster=False):
        x = np.ascontiguousarray(inputs, np.float32)
        out = np.zeros(self.outputs, np.float32)
        if raster:
            r = np.zeros((ticks, self.count), np.uint8)
            rc = self.lib.ref_step_raster(self.ptr, _ptr(x, _f), ticks, gain, _ptr(out, _f), _ptr(r, _u8))
            return rc, out, r
        rc = self.lib.ns_step(self.ptr, _ptr(x, _f), ticks, gain, _ptr(out, _f))
        return rc, out, None

    def dump(self):
        nw = np.zeros((self.count, NW), np.uint32)
        sw = np.zeros((max(self.edges, 1), SW), np.uint32)
        t = ct.c_int64(0)
        self.lib.ref_dump(self.ptr, _ptr(nw, _u32), _ptr(sw, _u32), ct.byref(t))
        return nw, sw[: self.edges], t.value

    def close(self):
        if self.ptr:
            self.lib.ns_destroy(self.ptr)
            self.ptr = None

    __del__ = close


def protocols():
    out = np.zeros(40, np.float32)
    n = oracle_lib().or_protocols(_ptr(out, _f), 40)
    return out[:n]


# ---- sampled stepping in worker processes (tests only) -------------------------
def _step_brain_jobs(jobs, calls, ticks, gain, pulse):
    """Steps each job's brain `calls` times from its reset in this process.
    jobs: (index, neuron rows, synapse rows, motors, channels, max delay,
    inputs, seed). Returns (index, outputs (calls x outputs), status (calls,),
    neuron dump, synapse dump, tick) per job."""
    out = []
    for idx, ng, sg, mo, channels, max_delay, inputs, seed in jobs:
        o = OracleBrain(ng, sg, mo, channels, max_delay)
        if pulse is not None:
            o.set_pulse(*pulse)
        o.reset(int(seed))
        outs = np.zeros((calls, len(mo)), np.float32)
        status = np.zeros(calls, np.int32)
        for c in range(calls):
            rc, oo, _ = o.step(inputs, ticks, gain, stop_on_nonfinite=False)
            outs[c] = oo
            status[c] = rc
        nw, sw, t = o.dump()
        o.close()
        out.append((idx, outs, status, nw, sw, t))
    return out


class SampledOracle:
    """The oracle stepping a sample of a batch's brains, split across worker
    processes (spawn start method, so the workers hold no CUDA state). Start it
    before the GPU run and collect with result(): the two then overlap."""

    def __init__(self, batch, indices, seeds, calls, ticks=16, gain=None, pulse=None, processes=None):
        import concurrent.futures as cf
        import multiprocessing as mp
        import os
        gain = batch.gain if gain is None else gain
        jobs = []
        for i in indices:
            ng, sg, mo = batch.brain(int(i))
            jobs.append((int(i), ng, sg, mo, batch.channels, batch.max_delay, batch.inputs[int(i)],
                         int(seeds[int(i)])))
        # largest brains first, dealt round-robin, so the workers finish together
        jobs.sort(key=lambda j: -len(j[1]))
        self.processes = max(1, min(processes or os.cpu_count() or 1, len(jobs)))
        parts = [jobs[k::self.processes] for k in range(self.processes)]
        self.pool = cf.ProcessPoolExecutor(self.processes, mp_context=mp.get_context("spawn"))
        self.futures = [self.pool.submit(_step_brain_jobs, p, calls, ticks, gain, pulse) for p in parts]

    def result(self):
        """{index: (outputs, status, neuron dump, synapse dump, tick)}."""
        res = {}
        try:
            for f in self.futures:
                for idx, outs, status, nw, sw, t in f.result():
                    res[idx] = (outs, status, nw, sw, t)
        finally:
            self.pool.shutdown()
        return res


def _host_package():
    """The product's Python package loaded by path in a worker process, for
    its host-side pool records (WorldPools) only; nothing here touches a GPU."""
    import importlib.util
    import sys
    name = "neural_selection_b200"
    if name not in sys.modules:
        pkg = HERE.parent / "neural-selection_b200"
        spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py",
                                                      submodule_search_locations=[str(pkg)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def _world_subset_run(fields_, subset, steps, senses_seed):
    """The oracle's world stage over `steps` world steps for the animals in
    `subset` only (every other animal marked not alive, so it is skipped): the
    senses of every step are drawn from `senses_seed` for the whole
    population, ages advance for living animals, homeostasis after each step.
    fields_: the WorldPools fields as a dict. Returns the motor counts of every
    step (steps x animals x 5) and the final pools as a dict."""
    pools = _host_package().world.WorldPools(**fields_)
    alive = pools.animals["alive"].copy()
    keep = np.zeros(len(alive), bool)
    keep[np.asarray(subset, np.int64)] = True
    pools.animals["alive"][~keep & (alive == 1)] = 0
    rng = np.random.default_rng(senses_seed)
    motors = np.zeros((steps,) + pools.motors.shape, np.int32)
    for step in range(1, steps + 1):
        pools.senses[:] = rng.random(pools.senses.shape).astype(np.float32)
        pools.motors[:] = 0
        world_step(pools, step)
        motors[step - 1] = pools.motors
        pools.animals["age"][pools.animals["alive"] == 1] += 1
        world_homeostasis(pools)
    pools.animals["alive"][:] = alive
    return motors, dict(pools.__dict__)


class SubsetWorldOracle:
    """The oracle's world stage on disjoint subsets of a population's animals
    in worker processes (spawn). Animals do not interact within the neural
    stage, so each subset's pools evolve exactly as in a run of the whole
    population."""

    def __init__(self, pools, steps, senses_seed, processes=None):
        import concurrent.futures as cf
        import multiprocessing as mp
        import os
        live = np.nonzero(pools.animals["alive"] == 1)[0]
        self.processes = max(1, min(processes or os.cpu_count() or 1, len(live)))
        self.subsets = [live[k::self.processes] for k in range(self.processes)]
        fields_ = dict(pools.__dict__)
        self.pool = cf.ProcessPoolExecutor(self.processes, mp_context=mp.get_context("spawn"))
        self.futures = [self.pool.submit(_world_subset_run, fields_, s, steps, senses_seed) for s in self.subsets]

    def result(self):
        """[(subset, motors per step, final pool fields)] per worker."""
        try:
            return [(s, *f.result()) for s, f in zip(self.subsets, self.futures)]
        finally:
            self.pool.shutdown()
