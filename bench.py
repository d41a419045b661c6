"""Benchmark of the B200 neural tick at full pools.

Workload (one step = one world step = 16 ticks of 1 ms): 32,768 brains of
uneven size (lognormal, median 96, sigma 1, clipped to 16-4,096 and rescaled to
fill 4,194,304 neuron slots), 8,388,608 synapses in proportion to size,
delays 1-16 ms, Poisson 10-40 Hz receptor drive; seeded synthetic inputs
(Philox4x32-10, seed 2). All device state (1.4 GB) exceeds the 126 MB L2, so
every step streams it from HBM.

value : neuron-ticks/s with inputs resident on the device, one persistent
        fused launch per step replayed from a captured CUDA graph, timed with
        CUDA events on the launching stream (max over ranks).
e2e   : the same metric through the reference's C ABI call ns_gpu_step with
        pinned host buffers (host->device observations, device->host motor
        outputs and status inside the timed region).
other_configs : (N=1, default run) the same metric, device-resident, on the
        plasticity-heavy full pools (config 4) and the plain small batch
        (config 1), each after its own per-bucket autotune.
reference_cuda : (N=1, default run) the reference's own CUDA forms on the
        same batch and GPU after this library's buffers are freed: the Gym
        batch kernel step_batch (gym_adapter/gpu.cu) and the world simulator's
        neural stage (src/main.cu) as fused global-slot kernels and as
        --block-brains tiers; best_ratio = value / the fastest form's.
--impl reference : the reference's own host executor (gym_adapter/native.cpp
        built from its sources into oracle/_ref) on the host cores.
--impl reference-cuda : the reference's CUDA forms alone, one line each.

--world : the world simulator's neural stage (config 2 founders, or --world-population
        full) through nsb_world_*, then the reference's world kernels on the same pools.
--world-loop : the world step (neural stage, body, bites, homeostasis,
        reclamation, reproduction, regrowth, senses), closed loop, then the
        reference's kernels for the same steps on the same initial pools.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
       (N > 1 under torch.distributed.run: one full-pool replica per GPU).
"""
import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
ALGO_BYTES_PER_NEURON = 172    # per world step: gene 64 + log-AMPA 4 + state 2x48 + delay-ring 2x4
ALGO_BYTES_PER_SYNAPSE = 176   # per world step: gene 40 + state 2x68
METRIC = "neuron-ticks/s at full pools"
UNIT = "neuron-ticks/s"


def load_package():
    name = "neural_selection_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = ROOT / "neural-selection_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_step():
    """DRAM bytes of one step's tick-kernel launches (every bucket) from the
    committed ncu summary of the full-pool workload."""
    p = ROOT / "profiles" / "tick_kernel_full_pools.txt"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("dram_bytes_per_step:"):
            return float(line.split(":")[1].split()[0])
    return None


def warp_instructions_per_neuron_tick():
    """Warp instructions the light tick kernel issues per neuron-tick, from
    the committed ncu summary of the benchmark's 1/8 slice."""
    p = ROOT / "profiles" / "tick_kernel_list_div8_full_set.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("warp_instructions_per_neuron_tick:"):
            return float(line.split(":")[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0])); mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, v in zip(names, parts[2:6]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


# Workloads the reference's own CUDA forms are timed on as well.
SMALL_OR_MAIN = ("batched_uneven", "plain_small", "heavy_smoke", "heavy_founders")


def workload(nsb, seed, fraction=1, kind="batched_uneven"):
    """The full-pool workload, or with --fraction D a 1/D slice of it (brains,
    neuron and synapse pools all divided by D; same size distribution) for
    profiler captures that must stay small. kind "plasticity_heavy": the same
    pools with every synapse on the triplet/dopamine profile (config 4)."""
    if kind == "plasticity_heavy":
        tag = "full" if fraction == 1 else f"div{fraction}"
        cache = Path(os.environ.get("NSB_BENCH_CACHE", "/tmp")) / f"nsb_heavy_{tag}_seed{seed}.npz"
        W = nsb.workloads
        meta = {"ticks_per_step": 16, "steps": 1000, "pulse_period": 50, "pulse_mod": 4, "burst_fraction": 0.3}
        if cache.exists():
            z = np.load(cache)
            return W.Batch(z["nr"], z["sr"], z["no"], z["so"], z["mo"], int(z["ch"]), int(z["md"]),
                           "plasticity_heavy", z["inp"], 230.0, meta)
        b = W.plasticity_heavy(seed=seed + 2, brains=32768 // fraction, total_neurons=4194304 // fraction,
                               total_synapses=8388608 // fraction)
        assert all(b.meta[k] == v for k, v in meta.items())
        try:
            np.savez(cache, nr=b.neuron_rows, sr=b.synapse_rows, no=b.neuron_offsets, so=b.synapse_offsets,
                     mo=b.motors, ch=b.channels, md=b.max_delay, inp=b.inputs)
        except OSError:
            pass
        return b
    if kind == "plain_small":
        # config 1: 64 brains x 48 neurons, 600 synapses each, 20 Hz receptor drive
        return nsb.workloads.plain_small(seed=seed)
    if kind == "heavy_smoke":
        # 4 brains of every cell type with 43 LP and Prinz cells among them
        return nsb.workloads.parity_mix(seed=seed + 1, brains=4)
    if kind == "heavy_founders":
        # 256 world founders with LP, Prinz and LFS cells (3 % each of hidden
        # cells), stepped as one batch
        return nsb.workloads.world_founders(seed=seed, founders=256, heavy_types=True)
    if kind == "serving_population":
        # the serving genomes (config 5) stepped as one static batch of 5,000
        # genomes (about 4.1 M neurons, 33 M synapses), every channel at 0.5
        b = nsb.workloads.serving_library(seed=5 + seed - 2, genomes=5000 // fraction)
        b.inputs = np.full((b.brains, b.channels), 0.5, np.float32)
        return b
    tag = "full" if fraction == 1 else f"div{fraction}"
    cache = Path(os.environ.get("NSB_BENCH_CACHE", "/tmp")) / f"nsb_uneven_{tag}_seed{seed}.npz"
    W = nsb.workloads
    if cache.exists():
        z = np.load(cache)
        return W.Batch(z["nr"], z["sr"], z["no"], z["so"], z["mo"], int(z["ch"]), int(z["md"]), "batched_uneven",
                       z["inp"], 230.0, {})
    b = W.batched_uneven(seed=seed, brains=32768 // fraction, total_neurons=4194304 // fraction,
                         total_synapses=8388608 // fraction)
    try:
        np.savez(cache, nr=b.neuron_rows, sr=b.synapse_rows, no=b.neuron_offsets, so=b.synapse_offsets,
                 mo=b.motors, ch=b.channels, md=b.max_delay, inp=b.inputs)
    except OSError:
        pass
    return b


# ---- CPU: the reference host executor -------------------------------------------
_WORKER_BRAINS = []


def _cpu_init(jobs, use_ref, pulse):
    sys.path.insert(0, str(ROOT))
    from oracle import pyoracle
    global _WORKER_BRAINS
    _WORKER_BRAINS = []
    for rows_n, rows_s, motors, channels, inputs in jobs:
        if use_ref:
            b = pyoracle.RefBrain(rows_n, rows_s, motors, channels)
        else:
            b = pyoracle.OracleBrain(rows_n, rows_s, motors, channels, 16, libm=True)
            if pulse:
                b.set_pulse(*pulse)
        b.reset(7)
        _WORKER_BRAINS.append((b, inputs, len(rows_n)))


def _cpu_step(ticks):
    t0 = time.perf_counter()
    nt = 0
    for b, inputs, n in _WORKER_BRAINS:
        b.step(inputs, ticks, 230.0)
        nt += n * ticks
    return nt, time.perf_counter() - t0


class CpuReference:
    """The reference host executor (gym_adapter/native.cpp built from its
    sources) over a strided sample of brains, the sample split across one
    process per host core; each process keeps its brains between steps."""

    def __init__(self, batch, stride, processes):
        import multiprocessing as mp
        sys.path.insert(0, str(ROOT))
        from oracle import pyoracle
        pulse = (batch.meta["pulse_period"], batch.meta["pulse_mod"]) if "pulse_period" in batch.meta else None
        # The reference has no profile 6 (triplet/dopamine): that workload runs on the oracle port.
        self.use_ref = pyoracle.ref_lib() is not None and pulse is None
        idx = np.argsort(np.diff(batch.neuron_offsets), kind="stable")[::stride]
        jobs = []
        for i in idx:
            ng, sg, mo = batch.brain(int(i))
            sg = sg.copy()
            if self.use_ref:   # the reference ABI accepts delays 1-8 only; fold longer ones
                sg[:, 4] = (sg[:, 4] - 1) % 8 + 1
            jobs.append((ng, sg, mo, batch.channels, batch.inputs[int(i)]))
        self.processes = max(1, min(processes, len(jobs)))
        parts = [jobs[k::self.processes] for k in range(self.processes)]
        ctx = mp.get_context("spawn")
        self.pools = [ctx.Pool(1, initializer=_cpu_init, initargs=(part, self.use_ref, pulse)) for part in parts]
        self.kind = "reference" if self.use_ref else "port"
        self.sample = (f"{len(jobs)} of {batch.brains} brains (every {stride}th by size, "
                       f"{sum(len(j[0]) for j in jobs)} neurons), 16-tick steps; " +
                       ("delays folded into 1-8 (the reference ABI accepts 1-8)" if self.use_ref else
                        "oracle port with the delay-16 ring"))

    def step(self, ticks=16):
        res = [p.apply_async(_cpu_step, (ticks,)) for p in self.pools]
        out = [r.get() for r in res]
        return sum(o[0] for o in out), max(o[1] for o in out)

    def close(self):
        for p in self.pools:
            p.terminate()


def run_reference(args, rank, world):
    if rank != 0:
        return
    nsb = load_package()
    batch = workload(nsb, 2)
    ref = CpuReference(batch, 8, os.cpu_count() or 1)
    for _ in range(args.warmup):
        ref.step(16)
    nt, secs = 0, 0.0
    for _ in range(args.steps):
        a, b = ref.step(16)
        nt += a; secs += b
    ref.close()
    value = nt / secs
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (Philox4x32-10 seed 2)",
            "config": {"workload": "batched_uneven_full_pools", "brains": batch.brains, "neurons": 4194304,
                       "synapses": 8388608, "ticks_per_step": 16, "delays_ms": "1-16"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.processes, "kind": ref.kind,
                             "sample": ref.sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_cuda_forms(batch, steps, warmup, gpu_index=0):
    """The reference's own CUDA forms of the neural tick on `batch`, timed with
    CUDA events on the default stream they launch on:
      step_batch   : gym_adapter/gpu.cu (one CTA of 32 threads per brain),
                     ns_gpu_step through its C ABI with host buffers, its flags
                     --fmad=false --prec-div=true --prec-sqrt=true;
      global_slot  : src/main.cu neural stage, fused global-slot kernels;
      block_tiers  : src/main.cu neural stage, --block-brains tiers with the
                     global-slot fallback (both --use_fast_math, as the world
                     binary is built).
    Delays are folded into 1-8 because the reference accepts 1-8 only; the
    cost per tick does not depend on the delay. Returns (forms, notes): forms
    maps a form to {ms_per_step, value, e2e_value, ...}; the world forms are
    timed only for the full-pool batch. Nothing of this library runs here."""
    import ctypes as ct
    import torch
    sys.path.insert(0, str(ROOT))
    from oracle import pyoracle
    forms, notes = {}, []
    lib = pyoracle.ref_gpu_lib()
    N = len(batch.neuron_rows)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if lib is None:
        notes.append("oracle/_ref/libns_ref_gpu.so not built")
    else:
        f, i32 = ct.POINTER(ct.c_float), ct.POINTER(ct.c_int)
        t_setup = time.perf_counter()
        handles = []
        for b in range(batch.brains):
            ng, sg, mo = batch.brain(b)
            sg = np.ascontiguousarray(sg.copy())
            sg[:, 4] = (sg[:, 4] - 1) % 8 + 1
            ng = np.ascontiguousarray(ng); mo = np.ascontiguousarray(mo, np.int32)
            h = lib.ns_create(len(ng), len(sg), batch.channels, batch.outputs, ng.ctypes.data_as(f),
                              sg.ctypes.data_as(f), mo.ctypes.data_as(i32))
            if not h:
                raise RuntimeError(lib.ns_error().decode())
            handles.append(h)
        arr = (ct.c_void_p * len(handles))(*handles)
        t0 = time.perf_counter()
        gb = lib.ns_gpu_create(arr, len(handles))
        create_s = time.perf_counter() - t0
        for h in handles:
            lib.ns_destroy(h)
        if not gb:
            raise RuntimeError(lib.ns_error().decode())
        mask = np.ones(batch.brains, np.uint8)
        seeds = np.arange(batch.brains, dtype=np.uint32)
        lib.ns_gpu_reset(gb, mask.ctypes.data_as(ct.POINTER(ct.c_uint8)),
                         seeds.ctypes.data_as(ct.POINTER(ct.c_uint32)))
        inp = np.ascontiguousarray(batch.inputs)
        out = np.zeros((batch.brains, batch.outputs), np.float32)
        st = np.zeros(batch.brains, np.int32)

        def step():
            rc = lib.ns_gpu_step(gb, inp.ctypes.data_as(f), mask.ctypes.data_as(ct.POINTER(ct.c_uint8)), 16,
                                 batch.gain, out.ctypes.data_as(f), st.ctypes.data_as(i32))
            if rc:
                raise RuntimeError(lib.ns_error().decode())
        for _ in range(max(warmup, 3)):
            step()
        torch.cuda.synchronize()
        with ClockSampler(gpu_index) as clk:
            t0 = time.perf_counter()
            e0.record()
            for _ in range(steps):
                step()
            e1.record()
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
        ms = e0.elapsed_time(e1) / steps
        lib.ns_gpu_destroy(gb)
        forms["step_batch"] = {
            "ms_per_step": ms, "value": N * 16 / (ms / 1e3), "e2e_value": N * 16 * steps / wall,
            "kernel": "gym_adapter/gpu.cu step_batch, 32 threads per brain, --fmad=false --prec-div=true "
                      "--prec-sqrt=true, sm_100a",
            "h2d_bytes_per_step": int(inp.nbytes + mask.nbytes), "d2h_bytes_per_step": int(out.nbytes + st.nbytes),
            "setup_s": time.perf_counter() - t_setup - wall, "ns_gpu_create_s": create_s, "steps": steps,
            "clocks": clk.summary()}
    if batch.brains != 32768:
        return forms, notes
    wlib = pyoracle.ref_world_lib()
    if wlib is None:
        notes.append("oracle/_ref/libns_ref_world.so not built")
        return forms, notes
    f, i32 = ct.POINTER(ct.c_float), ct.POINTER(ct.c_int)
    for mode, key, label in ((0, "global_slot", "fused global-slot kernels"),
                             (1, "block_tiers", "--block-brains tiers + global-slot fallback")):
        no = np.ascontiguousarray(batch.neuron_offsets, np.int64)
        so = np.ascontiguousarray(batch.synapse_offsets, np.int64)
        w = wlib.ref_world_create(batch.brains, no.ctypes.data_as(ct.POINTER(ct.c_int64)),
                                  so.ctypes.data_as(ct.POINTER(ct.c_int64)),
                                  np.ascontiguousarray(batch.neuron_rows).ctypes.data_as(f),
                                  np.ascontiguousarray(batch.synapse_rows).ctypes.data_as(f),
                                  np.ascontiguousarray(batch.motors, np.int32).ctypes.data_as(i32),
                                  batch.outputs, 7, mode)
        if not w:
            notes.append(f"{key}: pool setup failed")
            continue
        for _ in range(max(warmup, 3)):
            assert wlib.ref_world_step(w) == 0
        wlib.ref_world_sync()
        with ClockSampler(gpu_index) as clk:
            t0 = time.perf_counter()
            e0.record()
            for _ in range(steps):
                assert wlib.ref_world_step(w) == 0
            e1.record()
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
        ms = e0.elapsed_time(e1) / steps
        spikes = wlib.ref_world_total_spikes(w, N)
        wlib.ref_world_destroy(w)
        forms[key] = {"ms_per_step": ms, "value": N * 16 / (ms / 1e3), "e2e_value": N * 16 * steps / wall,
                      "kernel": f"src/main.cu neural stage, {label}, --use_fast_math, sm_100a",
                      "total_spikes_after": int(spikes), "steps": steps, "clocks": clk.summary()}
    return forms, notes


def run_reference_cuda(args, rank, world, local_rank):
    """The reference's own CUDA forms alone, one JSON line per form."""
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local_rank)
    nsb = load_package()
    batch = workload(nsb, 2, 1, args.workload if args.workload in SMALL_OR_MAIN else "batched_uneven")
    steps = max(3, min(args.steps, 20))
    forms, notes = reference_cuda_forms(batch, steps, args.warmup, local_rank)
    N = len(batch.neuron_rows)
    for key, fm in forms.items():
        line = {"impl": "reference-cuda" if key == "step_batch" else "reference-cuda-world", "metric": METRIC,
                "value": fm["value"], "unit": UNIT, "n_gpus": 1, "steps": fm["steps"], "warmup": max(args.warmup, 3),
                "ms_per_step": fm["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic (Philox4x32-10 seed 2)",
                "config": {"workload": ("batched_uneven_full_pools" if batch.brains == 32768 else batch.name),
                           "brains": batch.brains, "neurons": N, "synapses": len(batch.synapse_rows),
                           "ticks_per_step": 16, "delays_ms": "1-16 folded into 1-8 (reference ABI limit)",
                           "kernel": fm["kernel"]},
                "e2e": {"value": fm["e2e_value"], "unit": UNIT,
                        "h2d_bytes_per_step": fm.get("h2d_bytes_per_step", 0),
                        "d2h_bytes_per_step": fm.get("d2h_bytes_per_step", 16)},
                "clocks": fm["clocks"]}
        print(json.dumps(line), flush=True)
    for n in notes:
        print(json.dumps({"impl": "reference-cuda", "unavailable": n}), flush=True)


def device_rate(nsb, batch, steps, warmup, gpu_index):
    """One batch stepped device-resident from a captured CUDA graph after the
    per-bucket autotuner, timed with CUDA events on the launching stream:
    ms per step, neuron-ticks/s, synaptic events/s, the bucket plan and the
    clocks seen."""
    import torch
    gpu = nsb.GpuBatch.from_rows(batch)
    try:
        if "pulse_period" in batch.meta:
            gpu.set_modulation(batch.meta["pulse_period"], batch.meta["pulse_mod"])
        gpu.reset(np.arange(batch.brains, dtype=np.uint32))
        gpu.upload(batch.inputs, np.ones(batch.brains, np.uint8))
        stream = torch.cuda.Stream()
        s = stream.cuda_stream
        for _ in range(5):                 # the autotuner sees running activity, not the reset
            gpu.step_graph(16, batch.gain, s)
        gpu.autotune(16, batch.gain, s)
        torch.cuda.synchronize()
        for _ in range(max(warmup, 3)):
            gpu.step_graph(16, batch.gain, s)
        torch.cuda.synchronize()
        gpu.take_events()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with ClockSampler(gpu_index) as clk:
            e0.record(stream)
            for _ in range(steps):
                gpu.step_graph(16, batch.gain, s)
            e1.record(stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        events = gpu.take_events()
        plan = [{k: b[k] for k in ("name", "units", "block", "cooperative", "cluster", "meta_cap", "list")}
                for b in gpu.buckets() if b["units"]]
    finally:
        gpu.close()
    N = len(batch.neuron_rows)
    return {"ms_per_step": ms / steps, "value": N * 16 * steps / (ms / 1e3), "unit": UNIT,
            "synaptic_events_per_s": events / (ms / 1e3), "neurons": N, "synapses": len(batch.synapse_rows),
            "brains": batch.brains, "steps": steps, "warmup": max(warmup, 3), "plan": plan, "clocks": clk.summary()}


def run_ours(args, rank, world, local_rank):
    import torch
    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    nsb = load_package()
    if args.strong and world > 1:
        # strong scaling: one population split across the ranks by neurons + synapses
        full = workload(nsb, 2, args.fraction, args.workload)
        lo, hi = nsb.sharding.shard_ranges(full.neuron_offsets, full.synapse_offsets, world)[rank]
        batch = full.subset(range(lo, hi))
        total_neurons = len(full.neuron_rows)
        del full
    else:
        batch = workload(nsb, 2 + rank, args.fraction, args.workload)
        total_neurons = world * len(batch.neuron_rows)
    N = len(batch.neuron_rows)
    E = len(batch.synapse_rows)
    gpu = nsb.GpuBatch.from_rows(batch)
    if "pulse_period" in batch.meta:
        gpu.set_modulation(batch.meta["pulse_period"], batch.meta["pulse_mod"])
    st = gpu.stats()
    gpu.reset(np.arange(batch.brains, dtype=np.uint32) + 1000 * rank)
    gpu.upload(batch.inputs, np.ones(batch.brains, np.uint8))
    stream = torch.cuda.Stream()
    s = stream.cuda_stream
    # Per-bucket autotune (untimed; state restored afterwards), after a few
    # steps so that it sees the population's running activity, not its reset.
    if not args.no_autotune:
        for _ in range(5):
            gpu.step_graph(16, batch.gain, s)
        torch.cuda.synchronize()
    coop = gpu.autotune(16, batch.gain, s) if not args.no_autotune else gpu.buckets()[3]["cooperative"] != 0
    torch.cuda.synchronize()
    plan = [{k: b[k] for k in ("name", "units", "max_neurons", "block", "cooperative", "cluster", "meta_cap", "list",
                               "grid")}
            for b in gpu.buckets() if b["units"]]
    for _ in range(max(args.warmup, 3)):
        gpu.step_graph(16, batch.gain, s)
    torch.cuda.synchronize()
    gpu.take_events()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        torch.cuda.nvtx.range_push("timed")       # profiler captures: ncu --nvtx --nvtx-include timed/
        e0.record(stream)
        for _ in range(args.steps):
            gpu.step_graph(16, batch.gain, s)
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = e0.elapsed_time(e1)
    events = gpu.take_events()
    if dist:
        ms = nsb.sharding.max_over_ranks(ms, dist, "cuda")
        events = nsb.sharding.sum_over_ranks(events, dist, "cuda")
        dist.barrier()
    ms_step = ms / args.steps
    value = total_neurons * 16 * args.steps / (ms / 1e3)
    events_per_s = events / (ms / 1e3)
    launches_per_step = len(plan)          # one tick-kernel launch per non-empty bucket

    # e2e: reference-facing C ABI call with pinned host buffers
    inp = torch.from_numpy(batch.inputs).pin_memory()
    msk = torch.ones(batch.brains, dtype=torch.uint8).pin_memory()
    out = torch.zeros((batch.brains, batch.outputs), dtype=torch.float32).pin_memory()
    stat = torch.zeros(batch.brains, dtype=torch.int32).pin_memory()
    import ctypes as ct
    lib = nsb.native.library()
    f = ct.POINTER(ct.c_float)

    def abi_step():
        rc = lib.ns_gpu_step(gpu.ptr, ct.cast(inp.data_ptr(), f), ct.cast(msk.data_ptr(), ct.POINTER(ct.c_uint8)), 16,
                             batch.gain, ct.cast(out.data_ptr(), f), ct.cast(stat.data_ptr(), ct.POINTER(ct.c_int)))
        if rc:
            raise RuntimeError(lib.ns_error().decode())
    for _ in range(2):
        abi_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_steps = max(args.steps // 2, 3)
    for _ in range(e2e_steps):
        abi_step()
    e2e_s = time.perf_counter() - t0
    if dist:
        e2e_s = nsb.sharding.max_over_ranks(e2e_s, dist, "cuda")
    e2e_value = total_neurons * 16 * e2e_steps / e2e_s
    h2d = batch.inputs.nbytes + batch.brains
    d2h = out.numel() * 4 + stat.numel() * 4

    if rank == 0:
        peak, peak_kind = peaks()
        algo = ALGO_BYTES_PER_NEURON * N + ALGO_BYTES_PER_SYNAPSE * E
        achieved = algo / (ms_step / 1e3) / 1e9
        traffic = traffic_per_step() if args.workload == "batched_uneven" else None
        if traffic is not None:
            traffic /= args.fraction
        clocks = clk.summary()
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True,
                "scaling": "strong" if args.strong and world > 1 else "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (Philox4x32-10, seed 2 + rank)",
                "config": {"workload": ("plain_small_64x48" if args.workload == "plain_small" else
                                        "lp_prinz_smoke_4_brains" if args.workload == "heavy_smoke" else
                                        "heavy_world_founders_256" if args.workload == "heavy_founders" else
                                        f"{args.workload}_full_pools" if args.fraction == 1 else
                                        f"{args.workload}_1/{args.fraction}_pools"), "brains": batch.brains, "neurons": N,
                           "synapses": E, "ticks_per_step": 16, "delays_ms": f"1-{batch.max_delay}",
                           "parallelism": (f"shards x{world}" if args.strong and world > 1 else f"replicas x{world}"),
                           "units": st["units"], "grid": st["grid"], "block": st["block"],
                           "delivery": "warp-cooperative" if coop else "serial",
                           "plan": plan,
                           "l2": (f"device state {(120 * N + 108 * E) / 1e9:.2f} GB > 126 MB L2: inputs larger than L2"
                                  if 120 * N + 108 * E > 126e6 else
                                  f"device state {(120 * N + 108 * E) / 1e6:.1f} MB, L2-resident (not flushed)")},
                "synaptic_events_per_s": events_per_s,
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                             "algorithmic_bytes_per_launch": algo},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
                "gpu_launches": launches_per_step * args.steps,
                "clocks": clocks}
        wi = warp_instructions_per_neuron_tick()
        if wi is not None and clocks and args.workload == "batched_uneven":
            # Issue roofline: the kernel is bound by instruction issue, not HBM.
            # Peak = SMs x 4 schedulers x one warp instruction per cycle at the SM clock seen.
            sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
            peak_issue = sms * 4 * clocks["sm_mhz"] * 1e6
            line["roofline_issue"] = {"bound": "issue", "warp_inst_per_neuron_tick": wi,
                                      "achieved": wi * value / world / 1e9, "peak": peak_issue / 1e9,
                                      "unit": "G warp-instructions/s", "frac": wi * value / world / peak_issue,
                                      "source": "profiles/tick_kernel_list_div8_full_set.md (ncu, 1/8 slice)"}
        if not args.no_cpu_baseline:
            ref = CpuReference(batch, 8, os.cpu_count() or 1)
            ref.step(16)
            nt, secs = 0, 0.0
            for _ in range(2):
                a, b = ref.step(16)
                nt += a; secs += b
            ref.close()
            line["cpu_baseline"] = {"value": nt / secs, "unit": UNIT, "cores": ref.processes, "kind": ref.kind,
                                    "sample": ref.sample + "; 2 timed steps after 1 warm-up"}
    gpu.close()
    if rank == 0 and world == 1 and not args.no_other_configs and args.fraction == 1 \
            and args.workload == "batched_uneven":
        # The other configurations of the same metric, device-resident, in the same run:
        # plasticity-heavy full pools (every synapse triplet STDP + dopamine
        # eligibility, 30 % bursting, pulses every 50 ms) and the plain small
        # batch (64 brains x 48 neurons, 600 synapses each).
        line["other_configs"] = {
            "plasticity_heavy_full_pools": device_rate(nsb, workload(nsb, 2, 1, "plasticity_heavy"), 10, 3,
                                                       local_rank),
            "plain_small_64x48": device_rate(nsb, workload(nsb, 2, 1, "plain_small"), 50, 5, local_rank),
            "lp_prinz_smoke_4_brains": device_rate(nsb, workload(nsb, 2, 1, "heavy_smoke"), 20, 3, local_rank)}
    if rank == 0:
        if (world == 1 and not args.no_reference_cuda and args.fraction == 1
                and args.workload in SMALL_OR_MAIN):
            # The reference's own CUDA forms on the same batch and GPU, after
            # this library's buffers are freed (none of its code runs there).
            torch.cuda.synchronize()
            forms, notes = reference_cuda_forms(batch, max(3, min(args.steps, 20)), args.warmup, local_rank)
            rc = {k: {"ms_per_step": v["ms_per_step"], "value": v["value"], "e2e_value": v["e2e_value"],
                      "kernel": v["kernel"], "steps": v["steps"], "clocks": v["clocks"]} for k, v in forms.items()}
            if forms:
                best = min(forms, key=lambda k: forms[k]["ms_per_step"])
                rc["best_form"] = best
                rc["best_ms_per_step"] = forms[best]["ms_per_step"]
                rc["best_ratio"] = value / forms[best]["value"]
                rc["best_e2e_ratio"] = e2e_value / max(v["e2e_value"] for v in forms.values())
            rc["delays"] = "folded into 1-8 for the reference (its ABI accepts 1-8); cost per tick is delay-independent"
            if notes:
                rc["unavailable"] = notes
            line["reference_cuda"] = rc
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_serve(args, rank, world, local_rank):
    """Serving loop (config 5): genome-evaluation episodes on the pole-on-cart
    environment. Phases:
      1. saturation: a backlog larger than the in-flight cap; peak batched
         throughput = neuron-ticks launched per second over the last
         `serve_seconds / 2` seconds, in episodes/s through the mean episode
         work of the request mix;
      2. open loop at --serve-load x peak (Poisson), then drain: p50/p99
         latency (arrival -> result) of the requests that arrived after the
         first quarter of the window, and the achieved fraction of peak;
      3. open loop at --serve-rate (the configured 2,000 requests/s) for the
         same window: what completes, at what latency, and the backlog left.
    """
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local_rank)
    nsb = load_package()
    W = nsb.workloads
    lib = W.serving_library(seed=5, genomes=args.serve_genomes)
    sizes = np.diff(lib.neuron_offsets).astype(np.float64)
    mean_steps = (200 + 2000) / 2.0
    work_per_episode = sizes.mean() * mean_steps * 16      # neuron-ticks, library drawn uniformly

    def server():
        srv = nsb.Server(max_inflight_neurons=args.serve_cap, hbm_budget_bytes=150e9)
        ids = np.array(srv.register_batch(lib), np.int32)
        return srv, ids

    def wait(srv, until, results):
        while srv.now() < until:
            time.sleep(0.2)
            results.append(srv.poll())

    T = args.serve_seconds
    # 1. saturation
    srv, ids = server()
    n = int(max(20000, 3 * args.serve_cap / sizes.mean(), 1000 * T))   # outlasts the window at any rate seen
    sched = W.serving_schedule(11, 1e6, n / 1e6, len(ids))
    srv.submit(ids[sched["genome"]], sched["seed"], sched["steps"], tag=sched["tag"], arrival=0.0)
    srv.start()
    res = []
    wait(srv, T / 2, res)
    a = srv.stats()
    wait(srv, T, res)
    b = srv.stats()
    srv.stop()
    srv.close()
    peak_nt = (b["neuron_ticks_launched"] - a["neuron_ticks_launched"]) / (b["elapsed_s"] - a["elapsed_s"])
    peak_eps = peak_nt / work_per_episode
    peak_events = (b["events"] - a["events"]) / (b["elapsed_s"] - a["elapsed_s"])

    def open_loop(rate, drain):
        srv, ids = server()
        sch = W.serving_schedule(13, rate, T, len(ids))
        t0 = srv.now() + 0.5
        srv.submit(ids[sch["genome"]], sch["seed"], sch["steps"], tag=sch["tag"], arrival=sch["arrival"] + t0)
        srv.start()
        res = []
        wait(srv, t0 + T / 4, res)
        s0 = srv.stats()
        wait(srv, t0 + T, res)
        s1 = srv.stats()
        if drain:
            deadline = t0 + T + 120
            while srv.stats()["inflight"] + srv.stats()["queued"] > 0 and srv.now() < deadline:
                time.sleep(0.2)
                res.append(srv.poll())
        s2 = srv.stats()
        srv.stop()
        res.append(srv.poll_all())
        srv.close()
        r = np.concatenate(res)
        arr = r["arrival_s"] - t0
        window = r[(arr >= T / 4) & (arr < T)]
        lat = window["done_s"] - window["arrival_s"]
        nt = (s1["neuron_ticks_launched"] - s0["neuron_ticks_launched"]) / (s1["elapsed_s"] - s0["elapsed_s"])
        done_in_window = ((r["done_s"] - t0 >= T / 4) & (r["done_s"] - t0 < T)).sum()
        out = {"offered_per_s": rate, "arrived": int(len(sch["arrival"])), "completed": int(len(r)),
               "episodes_per_s": float(done_in_window / (0.75 * T)), "neuron_ticks_per_s": nt,
               "frac_of_peak": nt / peak_nt,
               "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
               "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
               "backlog_at_end": int(s1["queued"] + s1["inflight"]),
               "nonfinite": int((r["status"] != 0).sum())}
        if len(lat):
            out["p99_over_p50"] = out["p99_s"] / out["p50_s"]
        if not drain:
            out["note"] = "latency of requests completed within the window only (overloaded: the rest are queued)"
        return out

    loaded = open_loop(args.serve_load * peak_eps, drain=True)
    configured = open_loop(args.serve_rate, drain=False)
    line = {"metric": "p99 episode latency, serving loop at the measured load", "value": loaded["p99_s"],
            "unit": "s", "n_gpus": 1, "higher_is_better": False, "vs_baseline": None, "dtype": "f32",
            "data": f"synthetic (Philox4x32-10): {len(ids)} genomes, N log-uniform 32-4096, 8 synapses/neuron; "
                    "Poisson arrivals, episodes U[200, 2000] steps",
            "config": {"workload": "serving_cartpole_episodes", "inflight_cap_neurons": args.serve_cap,
                       "hbm_budget_bytes": 150e9, "window_s": T, "ticks_per_step": 16,
                       "mean_episode_neuron_ticks": work_per_episode},
            "peak": {"neuron_ticks_per_s": peak_nt, "episodes_per_s": peak_eps, "synaptic_events_per_s": peak_events,
                     "busy_frac": (b["busy_s"] - a["busy_s"]) / (b["elapsed_s"] - a["elapsed_s"]),
                     "queued_at_window_end": int(b["queued"])},
            "at_load": loaded, "at_configured_rate": configured}
    print(json.dumps(line), flush=True)


def world_population(nsb, population, founders=2048, compact=False, scatter=None, heavy=False):
    """World pools at the reference build's capacities (32,768 animals,
    4,194,304 neuron and 8,388,608 synapse slots). "founders": 2,048 founders
    of 32-96 neurons with 4-12 synapses per neuron (config 2; with `heavy`,
    3 % each of the hidden excitatory neurons are LP, Prinz and LFS cells, as
    mutation makes them, so nearly every animal carries one); "full": the
    full-pool batched-uneven population as animals (delays folded into the
    world's 1-8 ms ring, its 8 input channels as world senses 0-7)."""
    W = nsb.world
    if population == "founders":
        batch = nsb.workloads.world_founders(seed=2, founders=founders, heavy_types=heavy)
    else:
        full = workload(nsb, 2)
        sr = full.synapse_rows.copy()
        sr[:, 4] = (sr[:, 4] - 1) % 8 + 1
        senses = np.zeros((full.brains, 19), np.float32)
        senses[:, :full.channels] = full.inputs
        batch = nsb.workloads.Batch(full.neuron_rows, sr, full.neuron_offsets, full.synapse_offsets, full.motors, 19,
                                    8, "batched_uneven_world", senses, 230.0, {})
    recs = W.records_from_gpu(batch, np.arange(batch.brains, dtype=np.uint32) + 1)
    if compact:     # pools sized to the population (profiler captures; the reference needs its full capacities)
        N, E = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1])
        pools = W.place_population(batch, *recs, animal_capacity=batch.brains + 64, neuron_capacity=N + 4096,
                                   synapse_capacity=E + 8192)
    else:
        pools = W.place_population(batch, *recs, animal_capacity=32768, neuron_capacity=4194304,
                                   synapse_capacity=8388608, scatter_seed=scatter)
    return batch, pools


def run_world_stage(args, rank, world, local_rank):
    """The world simulator's neural stage on world pools through
    nsb_world_neural_step + nsb_world_homeostasis, then the reference's own
    world kernels (src/main.cu, the world binary's flags) on the same pools.
    Rank 0 only (one GPU)."""
    import ctypes as ct
    import torch
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    sys.path.insert(0, str(ROOT))
    nsb = load_package()
    W = nsb.world
    batch, pools = world_population(nsb, args.world_population, args.world_founders, args.world_compact,
                                    heavy=args.world_heavy)
    N, E, B = int(batch.neuron_offsets[-1]), int(batch.synapse_offsets[-1]), batch.brains
    stage = W.World(pools)
    counter = [0]

    def run(k):
        for _ in range(k):
            counter[0] += 1
            stage.neural_step(counter[0])
            stage.homeostasis()
    t0 = time.perf_counter()
    run(1)
    first_step_s = time.perf_counter() - t0          # includes compiling every brain on the device
    run(max(args.warmup, 3) - 1)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clk:
        t0 = time.perf_counter()
        e0.record()
        run(args.steps)
        e1.record()
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1) / args.steps
    st = stage.stats()
    stage.close()
    del stage
    torch.cuda.empty_cache()
    value = N * 16 / (ms / 1e3)
    peak, peak_kind = peaks()
    algo = ALGO_BYTES_PER_NEURON * N + ALGO_BYTES_PER_SYNAPSE * E
    achieved = algo / (ms / 1e3) / 1e9
    line = {"metric": "neuron-ticks/s of the world neural stage", "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (Philox4x32-10, seed 2)",
            "config": {"workload": (f"world_founders_{B}" if args.world_population == "founders" else "world_full"),
                       "animals": B, "neurons": N, "synapses": E,
                       "ticks_per_step": 16, "delays_ms": "1-8",
                       "pools": ("reference layouts sized to the population" if args.world_compact else
                                 "reference layouts at the reference capacities (32,768 / 4,194,304 / 8,388,608)"),
                       "step": "nsb_world_neural_step + nsb_world_homeostasis (5 kernels, one host sync)",
                       "first_step_s_with_compile": first_step_s,
                       "l2": f"pools touched per step {(364 * N + 200 * E) / 1e9:.2f} GB"},
            "synaptic_events_per_s": st["events"] / (ms / 1e3),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_kind, "algorithmic_bytes_per_launch": algo},
            "e2e": {"value": N * 16 * args.steps / wall, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 72},
            "gpu_launches": 5 * args.steps,
            "clocks": clk.summary()}
    if not args.no_cpu_baseline:
        from oracle import pyoracle
        sub = batch.subset(range(0, B, max(1, B // 64)))
        sp = W.place_population(sub, *W.records_from_gpu(sub, np.arange(sub.brains, dtype=np.uint32) + 1))
        pyoracle.world_step(sp, 1)
        t0 = time.perf_counter()
        for k in (2, 3):
            pyoracle.world_step(sp, k)
            pyoracle.world_homeostasis(sp)
        secs = time.perf_counter() - t0
        n_sub = int(sub.neuron_offsets[-1])
        line["cpu_baseline"] = {"value": n_sub * 16 * 2 / secs, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"{sub.brains} of {B} animals ({n_sub} neurons), oracle world "
                                          f"restatement, 2 steps after 1"}
    print(json.dumps(line), flush=True)

    if args.world_compact:
        return
    # the reference's world kernels on the same initial pools
    from oracle import pyoracle
    wlib = pyoracle.ref_world_lib()
    if wlib is None or not hasattr(wlib, "ref_world_pools_create"):
        print(json.dumps({"impl": "reference-cuda-world", "unavailable": "oracle/_ref/libns_ref_world.so not built"}))
        return
    wlib.ref_world_pools_create.restype = ct.c_void_p
    wlib.ref_world_pools_create.argtypes = [ct.c_void_p, ct.c_int]
    wlib.ref_world_pools_step.argtypes = [ct.c_void_p, ct.c_longlong]
    wlib.ref_world_pools_homeostasis.argtypes = [ct.c_void_p]
    wlib.ref_world_pools_destroy.argtypes = [ct.c_void_p]
    for mode, label in ((0, "fused global-slot kernels"), (1, "--block-brains tiers + global-slot fallback")):
        dev = {}
        stc = W.NsbWorldPools()
        for n in W.ARRAYS:
            a = getattr(pools, n)
            dev[n] = None if a is None else torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1)).cuda()
            setattr(stc, n, None if dev[n] is None else dev[n].data_ptr())
        stc.trace_animal, stc.silence_senses, stc.silence_contact = -1, 0, 0
        stc.animal_capacity, stc.neuron_capacity, stc.synapse_capacity = pools.capacities
        h = wlib.ref_world_pools_create(ct.byref(stc), mode)
        if not h:
            print(json.dumps({"impl": "reference-cuda-world", "unavailable": "pool setup failed"}))
            continue
        k = 0
        for _ in range(max(args.warmup, 3)):
            k += 1
            wlib.ref_world_pools_step(h, k)
            wlib.ref_world_pools_homeostasis(h)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record()
        for _ in range(args.steps):
            k += 1
            wlib.ref_world_pools_step(h, k)
            wlib.ref_world_pools_homeostasis(h)
        e1.record()
        torch.cuda.synchronize()
        rwall = time.perf_counter() - t0
        rms = e0.elapsed_time(e1) / args.steps
        wlib.ref_world_pools_destroy(h)
        del dev
        torch.cuda.empty_cache()
        ref_line = {"impl": "reference-cuda-world", "metric": line["metric"], "value": N * 16 / (rms / 1e3),
                    "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": rms,
                    "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                    "data": line["data"],
                    "config": dict(line["config"], kernel=f"src/main.cu neural stage, {label}, --use_fast_math, "
                                                          f"sm_100a", step="selection + 16 ticks + homeostasis"),
                    "e2e": {"value": N * 16 * args.steps / rwall, "unit": UNIT, "h2d_bytes_per_step": 0,
                            "d2h_bytes_per_step": 16}}
        ref_line["config"].pop("first_step_s_with_compile", None)
        print(json.dumps(ref_line), flush=True)


def run_world_loop(args, rank, world, local_rank):
    """The world step in the reference host loop's order (src/main.cu:2634-2770):
    neural stage, body step with spatial index, bites and predation deaths,
    homeostasis, genome reclamation, reproduction with mutation, regrowth and
    senses, closed loop (each step's senses drive the next; cohort
    observation, an observer, is left out). This library's stages,
    then the reference's own kernels (the world binary's flags, launched as
    its host loop launches them) on the same initial pools. Rank 0 only."""
    import ctypes as ct
    import torch
    if rank != 0:
        return
    torch.cuda.set_device(local_rank)
    sys.path.insert(0, str(ROOT))
    nsb = load_package()
    W = nsb.world
    # slots spread over the pools, as the simulator's hinted claims spread them
    # (init_animals, src/main.cu:547-611); packed slots would make every
    # claim_slot scan long runs of full bitmap words
    batch, pools = world_population(nsb, args.world_population, args.world_founders, False, scatter=3,
                                    heavy=args.world_heavy)
    W.place_bodies(pools, 3)
    if args.world_parents > 0:                    # a fraction of well-fed animals: births every step
        live = np.nonzero(pools.animals["alive"] == 1)[0]
        pools.animals["energy"][live[:int(len(live) * args.world_parents)]] = 200.0
    seed, renewal = 2, 0.0006                     # the simulator's defaults (src/main.cu:1937)
    eco = W.make_ecology(pools, seed=seed, initial_count=batch.brains, life_capacity=32768 * 16)
    B = batch.brains
    warm = max(args.warmup, 3)

    def timed(step_fn, label):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e = [None, torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)]
        k = 0
        for _ in range(warm):
            k += 1
            step_fn(k, None)
        torch.cuda.synchronize()
        eco_ms = 0.0
        neurons = 0
        with ClockSampler(local_rank) as clk:
            start.record()
            for _ in range(args.steps):
                k += 1
                neurons += step_fn(k, e)
                eco_ms += e[1].elapsed_time(e[2])
            end.record()
            torch.cuda.synchronize()
        return start.elapsed_time(end) / args.steps, eco_ms / args.steps, neurons, clk.summary()

    def live_neurons(p):
        A = p.animals
        return int(A["neuron_count"][A["alive"] == 1].sum())

    # ---- this library
    stage = W.World(pools)
    stage.attach_ecology(eco)
    stage.regrow_and_sense(0, seed, 0.0)
    alive_n = [live_neurons(pools)]

    def ours(k, ev):
        stage.neural_step(k)
        if ev:
            ev[1].record()
        stage.body_step(k)
        stage.homeostasis()
        stage.reclaim(k)
        stage.reproduce()
        stage.regrow_and_sense(k, seed, renewal)
        if ev:
            ev[2].record()
            ev[2].synchronize()
        n = stage.stats()["neurons"]
        return n

    ms, eco_ms, neuron_steps, clk = timed(ours, "ours")
    fin = stage.download_ecology()
    stage.close()
    del stage
    torch.cuda.empty_cache()
    line = {"metric": "neuron-ticks/s of the world step (neural stage + ecology)",
            "value": neuron_steps * 16 / (ms * args.steps / 1e3), "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (Philox4x32-10, seed 2); food grid of init_world seed 2",
            "config": {"workload": f"world_loop_founders_{B}" if args.world_population == "founders"
                       else "world_loop_full", "animals": B, "neurons_at_start": alive_n[0],
                       "food_renewal": renewal,
                       "pools": "reference capacities (32,768 / 4,194,304 / 8,388,608), slots scattered",
                       "well_fed_fraction": args.world_parents,
                       "step": "neural_step, body_step, homeostasis, reclaim, reproduce, regrow_and_sense (5 host syncs)"},
            "ecology_ms_per_step": eco_ms,
            "world_counts": {"deaths": int(fin.deaths[0]), "bites": int(fin.bites[0]),
                             "life_records": int(fin.life_count[0]), "births": int(fin.births[0])},
            "clocks": clk}
    print(json.dumps(line), flush=True)

    # ---- the reference's kernels on the same initial pools
    from oracle import pyoracle
    wlib = pyoracle.ref_world_lib()
    if wlib is None or not hasattr(wlib, "ref_world_eco_create"):
        print(json.dumps({"impl": "reference-cuda-world-loop", "unavailable": "oracle/_ref/libns_ref_world.so not built"}))
        return
    wlib.ref_world_pools_create.restype = ct.c_void_p
    wlib.ref_world_pools_create.argtypes = [ct.c_void_p, ct.c_int]
    wlib.ref_world_pools_step.argtypes = [ct.c_void_p, ct.c_longlong]
    wlib.ref_world_pools_homeostasis.argtypes = [ct.c_void_p]
    wlib.ref_world_pools_destroy.argtypes = [ct.c_void_p]
    wlib.ref_world_eco_create.restype = ct.c_void_p
    wlib.ref_world_eco_create.argtypes = [ct.c_void_p, ct.c_void_p]
    wlib.ref_world_eco_body.argtypes = [ct.c_void_p, ct.c_longlong, ct.c_int]
    wlib.ref_world_eco_reclaim.argtypes = [ct.c_void_p, ct.c_longlong, ct.c_int]
    wlib.ref_world_eco_regrow_and_sense.argtypes = [ct.c_void_p, ct.c_longlong, ct.c_ulonglong, ct.c_float,
                                                    ct.c_int]
    wlib.ref_world_eco_destroy.argtypes = [ct.c_void_p]
    wlib.ref_world_eco_reproduce.argtypes = [ct.c_void_p, ct.c_int]
    for mode, label in ((0, "fused global-slot kernels"), (1, "--block-brains tiers + global-slot fallback")):
        holder = W.World(pools)          # device copies of the pools and ecology, in the shared layouts
        holder.attach_ecology(eco)
        h = wlib.ref_world_pools_create(ct.byref(holder.struct), mode)
        x = wlib.ref_world_eco_create(ct.byref(holder.struct), ct.byref(holder.eco_struct))
        if not h or not x:
            print(json.dumps({"impl": "reference-cuda-world-loop", "unavailable": "pool setup failed"}))
            holder.close()
            continue
        wlib.ref_world_eco_regrow_and_sense(x, 0, seed, 0.0, 0)

        def theirs(k, ev):
            wlib.ref_world_pools_step(h, k)
            if ev:
                ev[1].record()
            wlib.ref_world_eco_body(x, k, 0)
            wlib.ref_world_pools_homeostasis(h)
            wlib.ref_world_eco_reclaim(x, k, 0)
            wlib.ref_world_eco_reproduce(x, 0)
            wlib.ref_world_eco_regrow_and_sense(x, k, seed, renewal, 0)
            if ev:
                ev[2].record()
                ev[2].synchronize()
            return 0

        rms, reco_ms, _, rclk = timed(theirs, label)
        wlib.ref_world_eco_destroy(x)
        wlib.ref_world_pools_destroy(h)
        holder.close()
        del holder
        torch.cuda.empty_cache()
        print(json.dumps({"impl": "reference-cuda-world-loop", "metric": "ms per world step (neural stage + "
                          "ecology)", "value": rms, "unit": "ms", "higher_is_better": False,
                          "steps": args.steps, "warmup": warm, "ecology_ms_per_step": reco_ms,
                          "ours_ms_per_step": ms, "ours_ecology_ms_per_step": eco_ms,
                          "config": dict(line["config"], kernel=f"src/main.cu, {label}, --use_fast_math, sm_100a"),
                          "clocks": rclk}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-cuda"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default bucket configurations (profiler captures: fewer launches before the timed ones)")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the plasticity-heavy and plain-small lines of the default run (N=1 only)")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip timing the reference's own CUDA forms on the same batch (N=1 only)")
    ap.add_argument("--fraction", type=int, default=1, choices=[1, 2, 4, 8, 16],
                    help="run a 1/D slice of the full pools (profiler captures only)")
    ap.add_argument("--workload", default="batched_uneven",
                    choices=["batched_uneven", "plasticity_heavy", "serving_population", "plain_small", "heavy_smoke",
                             "heavy_founders"],
                    help="full-pool workload: batched uneven brains (default) or the plasticity-heavy variant")
    ap.add_argument("--strong", action="store_true",
                    help="N > 1: split one full-pool population across the ranks (default: one replica per rank)")
    ap.add_argument("--serve", action="store_true", help="serving-loop latency/throughput (config 5)")
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-load", type=float, default=0.85, help="offered load as a fraction of peak")
    ap.add_argument("--serve-rate", type=float, default=2000.0, help="configured arrival rate (requests/s)")
    ap.add_argument("--serve-cap", type=int, default=4194304, help="neurons in flight")
    ap.add_argument("--serve-genomes", type=int, default=512)
    ap.add_argument("--world", action="store_true",
                    help="the world simulator's neural stage on its own pools (config 2)")
    ap.add_argument("--world-population", default="founders", choices=["founders", "full"])
    ap.add_argument("--world-founders", type=int, default=2048, help="founders of the config-2 population")
    ap.add_argument("--world-compact", action="store_true",
                    help="pools sized to the population, no reference leg (profiler captures)")
    ap.add_argument("--world-parents", type=float, default=0.0,
                    help="--world-loop: fraction of founders given energy 200 (they reproduce every step)")
    ap.add_argument("--world-heavy", action="store_true",
                    help="--world / --world-loop founders with LP, Prinz and LFS cells (3 %% each of hidden cells)")
    ap.add_argument("--world-loop", action="store_true",
                    help="the world step: neural stage + ecology with reproduction, closed loop")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus if "RANK" in os.environ else 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.serve:
        run_serve(args, rank, world, local_rank)
    elif args.world_loop:
        run_world_loop(args, rank, world, local_rank)
    elif args.world:
        run_world_stage(args, rank, world, local_rank)
    elif args.impl == "reference":
        run_reference(args, rank, world)
    elif args.impl == "reference-cuda":
        run_reference_cuda(args, rank, world, local_rank)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
