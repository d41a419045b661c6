"""Serving loop for genome-evaluation episodes (nsb_serve_* in libns_b200.so).

Each request is one episode: a registered genome controls the pole-on-cart
environment for a given number of steps (16 neural ticks per 20 ms
environment step), starting from its seed. The server admits requests as
they arrive, first come first served, while the neurons in flight stay under
an in-flight cap and the bytes of admitted episodes under an HBM budget;
admitted episodes keep their neural and environment state on the device and
are batched continuously into the persistent tick kernel. A result is the
same whatever else is in flight.

    srv = Server(max_inflight_neurons=4_194_304)
    ids = srv.register_batch(workloads.serving_library(genomes=512))
    srv.submit(genome, seed, steps, tag, arrival)   # arrival on srv.now()'s clock
    srv.start(); ...; results = srv.poll(); srv.stop()
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import native

RESULT_DTYPE = np.dtype([("tag", np.uint64), ("genome", np.int32), ("steps", np.int32), ("reward", np.int32),
                         ("failures", np.int32), ("trace", np.uint32), ("seed", np.uint32), ("status", np.int32),
                         ("pad", np.int32), ("arrival_s", np.float64), ("admit_s", np.float64),
                         ("done_s", np.float64)])
assert RESULT_DTYPE.itemsize == 64
STATS = ("steps", "admitted", "completed", "queued", "inflight", "inflight_neurons", "units", "neuron_ticks",
         "busy_s", "elapsed_s", "events", "pool_neurons", "pool_synapses", "pool_bytes", "inflight_bytes",
         "neuron_ticks_launched")


class Server:
    def __init__(self, max_inflight_neurons=4194304, hbm_budget_bytes=150e9, synapses_per_neuron=8.0,
                 max_slots=65536, max_brain_neurons=4096, ticks=16, gain=230.0, smoothing=0.4):
        self.lib = native.library()
        self.ptr = self.lib.nsb_serve_create(int(max_inflight_neurons), float(hbm_budget_bytes),
                                             float(synapses_per_neuron), int(max_slots), int(max_brain_neurons),
                                             int(ticks), float(gain), float(smoothing))
        if not self.ptr:
            raise RuntimeError(self.lib.ns_error().decode())
        self.ticks = ticks

    def _check(self, rc):
        if rc < 0:
            raise RuntimeError(self.lib.ns_error().decode())
        return rc

    def register(self, neuron_rows, synapse_rows, motors):
        ng = np.ascontiguousarray(neuron_rows, np.float32).reshape(-1, 10)
        sg = np.ascontiguousarray(synapse_rows, np.float32).reshape(-1, 11)
        mo = np.ascontiguousarray(motors, np.int32)
        sgp = sg if len(sg) else np.zeros((1, 11), np.float32)
        f = ct.POINTER(ct.c_float)
        return self._check(self.lib.nsb_serve_register(self.ptr, len(ng), len(sg), ng.ctypes.data_as(f),
                                                       sgp.ctypes.data_as(f),
                                                       mo.ctypes.data_as(ct.POINTER(ct.c_int))))

    def register_batch(self, batch):
        return [self.register(*batch.brain(i)) for i in range(batch.brains)]

    def submit(self, genome, seed, steps, tag=None, arrival=None):
        genome = np.ascontiguousarray(np.atleast_1d(genome), np.int32)
        n = len(genome)
        seed = np.ascontiguousarray(np.broadcast_to(np.asarray(seed, np.uint32), (n,)))
        steps = np.ascontiguousarray(np.broadcast_to(np.asarray(steps, np.int32), (n,)))
        tag = np.arange(n, dtype=np.uint64) if tag is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(tag, np.uint64), (n,)))
        arrival = np.full(n, self.now()) if arrival is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(arrival, np.float64), (n,)))
        self._check(self.lib.nsb_serve_submit(
            self.ptr, n, genome.ctypes.data_as(ct.POINTER(ct.c_int32)), seed.ctypes.data_as(ct.POINTER(ct.c_uint32)),
            steps.ctypes.data_as(ct.POINTER(ct.c_int32)), tag.ctypes.data_as(ct.POINTER(ct.c_uint64)),
            arrival.ctypes.data_as(ct.POINTER(ct.c_double))))

    def start(self):
        self._check(self.lib.nsb_serve_start(self.ptr))

    def stop(self):
        self._check(self.lib.nsb_serve_stop(self.ptr))

    def run(self, max_iterations=10**9):
        """Run the loop on this thread until nothing is queued or in flight."""
        self._check(self.lib.nsb_serve_run(self.ptr, int(max_iterations)))

    def poll(self, max_results=1 << 16):
        out = np.zeros(max_results, RESULT_DTYPE)
        n = self._check(self.lib.nsb_serve_poll(self.ptr, out.ctypes.data_as(ct.c_void_p), max_results))
        return out[:n]

    def poll_all(self):
        parts = []
        while True:
            r = self.poll()
            if len(r) == 0:
                break
            parts.append(r)
        return np.concatenate(parts) if parts else np.zeros(0, RESULT_DTYPE)

    def now(self):
        return self.lib.nsb_serve_now(self.ptr)

    def stats(self):
        v = np.zeros(len(STATS), np.float64)
        self._check(self.lib.nsb_serve_stats(self.ptr, v.ctypes.data_as(ct.POINTER(ct.c_double))))
        return dict(zip(STATS, v.tolist()))

    def close(self):
        if getattr(self, "ptr", None):
            self.lib.nsb_serve_destroy(self.ptr)
            self.ptr = None

    __del__ = close

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
