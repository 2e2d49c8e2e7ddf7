"""Continuous-batching Fock-build server on one GPU (Python face of the
native server, ``cqf_server_*`` in include/cqfock.h).

Requests (molecule, basis name, density) arrive at any time.  The native
server (csrc/cqf_server.cu)

* admits the oldest waiting request when an execution slot is free and its
  device-memory footprint (shell-pair data + contraction workspace,
  ``cqf_fock_footprint``, estimated before any allocation) fits in the budget
  that the running requests and the cached bases leave; idle cached bases are
  evicted (least recently used) to make room; no batch boundaries
  (continuous batching);
* runs every admitted request on its own worker thread and its basis' own
  CUDA stream, so the basis set-up and J/K kernels of different requests
  overlap on the device;
* keeps the device shell-pair data of recent geometries resident in HBM
  (LRU, counted in the budget), so repeated geometries (SCF iterations, RT
  steps) skip set-up.

This wrapper builds each request's basis from its molecule on a thread of
its own, submits it, waits (the C call releases the GIL) and resolves the
request's Future with G = 2 J[D] - K[D]; it records per-request latency
(completion - arrival) and phase times and reports p50 / p99.

Each request's result depends only on its own inputs: the kernels and the
work split are the same alone and in a mix (the only difference is the order
of floating-point atomics), which ``tests/test_gpu_serving.py`` checks.
"""
from __future__ import annotations

import ctypes as C
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Dict

import numpy as np

from . import _cabi
from .basis import BasisSet, Molecule
from .contraction import shell_array


@dataclass
class FockRequest:
    mol: Molecule
    basis: str
    D: np.ndarray
    precision: str = "mixed"
    fp32_cutoff: float = 1e-6
    arrival: float = 0.0            # perf_counter() time of arrival
    rid: int = 0
    future: Future = field(default_factory=Future)


def footprint_bytes(basis: BasisSet) -> int:
    """Device bytes the server charges a request of this basis
    (``cqf_fock_footprint``: shell-pair data, upper bound with every pair
    significant, plus the workspace of one J and one K)."""
    sh, _keep = shell_array(basis)
    return int(_cabi.lib().cqf_fock_footprint(sh, basis.nshell))


class FockServer:
    def __init__(self, device: int = 0, slots: int = 8,
                 mem_budget: int = 8 << 30, cache_entries: int = 16):
        L = _cabi.lib()
        o = _cabi.CqfServerOpts()
        L.cqf_server_opts_default(C.byref(o))
        o.device, o.slots = device, slots
        o.mem_budget, o.cache_entries = int(mem_budget), cache_entries
        h = C.c_void_p()
        _cabi.check(L.cqf_server_create(C.byref(o), C.byref(h)))
        self._h = h
        self._lock = threading.Lock()
        self._threads = []
        self.latencies: Dict[int, float] = {}
        # per request: (prep, queue, set-up, build) in seconds; prep = basis
        # construction on the host before submission
        self.phases: Dict[int, tuple] = {}

    # ------------------------------------------------------------ public
    def submit(self, req: FockRequest) -> Future:
        if not req.arrival:
            req.arrival = time.perf_counter()
        t = threading.Thread(target=self._serve, args=(req,), daemon=True)
        with self._lock:
            self._threads.append(t)
        t.start()
        return req.future

    def close(self):
        with self._lock:
            threads = list(self._threads)
        for t in threads:
            t.join()
        if self._h:
            _cabi.lib().cqf_server_destroy(self._h)
            self._h = None

    def stats(self):
        lat = np.array(list(self.latencies.values()))
        if len(lat) == 0:
            return {}
        st = _cabi.CqfServerStats()
        _cabi.check(_cabi.lib().cqf_server_get_stats(self._h, C.byref(st)))
        out = {"completed": len(lat), "failed": int(st.failed),
               "peak_inflight": int(st.peak_inflight),
               "p50_ms": float(np.percentile(lat, 50) * 1e3),
               "p99_ms": float(np.percentile(lat, 99) * 1e3),
               "mean_ms": float(lat.mean() * 1e3)}
        ph = np.array(list(self.phases.values())) * 1e3
        for i, name in enumerate(("prep", "queue", "setup", "build")):
            out[name + "_ms"] = {"p50": float(np.percentile(ph[:, i], 50)),
                                 "p99": float(np.percentile(ph[:, i], 99)),
                                 "mean": float(ph[:, i].mean())}
        return out

    # ------------------------------------------------------------ internals
    def _serve(self, req: FockRequest):
        try:
            L = _cabi.lib()
            basis = BasisSet.build(req.mol, req.basis)
            sh, keep = shell_array(basis)
            N = basis.nbasis
            D = np.asfortranarray(req.D, dtype=np.float64)
            if D.shape != (N, N):
                raise ValueError("density shape does not match the basis")
            G = np.zeros((N, N), order="F")
            dp = C.POINTER(C.c_double)
            q = _cabi.CqfFockRequest(sh, basis.nshell, 1e-12, D.ctypes.data_as(dp),
                                     G.ctypes.data_as(dp), 1.0,
                                     _cabi.CQF_MIXED if req.precision == "mixed"
                                     else _cabi.CQF_FP64, float(req.fp32_cutoff))
            t_sub = time.perf_counter()
            rid = C.c_longlong()
            _cabi.check(L.cqf_server_submit(self._h, C.byref(q), C.byref(rid)))
            info = _cabi.CqfRequestInfo()
            _cabi.check(L.cqf_server_wait(self._h, rid.value, -1.0, C.byref(info)))
            done = time.perf_counter()
            del keep
            with self._lock:
                self.latencies[req.rid] = done - req.arrival
                self.phases[req.rid] = (t_sub - req.arrival, info.queue_ms / 1e3,
                                        info.setup_ms / 1e3, info.build_ms / 1e3)
            req.future.set_result(G)
        except BaseException as e:  # report to the caller, keep serving
            req.future.set_exception(e)


def poisson_stream(n: int, rate_hz: float, seed: int = 5, max_waters: int = 32):
    """The serving workload: n requests, Poisson arrival offsets (s), water
    clusters of U{1..max_waters} molecules, cc-pVDZ or def2-SVP (50/50), each
    with its own seeded cluster and occupied-orbital density seed."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate_hz)
        nw = int(rng.integers(1, max_waters + 1))
        bname = "cc-pvdz" if rng.random() < 0.5 else "def2-svp"
        out.append(dict(rid=i, t=t, nwater=nw, basis=bname,
                        geom_seed=int(10_000 + i), dens_seed=int(20_000 + i)))
    return out
