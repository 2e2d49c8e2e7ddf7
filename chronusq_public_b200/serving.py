"""Continuous-batching Fock-build server on one GPU.

Requests (molecule, basis name, density) arrive at any time.  The server

* admits a request when an execution slot is free and its device-memory
  footprint (shell-pair data + contraction workspace, estimated before any
  allocation) fits in the budget that the requests already on the GPU leave;
  requests that do not fit wait in FIFO order and are admitted as soon as
  slots / memory free up (no batch boundaries: continuous batching);
* runs every admitted request on its own worker thread and its own CUDA
  stream (each device basis owns a stream), so the basis set-up and J/K
  kernels of different requests overlap on the device; ctypes releases the
  GIL for the duration of each C-ABI call;
* keeps the device shell-pair data (``DirectTPI``) of recent geometries
  resident in HBM (LRU, counted in the budget) so repeated geometries (SCF
  iterations, RT steps) skip set-up;
* records per-request latency (completion - arrival) and reports throughput
  with p50 / p99 latency.

Each request's result depends only on its own inputs: the kernels and the
work split are the same alone and in a mix (the only difference is the order
of floating-point atomics), which ``tests/test_gpu_serving.py`` checks.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Dict, Optional

import numpy as np

from .basis import BasisSet, Molecule
from .contraction import DirectTPI
from .fockbuilder import FockBuilder


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


def _geometry_key(mol: Molecule, basis: str):
    return (basis, mol.Z.tobytes(), np.round(mol.xyz, 10).tobytes())


def footprint_bytes(basis: BasisSet, nmat: int = 2) -> int:
    """Device bytes a request needs: shell/pair/primitive-pair data (upper
    bound: every pair significant) plus the per-call workspace."""
    ns, N, nc = basis.nshell, basis.nbasis, basis.ncart
    npair = ns * (ns + 1) // 2
    kprim = basis.max_prim ** 2
    pairs = npair * (64 + 96 * kprim) + ns * ns * 8 + 300_000
    ws = 8 * (2 * nmat * N * N + 2 * nmat * nc * nc + (nmat + 1) * ns * ns)
    return int(pairs + ws)


class FockServer:
    def __init__(self, device: int = 0, slots: int = 8,
                 mem_budget: int = 8 << 30, cache_entries: int = 16):
        self.device = device
        self.slots = slots
        self.mem_budget = mem_budget
        self.cache_entries = cache_entries
        self._lock = threading.Condition()
        self._queue: collections.deque = collections.deque()
        self._inflight = 0
        self._mem_in_use = 0
        self._cache: "collections.OrderedDict" = collections.OrderedDict()
        self._cache_mem = 0
        self._stop = False
        self.latencies: Dict[int, float] = {}
        # per request: (queue wait, device set-up, build) in seconds
        self.phases: Dict[int, tuple] = {}
        self.completed = 0
        self._sched = threading.Thread(target=self._schedule, daemon=True)
        self._sched.start()

    # ------------------------------------------------------------ public
    def submit(self, req: FockRequest) -> Future:
        if not req.arrival:
            req.arrival = time.perf_counter()
        with self._lock:
            self._queue.append(req)
            self._lock.notify_all()
        return req.future

    def close(self):
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        self._sched.join(timeout=60)
        for _, (tpi, _m) in self._cache.items():
            tpi.close()
        self._cache.clear()

    def stats(self):
        lat = np.array(list(self.latencies.values()))
        if len(lat) == 0:
            return {}
        out = {"completed": self.completed,
               "p50_ms": float(np.percentile(lat, 50) * 1e3),
               "p99_ms": float(np.percentile(lat, 99) * 1e3),
               "mean_ms": float(lat.mean() * 1e3)}
        if self.phases:
            ph = np.array(list(self.phases.values())) * 1e3
            for i, name in enumerate(("queue", "setup", "build")):
                out[name + "_ms"] = {"p50": float(np.percentile(ph[:, i], 50)),
                                     "p99": float(np.percentile(ph[:, i], 99)),
                                     "mean": float(ph[:, i].mean())}
        return out

    # ------------------------------------------------------------ internals
    def _schedule(self):
        while True:
            with self._lock:
                while not self._stop and not self._admissible():
                    self._lock.wait(timeout=0.5)
                if self._stop and not self._queue:
                    return
                if not self._admissible():
                    continue
                req, basis, need = self._queue.popleft()
                self._inflight += 1
                self._mem_in_use += need
            threading.Thread(target=self._run, args=(req, basis, need),
                             daemon=True).start()

    def _admissible(self) -> bool:
        """Head of the queue fits a slot and the memory budget (FIFO)."""
        if not self._queue or self._inflight >= self.slots:
            return False
        head = self._queue[0]
        if isinstance(head, FockRequest):
            basis = BasisSet.build(head.mol, head.basis)
            self._queue[0] = (head, basis, footprint_bytes(basis))
        req, basis, need = self._queue[0]
        key = _geometry_key(req.mol, req.basis)
        if key in self._cache:
            need -= self._cache[key][1]
        free = self.mem_budget - self._mem_in_use - self._cache_mem
        while free < need and self._evict_one():
            free = self.mem_budget - self._mem_in_use - self._cache_mem
        if free >= need or self._inflight == 0:
            self._queue[0] = (req, basis, max(need, 0))
            return True
        return False

    def _evict_one(self) -> bool:
        for key, (tpi, mem) in self._cache.items():
            if getattr(tpi, "_busy", 0) == 0:
                del self._cache[key]
                self._cache_mem -= mem
                tpi.close()
                return True
        return False

    def _get_tpi(self, req: FockRequest, basis: BasisSet):
        key = _geometry_key(req.mol, req.basis)
        with self._lock:
            hit = self._cache.pop(key, None)
            if hit is not None:
                self._cache_mem -= hit[1]
                hit[0]._busy = getattr(hit[0], "_busy", 0) + 1
                return hit[0], key
        tpi = DirectTPI(basis, device=self.device)
        tpi._busy = 1
        return tpi, key

    def _run(self, req: FockRequest, basis: BasisSet, need: int):
        try:
            t_start = time.perf_counter()
            tpi, key = self._get_tpi(req, basis)
            t_setup = time.perf_counter()
            try:
                G, _J, _K = FockBuilder(tpi).formRawGD(
                    req.D, precision=req.precision, fp32_cutoff=req.fp32_cutoff)
            finally:
                tpi._busy -= 1
            done = time.perf_counter()
            with self._lock:
                self.latencies[req.rid] = done - req.arrival
                self.phases[req.rid] = (t_start - req.arrival, t_setup - t_start,
                                        done - t_setup)
                self.completed += 1
                data_mem = footprint_bytes(basis) - 8 * 2 * 2 * basis.nbasis ** 2
                self._cache[key] = (tpi, max(data_mem, 0))
                self._cache_mem += max(data_mem, 0)
                while len(self._cache) > self.cache_entries and self._evict_one():
                    pass
            req.future.set_result(G)
        except BaseException as e:  # report to the caller, keep serving
            req.future.set_exception(e)
        finally:
            with self._lock:
                self._inflight -= 1
                self._mem_in_use -= need
                self._lock.notify_all()


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
