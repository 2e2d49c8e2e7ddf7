#!/usr/bin/env python
"""Fock builds/s of the direct J/K build on one B200 (replicas per GPU).

Workload (default): seeded (H2O)_16 cluster, def2-SVP (N = 384), one
closed-shell build G = 2 J[D] - K[D] per step with D = C C^T, C 384 x 40
seeded and S-orthonormalised.  A step is one Fock build (J and K of one
density in one ``twoBodyContract`` call).

value   = builds/s of the mixed-precision build (FP32 for quartets whose
          Schwarz x density bound is below --cutoff, FP64 otherwise), inputs
          resident in HBM (device pointers), timed per step with CUDA events
          on the build stream; L2 is flushed (256 MiB write) between steps,
          outside the events.
e2e     = the same build through the public Python API with host (numpy)
          buffers: H2D of D, D2H of J and K inside the timed region.
fp64    = the same, all quartets in FP64 (the reference precision).
cutoff_sweep = the mixed build at the configuration's cutoffs 1e-6 .. 1e-10
          (builds/s, FP32 quartets, Fock and energy error).
complex_build = the FP64 build of a complex Hermitian density (an RT-TDDFT
          step's), same workload, with its error against the oracle.
batched_dD_graph = config 4: (H2O)8 / cc-pVDZ, 64 dD densities per CUDA-graph
          launch, FP64 (incremental builds stay FP64) and mixed, each with
          its error against the oracle on two of the densities, beside the
          same work one density per call in FP64.
four_component_ag4 = config 3: the Ag4 four-component Dirac-Coulomb build
          (FP64 and mixed, one timed build each, the mixed build's deviation,
          a bounded CPU sample with the GPU's deviation from the oracle).
serving = config 5: 2,000 Poisson-arrival requests replayed at each of
          --serving-rates (the last above saturation), p50/p99 latency,
          per-phase times, sampled errors against the oracle.
Errors  = max |G - G_oracle| and |E2 - E2_oracle| against the CPU oracle
          (FP64), computed once outside the timed region.  The extra
          workloads run only with one rank.

--impl reference times the reference's algorithm on the host cores: the
C++/OpenMP restatement of directScaffoldNew in oracle/ (the reference
itself needs libint2/libcint and cannot be built here).

Multi-GPU: the build runs on one GPU; with --gpus N each rank runs
an independent replica of the same build (replicas only, no collective) and
value sums the builds of all ranks over the slowest rank's time.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("Fock builds/s (mixed vs FP64, same B200) at <=1e-6 Eh Fock err; "
          "p50/p99 latency")
# DRAM bytes of one mixed build from an ncu capture (profiles/), by workload
TRAFFIC_BYTES = {"h2o16_def2svp": 1.32e8}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="h2o16_def2svp")
    ap.add_argument("--cutoff", type=float, default=1e-2)
    ap.add_argument("--no-oracle", action="store_true")
    ap.add_argument("--four-comp", type=int, default=1,
                    help="also time the Ag4 four-component build (config 3)")
    ap.add_argument("--batched", type=int, default=1,
                    help="also time the 64-density dD build as a CUDA graph")
    ap.add_argument("--serving-requests", type=int, default=2000,
                    help="requests of the Poisson serving stream (0: skip)")
    ap.add_argument("--serving-rates", type=float, nargs="+", default=[20.0, 80.0, 160.0],
                    help="arrival rates (Hz) the stream is replayed at")
    ap.add_argument("--profile-case", default=None,
                    help="one untimed build of a named case for profiler captures "
                         "(h2o16_def2svp, h2o8_ccpvdz, ag4_dc, ag1_ssss, ag1_llss) and exit")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="precision of --profile-case")
    return ap.parse_args()


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return ws, rank, local, pg


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for n, v in zip(names, s[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def fma_peaks():
    from chronusq_public_b200.build import PEAK_LIB
    L = ctypes.CDLL(PEAK_LIB)
    L.cqf_fma_peak_tflops.restype = ctypes.c_double
    L.cqf_fma_peak_tflops.argtypes = [ctypes.c_int, ctypes.c_int]
    return L.cqf_fma_peak_tflops(1, 4096), L.cqf_fma_peak_tflops(0, 16384)


def build_launches(basis, Q, mixed):
    """Kernels one closed-shell J+K build launches (l <= 2 bases): block
    norms x2, max, norms_aux, Cartesian transforms x2, the FP32 density copy
    (mixed), per class pair and bra slab the planning pass and the FP64 (and
    FP32) class kernel, back transforms x2.  Class sizes are the significant
    pairs (nonzero Schwarz bound) per angular-momentum class; the slab size
    is the library's mask region (2^18 words per stream)."""
    sys.path.insert(0, os.path.join(ROOT, "chronusq_public_b200", "csrc"))
    from gen_jk import orientation
    ls = [s.l for s in basis.shells]
    cnt = {}
    for i in range(basis.nshell):
        for j in range(i + 1):
            if Q[i, j] > 0.0:
                c = (max(ls[i], ls[j]), min(ls[i], ls[j]))
                cnt[c] = cnt.get(c, 0) + 1
    cls = sorted(cnt)
    tiles = lambda n: (n + 31) // 32
    need = max([max(cnt[a] * tiles(cnt[b]), cnt[b] * tiles(cnt[a]))
                for i, a in enumerate(cls) for b in cls[:i + 1]] + [0])
    words = max(max(tiles(n) for n in cnt.values()), min(need, 1 << 18))
    n = 2 + 1 + 1 + 2 + (1 if mixed else 0) + 2
    for i, a in enumerate(cls):
        for b in cls[:i + 1]:
            bra, ket = orientation(a, b)
            slab = max(1, words // tiles(cnt[ket]))
            n += (-(-cnt[bra] // slab)) * (3 if mixed else 2)
    return n


def oracle_module():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def cpu_baseline(basis, D, budget_s=25.0):
    """Times the oracle (C++/OpenMP restatement of directScaffoldNew) on all
    host cores: one warm-up build then as many builds as fit the budget."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ob = O.OracleBasis(basis)
    ob.schwarz()
    t0 = time.perf_counter()
    J, K = ob.contract([D, D], [1, 1], [0, 1])
    first = time.perf_counter() - t0
    times = [first]
    while sum(times) < budget_s and len(times) < 5:
        t0 = time.perf_counter()
        ob.contract([D, D], [1, 1], [0, 1])
        times.append(time.perf_counter() - t0)
    med = statistics.median(times[1:] if len(times) > 1 else times)
    return dict(builds_per_s=1.0 / med, s_per_build=med, n=len(times),
                cores=os.cpu_count(), G=2 * J - K)


def run_batched(dev, steps, warmup, precision="fp64", cutoff=0.0, ndens=64, check=True):
    """(H2O)8 / cc-pVDZ (N = 192): 64 symmetric perturbations
    dD_k = 1e-3 (X_k + X_k^T) contracted (J and K) against one pass of
    screened ERIs, incremental (AX += G[dD]), captured once as a CUDA graph
    and replayed.  Unit: builds/s = densities per second."""
    import numpy as np
    import torch

    from chronusq_public_b200 import workloads
    from chronusq_public_b200.basis import BasisSet
    from chronusq_public_b200.contraction import (COULOMB, EXCHANGE, ContractionGraph,
                                                  DirectTPI, TwoBodyContraction)
    mol, bname, nocc, seed = workloads.config("h2o8_ccpvdz")
    basis = BasisSet.build(mol, bname)
    tpi = DirectTPI(basis, device=dev.index or 0)
    N = basis.nbasis
    dDs = workloads.delta_densities(N, ndens, eps=1e-3, seed_base=400)
    X = [torch.from_numpy(np.ascontiguousarray(d.T)).to(dev).t() for d in dDs]
    out = [torch.zeros((N, N), dtype=torch.float64, device=dev).t() for _ in range(2 * ndens)]
    cont = []
    for k in range(ndens):
        cont.append(TwoBodyContraction(X[k], out[2 * k], True, COULOMB))
        cont.append(TwoBodyContraction(X[k], out[2 * k + 1], True, EXCHANGE))
    stream = torch.cuda.Stream(dev)
    single = None
    if precision == "fp64":
        # the same work one density per call (J and K of dD_0, FP64, no
        # graph): the FP64 GPU build the batched rate is compared with
        from chronusq_public_b200.contraction import GTODirectTPIContraction
        con = GTODirectTPIContraction(tpi)
        one = [TwoBodyContraction(X[0], out[0], True, COULOMB),
               TwoBodyContraction(X[0], out[1], True, EXCHANGE)]
        for _ in range(warmup):
            con.twoBodyContract(one, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        ms1 = []
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            con.twoBodyContract(one, stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms1.append(e0.elapsed_time(e1))
        t1 = float(np.median(ms1)) / 1e3
        single = {"ms_per_build": t1 * 1e3, "builds_per_s": 1.0 / t1,
                  "what": "one dD per call (J+K), FP64, no graph"}
    g = ContractionGraph(tpi, cont, precision=precision, fp32_cutoff=cutoff)
    for _ in range(warmup):
        g.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    ms = []
    for _ in range(steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.launch(stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    # error of one launch against the oracle on two of the densities (the
    # graph accumulates, so the outputs are zeroed and it is replayed once)
    for o in out:
        o.zero_()
    g.launch(stream.cuda_stream)
    torch.cuda.synchronize()
    g.close()
    err = None
    if check:
        O = oracle_module()
        ob = O.OracleBasis(basis)
        errs = []
        for k in (0, 1):
            Jo, Ko = ob.contract([dDs[k], dDs[k]], [1, 1], [0, 1])
            J = out[2 * k].t().contiguous().t().cpu().numpy()
            K = out[2 * k + 1].t().contiguous().t().cpu().numpy()
            errs.append(float(np.abs((2 * J - K) - (2 * Jo - Ko)).max()))
        err = {"fock_maxabs_vs_oracle": max(errs), "densities_checked": 2,
               "what": "max |G_k - G_k(oracle)|, G = 2J - K of dD_0 and dD_1 (one launch)"}
    t = float(np.median(ms)) / 1e3
    res = {"workload": "h2o8_ccpvdz x 64 dD (J+K), CUDA graph", "nbasis": N,
           "densities_per_launch": ndens, "ms_per_launch": t * 1e3,
           "builds_per_s": ndens / t, "precision": precision, "fp32_cutoff": cutoff,
           "errors": err}
    if single:
        res["fp64_single_density"] = single
    return res


def prepare_serving(dev, nreq):
    """The requests of the serving stream (config 5): nreq seeded (H2O)_n,
    n ~ U{1..32}, cc-pVDZ or def2-SVP (50/50), each with its own seeded
    S-orthonormalised occupied-orbital density (5 per water); arrival offsets
    of a unit-rate Poisson process (divided by the rate when replayed).  S
    comes from the device, before any timed stream starts."""
    from chronusq_public_b200 import workloads
    from chronusq_public_b200.basis import BasisSet
    from chronusq_public_b200.contraction import DirectTPI
    from chronusq_public_b200.serving import poisson_stream
    prepared = []
    for r in poisson_stream(nreq, 1.0, seed=5):
        mol = workloads.water_cluster(r["nwater"], seed=r["geom_seed"],
                                      box=max(6.0, 10.0 * (r["nwater"] / 16.0) ** (1 / 3)))
        basis = BasisSet.build(mol, r["basis"])
        tpi = DirectTPI(basis, device=dev.index or 0)
        S, _ = tpi.one_electron()
        tpi.close()
        D = workloads.occupied_density(S, 5 * r["nwater"], r["dens_seed"])
        prepared.append((r, mol, D, basis))
    return prepared


def run_serving(dev, prepared, rate, cutoff, check=0):
    """Replays the prepared requests with Poisson arrivals at `rate` Hz into
    the native server (continuous batching, memory admission), mixed
    precision.  Latency = completion - arrival.  With check > 0 that many
    requests of at most 8 waters (every k-th of them) are compared with the
    oracle's G = 2J - K."""
    import numpy as np

    from chronusq_public_b200.serving import FockRequest, FockServer
    srv = FockServer(device=dev.index or 0, slots=8, mem_budget=16 << 30)
    futs = []
    t0 = time.perf_counter()
    for (r, mol, D, _b) in prepared:
        ta = r["t"] / rate
        now = time.perf_counter() - t0
        if ta > now:
            time.sleep(ta - now)
        futs.append(srv.submit(FockRequest(mol, r["basis"], D, precision="mixed",
                                           fp32_cutoff=cutoff, rid=r["rid"],
                                           arrival=t0 + ta)))
    results = [f.result(timeout=900) for f in futs]
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    out = {"requests": len(prepared), "arrival_rate_hz": rate, "wall_s": wall,
           "builds_per_s": len(prepared) / wall, "p50_ms": st["p50_ms"],
           "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"], "fp32_cutoff": cutoff,
           "peak_inflight": st.get("peak_inflight"),
           "phases_ms": {k: st[k] for k in ("prep_ms", "queue_ms", "setup_ms", "build_ms")
                         if k in st},
           "mix": "U{1..32} waters, cc-pVDZ/def2-SVP 50/50"}
    if check > 0:
        O = oracle_module()
        small = [i for i, p in enumerate(prepared) if p[0]["nwater"] <= 8]
        pick = small[::max(1, len(small) // check)][:check]
        errs = []
        for i in pick:
            D, basis = prepared[i][2], prepared[i][3]
            Jo, Ko = O.OracleBasis(basis).contract([D, D], [1, 1], [0, 1])
            errs.append(float(np.abs(results[i] - (2 * Jo - Ko)).max()))
        out["errors"] = {"fock_maxabs_vs_oracle": max(errs), "requests_checked": len(pick),
                         "what": "max |G - G(oracle)| over sampled requests of <= 8 waters"}
    return out


def reference_arm_4c(args, ws):
    """Oracle 4C build (bare Coulomb + LLSS) of one Ag atom of the Ag4
    workload's basis: the bounded CPU sample of config 3."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    from chronusq_public_b200 import workloads
    from chronusq_public_b200.basis import BasisSet, Molecule
    b1 = BasisSet.build(Molecule.from_angstrom([("Ag", 0.0, 0.0, 0.0)]),
                        "sapporo-dkh3-dzp-2012_no", uncontract=True)
    ob = O.OracleBasis(b1)
    S1, T1 = ob.overlap_kinetic()
    D1 = workloads.spinor_density_4c(S1, T1, 47, 3)
    times = []
    for _ in range(max(1, min(args.steps, 2))):
        t0 = time.perf_counter()
        ob.dirac_coulomb(D1, bare=True, dc=True, ssss=False)
        times.append(time.perf_counter() - t0)
    v = len(times) / sum(times)
    sample = ("one Ag atom (N = 152) of the ag4_dc basis, bare Coulomb + LLSS, "
              "C++/OpenMP restatement of directScaffoldLibcint + formGDDirect")
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": "builds/s",
                      "n_gpus": ws, "steps": len(times), "warmup": 0,
                      "ms_per_step": 1e3 * sum(times) / len(times),
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                      "dtype": "f64 (complex)", "data": "synthetic (seeded)",
                      "config": {"workload": "ag4_dc", "sample": sample},
                      "cpu_baseline": {"value": v, "unit": "builds/s",
                                       "cores": os.cpu_count(), "kind": "port",
                                       "sample": sample},
                      "e2e": {"value": v, "unit": "builds/s", "h2d_bytes_per_step": 0,
                              "d2h_bytes_per_step": 0}}), flush=True)


def reference_arm(args, ws, rank):
    if rank != 0:
        return
    if args.workload == "ag4_dc":
        reference_arm_4c(args, ws)
        return
    import numpy as np

    from chronusq_public_b200 import workloads
    from chronusq_public_b200.basis import BasisSet
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    mol, bname, nocc, seed = workloads.config(args.workload)
    basis = BasisSet.build(mol, bname)
    ob = O.OracleBasis(basis)
    S, _ = ob.overlap_kinetic()
    D = workloads.occupied_density(S, nocc, seed)
    ob.schwarz()
    for _ in range(max(1, min(args.warmup, 1))):
        ob.contract([D, D], [1, 1], [0, 1])
    times = []
    budget = 150.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ob.contract([D, D], [1, 1], [0, 1])
        times.append(time.perf_counter() - t0)
        if sum(times) > budget:
            break
    tot = sum(times)
    v = len(times) / tot
    line = {"impl": "reference", "metric": METRIC, "value": v,
            "unit": "builds/s", "n_gpus": ws, "steps": len(times),
            "warmup": 1, "ms_per_step": 1e3 * tot / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": args.workload, "nbasis": basis.nbasis,
                       "l2": "inputs smaller than L2; host CPU arm"},
            "cpu_baseline": {"value": v, "unit": "builds/s",
                             "cores": os.cpu_count(), "kind": "port",
                             "sample": "%d full builds of %s (C++/OpenMP "
                                       "restatement of directScaffoldNew; "
                                       "libint2/libcint unavailable)"
                                       % (len(times), args.workload)},
            "e2e": {"value": v, "unit": "builds/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_four_component_sub(args, local):
    """Config 3 inside the default run: the Ag4 four-component build
    (BareCoulomb + DiracCoulomb + SSSS, libcint branch; N = 608, 4C dimension
    2432), one FP64 and one mixed build timed with CUDA events after a
    warm-up on a zero density (which computes the 4C Schwarz tables with
    every quartet screened); the mixed build's largest deviation from the
    FP64 one; the bounded CPU sample (one Ag atom, bare Coulomb + LLSS) timed
    on the oracle and on the GPU, with the GPU's deviation from the oracle."""
    import numpy as np
    import torch

    from chronusq_public_b200 import workloads
    from chronusq_public_b200.basis import BasisSet, Molecule
    from chronusq_public_b200.contraction import DirectTPI
    from chronusq_public_b200.fockbuilder import FourCompFock

    dev = torch.device("cuda", local)
    basis, tpi, D = workloads.build_ag4_dc(lambda b: DirectTPI(b, device=local))
    N2 = 2 * basis.nbasis
    Dd = [torch.from_numpy(np.ascontiguousarray(d.T)).to(dev).t() for d in D]
    fb = FourCompFock(tpi)
    stream = torch.cuda.Stream(dev)
    fb.formGD([torch.zeros_like(d) for d in Dd], stream=stream.cuda_stream)
    torch.cuda.synchronize()

    def timed(**kw):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        G = fb.formGD(Dd, stream=stream.cuda_stream, **kw)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3, G, dict(fb.last_stats)

    with ClockSampler(local) as clk:
        t64, G, s64 = timed()
        t32, Gm, s32 = timed(precision="mixed", fp32_cutoff=args.cutoff)
    herm = max(float((g - g.conj().t()).abs().max()) for g in G)
    mixed_err = max(float((a - b).abs().max()) for a, b in zip(Gm, G))
    del Gm
    out = {"workload": "ag4_dc", "nbasis_1c": basis.nbasis, "dim_4c": 2 * N2,
           "hamiltonian": "BareCoulomb + DiracCoulomb + SSSS (libcint)",
           "fp64": {"s_per_build": t64, "builds_per_s": 1.0 / t64,
                    "quartets_computed": s64["fp64"], "quartets_screened": s64["screened"]},
           "mixed": {"s_per_build": t32, "builds_per_s": 1.0 / t32,
                     "fp32_cutoff": args.cutoff, "quartets_fp32": s32["fp32"],
                     "quartets_fp64": s32["fp64"], "speedup_vs_fp64": t64 / t32,
                     "G_maxabs_vs_fp64": mixed_err},
           "checks": {"G_hermiticity_maxabs": herm},
           "clocks": clk.summary()}
    if not args.no_oracle:
        O = oracle_module()
        b1 = BasisSet.build(Molecule.from_angstrom([("Ag", 0.0, 0.0, 0.0)]),
                            "sapporo-dkh3-dzp-2012_no", uncontract=True)
        tpi1 = DirectTPI(b1, device=local)
        S1, T1 = tpi1.one_electron()
        D1 = workloads.spinor_density_4c(S1, T1, 47, 3)
        ob = O.OracleBasis(b1)
        t0 = time.perf_counter()
        Go = ob.dirac_coulomb(D1, bare=True, dc=True, ssss=False)
        tcpu = time.perf_counter() - t0
        fb1 = FourCompFock(tpi1, DiracCoulombSSSS=False)
        fb1.formGD(D1)
        t0 = time.perf_counter()
        Gg = fb1.formGD(D1)
        tg = time.perf_counter() - t0
        out["cpu_baseline"] = {
            "value": 1.0 / tcpu, "unit": "builds/s", "cores": os.cpu_count(), "kind": "port",
            "sample": "one Ag atom (N = 152), bare Coulomb + LLSS, C++/OpenMP restatement "
                      "of directScaffoldLibcint + formGDDirect",
            "gpu_same_sample_builds_per_s": 1.0 / tg,
            "fock_maxabs_gpu_vs_oracle": max(float(np.abs(a - b).max())
                                             for a, b in zip(Gg, Go)),
            "G_maxabs_of_sample": max(float(np.abs(b).max()) for b in Go)}
        tpi1.close()
    tpi.close()
    return out


def run_four_component(args, ws, rank, local, pg):
    """Config 3: four-component Dirac-Coulomb build (BareCoulomb + DiracCoulomb
    + SSSS, libcint branch) of the seeded Ag4 tetrahedron, uncontracted
    sapporo-dkh3-dzp basis (N = 608, 4C dimension 2432), density from 188
    seeded complex spinors orthonormalised in the 4C metric; FP64.  A step is
    one full formGDDirect build.  The CPU baseline is the oracle on a bounded
    sample (one Ag atom, bare Coulomb + LLSS) with the GPU timed on the same
    sample.  The line's "mixed" object is one build with FP32 arithmetic on
    the quartets whose screening bound is below --cutoff, timed the same way,
    and its largest deviation from the FP64 build."""
    import numpy as np
    import torch

    from chronusq_public_b200 import workloads
    from chronusq_public_b200.basis import BasisSet, Molecule
    from chronusq_public_b200.contraction import DirectTPI
    from chronusq_public_b200.fockbuilder import FourCompFock

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    basis, tpi, D = workloads.build_ag4_dc(lambda b: DirectTPI(b, device=local))
    N2 = 2 * basis.nbasis
    Dd = [torch.from_numpy(np.ascontiguousarray(d.T)).to(dev).t() for d in D]
    fb = FourCompFock(tpi)
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        fb.formGD(Dd, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    ms = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            G = fb.formGD(Dd, stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    stats = dict(fb.last_stats)
    torch.cuda.synchronize()
    herm = max(float((g - g.conj().t()).abs().max()) for g in G)
    # mixed precision (FP32 on quartets with bound < cutoff): one timed build
    # after one warm-up, and its largest deviation from the FP64 build
    fb.formGD(Dd, precision="mixed", fp32_cutoff=args.cutoff, stream=stream.cuda_stream)
    flush.fill_(1.0)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    Gm = fb.formGD(Dd, precision="mixed", fp32_cutoff=args.cutoff, stream=stream.cuda_stream)
    e1.record(stream)
    e1.synchronize()
    ms_mixed = e0.elapsed_time(e1)
    smix = dict(fb.last_stats)
    mixed_err = max(float((a - b).abs().max()) for a, b in zip(Gm, G))
    del Gm
    # e2e: host numpy buffers through the public API
    te = []
    t0 = time.perf_counter()
    fb.formGD(D)
    te.append(time.perf_counter() - t0)
    t = torch.tensor([sum(ms) / 1e3, sum(te) / len(te)], dtype=torch.float64, device=dev)
    if pg:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    tdev, te2e = float(t[0]), float(t[1])
    if rank != 0:
        return
    K = args.steps
    line = {
        "metric": METRIC, "value": ws * K / tdev, "unit": "builds/s", "n_gpus": ws,
        "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * tdev / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64 (complex)", "data": "synthetic (seeded)",
        "config": {"workload": "ag4_dc", "nbasis_1c": basis.nbasis, "dim_4c": 2 * N2,
                   "nshell": basis.nshell, "npair": tpi.npair,
                   "hamiltonian": "BareCoulomb + DiracCoulomb + SSSS (libcint)",
                   "parallelism": "replicas",
                   "l2": "flushed between steps (256 MiB write)"},
        "quartets": {"computed": stats["fp64"], "screened": stats["screened"],
                     "total": stats["total"]},
        "checks": {"G_hermiticity_maxabs": herm},
        "mixed": {"builds_per_s": ws * 1e3 / ms_mixed, "fp32_cutoff": args.cutoff,
                  "G_maxabs_vs_fp64": mixed_err, "quartets_fp32": smix["fp32"],
                  "quartets_fp64": smix["fp64"], "speedup_vs_fp64": (tdev / K) / (ms_mixed / 1e3)},
        "e2e": {"value": ws / te2e, "unit": "builds/s",
                "h2d_bytes_per_step": 4 * 16 * N2 * N2,
                "d2h_bytes_per_step": 4 * 16 * N2 * N2},
        "clocks": clk.summary(),
    }
    if not args.no_oracle:
        # bounded CPU sample: one Ag atom, bare Coulomb + LLSS, oracle vs GPU
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as O
        mol1 = Molecule.from_angstrom([("Ag", 0.0, 0.0, 0.0)])
        b1 = BasisSet.build(mol1, "sapporo-dkh3-dzp-2012_no", uncontract=True)
        tpi1 = DirectTPI(b1, device=local)
        S1, T1 = tpi1.one_electron()
        D1 = workloads.spinor_density_4c(S1, T1, 47, 3)
        ob = O.OracleBasis(b1)
        t0 = time.perf_counter()
        Go = ob.dirac_coulomb(D1, bare=True, dc=True, ssss=False)
        tcpu = time.perf_counter() - t0
        fb1 = FourCompFock(tpi1, DiracCoulombSSSS=False)
        fb1.formGD(D1)
        t0 = time.perf_counter()
        Gg = fb1.formGD(D1)
        tg = time.perf_counter() - t0
        line["cpu_baseline"] = {
            "value": 1.0 / tcpu, "unit": "builds/s", "cores": os.cpu_count(), "kind": "port",
            "sample": "one Ag atom (N = 152), bare Coulomb + LLSS, C++/OpenMP restatement "
                      "of directScaffoldLibcint + formGDDirect",
            "gpu_same_sample_builds_per_s": 1.0 / tg,
            "fock_maxabs_gpu_vs_oracle": max(float(np.abs(a - b).max())
                                             for a, b in zip(Gg, Go))}
    print(json.dumps(line), flush=True)


def profile_case(args):
    """One untimed build of a named case on cuda:0 (the command ncu captures
    wrap; throughput numbers come from the timed runs, never from this)."""
    import numpy as np

    from chronusq_public_b200 import workloads
    from chronusq_public_b200.basis import BasisSet, Molecule
    from chronusq_public_b200.contraction import DirectTPI
    from chronusq_public_b200.fockbuilder import FockBuilder, FourCompFock
    name = args.profile_case
    cut = args.cutoff if args.precision == "mixed" else 0.0
    if name in ("ag1_ssss", "ag1_llss"):
        # one SSSS (or LLSS) contraction of a single Ag atom (uncontracted
        # basis) on a seeded Hermitian 17-entry input
        from chronusq_public_b200.contraction import (LLSS, SSSS, GTODirectRelERIContraction,
                                                      TwoBodyContraction)
        basis = BasisSet.build(Molecule.from_angstrom([("Ag", 0.0, 0.0, 0.0)]),
                               "sapporo-dkh3-dzp-2012_no", uncontract=True)
        tpi = DirectTPI(basis)
        N = basis.nbasis
        rng = np.random.default_rng(3)
        X = []
        for _ in range(17):
            A = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
            X.append(np.asfortranarray(0.05 * (A + A.conj().T)))
        lst = [TwoBodyContraction(x, np.zeros((N, N), complex)) for x in X]
        t0 = time.perf_counter()
        GTODirectRelERIContraction(tpi).twoBodyContract(
            lst, SSSS if name == "ag1_ssss" else LLSS, precision=args.precision,
            fp32_cutoff=cut)
    elif name == "ag4_dc":
        _basis, tpi, D = workloads.build_ag4_dc(lambda b: DirectTPI(b))
        t0 = time.perf_counter()
        FourCompFock(tpi).formGD(D, precision=args.precision, fp32_cutoff=cut)
    else:
        _mol, _basis, tpi, D = workloads.build_config(name, lambda b: DirectTPI(b))
        t0 = time.perf_counter()
        FockBuilder(tpi).formRawGD(D, precision=args.precision, fp32_cutoff=cut)
    print("%s (%s): one untimed build %.3f s" % (name, args.precision,
                                                  time.perf_counter() - t0), flush=True)


def main():
    args = parse()
    if args.profile_case:
        profile_case(args)
        return
    ws, rank, local, pg = dist_init(args)
    if args.impl == "ours" and args.workload == "ag4_dc":
        run_four_component(args, ws, rank, local, pg)
        if pg:
            pg.destroy_process_group()
        return
    if args.impl == "reference":
        reference_arm(args, ws, rank)
        if pg:
            pg.destroy_process_group()
        return

    import numpy as np
    import torch

    from chronusq_public_b200 import flops as FL
    from chronusq_public_b200 import workloads
    from chronusq_public_b200.basis import BasisSet
    from chronusq_public_b200.contraction import (COULOMB, EXCHANGE, DirectTPI,
                                                  GTODirectTPIContraction,
                                                  TwoBodyContraction)
    from chronusq_public_b200.fockbuilder import FockBuilder, two_electron_energy

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    mol, bname, nocc, seed = workloads.config(args.workload)
    basis = BasisSet.build(mol, bname)
    tpi = DirectTPI(basis, device=local)
    S, _ = tpi.one_electron()
    D = workloads.occupied_density(S, nocc, seed)
    N = basis.nbasis

    def colmajor(a):
        return torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).to(dev).t()

    Dd = colmajor(D)
    Jd = torch.zeros((N, N), dtype=torch.float64, device=dev).t().contiguous().t()
    Kd = torch.zeros_like(Jd).t().contiguous().t()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    con = GTODirectTPIContraction(tpi)
    stream = torch.cuda.Stream(dev)   # the build and its events on one stream

    def run(precision, cut, steps, warmup, collect=False):
        torch.cuda.set_stream(stream)
        for _ in range(warmup):
            Jd.zero_(); Kd.zero_()
            con.twoBodyContract([TwoBodyContraction(Dd, Jd, True, COULOMB),
                                 TwoBodyContraction(Dd, Kd, True, EXCHANGE)],
                                precision=precision, fp32_cutoff=cut,
                                stream=stream.cuda_stream)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        ms = []
        for _ in range(steps):
            flush.fill_(1.0)
            Jd.zero_(); Kd.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            con.twoBodyContract([TwoBodyContraction(Dd, Jd, True, COULOMB),
                                 TwoBodyContraction(Dd, Kd, True, EXCHANGE)],
                                precision=precision, fp32_cutoff=cut,
                                stream=stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        G = (2 * Jd - Kd).t().contiguous().t().cpu().numpy()
        return ms, G, dict(con.last_stats)

    with ClockSampler(local) as clk:
        ms64, G64, st64 = run("fp64", 0.0, args.steps, args.warmup)
        msmx, Gmx, stmx = run("mixed", args.cutoff, args.steps, args.warmup)
    clocks = clk.summary()
    # the configuration's cutoff sweep (1e-6 .. 1e-10): builds/s and, below,
    # the Fock and energy errors of each
    sweep = []
    for cut in (1e-6, 1e-7, 1e-8, 1e-9, 1e-10):
        msc, Gc, stc = run("mixed", cut, max(3, args.steps // 2), 1)
        sweep.append({"fp32_cutoff": cut, "builds_per_s": 1e3 * len(msc) / sum(msc),
                      "quartets_fp32": stc["fp32"], "G": Gc})

    # complex Hermitian density (an RT-TDDFT step's): J and K of D + i A, A a
    # seeded antisymmetric perturbation, FP64, device pointers
    rngc = np.random.default_rng(6)
    Ac = rngc.standard_normal((N, N))
    Xcx = torch.from_numpy(np.ascontiguousarray((D + 0.01j * (Ac - Ac.T)).T)).to(dev).t()
    Jcx = torch.zeros((N, N), dtype=torch.complex128, device=dev).t()
    Kcx = torch.zeros((N, N), dtype=torch.complex128, device=dev).t()
    cxl = [TwoBodyContraction(Xcx, Jcx, True, COULOMB), TwoBodyContraction(Xcx, Kcx, True, EXCHANGE)]
    for _ in range(args.warmup):
        con.twoBodyContract(cxl, stream=stream.cuda_stream)
    torch.cuda.synchronize()
    mscx = []
    for _ in range(max(3, args.steps // 2)):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        con.twoBodyContract(cxl, stream=stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        mscx.append(e0.elapsed_time(e1))
    complex_build = {"what": "complex Hermitian J+K (D + i A), FP64, device pointers",
                     "ms_per_build": float(np.median(mscx)),
                     "builds_per_s": 1e3 / float(np.median(mscx))}
    Zcx = D + 0.01j * (Ac - Ac.T)
    if not args.no_oracle and ws == 1:
        Jcx.zero_(); Kcx.zero_()
        con.twoBodyContract(cxl, stream=stream.cuda_stream)
        torch.cuda.synchronize()
        Jo, Ko = oracle_module().OracleBasis(basis).contract([Zcx, Zcx], [1, 1], [0, 1])
        Gc = (2 * Jcx - Kcx).t().contiguous().t().cpu().numpy()
        complex_build["errors"] = {
            "fock_maxabs_vs_oracle": float(np.abs(Gc - (2 * Jo - Ko)).max()),
            "what": "max |G - G(oracle)|, G = 2J - K of the complex Hermitian density"}

    # end-to-end through the public API with host buffers; J, K and G are
    # the caller's matrices, reused every build as an SCF loop reuses them
    fb = FockBuilder(tpi)
    Jh, Kh, Gh = (np.zeros((N, N), order="F") for _ in range(3))
    for _ in range(args.warmup):
        fb.formRawGD(D, precision="mixed", fp32_cutoff=args.cutoff, J=Jh, K=Kh, G=Gh)
    torch.cuda.synchronize()
    te = []
    with ClockSampler(local) as clk_e2e:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            fb.formRawGD(D, precision="mixed", fp32_cutoff=args.cutoff, J=Jh, K=Kh, G=Gh)
            te.append(time.perf_counter() - t0)

    def agg(x):
        t = torch.tensor([sum(x)], dtype=torch.float64, device=dev)
        if pg:
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
        return float(t.item())

    t64, tmx, te2e = agg(ms64) / 1e3, agg(msmx) / 1e3, agg(te)
    K = args.steps
    v64 = ws * K / t64
    vmx = ws * K / tmx
    ve2e = ws * K / te2e

    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return

    # roofline: algorithmic FLOPs of one build (count model) over the
    # measured FMA peaks
    Q = tpi.schwarz()
    fl = FL.build_flops(basis, Q, [D], nmat_digest=2, fp32_cut=args.cutoff)
    p64, p32 = fma_peaks()
    t_build = tmx / K
    achieved = (fl["f64"] + fl["f32"]) / t_build / 1e12
    frac = (fl["f64"] / (p64 * 1e12) + fl["f32"] / (p32 * 1e12)) / t_build
    fl64 = FL.build_flops(basis, Q, [D], nmat_digest=2)
    frac64 = (fl64["f64"] / (p64 * 1e12)) / (t64 / K)

    batched = None
    if args.batched and ws == 1:
        # config 4's incremental dD build runs in FP64 (FockBuilder keeps
        # increments in FP64); the mixed graph is reported beside it with its
        # error
        chk = not args.no_oracle
        batched = {"fp64": run_batched(dev, args.steps, args.warmup, check=chk),
                   "mixed": run_batched(dev, args.steps, args.warmup, "mixed", args.cutoff,
                                        check=chk)}
        batched["fp64_graph_over_fp64_single"] = (
            batched["fp64"]["builds_per_s"]
            / batched["fp64"]["fp64_single_density"]["builds_per_s"])
    four_comp = None
    if args.four_comp and ws == 1:
        four_comp = run_four_component_sub(args, local)
    serving = None
    if args.serving_requests > 0 and ws == 1:
        prepared = prepare_serving(dev, args.serving_requests)
        serving = {"rates": [run_serving(dev, prepared, r, args.cutoff,
                                         check=3 if k == 0 else 0)
                             for k, r in enumerate(args.serving_rates)]}

    cpu = None
    err = {}
    if not args.no_oracle:
        cpu = cpu_baseline(basis, D)
        Go = cpu["G"]
        err = {"fock_maxabs_fp64": float(np.abs(G64 - Go).max()),
               "fock_maxabs_mixed": float(np.abs(Gmx - Go).max()),
               "energy_err_mixed": abs(two_electron_energy(Gmx, D)
                                       - two_electron_energy(Go, D)),
               "energy_err_fp64": abs(two_electron_energy(G64, D)
                                      - two_electron_energy(Go, D))}
    Gref = cpu["G"] if cpu else G64
    for sw in sweep:
        Gc = sw.pop("G")
        sw["fock_maxabs"] = float(np.abs(Gc - Gref).max())
        sw["energy_err"] = abs(two_electron_energy(Gc, D) - two_electron_energy(Gref, D))
        sw["errors_against"] = "oracle" if cpu else "FP64 GPU build"
    launches_per_step = build_launches(basis, Q, mixed=True)
    line = {
        "metric": METRIC, "value": vmx, "unit": "builds/s", "n_gpus": ws,
        "steps": K, "warmup": args.warmup, "ms_per_step": 1e3 * tmx / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64+f32 (mixed)", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "nbasis": N,
                   "nshell": basis.nshell, "npair": tpi.npair,
                   "fp32_cutoff": args.cutoff, "parallelism": "replicas",
                   "l2": "flushed between steps (256 MiB write)"},
        "fp64": {"value": v64, "unit": "builds/s", "ms_per_step": 1e3 * t64 / K,
                 "roofline_frac": frac64},
        "mixed_over_fp64": vmx / v64,
        "cutoff_sweep": sweep,
        "complex_build": complex_build,
        "latency_ms": {"p50": float(np.percentile(msmx, 50)),
                       "p99": float(np.percentile(msmx, 99))},
        "errors_vs_oracle": err,
        "quartets": {"computed_fp32": stmx["fp32"], "computed_fp64": stmx["fp64"],
                     "screened": stmx["screened"], "total": stmx["total"]},
        "roofline": {"bound": "fp64+fp32 FMA (CUDA cores)", "achieved": achieved,
                     "peak": {"fp64_tflops": p64, "fp32_tflops": p32,
                              "source": "measured in this run (FMA microbenchmark)"},
                     "unit": "TFLOP/s", "frac": frac,
                     "gflop_per_build": {"f64": fl["f64"] / 1e9, "f32": fl["f32"] / 1e9},
                     "traffic": TRAFFIC_BYTES.get(args.workload),
                     "traffic_source": "constant: DRAM read+write bytes of one mixed build "
                                       "(all its launches) from the ncu capture in "
                                       "profiles/launches_jk_h2o16_def2svp.md, per-launch "
                                       "cache flush (an upper bound); not measured in "
                                       "this run"},
        "e2e": {"value": ve2e, "unit": "builds/s",
                "h2d_bytes_per_step": 8 * N * N,
                "d2h_bytes_per_step": 2 * 8 * N * N,
                "clocks": clk_e2e.summary()},
        "gpu_launches": launches_per_step * K,
        "clocks": clocks,
    }
    if batched:
        line["batched_dD_graph"] = batched
    if four_comp:
        line["four_component_ag4"] = four_comp
    if serving:
        line["serving"] = serving
    if cpu:
        line["cpu_baseline"] = {"value": cpu["builds_per_s"], "unit": "builds/s",
                                "cores": cpu["cores"], "kind": "port",
                                "sample": "%d full builds (1 warm-up) of %s, "
                                          "C++/OpenMP restatement of "
                                          "directScaffoldNew" % (cpu["n"], args.workload)}
    print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
