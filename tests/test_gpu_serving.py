"""Serving loop: continuous batching with memory admission; every result is
the same alone and in the mix (and matches the oracle)."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402
from chronusq_public_b200 import workloads  # noqa: E402
from chronusq_public_b200.basis import BasisSet  # noqa: E402
from chronusq_public_b200.contraction import DirectTPI  # noqa: E402
from chronusq_public_b200.serving import (FockRequest, FockServer,  # noqa: E402
                                          footprint_bytes)


def _requests(n, seed=7, nwater=None):
    reqs = []
    rng = np.random.default_rng(seed)
    for i in range(n):
        nw = nwater if nwater else int(rng.integers(1, 5))
        bname = "cc-pvdz" if i % 2 == 0 else "def2-svp"
        mol = workloads.water_cluster(nw, seed=100 + i, box=6.0)
        basis = BasisSet.build(mol, bname)
        tpi = DirectTPI(basis)
        S, _ = tpi.one_electron()
        tpi.close()
        D = workloads.occupied_density(S, 5 * nw, seed=200 + i)
        reqs.append((mol, bname, D, basis))
    return reqs


def test_alone_equals_mix_and_oracle():
    reqs = _requests(6)
    alone = []
    srv = FockServer(slots=1)
    for i, (mol, b, D, _) in enumerate(reqs):
        f = srv.submit(FockRequest(mol, b, D, precision="mixed", fp32_cutoff=1e-6, rid=i))
        alone.append(f.result(timeout=120))
    srv.close()
    srv = FockServer(slots=6)
    futs = [srv.submit(FockRequest(mol, b, D, precision="mixed", fp32_cutoff=1e-6, rid=i))
            for i, (mol, b, D, _) in enumerate(reqs)]
    mix = [f.result(timeout=120) for f in futs]
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs)
    # the mix really overlapped on the GPU (a server that serialised every
    # request would have peak_inflight == 1)
    assert st["peak_inflight"] > 1
    for a, m in zip(alone, mix):
        assert np.abs(a - m).max() < 1e-10
    # one request against the FP64 oracle at the mixed-path tolerance
    mol, b, D, basis = reqs[1]
    ob = O.OracleBasis(basis)
    Jo, Ko = ob.contract([D, D], [1, 1], [0, 1])
    assert np.abs(mix[1] - (2 * Jo - Ko)).max() < 1e-6


def test_memory_admission_limits_concurrency():
    reqs = [r for r in _requests(4, seed=9, nwater=3) if r[1] == "def2-svp"]
    reqs += [r for r in _requests(4, seed=11, nwater=3) if r[1] == "def2-svp"]
    need = max(footprint_bytes(r[3]) for r in reqs)
    assert min(footprint_bytes(r[3]) for r in reqs) * 2 > need * 1.5
    srv = FockServer(slots=8, mem_budget=int(need * 1.5), cache_entries=0)
    futs = [srv.submit(FockRequest(mol, b, D, rid=i)) for i, (mol, b, D, _) in enumerate(reqs)]
    for f in futs:
        f.result(timeout=120)
    st = srv.stats()
    srv.close()
    assert st["completed"] == len(reqs)
    assert st["peak_inflight"] == 1
