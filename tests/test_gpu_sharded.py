"""The sharded build on the GPU (cqf_opts::shard_index / shard_count): the
shards' results sum to the whole build on every kernel path -- the 1C fast
path (FP64 and mixed), the generic path (f shells, complex non-Hermitian),
and the whole 4C build with every term on -- and two processes sharing one
GPU through a gloo group reproduce the single-process build."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.contraction import (COULOMB, EXCHANGE, DirectTPI,
                                              GTODirectTPIContraction, TwoBodyContraction)
from chronusq_public_b200.fockbuilder import FourCompFock
from helpers import water_ref
from test_gpu_gaunt import gaunt_inputs
from test_gpu_rel import f_basis, water_631gd

pytestmark = pytest.mark.gpu


def _jk(tpi, mats, her, shard, **kw):
    N = tpi.nbasis
    out = []
    lst = []
    for X, h in zip(mats, her):
        dt = np.complex128 if np.iscomplexobj(X) else np.float64
        for t in (COULOMB, EXCHANGE):
            A = np.zeros((N, N), dtype=dt, order="F")
            out.append(A)
            lst.append(TwoBodyContraction(X, A, h, t))
    GTODirectTPIContraction(tpi).twoBodyContract(lst, shard=shard, **kw)
    return out


@pytest.mark.parametrize("case", ["fast_fp64", "fast_mixed", "f_shells", "complex_nonher"])
def test_shards_sum_to_the_whole_1c(case):
    rng = np.random.default_rng(41)
    bs = f_basis() if case == "f_shells" else BasisSet.build(water_ref(), "cc-pvdz")
    tpi = DirectTPI(bs)
    N = bs.nbasis
    A = rng.standard_normal((N, N))
    if case == "complex_nonher":
        mats = [0.1 * (A + 1j * rng.standard_normal((N, N)))]
        her = [False]
    else:
        mats = [0.1 * (A + A.T)]
        her = [True]
    kw = dict(precision="mixed", fp32_cutoff=1e-2) if case == "fast_mixed" else {}
    whole = _jk(tpi, mats, her, (0, 1), **kw)
    parts = [_jk(tpi, mats, her, (k, 3), **kw) for k in range(3)]
    for m in range(len(whole)):
        assert all(np.abs(p[m]).max() > 0 for p in parts), m  # each shard has work
        s = parts[0][m] + parts[1][m] + parts[2][m]
        tol = 1e-6 if case == "fast_mixed" else 1e-12
        assert np.abs(s - whole[m]).max() < tol * max(1.0, np.abs(whole[m]).max()), m


def test_shards_sum_to_the_whole_4c():
    bs = water_631gd()
    tpi = DirectTPI(bs)
    D, _X = gaunt_inputs(bs.nbasis, 42)
    fb = FourCompFock(tpi, Gaunt=True, Gauge=True)
    whole = fb.formGD(D)
    parts = [_four_comp_shard(fb, D, (k, 2)) for k in range(2)]
    for c in range(4):
        s = parts[0][c] + parts[1][c]
        assert np.abs(parts[0][c]).max() > 0 and np.abs(parts[1][c]).max() > 0
        assert np.abs(s - whole[c]).max() < 1e-11 * max(1.0, np.abs(whole[c]).max()), c


def _four_comp_shard(fb, D, shard):
    """formGD of one shard (the process-group path with a fixed shard)."""
    import chronusq_public_b200.fockbuilder as F
    saved = F._shard_of
    F._shard_of = lambda group: shard
    try:
        return fb.formGD(D)
    finally:
        F._shard_of = saved


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "oracle"), os.path.join(root, "tests")):
        sys.path.insert(0, p)
    import torch.distributed as dist

    from chronusq_public_b200.fockbuilder import FockBuilder, FourCompFock as FCF
    from test_gpu_gaunt import gaunt_inputs as gi
    from test_gpu_rel import water_631gd as w631
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world)
    try:
        bs = w631()
        tpi = DirectTPI(bs, device=0)
        N = bs.nbasis
        rng = np.random.default_rng(43)
        A = rng.standard_normal((N, N))
        D = 0.1 * (A + A.T)
        G1, _, _ = FockBuilder(tpi).formRawGD(D)
        Gs, _, _ = FockBuilder(tpi, group=dist.group.WORLD).formRawGD(D)
        D4, _ = gi(N, 44)
        H1 = FCF(tpi, Gaunt=True).formGD(D4)
        Hs = FCF(tpi, Gaunt=True, group=dist.group.WORLD).formGD(D4)
        e1 = float(np.abs(Gs - G1).max())
        e4 = max(float(np.abs(Hs[c] - H1[c]).max()) for c in range(4))
        out.put((rank, e1, e4))
    finally:
        dist.destroy_process_group()


def test_two_processes_one_gpu_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(900)
        assert p.exitcode == 0
    for rank, e1, e4 in sorted(q.get(timeout=10) for _ in range(2)):
        assert e1 < 1e-11, (rank, e1)
        assert e4 < 1e-11, (rank, e4)
