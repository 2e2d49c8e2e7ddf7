"""C-ABI library and host logic checks that need no GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from chronusq_public_b200 import _cabi, workloads
from chronusq_public_b200.basis import (BasisSet, cart_list, load_gbs,
                                        solid_harmonic_matrix)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_functions():
    txt = open(os.path.join(ROOT, "include", "cqfock.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cqf_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    lib = _cabi.lib()
    names = _header_functions()
    assert names, "no functions parsed from include/cqfock.h"
    for n in names:
        assert hasattr(lib, n), n
    assert sorted(_cabi.EXPORTS) == names


def test_no_device_reports_enodev_or_works():
    """Without a GPU, basis creation must fail with a status, not crash."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    lib = _cabi.lib()
    sh = (_cabi.CqfShell * 1)()
    a = (ctypes.c_double * 1)(1.0)
    c = (ctypes.c_double * 1)(1.0)
    sh[0].l, sh[0].pure, sh[0].nprim = 0, 0, 1
    sh[0].alpha = ctypes.cast(a, ctypes.POINTER(ctypes.c_double))
    sh[0].coeff = ctypes.cast(c, ctypes.POINTER(ctypes.c_double))
    h = ctypes.c_void_p()
    st = lib.cqf_basis_create(sh, 1, 1e-12, 0, ctypes.byref(h))
    assert st in (_cabi.CQF_ENODEV, _cabi.CQF_ECUDA)
    assert lib.cqf_last_error()


def test_bad_arguments_are_rejected():
    lib = _cabi.lib()
    h = ctypes.c_void_p()
    assert lib.cqf_basis_create(None, 0, 1e-12, 0, ctypes.byref(h)) == \
        _cabi.CQF_EINVAL
    assert lib.cqf_two_body_contract(None, None, 0, None, None) == \
        _cabi.CQF_EINVAL


def test_solid_harmonics_orthonormal():
    # with x^l-normalised Cartesian Gaussians the real solid harmonics are
    # unit-normalised and orthogonal: T^T M T = I with M the Cartesian
    # overlap metric of one centre (double factorial products)
    from math import prod

    def df(n):
        return prod(range(n, 0, -2)) if n > 0 else 1

    for l in range(5):
        carts = cart_list(l)
        M = np.zeros((len(carts), len(carts)))
        for i, a in enumerate(carts):
            for j, b in enumerate(carts):
                s = [a[k] + b[k] for k in range(3)]
                if any(x % 2 for x in s):
                    continue
                M[i, j] = prod(df(x - 1) for x in s) / df(2 * l - 1)
        T = solid_harmonic_matrix(l)
        assert np.allclose(T.T @ M @ T, np.eye(2 * l + 1), atol=1e-13)


def test_basis_sizes_of_the_workloads():
    mol, bname, nocc, seed = workloads.config("h2o_ccpvdz")
    assert BasisSet.build(mol, bname).nbasis == 24
    mol, bname, nocc, seed = workloads.config("h2o16_def2svp")
    b = BasisSet.build(mol, bname)
    assert b.nbasis == 384 and b.nshell == 192 and b.max_l == 2


def test_cluster_is_deterministic_and_respects_oo_distance():
    m1 = workloads.water_cluster(16, seed=2)
    m2 = workloads.water_cluster(16, seed=2)
    assert np.array_equal(m1.xyz, m2.xyz)
    O = m1.xyz[m1.Z == 8] * 0.52917721092
    d = np.linalg.norm(O[:, None] - O[None], axis=-1) + np.eye(len(O)) * 99
    assert d.min() >= 2.6 - 1e-12


def test_gbs_parser_splits_sp_and_sets_pure():
    g = load_gbs("def2-svp")
    ls = [(l, pure) for (l, pure, e, c) in g[8]]
    assert ls == [(0, False), (0, False), (0, False), (1, False), (1, False),
                  (2, True)]


def test_flop_model_matches_oracle_count():
    import oracle as O
    from chronusq_public_b200 import flops as FL
    mol, bname, nocc, seed = workloads.config("h2o_ccpvdz")
    basis = BasisSet.build(mol, bname)
    ob = O.OracleBasis(basis)
    S, _ = ob.overlap_kinetic()
    D = workloads.occupied_density(S, nocc, seed)
    Q = ob.schwarz()
    sig = np.zeros_like(Q)
    a, b = ob.sig_pairs()
    sig[a, b] = Q[a, b]
    mine = FL.build_flops(basis, sig, [D], nmat_digest=1, fp32_cut=1e-3)
    ref = ob.flops([D], fp32_cut=1e-3)
    assert mine["quartets"] == ref["quartets"]
    assert abs(mine["f64"] - ref["f64"]) <= 1e-9 * ref["f64"]
    assert abs(mine["f32"] - ref["f32"]) <= 1e-9 * max(ref["f32"], 1.0)


def _footprint_model(basis, nmat=2):
    """The server's footprint formula restated (cqf_fock_footprint)."""
    ns, N, nc = basis.nshell, basis.nbasis, basis.ncart
    npair = ns * (ns + 1) // 2
    kprim = basis.max_prim ** 2
    pairs = npair * (72 + (112 + 48 + 8 + 104 + 52) * kprim) + ns * ns * 8 + 300_000
    masks = 3 * 16 * min(npair * ((npair + 31) // 32), 1 << 18)
    ws = (8 * (2 * nmat * N * N + 2 * nmat * nc * nc + (nmat + 1) * ns * ns)
          + 4 * nmat * nc * nc + masks)
    return pairs + ws


def test_server_footprint_matches_model():
    from chronusq_public_b200.serving import footprint_bytes
    for nw, b in ((1, "cc-pvdz"), (3, "def2-svp")):
        basis = BasisSet.build(workloads.water_cluster(nw, seed=3, box=6.0), b)
        assert footprint_bytes(basis) == _footprint_model(basis)


def test_server_rejects_bad_arguments():
    L = _cabi.lib()
    o = _cabi.CqfServerOpts()
    L.cqf_server_opts_default(ctypes.byref(o))
    assert (o.slots, o.cache_entries) == (8, 16)
    o.slots = 0
    h = ctypes.c_void_p()
    assert L.cqf_server_create(ctypes.byref(o), ctypes.byref(h)) == _cabi.CQF_EINVAL
    o.slots = 2
    assert L.cqf_server_create(ctypes.byref(o), ctypes.byref(h)) == _cabi.CQF_OK
    q = _cabi.CqfFockRequest()
    rid = ctypes.c_longlong()
    assert L.cqf_server_submit(h, ctypes.byref(q), ctypes.byref(rid)) == _cabi.CQF_EINVAL
    assert L.cqf_server_wait(h, 12345, 0.0, None) == _cabi.CQF_EINVAL
    assert b"unknown request" in L.cqf_last_error()
    assert L.cqf_server_destroy(h) == _cabi.CQF_OK


def test_server_reports_failed_requests_without_device():
    """Without a GPU every request fails in basis set-up; the server reports
    the status and its text to the waiter, counts the failures and shuts
    down cleanly."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    from chronusq_public_b200.contraction import shell_array
    L = _cabi.lib()
    basis = BasisSet.build(workloads.water_cluster(1, seed=3, box=6.0), "cc-pvdz")
    sh, keep = shell_array(basis)
    N = basis.nbasis
    D = np.asfortranarray(np.eye(N))
    G = np.zeros((N, N), order="F")
    o = _cabi.CqfServerOpts()
    L.cqf_server_opts_default(ctypes.byref(o))
    o.slots = 2
    h = ctypes.c_void_p()
    assert L.cqf_server_create(ctypes.byref(o), ctypes.byref(h)) == _cabi.CQF_OK
    dp = ctypes.POINTER(ctypes.c_double)
    q = _cabi.CqfFockRequest(sh, basis.nshell, 1e-12, D.ctypes.data_as(dp),
                             G.ctypes.data_as(dp), 1.0, _cabi.CQF_FP64, 0.0)
    ids = []
    for _ in range(3):
        rid = ctypes.c_longlong()
        assert L.cqf_server_submit(h, ctypes.byref(q), ctypes.byref(rid)) == _cabi.CQF_OK
        ids.append(rid.value)
    assert len(set(ids)) == 3
    for rid in ids:
        info = _cabi.CqfRequestInfo()
        st = L.cqf_server_wait(h, rid, 30.0, ctypes.byref(info))
        assert st == _cabi.CQF_ENODEV and info.status == _cabi.CQF_ENODEV
        assert b"no CUDA device" in L.cqf_last_error()
    s = _cabi.CqfServerStats()
    assert L.cqf_server_get_stats(h, ctypes.byref(s)) == _cabi.CQF_OK
    assert (s.submitted, s.completed, s.failed) == (3, 0, 3)
    assert (G == 0).all()
    assert L.cqf_server_destroy(h) == _cabi.CQF_OK
