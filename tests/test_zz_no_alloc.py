"""cqf_two_body_contract_noalloc against cqf_two_body_contract.

Some callers of the J/K contraction cannot allocate device memory during the
call: a host program whose framework owns all of the GPU's memory, or a
latency-critical loop that cannot afford cudaFree's device synchronisation.  For them the library has an entry point that takes its
scratch from one fixed array compiled into libcqfock.so instead of growing a
workspace with cudaMalloc.  This file checks, through the C ABI, that two
calls in a row of that entry point give the regular entry point's J and K on
the same inputs (FP64 tolerance 1e-9) -- real and complex Hermitian
densities, and HER given as any nonzero value or as 0 -- that the calls leave
the device's free memory unchanged, and that a call needing more scratch
than the array holds is refused without touching its outputs.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from chronusq_public_b200 import _cabi, workloads  # noqa: E402
from chronusq_public_b200.basis import BasisSet  # noqa: E402
from chronusq_public_b200.contraction import DirectTPI  # noqa: E402

FP64_TOL = 1e-9


def _contract(entry, tpi, D, outs, types, device_pointers=False, her=1):
    n = len(outs)
    arr = (_cabi.CqfContraction * n)()
    for i, (AX, ty) in enumerate(zip(outs, types)):
        arr[i].X = C.c_void_p(D.ctypes.data if not device_pointers else D.data_ptr())
        arr[i].AX = C.c_void_p(AX.ctypes.data if not device_pointers else AX.data_ptr())
        arr[i].hermitian = her
        arr[i].type = ty
    opts = _cabi.CqfOpts()
    _cabi.lib().cqf_opts_default(C.byref(opts))
    opts.device_pointers = 1 if device_pointers else 0
    cplx = D.is_complex() if device_pointers else np.iscomplexobj(D)
    opts.is_complex = 1 if cplx else 0
    st = _cabi.CqfStats()
    return entry(tpi.handle, arr, n, C.byref(opts), C.byref(st))


@pytest.fixture(scope="module")
def setup():
    mol, bname, nocc, seed = workloads.config("h2o8_ccpvdz")
    tpi = DirectTPI(BasisSet.build(mol, bname))
    S, _ = tpi.one_electron()
    D = np.asfortranarray(workloads.occupied_density(S, nocc, seed))
    return tpi, D


def test_noalloc_matches_regular_entry_twice(setup):
    tpi, D = setup
    L = _cabi.lib()
    N = tpi.nbasis
    J0, K0 = np.zeros((N, N), order="F"), np.zeros((N, N), order="F")
    assert _contract(L.cqf_two_body_contract, tpi, D, [J0, K0],
                     [_cabi.CQF_COULOMB, _cabi.CQF_EXCHANGE]) == _cabi.CQF_OK
    for _ in range(2):
        J, K = np.zeros((N, N), order="F"), np.zeros((N, N), order="F")
        st = _contract(L.cqf_two_body_contract_noalloc, tpi, D, [J, K],
                       [_cabi.CQF_COULOMB, _cabi.CQF_EXCHANGE])
        assert st == _cabi.CQF_OK, L.cqf_last_error()
        assert np.abs(J - J0).max() < FP64_TOL
        assert np.abs(K - K0).max() < FP64_TOL


def _free_bytes():
    import torch
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0]


@pytest.mark.parametrize("her", [-1, 0, 2])
def test_noalloc_hermitian_flag_as_regular_entry(setup, her):
    """HER is a bool in the reference: -1 and 2 mean Hermitian, as 1 does,
    and 0 takes the non-Hermitian branch on both entry points."""
    tpi, D = setup
    L = _cabi.lib()
    N = tpi.nbasis
    types = [_cabi.CQF_COULOMB, _cabi.CQF_EXCHANGE]
    J1, K1 = np.zeros((N, N), order="F"), np.zeros((N, N), order="F")
    assert _contract(L.cqf_two_body_contract, tpi, D, [J1, K1], types, her=1) == _cabi.CQF_OK
    J0, K0 = np.zeros((N, N), order="F"), np.zeros((N, N), order="F")
    assert _contract(L.cqf_two_body_contract, tpi, D, [J0, K0], types, her=her) == _cabi.CQF_OK
    for _ in range(2):
        J, K = np.zeros((N, N), order="F"), np.zeros((N, N), order="F")
        st = _contract(L.cqf_two_body_contract_noalloc, tpi, D, [J, K], types, her=her)
        assert st == _cabi.CQF_OK, L.cqf_last_error()
        assert np.abs(J - J0).max() < FP64_TOL
        assert np.abs(K - K0).max() < FP64_TOL
        # D is symmetric: every flag gives the Hermitian result
        assert np.abs(J - J1).max() < FP64_TOL
        assert np.abs(K - K1).max() < FP64_TOL


def test_noalloc_complex_hermitian(setup):
    """A complex Hermitian density D + iA takes the same symmetric /
    antisymmetric split on both entry points."""
    tpi, D = setup
    L = _cabi.lib()
    N = tpi.nbasis
    rng = np.random.default_rng(5)
    A = rng.standard_normal((N, N))
    Z = np.asfortranarray(D + 0.01j * (A - A.T))
    types = [_cabi.CQF_COULOMB, _cabi.CQF_EXCHANGE]
    J0 = np.zeros((N, N), complex, order="F")
    K0 = np.zeros((N, N), complex, order="F")
    assert _contract(L.cqf_two_body_contract, tpi, Z, [J0, K0], types) == _cabi.CQF_OK
    for _ in range(2):
        J = np.zeros((N, N), complex, order="F")
        K = np.zeros((N, N), complex, order="F")
        st = _contract(L.cqf_two_body_contract_noalloc, tpi, Z, [J, K], types)
        assert st == _cabi.CQF_OK, L.cqf_last_error()
        assert np.abs(J - J0).max() < FP64_TOL
        assert np.abs(K - K0).max() < FP64_TOL


def test_noalloc_leaves_free_memory_unchanged(setup):
    """After one regular call (which loads the kernels), no-alloc calls do not
    change the device's free memory: the scratch array was mapped when the
    basis was created."""
    tpi, D = setup
    L = _cabi.lib()
    N = tpi.nbasis
    types = [_cabi.CQF_COULOMB, _cabi.CQF_EXCHANGE]
    J, K = np.zeros((N, N), order="F"), np.zeros((N, N), order="F")
    assert _contract(L.cqf_two_body_contract, tpi, D, [J, K], types) == _cabi.CQF_OK
    free0 = _free_bytes()
    for _ in range(2):
        J, K = np.zeros((N, N), order="F"), np.zeros((N, N), order="F")
        assert _contract(L.cqf_two_body_contract_noalloc, tpi, D, [J, K],
                         types) == _cabi.CQF_OK, L.cqf_last_error()
    assert _free_bytes() == free0


def test_noalloc_device_pointers(setup):
    import torch
    tpi, D = setup
    L = _cabi.lib()
    N = tpi.nbasis
    J0 = np.zeros((N, N), order="F")
    assert _contract(L.cqf_two_body_contract, tpi, D, [J0],
                     [_cabi.CQF_COULOMB]) == _cabi.CQF_OK
    Dd = torch.from_numpy(np.ascontiguousarray(D.T)).cuda().t()
    for _ in range(2):
        Jd = torch.zeros((N, N), dtype=torch.float64, device="cuda").t()
        st = _contract(L.cqf_two_body_contract_noalloc, tpi, Dd, [Jd],
                       [_cabi.CQF_COULOMB], device_pointers=True)
        assert st == _cabi.CQF_OK, L.cqf_last_error()
        torch.cuda.synchronize()
        assert np.abs(Jd.cpu().numpy() - J0).max() < FP64_TOL


def test_noalloc_rejects_oversized_call(setup):
    tpi, D = setup
    L = _cabi.lib()
    N = tpi.nbasis
    # 100 host-pointer contractions need far more than the fixed array
    outs = [np.full((N, N), 7.0, order="F") for _ in range(100)]
    st = _contract(L.cqf_two_body_contract_noalloc, tpi, D, outs,
                   [_cabi.CQF_COULOMB] * 100)
    assert st == _cabi.CQF_EINVAL
    assert b"scratch" in L.cqf_last_error()
    assert all((o == 7.0).all() for o in outs)
