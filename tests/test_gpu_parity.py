"""GPU parity of libcqfock.so (through the C ABI) against the reference's
golden data and the CPU oracle.  Tolerances: FP64 path max|dAX| <= 1e-9
(tests/func/contract.cxx:183 uses 1e-9); mixed path <= 1e-6 Eh."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

import oracle as O  # noqa: E402
from chronusq_public_b200 import workloads  # noqa: E402
from chronusq_public_b200.contraction import (  # noqa: E402
    COULOMB, EXCHANGE, DirectTPI, GTODirectTPIContraction, TwoBodyContraction)
from chronusq_public_b200.fockbuilder import (FockBuilder,  # noqa: E402
                                              two_electron_energy)
from helpers import (CONTRACT_CASES, contract_basis, golden,  # noqa: E402
                     readden_rhf_basis, tight_ao_scale, tight_d_basis)

FP64_TOL = 1e-9


@pytest.fixture(scope="module")
def contract_tpi():
    return DirectTPI(contract_basis())


@pytest.mark.parametrize("case", CONTRACT_CASES)
def test_contract_hdf5_cases(contract_tpi, case):
    g = golden("contract.npz")
    X = g[case + "_X"]
    AX = np.zeros_like(X, order="F")
    c = TwoBodyContraction(X, AX, bool(g[case + "_her"]), int(g[case + "_type"]))
    GTODirectTPIContraction(contract_tpi).twoBodyContract([c])
    assert np.abs(AX - g[case + "_AX"]).max() < FP64_TOL


def test_readden_rhf_build():
    g = golden("readden_rhf.npz")
    tpi = DirectTPI(readden_rhf_basis(g))
    S, T = tpi.one_electron()
    assert np.abs(S - g["S"]).max() < 1e-12
    assert np.abs(T - g["T"]).max() < 1e-9
    G, J, K = FockBuilder(tpi).formRawGD(g["D"])
    assert np.abs(G - (g["F"] - g["H"])).max() < FP64_TOL
    assert abs(two_electron_energy(G, g["D"]) - float(g["E_many_body"][0])) < 1e-8


def _oracle_and_device(name):
    mol, bname, nocc, seed = workloads.config(name)
    from chronusq_public_b200.basis import BasisSet
    basis = BasisSet.build(mol, bname)
    tpi = DirectTPI(basis)
    ob = O.OracleBasis(basis)
    S, _ = tpi.one_electron()
    So, _ = ob.overlap_kinetic()
    assert np.abs(S - So).max() < 1e-12
    D = workloads.occupied_density(S, nocc, seed)
    return basis, tpi, ob, D


def test_h2o_ccpvdz_fock_fp64():
    basis, tpi, ob, D = _oracle_and_device("h2o_ccpvdz")
    assert tpi.npair == len(ob.sig_pairs()[0])
    assert np.abs(tpi.schwarz() - ob.schwarz()).max() < 1e-12
    G, J, K = FockBuilder(tpi).formRawGD(D)
    Jo, Ko = ob.contract([D, D], [1, 1], [COULOMB, EXCHANGE])
    assert np.abs(J - Jo).max() < FP64_TOL
    assert np.abs(K - Ko).max() < FP64_TOL
    st = tpi and FockBuilder(tpi)
    assert st is not None


def test_h2o8_ccpvdz_fock_fp64_and_counts():
    basis, tpi, ob, D = _oracle_and_device("h2o8_ccpvdz")
    fb = FockBuilder(tpi)
    G, J, K = fb.formRawGD(D)
    Jo, Ko = ob.contract([D, D], [1, 1], [COULOMB, EXCHANGE])
    assert np.abs(2 * J - K - (2 * Jo - Ko)).max() < FP64_TOL
    s = fb.contraction.last_stats
    assert s["total"] == ob.last_stats["total"]
    assert s["screened"] == ob.last_stats["screened"]


def test_device_pointer_path_matches_host_path():
    import torch
    basis, tpi, ob, D = _oracle_and_device("h2o_ccpvdz")
    N = tpi.nbasis
    Jh = np.zeros((N, N), order="F")
    GTODirectTPIContraction(tpi).twoBodyContract(
        [TwoBodyContraction(D, Jh, True, COULOMB)])
    Dd = torch.from_numpy(np.asfortranarray(D)).cuda().t().contiguous().t()
    Jd = torch.zeros((N, N), dtype=torch.float64, device="cuda").t().contiguous().t()
    GTODirectTPIContraction(tpi).twoBodyContract(
        [TwoBodyContraction(Dd, Jd, True, COULOMB)])
    torch.cuda.synchronize()
    assert np.abs(Jd.cpu().numpy() - Jh).max() < 1e-12


def test_accumulate_semantics():
    basis, tpi, ob, D = _oracle_and_device("h2o_ccpvdz")
    N = tpi.nbasis
    J1 = np.zeros((N, N), order="F")
    c = GTODirectTPIContraction(tpi)
    c.twoBodyContract([TwoBodyContraction(D, J1, True, COULOMB)])
    J2 = J1.copy(order="F")
    c.twoBodyContract([TwoBodyContraction(D, J2, True, COULOMB)])
    assert np.abs(J2 - 2 * J1).max() < 1e-12


def test_output_buffers_and_increment():
    """Caller-owned J/K/G are zeroed and reused (the reference writes into
    the SingleSlater's matrices); an incremental build from dD accumulates
    into them, FP64 even when mixed is asked for (formGD, impl.hpp:80-88)."""
    basis, tpi, ob, D = _oracle_and_device("h2o_ccpvdz")
    N = tpi.nbasis
    fb = FockBuilder(tpi)
    J, K, G = (np.full((N, N), 7.0, order="F") for _ in range(3))
    G1, J1, K1 = fb.formRawGD(D, J=J, K=K, G=G)
    assert G1 is G and J1 is J and K1 is K
    Jo, Ko = ob.contract([D, D], [1, 1], [COULOMB, EXCHANGE])
    assert np.abs(J - Jo).max() < FP64_TOL
    assert np.abs(G - (2 * Jo - Ko)).max() < FP64_TOL
    rng = np.random.default_rng(11)
    X = rng.standard_normal((N, N))
    dD = np.asfortranarray(1e-3 * (X + X.T))
    fb.formRawGD(dD, J=J, K=K, G=G, increment=True, precision="mixed",
                 fp32_cutoff=1.0)
    Jo2, Ko2 = ob.contract([D + dD, D + dD], [1, 1], [COULOMB, EXCHANGE])
    assert np.abs(J - Jo2).max() < FP64_TOL
    assert np.abs(K - Ko2).max() < FP64_TOL
    assert fb.contraction.last_stats["fp32"] == 0
    with pytest.raises(ValueError):
        fb.formRawGD(D, J=np.zeros((N, N)), K=K)  # row-major output


def test_mixed_precision_within_1e6():
    basis, tpi, ob, D = _oracle_and_device("h2o8_ccpvdz")
    fb = FockBuilder(tpi)
    G64, _, _ = fb.formRawGD(D)
    Gm, _, _ = fb.formRawGD(D, precision="mixed", fp32_cutoff=1e-6)
    s = fb.contraction.last_stats
    assert s["fp32"] > 0
    assert np.abs(Gm - G64).max() <= 1e-6
    assert abs(two_electron_energy(Gm, D) - two_electron_energy(G64, D)) <= 1e-6


def test_mixed_precision_tight_primitives():
    """Quartets of very tight shells stay in FP64 on the mixed path even when
    their bound is below the cut (FP32 would overflow there)."""
    basis = tight_d_basis()
    tpi = DirectTPI(basis)
    ob = O.OracleBasis(basis)
    rng = np.random.default_rng(7)
    A = rng.standard_normal((basis.nbasis, basis.nbasis))
    f = tight_ao_scale(basis)
    D = 0.1 * (A + A.T) * f[:, None] * f[None, :]
    Jo, Ko = ob.contract([D, D], [1, 1], [0, 1])
    fb = FockBuilder(tpi)
    G, J, K = fb.formRawGD(D, precision="mixed", fp32_cutoff=1e-2)
    s = fb.contraction.last_stats
    assert s["fp32"] > 0 and s["fp64"] > 0, s
    assert np.isfinite(G).all()
    assert np.abs(J - Jo).max() <= 1e-6
    assert np.abs(K - Ko).max() <= 1e-6


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a).T)).cuda().t()


def test_batched_graph_matches_direct_calls():
    """64-density-style batch (here 6 dD + J/K) captured as a CUDA graph:
    replay == direct call, replays accumulate."""
    import torch
    from chronusq_public_b200.contraction import ContractionGraph
    basis, tpi, ob, D = _oracle_and_device("h2o_ccpvdz")
    N = tpi.nbasis
    dDs = workloads.delta_densities(N, 6, seed_base=400)
    Xs = [_dev(x) for x in dDs]
    outs = [torch.zeros((N, N), dtype=torch.float64, device="cuda").t() for _ in range(12)]
    cont = []
    for k, X in enumerate(Xs):
        cont.append(TwoBodyContraction(X, outs[2 * k], True, COULOMB))
        cont.append(TwoBodyContraction(X, outs[2 * k + 1], True, EXCHANGE))
    g = ContractionGraph(tpi, cont)
    g.launch()
    torch.cuda.synchronize()
    first = [o.cpu().numpy() for o in outs]
    g.launch()
    torch.cuda.synchronize()
    for o, f in zip(outs, first):
        assert np.abs(o.cpu().numpy() - 2 * f).max() < 1e-12
    Jo, Ko = ob.contract([dDs[0], dDs[0]], [1, 1], [COULOMB, EXCHANGE])
    assert np.abs(first[0] - Jo).max() < FP64_TOL
    assert np.abs(first[1] - Ko).max() < FP64_TOL
    g.close()


def test_many_densities_one_call_matches_oracle():
    basis, tpi, ob, D = _oracle_and_device("h2o_ccpvdz")
    N = tpi.nbasis
    dDs = workloads.delta_densities(N, 4, seed_base=400)
    fb = FockBuilder(tpi)
    Gs = fb.formRawGDBatch(dDs)
    for k, X in enumerate(dDs):
        Jo, Ko = ob.contract([X, X], [1, 1], [COULOMB, EXCHANGE])
        assert np.abs(Gs[k] - (2 * Jo - Ko)).max() < FP64_TOL


def _jk_vs_oracle(basis, seed=5):
    tpi = DirectTPI(basis)
    ob = O.OracleBasis(basis)
    N = basis.nbasis
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((N, N))
    D = 0.5 * (A + A.T)
    G, J, K = FockBuilder(tpi).formRawGD(D)
    Jo, Ko = ob.contract([D, D], [1, 1], [0, 1])
    assert np.abs(J - Jo).max() < FP64_TOL
    assert np.abs(K - Ko).max() < FP64_TOL
    return tpi


def test_edge_single_s_function():
    """N = 1: one H atom with one s shell (only the (ss|ss) class)."""
    from chronusq_public_b200.basis import BasisSet, Molecule, parse_gbs
    gbs = "****\nH 0\nS 1 1.00\n  0.8 1.0\n****\n"
    basis = BasisSet.build(Molecule.from_angstrom([("H", 0.0, 0.0, 0.0)]), parse_gbs(gbs))
    assert basis.nbasis == 1
    _jk_vs_oracle(basis)


def test_edge_distant_fragments_insignificant_pairs():
    """Two waters 60 Angstrom apart: no significant pair links them, the
    quartet list is two disconnected blocks."""
    from chronusq_public_b200.basis import BasisSet, Molecule
    w = workloads.water()
    xyz = np.vstack([w.xyz, w.xyz + np.array([60.0 / 0.52917721092, 0.0, 0.0])])
    mol = Molecule(np.concatenate([w.Z, w.Z]), xyz)
    basis = BasisSet.build(mol, "cc-pvdz")
    tpi = _jk_vs_oracle(basis)
    assert tpi.npair < basis.nshell * (basis.nshell + 1) // 2


def test_edge_empty_contraction_list():
    basis = contract_basis()
    tpi = DirectTPI(basis)
    GTODirectTPIContraction(tpi).twoBodyContract([])  # a no-op, no error
    import ctypes as C
    from chronusq_public_b200 import _cabi
    # the C ABI refuses an empty list with a status (the Python mirror, like
    # the reference's loop, does nothing)
    st = _cabi.CqfStats()
    assert _cabi.lib().cqf_two_body_contract(tpi.handle, None, 0, None,
                                             C.byref(st)) == _cabi.CQF_EINVAL


def test_nonhermitian_real_coulomb_fast_path():
    """Real non-Hermitian J (MOIntsTransformer's pseudo-densities) runs on the
    fast kernels through its symmetric part; it must match the oracle's
    non-Hermitian branch, several densities in one call."""
    basis, tpi, ob, D = _oracle_and_device("h2o8_ccpvdz")
    rng = np.random.default_rng(17)
    N = basis.nbasis
    Xs = [np.asfortranarray(0.1 * rng.standard_normal((N, N))) for _ in range(3)]
    outs = [np.zeros((N, N), order="F") for _ in Xs]
    GTODirectTPIContraction(tpi).twoBodyContract(
        [TwoBodyContraction(X, J, False, COULOMB) for X, J in zip(Xs, outs)])
    refs = ob.contract(Xs, [0, 0, 0], [0, 0, 0])
    for J, Jo in zip(outs, refs):
        assert np.abs(J - Jo).max() < FP64_TOL


def _herm_complex(N, seed, scale=0.1):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
    return np.asfortranarray(scale * 0.5 * (A + A.conj().T))


@pytest.mark.parametrize("name", ["h2o_ccpvdz", "h2o8_ccpvdz"])
def test_complex_hermitian_fast_split(name):
    """Complex Hermitian J and K (s..d basis) through the real fast kernels
    -- J[S], K[S] + i K[A] for X = S + iA -- against the oracle's complex
    Hermitian branch; AX accumulates into what it held."""
    basis, tpi, ob, _D = _oracle_and_device(name)
    N = basis.nbasis
    X1, X2 = _herm_complex(N, 31), _herm_complex(N, 32)
    J = np.asfortranarray(np.full((N, N), 0.25 + 0.5j))
    K1 = np.zeros((N, N), complex, order="F")
    K2 = np.zeros((N, N), complex, order="F")
    GTODirectTPIContraction(tpi).twoBodyContract(
        [TwoBodyContraction(X1, J, True, COULOMB), TwoBodyContraction(X1, K1, True, EXCHANGE),
         TwoBodyContraction(X2, K2, True, EXCHANGE)])
    Jo, K1o, K2o = ob.contract([X1, X1, X2], [1, 1, 1], [0, 1, 1])
    assert np.abs(J - (Jo + (0.25 + 0.5j))).max() < FP64_TOL
    assert np.abs(K1 - K1o).max() < FP64_TOL
    assert np.abs(K2 - K2o).max() < FP64_TOL
    assert np.abs(K1.imag).max() > 1e-3  # the antisymmetric part is exercised


def test_complex_hermitian_fast_split_device_pointers():
    import torch
    basis, tpi, ob, _D = _oracle_and_device("h2o_ccpvdz")
    N = basis.nbasis
    X = _herm_complex(N, 33)
    Xd = torch.from_numpy(np.ascontiguousarray(X.T)).cuda().t()
    Jd = torch.zeros((N, N), dtype=torch.complex128, device="cuda").t()
    Kd = torch.zeros((N, N), dtype=torch.complex128, device="cuda").t()
    GTODirectTPIContraction(tpi).twoBodyContract(
        [TwoBodyContraction(Xd, Jd, True, COULOMB), TwoBodyContraction(Xd, Kd, True, EXCHANGE)])
    torch.cuda.synchronize()
    Jo, Ko = ob.contract([X, X], [1, 1], [0, 1])
    assert np.abs(Jd.cpu().numpy() - Jo).max() < FP64_TOL
    assert np.abs(Kd.cpu().numpy() - Ko).max() < FP64_TOL


def test_complex_hermitian_f_shells_generic():
    """With f shells the complex Hermitian build stays on the generic kernel."""
    basis = contract_basis()
    assert basis.max_l == 3
    tpi = DirectTPI(basis)
    ob = O.OracleBasis(basis)
    X = _herm_complex(basis.nbasis, 34, 0.05)
    N = basis.nbasis
    K = np.zeros((N, N), complex, order="F")
    GTODirectTPIContraction(tpi).twoBodyContract([TwoBodyContraction(X, K, True, EXCHANGE)])
    Ko, = ob.contract([X], [1], [1])
    assert np.abs(K - Ko).max() < FP64_TOL


def test_complex_hermitian_graph_split():
    """Complex Hermitian J/K (the density of an RT-TDDFT step) captured as a
    CUDA graph on the real split: the first replay matches the oracle, the
    second accumulates the same again."""
    import torch
    from chronusq_public_b200.contraction import ContractionGraph
    basis, tpi, ob, _D = _oracle_and_device("h2o_ccpvdz")
    N = tpi.nbasis
    Xs = [_herm_complex(N, 40 + k) for k in range(3)]
    Xd = [torch.from_numpy(np.ascontiguousarray(x.T)).cuda().t() for x in Xs]
    outs = [torch.zeros((N, N), dtype=torch.complex128, device="cuda").t() for _ in range(6)]
    cont = []
    for k, X in enumerate(Xd):
        cont.append(TwoBodyContraction(X, outs[2 * k], True, COULOMB))
        cont.append(TwoBodyContraction(X, outs[2 * k + 1], True, EXCHANGE))
    g = ContractionGraph(tpi, cont)
    g.launch()
    torch.cuda.synchronize()
    first = [o.cpu().numpy() for o in outs]
    g.launch()
    torch.cuda.synchronize()
    for o, f in zip(outs, first):
        assert np.abs(o.cpu().numpy() - 2 * f).max() < 1e-12
    for k, X in enumerate(Xs):
        Jo, Ko = ob.contract([X, X], [1, 1], [COULOMB, EXCHANGE])
        assert np.abs(first[2 * k] - Jo).max() < FP64_TOL
        assert np.abs(first[2 * k + 1] - Ko).max() < FP64_TOL
    g.close()


def test_autotune_sets_shapes_and_caches(tmp_path):
    """cqf_autotune times the candidate launch shapes per class pair, keeps
    the fastest, leaves the results unchanged, and a second basis of the same
    system takes every choice from the cache file without timing."""
    basis, tpi, ob, D = _oracle_and_device("h2o8_ccpvdz")
    cache = str(tmp_path / "launch_shapes.txt")
    assert tpi.autotune(D, cache_path=cache) is False
    lines = open(cache).read().splitlines()
    assert lines and all(int(l.split()[-1]) in (2, 4, 8, 16) for l in lines)
    _G, J, K = FockBuilder(tpi).formRawGD(D)
    Jo, Ko = ob.contract([D, D], [1, 1], [0, 1])
    assert np.abs(J - Jo).max() < FP64_TOL
    assert np.abs(K - Ko).max() < FP64_TOL
    tpi2 = DirectTPI(basis)
    assert tpi2.autotune(D, cache_path=cache) is True
    assert open(cache).read().splitlines() == lines
    _G2, J2, K2 = FockBuilder(tpi2).formRawGD(D)
    assert np.abs(J2 - Jo).max() < FP64_TOL and np.abs(K2 - Ko).max() < FP64_TOL
