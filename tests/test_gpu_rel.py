"""Four-component Dirac-Coulomb build on the GPU (cqf_rel_two_body_contract,
cqf_four_comp_gd) against the oracle's restatement of directScaffoldLibcint /
formGDDirect and against the reference's own 4C golden builds."""
import numpy as np
import pytest

import oracle as O
from chronusq_public_b200.basis import BasisSet, Molecule, parse_gbs
from chronusq_public_b200.contraction import (BARE_COULOMB, LLSS, SSSS, DirectTPI,
                                              GTODirectRelERIContraction,
                                              TwoBodyContraction)
from chronusq_public_b200.fockbuilder import FourCompFock
from chronusq_public_b200.workloads import SPEED_OF_LIGHT
from helpers import golden, tight_ao_scale, tight_d_basis, water_ref

pytestmark = pytest.mark.gpu

PAULI = ("SCALAR", "MX", "MY", "MZ")

# a small two-centre basis with f shells on both centres (exercises the
# (ff|ff) classes and the LM = 3 kernels)
F_BASIS = """
****
He 0
S 2 1.00
  4.0 0.4
  0.9 0.7
S 1 1.00
  0.35 1.0
P 1 1.00
  1.1 1.0
D 1 1.00
  0.8 1.0
F 1 1.00
  0.7 1.0
****
H 0
S 2 1.00
  3.0 0.3
  0.5 0.8
P 1 1.00
  0.6 1.0
F 1 1.00
  0.9 1.0
****
"""


def f_basis():
    mol = Molecule.from_angstrom([("He", 0.0, 0.0, 0.0), ("H", 0.3, -0.2, 1.1)])
    return BasisSet.build(mol, parse_gbs(F_BASIS))


def water_631gd():
    return BasisSet.build(water_ref(), "6-31gd")


def herm(n, rng, scale=1.0):
    A = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    return scale * 0.5 * (A + A.conj().T)


def rel_inputs(N, seed):
    """The 17 X entries of a 4C contraction from random Hermitian Pauli
    components of a 2N x 2N density (LL, SS blocks Hermitian, LS general)."""
    rng = np.random.default_rng(seed)
    D = [herm(2 * N, rng, 0.1) for _ in range(4)]
    LL = [d[:N, :N] for d in D]
    SS = [d[N:, N:] for d in D]
    LS = [d[:N, N:] for d in D]
    X = [LL[0]] + LL + SS + SS + LS
    return D, [np.asfortranarray(x) for x in X]


def max_rel(a, b):
    return np.abs(a - b).max() / max(1.0, np.abs(b).max())


@pytest.fixture(scope="module")
def w631():
    bs = water_631gd()
    return bs, DirectTPI(bs), O.OracleBasis(bs)


@pytest.fixture(scope="module")
def fsys():
    bs = f_basis()
    return bs, DirectTPI(bs), O.OracleBasis(bs)


def _rel_case(sysfix, ctype, exchange, seed):
    bs, tpi, ob = sysfix
    N = bs.nbasis
    _D, X = rel_inputs(N, seed)
    ref = ob.rel_contract(X, ctype, exchange)
    lst = [TwoBodyContraction(X[m], np.zeros((N, N), complex)) for m in range(17)]
    GTODirectRelERIContraction(tpi).twoBodyContract(lst, ctype, computeExchange=exchange)
    return [c.AX for c in lst], ref


# outputs each type writes (direct4C_libcint.hpp:514, :810, :1841)
OUTS = {BARE_COULOMB: [0, 1, 2, 3, 4], LLSS: [0, 5, 6, 7, 8, 13, 14, 15, 16],
        SSSS: [5, 6, 7, 8, 9, 10, 11, 12]}


@pytest.mark.parametrize("ctype", [BARE_COULOMB, LLSS, SSSS])
def test_rel_contract_water(w631, ctype):
    got, ref = _rel_case(w631, ctype, True, 11 + ctype)
    for m in range(17):
        if m in OUTS[ctype]:
            assert np.abs(ref[m]).max() > 0, m
            assert max_rel(got[m], ref[m]) < 1e-11, m
        else:
            assert np.abs(got[m]).max() == 0, m


@pytest.mark.parametrize("ctype", [LLSS, SSSS])
def test_rel_contract_f_shells(fsys, ctype):
    got, ref = _rel_case(fsys, ctype, True, 21 + ctype)
    for m in OUTS[ctype]:
        assert max_rel(got[m], ref[m]) < 1e-11, m


def test_rel_contract_no_exchange(w631):
    got, ref = _rel_case(w631, LLSS, False, 5)
    for m in range(17):
        assert max_rel(got[m], ref[m]) < 1e-11, m
    assert all(np.abs(got[m]).max() == 0 for m in (13, 14, 15, 16))


def test_four_comp_gd_qn_golden():
    """Converged complex 4C-HF water / 6-31G(d): BareCoulomb (1C path,
    non-libcint) + Dirac-Coulomb LLSS, SSSS off -- G = F - H of the
    reference's stored build, FP64 bar 1e-9."""
    g = golden("qn_4chf_dc.npz")
    tpi = DirectTPI(water_631gd())
    fb = FourCompFock(tpi, DiracCoulombSSSS=False, Libcint=False)
    G = fb.formGD([g["D_" + c] for c in PAULI])
    for k, c in enumerate(PAULI):
        assert np.abs(G[k] - g["G_" + c]).max() < 1e-9, c


def test_four_comp_gd_readden_golden():
    """libcint bare Coulomb of the DC-HF-guess READDEN build (LL blocks)."""
    g = golden("readden_dchf_ll.npz")
    bs = BasisSet.build(water_ref(), parse_gbs(str(golden("readden_dc.npz")["basisdef"])))
    tpi = DirectTPI(bs)
    N = bs.nbasis
    D = []
    for c in PAULI:
        d = np.zeros((2 * N, 2 * N), complex)
        d[:N, :N] = g["D_" + c]
        D.append(d)
    G = FourCompFock(tpi, DiracCoulomb=False, DiracCoulombSSSS=False).formGD(D)
    for k, c in enumerate(PAULI):
        assert np.abs(G[k][:N, :N] - g["G_" + c]).max() < 1e-9, c


@pytest.mark.parametrize("libcint", [True, False])
def test_four_comp_gd_full_vs_oracle(w631, libcint):
    bs, tpi, ob = w631
    D, _X = rel_inputs(bs.nbasis, 3)
    ref = ob.dirac_coulomb(D, bare=True, dc=True, ssss=True, libcint=libcint)
    G = FourCompFock(tpi, Libcint=libcint).formGD(D)
    for k in range(4):
        assert np.abs(G[k] - ref[k]).max() < 1e-9, k


def test_four_comp_gd_device_pointers(w631):
    torch = pytest.importorskip("torch")
    bs, tpi, _ob = w631
    D, _X = rel_inputs(bs.nbasis, 4)
    fb = FourCompFock(tpi)
    Gh = fb.formGD(D)
    Dd = [torch.from_numpy(np.asfortranarray(d)).cuda().T.contiguous().T for d in D]
    Gd = fb.formGD(Dd)
    for k in range(4):
        assert np.abs(Gd[k].cpu().numpy() - Gh[k]).max() < 1e-12


def test_four_comp_gd_hermitian(fsys):
    bs, tpi, _ob = fsys
    D, _X = rel_inputs(bs.nbasis, 9)
    G = FourCompFock(tpi).formGD(D, xHFX=0.7)
    for k in range(4):
        assert np.abs(G[k] - G[k].conj().T).max() < 1e-9 * max(1.0, np.abs(G[k]).max())


# Mixed precision: quartets whose screening bound is below the cutoff run in
# FP32 arithmetic; the build must stay within 1e-6 Eh of the FP64 oracle.
MIXED_TOL = 1e-6
MIXED_CUT = 1e-2
# weight of each type's output in G (impl.hpp:3895-4636): 2 for the bare
# Coulomb J (libcint), 2 C^2 for LLSS, 2 C^4 for SSSS (C^2 = 1 / 4c^2), so
# the raw contraction's deviation times it is the deviation in Eh
_C2 = 1.0 / (4.0 * SPEED_OF_LIGHT ** 2)
FOCK_WEIGHT = {BARE_COULOMB: 2.0, LLSS: 2.0 * _C2, SSSS: 2.0 * _C2 * _C2}


@pytest.mark.parametrize("sysname,ctype", [("w631", BARE_COULOMB), ("w631", LLSS),
                                           ("w631", SSSS), ("fsys", LLSS), ("fsys", SSSS)])
def test_rel_contract_mixed(request, sysname, ctype):
    bs, tpi, ob = request.getfixturevalue(sysname)
    N = bs.nbasis
    _D, X = rel_inputs(N, 41 + ctype)
    ref = ob.rel_contract(X, ctype, True)
    c = GTODirectRelERIContraction(tpi)
    split = False
    # the small-component bounds carry c^-2 and c^-4 factors: sweep the
    # cutoff so that some launch splits its quartets between both precisions
    for cut in [MIXED_CUT * 10.0 ** -k for k in range(11)]:
        lst = [TwoBodyContraction(X[m], np.zeros((N, N), complex)) for m in range(17)]
        c.twoBodyContract(lst, ctype, precision="mixed", fp32_cutoff=cut)
        st = c.last_stats
        if cut == MIXED_CUT:
            assert st["fp32"] > 0, st
        split |= st["fp32"] > 0 and st["fp64"] > 0
        assert st["fp32"] + st["fp64"] + st["screened"] == st["total"], st
        for m in OUTS[ctype]:
            err = FOCK_WEIGHT[ctype] * np.abs(lst[m].AX - ref[m]).max()
            assert err < MIXED_TOL, (cut, m, err)
    assert split


def test_four_comp_gd_mixed(w631):
    bs, tpi, ob = w631
    D, _X = rel_inputs(bs.nbasis, 13)
    ref = ob.dirac_coulomb(D, bare=True, dc=True, ssss=True, libcint=True)
    fb = FourCompFock(tpi)
    G = fb.formGD(D, precision="mixed", fp32_cutoff=MIXED_CUT)
    smx = fb.last_stats
    assert smx["fp32"] > 0
    for k in range(4):
        assert np.abs(G[k] - ref[k]).max() < MIXED_TOL, k
    # FP64 and mixed builds visit and screen the same quartets
    fb.formGD(D)
    s64 = fb.last_stats
    assert s64["fp32"] == 0
    assert (s64["total"], s64["screened"]) == (smx["total"], smx["screened"])
    assert s64["fp64"] == smx["fp64"] + smx["fp32"]


@pytest.mark.parametrize("ctype", [BARE_COULOMB, LLSS, SSSS])
def test_rel_contract_mixed_tight_primitives(ctype):
    """Very tight d shells (exponent 1e5) with damped density blocks: their
    quartets fall below the cut but must stay in FP64 (FP32 overflows)."""
    bs = tight_d_basis()
    tpi, ob = DirectTPI(bs), O.OracleBasis(bs)
    N = bs.nbasis
    f = tight_ao_scale(bs)
    _D, X = rel_inputs(N, 51 + ctype)
    X = [np.asfortranarray(x * f[:, None] * f[None, :]) for x in X]
    ref = ob.rel_contract(X, ctype, True)
    lst = [TwoBodyContraction(X[m], np.zeros((N, N), complex)) for m in range(17)]
    c = GTODirectRelERIContraction(tpi)
    c.twoBodyContract(lst, ctype, precision="mixed", fp32_cutoff=MIXED_CUT)
    assert c.last_stats["fp32"] > 0, c.last_stats
    for m in OUTS[ctype]:
        assert np.isfinite(lst[m].AX).all(), m
        err = FOCK_WEIGHT[ctype] * np.abs(lst[m].AX - ref[m]).max()
        assert err < MIXED_TOL, (m, err)
