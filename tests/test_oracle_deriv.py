"""Independent pins of the four-component small-component terms (CPU only).

The SSSS term of the Dirac-Coulomb build has no reference golden file of its
own (the one that holds an SSSS build also needs the Gaunt and gauge terms),
so the GPU's SSSS path is checked against the oracle, and the oracle is
pinned here two ways that do not reuse its four-component code:

1. its derivative ERIs (d/dr of the orbitals on chosen centres, the engine
   behind LLSS and SSSS) against 5-point central differences of its plain
   ERIs -- which are pinned to the reference's golden files -- in the shell
   centres; and
2. the LLSS and SSSS two-electron matrices rebuilt from scratch: kinetically
   balanced small-component spinors (sigma.p) chi / (2c), their charge
   densities through sigma_i sigma_j = delta_ij + i eps_ijk sigma_k, and
   G = J - K over 2-spinor indices with numpy.  The overall Coulomb and
   exchange weights of the reference's Pauli-component storage are read off
   the LLSS term (itself pinned to water_6-31Gd_qn_4chf.bin.ref) and then
   must reproduce the SSSS term with no further freedom.
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
from chronusq_public_b200.basis import BasisSet
from helpers import water_ref
from twospinor import C2, SS, deriv_tensor as _tensor, pauli as _pauli, spin_blocks as _spin_blocks


@pytest.fixture(scope="module")
def water():
    return BasisSet.build(water_ref(), "6-31gd")


def _shifted(basis, s, axis, h):
    sh = list(basis.shells)
    o = np.array(sh[s].origin, dtype=float)
    o[axis] += h
    sh[s] = dataclasses.replace(sh[s], origin=o)
    return BasisSet(sh)


def _plain(basis, q):
    return O.OracleBasis(basis).eri_quartet(*q)


def _quartet(basis):
    """Four distinct shells on three centres with l = 1, 0, 2, 0."""
    ls = [s.l for s in basis.shells]
    cen = [tuple(np.round(s.origin, 8)) for s in basis.shells]
    p = ls.index(1)
    d = ls.index(2)
    h = [i for i, s in enumerate(basis.shells) if s.l == 0 and cen[i] != cen[p]]
    return (p, h[0], d, h[-1])


def test_derivative_eris_match_finite_differences(water):
    q = _quartet(water)
    ob = O.OracleBasis(water)
    h = 1e-3
    for c in range(4):  # one derivative on centre c
        der = ob.eri_deriv_quartet(*q, 1 << c)
        for x in range(3):
            f = [_plain(_shifted(water, q[c], x, k * h), q) for k in (-2, -1, 1, 2)]
            dA = (f[0] - 8 * f[1] + 8 * f[2] - f[3]) / (12 * h)
            # d/dr of the orbital = -d/dA of its centre
            assert np.abs(der[x] + dA).max() < 1e-7 * max(1.0, np.abs(dA).max()), (c, x)


def test_four_centre_derivative_eris_match_finite_differences(water):
    """(dA_i a dB_j b | dC_k c dD_l d): the fourth mixed derivative of the
    plain ERI in the four centres (16-point stencil), on three components."""
    q = _quartet(water)
    der = O.OracleBasis(water).eri_deriv_quartet(*q, 15)
    h = 4e-3
    for (i, j, k, l) in ((0, 1, 2, 0), (2, 2, 1, 1), (1, 0, 0, 2)):
        acc = 0.0
        for sg in np.ndindex(2, 2, 2, 2):
            b = water
            sign = 1.0
            for c, (ax, s) in enumerate(zip((i, j, k, l), sg)):
                b = _shifted(b, q[c], ax, h if s else -h)
                sign *= 1.0 if s else -1.0
            acc = acc + sign * _plain(b, q)
        fd = acc / (16 * h ** 4)
        comp = ((i * 3 + j) * 3 + k) * 3 + l
        assert np.abs(der[comp] - fd).max() < 2e-3 * np.abs(fd).max(), (i, j, k, l)


@pytest.fixture(scope="module")
def four_comp(water):
    N = water.nbasis
    rng = np.random.default_rng(21)
    D = []
    for _ in range(4):
        A = rng.standard_normal((2 * N, 2 * N)) + 1j * rng.standard_normal((2 * N, 2 * N))
        D.append(0.05 * (A + A.conj().T))
    ob = O.OracleBasis(water)
    g_llss = ob.dirac_coulomb(D, bare=False, dc=True, ssss=False, thresh=1e-16)
    g_ssss = ob.dirac_coulomb(D, bare=False, dc=False, ssss=True, thresh=1e-16)
    return N, D, g_llss, g_ssss


def _block(G, N, r, c):
    return [g[r * N:(r + 1) * N, c * N:(c + 1) * N] for g in G]


def test_llss_and_ssss_from_two_spinors(water, four_comp):
    N, D, g_llss, g_ssss = four_comp
    Db = _spin_blocks(D, N)
    I3 = _tensor(water, 3)     # (d_i mu d_j nu | ka la)
    I12 = _tensor(water, 12)   # (mu nu | d_k ka d_l la)
    # LLSS: J^LL from the SS density, J^SS from the LL density, K^LS
    W = np.einsum("klab,qbpa->klpq", SS, Db["SS"])  # sum_tt' S_kl[t,t'] D[la t', ka t]
    JLL = C2 * np.einsum("klmnpq,klpq->mn", I12, W)
    JLL_so = np.zeros((N, 2, N, 2), dtype=complex)
    JLL_so[:, 0, :, 0] = JLL_so[:, 1, :, 1] = JLL
    trLL = Db["LL"][:, 0, :, 0] + Db["LL"][:, 1, :, 1]   # sum_t D[la t, ka t]
    JSS = C2 * np.einsum("ijab,ijmnpq,qp->manb", SS, I3, trLL)
    KLS = C2 * np.einsum("klab,klmqpn,qspa->msnb", SS, I12, Db["LS"], optimize=True)
    ref_LL, ref_SS, ref_LS = (_block(g_llss, N, 0, 0), _block(g_llss, N, 1, 1),
                              _block(g_llss, N, 0, 1))
    # the reference's weights (Coulomb fJ, exchange fK) read off LLSS
    mine_J = _pauli(JLL_so)
    fJ = np.vdot(mine_J[0], ref_LL[0]).real / np.vdot(mine_J[0], mine_J[0]).real
    mine_K = _pauli(KLS)
    fK = -np.vdot(mine_K[0], ref_LS[0]).real / np.vdot(mine_K[0], mine_K[0]).real
    scale = max(np.abs(r).max() for r in ref_LL + ref_SS + ref_LS)
    for m, r in zip(_pauli(fJ * JLL_so), ref_LL):
        assert np.abs(m - r).max() < 1e-10 * scale
    for m, r in zip(_pauli(fJ * JSS), ref_SS):
        assert np.abs(m - r).max() < 1e-10 * scale
    for m, r in zip(_pauli(-fK * KLS), ref_LS):
        assert np.abs(m - r).max() < 1e-10 * scale
    # SSSS with the same weights: J^SS and K^SS from the SS density
    I15 = _tensor(water, 15)
    JS = C2 * C2 * np.einsum("ijab,ijklmnpq,klpq->manb", SS, I15, W, optimize=True)
    KS = C2 * C2 * np.einsum("ijac,klbd,ijklmqpn,qcpb->mand", SS, SS, I15, Db["SS"],
                             optimize=True)
    ref = _block(g_ssss, N, 1, 1)
    scale = max(np.abs(r).max() for r in ref)
    assert scale > 0.0
    for c, (m, r) in enumerate(zip(_pauli(fJ * JS - fK * KS), ref)):
        assert np.abs(m - r).max() < 1e-10 * scale, c
    # nothing outside the SS block
    for g in g_ssss:
        assert np.abs(g[:N, :]).max() == 0.0 and np.abs(g[:, :N]).max() == 0.0
