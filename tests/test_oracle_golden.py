"""Pins the CPU oracle to the reference's own golden data (no GPU)."""
import math

import numpy as np
import pytest

import oracle as O
from chronusq_public_b200.basis import BasisSet, parse_gbs
from helpers import (CONTRACT_CASES, contract_basis, golden,
                     readden_rhf_basis, water_ref)


@pytest.fixture(scope="module")
def contract_oracle():
    return O.OracleBasis(contract_basis())


@pytest.mark.parametrize("case", CONTRACT_CASES)
def test_contract_hdf5(contract_oracle, case):
    """tests/func/contract.cxx:97-190: max|AX - AX_ref| < 1e-9."""
    g = golden("contract.npz")
    AX, = contract_oracle.contract([g[case + "_X"]], [int(g[case + "_her"])],
                                   [int(g[case + "_type"])])
    assert np.abs(AX - g[case + "_AX"]).max() < 1e-9


def test_readden_rhf_fock():
    """One direct RHF build: FOCK - CORE_H = 2 J[D] - K[D]."""
    g = golden("readden_rhf.npz")
    ob = O.OracleBasis(readden_rhf_basis(g))
    S, T = ob.overlap_kinetic()
    assert np.abs(S - g["S"]).max() < 1e-12
    assert np.abs(T - g["T"]).max() < 1e-9
    J, K = ob.contract([g["D"], g["D"]], [1, 1], [0, 1])
    G = 2 * J - K
    assert np.abs(G - (g["F"] - g["H"])).max() < 1e-9
    # two-electron energy 1/4 Tr[G D] (singleslater/quantum.hpp:147-205)
    e2 = 0.25 * np.sum(G * g["D"].T) * 1.0
    assert abs(e2 - float(g["E_many_body"][0])) < 1e-8


def test_normalisation_agrees(contract_oracle):
    b = contract_basis()
    assert np.allclose(contract_oracle.coefs(), b.flat()["coef"],
                       rtol=1e-14, atol=0)


@pytest.mark.parametrize("m,T", [(0, 0.0), (0, 1e-8), (3, 0.37), (8, 12.3),
                                 (12, 35.9), (12, 36.1), (16, 80.0),
                                 (4, 200.0)])
def test_boys_against_series(m, T):
    # independent reference: F_m(T) = int_0^1 t^2m exp(-T t^2) dt by
    # composite Gauss-Legendre on [0,1]
    x, w = np.polynomial.legendre.leggauss(200)
    segs = 40
    tot = 0.0
    for s in range(segs):
        a, b = s / segs, (s + 1) / segs
        t = 0.5 * (b - a) * x + 0.5 * (a + b)
        tot += 0.5 * (b - a) * np.sum(w * t ** (2 * m) * np.exp(-T * t * t))
    assert abs(O.boys(m, T) - tot) <= 1e-14 * max(tot, 1e-300) + 1e-300


def _readden_dc_basis():
    return BasisSet.build(water_ref(), parse_gbs(str(golden("readden_dc.npz")["basisdef"])))


PAULI = ("SCALAR", "MX", "MY", "MZ")


def test_dirac_coulomb_bare_libcint():
    """4C bare Coulomb (libcint branch, twoeH_LL = 2 CLLMS,
    fourcompfock/impl.hpp:3901-3933) against the DC-HF-guess READDEN build,
    whose stored FOCK carries only the LL two-electron block."""
    g = golden("readden_dchf_ll.npz")
    ob = O.OracleBasis(_readden_dc_basis())
    N = ob.nbasis
    D = []
    for c in PAULI:
        d = np.zeros((2 * N, 2 * N), dtype=np.complex128)
        d[:N, :N] = g["D_" + c]
        D.append(d)
    G = ob.dirac_coulomb(D, bare=True, dc=False, ssss=False, libcint=True)
    for k, c in enumerate(PAULI):
        assert np.abs(G[k][:N, :N] - g["G_" + c]).max() < 1e-9, c
        assert np.abs(G[k][N:, :]).max() == 0 and np.abs(G[k][:, N:]).max() == 0


def test_dirac_coulomb_rhf_guess():
    """Same build from the RHF-guess READDEN density (spin components zero)."""
    g = golden("readden_dc.npz")
    ob = O.OracleBasis(_readden_dc_basis())
    D = [np.where(np.abs(g["D_" + c]) < 1e-200, 0, g["D_" + c]) for c in PAULI]
    G = ob.dirac_coulomb(D, bare=True, dc=False, ssss=False, libcint=True)
    for k, c in enumerate(PAULI):
        ref = g["F_" + c] - g["H_" + c]
        ref = np.where(np.abs(ref) < 1e-200, 0, ref)
        assert np.abs(G[k] - ref).max() < 1e-9, c


def test_dirac_coulomb_llss():
    """Converged complex 4C-HF water / 6-31G(d) with the Dirac-Coulomb LLSS
    terms (SS and LS blocks from the derivative ERIs, impl.hpp:4003-4147) and
    the non-libcint bare Coulomb (twoeH_LL = J, impl.hpp:3934-3969)."""
    g = golden("qn_4chf_dc.npz")
    ob = O.OracleBasis(BasisSet.build(water_ref(), "6-31gd"))
    D = [g["D_" + c] for c in PAULI]
    G = ob.dirac_coulomb(D, bare=True, dc=True, ssss=False, libcint=False)
    for k, c in enumerate(PAULI):
        assert np.abs(G[k] - g["G_" + c]).max() < 1e-9, c


def test_nuclear_point_rhf_core_hamiltonian():
    """Point nuclei: the reference stores the core Hamiltonian's scalar
    Pauli component, 2 (T + V) (INTS/CORE_HAMILTONIAN_SCALAR)."""
    g = golden("readden_rhf.npz")
    ob = O.OracleBasis(readden_rhf_basis(g))
    V = ob.nuclear(water_ref().nuclei())
    assert np.abs(V - (g["H"] / 2 - g["T"])).max() < 1e-10


def test_nuclear_finite_four_component_core_hamiltonian():
    """Gaussian nuclei (the 4C default): the LL block of the DC core
    Hamiltonian's scalar component is 2 V, its LS block 2 T; point nuclei
    would miss it by far more than the tolerance."""
    g = golden("readden_dc.npz")
    mol = water_ref()
    bs = BasisSet.build(mol, parse_gbs(str(g["basisdef"])))
    ob = O.OracleBasis(bs)
    N = bs.nbasis
    H = g["H_SCALAR"]
    Vf = ob.nuclear(mol.nuclei(finite=True))
    assert np.abs(H[:N, :N].real - 2 * Vf).max() < 1e-10
    assert np.abs(H[:N, :N].real - 2 * ob.nuclear(mol.nuclei())).max() > 1e-3
    _S, T = ob.overlap_kinetic()
    assert np.abs(H[:N, N:].real - 2 * T).max() < 1e-9


def test_finite_nucleus_exponent():
    from chronusq_public_b200.basis import finite_nucleus_exponent
    # O-16: r = 0.836 * 16^(1/3) + 0.570 fm
    r = (0.836 * 16 ** (1 / 3) + 0.570) * 1e-5 / 0.52917721092
    assert math.isclose(finite_nucleus_exponent(16), 1.5 / r ** 2, rel_tol=1e-14)
    nuc = water_ref().nuclei(finite=True)
    assert nuc.shape == (3, 5) and (nuc[:, 4] > 1e8).all()


def test_four_component_core_hamiltonian_ss_block():
    """SS block of the reference's 4C core Hamiltonian (compute4CCH,
    src/fourcomp/fourcomp.cxx:36-100): scalar 2 (pV.p / 4c^2 - T), MX/MY/MZ
    2i (pV x p)_k / 4c^2, with Gaussian nuclei."""
    g = golden("readden_dc.npz")
    mol = water_ref()
    bs = BasisSet.build(mol, parse_gbs(str(g["basisdef"])))
    ob = O.OracleBasis(bs)
    N = bs.nbasis
    W = ob.nuclear_pvp(mol.nuclei(finite=True))
    _S, T = ob.overlap_kinetic()
    C2 = 1.0 / (4.0 * 137.035999074 ** 2)
    ss = g["H_SCALAR"][N:, N:]
    assert np.abs(ss.real - 2 * (C2 * W[0] - T)).max() < 1e-9
    assert np.abs(ss.imag).max() == 0
    for k, comp in enumerate(("MX", "MY", "MZ")):
        h = g["H_" + comp]
        assert np.abs(h[N:, N:] - 2j * C2 * W[1 + k]).max() < 1e-12
        assert np.abs(h[:N, :]).max() == 0 and np.abs(h[N:, :N]).max() == 0
