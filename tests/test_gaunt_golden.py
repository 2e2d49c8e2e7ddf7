"""The Gaunt and Breit gauge terms restated from two-spinor physics
(tests/twospinor.py), pinned to the reference's converged SCF builds:
Dirac-Coulomb-Gaunt (tests/scf/reference/UPu_184+_P_DCG_finitenuc.bin.ref,
CuH3_321g_DCG.bin.ref; bare Coulomb + LLSS + Gaunt, SSSS off, libcint) and
Dirac-Coulomb-Breit (UPu_184+_P_DCGGS_finitenuc.bin.ref; SSSS, Gaunt and
Gauge on): G_golden = F - H must equal the builds on the stored density,
every block and Pauli component.  The Breit build also pins the oracle's
SSSS term, which no other reference file holds.  CPU only."""
import numpy as np
import pytest

import oracle as O
import twospinor as TS
from helpers import gaunt_system as _system

COMPS = ("SCALAR", "MX", "MY", "MZ")


@pytest.mark.parametrize("name", ["gaunt_upu.npz", "gaunt_cuh3.npz"])
def test_gaunt_reproduces_reference_dcg_build(name):
    basis, D, Gref = _system(name)
    assert 2 * basis.nbasis == D[0].shape[0]
    ob = O.OracleBasis(basis)
    Gdc = ob.dirac_coulomb(D, bare=True, dc=True, ssss=False, libcint=True)
    Gg = TS.gaunt(basis, D)
    scale = max(np.abs(g).max() for g in Gref)
    gaunt_size = max(np.abs(g).max() for g in Gg)
    for c in range(4):
        err = np.abs(Gdc[c] + Gg[c] - Gref[c]).max()
        assert err < 1e-8 * max(1.0, scale), (COMPS[c], err, scale)
    # the Gaunt term is visible at this tolerance (the check is not vacuous)
    miss = max(np.abs(Gdc[c] - Gref[c]).max() for c in range(4))
    assert miss > 1e3 * 1e-8 * max(1.0, scale), (miss, gaunt_size)


@pytest.mark.parametrize("name", ["gaunt_upu.npz", "gaunt_cuh3.npz"])
def test_oracle_gaunt_reproduces_reference_dcg_build(name):
    """The oracle's restatement of the reference's Gaunt contraction (its
    quartet set, Gaunt Schwarz screen and update sites) and assembly."""
    basis, D, Gref = _system(name)
    G = O.OracleBasis(basis).dirac_coulomb(D, bare=True, dc=True, ssss=False, libcint=True,
                                           gaunt=True)
    scale = max(np.abs(g).max() for g in Gref)
    for c in range(4):
        assert np.abs(G[c] - Gref[c]).max() < 1e-9 * max(1.0, scale), COMPS[c]


@pytest.mark.parametrize("name", ["gaunt_upu.npz", "gaunt_cuh3.npz"])
def test_oracle_gaunt_matches_two_spinors_on_a_random_density(name):
    """A random Hermitian 4C density (no SCF structure), screening off: the
    oracle's Gaunt-only build equals the two-spinor restatement."""
    basis, _, _ = _system(name)
    N = basis.nbasis
    rng = np.random.default_rng(5)
    A = [rng.standard_normal((2 * N, 2 * N)) + 1j * rng.standard_normal((2 * N, 2 * N))
         for _ in range(4)]
    # Pauli components of a Hermitian 2-spinor matrix are Hermitian
    D = [0.1 * (a + a.conj().T) for a in A]
    G = O.OracleBasis(basis).dirac_coulomb(D, bare=False, dc=False, ssss=False, gaunt=True,
                                           thresh=0.0)
    ref = TS.gaunt(basis, D)
    scale = max(np.abs(r).max() for r in ref)
    for c in range(4):
        assert np.abs(G[c] - ref[c]).max() < 1e-11 * scale, COMPS[c]


def test_r12_kernel_integrals_laplacian():
    """sum_i (ab| d_i d_i r12 |cd) = 2 (ab|cd): the r12 integrals behind the
    gauge term against the golden-pinned Coulomb ERIs, plain and with
    derivatives on the orbitals."""
    basis, _, _ = _system("gaunt_cuh3.npz")
    ob = O.OracleBasis(basis)
    ls = [sh.l for sh in basis.shells]
    q = (ls.index(2), ls.index(1), 0, len(ls) - 1)
    for dmask in (0, 6, 10, 15):
        lap = sum(ob.r12_deriv_quartet(*q, dmask, i, i) for i in range(3))
        c = ob.eri_deriv_quartet(*q, dmask)
        assert np.abs(c).max() > 0
        assert np.abs(lap - 2 * c).max() < 1e-12 * np.abs(c).max(), dmask


def test_breit_reproduces_reference_dcggs_build():
    """Bare Coulomb + Dirac-Coulomb (LLSS + SSSS) from the oracle, Gaunt and
    gauge from the two-spinor restatement, half of each (the Breit term)."""
    basis, D, Gref = _system("breit_upu.npz")
    ob = O.OracleBasis(basis)
    Gdc = ob.dirac_coulomb(D, bare=True, dc=True, ssss=True, libcint=True)
    Gg = TS.gaunt(basis, D)
    Gb = TS.gauge(basis, D)
    scale = max(np.abs(g).max() for g in Gref)
    for c in range(4):
        err = np.abs(Gdc[c] + 0.5 * (Gg[c] + Gb[c]) - Gref[c]).max()
        assert err < 1e-9 * max(1.0, scale), (COMPS[c], err)


def test_oracle_breit_reproduces_reference_dcggs_build():
    """The oracle's whole Dirac-Coulomb-Breit build (its SSSS, Gaunt and
    GAUGE restatements) against the reference's."""
    basis, D, Gref = _system("breit_upu.npz")
    G = O.OracleBasis(basis).dirac_coulomb(D, bare=True, dc=True, ssss=True, libcint=True,
                                           gaunt=True, gauge=True)
    scale = max(np.abs(g).max() for g in Gref)
    for c in range(4):
        assert np.abs(G[c] - Gref[c]).max() < 1e-9 * max(1.0, scale), COMPS[c]


def test_oracle_gauge_matches_two_spinors_on_a_random_density():
    basis, _, _ = _system("breit_upu.npz")
    N = basis.nbasis
    rng = np.random.default_rng(6)
    A = [rng.standard_normal((2 * N, 2 * N)) + 1j * rng.standard_normal((2 * N, 2 * N))
         for _ in range(4)]
    D = [0.1 * (a + a.conj().T) for a in A]
    G = O.OracleBasis(basis).dirac_coulomb(D, bare=False, dc=False, ssss=False, gauge=True,
                                           thresh=0.0)
    ref = TS.gauge(basis, D)
    scale = max(np.abs(r).max() for r in ref)
    for c in range(4):
        assert np.abs(G[c] - 0.5 * ref[c]).max() < 1e-11 * scale, COMPS[c]
