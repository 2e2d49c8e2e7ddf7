"""The Gaunt term restated from two-spinor physics (tests/twospinor.py),
pinned to the reference's converged Dirac-Coulomb-Gaunt SCF builds
(tests/scf/reference/UPu_184+_P_DCG_finitenuc.bin.ref and
CuH3_321g_DCG.bin.ref; bare Coulomb + LLSS + Gaunt, SSSS off, libcint):
G_golden = F - H must equal the oracle's bare Coulomb + LLSS build plus the
restated Gaunt matrix on the stored density, every block and Pauli
component.  CPU only."""
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
