"""One-electron matrices on the device (cqf_basis_one_electron,
cqf_basis_nuclear) against the reference's stored core Hamiltonians and the
oracle."""
import numpy as np
import pytest

import oracle as O
from chronusq_public_b200.basis import BasisSet, Molecule, parse_gbs
from chronusq_public_b200.contraction import DirectTPI
from helpers import golden, readden_rhf_basis, water_ref

pytestmark = pytest.mark.gpu


def test_nuclear_point_matches_rhf_core_hamiltonian():
    g = golden("readden_rhf.npz")
    tpi = DirectTPI(readden_rhf_basis(g))
    V = tpi.nuclear(water_ref().nuclei())
    _S, T = tpi.one_electron()
    assert np.abs(V - (g["H"] / 2 - g["T"])).max() < 1e-9
    assert np.abs(2 * (T + V) - g["H"]).max() < 1e-9


def test_nuclear_finite_matches_dc_core_hamiltonian():
    g = golden("readden_dc.npz")
    mol = water_ref()
    bs = BasisSet.build(mol, parse_gbs(str(g["basisdef"])))
    tpi = DirectTPI(bs)
    N = bs.nbasis
    V = tpi.nuclear(mol.nuclei(finite=True))
    assert np.abs(2 * V - g["H_SCALAR"][:N, :N].real).max() < 1e-9


@pytest.mark.parametrize("finite", [False, True])
def test_nuclear_ag_f_shells_vs_oracle(finite):
    """Two Ag atoms, uncontracted sapporo-dkh3-dzp (s..f, exponents to ~1e7)."""
    mol = Molecule.from_angstrom([("Ag", 0.0, 0.0, 0.0), ("Ag", 0.3, 0.5, 2.6)])
    bs = BasisSet.build(mol, "sapporo-dkh3-dzp-2012_no", uncontract=True)
    nuc = mol.nuclei(finite=finite)
    V = DirectTPI(bs).nuclear(nuc)
    Vo = O.OracleBasis(bs).nuclear(nuc)
    assert np.abs(V - Vo).max() < 1e-10 * max(1.0, np.abs(Vo).max())
    assert np.abs(V - V.T).max() < 1e-10 * np.abs(Vo).max()


def test_four_comp_core_hamiltonian_matches_reference():
    """All four Pauli components, every block, against the reference's stored
    4C core Hamiltonian (water, Gaussian nuclei)."""
    g = golden("readden_dc.npz")
    mol = water_ref()
    bs = BasisSet.build(mol, parse_gbs(str(g["basisdef"])))
    H = DirectTPI(bs).four_comp_core_hamiltonian(mol.nuclei(finite=True))
    for k, comp in enumerate(("SCALAR", "MX", "MY", "MZ")):
        ref = g["H_" + comp]
        assert np.abs(H[k] - ref).max() < 1e-9 * max(1.0, np.abs(ref).max()), comp


@pytest.mark.parametrize("finite", [False, True])
def test_nuclear_pvp_ag_f_shells_vs_oracle(finite):
    mol = Molecule.from_angstrom([("Ag", 0.0, 0.0, 0.0), ("Ag", 0.3, 0.5, 2.6)])
    bs = BasisSet.build(mol, "sapporo-dkh3-dzp-2012_no", uncontract=True)
    nuc = mol.nuclei(finite=finite)
    W = DirectTPI(bs).nuclear_pvp(nuc)
    Wo = O.OracleBasis(bs).nuclear_pvp(nuc)
    for k in range(4):
        assert np.abs(W[k] - Wo[k]).max() < 1e-10 * max(1.0, np.abs(Wo[k]).max()), k
    # pV.p symmetric, the spin-orbit parts antisymmetric
    assert np.abs(W[0] - W[0].T).max() < 1e-9 * np.abs(W[0]).max()
    for k in (1, 2, 3):
        assert np.abs(W[k] + W[k].T).max() < 1e-9 * np.abs(W[k]).max()
