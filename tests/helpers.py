"""Shared test inputs: the reference's test molecules and the golden data."""
import os

import numpy as np

from chronusq_public_b200.basis import BasisSet, Molecule, parse_gbs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# tests/func/input/contract_ref.inp and the READDEN inputs (Angstrom)
WATER_REF_GEOM = [("O", 0.0, -0.07579184359, 0.0),
                  ("H", 0.866811829, 0.6014357793, 0.0),
                  ("H", -0.866811829, 0.6014357793, 0.0)]


def golden(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def water_ref():
    return Molecule.from_angstrom(WATER_REF_GEOM)


def contract_basis():
    """water / cc-pVTZ of tests/func/input/contract_ref.inp (N = 58)."""
    return BasisSet.build(water_ref(), "cc-pvtz")


def readden_rhf_basis(g=None):
    g = golden("readden_rhf.npz") if g is None else g
    return BasisSet.build(water_ref(), parse_gbs(str(g["basisdef"])))


CONTRACT_CASES = ["HER_REAL_J", "NONHER_REAL_J", "HER_REAL_K", "NONHER_REAL_K",
                  "HER_COMPLEX_J", "NONHER_COMPLEX_J", "HER_COMPLEX_K",
                  "NONHER_COMPLEX_K"]


# Two centres with very tight d shells (exponent 1e5) beside ordinary ones:
# in FP32 the Hermite recursion of the tight-tight quartets would overflow
# ((2 alpha)^L past 2^128) while F_n(T) underflows, so the mixed path must
# keep them in FP64 whatever their screening bound.
TIGHT_D_BASIS = """
****
He 0
S 2 1.00
  4.0 0.4
  0.9 0.7
P 1 1.00
  1.1 1.0
D 1 1.00
  1.0e5 1.0
D 1 1.00
  0.8 1.0
****
H 0
S 1 1.00
  0.5 1.0
D 1 1.00
  1.0e5 1.0
****
"""


def tight_d_basis():
    mol = Molecule.from_angstrom([("He", 0.0, 0.0, 0.0), ("H", 0.4, -0.3, 1.3)])
    return BasisSet.build(mol, parse_gbs(TIGHT_D_BASIS))


def tight_ao_scale(basis, damp=1e-5):
    """Per-AO factor: `damp` on the AOs of shells with an exponent above
    1e4, 1 elsewhere (a density scaled by it on rows and columns has tiny
    blocks on the tight shells, so their quartets' bounds are small)."""
    f = np.ones(basis.nbasis)
    for s, sh in enumerate(basis.shells):
        if sh.alpha.max() > 1e4:
            f[basis.offsets[s]:basis.offsets[s] + sh.size] = damp
    return f


def gaunt_system(name):
    """(basis, D, G) of a Dirac-Coulomb-Gaunt golden build (gaunt_*.npz):
    the molecule and basis of the reference input, and the four Pauli
    components of its density and of G = F - H."""
    g = golden(name)
    atoms = []
    for line in str(g["geometry"]).splitlines():
        s, x, y, z = line.split()
        atoms.append((s, float(x), float(y), float(z)))
    mol = Molecule.from_angstrom(atoms)
    if "basisdef" in g:
        basis = BasisSet.build(mol, parse_gbs(str(g["basisdef"])))
    else:
        basis = BasisSet.build(mol, str(g["basisname"]))
    comps = ("SCALAR", "MX", "MY", "MZ")
    return (basis, [np.asarray(g["D_" + c]) for c in comps],
            [np.asarray(g["G_" + c]) for c in comps])
