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
