"""The oracle's restatement of DirectGradContraction::directScaffoldGrad
(direct.hpp:2198-2571), pinned independently (CPU only): its J- and K-type
derivative matrices for an atom's x / y / z equal central finite
differences of the golden-pinned J / K builds with that atom's shells
displaced (the density fixed in the AO basis), and they sum to zero over
the atoms (translational invariance)."""
import dataclasses

import numpy as np
import pytest

import oracle as O
from chronusq_public_b200.basis import BasisSet
from helpers import water_ref


@pytest.fixture(scope="module")
def system():
    b = BasisSet.build(water_ref(), "6-31gd")
    N = b.nbasis
    rng = np.random.default_rng(17)
    A = rng.standard_normal((N, N))
    D = 0.1 * (A + A.T)
    atoms = np.array([s.atom for s in b.shells], dtype=np.int32)
    natom = int(atoms.max()) + 1
    grad = O.OracleBasis(b).grad_contract([D, D], [O.COULOMB, O.EXCHANGE], atoms, natom)
    return b, D, atoms, natom, grad


def _moved(b, atom, axis, h):
    sh = []
    for s in b.shells:
        if s.atom == atom:
            o = np.array(s.origin, dtype=float)
            o[axis] += h
            s = dataclasses.replace(s, origin=o)
        sh.append(s)
    return BasisSet(sh)


def test_grad_matches_finite_differences(system):
    b, D, atoms, natom, grad = system
    h = 1e-3
    for atom, axis in ((0, 2), (1, 0), (2, 1)):
        f = []
        for k in (-2, -1, 1, 2):
            J, K = O.OracleBasis(_moved(b, atom, axis, k * h)).contract(
                [D, D], [1, 1], [O.COULOMB, O.EXCHANGE], screen=False)
            f.append((J, K))
        for m in range(2):
            fd = (f[0][m] - 8 * f[1][m] + 8 * f[2][m] - f[3][m]) / (12 * h)
            g = grad[atom * 3 + axis][m]
            assert np.abs(fd).max() > 1e-3
            assert np.abs(g - fd).max() < 1e-6 * np.abs(fd).max(), (atom, axis, m)


def test_grad_translational_invariance(system):
    _b, _D, _atoms, natom, grad = system
    for axis in range(3):
        for m in range(2):
            tot = sum(grad[a * 3 + axis][m] for a in range(natom))
            scale = max(np.abs(grad[a * 3 + axis][m]).max() for a in range(natom))
            assert np.abs(tot).max() < 1e-11 * scale, (axis, m)
