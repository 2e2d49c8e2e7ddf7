"""Seeded synthetic inputs of the Fock-build workloads.

Every workload is deterministic in its seed (numpy ``default_rng``):

* ``water``          H2O, O (0,0,0), H (+-0.757, 0, 0.587) Angstrom.
* ``water_cluster``  (H2O)_n: O positions by rejection sampling, uniform in a
                     cube of side ``box`` Angstrom with O-O >= 2.6 Angstrom,
                     rigid monomer above, uniformly random orientation (unit
                     quaternion from 4 normal deviates).
* ``occupied_density`` C ~ N(0,1) (N x nocc), C <- C (C^T S C)^{-1/2},
                     D = C C^T (what ChronusQ stores as onePDM.S for a
                     closed shell is 2 C C^T; the configs use C C^T as
                     written).
* ``delta_densities`` dD_k = eps (X_k + X_k^T), X_k ~ N(0,1), seeds base+k.
* ``ag4_cluster``    Ag4 tetrahedron, edge 2.7 Angstrom, every vertex
                     coordinate jittered by U(-0.05, 0.05) Angstrom.
* ``spinor_density_4c`` complex Gaussian occupied 4C spinors orthonormalised
                     in the metric diag(S, S, T/2c^2, T/2c^2), D = C C^H as
                     the four Pauli components of the 2N x 2N matrix.

S comes from the device one-electron integrals of libcqfock.so.
"""
from __future__ import annotations

from typing import List, Tuple

import numpy as np

from .basis import BasisSet, Molecule

WATER_GEOM = [("O", 0.0, 0.0, 0.0), ("H", 0.757, 0.0, 0.587),
              ("H", -0.757, 0.0, 0.587)]


def water() -> Molecule:
    return Molecule.from_angstrom(WATER_GEOM)


def _rotation(q: np.ndarray) -> np.ndarray:
    w, x, y, z = q / np.linalg.norm(q)
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
        [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
        [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def water_cluster(n: int, seed: int, box: float = 10.0,
                  dmin: float = 2.6) -> Molecule:
    """(H2O)_n by seeded rejection sampling (Angstrom inputs, Bohr output)."""
    rng = np.random.default_rng(seed)
    pos: List[np.ndarray] = []
    tries = 0
    while len(pos) < n:
        tries += 1
        if tries > 1000000:
            raise RuntimeError("could not place %d waters in a %g A box"
                               % (n, box))
        c = rng.uniform(0.0, box, size=3)
        if all(np.linalg.norm(c - p) >= dmin for p in pos):
            pos.append(c)
    mono = np.array([[a[1], a[2], a[3]] for a in WATER_GEOM])
    atoms: List[Tuple[str, float, float, float]] = []
    for c in pos:
        R = _rotation(rng.normal(size=4))
        for sym, xyz in zip(("O", "H", "H"), mono @ R.T + c):
            atoms.append((sym, float(xyz[0]), float(xyz[1]), float(xyz[2])))
    return Molecule.from_angstrom(atoms)


def occupied_density(S: np.ndarray, nocc: int, seed: int) -> np.ndarray:
    """D = C C^T with C (N x nocc) seeded N(0,1), S-orthonormalised."""
    rng = np.random.default_rng(seed)
    N = S.shape[0]
    C = rng.normal(size=(N, nocc))
    M = C.T @ S @ C
    w, V = np.linalg.eigh(M)
    C = C @ (V @ np.diag(w ** -0.5) @ V.T)
    return np.asfortranarray(C @ C.T)


def delta_densities(N: int, count: int, eps: float = 1e-3,
                    seed_base: int = 400) -> List[np.ndarray]:
    out = []
    for k in range(count):
        X = np.random.default_rng(seed_base + k).normal(size=(N, N))
        out.append(np.asfortranarray(eps * (X + X.T)))
    return out


def ag4_cluster(seed: int = 3, edge: float = 2.7, jitter: float = 0.05) -> Molecule:
    rng = np.random.default_rng(seed)
    a = edge / np.sqrt(2.0)  # tetrahedron from alternate cube corners
    v = 0.5 * a * np.array([[1, 1, 1], [1, -1, -1], [-1, 1, -1], [-1, -1, 1]], float)
    v = v + rng.uniform(-jitter, jitter, size=v.shape)
    return Molecule.from_angstrom([("Ag", *map(float, x)) for x in v])


SPEED_OF_LIGHT = 137.035999074  # atomic units (ChronusQ include/physcon.hpp)


def spinor_density_4c(S: np.ndarray, T: np.ndarray, nocc: int, seed: int):
    """Pauli components [scalar, MX, MY, MZ] (each 2N x 2N, LL block first)
    of D = C C^H, C (4N x nocc) complex Gaussian with rows (L alpha, L beta,
    S alpha, S beta), orthonormalised in the 4C metric."""
    rng = np.random.default_rng(seed)
    N = S.shape[0]
    C = rng.normal(size=(4 * N, nocc)) + 1j * rng.normal(size=(4 * N, nocc))
    Ms = T / (2.0 * SPEED_OF_LIGHT ** 2)
    Z = np.zeros_like(S)
    M = np.block([[S, Z, Z, Z], [Z, S, Z, Z], [Z, Z, Ms, Z], [Z, Z, Z, Ms]])
    w, V = np.linalg.eigh(C.conj().T @ M @ C)
    C = C @ (V @ np.diag(w ** -0.5) @ V.conj().T)
    Dfull = C @ C.conj().T
    idx_a = np.r_[0:N, 2 * N:3 * N]       # (L alpha, S alpha)
    idx_b = np.r_[N:2 * N, 3 * N:4 * N]   # (L beta, S beta)
    aa = Dfull[np.ix_(idx_a, idx_a)]
    bb = Dfull[np.ix_(idx_b, idx_b)]
    ab = Dfull[np.ix_(idx_a, idx_b)]
    ba = Dfull[np.ix_(idx_b, idx_a)]
    return [np.asfortranarray(aa + bb), np.asfortranarray(ab + ba),
            np.asfortranarray(1j * (ab - ba)), np.asfortranarray(aa - bb)]


# workload names -> (molecule factory, basis, occupied orbitals, seed)
def config(name: str):
    if name == "h2o_ccpvdz":
        return water(), "cc-pvdz", 5, 1
    if name == "h2o16_def2svp":
        return water_cluster(16, seed=2), "def2-svp", 40, 2
    if name == "h2o8_ccpvdz":
        return water_cluster(8, seed=4), "cc-pvdz", 40, 4
    if name == "ag4_dc":  # uncontracted basis, 188 occupied spinors
        return ag4_cluster(3), "sapporo-dkh3-dzp-2012_no", 188, 3
    raise KeyError(name)


def build_ag4_dc(tpi_factory, seed: int = 3):
    """(basis, DirectTPI, D[4]) of the Ag4 four-component workload."""
    mol, bname, nocc, _ = config("ag4_dc")
    basis = BasisSet.build(mol, bname, uncontract=True)
    tpi = tpi_factory(basis)
    S, T = tpi.one_electron()
    return basis, tpi, spinor_density_4c(S, T, nocc, seed)


def build_config(name: str, tpi_factory):
    """(basis, DirectTPI, D) of a named workload; ``tpi_factory(basis)``
    makes the device basis (S is taken from it)."""
    mol, bname, nocc, seed = config(name)
    basis = BasisSet.build(mol, bname)
    tpi = tpi_factory(basis)
    S, _T = tpi.one_electron()
    D = occupied_density(S, nocc, seed)
    return mol, basis, tpi, D

