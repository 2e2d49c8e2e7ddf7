"""The nuclear-gradient contraction on the GPU (cqf_grad_two_body_contract,
DirectGradContraction::gradTwoBodyContract) against the oracle's
restatement of directScaffoldGrad (itself pinned to finite differences of
the golden-pinned J / K builds, tests/test_oracle_grad.py), and the
two-electron energy gradient of FockBuilder::getGDGrad."""
import numpy as np
import pytest

import oracle as O
from chronusq_public_b200 import workloads
from chronusq_public_b200.basis import BasisSet
from chronusq_public_b200.contraction import (COULOMB, EXCHANGE, DirectGradContraction,
                                              DirectTPI, TwoBodyContraction)
from chronusq_public_b200.fockbuilder import FockBuilder
from helpers import water_ref
from test_gpu_rel import f_basis

pytestmark = pytest.mark.gpu


def _system(which, seed):
    b = f_basis() if which == "f_basis" else BasisSet.build(water_ref(), "6-31gd")
    N = b.nbasis
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((N, N))
    D = 0.1 * (A + A.T)
    atoms = np.array([s.atom for s in b.shells], dtype=np.int32)
    return b, D, atoms, int(atoms.max()) + 1


def _gpu_grad(tpi, D, atoms, natom, shard=(0, 1), device=False):
    N = tpi.nbasis
    cList = []
    for _ in range(3 * natom):
        if device:
            import torch
            J = torch.zeros((N, N), dtype=torch.float64, device="cuda").T
            K = torch.zeros((N, N), dtype=torch.float64, device="cuda").T
        else:
            J = np.zeros((N, N), order="F")
            K = np.zeros((N, N), order="F")
        cList.append([TwoBodyContraction(D, J, True, COULOMB),
                      TwoBodyContraction(D, K, True, EXCHANGE)])
    DirectGradContraction(tpi).gradTwoBodyContract(cList, atoms, shard=shard)
    if device:
        return [[c.AX.cpu().numpy() for c in comp] for comp in cList]
    return [[c.AX for c in comp] for comp in cList]


@pytest.mark.parametrize("which", ["water_631gd", "f_basis"])
def test_grad_contract_vs_oracle(which):
    b, D, atoms, natom = _system(which, 51)
    ref = O.OracleBasis(b).grad_contract([D, D], [O.COULOMB, O.EXCHANGE], atoms, natom)
    got = _gpu_grad(DirectTPI(b), D, atoms, natom)
    for g in range(3 * natom):
        for m in range(2):
            scale = max(1.0, np.abs(ref[g][m]).max())
            assert np.abs(got[g][m] - ref[g][m]).max() < 1e-11 * scale, (g, m)


def test_grad_contract_device_pointers_and_shards():
    import torch
    b, D, atoms, natom = _system("water_631gd", 52)
    tpi = DirectTPI(b)
    host = _gpu_grad(tpi, D, atoms, natom)
    Dd = torch.from_numpy(np.asfortranarray(D)).cuda().T.contiguous().T
    dev = _gpu_grad(tpi, Dd, atoms, natom, device=True)
    parts = [_gpu_grad(tpi, D, atoms, natom, shard=(k, 3)) for k in range(3)]
    for g in range(3 * natom):
        for m in range(2):
            assert np.abs(dev[g][m] - host[g][m]).max() < 1e-13
            s = parts[0][g][m] + parts[1][g][m] + parts[2][g][m]
            assert np.abs(s - host[g][m]).max() < 1e-12 * max(1.0, np.abs(host[g][m]).max())


def test_two_electron_gradient_translational_invariance():
    """(H2O)4 / cc-pVDZ: getGDGrad sums to zero over the atoms; (H2O)2: it
    equals 1/4 Tr[D (2 J^x - K^x)] from the oracle's contraction."""
    for n in (4, 2):
        mol = workloads.water_cluster(n, seed=3)
        b = BasisSet.build(mol, "cc-pvdz")
        tpi = DirectTPI(b)
        S, _ = tpi.one_electron()
        D = workloads.occupied_density(S, 5 * n, 5)
        atoms = np.array([s.atom for s in b.shells], dtype=np.int32)
        natom = mol.natom
        g = FockBuilder(tpi).getGDGrad(D, atoms, natom)
        assert np.abs(g).max() > 1e-2
        assert np.abs(g.sum(axis=0)).max() < 1e-9 * np.abs(g).max(), n
        if n == 2:
            ref = O.OracleBasis(b).grad_contract([D, D], [O.COULOMB, O.EXCHANGE], atoms,
                                                 natom)
            gr = np.array([0.25 * np.sum((2 * ref[k][0] - ref[k][1]) * D.T)
                           for k in range(3 * natom)])
            assert np.abs(g.ravel() - gr).max() < 1e-10 * np.abs(gr).max()
