"""The ChronusQ-side shims (chronusq_public_b200/shim/) compiled against test
stand-ins of the reference classes they derive from (tests/cpp/chronusq_stub/,
names and signatures of include/particleintegrals/twopints.hpp:31-260 and
twopints/gtodirect{tpi,releri}.hpp), then run across a geometry step: one
contraction object sees the shells move and must rebuild its device basis,
as the reference recomputes its Schwarz table for the new geometry."""
import os
import subprocess

import numpy as np
import pytest

from chronusq_public_b200 import _cabi
from chronusq_public_b200.basis import BasisSet, Molecule
from helpers import WATER_REF_GEOM

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp):
    exe = os.path.join(tmp, "shim_driver")
    subprocess.check_call(
        ["/usr/bin/g++", "-std=c++17", "-O2",
         "-I", os.path.join(ROOT, "tests", "cpp", "chronusq_stub"),
         "-I", os.path.join(ROOT, "chronusq_public_b200", "shim"),
         "-I", os.path.join(ROOT, "include"),
         os.path.join(ROOT, "tests", "cpp", "shim_driver.cpp"), "-o", exe,
         _cabi.LIB_PATH, "-Wl,-rpath," + os.path.dirname(_cabi.LIB_PATH)])
    return exe


def _write_shells(path, b):
    with open(path, "w") as f:
        f.write("%d\n" % b.nshell)
        for s in b.shells:
            f.write("%d %d %d %.17g %.17g %.17g\n" % (s.l, int(s.pure), s.nprim, *s.origin))
            f.write(" ".join("%.17g" % a for a in s.alpha) + "\n")
            f.write(" ".join("%.17g" % c for c in s.coef) + "\n")


def _geometries():
    """water / 6-31G(d) at the reference geometry and with one H moved by
    (0.12, 0.09, 0) Angstrom (a geometry-optimisation step)."""
    g1 = [list(a) for a in WATER_REF_GEOM]
    g1[1][1] += 0.12
    g1[1][2] += 0.09
    b0 = BasisSet.build(Molecule.from_angstrom(WATER_REF_GEOM), "6-31gd")
    b1 = BasisSet.build(Molecule.from_angstrom([tuple(a) for a in g1]), "6-31gd")
    return b0, b1


def test_shims_compile_against_reference_signatures(tmp_path):
    assert os.path.exists(_build(str(tmp_path)))


@pytest.mark.gpu
def test_shim_rebuilds_basis_after_geometry_step(tmp_path):
    import oracle as O
    exe = _build(str(tmp_path))
    b0, b1 = _geometries()
    _write_shells(tmp_path / "shells0.txt", b0)
    _write_shells(tmp_path / "shells1.txt", b1)
    N = b0.nbasis
    rng = np.random.default_rng(11)
    A = rng.standard_normal((N, N))
    D = 0.05 * (A + A.T)
    np.asfortranarray(D).T.tofile(str(tmp_path / "D.bin"))
    subprocess.check_call([exe, str(tmp_path), "1c"])
    refs = []
    for b in (b0, b1):
        J, K = O.OracleBasis(b).contract([D, D], [1, 1], [O.COULOMB, O.EXCHANGE])
        refs.append((J, K))
    assert np.abs(refs[0][0] - refs[1][0]).max() > 1e-3  # the step changes J
    for g, ref in enumerate([refs[0], refs[1], refs[1]]):
        JK = np.fromfile(str(tmp_path / ("JK%d.bin" % g)), dtype=np.float64)
        J = JK[:N * N].reshape(N, N, order="F")
        K = JK[N * N:].reshape(N, N, order="F")
        assert np.abs(J - ref[0]).max() < 1e-9, g
        assert np.abs(K - ref[1]).max() < 1e-9, g


@pytest.mark.gpu
def test_rel_shim_rebuilds_basis_after_geometry_step(tmp_path):
    import oracle as O
    exe = _build(str(tmp_path))
    b0, b1 = _geometries()
    _write_shells(tmp_path / "shells0.txt", b0)
    _write_shells(tmp_path / "shells1.txt", b1)
    N = b0.nbasis
    rng = np.random.default_rng(12)
    X = []
    for k in range(5):
        A = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))
        X.append(np.asfortranarray(0.05 * (A + A.conj().T)))
        X[k].T.tofile(str(tmp_path / ("R%d.bin" % k)))
    subprocess.check_call([exe, str(tmp_path), "4c"])
    X17 = X + [np.zeros((N, N), complex)] * 12
    refs = [O.OracleBasis(b).rel_contract(X17, 0, True)[:5] for b in (b0, b1)]
    for g, ref in enumerate([refs[0], refs[1], refs[1]]):
        out = np.fromfile(str(tmp_path / ("REL%d.bin" % g)), dtype=np.complex128)
        for k in range(5):
            AX = out[k * N * N:(k + 1) * N * N].reshape(N, N, order="F")
            assert np.abs(AX - ref[k]).max() < 1e-9, (g, k)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["gaunt", "gauge"])
def test_rel_shim_gaunt_list_with_aliased_outputs(tmp_path, mode):
    """The reference's 29-entry GAUNT / GAUGE list through the shim, its
    CSLM* / XSLM* AX pointing at the CLSM* / XLSM* outputs as in
    fourcompfock/impl.hpp:4237-4274, :4399-4436, against the oracle."""
    import oracle as O
    exe = _build(str(tmp_path))
    b0, _ = _geometries()
    _write_shells(tmp_path / "shells0.txt", b0)
    N = b0.nbasis
    rng = np.random.default_rng(13)
    # a Hermitian 4C density: Pauli components of a Hermitian 2N x 2N matrix
    blocks = []
    for _ in range(4):
        A = rng.standard_normal((2 * N, 2 * N)) + 1j * rng.standard_normal((2 * N, 2 * N))
        blocks.append(0.05 * (A + A.conj().T))
    ro, co = (0, N, 0, N), (0, N, N, 0)  # LL, SS, LS, SL
    G = []
    for k in range(4):
        for c in range(4):
            G.append(np.asfortranarray(blocks[c][ro[k]:ro[k] + N, co[k]:co[k] + N]))
    for i, g in enumerate(G):
        g.T.tofile(str(tmp_path / ("G%d.bin" % i)))
    subprocess.check_call([exe, str(tmp_path), mode])
    X = [G[0]] + G[0:4] + G[4:8] + G[4:8] + G[8:12] + G[8:12] + G[12:16] + G[12:16]
    ref = O.OracleBasis(b0).rel_contract(X, 3 if mode == "gaunt" else 4, True)
    out = np.fromfile(str(tmp_path / (mode + ".bin")), dtype=np.complex128)
    k = 0
    for base in (1, 9, 13, 17):
        for c in range(4):
            AX = out[k * N * N:(k + 1) * N * N].reshape(N, N, order="F")
            scale = max(1.0, np.abs(ref[base + c]).max())
            assert np.abs(AX - ref[base + c]).max() < 1e-9 * scale, (base, c)
            k += 1
