"""The C++ host layer (include/cqfock.hpp) compiled with g++ against
libcqfock.so reproduces the contract.hdf5 cases (tests/func/contract.cxx)."""
import os
import subprocess

import numpy as np
import pytest

from chronusq_public_b200 import _cabi
from helpers import CONTRACT_CASES, contract_basis, golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp):
    exe = os.path.join(tmp, "contract_cpp")
    subprocess.check_call(
        ["/usr/bin/g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
         os.path.join(ROOT, "tests", "cpp", "contract_cpp.cpp"), "-o", exe,
         _cabi.LIB_PATH, "-Wl,-rpath," + os.path.dirname(_cabi.LIB_PATH)])
    return exe


def test_cpp_host_layer_compiles(tmp_path):
    assert os.path.exists(_build(str(tmp_path)))


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["HER_REAL_J", "HER_REAL_K", "NONHER_COMPLEX_J",
                                  "NONHER_COMPLEX_K"])
def test_cpp_host_layer_contract_cases(tmp_path, case):
    exe = _build(str(tmp_path))
    b = contract_basis()
    with open(tmp_path / "shells.txt", "w") as f:
        f.write("%d\n" % b.nshell)
        for s in b.shells:
            f.write("%d %d %d %.17g %.17g %.17g\n" % (s.l, int(s.pure), s.nprim, *s.origin))
            f.write(" ".join("%.17g" % a for a in s.alpha) + "\n")
            f.write(" ".join("%.17g" % c for c in s.coef) + "\n")
    g = golden("contract.npz")
    X = g[case + "_X"]
    cplx = np.iscomplexobj(X)
    np.asfortranarray(X).T.tofile(str(tmp_path / "X.bin"))
    subprocess.check_call([exe, str(tmp_path), str(int(g[case + "_her"])),
                           str(int(g[case + "_type"])), str(int(cplx))])
    AX = np.fromfile(str(tmp_path / "AX.bin"), dtype=X.dtype).reshape(X.shape).T
    assert np.abs(AX - g[case + "_AX"]).max() < 1e-9


@pytest.mark.gpu
@pytest.mark.parametrize("libcint", [1, 0])
def test_cpp_host_layer_four_component(tmp_path, libcint):
    """FourCompFock::formGD through the C++ layer against the oracle's
    formGDDirect (water / 6-31G(d), random Hermitian 4C density)."""
    import oracle as O
    from chronusq_public_b200.basis import BasisSet
    from helpers import water_ref
    exe = _build(str(tmp_path))
    b = BasisSet.build(water_ref(), "6-31gd")
    with open(tmp_path / "shells.txt", "w") as f:
        f.write("%d\n" % b.nshell)
        for s in b.shells:
            f.write("%d %d %d %.17g %.17g %.17g\n" % (s.l, int(s.pure), s.nprim, *s.origin))
            f.write(" ".join("%.17g" % a for a in s.alpha) + "\n")
            f.write(" ".join("%.17g" % c for c in s.coef) + "\n")
    rng = np.random.default_rng(7)
    N2 = 2 * b.nbasis
    D = []
    for c in range(4):
        A = rng.standard_normal((N2, N2)) + 1j * rng.standard_normal((N2, N2))
        D.append(0.05 * (A + A.conj().T))
        np.asfortranarray(D[c]).T.tofile(str(tmp_path / ("D%d.bin" % c)))
    subprocess.check_call([exe, str(tmp_path), str(libcint), "4", "1"])
    ref = O.OracleBasis(b).dirac_coulomb(D, libcint=bool(libcint))
    for c in range(4):
        G = np.fromfile(str(tmp_path / ("G%d.bin" % c)), dtype=np.complex128).reshape(N2, N2).T
        assert np.abs(G - ref[c]).max() < 1e-9, c
