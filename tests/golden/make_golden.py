"""Generate the golden fixtures under tests/golden/ from the reference's own
test data.  Run once where the reference checkout is available:

    python tests/golden/make_golden.py /path/to/chronusq_public

Sources (paths within xsligroup/chronusq_public):
* tests/func/reference/contract.hdf5 -- direct J/K of random X on water /
  cc-pVTZ (tests/func/input/contract_ref.inp), checked by
  tests/func/contract.cxx:97-190 at max|dAX| < 1e-9.  The 8 cases and their
  (HER, contraction type) arguments follow contract.cxx:195-316, including the
  two quirks (NONHER/REAL/K runs COULOMB, NONHER/COMPLEX/K runs HERMITIAN
  EXCHANGE).
* tests/scf/reference/water_cc-pVDZ_RHF_RHFGuess_READDEN_scratch.bin.ref --
  one direct RHF build from a read density (tests/scf/rhf.cxx:74-110); the
  basis is the inline uncontracted cc-pVDZ of
  tests/scf/serial/rhf/water_cc-pVDZ_RHF_READDEN.inp.
* tests/scf/reference/water_cc-pVDZ_DC-HF_RHFGuess_READDEN.bin.ref -- one 4C
  Dirac-Coulomb build (tests/scf/fourcomphf.cxx:143-150).
* tests/scf/reference/UPu_184+_P_DCG_finitenuc.bin.ref and CuH3_321g_DCG.bin.ref
  -- converged 4C Dirac-Coulomb-Gaunt SCFs (inputs under
  tests/scf/serial/fourcomp/): D and G = F - H of the final build.
* tests/scf/reference/UPu_184+_P_DCGGS_finitenuc.bin.ref -- the same with
  SSSS, Gaunt and Gauge on (Dirac-Coulomb-Breit).

HDF5 datasets written from column-major buffers read back transposed; the
fixtures store them in natural (row = first index) orientation.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from h5lite import H5File  # noqa: E402

# (dataset group, HER flag, contraction type: 0 COULOMB / 1 EXCHANGE)
CONTRACT_CASES = [
    ("HER/REAL/J", 1, 0), ("NONHER/REAL/J", 0, 0),
    ("HER/REAL/K", 1, 1), ("NONHER/REAL/K", 0, 0),
    ("HER/COMPLEX/J", 1, 0), ("NONHER/COMPLEX/J", 0, 0),
    ("HER/COMPLEX/K", 1, 1), ("NONHER/COMPLEX/K", 1, 1),
]


def _inline_basis(inp_path):
    txt = open(inp_path).read()
    return txt.split("BasisDef:")[1].split("[MISC]")[0]


def _geometry(text):
    """The [Molecule] geom: lines as 'Sym x y z' strings (Angstrom)."""
    lines = text.splitlines()
    i = [k for k, l in enumerate(lines) if l.strip().lower().startswith("geom")][0]
    out = []
    for l in lines[i + 1:]:
        t = l.split()
        if len(t) != 4 or not t[0].isalpha():
            break
        out.append(" ".join(t))
    return "\n".join(out)


def _basis_name(text):
    for l in text.splitlines():
        t = l.replace("=", " ").split()
        if len(t) == 2 and t[0].lower() == "basis":
            return t[1].lower()
    raise ValueError("no basis name")


def main(ref_root):
    f = H5File(os.path.join(ref_root, "tests/func/reference/contract.hdf5"))
    out = {}
    for g, her, ty in CONTRACT_CASES:
        key = g.replace("/", "_")
        out[key + "_X"] = f.read("/CONTRACTION/%s/X" % g).T.copy()
        out[key + "_AX"] = f.read("/CONTRACTION/%s/AX" % g).T.copy()
        out[key + "_her"] = np.int32(her)
        out[key + "_type"] = np.int32(ty)
    np.savez_compressed(os.path.join(HERE, "contract.npz"), **out)

    rd = os.path.join(ref_root, "tests/scf/reference")
    f = H5File(os.path.join(
        rd, "water_cc-pVDZ_RHF_RHFGuess_READDEN_scratch.bin.ref"))
    rhf = {k: f.read(p).T.copy() for k, p in [
        ("D", "/SCF/1PDM_SCALAR"), ("F", "/SCF/FOCK_SCALAR"),
        ("H", "/INTS/CORE_HAMILTONIAN_SCALAR"), ("S", "/INTS/OVERLAP"),
        ("T", "/INTS/KINETIC")]}
    rhf["E_total"] = f.read("/SCF/TOTAL_ENERGY")
    rhf["E_many_body"] = f.read("/SCF/MANY_BODY_ENERGY")
    rhf["basisdef"] = np.array(_inline_basis(os.path.join(
        ref_root, "tests/scf/serial/rhf/water_cc-pVDZ_RHF_READDEN.inp")))
    np.savez_compressed(os.path.join(HERE, "readden_rhf.npz"), **rhf)

    f = H5File(os.path.join(rd, "water_cc-pVDZ_DC-HF_RHFGuess_READDEN.bin.ref"))
    dc = {}
    for comp in ("SCALAR", "MX", "MY", "MZ"):
        dc["D_" + comp] = f.read("/SCF/1PDM_" + comp).T.copy()
        dc["F_" + comp] = f.read("/SCF/FOCK_" + comp).T.copy()
        dc["H_" + comp] = f.read("/INTS/CORE_HAMILTONIAN_" + comp).T.copy()
    dc["S"] = f.read("/INTS/OVERLAP").T.copy()
    dc["T"] = f.read("/INTS/KINETIC").T.copy()
    dc["E_total"] = f.read("/SCF/TOTAL_ENERGY")
    dc["E_many_body"] = f.read("/SCF/MANY_BODY_ENERGY")
    dc["basisdef"] = np.array(_inline_basis(os.path.join(
        ref_root, "tests/scf/serial/fourcomp/water_cc-pVDZ_DC-HF_READDEN.inp")))
    np.savez_compressed(os.path.join(HERE, "readden_dc.npz"), **dc)

    # 4C build from a full 4C density (DC-HF guess, libcint, bare Coulomb
    # only -- the stored FOCK has zero SS / LS two-electron blocks): the LL
    # blocks of D and of G = FOCK - CORE_H, all four Pauli components.
    f = H5File(os.path.join(rd, "water_cc-pVDZ_DC-HF_DCHFGuess_READDEN_scratch.bin.ref"))
    N = 40
    out = {}
    for comp in ("SCALAR", "MX", "MY", "MZ"):
        D = f.read("/SCF/1PDM_" + comp).T
        G = f.read("/SCF/FOCK_" + comp).T - f.read("/INTS/CORE_HAMILTONIAN_" + comp).T
        out["D_" + comp] = np.where(np.abs(D) < 1e-200, 0, D)[:N, :N].copy()
        out["G_" + comp] = np.where(np.abs(G) < 1e-200, 0, G)[:N, :N].copy()
    np.savez_compressed(os.path.join(HERE, "readden_dchf_ll.npz"), **out)

    # converged complex 4C-HF water / 6-31G(d) with Dirac-Coulomb (LLSS) on,
    # SSSS off, non-libcint bare Coulomb
    # (tests/scf/serial/qn/water_6-31Gd_4chf_bfgs.inp): D and G = F - H.
    f = H5File(os.path.join(rd, "water_6-31Gd_qn_4chf.bin.ref"))
    out = {}
    for comp in ("SCALAR", "MX", "MY", "MZ"):
        D = f.read("/SCF/1PDM_" + comp).T
        G = f.read("/SCF/FOCK_" + comp).T - f.read("/INTS/CORE_HAMILTONIAN_" + comp).T
        out["D_" + comp] = np.where(np.abs(D) < 1e-200, 0, D).copy()
        out["G_" + comp] = np.where(np.abs(G) < 1e-200, 0, G).copy()
    np.savez_compressed(os.path.join(HERE, "qn_4chf_dc.npz"), **out)

    # converged four-component Dirac-Coulomb-Gaunt SCF references (bare
    # Coulomb + Dirac-Coulomb LLSS + Gaunt, SSSS off, libcint, in-core
    # integrals): D and G = F - H of the final build, with the molecule and
    # basis of each input
    for name, inp, key in [
            ("UPu_184+_P_DCG_finitenuc", "tests/scf/serial/fourcomp/UPu_184+_P_DCG_finitenuc.inp",
             "gaunt_upu"),
            ("CuH3_321g_DCG", "tests/scf/serial/fourcomp/CuH3_321g_DCG.inp", "gaunt_cuh3"),
            # bare + Dirac-Coulomb + SSSS + Gaunt + Gauge (Breit)
            ("UPu_184+_P_DCGGS_finitenuc",
             "tests/scf/serial/fourcomp/UPu_184+_P_DCGGS_finitenuc.inp", "breit_upu")]:
        f = H5File(os.path.join(rd, name + ".bin.ref"))
        out = {}
        for comp in ("SCALAR", "MX", "MY", "MZ"):
            D = f.read("/SCF/1PDM_" + comp).T
            G = f.read("/SCF/FOCK_" + comp).T - f.read("/INTS/CORE_HAMILTONIAN_" + comp).T
            out["D_" + comp] = np.where(np.abs(D) < 1e-200, 0, D).copy()
            out["G_" + comp] = np.where(np.abs(G) < 1e-200, 0, G).copy()
        text = open(os.path.join(ref_root, inp)).read()
        out["geometry"] = np.array(_geometry(text))
        if "DefineBasis" in text:
            out["basisdef"] = np.array(_inline_basis(os.path.join(ref_root, inp)))
        else:
            out["basisname"] = np.array(_basis_name(text))
        np.savez_compressed(os.path.join(HERE, key + ".npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the ChronusQ source tree>")
    main(sys.argv[1])
