"""ctypes front-end of the CPU oracle (test infrastructure only).

Loaded by tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline /
reference arm -- never by the chronusq_public_b200 package.  The C++ side
(``cqf_oracle.cpp``) restates ChronusQ's ``directScaffoldNew``
(include/particleintegrals/contract/direct.hpp:1412-2123) with its own
McMurchie-Davidson ERIs.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libcqf_oracle.so")

_lib = None


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB_PATH) or (
            os.path.getmtime(LIB_PATH)
            < os.path.getmtime(os.path.join(HERE, "cqf_oracle.cpp"))):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.orc_basis_new.restype = C.c_void_p
        L.orc_basis_new.argtypes = [C.c_int, ip, ip, ip, dp, dp, dp, C.c_int]
        L.orc_basis_free.argtypes = [C.c_void_p]
        L.orc_nbasis.argtypes = [C.c_void_p]
        L.orc_nbasis.restype = C.c_int
        L.orc_coefs.argtypes = [C.c_void_p, dp]
        L.orc_boys.argtypes = [C.c_int, C.c_double]
        L.orc_boys.restype = C.c_double
        L.orc_overlap_kinetic.argtypes = [C.c_void_p, dp, dp]
        L.orc_nuclear.argtypes = [C.c_void_p, C.c_int, dp, dp]
        L.orc_nuclear_pvp.argtypes = [C.c_void_p, C.c_int, dp, dp]
        L.orc_eri_quartet.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      C.c_int, dp]
        L.orc_eri_quartet.restype = C.c_int
        L.orc_schwarz.argtypes = [C.c_void_p, dp]
        L.orc_sig_pairs.argtypes = [C.c_void_p, ip, ip]
        L.orc_sig_pairs.restype = C.c_int
        L.orc_contract.argtypes = [C.c_void_p, C.c_int, C.c_int, ip, ip,
                                   C.POINTER(C.c_void_p),
                                   C.POINTER(C.c_void_p), C.c_double, C.c_int,
                                   C.c_int, C.POINTER(C.c_longlong)]
        L.orc_contract_part.argtypes = L.orc_contract.argtypes + [C.c_int, C.c_int]
        L.orc_contract_part.restype = C.c_int
        L.orc_grad_contract.argtypes = [C.c_void_p, ip, C.c_int, C.c_int, ip,
                                        C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int]
        L.orc_grad_contract.restype = C.c_int
        L.orc_flops.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                                C.c_double, C.c_double, dp]
        L.orc_dirac_coulomb.argtypes = [C.c_void_p, C.POINTER(C.c_void_p),
                                        C.POINTER(C.c_void_p), C.c_int, C.c_int,
                                        C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                        C.c_int]
        L.orc_dirac_coulomb.restype = C.c_int
        L.orc_rel_contract.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_void_p),
                                       C.POINTER(C.c_void_p), C.c_double, C.c_int]
        L.orc_rel_contract.restype = C.c_int
        L.orc_eri_deriv_quartet.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int,
                                            C.c_int, C.c_int, dp]
        L.orc_eri_deriv_quartet.restype = C.c_int
        L.orc_r12_deriv_quartet.argtypes = [C.c_void_p] + [C.c_int] * 7 + [dp]
        L.orc_r12_deriv_quartet.restype = C.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class OracleBasis:
    """Oracle view of a ``chronusq_public_b200.basis.BasisSet``.

    The oracle normalises the raw .gbs coefficients itself (independently of
    the package's Python normalisation) unless ``use_raw=False``.
    """

    def __init__(self, basis, use_raw: bool = True):
        f = basis.flat()
        self._keep = f
        self.nbasis = basis.nbasis
        self.nshell = basis.nshell
        coef = f["coef_raw"] if use_raw else f["coef"]
        coef = np.ascontiguousarray(coef, dtype=np.float64)
        self._coef = coef
        self.h = lib().orc_basis_new(
            basis.nshell, _ip(f["l"]), _ip(f["pure"]), _ip(f["nprim"]),
            _dp(f["alpha"]), _dp(coef), _dp(f["origin"]), 1 if use_raw else 0)
        self.sizes = basis.sizes
        self.offsets = basis.offsets

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_basis_free(self.h)
                self.h = None
        except Exception:
            pass

    def coefs(self):
        out = np.zeros(len(self._coef))
        lib().orc_coefs(self.h, _dp(out))
        return out

    def overlap_kinetic(self):
        N = self.nbasis
        S = np.zeros((N, N), order="F")
        T = np.zeros((N, N), order="F")
        lib().orc_overlap_kinetic(self.h, _dp(S), _dp(T))
        return S, T

    def nuclear(self, nuclei):
        """V (N x N): nuclei = (natom, 5) rows {Z, x, y, z, zeta}, zeta = 0
        for a point charge (orc_nuclear)."""
        N = self.nbasis
        nuc = np.ascontiguousarray(nuclei, dtype=np.float64)
        V = np.zeros((N, N), order="F")
        lib().orc_nuclear(self.h, len(nuc), _dp(nuc), _dp(V))
        return V

    def nuclear_pvp(self, nuclei):
        """[pV.p, (pVxp)_x, (pVxp)_y, (pVxp)_z], each N x N (orc_nuclear_pvp)."""
        N = self.nbasis
        nuc = np.ascontiguousarray(nuclei, dtype=np.float64)
        W = np.zeros((4, N, N))
        buf = np.zeros(4 * N * N)
        lib().orc_nuclear_pvp(self.h, len(nuc), _dp(nuc), _dp(buf))
        for k in range(4):
            W[k] = buf[k * N * N:(k + 1) * N * N].reshape(N, N, order="F")
        return W

    def eri_quartet(self, s1, s2, s3, s4):
        n = [int(self.sizes[s]) for s in (s1, s2, s3, s4)]
        out = np.zeros(int(np.prod(n)) * 16)
        k = lib().orc_eri_quartet(self.h, s1, s2, s3, s4, _dp(out))
        return out[:k].reshape(n)

    def eri_deriv_quartet(self, s1, s2, s3, s4, dmask):
        """(ncomp, n1, n2, n3, n4) derivative ERIs, derivatives (d/dr of the
        orbital) on the centres in dmask (bit 0..3 = s1..s4); component index
        over the differentiated centres in order, the last fastest."""
        n = [int(self.sizes[s]) for s in (s1, s2, s3, s4)]
        nd = bin(dmask & 15).count("1")
        out = np.zeros(3 ** nd * int(np.prod(n)))
        k = lib().orc_eri_deriv_quartet(self.h, s1, s2, s3, s4, dmask, _dp(out))
        return out[:k].reshape([3 ** nd] + n)

    def r12_deriv_quartet(self, s1, s2, s3, s4, dmask, i=-1, j=-1):
        """As eri_deriv_quartet with the kernel d_i d_j r12 (i, j = 0..2,
        -1 for none; derivatives in r = r1 - r2) in place of 1 / r12."""
        n = [int(self.sizes[s]) for s in (s1, s2, s3, s4)]
        nd = bin(dmask & 15).count("1")
        out = np.zeros(3 ** nd * int(np.prod(n)))
        k = lib().orc_r12_deriv_quartet(self.h, s1, s2, s3, s4, dmask, i, j, _dp(out))
        return out[:k].reshape([3 ** nd] + n)

    def schwarz(self):
        Q = np.zeros((self.nshell, self.nshell), order="F")
        lib().orc_schwarz(self.h, _dp(Q))
        return Q

    def sig_pairs(self):
        n = lib().orc_sig_pairs(self.h, None, None)
        a = np.zeros(n, dtype=np.int32)
        b = np.zeros(n, dtype=np.int32)
        lib().orc_sig_pairs(self.h, _ip(a), _ip(b))
        return a, b

    def contract(self, mats, her, types, thresh=1e-12, nthreads=0,
                 screen=True, AX=None, mpi=(0, 1)):
        """Restated ``twoBodyContract``: returns the list of AX (accumulated
        into ``AX`` when given).  ``mats``: N x N arrays (real or complex).
        ``mpi = (rank, size)``: this rank's part under the reference's MPI
        split of the shell-pair loop."""
        is_c = any(np.iscomplexobj(m) for m in mats)
        dt = np.complex128 if is_c else np.float64
        Xs = [np.asfortranarray(m, dtype=dt) for m in mats]
        if AX is None:
            AX = [np.zeros_like(x, order="F") for x in Xs]
        else:
            AX = [np.asfortranarray(a, dtype=dt) for a in AX]
        n = len(Xs)
        xp = (C.c_void_p * n)(*[x.ctypes.data for x in Xs])
        ap = (C.c_void_p * n)(*[a.ctypes.data for a in AX])
        h = np.array(her, dtype=np.int32)
        t = np.array(types, dtype=np.int32)
        st = (C.c_longlong * 3)()
        rc = lib().orc_contract_part(self.h, n, 1 if is_c else 0, _ip(h), _ip(t), xp, ap,
                                     thresh, nthreads, 1 if screen else 0, st,
                                     int(mpi[0]), int(mpi[1]))
        if rc:
            raise ValueError("mpi rank outside [0, size)")
        self.last_stats = dict(total=st[0], screened=st[1], computed=st[2])
        return AX

    def grad_contract(self, mats, types, shell_atom, natom, nthreads=0):
        """Restated ``DirectGradContraction::directScaffoldGrad`` on real
        symmetric ``mats``: returns [3 * natom][len(mats)] N x N arrays, the
        contractions of d(mu nu|la si)/dR for every atom and x, y, z."""
        N = self.nbasis
        Xs = [np.asfortranarray(m, dtype=np.float64) for m in mats]
        n = len(Xs)
        out = [[np.zeros((N, N), order="F") for _ in range(n)] for _ in range(3 * natom)]
        flat = [a for comp in out for a in comp]
        xp = (C.c_void_p * n)(*[x.ctypes.data for x in Xs])
        ap = (C.c_void_p * len(flat))(*[a.ctypes.data for a in flat])
        sa = np.ascontiguousarray(shell_atom, dtype=np.int32)
        t = np.ascontiguousarray(types, dtype=np.int32)
        lib().orc_grad_contract(self.h, _ip(sa), int(natom), n, _ip(t), xp, ap, nthreads)
        return out

    def dirac_coulomb(self, D, bare=True, dc=True, ssss=True, xHFX=1.0,
                      thresh=1e-12, libcint=True, gaunt=False, gauge=False):
        """FourCompFock::formGDDirect: D = [S, X, Y, Z] Pauli components of
        the 2N x 2N density; returns G = twoeH - xHFX K (same layout)."""
        Ds = [np.asfortranarray(d, dtype=np.complex128) for d in D]
        Gs = [np.zeros_like(d, order="F") for d in Ds]
        dp_ = (C.c_void_p * 4)(*[d.ctypes.data for d in Ds])
        gp_ = (C.c_void_p * 4)(*[g.ctypes.data for g in Gs])
        lib().orc_dirac_coulomb(self.h, dp_, gp_, int(bare), int(dc), int(ssss),
                                xHFX, thresh, int(libcint), int(gaunt), int(gauge))
        return Gs

    def rel_contract(self, X, contType, exchange=True, thresh=1e-12):
        """GTODirectRelERIContraction::twoBodyContract: X = the 17 N x N
        complex matrices (29 for GAUNT and GAUGE, contType 3 and 4;
        DIRAC_PAULI_SPINOR_COMP order); returns as many AX."""
        n = 29 if contType in (3, 4) else 17
        assert len(X) == n
        Xs = [np.asfortranarray(x, dtype=np.complex128) for x in X]
        AX = [np.zeros_like(x, order="F") for x in Xs]
        xp = (C.c_void_p * n)(*[x.ctypes.data for x in Xs])
        ap = (C.c_void_p * n)(*[a.ctypes.data for a in AX])
        lib().orc_rel_contract(self.h, int(contType), xp, ap, thresh,
                               1 if exchange else 0)
        return AX

    def flops(self, mats, thresh=1e-12, fp32_cut=0.0):
        Xs = [np.asfortranarray(np.abs(m), dtype=np.float64) for m in mats]
        n = len(Xs)
        xp = (C.c_void_p * n)(*[x.ctypes.data for x in Xs])
        out = np.zeros(4)
        lib().orc_flops(self.h, n, xp, thresh, fp32_cut, _dp(out))
        return dict(f64=out[0], f32=out[1], quartets=out[2], q32=out[3])


def boys(m: int, T: float) -> float:
    return lib().orc_boys(m, T)


COULOMB, EXCHANGE = 0, 1
