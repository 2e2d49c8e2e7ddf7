"""Host-side mirror of ChronusQ's direct two-body contraction interface.

``TwoBodyContraction`` and ``GTODirectTPIContraction.twoBodyContract`` keep
the names, argument meaning and accumulate semantics of
``include/particleintegrals/twopints.hpp:59-75`` and
``include/particleintegrals/twopints/gtodirecttpi.hpp:143-228``; the work is
done by libcqfock.so on the GPU through the C ABI of include/cqfock.h.

Matrices: N x N, column-major semantics (index [i, j] is row i, column j);
numpy arrays (host, any order) or CUDA torch tensors (device pointers, must
be Fortran-contiguous i.e. ``t.T.contiguous().T`` or symmetric use).  AX is
accumulated (AX += G[X]), as on the reference's multi-threaded path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from . import _cabi
from ._cabi import CQF_COULOMB, CQF_EXCHANGE  # noqa: F401
from .basis import BasisSet

COULOMB, EXCHANGE = CQF_COULOMB, CQF_EXCHANGE


@dataclass
class TwoBodyContraction:
    """``TwoBodyContraction<T>``: AX += G[X] of type contType."""
    X: object
    AX: object
    HER: bool = True
    contType: int = COULOMB


def shell_array(basis: BasisSet):
    """(cqf_shell array, owner) of a basis: the ctypes shells point into
    arrays held by `owner`, which must outlive every use of the shells."""
    f = basis.flat()
    alpha = np.ascontiguousarray(f["alpha"], dtype=np.float64)
    coef = np.ascontiguousarray(f["coef"], dtype=np.float64)
    sh = (_cabi.CqfShell * basis.nshell)()
    dp = C.POINTER(C.c_double)
    off = 0
    for s in range(basis.nshell):
        n = int(f["nprim"][s])
        sh[s].l = int(f["l"][s])
        sh[s].pure = int(f["pure"][s])
        sh[s].nprim = n
        sh[s].alpha = C.cast(alpha.ctypes.data + 8 * off, dp)
        sh[s].coeff = C.cast(coef.ctypes.data + 8 * off, dp)
        for x in range(3):
            sh[s].origin[x] = float(f["origin"][s, x])
        off += n
    return sh, (f, alpha, coef)


class DirectTPI:
    """Device-resident shell pairs and Schwarz bounds of one basis
    (``DirectTPI``, gtodirecttpi.hpp:30-141; threshSchwarz default 1e-12)."""

    def __init__(self, basis: BasisSet, threshSchwarz: float = 1e-12,
                 device: int = 0):
        L = _cabi.lib()
        self.basis = basis
        self.threshSchwarz = threshSchwarz
        self.device = device
        sh, self._keep = shell_array(basis)
        h = C.c_void_p()
        _cabi.check(L.cqf_basis_create(sh, basis.nshell, threshSchwarz, device,
                                       C.byref(h)))
        self.handle = h
        nb, ns, npair = C.c_int(), C.c_int(), C.c_int()
        _cabi.check(L.cqf_basis_info(h, C.byref(nb), C.byref(ns),
                                     C.byref(npair)))
        self.nbasis, self.nshell, self.npair = nb.value, ns.value, npair.value

    def schwarz(self) -> np.ndarray:
        Q = np.zeros((self.nshell, self.nshell), order="F")
        _cabi.check(_cabi.lib().cqf_basis_schwarz(
            self.handle, Q.ctypes.data_as(C.POINTER(C.c_double))))
        return Q

    def one_electron(self):
        """(S, T): overlap and kinetic matrices, computed on the device."""
        N = self.nbasis
        S = np.zeros((N, N), order="F")
        T = np.zeros((N, N), order="F")
        dp = C.POINTER(C.c_double)
        _cabi.check(_cabi.lib().cqf_basis_one_electron(
            self.handle, S.ctypes.data_as(dp), T.ctypes.data_as(dp)))
        return S, T

    def autotune(self, D, precision: str = "fp64", fp32_cutoff: float = 0.0,
                 cache_path: Optional[str] = None) -> bool:
        """``cqf_autotune`` on the closed-shell J and K of the real symmetric
        density D (host array): sets this basis' launch shapes; returns True
        when every class pair came from ``cache_path``."""
        N = self.nbasis
        X = np.asfortranarray(D, dtype=np.float64)
        out = np.zeros((N, N), order="F")
        arr = (_cabi.CqfContraction * 2)()
        for i, t in enumerate((COULOMB, EXCHANGE)):
            arr[i].X = C.c_void_p(X.ctypes.data)
            arr[i].AX = C.c_void_p(out.ctypes.data)
            arr[i].hermitian = 1
            arr[i].type = t
        opts = _cabi.CqfOpts()
        _cabi.lib().cqf_opts_default(C.byref(opts))
        opts.precision = _cabi.CQF_MIXED if precision == "mixed" else _cabi.CQF_FP64
        opts.fp32_cutoff = float(fp32_cutoff)
        hit = C.c_int(0)
        _cabi.check(_cabi.lib().cqf_autotune(
            self.handle, arr, 2, C.byref(opts),
            cache_path.encode() if cache_path else None, C.byref(hit)))
        return bool(hit.value)

    def nuclear(self, nuclei) -> np.ndarray:
        """V: nuclear-attraction matrix in the field of ``nuclei``
        ((natom, 5) rows {Z, x, y, z, zeta}; ``Molecule.nuclei``), computed
        on the device."""
        N = self.nbasis
        nuc = np.ascontiguousarray(nuclei, dtype=np.float64).reshape(-1, 5)
        V = np.zeros((N, N), order="F")
        dp = C.POINTER(C.c_double)
        _cabi.check(_cabi.lib().cqf_basis_nuclear(
            self.handle, len(nuc), nuc.ctypes.data_as(dp), V.ctypes.data_as(dp)))
        return V

    def nuclear_pvp(self, nuclei) -> np.ndarray:
        """(4, N, N): pV.p and the spin-orbit (pV x p)_x,y,z of the four-
        component core Hamiltonian, computed on the device."""
        N = self.nbasis
        nuc = np.ascontiguousarray(nuclei, dtype=np.float64).reshape(-1, 5)
        buf = np.zeros(4 * N * N)
        dp = C.POINTER(C.c_double)
        _cabi.check(_cabi.lib().cqf_basis_nuclear_pvp(
            self.handle, len(nuc), nuc.ctypes.data_as(dp), buf.ctypes.data_as(dp)))
        return np.stack([buf[k * N * N:(k + 1) * N * N].reshape(N, N, order="F")
                         for k in range(4)])

    def four_comp_core_hamiltonian(self, nuclei) -> list:
        """``FourComponent::compute4CCH``: the four Pauli components
        (scalar, MX, MY, MZ) of the 2N x 2N complex core Hamiltonian
        [[V, T], [T, W / 4c^2 - T]] as the reference stores them."""
        M = 2 * self.nbasis
        nuc = np.ascontiguousarray(nuclei, dtype=np.float64).reshape(-1, 5)
        H = [np.zeros((M, M), dtype=np.complex128, order="F") for _ in range(4)]
        hp = (C.c_void_p * 4)(*[h.ctypes.data for h in H])
        _cabi.check(_cabi.lib().cqf_four_comp_core_hamiltonian(
            self.handle, len(nuc), nuc.ctypes.data_as(C.POINTER(C.c_double)), hp))
        return H

    def close(self):
        if getattr(self, "handle", None):
            _cabi.lib().cqf_basis_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _is_torch(x):
    return type(x).__module__.startswith("torch")


def _stream_arg(stream):
    """CUDA stream handle for the C ABI.  None -> the basis' own stream;
    0 (torch's legacy default stream) -> cudaStreamLegacy, so that work is
    ordered with the caller's stream as the caller expects."""
    if stream is None:
        return None
    return C.c_void_p(1 if int(stream) == 0 else int(stream))


class ContractionGraph:
    """A contraction captured as a CUDA graph (``cqf_graph_create``): X and AX
    (CUDA tensors, column-major) are bound at capture; every ``launch`` adds
    G[X] into AX on ``stream`` without synchronising."""

    def __init__(self, tpi: DirectTPI, matList, precision="fp64",
                 fp32_cutoff=0.0, screen=True):
        self.tpi = tpi
        n = len(matList)
        arr = (_cabi.CqfContraction * n)()
        is_c = matList[0].X.is_complex()
        N = tpi.nbasis
        for i, c in enumerate(matList):
            for t in (c.X, c.AX):
                if not (_is_torch(t) and t.is_cuda and tuple(t.shape) == (N, N)
                        and t.stride() == (1, N)):
                    raise ValueError("graph matrices must be column-major CUDA "
                                     "tensors of shape (N, N)")
            arr[i].X = C.c_void_p(c.X.data_ptr())
            arr[i].AX = C.c_void_p(c.AX.data_ptr())
            arr[i].hermitian = 1 if c.HER else 0
            arr[i].type = int(c.contType)
        self._keep = list(matList)
        opts = _cabi.CqfOpts()
        _cabi.lib().cqf_opts_default(C.byref(opts))
        opts.is_complex = 1 if is_c else 0
        opts.screen = 1 if screen else 0
        opts.device_pointers = 1
        opts.precision = _cabi.CQF_MIXED if precision == "mixed" else _cabi.CQF_FP64
        opts.fp32_cutoff = float(fp32_cutoff)
        h = C.c_void_p()
        _cabi.check(_cabi.lib().cqf_graph_create(tpi.handle, arr, n, C.byref(opts),
                                                 C.byref(h)))
        self.handle = h

    def launch(self, stream=None):
        _cabi.check(_cabi.lib().cqf_graph_launch(self.handle, _stream_arg(stream)))

    def close(self):
        if getattr(self, "handle", None):
            _cabi.lib().cqf_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GTODirectTPIContraction:
    """``GTODirectTPIContraction<MatsT,double>`` on the GPU."""

    def __init__(self, tpi: DirectTPI):
        self.tpi = tpi
        self.last_stats: Optional[dict] = None

    def twoBodyContract(self, matList: List[TwoBodyContraction],
                        screen: bool = True, precision: str = "fp64",
                        fp32_cutoff: float = 0.0, stream=None,
                        shard: Tuple[int, int] = (0, 1)) -> None:
        """AX += G[X] for every entry (directScaffoldNew semantics).
        ``shard = (index, count)``: only this process's share of the
        shell-pair work (cqf_opts::shard_index / shard_count); the shares sum
        to the whole contraction."""
        if not matList:
            return
        N = self.tpi.nbasis
        dev = _is_torch(matList[0].X)
        is_c = any((x.X.is_complex() if _is_torch(x.X) else np.iscomplexobj(x.X))
                   for x in matList)
        n = len(matList)
        arr = (_cabi.CqfContraction * n)()
        keep = []
        writeback = []
        conv = {}  # one column-major copy per source X (J and K share D)
        for i, c in enumerate(matList):
            if dev:
                for t in (c.X, c.AX):
                    if tuple(t.shape) != (N, N):
                        raise ValueError("matrix shape must be (N, N)")
                    if not t.is_cuda:
                        raise ValueError("mixing host and device matrices")
                    if t.stride() != (1, N):
                        raise ValueError("device matrices must be column-major"
                                         " (stride (1, N))")
                arr[i].X = C.c_void_p(c.X.data_ptr())
                arr[i].AX = C.c_void_p(c.AX.data_ptr())
            else:
                dt = np.complex128 if is_c else np.float64
                X = conv.get(id(c.X))
                if X is None:
                    X = conv[id(c.X)] = np.asfortranarray(c.X, dtype=dt)
                if X.shape != (N, N):
                    raise ValueError("matrix shape must be (N, N)")
                if not (isinstance(c.AX, np.ndarray) and c.AX.dtype == dt
                        and c.AX.flags.f_contiguous and c.AX.shape == (N, N)):
                    AX = np.asfortranarray(c.AX, dtype=dt)
                    writeback.append((c, AX))
                else:
                    AX = c.AX
                keep += [X, AX]
                arr[i].X = C.c_void_p(X.ctypes.data)
                arr[i].AX = C.c_void_p(AX.ctypes.data)
            arr[i].hermitian = 1 if c.HER else 0
            arr[i].type = int(c.contType)
        opts = _cabi.CqfOpts()
        _cabi.lib().cqf_opts_default(C.byref(opts))
        opts.is_complex = 1 if is_c else 0
        opts.screen = 1 if screen else 0
        opts.device_pointers = 1 if dev else 0
        opts.precision = _cabi.CQF_MIXED if precision == "mixed" else _cabi.CQF_FP64
        opts.fp32_cutoff = float(fp32_cutoff)
        opts.stream = _stream_arg(stream)
        opts.shard_index, opts.shard_count = int(shard[0]), int(shard[1])
        st = _cabi.CqfStats()
        _cabi.check(_cabi.lib().cqf_two_body_contract(
            self.tpi.handle, arr, n, C.byref(opts), C.byref(st)))
        for c, AX in writeback:
            if isinstance(c.AX, np.ndarray):
                c.AX[...] = AX
            else:
                c.AX = AX
        self.last_stats = dict(total=st.quartets_total,
                               screened=st.quartets_screened,
                               fp32=st.quartets_fp32, fp64=st.quartets_fp64,
                               device_ms=st.device_ms)


# ---------------------------------------------------------------- 4C
BARE_COULOMB, LLSS, SSSS, GAUNT, GAUGE = (
    _cabi.CQF_REL_BARE_COULOMB, _cabi.CQF_REL_LLSS, _cabi.CQF_REL_SSSS, _cabi.CQF_REL_GAUNT,
    _cabi.CQF_REL_GAUGE)
# DIRAC_PAULI_SPINOR_COMP order of the 17 (X, AX) entries, and the 12 the
# GAUNT and GAUGE lists add (include/particleintegrals/contract/direct4C_libcint.hpp:
# 279-310)
REL_COMPS = ("CLLMS", "XLLMS", "XLLMX", "XLLMY", "XLLMZ", "CSSMS", "CSSMX",
             "CSSMY", "CSSMZ", "XSSMS", "XSSMX", "XSSMY", "XSSMZ", "XLSMS",
             "XLSMX", "XLSMY", "XLSMZ")
GAUNT_COMPS = REL_COMPS + ("CLSMS", "CLSMX", "CLSMY", "CLSMZ", "CSLMS", "CSLMX",
                           "CSLMY", "CSLMZ", "XSLMS", "XSLMX", "XSLMY", "XSLMZ")


def _stats(st):
    return dict(total=st.quartets_total, screened=st.quartets_screened,
                fp32=st.quartets_fp32, fp64=st.quartets_fp64,
                device_ms=st.device_ms)


def _rel_outputs(contType: int, exchange: bool) -> List[int]:
    """Entries a 4C contraction type writes."""
    four = lambda b: list(range(b, b + 4))  # noqa: E731
    if contType == BARE_COULOMB:
        return [_cabi.CQF_CLLMS] + (four(_cabi.CQF_XLLMS) if exchange else [])
    if contType == LLSS:
        return ([_cabi.CQF_CLLMS] + four(_cabi.CQF_CSSMS)
                + (four(_cabi.CQF_XLSMS) if exchange else []))
    if contType == SSSS:
        return four(_cabi.CQF_CSSMS) + (four(_cabi.CQF_XSSMS) if exchange else [])
    return four(_cabi.CQF_CLSMS) + ((four(_cabi.CQF_XLLMS) + four(_cabi.CQF_XSSMS)
                                     + four(_cabi.CQF_XLSMS)) if exchange else [])


class GTODirectRelERIContraction:
    """``GTODirectRelERIContraction<dcomplex,double>`` on the GPU
    (include/particleintegrals/twopints/gtodirectreleri.hpp:75-94)."""

    def __init__(self, tpi: DirectTPI):
        self.tpi = tpi
        self.last_stats: Optional[dict] = None

    def twoBodyContract(self, matList: List[TwoBodyContraction],
                        contType: int, computeExchange: bool = True,
                        screen: bool = True, precision: str = "fp64",
                        fp32_cutoff: float = 0.0, stream=None,
                        shard: Tuple[int, int] = (0, 1)) -> None:
        """17 entries in REL_COMPS order (29 in GAUNT_COMPS order for
        GAUNT and GAUGE; None for entries the type does not use).  The AX the
        type writes are overwritten (the reference zeroes AX on entry); X and
        AX are N x N complex (numpy, or column-major CUDA complex128 tensors).
        precision="mixed" runs the quartets whose screening bound is below
        fp32_cutoff in FP32 arithmetic (the reference is FP64 throughout;
        GAUNT and GAUGE always run in FP64)."""
        n = (_cabi.CQF_REL_NMAT_GAUNT if contType in (GAUNT, GAUGE)
             else _cabi.CQF_REL_NMAT)
        if len(matList) != n:
            raise ValueError("a 4C contraction list has %d entries" % n)
        N = self.tpi.nbasis
        present = [c for c in matList if c is not None]
        dev = bool(present) and _is_torch(present[0].X)
        outs = set(_rel_outputs(contType, computeExchange))
        xs = (C.c_void_p * n)()
        axs = (C.c_void_p * n)()
        keep, writeback = [], []
        for i, c in enumerate(matList):
            if c is None:
                continue
            if dev:
                for t in (c.X, c.AX):
                    if tuple(t.shape) != (N, N) or not t.is_cuda or t.stride() != (1, N):
                        raise ValueError("device matrices must be (N, N) column-major")
                xs[i] = c.X.data_ptr()
                axs[i] = c.AX.data_ptr()
            else:
                X = np.asfortranarray(c.X, dtype=np.complex128)
                if X.shape != (N, N):
                    raise ValueError("matrix shape must be (N, N)")
                keep.append(X)
                xs[i] = X.ctypes.data
                if i in outs:
                    AX = np.zeros((N, N), dtype=np.complex128, order="F")
                    keep.append(AX)
                    writeback.append((c, AX))
                    axs[i] = AX.ctypes.data
        opts = _cabi.CqfOpts()
        _cabi.lib().cqf_opts_default(C.byref(opts))
        opts.is_complex = 1
        opts.screen = 1 if screen else 0
        opts.precision = _cabi.CQF_MIXED if precision == "mixed" else _cabi.CQF_FP64
        opts.fp32_cutoff = float(fp32_cutoff)
        opts.device_pointers = 1 if dev else 0
        opts.stream = _stream_arg(stream)
        opts.shard_index, opts.shard_count = int(shard[0]), int(shard[1])
        st = _cabi.CqfStats()
        _cabi.check(_cabi.lib().cqf_rel_two_body_contract(
            self.tpi.handle, xs, axs, int(contType), 1 if computeExchange else 0,
            C.byref(opts), C.byref(st)))
        for c, AX in writeback:
            if isinstance(c.AX, np.ndarray) and c.AX.shape == (N, N):
                c.AX[...] = AX
            else:
                c.AX = AX
        self.last_stats = _stats(st)


class DirectGradContraction:
    """``DirectGradContraction<double,double>::gradTwoBodyContract``
    (include/particleintegrals/gradints.hpp:278-283 -> directScaffoldGrad,
    contract/direct.hpp:2198-2571) on the GPU."""

    def __init__(self, tpi: DirectTPI):
        self.tpi = tpi
        self.last_stats: Optional[dict] = None

    def gradTwoBodyContract(self, cList: List[List[TwoBodyContraction]],
                            shell_atom, stream=None,
                            shard: Tuple[int, int] = (0, 1)) -> None:
        """``cList[3 atom + xyz][m]``: the contraction of matrix m for that
        nuclear coordinate (all components share X, HER and contType; each
        its own AX, added into as 1/2 (A + A^T)).  X real symmetric N x N
        (numpy, or column-major CUDA float64 tensors); ``shell_atom[s]``:
        the atom of shell s.  Non-Hermitian and complex X are not built."""
        nGrad = len(cList)
        if nGrad == 0 or nGrad % 3:
            raise ValueError("cList has 3 entries per atom")
        nMat = len(cList[0])
        N = self.tpi.nbasis
        first = cList[0]
        dev = _is_torch(first[0].X)
        arr = (_cabi.CqfContraction * nMat)()
        keep, writeback = [], []
        for m, c in enumerate(first):
            if dev:
                X = c.X
                if tuple(X.shape) != (N, N) or not X.is_cuda or X.stride() != (1, N):
                    raise ValueError("device matrices must be (N, N) column-major")
                arr[m].X = C.c_void_p(X.data_ptr())
            else:
                X = np.asfortranarray(c.X, dtype=np.float64)
                if X.shape != (N, N):
                    raise ValueError("matrix shape must be (N, N)")
                keep.append(X)
                arr[m].X = C.c_void_p(X.ctypes.data)
            arr[m].hermitian = 1 if c.HER else 0
            arr[m].type = int(c.contType)
        axs = (C.c_void_p * (nGrad * nMat))()
        for g, comp in enumerate(cList):
            if len(comp) != nMat:
                raise ValueError("every component has the same matrices")
            for m, c in enumerate(comp):
                if dev:
                    if tuple(c.AX.shape) != (N, N) or c.AX.stride() != (1, N):
                        raise ValueError("device matrices must be (N, N) column-major")
                    axs[g * nMat + m] = c.AX.data_ptr()
                else:
                    if isinstance(c.AX, np.ndarray) and c.AX.dtype == np.float64 \
                            and c.AX.flags.f_contiguous and c.AX.shape == (N, N):
                        AX = c.AX
                    else:
                        AX = np.asfortranarray(c.AX, dtype=np.float64)
                        writeback.append((c, AX))
                    keep.append(AX)
                    axs[g * nMat + m] = AX.ctypes.data
        sa = np.ascontiguousarray(shell_atom, dtype=np.int32)
        if sa.shape != (self.tpi.nshell,):
            raise ValueError("shell_atom has one entry per shell")
        opts = _cabi.CqfOpts()
        _cabi.lib().cqf_opts_default(C.byref(opts))
        opts.device_pointers = 1 if dev else 0
        opts.stream = _stream_arg(stream)
        opts.shard_index, opts.shard_count = int(shard[0]), int(shard[1])
        st = _cabi.CqfStats()
        _cabi.check(_cabi.lib().cqf_grad_two_body_contract(
            self.tpi.handle, sa.ctypes.data_as(C.POINTER(C.c_int)), nGrad // 3, arr, nMat,
            axs, C.byref(opts), C.byref(st)))
        for c, AX in writeback:
            if isinstance(c.AX, np.ndarray) and c.AX.shape == (N, N):
                c.AX[...] = AX
            else:
                c.AX = AX
        self.last_stats = _stats(st)
