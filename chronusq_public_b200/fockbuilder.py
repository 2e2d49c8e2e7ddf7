"""``FockBuilder::formGD`` / ``formFock`` for closed-shell real densities.

Restates ``include/fockbuilder/impl.hpp``: ``formRawGDInBatches`` (:109-244)
zeroes J/K, contracts {D, J, HER, COULOMB} and {D, K, HER, EXCHANGE} in one
``twoBodyContract`` call (:139-212) and assembles G = 2J - xHFX K (:223-237);
``formFock`` adds the core Hamiltonian (:280-319).  D is ``onePDM.S``.

With a ``torch.distributed`` process group the builders split the work the
way the reference splits its shell-pair loop over MPI ranks
(direct.hpp:1600-1604; 4C direct4C_libcint.hpp:933-936): each rank computes
its shard of the bra shell pairs and the shards are summed over the group
(the reference's MPIReduce, direct.hpp:2085-2107), NCCL for device matrices
and host matrices on an NCCL group, the group's own backend otherwise.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np

from .contraction import (COULOMB, EXCHANGE, DirectGradContraction, DirectTPI,
                          GTODirectTPIContraction, TwoBodyContraction, _is_torch)


def _shard_of(group):
    if group is None:
        return (0, 1)
    import torch.distributed as dist
    return (dist.get_rank(group), dist.get_world_size(group))


def allreduce_sum(arrays, group, device: int = 0) -> None:
    """Sums each array (numpy, or torch) over the process group, in place."""
    if group is None:
        return
    import torch
    import torch.distributed as dist
    nccl = dist.get_backend(group) == "nccl"
    for a in arrays:
        if _is_torch(a):
            if not a.is_contiguous() and a.T.is_contiguous():
                a = a.T  # column-major matrices: the same storage
            if a.is_complex():
                a = torch.view_as_real(a)
            if not a.is_contiguous():
                raise ValueError("allreduce_sum: tensors must be contiguous")
            dist.all_reduce(a, group=group)
            continue
        flat = np.ravel(a, order="K")
        if not np.shares_memory(flat, a):
            raise ValueError("allreduce_sum: arrays must be contiguous")
        if np.iscomplexobj(flat):
            flat = flat.view(np.float64)
        t = torch.from_numpy(flat)
        if nccl:
            d = t.to("cuda:%d" % device)
            dist.all_reduce(d, group=group)
            t.copy_(d.cpu())
        else:
            dist.all_reduce(t, group=group)


class FockBuilder:
    """``group``: a torch.distributed process group whose ranks share the
    build (each its shard of the shell-pair work, then a sum); None: the
    whole build on this process."""

    def __init__(self, tpi: DirectTPI, group=None):
        self.tpi = tpi
        self.group = group
        self.contraction = GTODirectTPIContraction(tpi)

    def formRawGD(self, D, xHFX: float = 1.0, precision: str = "fp64",
                  fp32_cutoff: float = 0.0, increment: bool = False,
                  J=None, K=None, G=None):
        """Returns (G, J, K).  With ``increment`` the J/K passed in are
        accumulated (the incremental dD build of formGD, impl.hpp:80-88);
        that build always runs in FP64 -- mixed precision applies to builds
        from the full density, whose FP32 errors do not accumulate over SCF
        iterations the way the increments' would.

        J, K and G given as column-major N x N float64 arrays are the output
        storage, as the reference writes into the SingleSlater's own
        coulombMatrix / exchangeMatrix / twoeH (impl.hpp:131-137, :223-237):
        outside ``increment`` they are zeroed in place, so an SCF loop that
        passes the same arrays every iteration allocates nothing."""
        if increment:
            precision = "fp64"
        N = self.tpi.nbasis

        def _out(A, keep):
            if A is None:
                return np.zeros((N, N), order="F")
            if (not isinstance(A, np.ndarray) or A.shape != (N, N)
                    or A.dtype != np.float64 or not A.flags.f_contiguous):
                raise ValueError("formRawGD: outputs must be column-major "
                                 "(N, N) float64 arrays")
            if not keep:
                A.fill(0.0)
            return A

        if increment and (J is None or K is None):
            raise ValueError("formRawGD: increment accumulates into J and K")
        J = _out(J, increment)
        K = _out(K, increment)
        shard = _shard_of(self.group)
        if increment and shard[1] > 1:
            # the increments of every shard go into zeroed buffers; the sum
            # is added once
            J0, K0 = J, K
            J, K = np.zeros((N, N), order="F"), np.zeros((N, N), order="F")
        cont = [TwoBodyContraction(D, J, True, COULOMB)]
        if xHFX != 0.0:
            cont.append(TwoBodyContraction(D, K, True, EXCHANGE))
        self.contraction.twoBodyContract(cont, precision=precision,
                                         fp32_cutoff=fp32_cutoff, shard=shard)
        allreduce_sum([J, K], self.group, self.tpi.device)
        if increment and shard[1] > 1:
            J0 += J
            K0 += K
            J, K = J0, K0
        if G is None:
            G = 2.0 * J - xHFX * K
        else:
            G = _out(G, True)
            np.multiply(J, 2.0, out=G)
            if xHFX == 1.0:
                np.subtract(G, K, out=G)
            elif xHFX != 0.0:
                G -= xHFX * K
        return G, J, K

    def formRawGDBatch(self, Ds: List[np.ndarray], xHFX: float = 1.0,
                       precision: str = "fp64", fp32_cutoff: float = 0.0):
        """Many densities in one contraction (formRawGDInBatches with
        nBatch > 1, as MOIntsTransformer uses it)."""
        N = self.tpi.nbasis
        Js = [np.zeros((N, N), order="F") for _ in Ds]
        Ks = [np.zeros((N, N), order="F") for _ in Ds]
        cont = []
        for D, J, K in zip(Ds, Js, Ks):
            cont.append(TwoBodyContraction(D, J, True, COULOMB))
            if xHFX != 0.0:
                cont.append(TwoBodyContraction(D, K, True, EXCHANGE))
        self.contraction.twoBodyContract(cont, precision=precision,
                                         fp32_cutoff=fp32_cutoff,
                                         shard=_shard_of(self.group))
        allreduce_sum(Js + Ks, self.group, self.tpi.device)
        return [2.0 * J - xHFX * K for J, K in zip(Js, Ks)]

    def formFock(self, H, D, **kw):
        G, _J, _K = self.formRawGD(D, **kw)
        return H + G

    def getGDGrad(self, D, shell_atom, natom: int, xHFX: float = 1.0) -> np.ndarray:
        """``FockBuilder::getGDGrad`` (include/fockbuilder/impl.hpp:400-497)
        for a closed-shell real density: the two-electron energy gradient
        1/4 Tr[D (2 J^x - xHFX K^x)] for every nuclear coordinate, (natom, 3),
        with J^x / K^x from the gradient contraction."""
        N = self.tpi.nbasis
        cList, JL, KL = [], [], []
        for _ in range(3 * natom):
            J = np.zeros((N, N), order="F")
            comp = [TwoBodyContraction(D, J, True, COULOMB)]
            JL.append(J)
            if abs(xHFX) > 1e-12:
                K = np.zeros((N, N), order="F")
                comp.append(TwoBodyContraction(D, K, True, EXCHANGE))
                KL.append(K)
            cList.append(comp)
        DirectGradContraction(self.tpi).gradTwoBodyContract(
            cList, shell_atom, shard=_shard_of(self.group))
        allreduce_sum(JL + KL, self.group, self.tpi.device)
        Dt = np.asarray(D).T
        out = np.zeros(3 * natom)
        for g in range(3 * natom):
            G = 2.0 * JL[g] - (xHFX * KL[g] if KL else 0.0)
            out[g] = 0.25 * float(np.sum(G * Dt))
        return out.reshape(natom, 3)


def two_electron_energy(G, D) -> float:
    """1/4 Tr[G D] (the many-body term of singleslater/quantum.hpp:147-205
    for the scalar component)."""
    return 0.25 * float(np.sum(np.asarray(G) * np.asarray(D).T))


class FourCompFock:
    """``FourCompFock<dcomplex,double>::formGDDirect``
    (include/fockbuilder/fourcompfock/impl.hpp:3752-4636) on the GPU.

    Hamiltonian switches as the reference's HamiltonianOptions (BareCoulomb,
    DiracCoulomb, DiracCoulombSSSS, Libcint, Gaunt, Gauge; with Gauge the
    Gaunt and gauge terms are weighted C^2 / 2, the Breit interaction); the
    density is the four Pauli
    components (scalar, MX, MY, MZ) of the 2N x 2N complex 4C one-particle
    density (LL block first).  ``formGD`` returns the same four components of
    G = twoeH - xHFX K.
    """

    def __init__(self, tpi: DirectTPI, BareCoulomb: bool = True,
                 DiracCoulomb: bool = True, DiracCoulombSSSS: bool = True,
                 Libcint: bool = True, Gaunt: bool = False, Gauge: bool = False,
                 group=None):
        self.tpi = tpi
        self.group = group
        self.BareCoulomb = BareCoulomb
        self.DiracCoulomb = DiracCoulomb
        self.DiracCoulombSSSS = DiracCoulombSSSS
        self.Libcint = Libcint
        self.Gaunt = Gaunt
        self.Gauge = Gauge
        self.last_stats = None

    def formGD(self, D: List, xHFX: float = 1.0, screen: bool = True,
               precision: str = "fp64", fp32_cutoff: float = 0.0,
               stream=None) -> List:
        import ctypes as C

        from . import _cabi
        from .contraction import _is_torch, _stats, _stream_arg
        if len(D) != 4:
            raise ValueError("D is the list of 4 Pauli components")
        N2 = 2 * self.tpi.nbasis
        dev = _is_torch(D[0])
        dp = (C.c_void_p * 4)()
        gp = (C.c_void_p * 4)()
        keep = []
        if dev:
            import torch
            G = [torch.zeros((N2, N2), dtype=torch.complex128, device=D[0].device).T
                 for _ in range(4)]
            for c in range(4):
                if tuple(D[c].shape) != (N2, N2) or D[c].stride() != (1, N2):
                    raise ValueError("device densities must be (2N, 2N) column-major")
                dp[c] = D[c].data_ptr()
                gp[c] = G[c].data_ptr()
        else:
            G = [np.zeros((N2, N2), dtype=np.complex128, order="F") for _ in range(4)]
            for c in range(4):
                Dc = np.asfortranarray(D[c], dtype=np.complex128)
                if Dc.shape != (N2, N2):
                    raise ValueError("density components must be (2N, 2N)")
                keep.append(Dc)
                dp[c] = Dc.ctypes.data
                gp[c] = G[c].ctypes.data
        dco = _cabi.CqfDcOpts()
        _cabi.lib().cqf_dc_opts_default(C.byref(dco))
        dco.bare_coulomb = int(self.BareCoulomb)
        dco.dirac_coulomb = int(self.DiracCoulomb)
        dco.dirac_coulomb_ssss = int(self.DiracCoulombSSSS)
        dco.libcint = int(self.Libcint)
        dco.gaunt = int(self.Gaunt)
        dco.gauge = int(self.Gauge)
        dco.xHFX = float(xHFX)
        opts = _cabi.CqfOpts()
        _cabi.lib().cqf_opts_default(C.byref(opts))
        opts.is_complex = 1
        opts.screen = 1 if screen else 0
        opts.precision = _cabi.CQF_MIXED if precision == "mixed" else _cabi.CQF_FP64
        opts.fp32_cutoff = float(fp32_cutoff)
        opts.device_pointers = 1 if dev else 0
        opts.stream = _stream_arg(stream)
        opts.shard_index, opts.shard_count = _shard_of(self.group)
        st = _cabi.CqfStats()
        _cabi.check(_cabi.lib().cqf_four_comp_gd(
            self.tpi.handle, dp, gp, C.byref(dco), C.byref(opts), C.byref(st)))
        if dev and self.group is not None:
            import torch
            torch.cuda.synchronize(D[0].device)
        allreduce_sum(G, self.group, self.tpi.device)
        self.last_stats = _stats(st)
        return G
