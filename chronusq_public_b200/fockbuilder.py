"""``FockBuilder::formGD`` / ``formFock`` for closed-shell real densities.

Restates ``include/fockbuilder/impl.hpp``: ``formRawGDInBatches`` (:109-244)
zeroes J/K, contracts {D, J, HER, COULOMB} and {D, K, HER, EXCHANGE} in one
``twoBodyContract`` call (:139-212) and assembles G = 2J - xHFX K (:223-237);
``formFock`` adds the core Hamiltonian (:280-319).  D is ``onePDM.S``.
"""
from __future__ import annotations

from typing import List, Optional

import numpy as np

from .contraction import (COULOMB, EXCHANGE, DirectTPI,
                          GTODirectTPIContraction, TwoBodyContraction)


class FockBuilder:
    def __init__(self, tpi: DirectTPI):
        self.tpi = tpi
        self.contraction = GTODirectTPIContraction(tpi)

    def formRawGD(self, D, xHFX: float = 1.0, precision: str = "fp64",
                  fp32_cutoff: float = 0.0, increment: bool = False,
                  J=None, K=None):
        """Returns (G, J, K).  With ``increment`` the J/K passed in are
        accumulated (the incremental dD build of formGD, impl.hpp:80-88)."""
        N = self.tpi.nbasis
        if J is None or not increment:
            J = np.zeros((N, N), order="F")
        if K is None or not increment:
            K = np.zeros((N, N), order="F")
        cont = [TwoBodyContraction(D, J, True, COULOMB)]
        if xHFX != 0.0:
            cont.append(TwoBodyContraction(D, K, True, EXCHANGE))
        self.contraction.twoBodyContract(cont, precision=precision,
                                         fp32_cutoff=fp32_cutoff)
        G = 2.0 * J - xHFX * K
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
                                         fp32_cutoff=fp32_cutoff)
        return [2.0 * J - xHFX * K for J, K in zip(Js, Ks)]

    def formFock(self, H, D, **kw):
        G, _J, _K = self.formRawGD(D, **kw)
        return H + G


def two_electron_energy(G, D) -> float:
    """1/4 Tr[G D] (the many-body term of singleslater/quantum.hpp:147-205
    for the scalar component)."""
    return 0.25 * float(np.sum(np.asarray(G) * np.asarray(D).T))
