"""The Gaunt and gauge (Breit) terms on the GPU (cqf_rel_two_body_contract
with GAUNT / GAUGE, cqf_four_comp_gd with gaunt / gauge on) against the
oracle's restatement of the reference's contractions (direct4C_libcint.hpp:
2833-3907, :3908-5160) and against the reference's converged
Dirac-Coulomb-Gaunt and Dirac-Coulomb-Breit builds."""
import numpy as np
import pytest

import oracle as O
from chronusq_public_b200.contraction import (GAUGE, GAUNT, DirectTPI,
                                              GTODirectRelERIContraction, TwoBodyContraction)
from chronusq_public_b200.fockbuilder import FourCompFock
from helpers import gaunt_system
from test_gpu_rel import f_basis, herm, max_rel, water_631gd

pytestmark = pytest.mark.gpu

# entries the GAUNT contraction writes: XLLM*, XSSM*, XLSM*, CLSM*
OUTS_X = [1, 2, 3, 4, 9, 10, 11, 12, 13, 14, 15, 16]
OUTS_C = [17, 18, 19, 20]


def gaunt_inputs(N, seed):
    """The 29 X entries from random Hermitian Pauli components of a 2N x 2N
    density: LL, SS, LS (exchange and Coulomb) and SL blocks."""
    rng = np.random.default_rng(seed)
    D = [herm(2 * N, rng, 0.1) for _ in range(4)]
    LL = [d[:N, :N] for d in D]
    SS = [d[N:, N:] for d in D]
    LS = [d[:N, N:] for d in D]
    SL = [d[N:, :N] for d in D]
    X = [LL[0]] + LL + SS + SS + LS + LS + SL + SL
    return D, [np.asfortranarray(x) for x in X]


def _case(bs, seed, exchange=True, screen=True, ctype=GAUNT):
    tpi, ob = DirectTPI(bs), O.OracleBasis(bs)
    N = bs.nbasis
    _D, X = gaunt_inputs(N, seed)
    ref = ob.rel_contract(X, ctype, exchange, thresh=1e-12 if screen else 0.0)
    lst = [TwoBodyContraction(X[m], np.zeros((N, N), complex)) for m in range(29)]
    GTODirectRelERIContraction(tpi).twoBodyContract(lst, ctype, computeExchange=exchange,
                                                   screen=screen)
    return [c.AX for c in lst], ref


@pytest.mark.parametrize("which", ["water_631gd", "f_basis"])
def test_gaunt_contract_vs_oracle(which):
    bs = water_631gd() if which == "water_631gd" else f_basis()
    got, ref = _case(bs, 31)
    for m in range(29):
        if m in OUTS_X + OUTS_C:
            assert np.abs(ref[m]).max() > 0, m
            assert max_rel(got[m], ref[m]) < 1e-11, m
        else:
            assert np.abs(got[m]).max() == 0, m


def test_gaunt_contract_unscreened_and_no_exchange():
    bs = water_631gd()
    got, ref = _case(bs, 32, exchange=True, screen=False)
    for m in OUTS_X + OUTS_C:
        assert max_rel(got[m], ref[m]) < 1e-11, m
    got, ref = _case(bs, 33, exchange=False)
    for m in OUTS_C:
        assert max_rel(got[m], ref[m]) < 1e-11, m
    for m in OUTS_X:
        assert np.abs(got[m]).max() == 0, m


@pytest.mark.parametrize("name", ["gaunt_upu.npz", "gaunt_cuh3.npz"])
def test_four_comp_gd_gaunt_golden(name):
    """The reference's converged DCG builds: bare Coulomb (libcint) + LLSS +
    Gaunt, SSSS off; G = F - H at the FP64 bar of 1e-9 Eh."""
    bs, D, Gref = gaunt_system(name)
    G = FourCompFock(DirectTPI(bs), DiracCoulombSSSS=False, Gaunt=True).formGD(D)
    for k in range(4):
        assert np.abs(G[k] - Gref[k]).max() < 1e-9, k


def test_four_comp_gd_gaunt_vs_oracle():
    """Every term on (bare, LLSS, SSSS, Gaunt), random Hermitian density,
    exchange scaled."""
    bs = water_631gd()
    D, _X = gaunt_inputs(bs.nbasis, 34)
    ref = O.OracleBasis(bs).dirac_coulomb(D, bare=True, dc=True, ssss=True, gaunt=True,
                                          xHFX=0.6)
    G = FourCompFock(DirectTPI(bs), Gaunt=True).formGD(D, xHFX=0.6)
    for k in range(4):
        assert np.abs(G[k] - ref[k]).max() < 1e-9, k


@pytest.mark.parametrize("which", ["water_631gd", "f_basis"])
def test_gauge_contract_vs_oracle(which):
    bs = water_631gd() if which == "water_631gd" else f_basis()
    got, ref = _case(bs, 35, ctype=GAUGE)
    for m in range(29):
        if m in OUTS_X + OUTS_C:
            assert np.abs(ref[m]).max() > 0, m
            assert max_rel(got[m], ref[m]) < 1e-11, m
        else:
            assert np.abs(got[m]).max() == 0, m


def test_gauge_contract_unscreened_no_exchange():
    bs = water_631gd()
    got, ref = _case(bs, 36, exchange=False, screen=False, ctype=GAUGE)
    for m in OUTS_C:
        assert max_rel(got[m], ref[m]) < 1e-11, m
    for m in OUTS_X:
        assert np.abs(got[m]).max() == 0, m


def test_four_comp_gd_breit_golden():
    """The reference's converged Dirac-Coulomb-Breit build of UPu(184+):
    bare Coulomb + LLSS + SSSS + Gaunt + Gauge, G = F - H at 1e-9 Eh."""
    bs, D, Gref = gaunt_system("breit_upu.npz")
    G = FourCompFock(DirectTPI(bs), Gaunt=True, Gauge=True).formGD(D)
    for k in range(4):
        assert np.abs(G[k] - Gref[k]).max() < 1e-9, k


def test_four_comp_gd_breit_vs_oracle():
    bs = water_631gd()
    D, _X = gaunt_inputs(bs.nbasis, 37)
    ref = O.OracleBasis(bs).dirac_coulomb(D, bare=True, dc=True, ssss=True, gaunt=True,
                                          gauge=True, xHFX=0.8)
    G = FourCompFock(DirectTPI(bs), Gaunt=True, Gauge=True).formGD(D, xHFX=0.8)
    for k in range(4):
        assert np.abs(G[k] - ref[k]).max() < 1e-9, k
