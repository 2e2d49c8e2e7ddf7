"""Algorithmic FLOP count of one direct J/K build (the frozen
McMurchie-Davidson count model).

Per primitive quartet (l_ab = la+lb, l_cd = lc+ld, L = l_ab+l_cd,
H(n) = (n+1)(n+2)(n+3)/6, c(l) = (l+1)(l+2)/2):
  20 + 3L + 3 sum_{n=0..L} H(L-n) + 2 H(lab) H(lcd) c(lc) c(ld)
  + 2 c(la) c(lb) H(lab) c(lc) c(ld) + 3 [c(la) c(lb) H(lab) + c(lc) c(ld) H(lcd)]
per contracted quartet: + Cartesian-to-spherical transform
  (2 sum over centres of n_sph n_cart x remaining dims) + 12 n1 n2 n3 n4 per
density (J: 2 FMAs, K: 4 FMAs per integral).
Quartets: the unique (8-fold) quartets over significant pairs that survive
the reference screen max(shell-block norms) x Q12 x Q34 >= thresh
(include/particleintegrals/contract/direct.hpp:1642-1762).  Quartets whose
bound is below ``fp32_cut`` are counted as FP32 work.
"""
from __future__ import annotations

import numpy as np


def _H(n):
    return (n + 1.0) * (n + 2.0) * (n + 3.0) / 6.0


def _c(l):
    return (l + 1.0) * (l + 2.0) / 2.0


def flop_prim(la, lb, lc, ld):
    lab, lcd = la + lb, lc + ld
    L = lab + lcd
    s = sum(_H(L - n) for n in range(int(L) + 1))
    return (20 + 3.0 * L + 3.0 * s + 2 * _H(lab) * _H(lcd) * _c(lc) * _c(ld)
            + 2 * _c(la) * _c(lb) * _H(lab) * _c(lc) * _c(ld)
            + 3 * (_c(la) * _c(lb) * _H(lab) + _c(lc) * _c(ld) * _H(lcd)))


def _sph_flops(ls, pure):
    dims = [_c(l) for l in ls]
    f = 0.0
    for k in range(4):
        if not pure[k]:
            continue
        rest = 1.0
        for q in range(4):
            if q != k:
                rest *= dims[q]
        f += 2.0 * (2 * ls[k] + 1) * _c(ls[k]) * rest
        dims[k] = 2 * ls[k] + 1
    return f


def shell_block_norms(basis, X):
    """Infinity norms of all shell blocks (direct.hpp:73-90)."""
    A = np.abs(np.asarray(X))
    ns = basis.nshell
    out = np.zeros((ns, ns))
    offs, sizes = basis.offsets, basis.sizes
    for s1 in range(ns):
        rows = A[offs[s1]:offs[s1] + sizes[s1]]
        for s2 in range(ns):
            out[s1, s2] = rows[:, offs[s2]:offs[s2] + sizes[s2]].sum(1).max()
    return out


def build_flops(basis, Q, mats, nmat_digest=None, thresh=1e-12, fp32_cut=0.0):
    """dict(f64, f32, quartets, q32) for one build with densities ``mats``.

    Q: Schwarz table (nshell x nshell, zero for insignificant pairs)."""
    ns = basis.nshell
    norms = np.zeros((ns, ns))
    for X in mats:
        norms = np.maximum(norms, shell_block_norms(basis, X))
    nd = len(mats) if nmat_digest is None else nmat_digest
    ls = np.array([s.l for s in basis.shells])
    pure = np.array([s.pure for s in basis.shells])
    npr = np.array([s.nprim for s in basis.shells], dtype=np.float64)
    size = basis.sizes.astype(np.float64)
    s1s, s2s = [], []
    for s1 in range(ns):
        for s2 in range(s1 + 1):
            if Q[s1, s2] > 0.0:
                s1s.append(s1)
                s2s.append(s2)
    s1s = np.array(s1s)
    s2s = np.array(s2s)
    qp = Q[s1s, s2s]
    f64 = f32 = nq = n32 = 0.0
    cache = {}
    for p in range(len(s1s)):
        a, b = s1s[p], s2s[p]
        k = np.arange(p + 1)            # kets (s3, s4) <= (s1, s2) in loop order
        c, d = s1s[k], s2s[k]
        sm = np.maximum.reduce([norms[c, d], norms[a, d], norms[b, d],
                                norms[a, c], norms[b, c],
                                np.full(len(k), norms[a, b])])
        bound = sm * qp[p] * qp[k]
        keep = bound >= thresh
        if not keep.any():
            continue
        c, d, bound = c[keep], d[keep], bound[keep]
        key_ab = (ls[a], ls[b], pure[a], pure[b])
        lc, ld = ls[c], ls[d]
        # per-class flop per primitive quartet and transform
        fq = np.empty(len(c))
        cls = lc * 8 + ld + 64 * pure[c] + 128 * pure[d]
        for u in np.unique(cls):
            sel = cls == u
            i0 = np.flatnonzero(sel)[0]
            kk = key_ab + (int(lc[i0]), int(ld[i0]), int(pure[c][i0]),
                           int(pure[d][i0]))
            if kk not in cache:
                cache[kk] = (flop_prim(kk[0], kk[1], kk[4], kk[5]),
                             _sph_flops([kk[0], kk[1], kk[4], kk[5]],
                                        [kk[2], kk[3], kk[6], kk[7]]))
            fp, fs = cache[kk]
            fq[sel] = fp * npr[a] * npr[b] * npr[c[sel]] * npr[d[sel]] + fs
        fq += 12.0 * nd * size[a] * size[b] * size[c] * size[d]
        if fp32_cut > 0:
            lo = bound < fp32_cut
            f32 += fq[lo].sum()
            n32 += lo.sum()
            f64 += fq[~lo].sum()
        else:
            f64 += fq.sum()
        nq += len(c)
    return dict(f64=f64, f32=f32, quartets=nq, q32=n32)
