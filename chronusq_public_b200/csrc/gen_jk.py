"""Generates cqf_gen_jk.cuh: straight-line McMurchie-Davidson kernels for the
closed-shell (real, symmetric density) J/K build, one per shell-quartet class.

Run by chronusq_public_b200/build.py before nvcc; the output goes to
csrc/gen/ (not tracked).  For each class the generator

* picks the orientation (which pair class is the block's bra) that keeps the
  Hermite intermediate G[cd][tuv] smallest,
* splits the ket Cartesian components c into chunks so that the live set
  (integral block + G + R) stays inside the register file -- separately for
  each precision: an FP32 kernel keeps its integrals, Hermite intermediates
  and digestion products in FP32 (half the registers of FP64), so its chunks
  are larger,
* emits E coefficients, Boys/R recursion, the G and integral contractions as
  scalar code with Hermite coefficients constant-folded (E^{00}_0 = 1,
  E^{ij}_t = 0 for t > i + j),
* emits the digestion of each density: J_ab (warp-reduced over the block's
  kets, which share the bra pair), J_cd, and the four exchange blocks
  (K_ac, K_bd, K_ad, K_bc) stored transposed, in the bra function's column
  (a warp's atomics then land in one column: the bra is warp-uniform); with a
  symmetric density and the final 1/2 (A + A^T) these equal the reference's
  updates
  (include/particleintegrals/contract/direct.hpp:1858-1918).  Products are
  formed in the kernel's precision; every update is accumulated with an FP64
  atomic.
"""
import itertools
import os
import sys

LMAX_FAST = 2  # classes with every l <= 2 get generated kernels


def ncart(l):
    return (l + 1) * (l + 2) // 2


def carts(l):
    out = []
    for i in range(l + 1):
        for j in range(i + 1):
            out.append((l - i, i - j, j))
    return out


def nherm(L):
    return (L + 1) * (L + 2) * (L + 3) // 6


def herm_list(L):
    return [(t, u, v) for n in range(L + 1) for t in range(n, -1, -1)
            for u in range(n - t, -1, -1) for v in [n - t - u]]


class E1D:
    """Symbolic 1D Hermite coefficients E^{ij}_t of one pair (axis x)."""

    def __init__(self, w, li, lj, tag, o2p, PA, PB):
        self.w = w
        self.val = {}
        self.val[(0, 0, 0)] = "1"
        for i in range(li + 1):
            for j in range(lj + 1):
                if i == 0 and j == 0:
                    continue
                up = (j == 0)
                pi, pj = (i - 1, j) if up else (i, j - 1)
                X = PA if up else PB
                for t in range(i + j + 1):
                    terms = []
                    a = self.get(pi, pj, t)
                    if a is not None:
                        terms.append(a if X is None else self._mul(X, a))
                    b = self.get(pi, pj, t - 1)
                    if b is not None:
                        terms.append(self._mul(o2p, b))
                    c = self.get(pi, pj, t + 1)
                    if c is not None:
                        terms.append(self._mul("T(%d)" % (t + 1), c) if t + 1 != 1 else c)
                    if not terms:
                        continue
                    name = "%s_%d_%d_%d" % (tag, i, j, t)
                    w.line("const T %s = %s;" % (name, " + ".join(terms)))
                    self.val[(i, j, t)] = name

    @staticmethod
    def _mul(a, b):
        if a == "1":
            return b
        if b == "1":
            return a
        return "%s * %s" % (a, b)

    def get(self, i, j, t):
        if t < 0 or t > i + j or i < 0 or j < 0:
            return None
        return self.val.get((i, j, t))


class W:
    def __init__(self):
        self.lines = []
        self.ind = 0

    def line(self, s):
        self.lines.append("  " * self.ind + s)

    def open(self, s):
        self.line(s)
        self.ind += 1

    def close(self, s="}"):
        self.ind -= 1
        self.line(s)


def orientation(c1, c2):
    """(bra, ket) pair classes minimising NCD * H(lab)."""
    (a1, b1), (a2, b2) = c1, c2
    g12 = ncart(a2) * ncart(b2) * nherm(a1 + b1)
    g21 = ncart(a1) * ncart(b1) * nherm(a2 + b2)
    return (c1, c2) if g12 <= g21 else (c2, c1)


def chunk_size(la, lb, lc, ld, prec):
    """ket component pairs (flattened cd index) per chunk, so that the live
    set (integral chunk + G chunk + R, in 4-byte register units: 2 per FP64
    value, 1 per FP32 value) stays under the budget."""
    nab = ncart(la) * ncart(lb)
    ncd = ncart(lc) * ncart(ld)
    hab = nherm(la + lb)
    hl = nherm(la + lb + lc + ld)
    w = 2 if prec == 64 else 1
    best = 1
    for cs in range(1, ncd + 1):
        live = w * (nab * cs + cs * hab + hl)
        if live <= 176:
            best = cs
    return best


def use_mirror(la, lb, lc, ld, nchunk, prec):
    """Ket-outer primitive loops (emit_eri_mirror) for single-chunk classes
    whose live set -- integral block, bra-side Hermite accumulators
    G'[ab][tau nu phi] and R, in 4-byte register units -- fits the budget."""
    if nchunk != 1:
        return False
    nab = ncart(la) * ncart(lb)
    ncd = ncart(lc) * ncart(ld)
    w = 2 if prec == 64 else 1
    live = w * (nab * ncd + nab * nherm(lc + ld) + nherm(la + lb + lc + ld))
    return live <= 176


def emit_R(w, L, hall):
    """R^{(n)}_tuv recursion for total order L as straight-line code; returns
    the name of each R^{(n)}_tuv."""
    R = {}
    w.line("const T m2a = T(-2) * alpha;")
    pw = ["T(1)"]
    for n in range(1, L + 1):
        w.line("const T a%d = %s;" % (n, "m2a" if n == 1 else "a%d * m2a" % (n - 1)))
        pw.append("a%d" % n)
    for n in range(L, -1, -1):
        w.line("const T r%d_0_0_0 = %s;" % (n, "F[0]" if n == 0 else "%s * F[%d]" % (pw[n], n)))
        R[(n, 0, 0, 0)] = "r%d_0_0_0" % n
    for tot in range(1, L + 1):
        for n in range(L - tot, -1, -1):
            for (t, u, v) in [h for h in hall if sum(h) == tot]:
                if t > 0:
                    e = "X * %s" % R[(n + 1, t - 1, u, v)]
                    if t > 1:
                        e += " + T(%d) * %s" % (t - 1, R[(n + 1, t - 2, u, v)])
                elif u > 0:
                    e = "Y * %s" % R[(n + 1, t, u - 1, v)]
                    if u > 1:
                        e += " + T(%d) * %s" % (u - 1, R[(n + 1, t, u - 2, v)])
                else:
                    e = "Z * %s" % R[(n + 1, t, u, v - 1)]
                    if v > 1:
                        e += " + T(%d) * %s" % (v - 1, R[(n + 1, t, u, v - 2)])
                nm = "r%d_%d_%d_%d" % (n, t, u, v)
                w.line("const T %s = %s;" % (nm, e))
                R[(n, t, u, v)] = nm
    return R


def emit_eri_mirror(w, la, lb, lc, ld, CS, prec):
    """eri() body with the ket primitives (per lane) in the outer loop and the
    bra primitives (shared by the warp) in the inner one:
        G'[ab][tnp] = sum_ip pref sum_tuv E^ab_tuv R_{t+tau,u+nu,v+phi}
        I[ab][cd]  += sum_tnp (-1)^(tau+nu+phi) E^cd_tnp G'[ab][tnp]
    (the same integrals as the bra-outer order; each lane loads its ket
    primitive data and builds its ket E coefficients once per ket primitive
    instead of once per primitive pair)."""
    A, B, Cc, Dd = carts(la), carts(lb), carts(lc), carts(ld)
    NA, NB, ND = len(A), len(B), len(Dd)
    NCD = len(Cc) * ND
    lab, lcd = la + lb, lc + ld
    L = lab + lcd
    hcd = herm_list(lcd)
    hall = herm_list(L)
    axes = "xyz"
    w.line("#pragma unroll")
    w.line("for (int i = 0; i < %d; i++) I[i] = 0.0;" % (NA * NB * CS))
    w.line("const T PI52x2 = T(34.986836655249725693);")
    w.line("const double qbMax = eps > 0.0 ? __ldg(ppQ + P.pp_off) : 0.0;")
    w.line("#pragma unroll 1")
    w.open("for (int iq = 0; iq < Q.npp; iq++) {")
    w.line("const double qk = eps > 0.0 ? kq.Qp(iq) : 0.0;")
    w.line("if (qk * qbMax < eps) break;")
    w.line("const T q = T(kq.p(iq)), Kcd = T(kq.Kp(iq)), o2q = T(kq.o2p(iq));")
    w.line("const T Qx = T(kq.P(iq, 0)), Qy = T(kq.P(iq, 1)), Qz = T(kq.P(iq, 2));")
    if lcd > 0:
        for x in range(3):
            w.line("const T QC%s = T(kq.PA(iq, %d)), QD%s = T(kq.PB(iq, %d));"
                   % (axes[x], x, axes[x], x))
    ek = [E1D(w, lc, ld, "ec" + axes[x], "o2q", "QC" + axes[x], "QD" + axes[x])
          for x in range(3)] if lcd > 0 else None
    for ia in range(NA):
        for ib in range(NB):
            for (t, u, v) in hcd:
                w.line("T h_%d_%d_%d_%d_%d = T(0);" % (ia, ib, t, u, v))
    w.line("#pragma unroll 1")
    w.open("for (int ip = 0; ip < P.npp; ip++) {")
    w.line("if (eps > 0.0 && __ldg(ppQ + P.pp_off + ip) * qk < eps) break;")
    w.line("const auto& pa = pp[P.pp_off + ip];")
    w.line("const T p = T(pa.p), Kab = T(pa.Kp), o2p = T(pa.o2p);")
    w.line("const T X = T(pa.P[0]) - Qx, Y = T(pa.P[1]) - Qy, Z = T(pa.P[2]) - Qz;")
    if lab > 0:
        for x in range(3):
            w.line("const T PA%s = T(pa.PA[%d]), PB%s = T(pa.PB[%d]);" % (axes[x], x, axes[x], x))
    emit_boys(w, L, prec)
    w.line("const T pref = PI52x2 * rpq * Kab * Kcd;")
    R = emit_R(w, L, hall)
    eb = [E1D(w, la, lb, "ea" + axes[x], "o2p", "PA" + axes[x], "PB" + axes[x])
          for x in range(3)] if lab > 0 else None
    for ia, (ax, ay, az) in enumerate(A):
        for ib, (bx, by, bz) in enumerate(B):
            names = []
            for t in range(ax + bx + 1):
                for u in range(ay + by + 1):
                    for v in range(az + bz + 1):
                        if lab > 0:
                            fx, fy, fz = eb[0].get(ax, bx, t), eb[1].get(ay, by, u), eb[2].get(az, bz, v)
                            if fx is None or fy is None or fz is None:
                                continue
                            fac = [f for f in (fx, fy, fz) if f != "1"]
                        else:
                            fac = []
                        if fac:
                            nm = "v_%d_%d_%d_%d_%d" % (ia, ib, t, u, v)
                            w.line("const T %s = %s;" % (nm, " * ".join(fac)))
                            names.append((t, u, v, nm))
                        else:
                            names.append((t, u, v, None))
            for (tk, uk, vk) in hcd:
                sm = " + ".join(("%s * " % nm if nm else "") + R[(0, t + tk, u + uk, v + vk)]
                                for (t, u, v, nm) in names)
                w.line("h_%d_%d_%d_%d_%d += pref * (%s);" % (ia, ib, tk, uk, vk, sm))
    w.close("}")  # ip
    for k in range(NCD):
        c, di = divmod(k, ND)
        cx, cy, cz = Cc[c]
        dx, dy, dz = Dd[di]
        terms = []
        for ta in range(cx + dx + 1):
            for nu in range(cy + dy + 1):
                for ph in range(cz + dz + 1):
                    if lcd > 0:
                        ex, ey, ez = ek[0].get(cx, dx, ta), ek[1].get(cy, dy, nu), ek[2].get(cz, dz, ph)
                        if ex is None or ey is None or ez is None:
                            continue
                        fac = [f for f in (ex, ey, ez) if f != "1"]
                    else:
                        fac = []
                    terms.append((ta, nu, ph, fac, (ta + nu + ph) & 1))
        for ia in range(NA):
            for ib in range(NB):
                sm = " + ".join(("-" if sg else "") + " * ".join(fac + ["h_%d_%d_%d_%d_%d" % (ia, ib, ta, nu, ph)])
                                for (ta, nu, ph, fac, sg) in terms)
                w.line("I[%d] += %s;" % ((ia * NB + ib) * CS + k, sm))
    w.close("}")  # iq
    w.close("}")  # eri


def emit_boys(w, L, prec):
    """1/sqrt(p + q), alpha, T and F_0..F_L in the kernel's precision (the
    FP32 kernels evaluate T >= 36 in FP64, boys_f32)."""
    w.line("const T pq = p + q;")
    w.line("const T rpq = %s;" % ("rsqrt(pq)" if prec == 64 else "rsqrtf(pq)"))
    w.line("const T alpha = p * q * (rpq * rpq);")
    w.line("const T Targ = alpha * (X * X + Y * Y + Z * Z);")
    w.line("T F[%d];" % (L + 1))
    w.line("boys_f%d<%d>(Targ, F, boys);  // rows of L" % (prec, L))


def gen_class(la, lb, lc, ld, prec):
    """Struct GenJK<prec>_<class>: eri() computes chunk ch (a contiguous range
    of the flattened ket component index cd) of the contracted Cartesian
    block in the struct's precision T; digest() adds that chunk's J/K
    contributions of one density (products in T, FP64 atomics)."""
    w = W()
    A, B, Cc, Dd = carts(la), carts(lb), carts(lc), carts(ld)
    NA, NB, NC, ND = len(A), len(B), len(Cc), len(Dd)
    NAB, NCD = NA * NB, NC * ND
    lab, lcd = la + lb, lc + ld
    L = lab + lcd
    CS = chunk_size(la, lb, lc, ld, prec)
    nchunk = (NCD + CS - 1) // CS
    mirror = use_mirror(la, lb, lc, ld, nchunk, prec)
    chunks = [list(range(k * CS, min(NCD, (k + 1) * CS))) for k in range(nchunk)]
    hab = herm_list(lab)
    hall = herm_list(L)
    T = "double" if prec == 64 else "float"
    name = "%d_%d%d%d%d" % (prec, la, lb, lc, ld)
    w.line("// (%s%s|%s%s), FP%d: NAB=%d NCD=%d L=%d, %d chunk(s) of <= %d cd pairs%s"
           % ("spdf"[la], "spdf"[lb], "spdf"[lc], "spdf"[ld], prec, NAB, NCD, L, nchunk, CS,
              ", ket-outer primitive loops" if mirror else ""))
    w.open("struct GenJK%s {" % name)
    w.line("using T = %s;" % T)
    w.line("static constexpr int LA = %d, LB = %d, LC = %d, LD = %d;" % (la, lb, lc, ld))
    w.line("static constexpr int NCHUNK = %d;" % nchunk)
    w.line("static constexpr int NI = %d;  // integrals per chunk" % (NAB * CS))
    # resident blocks per SM the register allocator should target: small
    # low-L classes are latency bound and gain from occupancy
    live = (2 if prec == 64 else 1) * (NAB * CS + CS * len(hab) + len(hall))
    minb = 6 if L <= 1 else (4 if live <= 96 else (2 if live <= 150 else 1))
    w.line("static constexpr int MINB = %d;" % minb)
    # ket primitive data through an accessor (KetAoS / KetSoA, cqf_jk_fast.cuh)
    # bra primitive records through PP: PrimPairDev (FP64) or its FP32 copy
    w.line("template <class KA, class PP>")
    # primitive screen (the reference's engine precision, direct.hpp:1563-1589):
    # primitive quartets with Qp_ab Qp_cd < eps are skipped; a pair's
    # primitive pairs are sorted by Qp (descending), so a loop stops at the
    # first one below the bound.  eps = 0 computes every primitive quartet.
    w.open("static __device__ __forceinline__ void eri(const PairDev& P, const PairDev& Q, "
           "const PP* __restrict__ pp, const KA& kq, const T* __restrict__ boys, "
           "const int ch, T (&I)[%d], const double* __restrict__ ppQ, const double eps) {"
           % (NAB * CS))
    if mirror:
        emit_eri_mirror(w, la, lb, lc, ld, CS, prec)
    else:
        w.line("#pragma unroll")
        w.line("for (int i = 0; i < %d; i++) I[i] = T(0);" % (NAB * CS))
        w.line("const T PI52x2 = T(34.986836655249725693);")
        w.line("const double qkMax = eps > 0.0 && Q.npp > 0 ? kq.Qp(0) : 0.0;")
        w.line("#pragma unroll 1")
        w.open("for (int ip = 0; ip < P.npp; ip++) {")
        w.line("const double qb = eps > 0.0 ? __ldg(ppQ + P.pp_off + ip) : 0.0;")
        w.line("if (qb * qkMax < eps) break;")
        w.line("const auto& pa = pp[P.pp_off + ip];")
        w.line("const T p = T(pa.p), Kab = T(pa.Kp), o2p = T(pa.o2p);")
        w.line("const T Px = T(pa.P[0]), Py = T(pa.P[1]), Pz = T(pa.P[2]);")
        axes = "xyz"
        if lab > 0:
            for x in range(3):
                w.line("const T PA%s = T(pa.PA[%d]), PB%s = T(pa.PB[%d]);" % (axes[x], x, axes[x], x))
        for k in range(CS):
            for (t, u, v) in hab:
                w.line("T g_%d_%d_%d_%d = T(0);" % (k, t, u, v))
        w.line("#pragma unroll 1")
        w.open("for (int iq = 0; iq < Q.npp; iq++) {")
        w.line("if (eps > 0.0 && qb * kq.Qp(iq) < eps) break;")
        w.line("const T q = T(kq.p(iq)), Kcd = T(kq.Kp(iq)), o2q = T(kq.o2p(iq));")
        w.line("const T X = Px - T(kq.P(iq, 0)), Y = Py - T(kq.P(iq, 1)), Z = Pz - T(kq.P(iq, 2));")
        emit_boys(w, L, prec)
        w.line("const T pref = PI52x2 * rpq * Kab * Kcd;")
        if lcd > 0:
            for x in range(3):
                w.line("const T QC%s = T(kq.PA(iq, %d)), QD%s = T(kq.PB(iq, %d));"
                       % (axes[x], x, axes[x], x))
        ek = [E1D(w, lc, ld, "ec" + axes[x], "o2q", "QC" + axes[x], "QD" + axes[x])
              for x in range(3)] if lcd > 0 else None
        R = emit_R(w, L, hall)
        if nchunk > 1:
            w.open("switch (ch) {")
        for chv, cdl in enumerate(chunks):
            if nchunk > 1:
                w.open("case %d: {" % chv)
            for k, cd in enumerate(cdl):
                c, di = divmod(cd, ND)
                cx, cy, cz = Cc[c]
                dx, dy, dz = Dd[di]
                wn = []
                for ta in range(cx + dx + 1):
                    for nu in range(cy + dy + 1):
                        for ph in range(cz + dz + 1):
                            if lcd > 0:
                                ex = ek[0].get(cx, dx, ta)
                                ey = ek[1].get(cy, dy, nu)
                                ez = ek[2].get(cz, dz, ph)
                                if ex is None or ey is None or ez is None:
                                    continue
                                fac = [f for f in (ex, ey, ez) if f != "1"]
                            else:
                                fac = []
                            sgn = -1 if (ta + nu + ph) & 1 else 1
                            nm = "w_%d_%d_%d_%d" % (k, ta, nu, ph)
                            w.line("const T %s = %s%s;" % (nm, "-" if sgn < 0 else "",
                                                            " * ".join(["pref"] + fac)))
                            wn.append((ta, nu, ph, nm))
                for (t, u, v) in hab:
                    sm = " + ".join("%s * %s" % (nm, R[(0, t + ta, u + nu, v + ph)])
                                    for (ta, nu, ph, nm) in wn)
                    w.line("g_%d_%d_%d_%d += %s;" % (k, t, u, v, sm))
            if nchunk > 1:
                w.line("break;")
                w.close("}")
        if nchunk > 1:
            w.close("}")
        w.close("}")  # iq
        eb = [E1D(w, la, lb, "ea" + axes[x], "o2p", "PA" + axes[x], "PB" + axes[x])
              for x in range(3)] if lab > 0 else None
        for ia, (ax, ay, az) in enumerate(A):
            for ib, (bx, by, bz) in enumerate(B):
                names = []
                for t in range(ax + bx + 1):
                    for u in range(ay + by + 1):
                        for v in range(az + bz + 1):
                            if lab > 0:
                                fx, fy, fz = eb[0].get(ax, bx, t), eb[1].get(ay, by, u), eb[2].get(az, bz, v)
                                if fx is None or fy is None or fz is None:
                                    continue
                                fac = [f for f in (fx, fy, fz) if f != "1"]
                            else:
                                fac = []
                            if fac:
                                nm = "v_%d_%d_%d_%d_%d" % (ia, ib, t, u, v)
                                w.line("const T %s = %s;" % (nm, " * ".join(fac)))
                                names.append((t, u, v, nm))
                            else:
                                names.append((t, u, v, None))
                for k in range(CS):
                    sm = " + ".join(("%s * " % nm if nm else "") + "g_%d_%d_%d_%d" % (k, t, u, v)
                                    for (t, u, v, nm) in names)
                    w.line("I[%d] += %s;" % ((ia * NB + ib) * CS + k, sm))
        w.close("}")  # ip
        w.close("}")  # eri
    # ---- digestion
    w.line("// J/K contributions of chunk ch for one density (symmetric X, in the")
    w.line("// kernel's precision).  The K_ac update reads X(d, b) (the other three read")
    w.line("// X in bra-row order): sKac = sK for a symmetric X, -sK for an antisymmetric")
    w.line("// one.  Every update is one FP64 atomic.")
    w.open("static __device__ __forceinline__ void digest(const T (&I)[%d], const int ch, "
           "const T* __restrict__ X, double* __restrict__ Acc, size_t nc, int cA, int cB, "
           "int cC, int cD, T sJ, T sK, T sKac, bool doJ, bool doK, T (&jab)[%d]) {"
           % (NAB * CS, NAB))
    w.line("auto ld = [&](int r, int c) { return __ldg(X + (size_t)r + (size_t)c * nc); };")
    w.line("auto add = [&](int r, int c, T v) { atomicAdd(Acc + (size_t)r + (size_t)c * nc, double(v)); };")
    if nchunk > 1:
        w.open("switch (ch) {")
    for chv, cdl in enumerate(chunks):
        if nchunk > 1:
            w.open("case %d: {" % chv)
        els = [(k,) + divmod(cd, ND) for k, cd in enumerate(cdl)]  # (k, c, d)
        cs_ = sorted(set(c for (_, c, _) in els))
        ds_ = sorted(set(d for (_, _, d) in els))

        def Iv(a, b, k):
            return "I[%d]" % ((a * NB + b) * CS + k)
        w.open("if (doJ) {")
        for (k, c, d) in els:
            w.line("const T dcd_%d = ld(cD + %d, cC + %d);" % (k, d, c))
        for a_ in range(NA):
            for b_ in range(NB):
                sm = " + ".join("%s * dcd_%d" % (Iv(a_, b_, k), k) for (k, c, d) in els)
                w.line("jab[%d] += %s;" % (a_ * NB + b_, sm))
        for a_ in range(NA):
            for b_ in range(NB):
                w.line("const T dab_%d_%d = ld(cA + %d, cB + %d);" % (a_, b_, a_, b_))
        for (k, c, d) in els:
            sm = " + ".join("%s * dab_%d_%d" % (Iv(a_, b_, k), a_, b_)
                            for a_ in range(NA) for b_ in range(NB))
            w.line("add(cC + %d, cD + %d, sJ * (%s));" % (c, d, sm))
        w.close()
        w.open("if (doK) {")
        # K_ac += sum_bd I D[d,b]
        for b_ in range(NB):
            for d in ds_:
                w.line("const T ddb_%d_%d = ld(cD + %d, cB + %d);" % (d, b_, d, b_))
        for a_ in range(NA):
            for c in cs_:
                sm = " + ".join("%s * ddb_%d_%d" % (Iv(a_, b_, k), d, b_)
                                for b_ in range(NB) for (k, cc, d) in els if cc == c)
                w.line("add(cC + %d, cA + %d, sKac * (%s));" % (c, a_, sm))
        # K_bd += sum_ac I D[a,c]
        for a_ in range(NA):
            for c in cs_:
                w.line("const T dac_%d_%d = ld(cA + %d, cC + %d);" % (a_, c, a_, c))
        for b_ in range(NB):
            for d in ds_:
                sm = " + ".join("%s * dac_%d_%d" % (Iv(a_, b_, k), a_, c)
                                for a_ in range(NA) for (k, c, dd) in els if dd == d)
                w.line("add(cD + %d, cB + %d, sK * (%s));" % (d, b_, sm))
        # K_ad += sum_bc I D[b,c]
        for b_ in range(NB):
            for c in cs_:
                w.line("const T dbc_%d_%d = ld(cB + %d, cC + %d);" % (b_, c, b_, c))
        for a_ in range(NA):
            for d in ds_:
                sm = " + ".join("%s * dbc_%d_%d" % (Iv(a_, b_, k), b_, c)
                                for b_ in range(NB) for (k, c, dd) in els if dd == d)
                w.line("add(cD + %d, cA + %d, sK * (%s));" % (d, a_, sm))
        # K_bc += sum_ad I D[a,d]
        for a_ in range(NA):
            for d in ds_:
                w.line("const T dad_%d_%d = ld(cA + %d, cD + %d);" % (a_, d, a_, d))
        for b_ in range(NB):
            for c in cs_:
                sm = " + ".join("%s * dad_%d_%d" % (Iv(a_, b_, k), a_, d)
                                for a_ in range(NA) for (k, cc, d) in els if cc == c)
                w.line("add(cC + %d, cB + %d, sK * (%s));" % (c, b_, sm))
        w.close()
        if nchunk > 1:
            w.line("break;")
            w.close("}")
    if nchunk > 1:
        w.close("}")
    w.close("}")  # digest
    w.close("};")
    return "\n".join(w.lines), name


def main(out_path):
    pclasses = [(a, b) for a in range(LMAX_FAST + 1) for b in range(a + 1)]
    parts = ["// Generated by gen_jk.py -- do not edit.",
             "#pragma once", '#include "../cqf_common.cuh"', "namespace cqf {", ""]
    table = []
    for i, c1 in enumerate(pclasses):
        for c2 in pclasses[:i + 1]:
            bra, ket = orientation(c1, c2)
            names = []
            for prec in (64, 32):
                code, name = gen_class(bra[0], bra[1], ket[0], ket[1], prec)
                parts.append(code)
                parts.append("")
                names.append(name)
            table.append((bra, ket, names))
    parts.append("// (bra la, lb, ket lc, ld) of each generated class, FP64 / FP32 structs")
    parts.append("#define CQF_GEN_JK_CLASSES(X) \\")
    parts.append(" \\\n".join("  X(%d, %d, %d, %d, GenJK%s, GenJK%s)"
                             % (b[0], b[1], k[0], k[1], n[0], n[1]) for (b, k, n) in table))
    parts.append("")
    parts.append("}  // namespace cqf")
    txt = "\n".join(parts) + "\n"
    os.makedirs(os.path.dirname(out_path), exist_ok=True)
    if not os.path.exists(out_path) or open(out_path).read() != txt:
        with open(out_path, "w") as f:
            f.write(txt)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(
        os.path.dirname(os.path.abspath(__file__)), "gen", "cqf_gen_jk.cuh"))
