// Four-component Dirac-Coulomb direct contraction on the device.
//
// Replaces GTODirectRelERIContraction::twoBodyContract -> directScaffoldLibcint
// (include/particleintegrals/contract/direct4C_libcint.hpp:138-2832) and the
// FourCompFock::formGDDirect assembly (include/fockbuilder/fourcompfock/
// impl.hpp:3752-4636).
//
// Small-component functions are the large-component ones differentiated
// (restricted kinetic balance), so the LLSS and SSSS terms need derivative
// ERIs.  A differentiated pair (m, n) acts on the electron's spin as the
// operator P_mn = dm.dn + i sigma.(dm x dn): four real operator components
// (dot, cross x, y, z) per integral.  The reference takes the 9 / 81 raw
// derivative components from libcint and writes each spin product out; here
// the components come from McMurchie-Davidson over the pair's Hermite tables
// raised by one on each centre,
//     d/dx [x^i e^{-a x^2}] = i x^{i-1} e^{-a x^2} - 2a x^{i+1} e^{-a x^2},
// and the digestion is the Pauli algebra of P:
//   Coulomb   J^a(12) += P^a(12|34) rho(43), rho = (Re D^S, -Im D^x, -Im D^y, -Im D^z)
//   LS exchange  K(3,2) -= D(4,1) P_12                          (LLSS)
//   SS exchange  K(1,4) -= P_12 D(2,3) P_34                     (SSSS)
// with the reference's quartet sets, screens and degeneracy factors.
//
// Layout: densities and accumulators live in the Cartesian AO basis (exact
// transforms before and after, as on the 1C path); Coulomb accumulators are
// real, exchange accumulators complex.  One thread per unique shell quartet
// loops over the ket's Cartesian components; for each it sums the primitive
// quartets into the operator components of every bra component pair and
// digests them with FP64 atomics.  Hermitian outputs are completed from the
// accumulated half at the back transform (the reference's "upper =
// conj(lower)" after Hermitian digestion).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cqf_deriv.cuh"
#include "cqf_eri.cuh"
#include "cqf_internal.hpp"

namespace cqf {
namespace {

#define CQF_RCUDA(call)                                                                    \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(e_ == cudaErrorMemoryAllocation ? CQF_ENOMEM : CQF_ECUDA,                \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                     \
  } while (0)

#define CQF_RTRY(expr)           \
  do {                           \
    cqf_status s_ = (expr);      \
    if (s_ != CQF_OK) return s_; \
  } while (0)

unsigned rgrid(size_t n, int b) { return (unsigned)((n + b - 1) / b); }

// max of the six shell-block norms of a quartet in the reference's roles
// (direct4C_libcint.hpp:602-620, :940-948)
__device__ __forceinline__ double sh_max(const double* __restrict__ n, int s1, int s2, int s3,
                                         int s4, int ns) {
  auto B = [&](int a, int b) { return __ldg(n + a + (size_t)b * ns); };
  return fmax(fmax(fmax(B(s1, s2), B(s1, s3)), fmax(B(s2, s3), B(s1, s4))),
              fmax(B(s2, s4), B(s3, s4)));
}

// ------------------------------------------------------------ spin algebra
struct __align__(16) Q4 {  // s + v . sigma, complex components
  double2 s, x, y, z;
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 ctimes_i(double2 a) { return make_double2(-a.y, a.x); }

// (p.s + p.v sigma)(q.s + q.v sigma) = p.s q.s + p.v.q.v
//   + (p.s q.v + q.s p.v + i p.v x q.v) . sigma
__device__ __forceinline__ Q4 qmul(const Q4& p, const Q4& q) {
  Q4 r;
  r.s = cadd(cadd(cmul(p.s, q.s), cmul(p.x, q.x)), cadd(cmul(p.y, q.y), cmul(p.z, q.z)));
  r.x = cadd(cadd(cmul(p.s, q.x), cmul(q.s, p.x)),
             ctimes_i(csub(cmul(p.y, q.z), cmul(p.z, q.y))));
  r.y = cadd(cadd(cmul(p.s, q.y), cmul(q.s, p.y)),
             ctimes_i(csub(cmul(p.z, q.x), cmul(p.x, q.z))));
  r.z = cadd(cadd(cmul(p.s, q.z), cmul(q.s, p.z)),
             ctimes_i(csub(cmul(p.x, q.y), cmul(p.y, q.x))));
  return r;
}

// p (m0 + i w . sigma) for real m0 and w: m0 p.s + i p.v.w, and
// i p.s w + m0 p.v - p.v x w (the general product with the zero parts of the
// right factor left out)
__device__ __forceinline__ Q4 qmul_ri(const Q4& p, double m0, double w1, double w2,
                                      double w3) {
  const double2 pw = make_double2(p.x.x * w1 + p.y.x * w2 + p.z.x * w3,
                                  p.x.y * w1 + p.y.y * w2 + p.z.y * w3);
  Q4 r;
  r.s = make_double2(m0 * p.s.x - pw.y, m0 * p.s.y + pw.x);
  // i p.s w_k = (-p.s.y w_k, p.s.x w_k)
  r.x = make_double2(-p.s.y * w1 + m0 * p.x.x - (p.y.x * w3 - p.z.x * w2),
                     p.s.x * w1 + m0 * p.x.y - (p.y.y * w3 - p.z.y * w2));
  r.y = make_double2(-p.s.y * w2 + m0 * p.y.x - (p.z.x * w1 - p.x.x * w3),
                     p.s.x * w2 + m0 * p.y.y - (p.z.y * w1 - p.x.y * w3));
  r.z = make_double2(-p.s.y * w3 + m0 * p.z.x - (p.x.x * w2 - p.y.x * w1),
                     p.s.x * w3 + m0 * p.z.y - (p.x.y * w2 - p.y.y * w1));
  return r;
}

// t sigma_k (k = 1, 2, 3): sigma_j sigma_k = delta_jk + i eps_jkl sigma_l, so
// t sigma_x = (t.x, t.s, i t.z, -i t.y), t sigma_y = (t.y, -i t.z, t.s, i t.x),
// t sigma_z = (t.z, i t.y, -i t.x, t.s)
__device__ __forceinline__ Q4 qsig(const Q4& t, int k) {
  auto mi = [](double2 a) { return make_double2(a.y, -a.x); };  // -i a
  if (k == 1) return Q4{t.x, t.s, ctimes_i(t.z), mi(t.y)};
  if (k == 2) return Q4{t.y, mi(t.z), t.s, ctimes_i(t.x)};
  return Q4{t.z, ctimes_i(t.y), mi(t.x), t.s};
}

__device__ __forceinline__ double2 ldz(const double* X, size_t e) {
  return __ldg(reinterpret_cast<const double2*>(X) + e);
}
__device__ __forceinline__ void addz(double* A, size_t e, double2 v, double w) {
  atomicAdd(A + 2 * e, v.x * w);
  atomicAdd(A + 2 * e + 1, v.y * w);
}

struct RelLaunch {
  const PairDev* pairs;
  const PrimPairDev* pp;
  const ShellDev* shells;
  const double* prim;
  const double* boys;
  const float* boys32;
  const float2* pairRange;  // per pair: FP32 range data (fp32_range_ok)
  int mixed;      // 1: quartets with bound < cut run in FP32 (second launch)
  double cut;
  int braBeg, nBra, ketBeg, nKet, same;
  int screen;
  double thresh;
  const double* norms;  // max shell-block norms of the screening matrices
  const double* qLL;
  const double* qSS;
  int nShell, ncart, exchange;
  const double* Xll;     // Cartesian complex X[CLLMS]
  const double* Xss[4];  // Cartesian complex X[CSSM*]
  const double* Xk[4];   // exchange densities: X[XLSM*] (LLSS) / X[XSSM*] (SSSS)
  double* Jll;           // real
  double* Jss[4];        // real
  double* K[4];          // complex
  int shardIdx, shardCnt;  // bra pairs p with p % shardCnt == shardIdx only
  int skipSingle;          // single-primitive quartets: rel_gemm / rel_llss_single_kernel's
  int contracted;          // some bra or ket pair has more than one primitive pair
  int nsm;                 // multiprocessors of the device
  unsigned long long* counters;
};

constexpr int REL_THREADS = 64;

// Digestion of the operator components m of one bra component pair (a, b)
// against ket component pair (c, d) = (gC, gD) (Cartesian AO indices): the
// update formulas of the reference with the Pauli algebra of P.  jcol gets
// the caller's per-column Coulomb sum (J_LL(C,D) for LLSS, J_SS(C,D) for SSSS).
struct RelCol {
  int gC, gD;
  bool dAB, dCD, samePQ;
  double s34d, w12, wx;
  double rhoLL;    // LLSS: Re X_CLL(D, C)
  double rvDC[4];  // SSSS: (Re S, -Im X, -Im Y, -Im Z) of X_CSS(D, C)
};

template <int TYPE>
__device__ __forceinline__ void rel_digest(const RelLaunch& a, const PairDev& P, const RelCol& col,
                                           int ai, int bi, const double* m, double* jcol) {
  const size_t nc = a.ncart;
  auto ix = [nc](int r, int c) -> size_t { return (size_t)r + (size_t)c * nc; };
  const int gC = col.gC, gD = col.gD;
  const bool dAB = col.dAB, dCD = col.dCD, samePQ = col.samePQ;
  const double s34d = col.s34d, w12 = col.w12, wx = col.wx, rhoLL = col.rhoLL;
  const double* rvDC = col.rvDC;
  const int gA = P.cA + ai, gB = P.cB + bi;
  if (TYPE == 1) {
    // Coulomb SS(1,2) from the LL density (:1145-1190)
    const double wj = w12 * s34d * rhoLL;
    if (wj != 0.0)
#pragma unroll
      for (int op = 0; op < 4; op++) atomicAdd(a.Jss[op] + ix(gA, gB), wj * m[op]);
    // Coulomb LL(3,4) from the SS density
    const size_t eBA = ix(gB, gA);
    jcol[0] += m[0] * __ldg(a.Xss[0] + 2 * eBA) - m[1] * __ldg(a.Xss[1] + 2 * eBA + 1) -
               m[2] * __ldg(a.Xss[2] + 2 * eBA + 1) - m[3] * __ldg(a.Xss[3] + 2 * eBA + 1);
    if (!a.exchange) return;
    // exchange LS: K(t1, t2) -= D(d1, d2) P (:1200-1299)
    auto ls = [&](int t1, int t2, int d1, int d2, double flip) {
      const size_t e = ix(d1, d2);
      Q4 dq{ldz(a.Xk[0], e), ldz(a.Xk[1], e), ldz(a.Xk[2], e), ldz(a.Xk[3], e)};
      // dq (m0 + i flip m.sigma)
      const Q4 r = qmul_ri(dq, m[0], flip * m[1], flip * m[2], flip * m[3]);
      const size_t t = ix(t1, t2);
      addz(a.K[0], t, r.s, -1.0);
      addz(a.K[1], t, r.x, -1.0);
      addz(a.K[2], t, r.y, -1.0);
      addz(a.K[3], t, r.z, -1.0);
    };
    ls(gC, gB, gD, gA, 1.0);
    if (!dAB) ls(gC, gA, gD, gB, -1.0);
    if (!dCD) {
      ls(gD, gB, gC, gA, 1.0);
      if (!dAB) ls(gD, gA, gC, gB, -1.0);
    }
  } else {
    // m[a * 4 + b]; Coulomb SS(1,2) from D(4,3), and SS(3,4) from
    // D(2,1) when the bra and ket pairs differ (:2342-2380)
#pragma unroll
    for (int op = 0; op < 4; op++) {
      const double v = m[op * 4 + 0] * rvDC[0] + m[op * 4 + 1] * rvDC[1] +
                       m[op * 4 + 2] * rvDC[2] + m[op * 4 + 3] * rvDC[3];
      if (v != 0.0) atomicAdd(a.Jss[op] + ix(gA, gB), w12 * s34d * v);
    }
    if (!samePQ) {
      const size_t eBA = ix(gB, gA);
      const double rvBA[4] = {__ldg(a.Xss[0] + 2 * eBA), -__ldg(a.Xss[1] + 2 * eBA + 1),
                              -__ldg(a.Xss[2] + 2 * eBA + 1),
                              -__ldg(a.Xss[3] + 2 * eBA + 1)};
#pragma unroll
      for (int b = 0; b < 4; b++)
        jcol[b] += m[0 * 4 + b] * rvBA[0] + m[1 * 4 + b] * rvBA[1] +
                   m[2 * 4 + b] * rvBA[2] + m[3 * 4 + b] * rvBA[3];
    }
    if (!a.exchange) return;
    // exchange SS: K(t1, t2) -= P_12 D(d1, d2) P_34 with the bra / ket
    // orientation signs f1, f2 (:2381-2445); the Hermitian-conjugate
    // images come from the completion in the back transform
    auto ex = [&](int t1, int t2, int d1, int d2, double f1, double f2) {
      const size_t e = ix(d1, d2);
      const Q4 dq{ldz(a.Xk[0], e), ldz(a.Xk[1], e), ldz(a.Xk[2], e), ldz(a.Xk[3], e)};
      Q4 r{make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
#pragma unroll 1
      for (int b = 0; b < 4; b++) {
        // left operator sum_a c_ab sigma_a, c_ab = m_ab (i f1)^[a>0] (i f2)^[b>0]
        double2 cs = make_double2(m[0 * 4 + b], 0.0);
        double2 cx = make_double2(0.0, f1 * m[1 * 4 + b]);
        double2 cy = make_double2(0.0, f1 * m[2 * 4 + b]);
        double2 cz = make_double2(0.0, f1 * m[3 * 4 + b]);
        if (b > 0) {
          cs = make_double2(-f2 * cs.y, f2 * cs.x);
          cx = make_double2(-f2 * cx.y, f2 * cx.x);
          cy = make_double2(-f2 * cy.y, f2 * cy.x);
          cz = make_double2(-f2 * cz.y, f2 * cz.x);
        }
        const Q4 Lq{cs, cx, cy, cz};
        const Q4 ld = qmul(Lq, dq);
        const Q4 t = b == 0 ? ld : qsig(ld, b);  // (Lq dq) sigma_b
        r.s = cadd(r.s, t.s);
        r.x = cadd(r.x, t.x);
        r.y = cadd(r.y, t.y);
        r.z = cadd(r.z, t.z);
      }
      const size_t t = ix(t1, t2);
      addz(a.K[0], t, r.s, -wx);
      addz(a.K[1], t, r.x, -wx);
      addz(a.K[2], t, r.y, -wx);
      addz(a.K[3], t, r.z, -wx);
    };
    ex(gA, gD, gB, gC, 1.0, 1.0);
    if (!dCD) ex(gA, gC, gB, gD, 1.0, -1.0);
    if (!dAB) {
      ex(gB, gD, gA, gC, -1.0, 1.0);
      if (!dCD) ex(gB, gC, gA, gD, -1.0, -1.0);
    }
  }
}

// TYPE 1: LLSS (bra = SS pair, differentiated; ket = LL pair), all
// (bra, ket) combinations (direct4C_libcint.hpp:907-929).
// TYPE 2: SSSS, unique quartets of pairs (:2018-2047).
// The ket's Cartesian component pairs (c, d) of a quartet are split over
// nsplit threads (grid y = ket tiles x nsplit): the heavy classes with few
// quartets (f shells) still fill the GPU.
// T: primitive arithmetic (double; float for the small-bound quartets of a
// mixed launch); operator components, digestion and accumulation in FP64.
template <int LM, int TYPE, typename T>
__global__ void __launch_bounds__(REL_THREADS)
    rel_kernel(const RelLaunch a, int la, int lb, int lc, int ld, int nsplit) {
  constexpr bool IS32 = sizeof(T) == 4;
  const int ib = blockIdx.x;
  if (!in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) return;  // another shard's bra
  const int split = blockIdx.y % nsplit;
  const int jk = (blockIdx.y / nsplit) * REL_THREADS + threadIdx.x;
  const int ns = a.nShell;
  bool visited = jk < a.nKet && !(TYPE == 2 && a.same && jk > ib);
  const PairDev P = a.pairs[a.braBeg + ib];
  PairDev Q = P;
  bool work = false, mine = false;
  if (visited) {
    Q = a.pairs[a.ketBeg + jk];
    if (a.skipSingle && P.npp == 1 && Q.npp == 1) visited = false;  // rel_gemm_kernel's
  }
  if (visited) {
    int s1, s2, s3, s4;
    double q12, q34;
    if (TYPE == 1) {
      s1 = P.s1; s2 = P.s2; s3 = Q.s1; s4 = Q.s2;
      q12 = __ldg(a.qSS + s1 + (size_t)s2 * ns);
      q34 = __ldg(a.qLL + s3 + (size_t)s4 * ns);
    } else {
      const bool pRef = P.lex >= Q.lex;
      const PairDev& R12 = pRef ? P : Q;
      const PairDev& R34 = pRef ? Q : P;
      s1 = R12.s1; s2 = R12.s2; s3 = R34.s1; s4 = R34.s2;
      q12 = __ldg(a.qSS + s1 + (size_t)s2 * ns);
      q34 = __ldg(a.qSS + s3 + (size_t)s4 * ns);
    }
    // shMax * Q12 * Q34 < thresh (:947-948, :2059-2061)
    const double bound = sh_max(a.norms, s1, s2, s3, s4, ns) * q12 * q34;
    work = !a.screen || bound >= a.thresh;
    const bool lo = a.mixed && bound < a.cut &&
                    fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib),
                                  __ldg(a.pairRange + a.ketBeg + jk),
                                  la + lb + lc + ld + 2 + 2 * (TYPE == 2), 1, TYPE == 2);
    mine = work && (IS32 ? lo : !lo);
  }
  if (split == 0) {
    const unsigned mask = __activemask();
    const unsigned bv = __ballot_sync(mask, visited), bw = __ballot_sync(mask, work);
    const unsigned bm = __ballot_sync(mask, mine);
    if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) {
      if (!IS32 && bv) atomicAdd(a.counters + 0, (unsigned long long)__popc(bv));
      if (!IS32 && (bv & ~bw)) atomicAdd(a.counters + 1, (unsigned long long)__popc(bv & ~bw));
      if (bm) atomicAdd(a.counters + (IS32 ? 2 : 3), (unsigned long long)__popc(bm));
    }
  }

  constexpr int NB = (TYPE == 2) ? 4 : 1;  // ket operator components
  constexpr int NC = 4 * NB;               // operator components per integral
  constexpr int NCL = ncart(LM);
  constexpr int E1 = (LM + 2) * (LM + 2) * (2 * LM + 3);
  constexpr int HB = nherm(2 * LM + 2);
  constexpr int HL = nherm(4 * LM + 2 + 2 * (TYPE == 2));
  constexpr int FL = 2 * LM + 3;
  const int na = ncart(la), nb = ncart(lb), ncc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb;
  const ShellDev SA = a.shells[P.shA], SB = a.shells[P.shB];
  if (!mine) return;
  const T* boysT = reinterpret_cast<const T*>(IS32 ? (const void*)a.boys32 : (const void*)a.boys);

  const int dK = (TYPE == 2) ? 1 : 0;
  const int Lb = la + lb + 2, Lk = lc + ld + 2 * dK, L = Lb + Lk;
  const ShellDev SC = a.shells[Q.shA], SD = a.shells[Q.shB];
  const bool dAB = P.shA == P.shB, dCD = Q.shA == Q.shB, samePQ = P.lex == Q.lex;
  const double s12d = dAB ? 1.0 : 2.0, s34d = dCD ? 1.0 : 2.0;
  // the back transform adds the transpose (Hermitian completion): a
  // contribution on a pair's own diagonal block is counted twice there
  const double w12 = dAB ? 0.5 : 1.0, w34 = dCD ? 0.5 : 1.0;
  const bool single = P.npp == 1 && Q.npp == 1;  // digest without accumulating
  const size_t nc = a.ncart;
  auto ix = [nc](int r, int c) -> size_t { return (size_t)r + (size_t)c * nc; };

  T Ea[3][E1], Ec[3][E1];
  T G[NB][HB];
  T Rv[HL];
  T F[4 * LM + 5];
  double acc[NCL * NCL * NC];
  T fa[3][4][FL], fc[3][4][FL];
  int nfa[3][4], nfc[3][4];

#pragma unroll 1
  for (int cd = split; cd < ncc * nd; cd += nsplit) {
    {
      const int c = cd / nd, d = cd % nd;
      const int ci[3] = {cart_lx(lc, c), cart_ly(lc, c), cart_lz(lc, c)};
      const int di[3] = {cart_lx(ld, d), cart_ly(ld, d), cart_lz(ld, d)};
      const int gC = Q.cA + c, gD = Q.cB + d;
      // per-column Coulomb accumulators (LLSS: J_LL(C,D); SSSS: J_SS(C,D))
      double jcol[4] = {0.0, 0.0, 0.0, 0.0};
      double rhoLL = 0.0;
      double rvDC[4] = {0.0, 0.0, 0.0, 0.0};
      if (TYPE == 1) {
        rhoLL = __ldg(a.Xll + 2 * ix(gD, gC));
      } else {
        const size_t eDC = ix(gD, gC);
        rvDC[0] = __ldg(a.Xss[0] + 2 * eDC);
        rvDC[1] = -__ldg(a.Xss[1] + 2 * eDC + 1);
        rvDC[2] = -__ldg(a.Xss[2] + 2 * eDC + 1);
        rvDC[3] = -__ldg(a.Xss[3] + 2 * eDC + 1);
      }

      const RelCol col{gC, gD, dAB, dCD, samePQ, s34d, w12, samePQ ? 0.5 : 1.0, rhoLL,
                       {rvDC[0], rvDC[1], rvDC[2], rvDC[3]}};

      if (!single)
#pragma unroll 1
        for (int k = 0; k < nab * NC; k++) acc[k] = 0.0;
#pragma unroll 1
      for (int ip = 0; ip < P.npp; ip++) {
        const PrimPairDev& A = a.pp[P.pp_off + ip];
        double ea, eb;
        pair_exps(SA, SB, a.prim, A, ea, eb);
#pragma unroll 1
        for (int x = 0; x < 3; x++)
          hermite_E_rt<T, LM + 1>(la + 1, lb + 1, T(A.o2p), T(A.PA[x]), T(A.PB[x]), Ea[x]);
        const T p = T(A.p);
#pragma unroll 1
        for (int b = 0; b < NB; b++)
#pragma unroll 1
          for (int h = 0; h < nherm(Lb); h++) G[b][h] = T(0);
#pragma unroll 1
        for (int iq = 0; iq < Q.npp; iq++) {
          const PrimPairDev& B = a.pp[Q.pp_off + iq];
          double ec, ed;
          pair_exps(SC, SD, a.prim, B, ec, ed);
          const T q = T(B.p);
#pragma unroll 1
          for (int x = 0; x < 3; x++)
            hermite_E_rt<T, LM + 1>(lc + dK, ld + dK, T(B.o2p), T(B.PA[x]), T(B.PB[x]), Ec[x]);
          const T X = T(A.P[0] - B.P[0]), Y = T(A.P[1] - B.P[1]), Z = T(A.P[2] - B.P[2]);
          const T pq = p + q, alpha = p * q / pq;
          const T Targ = alpha * (X * X + Y * Y + Z * Z);
          const T pref = T(PI52X2) / sqrt(pq) * T(A.Kp) * T(B.Kp);
          boys_rt<T>(L, Targ, F, boysT);
          hermite_R_rt<T>(L, alpha, X, Y, Z, F, Rv);
          const int ntk = (TYPE == 2) ? 4 : 1;
#pragma unroll 1
          for (int x = 0; x < 3; x++)
#pragma unroll 1
            for (int ty = 0; ty < ntk; ty++) {
              nfc[x][ty] = axis_factor<T>(Ec[x], ld + dK, lc + ld + 2 * dK + 1, ci[x], di[x], ty,
                                          T(2.0 * ec), T(2.0 * ed), fc[x][ty]);
#pragma unroll 1
              for (int t = 1; t < nfc[x][ty]; t += 2) fc[x][ty][t] = -fc[x][ty][t];
            }
          if (TYPE == 1) {
            ket_add<T>(G[0], pref, fc[0][0], nfc[0][0], fc[1][0], nfc[1][0], fc[2][0], nfc[2][0],
                       Lb, Rv);
          } else {
#pragma unroll 1
            for (int kk = 0; kk < 3; kk++)
#pragma unroll 1
              for (int ll = 0; ll < 3; ll++) {
                int op;
                double sg;
                op_of(kk, ll, op, sg);
                const int tx = (kk == 0) | ((ll == 0) << 1), ty = (kk == 1) | ((ll == 1) << 1),
                          tz = (kk == 2) | ((ll == 2) << 1);
                ket_add<T>(G[op < NB ? op : 0], T(sg) * pref, fc[0][tx], nfc[0][tx], fc[1][ty],
                           nfc[1][ty], fc[2][tz], nfc[2][tz], Lb, Rv);
              }
          }
        }
        // bra: the 9 derivative pairs of every component pair (a, b)
#pragma unroll 1
        for (int ai = 0; ai < na; ai++)
#pragma unroll 1
          for (int bi = 0; bi < nb; bi++) {
            const int ab = ai * nb + bi;
            const int ax[3] = {cart_lx(la, ai), cart_ly(la, ai), cart_lz(la, ai)};
            const int bx[3] = {cart_lx(lb, bi), cart_ly(lb, bi), cart_lz(lb, bi)};
#pragma unroll 1
            for (int x = 0; x < 3; x++)
#pragma unroll 1
              for (int ty = 0; ty < 4; ty++)
                nfa[x][ty] = axis_factor<T>(Ea[x], lb + 1, la + lb + 3, ax[x], bx[x], ty,
                                            T(2.0 * ea), T(2.0 * eb), fa[x][ty]);
            double mloc[NC];
            double* m = single ? mloc : acc + ab * NC;
            if (single)
#pragma unroll
              for (int k = 0; k < NC; k++) mloc[k] = 0.0;
#pragma unroll 1
            for (int mu = 0; mu < 3; mu++)
#pragma unroll 1
              for (int nu = 0; nu < 3; nu++) {
                int op;
                double sg;
                op_of(mu, nu, op, sg);
                const int tx = (mu == 0) | ((nu == 0) << 1), ty = (mu == 1) | ((nu == 1) << 1),
                          tz = (mu == 2) | ((nu == 2) << 1);
#pragma unroll 1
                for (int b = 0; b < NB; b++)
                  m[op * NB + b] += sg * double(bra_dot<T>(fa[0][tx], nfa[0][tx], fa[1][ty],
                                                           nfa[1][ty], fa[2][tz], nfa[2][tz], G[b]));
              }
            if (single) rel_digest<TYPE>(a, P, col, ai, bi, mloc, jcol);
          }
      }
      if (!single)
#pragma unroll 1
        for (int ab = 0; ab < nab; ab++) rel_digest<TYPE>(a, P, col, ab / nb, ab % nb, acc + ab * NC, jcol);

      // per-column Coulomb flush
      if (TYPE == 1) {
        if (jcol[0] != 0.0) atomicAdd(a.Jll + ix(gC, gD), w34 * s12d * jcol[0]);
      } else if (!samePQ) {
#pragma unroll
        for (int b = 0; b < 4; b++)
          if (jcol[b] != 0.0) atomicAdd(a.Jss[b] + ix(gC, gD), w34 * s12d * jcol[b]);
      }
    }
  }
}

// Hermite index (t, u, v) of compact index e (inverse of hidx).
__device__ __forceinline__ void hinv(int e, int& t, int& u, int& v) {
  int sdeg = 0;
  while (nherm(sdeg) <= e) sdeg++;
  int r = e - nherm(sdeg - 1), k = 0;
  while ((k + 1) * (k + 2) / 2 <= r) k++;
  v = r - k * (k + 1) / 2;
  u = k - v;
  t = sdeg - k;
}

constexpr int RB_THREADS = 128;

// The block kernels' table of Hermite indices: tab[h] = t | u << 8 | v << 16
// for h < n (hinv once per block instead of per use).
__device__ __forceinline__ void htab_fill(int* tab, int n) {
  for (int h = threadIdx.x; h < n; h += blockDim.x) {
    int t, u, v;
    hinv(h, t, u, v);
    tab[h] = t | (u << 8) | (v << 16);
  }
}
__device__ __forceinline__ void htab_get(const int* tab, int h, int& t, int& u, int& v) {
  const int w = tab[h];
  t = w & 255;
  u = (w >> 8) & 255;
  v = w >> 16;
}

// Division by a runtime divisor d >= 1 as a multiply-high: with
// m = ceil(2^32 / d), floor(x m / 2^32) = floor(x / d) for 0 <= x < 2^32 / d
// (the error of m is below d).  The kernels' element indices are < 2^20.
struct FastDiv {
  unsigned m;
  int d;
  __device__ __forceinline__ explicit FastDiv(int dv)
      : m(dv == 1 ? 0u : 0xFFFFFFFFu / (unsigned)dv + 1u), d(dv) {}
  __device__ __forceinline__ int div(int x) const {
    return d == 1 ? x : (int)__umulhi((unsigned)x, m);
  }
  __device__ __forceinline__ void divmod(int x, int& q, int& r) const {
    q = div(x);
    r = x - q * d;
  }
};

// Shared-memory layout of rel_block_kernel (doubles), per launch.
struct RelBlockLayout {
  int oR0, oR1, oEb, oEk, oFa, oFc, oG, oM, oF, oJ, oT, total;
};
__host__ __device__ inline RelBlockLayout rel_block_layout(int la, int lb, int lc, int ld,
                                                           int type) {
  const int dK = type == 2 ? 1 : 0;
  const int Lb = la + lb + 2, L = Lb + lc + ld + 2 * dK;
  const int NB = type == 2 ? 4 : 1;
  const int nab = ncart(la) * ncart(lb);
  const int FL = 2 * (la > lb ? la : lb) + 3;
  const int FLk = 2 * (lc > ld ? lc : ld) + 3;
  RelBlockLayout Lo;
  int o = 0;
  auto take = [&](int n) { int r = o; o += (n + 1) / 2 * 2; return r; };
  Lo.oR0 = take(nherm(L));
  Lo.oR1 = take(nherm(L));
  Lo.oEb = take(3 * (la + 2) * (lb + 2) * (la + lb + 3));
  Lo.oEk = take(3 * (lc + 1 + dK) * (ld + 1 + dK) * (lc + ld + 1 + 2 * dK));
  Lo.oFa = take(3 * (la + 1) * (lb + 1) * 4 * FL);  // per (axis, exponent pair, type)
  Lo.oFc = take(12 * FLk);
  Lo.oG = take(NB * nherm(Lb));
  Lo.oM = take(nab * 4 * NB);
  Lo.oF = take(L + 1);
  Lo.oJ = take(4);
  Lo.oT = take((nherm(L) + 1) / 2);  // packed (t, u, v) of each Hermite index, int
  Lo.total = o;
  return Lo;
}

// Block-cooperative form of rel_kernel for the heavy classes (d and f
// shells): one block per unique quartet, everything in shared memory.  Per
// primitive quartet: E tables, R (level by level, ping-pong buffers, all
// threads), the bra factors of every component pair; per ket component pair
// (c, d): its ket factors, G[b][tuv] (one entry per thread), the operator
// components of every bra component pair (one (ab, b) unit per thread) and
// their digestion (one ab per thread), the per-column Coulomb sum reduced in
// shared memory.  Same quartet set, screens and updates as rel_kernel.
template <int TYPE, typename T>
__global__ void __launch_bounds__(RB_THREADS)
    rel_block_kernel(const RelLaunch a, int la, int lb, int lc, int ld) {
  constexpr bool IS32 = sizeof(T) == 4;
  extern __shared__ double sm[];
  const long long q = blockIdx.x + (long long)blockIdx.y * gridDim.x;
  int ib, jk;
  if (TYPE == 2 && a.same) {  // SSSS, one class: unordered pairs jk <= ib
    long long r = (long long)((sqrt(8.0 * (double)q + 1.0) - 1.0) * 0.5);
    while (r * (r + 1) / 2 > q) r--;
    while ((r + 1) * (r + 2) / 2 <= q) r++;
    ib = (int)r;
    jk = (int)(q - r * (r + 1) / 2);
  } else {
    ib = (int)(q / a.nKet);
    jk = (int)(q % a.nKet);
  }
  if (ib >= a.nBra || !in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) return;
  const int ns = a.nShell;
  const PairDev P = a.pairs[a.braBeg + ib];
  const PairDev Q = a.pairs[a.ketBeg + jk];
  if (a.skipSingle && P.npp == 1 && Q.npp == 1) return;  // rel_gemm_kernel's
  bool work, mine;
  {
    int s1, s2, s3, s4;
    double q12, q34;
    if (TYPE == 1) {
      s1 = P.s1; s2 = P.s2; s3 = Q.s1; s4 = Q.s2;
      q12 = __ldg(a.qSS + s1 + (size_t)s2 * ns);
      q34 = __ldg(a.qLL + s3 + (size_t)s4 * ns);
    } else {
      const bool pRef = P.lex >= Q.lex;
      const PairDev& R12 = pRef ? P : Q;
      const PairDev& R34 = pRef ? Q : P;
      s1 = R12.s1; s2 = R12.s2; s3 = R34.s1; s4 = R34.s2;
      q12 = __ldg(a.qSS + s1 + (size_t)s2 * ns);
      q34 = __ldg(a.qSS + s3 + (size_t)s4 * ns);
    }
    const double bound = sh_max(a.norms, s1, s2, s3, s4, ns) * q12 * q34;
    work = !a.screen || bound >= a.thresh;
    const bool lo = a.mixed && bound < a.cut &&
                    fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib),
                                  __ldg(a.pairRange + a.ketBeg + jk),
                                  la + lb + lc + ld + 2 + 2 * (TYPE == 2), 1, TYPE == 2);
    mine = work && (IS32 ? lo : !lo);
  }
  if (threadIdx.x == 0) {
    if (!IS32) atomicAdd(a.counters + 0, 1ull);
    if (!IS32 && !work) atomicAdd(a.counters + 1, 1ull);
    if (mine) atomicAdd(a.counters + (IS32 ? 2 : 3), 1ull);
  }
  if (!mine) return;  // block-uniform
  const T* boysT = reinterpret_cast<const T*>(IS32 ? (const void*)a.boys32 : (const void*)a.boys);

  constexpr int NB = (TYPE == 2) ? 4 : 1;
  constexpr int NC = 4 * NB;
  const int tid = threadIdx.x;
  const int na = ncart(la), nb = ncart(lb), ncc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb;
  const int dK = (TYPE == 2) ? 1 : 0;
  const int Lb = la + lb + 2, L = Lb + lc + ld + 2 * dK;
  const int FL = 2 * max(la, lb) + 3, FLk = 2 * max(lc, ld) + 3;
  const RelBlockLayout Lo = rel_block_layout(la, lb, lc, ld, TYPE);
  int* htab = reinterpret_cast<int*>(sm + Lo.oT);
  htab_fill(htab, nherm(L));  // read after prep's first barrier
  const FastDiv fhbB(nherm(Lb)), fnbB(nb);
  T* Rb[2] = {reinterpret_cast<T*>(sm + Lo.oR0), reinterpret_cast<T*>(sm + Lo.oR1)};
  T* Eb = reinterpret_cast<T*>(sm + Lo.oEb);
  T* Ek = reinterpret_cast<T*>(sm + Lo.oEk);
  T* fa = reinterpret_cast<T*>(sm + Lo.oFa);
  T* fc = reinterpret_cast<T*>(sm + Lo.oFc);
  T* G = reinterpret_cast<T*>(sm + Lo.oG);
  double* Mc = sm + Lo.oM;
  T* Fs = reinterpret_cast<T*>(sm + Lo.oF);
  double* Js = sm + Lo.oJ;
  const int E1b = (la + 2) * (lb + 2) * (la + lb + 3);
  const int E1k = (lc + 1 + dK) * (ld + 1 + dK) * (lc + ld + 1 + 2 * dK);
  const ShellDev SA = a.shells[P.shA], SB = a.shells[P.shB];
  const ShellDev SC = a.shells[Q.shA], SD = a.shells[Q.shB];
  const bool dAB = P.shA == P.shB, dCD = Q.shA == Q.shB, samePQ = P.lex == Q.lex;
  const double s12d = dAB ? 1.0 : 2.0, s34d = dCD ? 1.0 : 2.0;
  const double w12 = dAB ? 0.5 : 1.0, w34 = dCD ? 0.5 : 1.0;
  const size_t nc = a.ncart;
  const T* R = Rb[0];  // R^(0) after the recursion
  double ec = 0.0, ed = 0.0;
  T pref = T(0);

  // E tables, R and the bra factors of primitive quartet (ip, iq)
  auto prep = [&](int ip, int iq) {
    const PrimPairDev& A = a.pp[P.pp_off + ip];
    const PrimPairDev& B = a.pp[Q.pp_off + iq];
    double ea, eb;
    pair_exps(SA, SB, a.prim, A, ea, eb);
    pair_exps(SC, SD, a.prim, B, ec, ed);
    if (tid < 3)
      hermite_E_rt<T, LMAX + 1>(la + 1, lb + 1, T(A.o2p), T(A.PA[tid]), T(A.PB[tid]),
                                Eb + tid * E1b);
    else if (tid < 6)
      hermite_E_rt<T, LMAX + 1>(lc + dK, ld + dK, T(B.o2p), T(B.PA[tid - 3]), T(B.PB[tid - 3]),
                                Ek + (tid - 3) * E1k);
    const T X = T(A.P[0] - B.P[0]), Y = T(A.P[1] - B.P[1]), Z = T(A.P[2] - B.P[2]);
    const T pq = T(A.p) + T(B.p), alpha = T(A.p) * T(B.p) / pq;
    pref = T(PI52X2) / sqrt(pq) * T(A.Kp) * T(B.Kp);
    if (tid >= 32 && tid < 64)
      boys_lanes<T>(L, alpha * (X * X + Y * Y + Z * Z), Fs, boysT, tid - 32);
    __syncthreads();
    // R^(n)_tuv, n = L .. 0, from R^(n+1); level n in Rb[n & 1]
    const T m2a = T(-2) * alpha;
    for (int n = L; n >= 0; n--) {
      T* cur = Rb[n & 1];
      const T* prv = Rb[(n + 1) & 1];
      const int cnt = nherm(L - n);
      for (int e = tid; e < cnt; e += RB_THREADS) {
        int t, u, v;
        htab_get(htab, e, t, u, v);
        T val;
        if (e == 0) {
          T f = T(1);
          for (int k = 0; k < n; k++) f *= m2a;
          val = f * Fs[n];
        } else if (t > 0) {
          val = X * prv[hidx(t - 1, u, v)];
          if (t > 1) val += T(t - 1) * prv[hidx(t - 2, u, v)];
        } else if (u > 0) {
          val = Y * prv[hidx(0, u - 1, v)];
          if (u > 1) val += T(u - 1) * prv[hidx(0, u - 2, v)];
        } else {
          val = Z * prv[hidx(0, 0, v - 1)];
          if (v > 1) val += T(v - 1) * prv[hidx(0, 0, v - 2)];
        }
        cur[e] = val;
      }
      __syncthreads();
    }
    // bra factors of every axis, exponent pair and derivative type
    for (int it = tid; it < 3 * (la + 1) * (lb + 1) * 4; it += RB_THREADS) {
      const int ty = it % 4, jb = (it / 4) % (lb + 1), ia = (it / 4 / (lb + 1)) % (la + 1),
                x = it / 4 / (lb + 1) / (la + 1);
      axis_factor<T>(Eb + x * E1b, lb + 1, la + lb + 3, ia, jb, ty, T(2.0 * ea), T(2.0 * eb),
                     fa + (size_t)it * FL);
    }
    __syncthreads();
  };
  auto faOf = [&](int x, int i, int j, int ty) {
    return fa + (size_t)(((x * (la + 1) + i) * (lb + 1) + j) * 4 + ty) * FL;
  };

  const bool single = P.npp == 1 && Q.npp == 1;
  if (single) prep(0, 0);
  if (tid < 4) Js[tid] = 0.0;
#pragma unroll 1
  for (int cd = 0; cd < ncc * nd; cd++) {
    const int c = cd / nd, d = cd % nd;
    const int gC = Q.cA + c, gD = Q.cB + d;
    for (int e = tid; e < nab * NC; e += RB_THREADS) Mc[e] = 0.0;
#pragma unroll 1
    for (int ip = 0; ip < P.npp; ip++)
#pragma unroll 1
      for (int iq = 0; iq < Q.npp; iq++) {
        if (!single) prep(ip, iq);  // ends with a barrier
        // ket factors of this component pair (sign (-1)^t folded in)
        const int ntk = (TYPE == 2) ? 4 : 1;
        if (tid < 3 * ntk) {
          const int x = tid / ntk, ty = tid % ntk;
          const int ci = x == 0 ? cart_lx(lc, c) : (x == 1 ? cart_ly(lc, c) : cart_lz(lc, c));
          const int di = x == 0 ? cart_lx(ld, d) : (x == 1 ? cart_ly(ld, d) : cart_lz(ld, d));
          T* f = fc + (x * 4 + ty) * FLk;
          const int n = axis_factor<T>(Ek + x * E1k, ld + dK, lc + ld + 2 * dK + 1, ci, di, ty,
                                       T(2.0 * ec), T(2.0 * ed), f);
          for (int t = 1; t < n; t += 2) f[t] = -f[t];
        }
        __syncthreads();
        // G[b][tuv]
        const int hb = nherm(Lb);
        for (int e = tid; e < NB * hb; e += RB_THREADS) {
          int b, h;
          fhbB.divmod(e, b, h);
          int t, u, v;
          htab_get(htab, h, t, u, v);
          const int ci[3] = {cart_lx(lc, c), cart_ly(lc, c), cart_lz(lc, c)};
          const int di[3] = {cart_lx(ld, d), cart_ly(ld, d), cart_lz(ld, d)};
          T gsum = T(0);
          for (int kk = 0; kk < (TYPE == 2 ? 3 : 1); kk++)
            for (int ll = 0; ll < (TYPE == 2 ? 3 : 1); ll++) {
              int op = 0;
              double sg = 1.0;
              int tyx = 0, tyy = 0, tyz = 0;
              if (TYPE == 2) {
                op_of(kk, ll, op, sg);
                if (op != b) continue;
                tyx = (kk == 0) | ((ll == 0) << 1);
                tyy = (kk == 1) | ((ll == 1) << 1);
                tyz = (kk == 2) | ((ll == 2) << 1);
              }
              const T* fx = fc + (0 * 4 + tyx) * FLk;
              const T* fy = fc + (1 * 4 + tyy) * FLk;
              const T* fz = fc + (2 * 4 + tyz) * FLk;
              const int nx = ci[0] + di[0] + (tyx & 1) + (tyx >> 1) + 1;
              const int ny = ci[1] + di[1] + (tyy & 1) + (tyy >> 1) + 1;
              const int nz = ci[2] + di[2] + (tyz & 1) + (tyz >> 1) + 1;
              T acc = T(0);
              for (int i = 0; i < nx; i++) {
                if (fx[i] == T(0)) continue;
                for (int j = 0; j < ny; j++) {
                  const T fxy = fx[i] * fy[j];
                  if (fxy == T(0)) continue;
                  acc += fxy * hdot_v(fz, nz, R, t + i, u + j, v);
                }
              }
              gsum += T(sg) * acc;
            }
          G[e] = pref * gsum;
        }
        __syncthreads();
        // operator components of every bra component pair: unit (ab, b)
        for (int e = tid; e < nab * NB; e += RB_THREADS) {
          const int ab = e / NB, b = e % NB;
          int ai, bi;
          fnbB.divmod(ab, ai, bi);
          const int ax[3] = {cart_lx(la, ai), cart_ly(la, ai), cart_lz(la, ai)};
          const int bx[3] = {cart_lx(lb, bi), cart_ly(lb, bi), cart_lz(lb, bi)};
          double m4[4] = {0.0, 0.0, 0.0, 0.0};
          for (int mu = 0; mu < 3; mu++)
            for (int nu = 0; nu < 3; nu++) {
              int op;
              double sg;
              op_of(mu, nu, op, sg);
              const int tx = (mu == 0) | ((nu == 0) << 1), ty = (mu == 1) | ((nu == 1) << 1),
                        tz = (mu == 2) | ((nu == 2) << 1);
              const T* gx = faOf(0, ax[0], bx[0], tx);
              const T* gy = faOf(1, ax[1], bx[1], ty);
              const T* gz = faOf(2, ax[2], bx[2], tz);
              m4[op] += sg * (double)bra_dot<T>(gx, ax[0] + bx[0] + (tx & 1) + (tx >> 1) + 1, gy,
                                     ax[1] + bx[1] + (ty & 1) + (ty >> 1) + 1, gz,
                                     ax[2] + bx[2] + (tz & 1) + (tz >> 1) + 1, G + b * hb);
            }
          for (int op = 0; op < 4; op++) Mc[ab * NC + op * NB + b] += m4[op];
        }
        __syncthreads();
      }
    // digestion, one bra component pair per thread
    RelCol col{gC, gD, dAB, dCD, samePQ, s34d, w12, samePQ ? 0.5 : 1.0, 0.0, {0, 0, 0, 0}};
    if (TYPE == 1) {
      col.rhoLL = __ldg(a.Xll + 2 * ((size_t)gD + (size_t)gC * nc));
    } else {
      const size_t eDC = (size_t)gD + (size_t)gC * nc;
      col.rvDC[0] = __ldg(a.Xss[0] + 2 * eDC);
      col.rvDC[1] = -__ldg(a.Xss[1] + 2 * eDC + 1);
      col.rvDC[2] = -__ldg(a.Xss[2] + 2 * eDC + 1);
      col.rvDC[3] = -__ldg(a.Xss[3] + 2 * eDC + 1);
    }
    for (int ab = tid; ab < nab; ab += RB_THREADS) {
      double jl[4] = {0.0, 0.0, 0.0, 0.0};
      rel_digest<TYPE>(a, P, col, ab / nb, ab % nb, Mc + ab * NC, jl);
      for (int b = 0; b < 4; b++)
        if (jl[b] != 0.0) atomicAdd(Js + b, jl[b]);
    }
    __syncthreads();
    if (tid == 0) {
      const size_t eCD = (size_t)gC + (size_t)gD * nc;
      if (TYPE == 1) {
        if (Js[0] != 0.0) atomicAdd(a.Jll + eCD, w34 * s12d * Js[0]);
      } else if (!samePQ) {
        for (int b = 0; b < 4; b++)
          if (Js[b] != 0.0) atomicAdd(a.Jss[b] + eCD, w34 * s12d * Js[b]);
      }
      for (int b = 0; b < 4; b++) Js[b] = 0.0;
    }
    __syncthreads();
  }
}

// Shared-memory layout of rel_llss_block_kernel (doubles).  The axis
// factors depend on a component pair only through its two exponents on the
// axis, so they are kept per (axis, i, j[, derivative type]); single-primitive
// launches digest each element as it is made and keep no accumulator Mc.
struct LlssBlockLayout {
  int oR0, oR1, oEb, oEk, oFa, oFc, oG, oM, oF, oJ, oT, total;
};
__host__ __device__ inline LlssBlockLayout llss_block_layout(int la, int lb, int lc, int ld,
                                                             bool single) {
  const int Lb = la + lb + 2, L = Lb + lc + ld;
  const int nab = ncart(la) * ncart(lb), ncd = ncart(lc) * ncart(ld);
  const int FL = 2 * (la > lb ? la : lb) + 3, FLk = lc + ld + 1;
  LlssBlockLayout Lo;
  int o = 0;
  auto take = [&](int n) { int r = o; o += (n + 1) / 2 * 2; return r; };
  Lo.oR0 = take(nherm(L));
  Lo.oR1 = take(nherm(L));
  Lo.oEb = take(3 * (la + 2) * (lb + 2) * (la + lb + 3));
  Lo.oEk = take(3 * (lc + 1) * (ld + 1) * (lc + ld + 1));
  Lo.oFa = take(3 * (la + 1) * (lb + 1) * 4 * FL);
  Lo.oFc = take(3 * (lc + 1) * (ld + 1) * FLk);
  Lo.oG = take(ncd * nherm(Lb));
  Lo.oM = take(single ? 0 : nab * ncd * 4);
  Lo.oF = take(L + 1);
  Lo.oJ = take(ncd);
  Lo.oT = take((nherm(L) + 1) / 2);  // packed (t, u, v) of each Hermite index, int
  Lo.total = o;
  return Lo;
}

// LLSS form of the block kernel: the ket pair is undifferentiated, so the
// ket-contracted Hermite sums G[cd][tuv] of every ket component pair are
// built at once, and the operator components of every (bra, ket) component
// element are one work unit per thread (nab x ncd units); digestion per
// element, the per-column Coulomb sums J_LL(C,D) reduced in shared memory.
// With skipSingle set the quartets of two single-primitive pairs are
// rel_llss_single_kernel's.
template <typename T>
__global__ void __launch_bounds__(RB_THREADS)
    rel_llss_block_kernel(const RelLaunch a, int la, int lb, int lc, int ld) {
  constexpr bool IS32 = sizeof(T) == 4;
  extern __shared__ double sm[];
  const long long q = blockIdx.x + (long long)blockIdx.y * gridDim.x;
  const int ib = (int)(q / a.nKet), jk = (int)(q % a.nKet);
  if (ib >= a.nBra || !in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) return;
  const int ns = a.nShell;
  const PairDev P = a.pairs[a.braBeg + ib];
  const PairDev Q = a.pairs[a.ketBeg + jk];
  if (a.skipSingle && P.npp == 1 && Q.npp == 1) return;  // rel_llss_single_kernel's
  const double bound = sh_max(a.norms, P.s1, P.s2, Q.s1, Q.s2, ns) *
                       __ldg(a.qSS + P.s1 + (size_t)P.s2 * ns) *
                       __ldg(a.qLL + Q.s1 + (size_t)Q.s2 * ns);
  const bool work = !a.screen || bound >= a.thresh;
  const bool lo = a.mixed && bound < a.cut &&
                  fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib),
                                __ldg(a.pairRange + a.ketBeg + jk), la + lb + lc + ld + 2, 1, 0);
  const bool mine = work && (IS32 ? lo : !lo);
  if (threadIdx.x == 0) {
    if (!IS32) atomicAdd(a.counters + 0, 1ull);
    if (!IS32 && !work) atomicAdd(a.counters + 1, 1ull);
    if (mine) atomicAdd(a.counters + (IS32 ? 2 : 3), 1ull);
  }
  if (!mine) return;  // block-uniform
  const T* boysT = reinterpret_cast<const T*>(IS32 ? (const void*)a.boys32 : (const void*)a.boys);

  const int tid = threadIdx.x;
  const int na = ncart(la), nb = ncart(lb), ncc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb, ncd = ncc * nd;
  const int Lb = la + lb + 2, L = Lb + lc + ld;
  const int hb = nherm(Lb);
  const int FL = 2 * max(la, lb) + 3, FLk = lc + ld + 1;
  const LlssBlockLayout Lo = llss_block_layout(la, lb, lc, ld, false);
  int* htab = reinterpret_cast<int*>(sm + Lo.oT);
  htab_fill(htab, nherm(L));  // read after the first barrier of the primitive loop
  T* Rb[2] = {reinterpret_cast<T*>(sm + Lo.oR0), reinterpret_cast<T*>(sm + Lo.oR1)};
  T* Eb = reinterpret_cast<T*>(sm + Lo.oEb);
  T* Ek = reinterpret_cast<T*>(sm + Lo.oEk);
  T* fa = reinterpret_cast<T*>(sm + Lo.oFa);
  T* fc = reinterpret_cast<T*>(sm + Lo.oFc);
  T* G = reinterpret_cast<T*>(sm + Lo.oG);
  double* Mc = sm + Lo.oM;
  T* Fs = reinterpret_cast<T*>(sm + Lo.oF);
  double* Js = sm + Lo.oJ;
  const int E1b = (la + 2) * (lb + 2) * (la + lb + 3);
  const int E1k = (lc + 1) * (ld + 1) * (lc + ld + 1);
  const ShellDev SA = a.shells[P.shA], SB = a.shells[P.shB];
  const ShellDev SC = a.shells[Q.shA], SD = a.shells[Q.shB];
  const bool dAB = P.shA == P.shB, dCD = Q.shA == Q.shB;
  const double s12d = dAB ? 1.0 : 2.0, s34d = dCD ? 1.0 : 2.0;
  const double w12 = dAB ? 0.5 : 1.0, w34 = dCD ? 0.5 : 1.0;
  const size_t nc = a.ncart;
  const T* R = Rb[0];

  for (int e = tid; e < nab * ncd * 4; e += RB_THREADS) Mc[e] = 0.0;
  for (int e = tid; e < ncd; e += RB_THREADS) Js[e] = 0.0;
  // the axis factor vectors of (axis x, bra exponents i, j, type ty) and
  // (axis x, ket exponents i, j)
  auto faOf = [&](int x, int i, int j, int ty) {
    return fa + (size_t)(((x * (la + 1) + i) * (lb + 1) + j) * 4 + ty) * FL;
  };
  auto fcOf = [&](int x, int i, int j) {
    return fc + (size_t)((x * (lc + 1) + i) * (ld + 1) + j) * FLk;
  };
#pragma unroll 1
  for (int ip = 0; ip < P.npp; ip++)
#pragma unroll 1
    for (int iq = 0; iq < Q.npp; iq++) {
      const PrimPairDev& A = a.pp[P.pp_off + ip];
      const PrimPairDev& B = a.pp[Q.pp_off + iq];
      double ea, eb, ec, ed;
      pair_exps(SA, SB, a.prim, A, ea, eb);
      pair_exps(SC, SD, a.prim, B, ec, ed);
      __syncthreads();  // the previous primitive quartet's readers are done
      if (tid < 3)
        hermite_E_rt<T, LMAX + 1>(la + 1, lb + 1, T(A.o2p), T(A.PA[tid]), T(A.PB[tid]),
                                  Eb + tid * E1b);
      else if (tid < 6)
        hermite_E_rt<T, LMAX + 1>(lc, ld, T(B.o2p), T(B.PA[tid - 3]), T(B.PB[tid - 3]),
                                  Ek + (tid - 3) * E1k);
      const T X = T(A.P[0] - B.P[0]), Y = T(A.P[1] - B.P[1]), Z = T(A.P[2] - B.P[2]);
      const T pq = T(A.p) + T(B.p), alpha = T(A.p) * T(B.p) / pq;
      const T pref = T(PI52X2) / sqrt(pq) * T(A.Kp) * T(B.Kp);
      if (tid >= 32 && tid < 64)
        boys_lanes<T>(L, alpha * (X * X + Y * Y + Z * Z), Fs, boysT, tid - 32);
      __syncthreads();
      const T m2a = T(-2) * alpha;
      for (int n = L; n >= 0; n--) {
        T* cur = Rb[n & 1];
        const T* prv = Rb[(n + 1) & 1];
        const int cnt = nherm(L - n);
        for (int e = tid; e < cnt; e += RB_THREADS) {
          int t, u, v;
          htab_get(htab, e, t, u, v);
          T val;
          if (e == 0) {
            T f = T(1);
            for (int k = 0; k < n; k++) f *= m2a;
            val = f * Fs[n];
          } else if (t > 0) {
            val = X * prv[hidx(t - 1, u, v)];
            if (t > 1) val += T(t - 1) * prv[hidx(t - 2, u, v)];
          } else if (u > 0) {
            val = Y * prv[hidx(0, u - 1, v)];
            if (u > 1) val += T(u - 1) * prv[hidx(0, u - 2, v)];
          } else {
            val = Z * prv[hidx(0, 0, v - 1)];
            if (v > 1) val += T(v - 1) * prv[hidx(0, 0, v - 2)];
          }
          cur[e] = val;
        }
        __syncthreads();
      }
      // bra factors (every axis, exponent pair, derivative type); ket factors
      // (undifferentiated, sign (-1)^t folded in)
      for (int it = tid; it < 3 * (la + 1) * (lb + 1) * 4; it += RB_THREADS) {
        const int ty = it % 4, jb = (it / 4) % (lb + 1), ia = (it / 4 / (lb + 1)) % (la + 1),
                  x = it / 4 / (lb + 1) / (la + 1);
        axis_factor<T>(Eb + x * E1b, lb + 1, la + lb + 3, ia, jb, ty, T(2.0 * ea), T(2.0 * eb),
                       fa + (size_t)it * FL);
      }
      for (int it = tid; it < 3 * (lc + 1) * (ld + 1); it += RB_THREADS) {
        const int di = it % (ld + 1), ci = (it / (ld + 1)) % (lc + 1),
                  x = it / (ld + 1) / (lc + 1);
        T* f = fc + (size_t)it * FLk;
        const int n = axis_factor<T>(Ek + x * E1k, ld, lc + ld + 1, ci, di, 0, T(0), T(0), f);
        for (int t = 1; t < n; t += 2) f[t] = -f[t];
      }
      __syncthreads();
      // G[cd][tuv] of every ket component pair
      for (int e = tid; e < ncd * hb; e += RB_THREADS) {
        const int cd = e / hb, h = e % hb, c = cd / nd, d = cd % nd;
        int t, u, v;
        htab_get(htab, h, t, u, v);
        const T* fx = fcOf(0, cart_lx(lc, c), cart_lx(ld, d));
        const T* fy = fcOf(1, cart_ly(lc, c), cart_ly(ld, d));
        const T* fz = fcOf(2, cart_lz(lc, c), cart_lz(ld, d));
        const int nx = cart_lx(lc, c) + cart_lx(ld, d) + 1;
        const int ny = cart_ly(lc, c) + cart_ly(ld, d) + 1;
        const int nz = cart_lz(lc, c) + cart_lz(ld, d) + 1;
        T acc = T(0);
        for (int i = 0; i < nx; i++) {
          if (fx[i] == T(0)) continue;
          for (int j = 0; j < ny; j++) {
            const T fxy = fx[i] * fy[j];
            if (fxy == T(0)) continue;
            acc += fxy * hdot_v(fz, nz, R, t + i, u + j, v);
          }
        }
        G[e] = pref * acc;
      }
      __syncthreads();
      // operator components of every (bra, ket) component element
      for (int e = tid; e < nab * ncd; e += RB_THREADS) {
        const int ab = e / ncd, cd = e % ncd;
        const int ai = ab / nb, bi = ab % nb;
        const int ax[3] = {cart_lx(la, ai), cart_ly(la, ai), cart_lz(la, ai)};
        const int bx[3] = {cart_lx(lb, bi), cart_ly(lb, bi), cart_lz(lb, bi)};
        double m4[4] = {0.0, 0.0, 0.0, 0.0};
        for (int mu = 0; mu < 3; mu++)
          for (int nu = 0; nu < 3; nu++) {
            int op;
            double sg;
            op_of(mu, nu, op, sg);
            const int tx = (mu == 0) | ((nu == 0) << 1), ty = (mu == 1) | ((nu == 1) << 1),
                      tz = (mu == 2) | ((nu == 2) << 1);
            m4[op] += sg * (double)bra_dot<T>(faOf(0, ax[0], bx[0], tx),
                                   ax[0] + bx[0] + (tx & 1) + (tx >> 1) + 1,
                                   faOf(1, ax[1], bx[1], ty),
                                   ax[1] + bx[1] + (ty & 1) + (ty >> 1) + 1,
                                   faOf(2, ax[2], bx[2], tz),
                                   ax[2] + bx[2] + (tz & 1) + (tz >> 1) + 1, G + (size_t)cd * hb);
          }
        for (int op = 0; op < 4; op++) Mc[(size_t)e * 4 + op] += m4[op];
      }
    }
  __syncthreads();
  // digestion, one (bra, ket) component element per thread
  for (int e = tid; e < nab * ncd; e += RB_THREADS) {
    const int ab = e / ncd, cd = e % ncd;
    const int gC = Q.cA + cd / nd, gD = Q.cB + cd % nd;
    RelCol col{gC, gD, dAB, dCD, false, s34d, w12, 1.0,
               __ldg(a.Xll + 2 * ((size_t)gD + (size_t)gC * nc)), {0, 0, 0, 0}};
    double jl[4] = {0.0, 0.0, 0.0, 0.0};
    rel_digest<1>(a, P, col, ab / nb, ab % nb, Mc + (size_t)e * 4, jl);
    if (jl[0] != 0.0) atomicAdd(Js + cd, jl[0]);
  }
  __syncthreads();
  for (int cd = tid; cd < ncd; cd += RB_THREADS)
    if (Js[cd] != 0.0)
      atomicAdd(a.Jll + (size_t)(Q.cA + cd / nd) + (size_t)(Q.cB + cd % nd) * nc,
                w34 * s12d * Js[cd]);
}

// LLSS quartets of two single-primitive pairs (every quartet of an
// uncontracted basis): one block per bra pair and tile of kt ket pairs (kt
// up to LS_KT; 1 for launches too small to fill the GPU otherwise).
// The bra pair's E tables and axis factors are made once; per ket its E
// tables, Boys values and R (level by level over the block), the ket factors,
// G[cd][tuv] of every ket component pair, then the operator components of
// every (bra, ket) component element, digested as they are made (one
// primitive quartet: nothing to accumulate).  Same quartet set, screens and
// updates as rel_llss_block_kernel.
constexpr int LS_KT = 8;

template <typename T>
__global__ void __launch_bounds__(RB_THREADS, 8)
    rel_llss_single_kernel(const RelLaunch a, int la, int lb, int lc, int ld, int kt) {
  constexpr bool IS32 = sizeof(T) == 4;
  extern __shared__ double sm[];
  const int nTiles = (a.nKet + kt - 1) / kt;
  const long long q = blockIdx.x + (long long)blockIdx.y * gridDim.x;
  const int ib = (int)(q / nTiles), tile = (int)(q % nTiles);
  if (ib >= a.nBra || !in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) return;
  const PairDev P = a.pairs[a.braBeg + ib];
  if (P.npp != 1) return;  // contracted bra: rel_llss_block_kernel
  const int jkEnd = min(tile * kt + kt, a.nKet);
  const int ns = a.nShell;
  const T* boysT = reinterpret_cast<const T*>(IS32 ? (const void*)a.boys32 : (const void*)a.boys);

  const int tid = threadIdx.x;
  const int na = ncart(la), nb = ncart(lb), ncc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb, ncd = ncc * nd;
  const int Lb = la + lb + 2, L = Lb + lc + ld;
  const int hb = nherm(Lb);
  const int FL = 2 * max(la, lb) + 3, FLk = lc + ld + 1;
  const LlssBlockLayout Lo = llss_block_layout(la, lb, lc, ld, true);
  int* htab = reinterpret_cast<int*>(sm + Lo.oT);
  htab_fill(htab, nherm(L));  // read after the bra phase's barrier
  T* Rb[2] = {reinterpret_cast<T*>(sm + Lo.oR0), reinterpret_cast<T*>(sm + Lo.oR1)};
  T* Eb = reinterpret_cast<T*>(sm + Lo.oEb);
  T* Ek = reinterpret_cast<T*>(sm + Lo.oEk);
  T* fa = reinterpret_cast<T*>(sm + Lo.oFa);
  T* fc = reinterpret_cast<T*>(sm + Lo.oFc);
  T* G = reinterpret_cast<T*>(sm + Lo.oG);
  T* Fs = reinterpret_cast<T*>(sm + Lo.oF);
  double* Js = sm + Lo.oJ;
  const int E1b = (la + 2) * (lb + 2) * (la + lb + 3);
  const int E1k = (lc + 1) * (ld + 1) * (lc + ld + 1);
  const ShellDev SA = a.shells[P.shA], SB = a.shells[P.shB];
  const bool dAB = P.shA == P.shB;
  const double s12d = dAB ? 1.0 : 2.0, w12 = dAB ? 0.5 : 1.0;
  const size_t nc = a.ncart;
  const T* R = Rb[0];
  auto faOf = [&](int x, int i, int j, int ty) {
    return fa + (size_t)(((x * (la + 1) + i) * (lb + 1) + j) * 4 + ty) * FL;
  };
  auto fcOf = [&](int x, int i, int j) {
    return fc + (size_t)((x * (lc + 1) + i) * (ld + 1) + j) * FLk;
  };
  const FastDiv fncd(ncd), fnb(nb), fnd(nd), fhb(hb);

  // ---- bra phase: E tables and axis factors of every axis, exponent pair
  // and derivative type
  const PrimPairDev& A = a.pp[P.pp_off];
  double ea, eb;
  pair_exps(SA, SB, a.prim, A, ea, eb);
  if (tid < 3)
    hermite_E_rt<T, LMAX + 1>(la + 1, lb + 1, T(A.o2p), T(A.PA[tid]), T(A.PB[tid]),
                              Eb + tid * E1b);
  __syncthreads();
  for (int it = tid; it < 3 * (la + 1) * (lb + 1) * 4; it += RB_THREADS) {
    const int ty = it % 4, jb = (it / 4) % (lb + 1), ia = (it / 4 / (lb + 1)) % (la + 1),
              x = it / 4 / (lb + 1) / (la + 1);
    axis_factor<T>(Eb + x * E1b, lb + 1, la + lb + 3, ia, jb, ty, T(2.0 * ea), T(2.0 * eb),
                   fa + (size_t)it * FL);
  }
  // (read after the barriers of the first ket)

  // ---- the tile's kets
#pragma unroll 1
  for (int jk = tile * kt; jk < jkEnd; jk++) {
    const PairDev Q = a.pairs[a.ketBeg + jk];
    if (Q.npp != 1) continue;  // contracted ket: rel_llss_block_kernel (block-uniform)
    const double bound = sh_max(a.norms, P.s1, P.s2, Q.s1, Q.s2, ns) *
                         __ldg(a.qSS + P.s1 + (size_t)P.s2 * ns) *
                         __ldg(a.qLL + Q.s1 + (size_t)Q.s2 * ns);
    const bool work = !a.screen || bound >= a.thresh;
    const bool lo = a.mixed && bound < a.cut &&
                    fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib),
                                  __ldg(a.pairRange + a.ketBeg + jk), la + lb + lc + ld + 2, 1,
                                  0);
    const bool mine = work && (IS32 ? lo : !lo);
    if (tid == 0) {
      if (!IS32) atomicAdd(a.counters + 0, 1ull);
      if (!IS32 && !work) atomicAdd(a.counters + 1, 1ull);
      if (mine) atomicAdd(a.counters + (IS32 ? 2 : 3), 1ull);
    }
    if (!mine) continue;  // block-uniform
    const bool dCD = Q.shA == Q.shB;
    const double s34d = dCD ? 1.0 : 2.0, w34 = dCD ? 0.5 : 1.0;
    const PrimPairDev& B = a.pp[Q.pp_off];
    const T X = T(A.P[0] - B.P[0]), Y = T(A.P[1] - B.P[1]), Z = T(A.P[2] - B.P[2]);
    const T pq = T(A.p) + T(B.p), alpha = T(A.p) * T(B.p) / pq;
    const T pref = T(PI52X2) / sqrt(pq) * T(A.Kp) * T(B.Kp);
    // the previous ket's readers are past the barrier that ended its loop
    if (tid < 3)
      hermite_E_rt<T, LMAX + 1>(lc, ld, T(B.o2p), T(B.PA[tid]), T(B.PB[tid]), Ek + tid * E1k);
    else if (tid >= 32 && tid < 64)
      boys_lanes<T>(L, alpha * (X * X + Y * Y + Z * Z), Fs, boysT, tid - 32);
    for (int e = tid; e < ncd; e += RB_THREADS) Js[e] = 0.0;
    __syncthreads();
    const T m2a = T(-2) * alpha;
    for (int n = L; n >= 0; n--) {
      T* cur = Rb[n & 1];
      const T* prv = Rb[(n + 1) & 1];
      const int cnt = nherm(L - n);
      for (int e = tid; e < cnt; e += RB_THREADS) {
        int t, u, v;
        htab_get(htab, e, t, u, v);
        T val;
        if (e == 0) {
          T f = T(1);
          for (int k = 0; k < n; k++) f *= m2a;
          val = f * Fs[n];
        } else if (t > 0) {
          val = X * prv[hidx(t - 1, u, v)];
          if (t > 1) val += T(t - 1) * prv[hidx(t - 2, u, v)];
        } else if (u > 0) {
          val = Y * prv[hidx(0, u - 1, v)];
          if (u > 1) val += T(u - 1) * prv[hidx(0, u - 2, v)];
        } else {
          val = Z * prv[hidx(0, 0, v - 1)];
          if (v > 1) val += T(v - 1) * prv[hidx(0, 0, v - 2)];
        }
        cur[e] = val;
      }
      if (n == L) {  // the ket factors beside the first level (Ek is complete)
        for (int it = tid; it < 3 * (lc + 1) * (ld + 1); it += RB_THREADS) {
          const int di = it % (ld + 1), ci = (it / (ld + 1)) % (lc + 1),
                    x = it / (ld + 1) / (lc + 1);
          T* f = fc + (size_t)it * FLk;
          const int nf = axis_factor<T>(Ek + x * E1k, ld, lc + ld + 1, ci, di, 0, T(0), T(0), f);
          for (int t = 1; t < nf; t += 2) f[t] = -f[t];
        }
      }
      __syncthreads();
    }
    // G[cd][tuv] of every ket component pair
    for (int e = tid; e < ncd * hb; e += RB_THREADS) {
      int cd, h, c, d;
      fhb.divmod(e, cd, h);
      fnd.divmod(cd, c, d);
      int t, u, v;
      htab_get(htab, h, t, u, v);
      const T* fx = fcOf(0, cart_lx(lc, c), cart_lx(ld, d));
      const T* fy = fcOf(1, cart_ly(lc, c), cart_ly(ld, d));
      const T* fz = fcOf(2, cart_lz(lc, c), cart_lz(ld, d));
      const int nx = cart_lx(lc, c) + cart_lx(ld, d) + 1;
      const int ny = cart_ly(lc, c) + cart_ly(ld, d) + 1;
      const int nz = cart_lz(lc, c) + cart_lz(ld, d) + 1;
      T acc = T(0);
      for (int i = 0; i < nx; i++) {
        if (fx[i] == T(0)) continue;
        for (int j = 0; j < ny; j++) {
          const T fxy = fx[i] * fy[j];
          if (fxy == T(0)) continue;
          acc += fxy * hdot_v(fz, nz, R, t + i, u + j, v);
        }
      }
      G[e] = pref * acc;
    }
    __syncthreads();
    // operator components of every (bra, ket) component element, digested
    for (int e = tid; e < nab * ncd; e += RB_THREADS) {
      int ab, cd, ai, bi, c, d;
      fncd.divmod(e, ab, cd);
      fnb.divmod(ab, ai, bi);
      fnd.divmod(cd, c, d);
      const int ax[3] = {cart_lx(la, ai), cart_ly(la, ai), cart_lz(la, ai)};
      const int bx[3] = {cart_lx(lb, bi), cart_ly(lb, bi), cart_lz(lb, bi)};
      double m4[4] = {0.0, 0.0, 0.0, 0.0};
      for (int mu = 0; mu < 3; mu++)
        for (int nu = 0; nu < 3; nu++) {
          int op;
          double sg;
          op_of(mu, nu, op, sg);
          const int tx = (mu == 0) | ((nu == 0) << 1), ty = (mu == 1) | ((nu == 1) << 1),
                    tz = (mu == 2) | ((nu == 2) << 1);
          m4[op] += sg * (double)bra_dot<T>(faOf(0, ax[0], bx[0], tx),
                                 ax[0] + bx[0] + (tx & 1) + (tx >> 1) + 1,
                                 faOf(1, ax[1], bx[1], ty),
                                 ax[1] + bx[1] + (ty & 1) + (ty >> 1) + 1,
                                 faOf(2, ax[2], bx[2], tz),
                                 ax[2] + bx[2] + (tz & 1) + (tz >> 1) + 1, G + (size_t)cd * hb);
        }
      const int gC = Q.cA + c, gD = Q.cB + d;
      RelCol col{gC, gD, dAB, dCD, false, s34d, w12, 1.0,
                 __ldg(a.Xll + 2 * ((size_t)gD + (size_t)gC * nc)), {0, 0, 0, 0}};
      double jl[4] = {0.0, 0.0, 0.0, 0.0};
      rel_digest<1>(a, P, col, ai, bi, m4, jl);
      if (jl[0] != 0.0) atomicAdd(Js + cd, jl[0]);
    }
    __syncthreads();
    for (int cd = tid; cd < ncd; cd += RB_THREADS)
      if (Js[cd] != 0.0)
        atomicAdd(a.Jll + (size_t)(Q.cA + cd / nd) + (size_t)(Q.cB + cd % nd) * nc,
                  w34 * s12d * Js[cd]);
    __syncthreads();  // the ket's shared memory is free for the next one
  }
}

// ---------------------------------------- GEMM form of the block kernels
// For a single-primitive quartet (every quartet of an uncontracted basis)
// the block kernels' work is two dense products per ket chunk:
//   G[h][(cd, b)] = sum_h' K[h'][(cd, b)] Rm[h'][h],
//   M[(ab, op)][(cd, b)] = sum_h H[h][(ab, op)] G[h][(cd, b)],
// with H / K the bra / ket Hermite coefficients of every component pair
// already combined over the derivative pairs of each operator component
// (H[(ab, op)][tuv] = sum_{mu nu -> op} sg f_x f_y f_z), and
// Rm[h'][h] = pref R_{t+tau, u+nu, v+phi} (ket sign folded into K).  Both
// run as register-tiled loops over shared memory, every lane busy: a thread
// owns a 4 x 4 tile, for the second product (one bra pair's 4 operator
// components) x (one ket pair's 4 components; LLSS: 4 ket pairs), which is
// then digested from registers at the reference's update sites.  A block
// takes one bra pair and a tile of up to KT ket pairs: the bra's E tables,
// axis factors and H are built once and stay in shared memory while the
// block walks its kets; per ket the R recursion runs over the block from a
// table of Hermite indices.  Same quartet set, screens
// and digestion as the block kernels, which keep the contracted quartets
// (and the classes whose layout does not fit).
constexpr int RG_THREADS = 256;
constexpr size_t RG_SMEM_MAX = 224 * 1024;
constexpr size_t RG_SMEM_HALF = 112 * 1024;  // two blocks per SM (228 KB, 1 KB reserved each)

struct RelGemmLayout {
  int HB, HBp, HK, HR, CH, CR, CRp, NT;
  int oH, oRm, oFk, oJs, oTuv, oScr;
  int oEb, oFa;                 // bra phase, in the scratch area
  int oEk, oR0, oR1, oF;        // per-ket phase, in the scratch area
  int oK, oG;                   // per ket chunk, in the scratch area
  int total;
};
__host__ __device__ inline int rg_round(int n, int m) { return (n + m - 1) / m * m; }
// offsets and total in elements of esz bytes (8: FP64, 4: FP32 arithmetic)
__host__ __device__ inline RelGemmLayout rel_gemm_layout(int la, int lb, int lc, int ld, int type,
                                                         int CH, int esz) {
  const int dK = type == 2 ? 1 : 0, NB = type == 2 ? 4 : 1;
  const int Lb = la + lb + 2, Lk = lc + ld + 2 * dK, L = Lb + Lk;
  const int nab = ncart(la) * ncart(lb), ncd = ncart(lc) * ncart(ld);
  const int FL = 2 * (la > lb ? la : lb) + 3, FLk = 2 * (lc > ld ? lc : ld) + 3;
  RelGemmLayout Lo;
  Lo.HB = nherm(Lb);
  Lo.HBp = rg_round(Lo.HB, 4);
  Lo.HK = nherm(Lk);
  Lo.HR = nab * 4;
  Lo.CH = CH;
  Lo.CR = CH * NB;
  Lo.CRp = rg_round(Lo.CR, 4);
  Lo.NT = nherm(L);
  int o = 0;
  auto take = [&](int n) { int r = o; o += rg_round(n, 4); return r; };
  Lo.oH = take(Lo.HB * Lo.HR);
  Lo.oRm = take(Lo.HK * Lo.HBp);
  Lo.oFk = take(ncd * 12 * FLk);
  Lo.oJs = take(CH * 4 * 8 / esz);           // per-column Coulomb sums, double
  Lo.oTuv = take((Lo.NT * 4 + esz - 1) / esz);  // packed (t, u, v) of each Hermite index, int
  Lo.oScr = o;
  int p = o;
  auto takeB = [&](int n) { int r = p; p += rg_round(n, 4); return r; };
  Lo.oEb = takeB(3 * (la + 2) * (lb + 2) * (la + lb + 3));
  Lo.oFa = takeB(3 * (la + 1) * (lb + 1) * 4 * FL);  // per (axis, exponent pair, type)
  int k = o;
  auto takeK = [&](int n) { int r = k; k += rg_round(n, 4); return r; };
  Lo.oEk = takeK(3 * (lc + 1 + dK) * (ld + 1 + dK) * (lc + ld + 1 + 2 * dK));
  Lo.oR0 = takeK(nherm(L));
  Lo.oR1 = takeK(nherm(L));
  Lo.oF = takeK(L + 1);
  int q = o;
  auto takeC = [&](int n) { int r = q; q += rg_round(n, 4); return r; };
  Lo.oK = takeC(Lo.HK * Lo.CRp);
  Lo.oG = takeC(Lo.HBp * Lo.CRp);
  Lo.total = p > k ? p : k;
  if (q > Lo.total) Lo.total = q;
  return Lo;
}
// the ket chunk: the largest whose layout leaves two blocks per SM, if that
// is at least 4 ket pairs (or all of them); else the largest that fits at
// all (one block per SM); 0: the class does not fit
inline int rel_gemm_chunk(int la, int lb, int lc, int ld, int type, int esz) {
  const int ncd = ncart(lc) * ncart(ld);
  for (int ch = ncd; ch >= 1; ch--)
    if ((size_t)rel_gemm_layout(la, lb, lc, ld, type, ch, esz).total * esz <= RG_SMEM_HALF) {
      if (ch >= 4 || ch == ncd) return ch;
      break;
    }
  for (int ch = ncd; ch >= 1; ch--)
    if ((size_t)rel_gemm_layout(la, lb, lc, ld, type, ch, esz).total * esz <= RG_SMEM_MAX)
      return ch;
  return 0;
}
// four consecutive elements (16-byte aligned)
__device__ __forceinline__ void rg_ld4(const double* p, double (&v)[4]) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void rg_ld4(const float* p, float (&v)[4]) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void rg_st4(double* p, double a, double b, double c, double d) {
  reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
  reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
}
__device__ __forceinline__ void rg_st4(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}
// ket pairs per block
constexpr int RG_KT = 8;

// T: primitive arithmetic (double; float for the small-bound quartets of a
// mixed launch); the operator components are digested in FP64.
template <int TYPE, typename T>
__global__ void __launch_bounds__(RG_THREADS, 2)
    rel_gemm_kernel(const RelLaunch a, int la, int lb, int lc, int ld, int CH) {
  constexpr bool IS32 = sizeof(T) == 4;
  extern __shared__ double sm[];
  T* smT = reinterpret_cast<T*>(sm);
  const int nTiles = (a.nKet + RG_KT - 1) / RG_KT;
  const long long q = blockIdx.x + (long long)blockIdx.y * gridDim.x;
  const int ib = (int)(q / nTiles), tile = (int)(q % nTiles);
  if (ib >= a.nBra || !in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) return;
  const bool tri = (TYPE == 2 && a.same);  // SSSS, one class: kets jk <= ib
  if (tri && tile * RG_KT > ib) return;
  const PairDev P = a.pairs[a.braBeg + ib];
  if (P.npp != 1) return;  // contracted: the block kernels
  const int jkEnd = min(tile * RG_KT + RG_KT, tri ? ib + 1 : a.nKet);
  const int ns = a.nShell;

  constexpr int NB = (TYPE == 2) ? 4 : 1;
  const int tid = threadIdx.x;
  const int na = ncart(la), nb = ncart(lb), ncc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb, ncd = ncc * nd;
  const int dK = (TYPE == 2) ? 1 : 0;
  const int Lb = la + lb + 2, Lk = lc + ld + 2 * dK, L = Lb + Lk;
  const int FL = 2 * max(la, lb) + 3, FLk = 2 * max(lc, ld) + 3;
  const RelGemmLayout Lo = rel_gemm_layout(la, lb, lc, ld, TYPE, CH, (int)sizeof(T));
  const int HB = Lo.HB, HBp = Lo.HBp, HK = Lo.HK, HR = Lo.HR, CRp = Lo.CRp;
  const FastDiv fHBp(HBp), fCRp(CRp), ftr(CRp / 4), fnab(nab), fnb(nb), fnd(nd);
  T* Hs = smT + Lo.oH;
  T* Rm = smT + Lo.oRm;
  T* fk = smT + Lo.oFk;
  double* Js = reinterpret_cast<double*>(smT + Lo.oJs);
  int* tuv = reinterpret_cast<int*>(smT + Lo.oTuv);
  T* Eb = smT + Lo.oEb;
  T* fa = smT + Lo.oFa;
  T* Ek = smT + Lo.oEk;
  T* Rb[2] = {smT + Lo.oR0, smT + Lo.oR1};
  T* Fs = smT + Lo.oF;
  T* Ks = smT + Lo.oK;
  T* Gs = smT + Lo.oG;
  const T* boysT = reinterpret_cast<const T*>(IS32 ? (const void*)a.boys32 : (const void*)a.boys);
  const int E1b = (la + 2) * (lb + 2) * (la + lb + 3);
  const int E1k = (lc + 1 + dK) * (ld + 1 + dK) * (lc + ld + 1 + 2 * dK);
  const ShellDev SA = a.shells[P.shA], SB = a.shells[P.shB];
  const bool dAB = P.shA == P.shB;
  const double s12d = dAB ? 1.0 : 2.0;
  const double w12 = dAB ? 0.5 : 1.0;
  const size_t nc = a.ncart;
  auto unpack = [&](int h, int& t, int& u, int& v) {
    const int w = tuv[h];
    t = w & 255;
    u = (w >> 8) & 255;
    v = w >> 16;
  };

  // ---- bra phase, once per block: E tables, axis factors, H
  const PrimPairDev& A = a.pp[P.pp_off];
  double ea, eb;
  pair_exps(SA, SB, a.prim, A, ea, eb);
  if (tid < 3)
    hermite_E_rt<T, LMAX + 1>(la + 1, lb + 1, T(A.o2p), T(A.PA[tid]), T(A.PB[tid]),
                              Eb + tid * E1b);
  for (int h = tid; h < Lo.NT; h += RG_THREADS) {
    int t, u, v;
    hinv(h, t, u, v);
    tuv[h] = t | (u << 8) | (v << 16);
  }
  for (int e = tid; e < 4 * CH; e += RG_THREADS) Js[e] = 0.0;
  __syncthreads();
  for (int it = tid; it < 3 * (la + 1) * (lb + 1) * 4; it += RG_THREADS) {
    const int ty = it % 4, jb = (it / 4) % (lb + 1), ia = (it / 4 / (lb + 1)) % (la + 1),
              x = it / 4 / (lb + 1) / (la + 1);
    axis_factor<T>(Eb + x * E1b, lb + 1, la + lb + 3, ia, jb, ty, T(2.0 * ea), T(2.0 * eb),
                   fa + (size_t)it * FL);
  }
  __syncthreads();
  auto faOf = [&](int x, int i, int j, int ty) {
    return fa + (size_t)(((x * (la + 1) + i) * (lb + 1) + j) * 4 + ty) * FL;
  };
  for (int e = tid; e < HB * HR; e += RG_THREADS) {
    const int h = e / HR, row = e % HR, ab = row / 4, op = row % 4;
    const int ai = ab / nb, bi = ab % nb;
    int t, u, v;
    unpack(h, t, u, v);
    const int ax[3] = {cart_lx(la, ai), cart_ly(la, ai), cart_lz(la, ai)};
    const int bx[3] = {cart_lx(lb, bi), cart_ly(lb, bi), cart_lz(lb, bi)};
    T val = T(0);
    for (int mu = 0; mu < 3; mu++)
      for (int nu = 0; nu < 3; nu++) {
        int o2;
        double sg;
        op_of(mu, nu, o2, sg);
        if (o2 != op) continue;
        const int tx = (mu == 0) | ((nu == 0) << 1), ty = (mu == 1) | ((nu == 1) << 1),
                  tz = (mu == 2) | ((nu == 2) << 1);
        if (t >= ax[0] + bx[0] + (tx & 1) + (tx >> 1) + 1 ||
            u >= ax[1] + bx[1] + (ty & 1) + (ty >> 1) + 1 ||
            v >= ax[2] + bx[2] + (tz & 1) + (tz >> 1) + 1)
          continue;
        val += T(sg) * faOf(0, ax[0], bx[0], tx)[t] * faOf(1, ax[1], bx[1], ty)[u] *
               faOf(2, ax[2], bx[2], tz)[v];
      }
    Hs[e] = val;
  }
  __syncthreads();  // H is complete; the bra scratch (Eb, fa) is free

  // ---- the block's kets, one at a time
#pragma unroll 1
  for (int jk = tile * RG_KT; jk < jkEnd; jk++) {
    const PairDev Q = a.pairs[a.ketBeg + jk];
    if (Q.npp != 1) continue;  // contracted: the block kernels (block-uniform)
    bool work, mine;
    {
      int s1, s2, s3, s4;
      double q12, q34;
      if (TYPE == 1) {
        s1 = P.s1; s2 = P.s2; s3 = Q.s1; s4 = Q.s2;
        q12 = __ldg(a.qSS + s1 + (size_t)s2 * ns);
        q34 = __ldg(a.qLL + s3 + (size_t)s4 * ns);
      } else {
        const bool pRef = P.lex >= Q.lex;
        const PairDev& R12 = pRef ? P : Q;
        const PairDev& R34 = pRef ? Q : P;
        s1 = R12.s1; s2 = R12.s2; s3 = R34.s1; s4 = R34.s2;
        q12 = __ldg(a.qSS + s1 + (size_t)s2 * ns);
        q34 = __ldg(a.qSS + s3 + (size_t)s4 * ns);
      }
      const double bound = sh_max(a.norms, s1, s2, s3, s4, ns) * q12 * q34;
      work = !a.screen || bound >= a.thresh;
      const bool lo = a.mixed && bound < a.cut &&
                      fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib),
                                    __ldg(a.pairRange + a.ketBeg + jk),
                                    la + lb + lc + ld + 2 + 2 * (TYPE == 2), 1, TYPE == 2);
      mine = work && (IS32 ? lo : !lo);
    }
    if (tid == 0) {
      if (!IS32) atomicAdd(a.counters + 0, 1ull);
      if (!IS32 && !work) atomicAdd(a.counters + 1, 1ull);
      if (mine) atomicAdd(a.counters + (IS32 ? 2 : 3), 1ull);
    }
    if (!mine) continue;  // block-uniform
    const ShellDev SC = a.shells[Q.shA], SD = a.shells[Q.shB];
    const bool dCD = Q.shA == Q.shB, samePQ = P.lex == Q.lex;
    const double w34 = dCD ? 0.5 : 1.0;
    const PrimPairDev& B = a.pp[Q.pp_off];
    double ec, ed;
    pair_exps(SC, SD, a.prim, B, ec, ed);
    const T X = T(A.P[0] - B.P[0]), Y = T(A.P[1] - B.P[1]), Z = T(A.P[2] - B.P[2]);
    const T pq = T(A.p) + T(B.p), alpha = T(A.p) * T(B.p) / pq;
    const T pref = T(PI52X2) / sqrt(pq) * T(A.Kp) * T(B.Kp);
    // Boys (one thread) and the ket E tables, then R level by level over the
    // block, indices from the table
    if (tid < 32) boys_lanes<T>(L, alpha * (X * X + Y * Y + Z * Z), Fs, boysT, tid);
    else if (tid >= 32 && tid < 35)
      hermite_E_rt<T, LMAX + 1>(lc + dK, ld + dK, T(B.o2p), T(B.PA[tid - 32]),
                                T(B.PB[tid - 32]), Ek + (tid - 32) * E1k);
    __syncthreads();
    {
      const T m2a = T(-2) * alpha;
      for (int n = L; n >= 0; n--) {
        T* cur = Rb[n & 1];
        const T* prv = Rb[(n + 1) & 1];
        const int cnt = nherm(L - n);
        for (int e = tid; e < cnt; e += RG_THREADS) {
          int t, u, v;
          unpack(e, t, u, v);
          T val;
          if (e == 0) {
            T f = T(1);
            for (int k = 0; k < n; k++) f *= m2a;
            val = f * Fs[n];
          } else if (t > 0) {
            val = X * prv[hidx(t - 1, u, v)];
            if (t > 1) val += T(t - 1) * prv[hidx(t - 2, u, v)];
          } else if (u > 0) {
            val = Y * prv[hidx(0, u - 1, v)];
            if (u > 1) val += T(u - 1) * prv[hidx(0, u - 2, v)];
          } else {
            val = Z * prv[hidx(0, 0, v - 1)];
            if (v > 1) val += T(v - 1) * prv[hidx(0, 0, v - 2)];
          }
          cur[e] = val;
        }
        __syncthreads();
      }
    }
    const T* R = Rb[0];
    for (int it = tid; it < ncd * 12; it += RG_THREADS) {
      const int cd = it / 12, x = (it % 12) / 4, ty = it % 4;
      if (TYPE == 1 && ty) continue;
      const int c = cd / nd, d = cd % nd;
      const int ci = x == 0 ? cart_lx(lc, c) : (x == 1 ? cart_ly(lc, c) : cart_lz(lc, c));
      const int di = x == 0 ? cart_lx(ld, d) : (x == 1 ? cart_ly(ld, d) : cart_lz(ld, d));
      T* f = fk + (size_t)it * FLk;
      const int n = axis_factor<T>(Ek + x * E1k, ld + dK, lc + ld + 2 * dK + 1, ci, di, ty,
                                   T(2.0 * ec), T(2.0 * ed), f);
      for (int t = 1; t < n; t += 2) f[t] = -f[t];
    }
    for (int e = tid; e < HK * HBp; e += RG_THREADS) {
      int hp, h;
      fHBp.divmod(e, hp, h);
      T val = T(0);
      if (h < HB) {
        int t, u, v, t2, u2, v2;
        unpack(h, t, u, v);
        unpack(hp, t2, u2, v2);
        val = pref * R[hidx(t + t2, u + u2, v + v2)];
      }
      Rm[e] = val;
    }
    __syncthreads();  // fk and Rm are complete; the per-ket scratch is free

    // ---- ket chunks
#pragma unroll 1
    for (int cd0 = 0; cd0 < ncd; cd0 += CH) {
      const int nch = min(CH, ncd - cd0);
      // K[h'][(cdl, b)]
      for (int e = tid; e < HK * CRp; e += RG_THREADS) {
        int hp, r;
        fCRp.divmod(e, hp, r);
        const int cdl = r / NB, b = r % NB;
        T val = T(0);
        if (cdl < nch) {
          const int cd = cd0 + cdl;
          int c, d;
          fnd.divmod(cd, c, d);
          const int ci[3] = {cart_lx(lc, c), cart_ly(lc, c), cart_lz(lc, c)};
          const int di[3] = {cart_lx(ld, d), cart_ly(ld, d), cart_lz(ld, d)};
          int t, u, v;
          unpack(hp, t, u, v);
          const T* f0 = fk + (size_t)cd * 12 * FLk;
          if (TYPE == 1) {
            if (t <= ci[0] + di[0] && u <= ci[1] + di[1] && v <= ci[2] + di[2])
              val = f0[(0 * 4) * FLk + t] * f0[(1 * 4) * FLk + u] * f0[(2 * 4) * FLk + v];
          } else {
            for (int kk = 0; kk < 3; kk++)
              for (int ll = 0; ll < 3; ll++) {
                int o2;
                double sg;
                op_of(kk, ll, o2, sg);
                if (o2 != b) continue;
                const int tx = (kk == 0) | ((ll == 0) << 1), ty = (kk == 1) | ((ll == 1) << 1),
                          tz = (kk == 2) | ((ll == 2) << 1);
                if (t >= ci[0] + di[0] + (tx & 1) + (tx >> 1) + 1 ||
                    u >= ci[1] + di[1] + (ty & 1) + (ty >> 1) + 1 ||
                    v >= ci[2] + di[2] + (tz & 1) + (tz >> 1) + 1)
                  continue;
                val += T(sg) * f0[(0 * 4 + tx) * FLk + t] * f0[(1 * 4 + ty) * FLk + u] *
                       f0[(2 * 4 + tz) * FLk + v];
              }
          }
        }
        Ks[e] = val;
      }
      __syncthreads();
      // G = K^T Rm, 4 x 4 tiles (rows of K, columns h)
      {
        const int tr = CRp / 4, th = HBp / 4;
        for (int unit = tid; unit < tr * th; unit += RG_THREADS) {
          int hq, rq;
          ftr.divmod(unit, hq, rq);
          const int r0 = rq * 4, h0 = hq * 4;
          T acc[4][4];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = T(0);
#pragma unroll 2
          for (int hp = 0; hp < HK; hp++) {
            T kv[4], mv[4];
            rg_ld4(Ks + (size_t)hp * CRp + r0, kv);
            rg_ld4(Rm + (size_t)hp * HBp + h0, mv);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
              for (int j = 0; j < 4; j++) acc[i][j] = fma(kv[i], mv[j], acc[i][j]);
          }
#pragma unroll
          for (int j = 0; j < 4; j++) {
            rg_st4(Gs + (size_t)(h0 + j) * CRp + r0, acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
          }
        }
      }
      __syncthreads();
      // M = H^T G, one 4 x 4 tile per unit, digested from registers
      {
        const int ngrp = (TYPE == 2) ? nch : (nch + 3) / 4;
        for (int unit = tid; unit < nab * ngrp; unit += RG_THREADS) {
          int grp, ab;
          fnab.divmod(unit, grp, ab);
          const int col0 = (TYPE == 2) ? grp * 4 : grp * 4;  // first column of the tile
          T acc[4][4];
#pragma unroll
          for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) acc[i][j] = T(0);
#pragma unroll 2
          for (int h = 0; h < HB; h++) {
            T hv[4], gv[4];
            rg_ld4(Hs + (size_t)h * HR + ab * 4, hv);
            rg_ld4(Gs + (size_t)h * CRp + col0, gv);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
              for (int j = 0; j < 4; j++) acc[i][j] = fma(hv[i], gv[j], acc[i][j]);
          }
          int ai, bi;
          fnb.divmod(ab, ai, bi);
          auto column = [&](int cdl) {
            int c, d;
            fnd.divmod(cd0 + cdl, c, d);
            const int gC = Q.cA + c, gD = Q.cB + d;
            RelCol col{gC, gD, dAB, dCD, samePQ, dCD ? 1.0 : 2.0, w12, samePQ ? 0.5 : 1.0, 0.0,
                       {0, 0, 0, 0}};
            if (TYPE == 1) {
              col.rhoLL = __ldg(a.Xll + 2 * ((size_t)gD + (size_t)gC * nc));
            } else {
              const size_t eDC = (size_t)gD + (size_t)gC * nc;
              col.rvDC[0] = __ldg(a.Xss[0] + 2 * eDC);
              col.rvDC[1] = -__ldg(a.Xss[1] + 2 * eDC + 1);
              col.rvDC[2] = -__ldg(a.Xss[2] + 2 * eDC + 1);
              col.rvDC[3] = -__ldg(a.Xss[3] + 2 * eDC + 1);
            }
            return col;
          };
          if (TYPE == 2) {
            double m[16];
#pragma unroll
            for (int op = 0; op < 4; op++)
#pragma unroll
              for (int b = 0; b < 4; b++) m[op * 4 + b] = (double)acc[op][b];
            double jl[4] = {0.0, 0.0, 0.0, 0.0};
            rel_digest<TYPE>(a, P, column(grp), ai, bi, m, jl);
#pragma unroll
            for (int b = 0; b < 4; b++)
              if (jl[b] != 0.0) atomicAdd(Js + grp * 4 + b, jl[b]);
          } else {
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const int cdl = grp * 4 + k;
              if (cdl >= nch) break;
              double m[4] = {(double)acc[0][k], (double)acc[1][k], (double)acc[2][k],
                             (double)acc[3][k]};
              double jl[4] = {0.0, 0.0, 0.0, 0.0};
              rel_digest<TYPE>(a, P, column(cdl), ai, bi, m, jl);
              if (jl[0] != 0.0) atomicAdd(Js + cdl * 4, jl[0]);
            }
          }
        }
      }
      __syncthreads();
      // per-column Coulomb flush (as the block kernels)
      for (int cdl = tid; cdl < nch; cdl += RG_THREADS) {
        const int cd = cd0 + cdl, c = cd / nd, d = cd % nd;
        const size_t eCD = (size_t)(Q.cA + c) + (size_t)(Q.cB + d) * nc;
        if (TYPE == 1) {
          if (Js[cdl * 4] != 0.0) atomicAdd(a.Jll + eCD, w34 * s12d * Js[cdl * 4]);
        } else if (!samePQ) {
          for (int b = 0; b < 4; b++)
            if (Js[cdl * 4 + b] != 0.0) atomicAdd(a.Jss[b] + eCD, w34 * s12d * Js[cdl * 4 + b]);
        }
        for (int b = 0; b < 4; b++) Js[cdl * 4 + b] = 0.0;
      }
      __syncthreads();
    }
  }  // kets
}

// Dynamic shared-memory limit of the block kernels (SSSS (ff|ff) takes 51 KB;
// the one LLSS layout above the limit, (ff|ff) at 165 KB, runs per thread).
constexpr size_t REL_SMEM_MAX = 160 * 1024;

// One class in one arithmetic precision: the instance in T computes the
// quartets that precision owns (every surviving one for double without the
// mixed mode; with it, double takes bound >= cut and float the rest).
template <int TYPE, typename T>
void launch_rel_prec(const RelLaunch& aIn, int la, int lb, int lc, int ld, cudaStream_t st) {
  RelLaunch a = aIn;
  a.skipSingle = 0;
  const int lmax = std::max(std::max(la, lb), std::max(lc, ld));
  if constexpr (TYPE == 2) if (lmax >= 2) {
    // single-primitive SSSS quartets of the d and f classes: the GEMM form,
    // when its layout fits; the other kernels skip them.  (LLSS quartets are
    // lighter -- one ket operator -- and the LLSS kernels, with every ket
    // component pair's Hermite sums built at once, measured faster: one Ag
    // atom 0.31 s in the GEMM form against 0.27 s for the first of them.)
    const int esz = (int)sizeof(T);
    const int CH = rel_gemm_chunk(la, lb, lc, ld, TYPE, esz);
    if (CH > 0) {
      const size_t smem = (size_t)rel_gemm_layout(la, lb, lc, ld, TYPE, CH, esz).total * esz;
      cudaFuncSetAttribute(rel_gemm_kernel<TYPE, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)RG_SMEM_MAX);
      const long long nb = (long long)a.nBra * ((a.nKet + RG_KT - 1) / RG_KT);
      const unsigned gx = (unsigned)std::min<long long>(nb, 65535);
      const unsigned gy = (unsigned)((nb + gx - 1) / gx);
      rel_gemm_kernel<TYPE, T><<<dim3(gx, gy), RG_THREADS, smem, st>>>(a, la, lb, lc, ld, CH);
      a.skipSingle = 1;
    }
  }
  const int tiles = (a.nKet + REL_THREADS - 1) / REL_THREADS;
  // split each quartet's ket components over enough threads to fill the GPU
  // (~256k threads per launch), at most one component pair per thread
  const long long quartets = (long long)a.nBra * a.nKet;
  const int ncd = ncart(lc) * ncart(ld);
  int nsplit = (int)std::min<long long>(ncd, std::max<long long>(1, (1 << 18) / quartets));
  nsplit = std::max(1, std::min(nsplit, 65535 / tiles));
  dim3 grid(a.nBra, tiles * nsplit);
  const int lm = std::max(std::max(la, lb), std::max(lc, ld));
  if (lm <= 1) {
    rel_kernel<1, TYPE, T><<<grid, REL_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit);
    return;
  }
  if constexpr (TYPE == 1) {
    // LLSS d/f classes: one block per quartet with every ket component at
    // once, when it fits in shared memory (single-primitive quartets in
    // their own instance); else per thread
    const long long nq = (long long)a.nBra * a.nKet;
    const unsigned gx = (unsigned)std::min<long long>(nq, 65535);
    const unsigned gy = (unsigned)((nq + gx - 1) / gx);
    const size_t smem1 = (size_t)llss_block_layout(la, lb, lc, ld, true).total * sizeof(double);
    if (smem1 <= REL_SMEM_MAX) {
      // always the same limit (on the current device), never one below a
      // launch still queued
      cudaFuncSetAttribute(rel_llss_single_kernel<T>,
                           cudaFuncAttributeMaxDynamicSharedMemorySize, (int)REL_SMEM_MAX);
      // ket tiles only where the launch keeps ~64 blocks per SM without them
      const int kt = (int)std::max<long long>(
          1, std::min<long long>(LS_KT, nq / (64LL * std::max(1, a.nsm))));
      const long long nb1 = (long long)a.nBra * ((a.nKet + kt - 1) / kt);
      const unsigned gx1 = (unsigned)std::min<long long>(nb1, 65535);
      const unsigned gy1 = (unsigned)((nb1 + gx1 - 1) / gx1);
      rel_llss_single_kernel<T><<<dim3(gx1, gy1), RB_THREADS, smem1, st>>>(a, la, lb, lc, ld,
                                                                           kt);
      a.skipSingle = 1;
      if (!a.contracted) return;
    }
    const size_t smem = (size_t)llss_block_layout(la, lb, lc, ld, false).total * sizeof(double);
    if (smem <= REL_SMEM_MAX) {
      cudaFuncSetAttribute(rel_llss_block_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)REL_SMEM_MAX);
      rel_llss_block_kernel<T><<<dim3(gx, gy), RB_THREADS, smem, st>>>(a, la, lb, lc, ld);
    } else if (lm == 2) {
      rel_kernel<2, TYPE, T><<<grid, REL_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit);
    } else {
      rel_kernel<3, TYPE, T><<<grid, REL_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit);
    }
  } else {
    // SSSS d and f classes: one block per quartet, intermediates in shared memory
    const RelBlockLayout Lo = rel_block_layout(la, lb, lc, ld, TYPE);
    const size_t smem = (size_t)Lo.total * sizeof(double);
    cudaFuncSetAttribute(rel_block_kernel<TYPE, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)REL_SMEM_MAX);
    const long long nq = a.same ? (long long)a.nBra * (a.nBra + 1) / 2
                                : (long long)a.nBra * a.nKet;
    const unsigned gx = (unsigned)std::min<long long>(nq, 65535);
    const unsigned gy = (unsigned)((nq + gx - 1) / gx);
    rel_block_kernel<TYPE, T><<<dim3(gx, gy), RB_THREADS, smem, st>>>(a, la, lb, lc, ld);
  }
}

template <int TYPE>
void launch_rel(const RelLaunch& a, int la, int lb, int lc, int ld, cudaStream_t st) {
  if (a.nBra == 0 || a.nKet == 0) return;
  launch_rel_prec<TYPE, double>(a, la, lb, lc, ld, st);
  if (a.mixed) launch_rel_prec<TYPE, float>(a, la, lb, lc, ld, st);
}

// ------------------------------------------------------------------ Gaunt
// The Gaunt term -alpha_1.alpha_2 / r12 (direct4C_libcint.hpp:2833-3907).
// The reference runs over unordered pairs of (differentiated, other) shell
// pairs X = (s2, s1), Y = (s3, s4) with the integrals (m d_j n | d_l k l).
// Here a thread takes an unordered quartet of unordered significant pairs
// {P, Q} (P = (A, B), Q = (C, D)) and computes, per Cartesian element, the
// 36 blocks (A B with d_j on A or B | C D with d_l on C or D) at once: the
// four (or, for P = Q, three) reference quartets {X, Y} the placements
// make, each screened on its own by shMax Q^G(X) Q^G(Y).  Per element and
// surviving quartet, in the reference's orientation (X >= Y as (deriv,
// other) shell indices), its update sites and conditions with T and, for
// the image, T^T -- the four update kinds as Pauli-algebra maps of the
// invariants t = tr T, tau (cross vector) and S' = T + T^T - t:
//   LL exchange from SS:  3 (d0 t - i d.tau),   -(i d0 tau + S' d)
//   SS exchange from LL:  3 d0 t - i d.tau,     -3 i d0 tau - S' d
//   LS Coulomb from SL (1), LS (2):  (d1_0 - d2_0) t + i (d1 + d2).tau,
//                                     i (d2_0 - d1_0) tau + (T^T - t)(d1 + d2)
//   LS exchange from SL:  d0 t - i d.tau,       i d0 tau + S' d - 4 T^T d
// LL and SS exchange are accumulated in the lower shell triangle (half
// weight on diagonal shell blocks) and completed as B + B^H by the back
// transform, the reference's "upper = conj(lower)" (:3833-3858).  FP64.
struct GauntLaunch {
  const PairDev* pairs;
  const PrimPairDev* pp;
  const ShellDev* shells;
  const double* prim;
  const double* boys;
  int braBeg, nBra, ketBeg, nKet, same;
  int screen;
  double thresh;
  const double* norms;  // max shell-block norms of the 16 exchange densities
  const double* qG;     // Gaunt Schwarz, qG[deriv + other * nshell]
  int nShell, ncart, exchange;
  const double* Xll[4];  // Cartesian complex densities: XLLM*, XSSM*, CLSM*, CSLM*, XSLM*
  const double* Xss[4];
  const double* Cls[4];
  const double* Csl[4];
  const double* Xsl[4];
  double* Kll[4];  // complex accumulators: LL / SS exchange, LS Coulomb, LS exchange
  double* Kss[4];
  double* Jls[4];
  double* Kls[4];
  int shardIdx, shardCnt;  // bra pairs p with p % shardCnt == shardIdx only
  unsigned long long* counters;
};

// bra component pairs per unit of work (the accumulator holds 36 blocks
// of each): a whole (pp) or (dd) pair, a fifth of an (ff) one
__host__ __device__ constexpr int gaunt_abch(int lm) { return lm <= 1 ? 9 : (lm == 2 ? 36 : 20); }

struct GInv {
  double T[3][3], t, tau[3], S[3][3];
};
__device__ __forceinline__ void gaunt_inv(const double* v, bool tr, GInv& g) {
#pragma unroll
  for (int j = 0; j < 3; j++)
#pragma unroll
    for (int l = 0; l < 3; l++) g.T[j][l] = tr ? v[3 * l + j] : v[3 * j + l];
  g.t = g.T[0][0] + g.T[1][1] + g.T[2][2];
  g.tau[0] = g.T[1][2] - g.T[2][1];
  g.tau[1] = g.T[2][0] - g.T[0][2];
  g.tau[2] = g.T[0][1] - g.T[1][0];
#pragma unroll
  for (int j = 0; j < 3; j++)
#pragma unroll
    for (int l = 0; l < 3; l++) g.S[j][l] = g.T[j][l] + g.T[l][j] - (j == l ? g.t : 0.0);
}

struct Z4 {  // Pauli components (s, x, y, z), complex
  double2 c[4];
};
__device__ __forceinline__ Z4 ld4(const double* const* X, size_t e) {
  return Z4{{ldz(X[0], e), ldz(X[1], e), ldz(X[2], e), ldz(X[3], e)}};
}
__device__ __forceinline__ void add4(double* const* A, size_t e, const Z4& v, double w) {
#pragma unroll
  for (int k = 0; k < 4; k++) addz(A[k], e, v.c[k], w);
}
__device__ __forceinline__ double2 cscale(double2 a, double f) {
  return make_double2(a.x * f, a.y * f);
}
// sum_x w[x] d_x over the vector part
__device__ __forceinline__ double2 vdot(const Z4& d, const double* w) {
  return make_double2(d.c[1].x * w[0] + d.c[2].x * w[1] + d.c[3].x * w[2],
                      d.c[1].y * w[0] + d.c[2].y * w[1] + d.c[3].y * w[2]);
}
// sum_y M[x][y] d_y (trans: M[y][x])
__device__ __forceinline__ double2 vmat(const Z4& d, const double (*M)[3], int x, bool trans) {
  double2 r = make_double2(0.0, 0.0);
#pragma unroll
  for (int y = 0; y < 3; y++) {
    const double m = trans ? M[y][x] : M[x][y];
    r.x += m * d.c[1 + y].x;
    r.y += m * d.c[1 + y].y;
  }
  return r;
}

__device__ __forceinline__ Z4 gaunt_ll(const GInv& g, const Z4& d) {
  Z4 r;
  r.c[0] = cscale(csub(cscale(d.c[0], g.t), ctimes_i(vdot(d, g.tau))), 3.0);
#pragma unroll
  for (int x = 0; x < 3; x++)
    r.c[1 + x] = cscale(cadd(ctimes_i(cscale(d.c[0], g.tau[x])), vmat(d, g.S, x, false)), -1.0);
  return r;
}
__device__ __forceinline__ Z4 gaunt_ss(const GInv& g, const Z4& d) {
  Z4 r;
  r.c[0] = csub(cscale(d.c[0], 3.0 * g.t), ctimes_i(vdot(d, g.tau)));
#pragma unroll
  for (int x = 0; x < 3; x++)
    r.c[1 + x] = csub(ctimes_i(cscale(d.c[0], -3.0 * g.tau[x])), vmat(d, g.S, x, false));
  return r;
}
__device__ __forceinline__ Z4 gaunt_cls(const GInv& g, const Z4& d1, const Z4& d2) {
  Z4 e;
  e.c[0] = csub(d1.c[0], d2.c[0]);
#pragma unroll
  for (int x = 1; x < 4; x++) e.c[x] = cadd(d1.c[x], d2.c[x]);
  Z4 r;
  r.c[0] = cadd(cscale(e.c[0], g.t), ctimes_i(vdot(e, g.tau)));
#pragma unroll
  for (int x = 0; x < 3; x++)
    r.c[1 + x] = cadd(ctimes_i(cscale(e.c[0], -g.tau[x])),
                      csub(vmat(e, g.T, x, true), cscale(e.c[1 + x], g.t)));
  return r;
}
__device__ __forceinline__ Z4 gaunt_xls(const GInv& g, const Z4& d) {
  Z4 r;
  r.c[0] = csub(cscale(d.c[0], g.t), ctimes_i(vdot(d, g.tau)));
#pragma unroll
  for (int x = 0; x < 3; x++)
    r.c[1 + x] = cadd(ctimes_i(cscale(d.c[0], g.tau[x])),
                      csub(vmat(d, g.S, x, false), cscale(vmat(d, g.T, x, true), 4.0)));
  return r;
}

// The update sites of one reference quartet (s1 s2 | s3 s4) at element
// (m1 m2 | m3 m4) (Cartesian AO indices), T = v (row: the s2 direction).
__device__ __forceinline__ void gaunt_sites(const GauntLaunch& a, const double* v, int s1, int s2,
                                            int s3, int s4, int m1, int m2, int m3, int m4) {
  const size_t nc = a.ncart;
  auto ix = [nc](int r, int c) -> size_t { return (size_t)r + (size_t)c * nc; };
  GInv T, Tt;
  gaunt_inv(v, false, T);
  gaunt_inv(v, true, Tt);
  const bool img = (s1 != s4) || (s2 != s3);
  if (a.exchange) {
    const double w14 = (s1 == s4) ? 0.5 : 1.0, w23 = (s2 == s3) ? 0.5 : 1.0;
    if (s1 >= s4) add4(a.Kll, ix(m1, m4), gaunt_ll(T, ld4(a.Xss, ix(m2, m3))), w14);
    if (s1 < s4 || (s1 == s4 && s2 != s3))
      add4(a.Kll, ix(m4, m1), gaunt_ll(Tt, ld4(a.Xss, ix(m3, m2))), w14);
    add4(a.Kss, ix(m2, m3), gaunt_ss(Tt, ld4(a.Xll, ix(m1, m4))), w23);
    if (s1 != s4 && s2 == s3) add4(a.Kss, ix(m3, m2), gaunt_ss(T, ld4(a.Xll, ix(m4, m1))), 0.5);
  }
  add4(a.Jls, ix(m1, m2), gaunt_cls(T, ld4(a.Csl, ix(m3, m4)), ld4(a.Cls, ix(m4, m3))), 1.0);
  if (img)
    add4(a.Jls, ix(m4, m3), gaunt_cls(Tt, ld4(a.Csl, ix(m2, m1)), ld4(a.Cls, ix(m1, m2))), 1.0);
  if (a.exchange) {
    add4(a.Kls, ix(m1, m3), gaunt_xls(T, ld4(a.Xsl, ix(m2, m4))), 1.0);
    if (img) add4(a.Kls, ix(m4, m2), gaunt_xls(Tt, ld4(a.Xsl, ix(m3, m1))), 1.0);
  }
}

// ------------------------------------------------ gauge (Breit) term
// The gauge part of the Breit interaction (direct4C_libcint.hpp:3908-5160):
// the GAUNT list, quartets and update sites with the kernel
// K_ii' = -r_i r_i' / r12^3 between the densities rho^i, rho^i' in place of
// Gaunt's -delta_ii' / r12.  Per element
//   V[i][i'][j][l] = (m d_j n | K_ii' | d_l k l)
//                  = -delta_ii' T[j][l] + (m d_j n | d_i d_i' r12 | d_l k l)
// (r_i r_i' / r^3 = delta_ii' / r - d_i d_i' r), and with
// W(M, D) = sum_jl M_jl s_j D s_l (the closed form above) the update kinds
// are, Q_ij = s_i s_j:
//   LL exchange from SS:  -sum_ii' s_i W(V^{ii'}, D) s_i'
//   SS exchange from LL:  -sum_jl  s_j W(V_{jl}, D) s_l     (M_ii' = V^{ii'}_jl)
//   LS Coulomb from SL (1), LS (2):  1/2 sum_ij Q_ij sum_i'l V^{ii'}_jl
//                                     (tr[Q_li' D2] - tr[Q_i'l D1])
//   LS exchange from SL:  sum_il s_i W(N_il, D) s_l         (N_ji' = V^{ii'}_jl)
// (for V = -delta T they are the Gaunt maps).  The image takes V with j
// and l exchanged (the kernel is even in r12 and symmetric in i, i').
struct GVd {
  double v[3][3][3][3];  // [i][i'][j][l]
};
__device__ __forceinline__ Q4 qunit(int a) {  // sigma_a
  Q4 r{make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  if (a == 0) r.x = make_double2(1, 0);
  else if (a == 1) r.y = make_double2(1, 0);
  else r.z = make_double2(1, 0);
  return r;
}
__device__ __forceinline__ void zacc(Z4& a, const Q4& b, double f) {
  a.c[0] = cadd(a.c[0], cscale(b.s, f));
  a.c[1] = cadd(a.c[1], cscale(b.x, f));
  a.c[2] = cadd(a.c[2], cscale(b.y, f));
  a.c[3] = cadd(a.c[3], cscale(b.z, f));
}
// W(M, D) = sum_jl M_jl s_j D s_l = d0 t - i d.tau + (i d0 tau + S' d).s
__device__ __forceinline__ Q4 w_map(const double (*M)[3], const Z4& d) {
  GInv g;
  double v[9];
#pragma unroll
  for (int k = 0; k < 9; k++) v[k] = M[k / 3][k % 3];
  gaunt_inv(v, false, g);
  Q4 r;
  r.s = csub(cscale(d.c[0], g.t), ctimes_i(vdot(d, g.tau)));
  double2 w[3];
#pragma unroll
  for (int x = 0; x < 3; x++) w[x] = cadd(ctimes_i(cscale(d.c[0], g.tau[x])), vmat(d, g.S, x, false));
  r.x = w[0];
  r.y = w[1];
  r.z = w[2];
  return r;
}
__device__ Z4 gauge_ll(const GVd& V, const Z4& d) {
  Z4 r{{make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)}};
#pragma unroll 1
  for (int i = 0; i < 3; i++)
#pragma unroll 1
    for (int ip = 0; ip < 3; ip++)
      zacc(r, qmul(qmul(qunit(i), w_map(V.v[i][ip], d)), qunit(ip)), -1.0);
  return r;
}
__device__ Z4 gauge_ss(const GVd& V, const Z4& d) {
  Z4 r{{make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)}};
#pragma unroll 1
  for (int j = 0; j < 3; j++)
#pragma unroll 1
    for (int l = 0; l < 3; l++) {
      double M[3][3];
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int ip = 0; ip < 3; ip++) M[i][ip] = V.v[i][ip][j][l];
      zacc(r, qmul(qmul(qunit(j), w_map(M, d)), qunit(l)), -1.0);
    }
  return r;
}
__device__ Z4 gauge_xls(const GVd& V, const Z4& d) {
  Z4 r{{make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)}};
#pragma unroll 1
  for (int i = 0; i < 3; i++)
#pragma unroll 1
    for (int l = 0; l < 3; l++) {
      double M[3][3];
#pragma unroll
      for (int j = 0; j < 3; j++)
#pragma unroll
        for (int ip = 0; ip < 3; ip++) M[j][ip] = V.v[i][ip][j][l];
      zacc(r, qmul(qmul(qunit(i), w_map(M, d)), qunit(l)), 1.0);
    }
  return r;
}
// tr[s_a s_b D] = 2 (delta_ab d0 + i eps_abm d_m)
__device__ __forceinline__ double2 tr_qq(int a, int b, const Z4& d) {
  if (a == b) return cscale(d.c[0], 2.0);
  const int m = 3 - a - b;
  const double e = (b == (a + 1) % 3) ? 2.0 : -2.0;
  return ctimes_i(cscale(d.c[1 + m], e));
}
__device__ Z4 gauge_cls(const GVd& V, const Z4& d1, const Z4& d2) {
  double2 sv[3][3];  // [l][i']
#pragma unroll 1
  for (int l = 0; l < 3; l++)
#pragma unroll 1
    for (int ip = 0; ip < 3; ip++) sv[l][ip] = csub(tr_qq(l, ip, d2), tr_qq(ip, l, d1));
  Z4 r{{make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)}};
#pragma unroll 1
  for (int i = 0; i < 3; i++)
#pragma unroll 1
    for (int j = 0; j < 3; j++) {
      double2 c = make_double2(0, 0);
#pragma unroll
      for (int ip = 0; ip < 3; ip++)
#pragma unroll
        for (int l = 0; l < 3; l++) c = cadd(c, cscale(sv[l][ip], V.v[i][ip][j][l]));
      c = cscale(c, 0.5);
      // Q_ij = delta_ij + i eps_ijm s_m
      if (i == j) r.c[0] = cadd(r.c[0], c);
      else {
        const int m = 3 - i - j;
        const double e = (j == (i + 1) % 3) ? 1.0 : -1.0;
        r.c[1 + m] = cadd(r.c[1 + m], ctimes_i(cscale(c, e)));
      }
    }
  return r;
}

// The gauge update sites of one reference quartet at one element (as
// gaunt_sites), V and its image Vt.
__device__ void gauge_sites(const GauntLaunch& a, const GVd& V, const GVd& Vt, int s1, int s2,
                            int s3, int s4, int m1, int m2, int m3, int m4) {
  const size_t nc = a.ncart;
  auto ix = [nc](int r, int c) -> size_t { return (size_t)r + (size_t)c * nc; };
  const bool img = (s1 != s4) || (s2 != s3);
  if (a.exchange) {
    const double w14 = (s1 == s4) ? 0.5 : 1.0, w23 = (s2 == s3) ? 0.5 : 1.0;
    if (s1 >= s4) add4(a.Kll, ix(m1, m4), gauge_ll(V, ld4(a.Xss, ix(m2, m3))), w14);
    if (s1 < s4 || (s1 == s4 && s2 != s3))
      add4(a.Kll, ix(m4, m1), gauge_ll(Vt, ld4(a.Xss, ix(m3, m2))), w14);
    add4(a.Kss, ix(m2, m3), gauge_ss(V, ld4(a.Xll, ix(m1, m4))), w23);
    if (s1 != s4 && s2 == s3) add4(a.Kss, ix(m3, m2), gauge_ss(Vt, ld4(a.Xll, ix(m4, m1))), 0.5);
  }
  add4(a.Jls, ix(m1, m2), gauge_cls(V, ld4(a.Csl, ix(m3, m4)), ld4(a.Cls, ix(m4, m3))), 1.0);
  if (img)
    add4(a.Jls, ix(m4, m3), gauge_cls(Vt, ld4(a.Csl, ix(m2, m1)), ld4(a.Cls, ix(m1, m2))), 1.0);
  if (a.exchange) {
    add4(a.Kls, ix(m1, m3), gauge_xls(V, ld4(a.Xsl, ix(m2, m4))), 1.0);
    if (img) add4(a.Kls, ix(m4, m2), gauge_xls(Vt, ld4(a.Xsl, ix(m3, m1))), 1.0);
  }
}

// bra component pairs per unit of work of the gauge kernel (its
// accumulator holds 7 x 36 blocks of each)
__host__ __device__ constexpr int gauge_abch(int lm) { return lm <= 2 ? 9 : 4; }

// One thread per (quartet {P, Q}, unit); units = ket component pairs (c, d)
// x slices of bra component pairs, split over nsplit threads.  GAUNT: one
// operator, 1 / r12.  GAUGE: seven -- 1 / r12 and d_i d_i' r12 for the six
// pairs i <= i' -- each a pass over the primitive pairs (the r12 passes on
// the auxiliary functions of r12_aux, the Hermite index shifted by
// e_i + e_i').
template <int LM, bool GAUGE>
__global__ void __launch_bounds__(REL_THREADS)
    gaunt_kernel(const GauntLaunch a, int la, int lb, int lc, int ld, int nsplit, int nslice) {
  const int ib = blockIdx.x;
  if (!in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) return;  // another shard's bra
  const int split = blockIdx.y % nsplit;
  const int jk = (blockIdx.y / nsplit) * REL_THREADS + threadIdx.x;
  const int ns = a.nShell;
  const bool visited = jk < a.nKet && !(a.same && jk > ib);
  const PairDev P = a.pairs[a.braBeg + ib];
  PairDev Q = P;
  unsigned alive = 0;  // bit 2 pb + pk: derivative on B (pb) / D (pk)
  if (visited) {
    Q = a.pairs[a.ketBeg + jk];
    const double shMax = sh_max(a.norms, P.s1, P.s2, Q.s1, Q.s2, ns);
    const bool samePQ = P.lex == Q.lex;
#pragma unroll
    for (int pb = 0; pb < 2; pb++)
#pragma unroll
      for (int pk = 0; pk < 2; pk++) {
        if ((pb && P.shA == P.shB) || (pk && Q.shA == Q.shB) || (samePQ && pb > pk)) continue;
        const int xd = pb ? P.shB : P.shA, xo = pb ? P.shA : P.shB;
        const int yd = pk ? Q.shB : Q.shA, yo = pk ? Q.shA : Q.shB;
        const double bound = shMax * __ldg(a.qG + xd + (size_t)xo * ns) *
                             __ldg(a.qG + yd + (size_t)yo * ns);
        if (!a.screen || bound >= a.thresh) alive |= 1u << (2 * pb + pk);
      }
  }
  if (split == 0) {
    const unsigned mask = __activemask();
    const unsigned bv = __ballot_sync(mask, visited), bw = __ballot_sync(mask, alive != 0);
    if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) {
      if (bv) atomicAdd(a.counters + 0, (unsigned long long)__popc(bv));
      if (bv & ~bw) atomicAdd(a.counters + 1, (unsigned long long)__popc(bv & ~bw));
      if (bw) atomicAdd(a.counters + 3, (unsigned long long)__popc(bw));
    }
  }
  if (!alive) return;

  constexpr int NOP = GAUGE ? 7 : 1;
  constexpr int E1 = (LM + 2) * (LM + 2) * (2 * LM + 3);
  constexpr int HB = nherm(2 * LM + 1);
  constexpr int HL = nherm(4 * LM + 2 + (GAUGE ? 2 : 0));
  constexpr int FL = 2 * LM + 3;
  constexpr int ABCH = GAUGE ? gauge_abch(LM) : gaunt_abch(LM);
  const int na = ncart(la), nb = ncart(lb), ncc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb, ncd = ncc * nd;
  const ShellDev SA = a.shells[P.shA], SB = a.shells[P.shB];
  const ShellDev SC = a.shells[Q.shA], SD = a.shells[Q.shB];
  const int Lb = la + lb + 1, Lk = lc + ld + 1;
  // which placements some surviving quartet needs
  const bool needB[2] = {(alive & 3u) != 0, (alive & 12u) != 0};
  const bool needK[2] = {(alive & 5u) != 0, (alive & 10u) != 0};

  double Ea[3][E1], Ec[3][E1];
  double G[6][HB];  // [pk * 3 + l]
  double Rv[HL];
  double F[4 * LM + 5];
  double acc[ABCH * NOP * 36];
  double fa[3][3][FL], fc[3][3][FL];
  int nfa[3][3], nfc[3][3];

#pragma unroll 1
  for (int u = split; u < ncd * nslice; u += nsplit) {
    const int cd = u / nslice, sl = u % nslice;
    const int ab0 = sl * ABCH, ab1 = min(nab, ab0 + ABCH);
    if (ab0 >= ab1) continue;
    const int c = cd / nd, d = cd % nd;
    const int ci[3] = {cart_lx(lc, c), cart_ly(lc, c), cart_lz(lc, c)};
    const int di[3] = {cart_lx(ld, d), cart_ly(ld, d), cart_lz(ld, d)};
#pragma unroll 1
    for (int k = 0; k < (ab1 - ab0) * NOP * 36; k++) acc[k] = 0.0;
#pragma unroll 1
    for (int op = 0; op < NOP; op++) {
      int oi = -1, oj = -1;
      if (op > 0) op_pair(op - 1, oi, oj);
      const int sx = (oi == 0) + (oj == 0), sy = (oi == 1) + (oj == 1), sz = (oi == 2) + (oj == 2);
      const int L = Lb + Lk + (op > 0 ? 2 : 0);
#pragma unroll 1
      for (int ip = 0; ip < P.npp; ip++) {
        const PrimPairDev& A = a.pp[P.pp_off + ip];
        double ea, eb;
        pair_exps(SA, SB, a.prim, A, ea, eb);
#pragma unroll 1
        for (int x = 0; x < 3; x++)
          hermite_E_rt<double, LM + 1>(la + 1, lb + 1, A.o2p, A.PA[x], A.PB[x], Ea[x]);
#pragma unroll 1
        for (int k = 0; k < 6; k++)
#pragma unroll 1
          for (int h = 0; h < nherm(Lb); h++) G[k][h] = 0.0;
#pragma unroll 1
        for (int iq = 0; iq < Q.npp; iq++) {
          const PrimPairDev& Bq = a.pp[Q.pp_off + iq];
          double ec, ed;
          pair_exps(SC, SD, a.prim, Bq, ec, ed);
#pragma unroll 1
          for (int x = 0; x < 3; x++)
            hermite_E_rt<double, LM + 1>(lc + 1, ld + 1, Bq.o2p, Bq.PA[x], Bq.PB[x], Ec[x]);
          const double X = A.P[0] - Bq.P[0], Y = A.P[1] - Bq.P[1], Z = A.P[2] - Bq.P[2];
          const double pq = A.p + Bq.p, alpha = A.p * Bq.p / pq;
          double pref = PI52X2 / sqrt(pq) * A.Kp * Bq.Kp;
          const double Targ = alpha * (X * X + Y * Y + Z * Z);
          boys_rt<double>(L, Targ, F, a.boys);
          if (op > 0) {
            r12_aux(L, Targ, F);
            pref /= 2.0 * alpha;
          }
          hermite_R_rt<double>(L, alpha, X, Y, Z, F, Rv);
#pragma unroll 1
          for (int x = 0; x < 3; x++)
#pragma unroll 1
            for (int ty = 0; ty < 3; ty++) {
              if (ty > 0 && !needK[ty - 1]) continue;
              nfc[x][ty] = axis_factor<double>(Ec[x], ld + 1, lc + ld + 3, ci[x], di[x], ty,
                                               2.0 * ec, 2.0 * ed, fc[x][ty]);
#pragma unroll 1
              for (int t = 1; t < nfc[x][ty]; t += 2) fc[x][ty][t] = -fc[x][ty][t];
            }
#pragma unroll 1
          for (int pk = 0; pk < 2; pk++) {
            if (!needK[pk]) continue;
#pragma unroll 1
            for (int l = 0; l < 3; l++) {
              const int tx = (l == 0) ? 1 + pk : 0, ty = (l == 1) ? 1 + pk : 0,
                        tz = (l == 2) ? 1 + pk : 0;
              ket_add<double>(G[pk * 3 + l], pref, fc[0][tx], nfc[0][tx], fc[1][ty],
                              nfc[1][ty], fc[2][tz], nfc[2][tz], Lb, Rv, sx, sy, sz);
            }
          }
        }
#pragma unroll 1
        for (int ab = ab0; ab < ab1; ab++) {
          const int ai = ab / nb, bi = ab % nb;
          const int ax[3] = {cart_lx(la, ai), cart_ly(la, ai), cart_lz(la, ai)};
          const int bx[3] = {cart_lx(lb, bi), cart_ly(lb, bi), cart_lz(lb, bi)};
#pragma unroll 1
          for (int x = 0; x < 3; x++)
#pragma unroll 1
            for (int ty = 0; ty < 3; ty++) {
              if (ty > 0 && !needB[ty - 1]) continue;
              nfa[x][ty] = axis_factor<double>(Ea[x], lb + 1, la + lb + 3, ax[x], bx[x], ty,
                                               2.0 * ea, 2.0 * eb, fa[x][ty]);
            }
          double* m = acc + ((ab - ab0) * NOP + op) * 36;
#pragma unroll 1
          for (int pb = 0; pb < 2; pb++) {
            if (!needB[pb]) continue;
#pragma unroll 1
            for (int j = 0; j < 3; j++) {
              const int tx = (j == 0) ? 1 + pb : 0, ty = (j == 1) ? 1 + pb : 0,
                        tz = (j == 2) ? 1 + pb : 0;
#pragma unroll 1
              for (int pk = 0; pk < 2; pk++) {
                if (!(alive & (1u << (2 * pb + pk)))) continue;
#pragma unroll 1
                for (int l = 0; l < 3; l++)
                  m[((pb * 3 + j) * 2 + pk) * 3 + l] +=
                      bra_dot<double>(fa[0][tx], nfa[0][tx], fa[1][ty], nfa[1][ty], fa[2][tz],
                                      nfa[2][tz], G[pk * 3 + l]);
              }
            }
          }
        }
      }
    }
    // digestion: every surviving reference quartet of every element
    const int gC = Q.cA + c, gD = Q.cB + d;
#pragma unroll 1
    for (int ab = ab0; ab < ab1; ab++) {
      const int gA = P.cA + ab / nb, gB = P.cB + ab % nb;
      const double* m = acc + (ab - ab0) * NOP * 36;
#pragma unroll 1
      for (int pb = 0; pb < 2; pb++)
#pragma unroll 1
        for (int pk = 0; pk < 2; pk++) {
          if (!(alive & (1u << (2 * pb + pk)))) continue;
          const int xd = pb ? P.shB : P.shA, xo = pb ? P.shA : P.shB;
          const int yd = pk ? Q.shB : Q.shA, yo = pk ? Q.shA : Q.shB;
          const int xdA = pb ? gB : gA, xoA = pb ? gA : gB;
          const int ydA = pk ? gD : gC, yoA = pk ? gC : gD;
          const bool xb = xd > yd || (xd == yd && xo >= yo);
          // the reference's orientation: bra X (j on X) or Y (j on Y)
          auto comp = [&](int o, int j, int l) -> double {
            return xb ? m[o * 36 + ((pb * 3 + j) * 2 + pk) * 3 + l]
                      : m[o * 36 + ((pb * 3 + l) * 2 + pk) * 3 + j];
          };
          if (!GAUGE) {
            double v[9];
#pragma unroll
            for (int j = 0; j < 3; j++)
#pragma unroll
              for (int l = 0; l < 3; l++) v[3 * j + l] = comp(0, j, l);
            if (xb) gaunt_sites(a, v, xo, xd, yd, yo, xoA, xdA, ydA, yoA);
            else gaunt_sites(a, v, yo, yd, xd, xo, yoA, ydA, xdA, xoA);
          } else {
            GVd V, Vt;
#pragma unroll 1
            for (int k = 0; k < 6; k++) {
              int i, ip;
              op_pair(k, i, ip);
#pragma unroll 1
              for (int j = 0; j < 3; j++)
#pragma unroll 1
                for (int l = 0; l < 3; l++) {
                  double v = comp(1 + k, j, l), vt = comp(1 + k, l, j);
                  if (i == ip) {
                    v -= comp(0, j, l);
                    vt -= comp(0, l, j);
                  }
                  V.v[i][ip][j][l] = V.v[ip][i][j][l] = v;
                  Vt.v[i][ip][j][l] = Vt.v[ip][i][j][l] = vt;
                }
            }
            if (xb) gauge_sites(a, V, Vt, xo, xd, yd, yo, xoA, xdA, ydA, yoA);
            else gauge_sites(a, V, Vt, yo, yd, xd, xo, yoA, ydA, xdA, xoA);
          }
        }
    }
  }
}

template <bool GAUGE>
void launch_gaunt(const GauntLaunch& a, int la, int lb, int lc, int ld, cudaStream_t st) {
  if (a.nBra == 0 || a.nKet == 0) return;
  const int tiles = (a.nKet + REL_THREADS - 1) / REL_THREADS;
  const int lm = std::max(std::max(la, lb), std::max(lc, ld));
  const int nab = ncart(la) * ncart(lb);
  const int abch = GAUGE ? gauge_abch(std::max(lm, 1)) : gaunt_abch(std::max(lm, 1));
  const int nslice = (nab + abch - 1) / abch;
  const long long quartets = (long long)a.nBra * a.nKet;
  const int units = ncart(lc) * ncart(ld) * nslice;
  int nsplit = (int)std::min<long long>(units, std::max<long long>(1, (1 << 18) / quartets));
  nsplit = std::max(1, std::min(nsplit, 65535 / tiles));
  dim3 grid(a.nBra, tiles * nsplit);
  if (lm <= 1)
    gaunt_kernel<1, GAUGE><<<grid, REL_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit, nslice);
  else if (lm == 2)
    gaunt_kernel<2, GAUGE><<<grid, REL_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit, nslice);
  else
    gaunt_kernel<3, GAUGE><<<grid, REL_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit, nslice);
}

// ------------------------------------------------------------ 4C Schwarz
// Q^LL(a,b) = sqrt(max |(ab|ab)|) and Q^SS(a,b) = C2 sqrt(max over the 81
// components of |(dA dB ab|dA dB ab)|), both over every element of the
// spherical quartet block (direct4C_libcint.hpp:341-481).  Every (pair,
// component) is one unit of work for a group of threads, one Cartesian ket
// column per thread (rel_schwarz_kernel).

// Cartesian column out[(a*nb + b) * stride] += w (d ab | K | d cd) of the
// ket component pair (c, d) with derivative directions dir[0..3] (-1:
// none), summed over the bra primitive pairs ip = ip0, ip0 + ipStep, ...
// (shared memory, added atomically: several threads may share a column).
// K = 1 / r12, or d_opi d_opj r12 when opi >= 0.
template <int LM>
__device__ void deriv_column(int la, int lb, int lc, int ld, int c, int d, const int* dir,
                             const PairDev& P, const PairDev& Q, const PrimPairDev* pp,
                             const ShellDev* shells, const double* prim, const double* boys,
                             double* out, int stride, int ip0, int ipStep, int opi = -1,
                             int opj = -1, double w = 1.0) {
  constexpr int E1 = (LM + 2) * (LM + 2) * (2 * LM + 3);
  constexpr int HB = nherm(2 * LM + 2);
  constexpr int HL = nherm(4 * LM + 4);
  constexpr int FL = 2 * LM + 3;
  const int na = ncart(la), nb = ncart(lb);
  const int rb = (dir[0] >= 0 || dir[1] >= 0) ? 1 : 0, rk = (dir[2] >= 0 || dir[3] >= 0) ? 1 : 0;
  const int Lb = la + lb + (dir[0] >= 0) + (dir[1] >= 0);
  const int Lk = lc + ld + (dir[2] >= 0) + (dir[3] >= 0);
  const int sh[3] = {(opi == 0) + (opj == 0), (opi == 1) + (opj == 1), (opi == 2) + (opj == 2)};
  const int L = Lb + Lk + (opi >= 0 ? 2 : 0);
  const ShellDev SA = shells[P.shA], SB = shells[P.shB], SC = shells[Q.shA], SD = shells[Q.shB];
  const int ci[3] = {cart_lx(lc, c), cart_ly(lc, c), cart_lz(lc, c)};
  const int di[3] = {cart_lx(ld, d), cart_ly(ld, d), cart_lz(ld, d)};
  double Ea[3][E1], Ec[3][E1], G[HB], Rv[HL], F[4 * LM + 5], f[3][FL], g[3][FL];
  int nf[3], ng[3];
  for (int ip = ip0; ip < P.npp; ip += ipStep) {
    const PrimPairDev& A = pp[P.pp_off + ip];
    double ea, eb;
    pair_exps(SA, SB, prim, A, ea, eb);
    for (int x = 0; x < 3; x++)
      hermite_E_rt<double, LM + 1>(la + rb, lb + rb, A.o2p, A.PA[x], A.PB[x], Ea[x]);
    for (int h = 0; h < nherm(Lb); h++) G[h] = 0.0;
    for (int iq = 0; iq < Q.npp; iq++) {
      const PrimPairDev& B = pp[Q.pp_off + iq];
      double ec, ed;
      pair_exps(SC, SD, prim, B, ec, ed);
      for (int x = 0; x < 3; x++)
        hermite_E_rt<double, LM + 1>(lc + rk, ld + rk, B.o2p, B.PA[x], B.PB[x], Ec[x]);
      const double X = A.P[0] - B.P[0], Y = A.P[1] - B.P[1], Z = A.P[2] - B.P[2];
      const double pq = A.p + B.p, alpha = A.p * B.p / pq;
      double pref = PI52X2 / sqrt(pq) * A.Kp * B.Kp;
      const double Targ = alpha * (X * X + Y * Y + Z * Z);
      boys_rt<double>(L, Targ, F, boys);
      if (opi >= 0) {
        r12_aux(L, Targ, F);
        pref /= 2.0 * alpha;
      }
      hermite_R_rt<double>(L, alpha, X, Y, Z, F, Rv);
      for (int x = 0; x < 3; x++) {
        const int ty = (dir[2] == x) | ((dir[3] == x) << 1);
        nf[x] = axis_factor(Ec[x], ld + rk, lc + ld + 2 * rk + 1, ci[x], di[x], ty, 2.0 * ec,
                            2.0 * ed, f[x]);
        for (int t = 1; t < nf[x]; t += 2) f[x][t] = -f[x][t];
      }
      ket_add(G, pref, f[0], nf[0], f[1], nf[1], f[2], nf[2], Lb, Rv, sh[0], sh[1], sh[2]);
    }
    for (int ai = 0; ai < na; ai++)
      for (int bi = 0; bi < nb; bi++) {
        const int ax[3] = {cart_lx(la, ai), cart_ly(la, ai), cart_lz(la, ai)};
        const int bx[3] = {cart_lx(lb, bi), cart_ly(lb, bi), cart_lz(lb, bi)};
        for (int x = 0; x < 3; x++) {
          const int ty = (dir[0] == x) | ((dir[1] == x) << 1);
          ng[x] = axis_factor(Ea[x], lb + rb, la + lb + 2 * rb + 1, ax[x], bx[x], ty, 2.0 * ea,
                              2.0 * eb, g[x]);
        }
        atomicAdd(out + (ai * nb + bi) * stride,
                  w * bra_dot(g[0], ng[0], g[1], ng[1], g[2], ng[2], G));
      }
  }
}

// one index of a 4-index block (row-major, index 3 fastest) from Cartesian
// to spherical: out[.. mu ..] = sum_c T[c][mu] in[.. c ..]; the gs threads
// of a group (g0 = this thread's index in it) share the work
__device__ void sph_index(const double* in, double* out, int* dims, int k, const double* T,
                          int nsk, int g0, int gs) {
  int od[4] = {dims[0], dims[1], dims[2], dims[3]};
  od[k] = nsk;
  const int tot = od[0] * od[1] * od[2] * od[3];
  for (int e = g0; e < tot; e += gs) {
    int i[4], r = e;
    for (int q = 3; q >= 0; q--) {
      i[q] = r % od[q];
      r /= od[q];
    }
    const int mu = i[k];
    double s = 0.0;
    for (int c = 0; c < dims[k]; c++) {
      const double t = T[c * nsk + mu];
      if (t == 0.0) continue;
      i[k] = c;
      s += t * in[((i[0] * dims[1] + i[1]) * dims[2] + i[2]) * dims[3] + i[3]];
    }
    out[e] = s;
  }
  dims[k] = nsk;
}

constexpr int SCH_THREADS = 128;

// One (pair, component) per group of gsize threads, SCH_THREADS / gsize
// groups per block, units enumerated pair-major over the components of a
// pair: the plain (ab|ab) block (when lowLL), the 81 blocks
// (dA_i dB_j ab | dA_k dB_l ab) (nSS = 81), the 18 Gaunt blocks
// (dA_i b | dA_k b), (a dB_i | a dB_k) (nG = 18) and the 108 gauge blocks
// (dA_j b | -r_i r_i' / r^3 | dA_l b) and the same on B (nB = 108; i <= i',
// the kernel -delta_ii' / r12 + d_i d_i' r12).  A group builds the
// Cartesian block in shared memory -- thread g0 takes ket column g0 % cpow
// (cpow: the column count rounded up to a power of two) and every
// (gsize / cpow)-th bra primitive pair from g0 / cpow -- transforms it to
// the spherical basis index by index, and folds its largest |element| into
// the pair's maximum (mx[6 pair + 0..5]: plain, SS, Gaunt on A, Gaunt on B,
// gauge on A, gauge on B) with an atomic max on the bit pattern
// (non-negative doubles order as integers).
constexpr int SCH_SLOTS = 6;
template <int LM>
__global__ void __launch_bounds__(SCH_THREADS)
    rel_schwarz_kernel(const PairDev* __restrict__ pairs, const PrimPairDev* __restrict__ pp,
                       const ShellDev* __restrict__ shells, const double* __restrict__ prim,
                       const double* __restrict__ boys, const double* __restrict__ sph,
                       const int* __restrict__ sphOff, int beg, int npair, int la, int lb,
                       int lowLL, int nSS, int nG, int nB, int gsize, int cpow,
                       unsigned long long* mx) {
  extern __shared__ double sm[];
  const int na = ncart(la), nb = ncart(lb);
  const int n4 = na * nb * na * nb;
  const int groups = SCH_THREADS / gsize;
  const int ncomp = lowLL + nSS + nG + nB;
  const int g = threadIdx.x / gsize, g0 = threadIdx.x % gsize;
  const long long unit = (long long)blockIdx.x * groups + g;
  const bool live = unit < (long long)npair * ncomp;
  const int ip = live ? (int)(unit / ncomp) : 0;
  const int comp = live ? (int)(unit % ncomp) : 0;
  const PairDev P = pairs[beg + ip];
  const ShellDev SA = shells[P.shA], SB = shells[P.shB];
  int dir[4] = {-1, -1, -1, -1};
  int slot = 0, opi = -1, opj = -1;
  if (comp >= lowLL + nSS + nG) {  // gauge: one derivative in each pair
    const int gc = comp - lowLL - nSS - nG;
    const int side = gc / 54, r = gc % 54;
    op_pair(r / 9, opi, opj);
    dir[side] = (r % 9) / 3;
    dir[2 + side] = r % 3;
    slot = 4 + side;
  } else if (comp >= lowLL + nSS) {  // Gaunt: one derivative in each pair
    const int gc = comp - lowLL - nSS;
    const int side = gc / 9;  // 0: on A, 1: on B
    dir[side] = (gc % 9) / 3;
    dir[2 + side] = gc % 3;
    slot = 2 + side;
  } else if (comp >= lowLL) {
    const int dc = comp - lowLL;  // derivative component 0..80
    dir[0] = dc / 27;
    dir[1] = (dc / 9) % 3;
    dir[2] = (dc / 3) % 3;
    dir[3] = dc % 3;
    slot = 1;
  }
  double* cur = sm + (size_t)g * 2 * n4;
  double* nxt = cur + n4;
  for (int e = g0; e < n4; e += gsize) cur[e] = 0.0;
  __syncthreads();
  const int col = g0 % cpow, slice = g0 / cpow, nslice = gsize / cpow;
  if (live && col < na * nb) {
    deriv_column<LM>(la, lb, la, lb, col / nb, col % nb, dir, P, P, pp, shells, prim, boys,
                     cur + col, na * nb, slice, nslice, opi, opj);
    if (opi >= 0 && opi == opj)  // the -delta_ii' / r12 part of the gauge kernel
      deriv_column<LM>(la, lb, la, lb, col / nb, col % nb, dir, P, P, pp, shells, prim, boys,
                       cur + col, na * nb, slice, nslice, -1, -1, -1.0);
  }
  __syncthreads();
  int dims[4] = {na, nb, na, nb};
  const ShellDev* S4[4] = {&SA, &SB, &SA, &SB};
  for (int k = 0; k < 4; k++) {  // every thread reaches each barrier
    const ShellDev& S = *S4[k];
    if (live && S.pure) {
      sph_index(cur, nxt, dims, k, sph + sphOff[S.l], nsph(S.l), g0, gsize);
      double* t = cur;
      cur = nxt;
      nxt = t;
    }
    __syncthreads();
  }
  if (!live) return;
  double m = 0.0;
  const int tot = dims[0] * dims[1] * dims[2] * dims[3];
  for (int e = g0; e < tot; e += gsize) m = fmax(m, fabs(cur[e]));
  if (m > 0.0)
    atomicMax(mx + SCH_SLOTS * (size_t)ip + slot, (unsigned long long)__double_as_longlong(m));
}

// Q^LL = sqrt(max), Q^SS = C2 sqrt(max) of each pair of a class into both
// triangles of the nshell x nshell tables (direct4C_libcint.hpp:388-394,
// :464-470); Q^G(d, o) = C1 sqrt(max) with the derivative on shell d
// (SchwarzGaunt, :2910-2955, C1 = 1 / 2c), not symmetric; the same for the
// gauge kernel, Q^B(d, o) (SchwarzGauge, :3960-4005, which maxes over
// libcint's 16 spin components of the operator where this maxes over its
// 81 spatial components).
__global__ void rel_schwarz_finish_kernel(const PairDev* __restrict__ pairs, int beg, int npair,
                                          const unsigned long long* __restrict__ mx,
                                          int needLL, int needSS, int needG, int needB,
                                          int nshell, double* qLL, double* qSS, double* qG,
                                          double* qB) {
  const int ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= npair) return;
  const PairDev P = pairs[beg + ip];
  const size_t e1 = P.s1 + (size_t)P.s2 * nshell, e2 = P.s2 + (size_t)P.s1 * nshell;
  auto v = [&](int k) {
    return sqrt(__longlong_as_double((long long)mx[SCH_SLOTS * ip + k]));
  };
  if (needLL) qLL[e1] = qLL[e2] = v(0);
  if (needSS) {
    const double C2 = 1.0 / (4.0 * SPEED_OF_LIGHT * SPEED_OF_LIGHT);
    qSS[e1] = qSS[e2] = C2 * v(1);
  }
  if (needG) {
    const double C1 = 1.0 / (2.0 * SPEED_OF_LIGHT);
    qG[P.shA + (size_t)P.shB * nshell] = C1 * v(2);
    qG[P.shB + (size_t)P.shA * nshell] = C1 * v(3);
  }
  if (needB) {
    const double C1 = 1.0 / (2.0 * SPEED_OF_LIGHT);
    qB[P.shA + (size_t)P.shB * nshell] = C1 * v(4);
    qB[P.shB + (size_t)P.shA * nshell] = C1 * v(5);
  }
}

cqf_status ensure_rel_schwarz(cqf_basis* B, bool needLL, bool needSS, bool needG,
                              bool needB, cudaStream_t st) {
  needLL = needLL && !B->rel_qLL;
  needSS = needSS && !B->rel_qSS;
  needG = needG && !B->rel_qG;
  needB = needB && !B->rel_qB;
  if (!needLL && !needSS && !needG && !needB) return CQF_OK;
  const size_t ns2 = (size_t)B->nshell * B->nshell;
  // basis-owned, stream-ordered on the basis' stream (freed by free_basis)
  for (double** q : {&B->d_qLL, &B->d_qSS, &B->d_qG, &B->d_qB})
    if (!*q) {
      CQF_RCUDA(cudaMallocAsync(q, ns2 * sizeof(double), B->stream));
      CQF_RCUDA(cudaMemsetAsync(*q, 0, ns2 * sizeof(double), B->stream));
    }
  CQF_RCUDA(cudaStreamSynchronize(B->stream));
  unsigned long long* mx = nullptr;
  const size_t mxn = SCH_SLOTS * (size_t)std::max(1, B->npair);
  CQF_RCUDA(cudaMallocAsync(&mx, mxn * sizeof(unsigned long long), st));
  CQF_RCUDA(cudaMemsetAsync(mx, 0, mxn * sizeof(unsigned long long), st));
  const int nSS = needSS ? 81 : 0, nG = needG ? 18 : 0, nB = needB ? 108 : 0;
  const int ncomp = (needLL ? 1 : 0) + nSS + nG + nB;
  for (int c = 0; c < NCLS; c++) {
    if (B->cls_cnt[c] <= 0) continue;
    int la, lb;
    class_ls(c, la, lb);
    const int n4 = ncart(la) * ncart(lb) * ncart(la) * ncart(lb);
    // threads per (pair, component): at least a warp, and the Cartesian
    // column count rounded up to a power of two (the spare threads split the
    // bra primitive pairs)
    int cpow = 1;
    while (cpow < ncart(la) * ncart(lb)) cpow *= 2;
    const int gsize = std::min(SCH_THREADS, std::max(32, cpow));
    const int groups = SCH_THREADS / gsize;
    const size_t smem = (size_t)groups * 2 * n4 * sizeof(double);
    const long long units = (long long)B->cls_cnt[c] * ncomp;
    const unsigned nblk = (unsigned)((units + groups - 1) / groups);
    unsigned long long* mxc = mx + SCH_SLOTS * (size_t)B->cls_beg[c];
    const int lm = std::max(la, 1);
#define CQF_SCH(LMV)                                                                          \
  if (lm == LMV) {                                                                            \
    CQF_RCUDA(cudaFuncSetAttribute(rel_schwarz_kernel<LMV>,                                   \
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));  \
    rel_schwarz_kernel<LMV><<<nblk, SCH_THREADS, smem, st>>>(                                 \
        B->d_pairs, B->d_pp, B->d_shells, B->d_prim, B->d_boys64, B->d_sph, B->d_sphOff,      \
        B->cls_beg[c], B->cls_cnt[c], la, lb, needLL ? 1 : 0, nSS, nG, nB, gsize, cpow, mxc); \
  }
    CQF_SCH(1)
    CQF_SCH(2)
    CQF_SCH(3)
#undef CQF_SCH
    rel_schwarz_finish_kernel<<<(B->cls_cnt[c] + 127) / 128, 128, 0, st>>>(
        B->d_pairs, B->cls_beg[c], B->cls_cnt[c], mxc, needLL, needSS, needG, needB,
        B->nshell, B->d_qLL, B->d_qSS, B->d_qG, B->d_qB);
    CQF_RCUDA(cudaGetLastError());
  }
  cudaFreeAsync(mx, st);
  CQF_RCUDA(cudaStreamSynchronize(st));
  B->rel_qLL = B->rel_qLL || needLL;
  B->rel_qSS = B->rel_qSS || needSS;
  B->rel_qG = B->rel_qG || needG;
  B->rel_qB = B->rel_qB || needB;
  return CQF_OK;
}

// ---------------------------------------------------------- back transform
// AX (complex N x N, assigned) from a Cartesian accumulator, B = T^T Ac T:
//   mode 0: B (complex)             mode 1: B + B^T (real Ac)
//   mode 2: i (B - B^T) (real Ac)   mode 3: B + B^H (complex)
__global__ void rel_from_cart_kernel(const double* __restrict__ Ac, int mode, int N, int nc,
                                     const ShellDev* __restrict__ sh,
                                     const int* __restrict__ ao2s,
                                     const double* __restrict__ sph,
                                     const int* __restrict__ sphOff, double* AX) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= (size_t)N * N) return;
  const int i = (int)(k % N), j = (int)(k / N);
  const bool cplx = (mode == 0 || mode == 3);
  auto bval = [&](int r, int c, double& bre, double& bim) {
    const ShellDev A = sh[ao2s[r]], B = sh[ao2s[c]];
    const int mu = r - A.sph_off, nu = c - B.sph_off;
    const double* TA = sph + sphOff[A.l];
    const double* TB = sph + sphOff[B.l];
    bre = 0.0;
    bim = 0.0;
    for (int a = 0; a < ncart(A.l); a++) {
      const double ta = A.pure ? TA[a * nsph(A.l) + mu] : (a == mu);
      if (ta == 0.0) continue;
      for (int b = 0; b < ncart(B.l); b++) {
        const double tb = B.pure ? TB[b * nsph(B.l) + nu] : (b == nu);
        if (tb == 0.0) continue;
        const size_t e = (size_t)(A.cart_off + a) + (size_t)(B.cart_off + b) * nc;
        if (cplx) {
          bre += ta * tb * Ac[2 * e];
          bim += ta * tb * Ac[2 * e + 1];
        } else {
          bre += ta * tb * Ac[e];
        }
      }
    }
  };
  double r1, i1, r2 = 0.0, i2 = 0.0;
  bval(i, j, r1, i1);
  if (mode != 0) bval(j, i, r2, i2);
  double outr, outi;
  if (mode == 0) { outr = r1; outi = i1; }
  else if (mode == 1) { outr = r1 + r2; outi = 0.0; }
  else if (mode == 2) { outr = 0.0; outi = r1 - r2; }
  else { outr = r1 + r2; outi = i1 - i2; }
  AX[2 * k] = outr;
  AX[2 * k + 1] = outi;
}

// imaginary part set to zero (the Coulomb density of the bare term)
__global__ void real_part_kernel(const double* __restrict__ X, size_t n, double* Y) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  Y[2 * k] = X[2 * k];
  Y[2 * k + 1] = 0.0;
}

// ------------------------------------------------------ 4C assembly kernels
// blk(i, j) = D(ro + i, co + j), N x N out of 2N x 2N
__global__ void get_block_kernel(const double* __restrict__ D, int N, int ro, int co,
                                 double* blk) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= (size_t)N * N) return;
  const int i = (int)(k % N), j = (int)(k / N);
  const size_t e = (size_t)(ro + i) + (size_t)(co + j) * 2 * N;
  blk[2 * k] = D[2 * e];
  blk[2 * k + 1] = D[2 * e + 1];
}

// M(ro + i, co + j) += f * src(i, j)
__global__ void add_block_kernel(double* M, int N, int ro, int co, const double* __restrict__ src,
                                 double f) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= (size_t)N * N) return;
  const int i = (int)(k % N), j = (int)(k / N);
  const size_t e = (size_t)(ro + i) + (size_t)(co + j) * 2 * N;
  M[2 * e] += f * src[2 * k];
  M[2 * e + 1] += f * src[2 * k + 1];
}

// SL = LS^H (impl.hpp:4560-4575), then G = twoeH - xHFX K
__global__ void finish_gd_kernel(double* twoeH, double* K, int N, double xHFX, int exch,
                                 double* G) {
  const int N2 = 2 * N;
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= (size_t)N2 * N2) return;
  const int r = (int)(k % N2), c = (int)(k / N2);
  size_t src = k;
  bool conj = false;
  if (r >= N && c < N) {  // SL block element (N + j, i) = conj(LS(i, N + j))
    src = (size_t)c + (size_t)r * N2;
    conj = true;
  }
  double hr = twoeH[2 * src], hi = twoeH[2 * src + 1];
  double kr = K[2 * src], ki = K[2 * src + 1];
  if (conj) {
    hi = -hi;
    ki = -ki;
  }
  G[2 * k] = hr - (exch ? xHFX * kr : 0.0);
  G[2 * k + 1] = hi - (exch ? xHFX * ki : 0.0);
}

// ------------------------------------------------------------ host driver
cqf_status ensure_relws(cqf_basis* B, size_t bytes) {
  if (bytes <= B->relws_bytes) return CQF_OK;
  if (B->d_relws) CQF_RCUDA(cudaFreeAsync(B->d_relws, B->stream));
  B->d_relws = nullptr;
  B->relws_bytes = 0;
  CQF_RCUDA(cudaMallocAsync(&B->d_relws, bytes, B->stream));
  CQF_RCUDA(cudaStreamSynchronize(B->stream));
  B->relws_bytes = bytes;
  return CQF_OK;
}

size_t align32(size_t n) { return (n + 31) / 32 * 32; }

// One contraction type on device pointers (X, AX: 17 entries, N x N complex).
// ws: device scratch of rel_ws_doubles() doubles.  From opts: screen, and
// precision / fp32_cutoff (CQF_MIXED: quartets whose screening bound is below
// the cutoff run in FP32 arithmetic, the rest in FP64).  cnt: total,
// screened, FP32, FP64 quartet counts, added to.
size_t rel_ws_doubles(const cqf_basis* B) {
  const size_t nc2 = (size_t)B->ncart * B->ncart, ns2 = (size_t)B->nshell * B->nshell;
  const size_t dc = align32(9 * 2 * nc2) + align32(13 * nc2) + align32(10 * ns2);
  // Gaunt: 20 Cartesian complex densities | 16 complex accumulators | norms
  const size_t ga = align32(20 * 2 * nc2) + align32(16 * 2 * nc2) + align32(18 * ns2);
  return std::max(dc, ga) + 64;
}

// The entries a contraction type writes (the others are neither zeroed nor
// written: the reference's GAUNT list points its CSLM* / XSLM* entries at
// the CLSM* / XLSM* outputs).
std::vector<int> rel_outputs(int type, bool exch) {
  std::vector<int> o;
  auto four = [&](int base) {
    for (int c = 0; c < 4; c++) o.push_back(base + c);
  };
  if (type == CQF_REL_BARE_COULOMB) {
    o.push_back(CQF_CLLMS);
    if (exch) four(CQF_XLLMS);
  } else if (type == CQF_REL_LLSS) {
    o.push_back(CQF_CLLMS);
    four(CQF_CSSMS);
    if (exch) four(CQF_XLSMS);
  } else if (type == CQF_REL_SSSS) {
    four(CQF_CSSMS);
    if (exch) four(CQF_XSSMS);
  } else {
    four(CQF_CLSMS);
    if (exch) {
      four(CQF_XLLMS);
      four(CQF_XSSMS);
      four(CQF_XLSMS);
    }
  }
  return o;
}

cqf_status gaunt_contract_dev(cqf_basis* B, const double* const* X, double* const* AX, int exch,
                              bool gauge, const cqf_opts& opts, cudaStream_t st, double* ws,
                              unsigned long long* cnt);

cqf_status rel_contract_dev(cqf_basis* B, const double* const* X, double* const* AX, int type,
                            int exch, const cqf_opts& opts, cudaStream_t st, double* ws,
                            unsigned long long* cnt) {
  if (opts.shard_count < 1 || opts.shard_index < 0 || opts.shard_index >= opts.shard_count)
    return fail(CQF_EINVAL, "shard_index must lie in [0, shard_count)");
  const int screen = opts.screen;
  const bool mixed = opts.precision == CQF_MIXED && opts.fp32_cutoff > 0.0;
  const int N = B->nbasis, nc = B->ncart, ns = B->nshell;
  const size_t NN = (size_t)N * N, nc2 = (size_t)nc * nc, ns2 = (size_t)ns * ns;
  for (int m : rel_outputs(type, exch))
    if (AX[m]) CQF_RCUDA(cudaMemsetAsync(AX[m], 0, 2 * NN * sizeof(double), st));
  if (type == CQF_REL_GAUNT || type == CQF_REL_GAUGE)
    return gaunt_contract_dev(B, X, AX, exch, type == CQF_REL_GAUGE, opts, st, ws, cnt);

  if (type == CQF_REL_BARE_COULOMB) {
    // (LL|LL): the 1C engine on J[Re X] and K[X] (the same quartets, screen
    // and digestion as the reference's BARE_COULOMB branch, :514-790)
    if (!X[CQF_CLLMS] || !AX[CQF_CLLMS]) return fail(CQF_EINVAL, "BARE_COULOMB needs CLLMS");
    double* reX = ws;  // N x N complex
    real_part_kernel<<<rgrid(NN, 256), 256, 0, st>>>(X[CQF_CLLMS], NN, reX);
    CQF_RCUDA(cudaGetLastError());
    std::vector<cqf_contraction> list;
    list.push_back({reX, AX[CQF_CLLMS], 1, CQF_COULOMB});
    if (exch)
      for (int c = 0; c < 4; c++) {
        if (!X[CQF_XLLMS + c] || !AX[CQF_XLLMS + c])
          return fail(CQF_EINVAL, "BARE_COULOMB exchange needs XLLM*");
        list.push_back({X[CQF_XLLMS + c], AX[CQF_XLLMS + c], 1, CQF_EXCHANGE});
      }
    cqf_opts o;
    cqf_opts_default(&o);
    o.is_complex = 1;
    o.device_pointers = 1;
    o.screen = screen;
    o.precision = opts.precision;
    o.fp32_cutoff = opts.fp32_cutoff;
    o.stream = st;
    o.shard_index = opts.shard_index;
    o.shard_count = opts.shard_count;
    cqf_stats s1{};
    const int n = (int)list.size();
    if (split_eligible(B, list.data(), n, o)) {
      // Hermitian entries: real and imaginary parts on the real kernels
      CQF_RTRY(basis_workspace(
          B, split_ws_doubles(B, split_real_count(list.data(), n), o) * sizeof(double)));
      CQF_RTRY(split_core(B, list.data(), n, o, &s1, static_cast<double*>(B->d_ws), false,
                          nullptr));
    } else {
      CQF_RTRY(basis_workspace(B, ws_layout(B, n, o).total * sizeof(double)));
      CQF_RTRY(contract_core(B, list.data(), n, o, &s1, static_cast<double*>(B->d_ws), false,
                             nullptr));
    }
    cnt[0] += s1.quartets_total;
    cnt[1] += s1.quartets_screened;
    cnt[2] += s1.quartets_fp32;
    cnt[3] += s1.quartets_fp64;
    return CQF_OK;
  }

  const bool llss = (type == CQF_REL_LLSS);
  CQF_RTRY(ensure_rel_schwarz(B, llss, true, false, false, st));
  // required entries
  std::vector<int> need = {CQF_CSSMS, CQF_CSSMX, CQF_CSSMY, CQF_CSSMZ};
  if (llss) need.push_back(CQF_CLLMS);
  if (exch)
    for (int c = 0; c < 4; c++) need.push_back((llss ? CQF_XLSMS : CQF_XSSMS) + c);
  for (int m : need)
    if (!X[m]) return fail(CQF_EINVAL, "missing X entry for this contraction type");
  std::vector<int> outs = {CQF_CSSMS, CQF_CSSMX, CQF_CSSMY, CQF_CSSMZ};
  if (llss) outs.push_back(CQF_CLLMS);
  if (exch)
    for (int c = 0; c < 4; c++) outs.push_back((llss ? CQF_XLSMS : CQF_XSSMS) + c);
  for (int m : outs)
    if (!AX[m]) return fail(CQF_EINVAL, "missing AX entry for this contraction type");

  // workspace: 9 Cartesian complex densities | 13 real accumulators (Jll,
  // Jss x4, K x4 complex) | norms
  double* xc = ws;
  double* accb = ws + align32(9 * 2 * nc2);
  double* nrm = accb + align32(13 * nc2);
  double* Jll = accb;
  double* Jss[4] = {accb + nc2, accb + 2 * nc2, accb + 3 * nc2, accb + 4 * nc2};
  double* Kc[4] = {accb + 5 * nc2, accb + 7 * nc2, accb + 9 * nc2, accb + 11 * nc2};
  auto XC = [&](int slot) { return xc + (size_t)slot * 2 * nc2; };
  // slots: 0 CLLMS, 1..4 CSSM*, 5..8 exchange densities
  if (llss) launch_to_cart(B, X[CQF_CLLMS], 1, XC(0), st);
  for (int c = 0; c < 4; c++) launch_to_cart(B, X[CQF_CSSMS + c], 1, XC(1 + c), st);
  if (exch)
    for (int c = 0; c < 4; c++)
      launch_to_cart(B, X[(llss ? CQF_XLSMS : CQF_XSSMS) + c], 1, XC(5 + c), st);
  // screening norms: max over CLLMS, CSSM*, XLSM* (LLSS) or CSSM* (SSSS)
  std::vector<int> smats = {CQF_CSSMS, CQF_CSSMX, CQF_CSSMY, CQF_CSSMZ};
  if (llss) {
    smats.insert(smats.begin(), CQF_CLLMS);
    for (int c = 0; c < 4; c++)
      if (X[CQF_XLSMS + c]) smats.push_back(CQF_XLSMS + c);
  }
  double* nmAll = nrm + ns2;
  for (size_t i = 0; i < smats.size(); i++)
    launch_block_norms(B, X[smats[i]], 1, nmAll + i * ns2, st);
  launch_max_norms(nmAll, (int)smats.size(), ns2, nrm,
                   reinterpret_cast<unsigned long long*>(nmAll + 9 * ns2), st);
  CQF_RCUDA(cudaMemsetAsync(accb, 0, 13 * nc2 * sizeof(double), st));
  unsigned long long* dcnt = B->d_counters;
  CQF_RCUDA(cudaMemsetAsync(dcnt, 0, 4 * sizeof(unsigned long long), st));
  CQF_RCUDA(cudaGetLastError());

  RelLaunch a{};
  a.pairs = B->d_pairs;
  a.pp = B->d_pp;
  a.shells = B->d_shells;
  a.prim = B->d_prim;
  a.boys = B->d_boys64;
  a.boys32 = B->d_boys32;
  a.pairRange = B->d_pairRange;
  a.mixed = mixed ? 1 : 0;
  a.cut = opts.fp32_cutoff;
  a.screen = screen;
  a.thresh = B->thresh;
  a.norms = nrm;
  a.qLL = B->d_qLL;
  a.qSS = B->d_qSS;
  a.nShell = ns;
  a.ncart = nc;
  a.exchange = exch;
  a.Xll = XC(0);
  for (int c = 0; c < 4; c++) {
    a.Xss[c] = XC(1 + c);
    a.Xk[c] = XC(5 + c);
    a.Jss[c] = Jss[c];
    a.K[c] = Kc[c];
  }
  a.Jll = Jll;
  a.shardIdx = opts.shard_index;
  a.shardCnt = std::max(1, opts.shard_count);
  a.counters = dcnt;
  a.nsm = B->nsm;
  for (int cb = 0; cb < NCLS; cb++)
    for (int ck = 0; ck < NCLS; ck++) {
      if (!llss && ck > cb) continue;
      if (!B->cls_cnt[cb] || !B->cls_cnt[ck]) continue;
      int la, lb, lc, ld;
      class_ls(cb, la, lb);
      class_ls(ck, lc, ld);
      a.braBeg = B->cls_beg[cb];
      a.nBra = B->cls_cnt[cb];
      a.ketBeg = B->cls_beg[ck];
      a.nKet = B->cls_cnt[ck];
      a.same = (cb == ck);
      a.contracted = 0;
      for (int i = 0; i < a.nBra && !a.contracted; i++)
        a.contracted = B->h_pairs[a.braBeg + i].npp > 1;
      for (int i = 0; i < a.nKet && !a.contracted; i++)
        a.contracted = B->h_pairs[a.ketBeg + i].npp > 1;
      if (llss) launch_rel<1>(a, la, lb, lc, ld, st);
      else launch_rel<2>(a, la, lb, lc, ld, st);
    }
  CQF_RCUDA(cudaGetLastError());
  auto back = [&](const double* src, int mode, double* dst) {
    rel_from_cart_kernel<<<rgrid(NN, 256), 256, 0, st>>>(src, mode, N, nc, B->d_shells,
                                                         B->d_ao2shell, B->d_sph, B->d_sphOff,
                                                         dst);
  };
  if (llss) back(Jll, 1, AX[CQF_CLLMS]);
  back(Jss[0], 1, AX[CQF_CSSMS]);
  for (int c = 1; c < 4; c++) back(Jss[c], 2, AX[CQF_CSSMS + c]);
  if (exch)
    for (int c = 0; c < 4; c++)
      back(Kc[c], llss ? 0 : 3, AX[(llss ? CQF_XLSMS : CQF_XSSMS) + c]);
  CQF_RCUDA(cudaGetLastError());
  unsigned long long h[4];
  CQF_RCUDA(cudaMemcpyAsync(h, dcnt, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CQF_RCUDA(cudaStreamSynchronize(st));
  cnt[0] += h[0];
  cnt[1] += h[1];
  cnt[2] += h[2];
  cnt[3] += h[3];
  return CQF_OK;
}


// The GAUNT (or GAUGE) contraction on device pointers (X, AX: 29
// entries).  Needs X[CLSM*], X[CSLM*] and, with exchange, X[XLLM*],
// X[XSSM*], X[XSLM*]; writes AX[CLSM*] and, with exchange, AX[XLLM*],
// AX[XSSM*], AX[XLSM*].  The screening norms are the max over the 16
// exchange densities the reference uses (:2957-3020, :4060-4130), of those
// given.  FP64 (opts.precision is not applied to these terms).
cqf_status gaunt_contract_dev(cqf_basis* B, const double* const* X, double* const* AX, int exch,
                              bool gauge, const cqf_opts& opts, cudaStream_t st, double* ws,
                              unsigned long long* cnt) {
  const int N = B->nbasis, nc = B->ncart, ns = B->nshell;
  const size_t NN = (size_t)N * N, nc2 = (size_t)nc * nc, ns2 = (size_t)ns * ns;
  (void)NN;
  std::vector<int> need;
  for (int c = 0; c < 4; c++) {
    need.push_back(CQF_CLSMS + c);
    need.push_back(CQF_CSLMS + c);
    if (exch) {
      need.push_back(CQF_XLLMS + c);
      need.push_back(CQF_XSSMS + c);
      need.push_back(CQF_XSLMS + c);
    }
  }
  for (int m : need)
    if (!X[m]) return fail(CQF_EINVAL, "missing X entry for the GAUNT / GAUGE contraction");
  for (int m : rel_outputs(CQF_REL_GAUNT, exch))
    if (!AX[m]) return fail(CQF_EINVAL, "missing AX entry for the GAUNT / GAUGE contraction");
  CQF_RTRY(ensure_rel_schwarz(B, false, false, !gauge, gauge, st));

  double* xc = ws;
  double* accb = ws + align32(20 * 2 * nc2);
  double* nrm = accb + align32(16 * 2 * nc2);
  auto XC = [&](int slot) { return xc + (size_t)slot * 2 * nc2; };
  auto AC = [&](int slot) { return accb + (size_t)slot * 2 * nc2; };
  // density slots: 0 XLLM*, 4 XSSM*, 8 CLSM*, 12 CSLM*, 16 XSLM*
  const int src[5] = {CQF_XLLMS, CQF_XSSMS, CQF_CLSMS, CQF_CSLMS, CQF_XSLMS};
  for (int k = 0; k < 5; k++)
    for (int c = 0; c < 4; c++)
      if (X[src[k] + c]) launch_to_cart(B, X[src[k] + c], 1, XC(4 * k + c), st);
  // screening norms: max over XLSM*, XSLM*, XLLM*, XSSM*
  // (without exchange, the LS / SL Coulomb entries stand for the same
  // LS / SL blocks)
  std::vector<int> smats;
  for (int base : {(int)CQF_XLSMS, (int)CQF_XSLMS, (int)CQF_XLLMS, (int)CQF_XSSMS})
    for (int c = 0; c < 4; c++) {
      int m = base + c;
      if (!X[m] && base == CQF_XLSMS) m = CQF_CLSMS + c;
      if (!X[m] && base == CQF_XSLMS) m = CQF_CSLMS + c;
      if (X[m]) smats.push_back(m);
    }
  double* nmAll = nrm + ns2;
  for (size_t i = 0; i < smats.size(); i++)
    launch_block_norms(B, X[smats[i]], 1, nmAll + i * ns2, st);
  launch_max_norms(nmAll, (int)smats.size(), ns2, nrm,
                   reinterpret_cast<unsigned long long*>(nmAll + 16 * ns2), st);
  CQF_RCUDA(cudaMemsetAsync(accb, 0, 16 * 2 * nc2 * sizeof(double), st));
  unsigned long long* dcnt = B->d_counters;
  CQF_RCUDA(cudaMemsetAsync(dcnt, 0, 4 * sizeof(unsigned long long), st));
  CQF_RCUDA(cudaGetLastError());

  GauntLaunch a{};
  a.pairs = B->d_pairs;
  a.pp = B->d_pp;
  a.shells = B->d_shells;
  a.prim = B->d_prim;
  a.boys = B->d_boys64;
  a.screen = opts.screen;
  a.thresh = B->thresh;
  a.norms = nrm;
  a.qG = gauge ? B->d_qB : B->d_qG;
  a.nShell = ns;
  a.ncart = nc;
  a.exchange = exch;
  for (int c = 0; c < 4; c++) {
    a.Xll[c] = XC(0 + c);
    a.Xss[c] = XC(4 + c);
    a.Cls[c] = XC(8 + c);
    a.Csl[c] = XC(12 + c);
    a.Xsl[c] = XC(16 + c);
    a.Kll[c] = AC(0 + c);
    a.Kss[c] = AC(4 + c);
    a.Jls[c] = AC(8 + c);
    a.Kls[c] = AC(12 + c);
  }
  a.shardIdx = opts.shard_index;
  a.shardCnt = std::max(1, opts.shard_count);
  a.counters = dcnt;
  for (int cb = 0; cb < NCLS; cb++)
    for (int ck = 0; ck <= cb; ck++) {
      if (!B->cls_cnt[cb] || !B->cls_cnt[ck]) continue;
      int la, lb, lc, ld;
      class_ls(cb, la, lb);
      class_ls(ck, lc, ld);
      a.braBeg = B->cls_beg[cb];
      a.nBra = B->cls_cnt[cb];
      a.ketBeg = B->cls_beg[ck];
      a.nKet = B->cls_cnt[ck];
      a.same = (cb == ck);
      if (gauge) launch_gaunt<true>(a, la, lb, lc, ld, st);
      else launch_gaunt<false>(a, la, lb, lc, ld, st);
    }
  CQF_RCUDA(cudaGetLastError());
  auto back = [&](const double* srcAcc, int mode, double* dst) {
    rel_from_cart_kernel<<<rgrid(NN, 256), 256, 0, st>>>(srcAcc, mode, N, nc, B->d_shells,
                                                         B->d_ao2shell, B->d_sph, B->d_sphOff,
                                                         dst);
  };
  for (int c = 0; c < 4; c++) {
    back(AC(8 + c), 0, AX[CQF_CLSMS + c]);
    if (exch) {
      back(AC(0 + c), 3, AX[CQF_XLLMS + c]);
      back(AC(4 + c), 3, AX[CQF_XSSMS + c]);
      back(AC(12 + c), 0, AX[CQF_XLSMS + c]);
    }
  }
  CQF_RCUDA(cudaGetLastError());
  unsigned long long h[4];
  CQF_RCUDA(cudaMemcpyAsync(h, dcnt, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CQF_RCUDA(cudaStreamSynchronize(st));
  for (int k = 0; k < 4; k++) cnt[k] += h[k];
  return CQF_OK;
}

}  // namespace
}  // namespace cqf

using namespace cqf;

extern "C" {

cqf_status cqf_rel_two_body_contract(cqf_basis* B, const void* const* X, void* const* AX,
                                     int type, int compute_exchange, const cqf_opts* optsIn,
                                     cqf_stats* stats) {
  if (!B || !X || !AX) return fail(CQF_EINVAL, "cqf_rel_two_body_contract: null argument");
  if (type < CQF_REL_BARE_COULOMB || type > CQF_REL_GAUGE)
    return fail(CQF_EINVAL, "cqf_rel_two_body_contract: unknown contraction type");
  cqf_opts o;
  cqf_opts_default(&o);
  if (optsIn) o = *optsIn;
  std::lock_guard<std::mutex> lk(B->mu);
  CQF_RCUDA(cudaSetDevice(B->device));
  cudaStream_t st = o.stream ? (cudaStream_t)o.stream : B->stream;
  const int nmat = (type >= CQF_REL_GAUNT) ? CQF_REL_NMAT_GAUNT : CQF_REL_NMAT;
  const std::vector<int> outs = rel_outputs(type, compute_exchange != 0);
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  const size_t wsd = rel_ws_doubles(B);
  const size_t hostd = o.device_pointers ? 0 : align32(2 * NN) * 2 * nmat;
  CQF_RTRY(ensure_relws(B, (wsd + hostd) * sizeof(double)));
  double* ws = static_cast<double*>(B->d_relws);
  double* hbuf = ws + wsd;
  const double* Xd[CQF_REL_NMAT_GAUNT] = {};
  double* AXd[CQF_REL_NMAT_GAUNT] = {};
  for (int m = 0; m < nmat; m++) {
    if (o.device_pointers) {
      Xd[m] = static_cast<const double*>(X[m]);
      AXd[m] = static_cast<double*>(AX[m]);
    } else {
      double* xd = hbuf + (size_t)m * align32(2 * NN);
      double* ad = hbuf + (size_t)(nmat + m) * align32(2 * NN);
      Xd[m] = X[m] ? xd : nullptr;
      AXd[m] = AX[m] ? ad : nullptr;
      if (X[m])
        CQF_RCUDA(cudaMemcpyAsync(xd, X[m], 2 * NN * sizeof(double), cudaMemcpyHostToDevice, st));
    }
  }
  CQF_RCUDA(cudaEventRecord(B->ev0, st));
  unsigned long long cnt[4] = {0, 0, 0, 0};
  CQF_RTRY(rel_contract_dev(B, Xd, AXd, type, compute_exchange, o, st, ws, cnt));
  CQF_RCUDA(cudaEventRecord(B->ev1, st));
  // only the entries the type writes come back (a list may alias the others)
  if (!o.device_pointers)
    for (int m : outs)
      if (AX[m])
        CQF_RCUDA(cudaMemcpyAsync(AX[m], AXd[m], 2 * NN * sizeof(double), cudaMemcpyDeviceToHost,
                                  st));
  CQF_RCUDA(cudaStreamSynchronize(st));
  if (stats) {
    stats->quartets_total = (long long)cnt[0];
    stats->quartets_screened = (long long)cnt[1];
    stats->quartets_fp32 = (long long)cnt[2];
    stats->quartets_fp64 = (long long)cnt[3];
    float ms = 0.f;
    cudaEventElapsedTime(&ms, B->ev0, B->ev1);
    stats->device_ms = ms;
  }
  return CQF_OK;
}

void cqf_dc_opts_default(cqf_dc_opts* o) {
  if (!o) return;
  o->bare_coulomb = 1;
  o->dirac_coulomb = 1;
  o->dirac_coulomb_ssss = 1;
  o->libcint = 1;
  o->xHFX = 1.0;
  o->gaunt = 0;
  o->gauge = 0;
}

cqf_status cqf_four_comp_gd(cqf_basis* B, const void* const* D, void* const* G,
                            const cqf_dc_opts* dcIn, const cqf_opts* optsIn, cqf_stats* stats) {
  if (!B || !D || !G) return fail(CQF_EINVAL, "cqf_four_comp_gd: null argument");
  for (int c = 0; c < 4; c++)
    if (!D[c] || !G[c]) return fail(CQF_EINVAL, "cqf_four_comp_gd: null D or G component");
  cqf_dc_opts dc;
  cqf_dc_opts_default(&dc);
  if (dcIn) dc = *dcIn;
  cqf_opts o;
  cqf_opts_default(&o);
  if (optsIn) o = *optsIn;
  std::lock_guard<std::mutex> lk(B->mu);
  CQF_RCUDA(cudaSetDevice(B->device));
  cudaStream_t st = o.stream ? (cudaStream_t)o.stream : B->stream;
  const int N = B->nbasis;
  const size_t NN = (size_t)N * N, NN2 = 4 * NN;
  const double c2 = SPEED_OF_LIGHT * SPEED_OF_LIGHT;
  const double C2 = 1.0 / (4.0 * c2), C4 = 1.0 / (16.0 * c2 * c2);
  const bool exch = std::fabs(dc.xHFX) >= 1e-12;
  // workspace: rel scratch | blocks 16 x N^2 | AX 29 x N^2 | twoeH 4 x 4N^2 |
  // K 4 x 4N^2 | D/G staging (host pointers) 8 x 4N^2, all complex
  const size_t wsd = rel_ws_doubles(B);
  const size_t blkd = align32(2 * NN), bigd = align32(2 * NN2);
  const size_t total = wsd + 16 * blkd + CQF_REL_NMAT_GAUNT * blkd + 8 * bigd +
                       (o.device_pointers ? 0 : 8 * bigd);
  CQF_RTRY(ensure_relws(B, total * sizeof(double)));
  double* ws = static_cast<double*>(B->d_relws);
  double* blk = ws + wsd;
  double* axb = blk + 16 * blkd;
  double* twoeH = axb + CQF_REL_NMAT_GAUNT * blkd;
  double* Kb = twoeH + 4 * bigd;
  double* stage = Kb + 4 * bigd;
  const double* Dd[4];
  double* Gd[4];
  for (int c = 0; c < 4; c++) {
    if (o.device_pointers) {
      Dd[c] = static_cast<const double*>(D[c]);
      Gd[c] = static_cast<double*>(G[c]);
    } else {
      double* dd = stage + c * bigd;
      Dd[c] = dd;
      Gd[c] = stage + (4 + c) * bigd;
      CQF_RCUDA(cudaMemcpyAsync(dd, D[c], 2 * NN2 * sizeof(double), cudaMemcpyHostToDevice, st));
    }
  }
  CQF_RCUDA(cudaEventRecord(B->ev0, st));
  // LL / SS / LS (/ SL, for Gaunt) blocks of each Pauli component
  // (impl.hpp:3847-3857)
  auto B3 = [&](int k, int c) { return blk + (size_t)(k * 4 + c) * blkd; };
  const int ro[4] = {0, N, 0, N}, co[4] = {0, N, N, 0};
  for (int k = 0; k < (dc.gaunt || dc.gauge ? 4 : 3); k++)
    for (int c = 0; c < 4; c++)
      get_block_kernel<<<rgrid(NN, 256), 256, 0, st>>>(Dd[c], N, ro[k], co[k], B3(k, c));
  CQF_RCUDA(cudaMemsetAsync(twoeH, 0, 8 * bigd * sizeof(double), st));
  CQF_RCUDA(cudaGetLastError());
  const double* X[CQF_REL_NMAT_GAUNT];
  double* AX[CQF_REL_NMAT_GAUNT];
  X[CQF_CLLMS] = B3(0, 0);
  for (int c = 0; c < 4; c++) {
    X[CQF_XLLMS + c] = B3(0, c);
    X[CQF_CSSMS + c] = B3(1, c);
    X[CQF_XSSMS + c] = B3(1, c);
    X[CQF_XLSMS + c] = B3(2, c);
    X[CQF_CLSMS + c] = B3(2, c);
    X[CQF_CSLMS + c] = B3(3, c);
    X[CQF_XSLMS + c] = B3(3, c);
  }
  for (int m = 0; m < CQF_REL_NMAT_GAUNT; m++) AX[m] = axb + (size_t)m * blkd;
  auto H = [&](int c) { return twoeH + (size_t)c * bigd; };
  auto Kk = [&](int c) { return Kb + (size_t)c * bigd; };
  auto add = [&](double* M, int r0, int c0, const double* src, double f) {
    add_block_kernel<<<rgrid(NN, 256), 256, 0, st>>>(M, N, r0, c0, src, f);
  };
  unsigned long long cnt[4] = {0, 0, 0, 0};
  if (dc.bare_coulomb) {  // impl.hpp:3895-3969
    CQF_RTRY(rel_contract_dev(B, X, AX, CQF_REL_BARE_COULOMB, exch, o, st, ws, cnt));
    add(H(0), 0, 0, AX[CQF_CLLMS], dc.libcint ? 2.0 : 1.0);
    if (exch)
      for (int c = 0; c < 4; c++) add(Kk(c), 0, 0, AX[CQF_XLLMS + c], 1.0);
  }
  if (dc.dirac_coulomb) {  // impl.hpp:4003-4147
    CQF_RTRY(rel_contract_dev(B, X, AX, CQF_REL_LLSS, exch, o, st, ws, cnt));
    add(H(0), 0, 0, AX[CQF_CLLMS], 2.0 * C2);
    for (int c = 0; c < 4; c++) add(H(c), N, N, AX[CQF_CSSMS + c], 2.0 * C2);
    if (exch)
      for (int c = 0; c < 4; c++) add(Kk(c), 0, N, AX[CQF_XLSMS + c], -C2);
  }
  if (dc.dirac_coulomb_ssss) {  // impl.hpp:4149-4233
    CQF_RTRY(rel_contract_dev(B, X, AX, CQF_REL_SSSS, exch, o, st, ws, cnt));
    for (int c = 0; c < 4; c++) add(H(c), N, N, AX[CQF_CSSMS + c], 2.0 * C4);
    if (exch)
      for (int c = 0; c < 4; c++) add(Kk(c), N, N, AX[CQF_XSSMS + c], -C4);
  }
  // Gaunt and Gauge (impl.hpp:4228-4540): with the gauge term both are
  // weighted C2 / 2 (their sum is the Breit term)
  const double C2b = dc.gauge ? 0.5 * C2 : C2;
  for (int t : {(int)CQF_REL_GAUNT, (int)CQF_REL_GAUGE}) {
    if (!(t == CQF_REL_GAUNT ? dc.gaunt : dc.gauge)) continue;
    CQF_RTRY(rel_contract_dev(B, X, AX, t, exch, o, st, ws, cnt));
    for (int c = 0; c < 4; c++) add(H(c), 0, N, AX[CQF_CLSMS + c], 2.0 * C2b);
    if (exch)
      for (int c = 0; c < 4; c++) {
        add(Kk(c), 0, 0, AX[CQF_XLLMS + c], -C2b);
        add(Kk(c), N, N, AX[CQF_XSSMS + c], -C2b);
        add(Kk(c), 0, N, AX[CQF_XLSMS + c], -C2b);
      }
  }
  for (int c = 0; c < 4; c++)
    finish_gd_kernel<<<rgrid(NN2, 256), 256, 0, st>>>(H(c), Kk(c), N, dc.xHFX, exch ? 1 : 0,
                                                      Gd[c]);
  CQF_RCUDA(cudaGetLastError());
  CQF_RCUDA(cudaEventRecord(B->ev1, st));
  if (!o.device_pointers)
    for (int c = 0; c < 4; c++)
      CQF_RCUDA(cudaMemcpyAsync(G[c], Gd[c], 2 * NN2 * sizeof(double), cudaMemcpyDeviceToHost,
                                st));
  CQF_RCUDA(cudaStreamSynchronize(st));
  if (stats) {
    stats->quartets_total = (long long)cnt[0];
    stats->quartets_screened = (long long)cnt[1];
    stats->quartets_fp32 = (long long)cnt[2];
    stats->quartets_fp64 = (long long)cnt[3];
    float ms = 0.f;
    cudaEventElapsedTime(&ms, B->ev0, B->ev1);
    stats->device_ms = ms;
  }
  return CQF_OK;
}

}  // extern "C"
