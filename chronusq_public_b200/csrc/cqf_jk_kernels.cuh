// J/K digestion kernels.  One launch per shell-quartet class (bra pair class
// x ket pair class); one thread per unique shell quartet.
//
// Quartet set, screening and update formulas restate
// GTODirectTPIContraction::directScaffoldNew
// (include/particleintegrals/contract/direct.hpp:1642-2002):
//  * unique quartets: pairs of significant pairs (s1 s2 | s3 s4) with
//    (s3, s4) <= (s1, s2) in the reference loop order (:1643-1730);
//  * screen: max of six shell-block norms x Q12 x Q34 < thresh (:1733-1762),
//    per matrix when several are contracted (:1764-1786);
//  * degeneracy and the 0.5 * deg scaling (:1791-1803, :1849-1850);
//  * the four digestion branches (HER/non-HER x COULOMB/EXCHANGE,
//    :1858-2002), applied with the reference's shell roles 1..4 so that even
//    the Hermitian-exchange branch on a non-Hermitian X matches.
// Updates land in Cartesian-AO accumulators with FP64 atomics (L2 resident);
// the Hermitisation / 0.5 scaling of :2036-2066 happens in the back transform.
#pragma once

#include "cqf_eri.cuh"
#include "cqf_internal.hpp"

namespace cqf {

__device__ __forceinline__ double block_norm(const double* __restrict__ n, int a, int b,
                                             int ns) {
  return __ldg(n + a + (size_t)b * ns);
}

// max of the six shell-block norms the reference combines (direct.hpp:1693-1736)
__device__ __forceinline__ double sh_max(const double* __restrict__ n, int s1, int s2, int s3,
                                         int s4, int ns) {
  double m = block_norm(n, s3, s4, ns);
  m = fmax(m, fmax(block_norm(n, s1, s4, ns), block_norm(n, s2, s4, ns)));
  double m123 = fmax(block_norm(n, s1, s3, ns), block_norm(n, s2, s3, ns));
  m123 = fmax(m123, block_norm(n, s1, s2, ns));
  return fmax(m, m123);
}

template <bool CPLX>
struct Mat;

template <>
struct Mat<false> {
  static __device__ __forceinline__ double ld(const double* X, size_t i) { return __ldg(X + i); }
  static __device__ __forceinline__ double ldc(const double* X, size_t i) { return __ldg(X + i); }
  static __device__ __forceinline__ double ldre(const double* X, size_t i) { return __ldg(X + i); }
  static __device__ __forceinline__ void add(double* A, size_t i, double v, double w) {
    atomicAdd(A + i, v * w);
  }
  static __device__ __forceinline__ void addre(double* A, size_t i, double v) {
    atomicAdd(A + i, v);
  }
};

template <>
struct Mat<true> {
  static __device__ __forceinline__ double2 ld(const double* X, size_t i) {
    return __ldg(reinterpret_cast<const double2*>(X) + i);
  }
  static __device__ __forceinline__ double2 ldc(const double* X, size_t i) {
    double2 z = __ldg(reinterpret_cast<const double2*>(X) + i);
    z.y = -z.y;
    return z;
  }
  static __device__ __forceinline__ double ldre(const double* X, size_t i) {
    return __ldg(X + 2 * i);
  }
  static __device__ __forceinline__ void add(double* A, size_t i, double2 v, double w) {
    atomicAdd(A + 2 * i, v.x * w);
    atomicAdd(A + 2 * i + 1, v.y * w);
  }
  static __device__ __forceinline__ void addre(double* A, size_t i, double v) {
    atomicAdd(A + 2 * i, v);
  }
};

__device__ __forceinline__ double2 operator+(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}

// Digest one integral v (already x 0.5 deg) with role indices i1..i4 into
// matrix m (direct.hpp:1858-2002).
template <bool CPLX>
__device__ __forceinline__ void digest_one(int flags, const double* __restrict__ X, double* A,
                                           size_t nc, int i1, int i2, int i3, int i4, double v) {
  using M = Mat<CPLX>;
  const bool her = flags & 1, exch = flags & 2;
  auto ix = [nc](int r, int c) -> size_t { return (size_t)r + (size_t)c * nc; };
  if (her) {
    if (!exch) {
      // J(1,2) += X(4,3) I ; J(4,3) += X(1,2) I   (real parts)
      M::addre(A, ix(i1, i2), M::ldre(X, ix(i4, i3)) * v);
      M::addre(A, ix(i4, i3), M::ldre(X, ix(i1, i2)) * v);
    } else {
      // (bit 2, the antisymmetric part of a split complex Hermitian density,
      // needs nothing here: these four updates read X in the orientation
      // the antisymmetric back transform expects, as the class kernels' do)
      const double h = 0.5 * v;
      M::add(A, ix(i1, i3), M::ldc(X, ix(i4, i2)), h);
      M::add(A, ix(i4, i2), M::ldc(X, ix(i1, i3)), h);
      M::add(A, ix(i4, i1), M::ldc(X, ix(i2, i3)), h);
      M::add(A, ix(i2, i3), M::ldc(X, ix(i4, i1)), h);
    }
  } else {
    const double h = 0.5 * v;
    if (!exch) {
      auto x34 = M::ld(X, ix(i4, i3)) + M::ld(X, ix(i3, i4));
      auto x12 = M::ld(X, ix(i2, i1)) + M::ld(X, ix(i1, i2));
      M::add(A, ix(i1, i2), x34, h);
      M::add(A, ix(i3, i4), x12, h);
      M::add(A, ix(i2, i1), x34, h);
      M::add(A, ix(i4, i3), x12, h);
    } else {
      M::add(A, ix(i3, i1), M::ld(X, ix(i4, i2)), h);
      M::add(A, ix(i4, i2), M::ld(X, ix(i3, i1)), h);
      M::add(A, ix(i4, i1), M::ld(X, ix(i3, i2)), h);
      M::add(A, ix(i3, i2), M::ld(X, ix(i4, i1)), h);
      M::add(A, ix(i1, i3), M::ld(X, ix(i2, i4)), h);
      M::add(A, ix(i2, i4), M::ld(X, ix(i1, i3)), h);
      M::add(A, ix(i1, i4), M::ld(X, ix(i2, i3)), h);
      M::add(A, ix(i2, i3), M::ld(X, ix(i1, i4)), h);
    }
  }
}

constexpr int JK_THREADS = 128;

// Adds the block's quartet counts to counters[0..3] with one atomic each.
__device__ __forceinline__ void count_block(unsigned long long* counters, bool visited,
                                            bool screened, bool f32, bool f64) {
  __shared__ unsigned int cnt[4];
  if (threadIdx.x < 4) cnt[threadIdx.x] = 0;
  __syncthreads();
  const unsigned mask = __activemask();
  const unsigned b0 = __ballot_sync(mask, visited), b1 = __ballot_sync(mask, screened);
  const unsigned b2 = __ballot_sync(mask, f32), b3 = __ballot_sync(mask, f64);
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&cnt[0], __popc(b0));
    atomicAdd(&cnt[1], __popc(b1));
    atomicAdd(&cnt[2], __popc(b2));
    atomicAdd(&cnt[3], __popc(b3));
  }
  __syncthreads();
  if (threadIdx.x < 4 && cnt[threadIdx.x])
    atomicAdd(counters + threadIdx.x, (unsigned long long)cnt[threadIdx.x]);
}

template <int LM, bool CPLX>
__global__ void __launch_bounds__(JK_THREADS)
    jk_generic_kernel(const JKLaunch a, int la, int lb, int lc, int ld) {
  const int ib = blockIdx.x;
  const int jk = blockIdx.y * JK_THREADS + threadIdx.x;
  if (!in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) return;  // another shard's bra
  const PairDev P = a.pairs[a.braBeg + ib];
  const int ns = a.nShell;

  bool visited = false, screened = false, work = false, fp32 = false;
  int s1 = 0, s2 = 0, s3 = 0, s4 = 0;
  double bound = 0.0;
  bool pRef = true;
  PairDev Q;
  if (a.same && blockIdx.y * JK_THREADS > ib) {  // tile wholly above the diagonal
    count_block(a.counters, false, false, false, false);
    return;
  }
  if (jk < a.nKet && !(a.same && jk > ib)) {  // each unordered pair once
    Q = a.pairs[a.ketBeg + jk];
    visited = true;
  }
  // tile-level screen: the largest Q of the block's kets (window maxima)
  double tq = 0.0;
  for (int k = blockIdx.y * JK_THREADS; k < min((int)(blockIdx.y + 1) * JK_THREADS, a.nKet);
       k += WTILE)
    tq = fmax(tq, __ldg(a.qWin + a.ketBeg + k));
  const bool tileDead = a.screen && __ldg(a.maxNorm) * P.Q * tq < a.thresh;
  if (tileDead) {
    count_block(a.counters, visited, visited, false, false);
    return;
  }
  if (visited) {
    pRef = P.lex >= Q.lex;
    const PairDev& R12 = pRef ? P : Q;
    const PairDev& R34 = pRef ? Q : P;
    s1 = R12.s1; s2 = R12.s2; s3 = R34.s1; s4 = R34.s2;
    if (a.screen) {
      bound = sh_max(a.norms, s1, s2, s3, s4, ns) * P.Q * Q.Q;
      screened = bound < a.thresh;
    }
    work = !screened;
    fp32 = work && a.precision == 1 && bound < a.fp32_cut &&
           fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib), __ldg(a.pairRange + a.ketBeg + jk),
                         la + lb + lc + ld, 0, 0);
  }
  count_block(a.counters, visited, screened, fp32, work && !fp32);
  if (!work) return;

  // per-matrix screening (direct.hpp:1764-1786)
  unsigned long long live[MAXMAT / 64];
  const int nw = (a.nMat + 63) / 64;
  for (int w = 0; w < nw; w++) live[w] = ~0ull;
  if (a.screen && a.nMat > 1) {
    const size_t ns2 = (size_t)ns * ns;
    for (int m = 0; m < a.nMat; m++) {
      double sm = sh_max(a.normsMat + m * ns2, s1, s2, s3, s4, ns);
      if (sm * P.Q * Q.Q < a.thresh) live[m >> 6] &= ~(1ull << (m & 63));
    }
  }

  const double deg = ((s1 == s2) ? 1.0 : 2.0) * ((s3 == s4) ? 1.0 : 2.0) *
                     ((s1 == s3 && s2 == s4) ? 1.0 : 2.0);
  const double scale = 0.5 * deg;
  const bool swP = P.shA != P.s1, swQ = Q.shA != Q.s1;
  const size_t nc = a.ncart;
  const size_t matStride = (size_t)a.ncart * a.ncart * (CPLX ? 2 : 1);
  const int na = ncart(la), nb = ncart(lb), ncc = ncart(lc), nd = ncart(ld);

  double col[RtBounds<LM>::NAB];
#pragma unroll 1
  for (int c = 0; c < ncc; c++)
#pragma unroll 1
    for (int d = 0; d < nd; d++) {
      if (fp32)
        eri_column_rt<float, LM>(la, lb, lc, ld, c, d, P, Q, a.pp, a.boys32, col);
      else
        eri_column_rt<double, LM>(la, lb, lc, ld, c, d, P, Q, a.pp, a.boys64, col);
      const int gc = Q.cA + c, gd = Q.cB + d;
      const int qc = swQ ? gd : gc, qd = swQ ? gc : gd;
#pragma unroll 1
      for (int ia = 0; ia < na; ia++)
#pragma unroll 1
        for (int ibb = 0; ibb < nb; ibb++) {
          const int ga = P.cA + ia, gb = P.cB + ibb;
          const int pa = swP ? gb : ga, pb = swP ? ga : gb;
          const int i1 = pRef ? pa : qc, i2 = pRef ? pb : qd;
          const int i3 = pRef ? qc : pa, i4 = pRef ? qd : pb;
          const double v = col[ia * nb + ibb] * scale;
          for (int m = 0; m < a.nMat; m++) {
            if (!((live[m >> 6] >> (m & 63)) & 1ull)) continue;
            digest_one<CPLX>(__ldg(a.flags + m), a.Xc + m * matStride, a.Ac + m * matStride, nc,
                             i1, i2, i3, i4, v);
          }
        }
    }
}

// One class-quartet launch of the generic kernel.
inline void launch_jk_generic(const JKLaunch& a, int la, int lb, int lc, int ld,
                              cudaStream_t st) {
  if (a.nBra == 0 || a.nKet == 0) return;
  dim3 grid(a.nBra, (a.nKet + JK_THREADS - 1) / JK_THREADS);
  const int lm = max(max(la, lb), max(lc, ld));
#define CQF_GEN_CASE(LMV)                                                                   \
  if (lm <= LMV) {                                                                          \
    if (a.cplx)                                                                             \
      jk_generic_kernel<LMV, true><<<grid, JK_THREADS, 0, st>>>(a, la, lb, lc, ld);         \
    else                                                                                    \
      jk_generic_kernel<LMV, false><<<grid, JK_THREADS, 0, st>>>(a, la, lb, lc, ld);        \
    return;                                                                                 \
  }
  CQF_GEN_CASE(1)
  CQF_GEN_CASE(2)
  CQF_GEN_CASE(3)
#undef CQF_GEN_CASE
}

// ---------------------------------------------------------------- Schwarz
// Q(s1,s2) = sqrt(|| D ||_inf), D(i,j) = (ij|ij) over the AOs of s1 (rows)
// and s2 (columns): max row sum (aointegrals_utilities.cxx:78-104).
__global__ void __launch_bounds__(64)
    schwarz_kernel(const PairDev* __restrict__ pairs, const PrimPairDev* __restrict__ pp,
                   const double* __restrict__ boys, const double* __restrict__ sph,
                   const int* __restrict__ sphOff, const ShellDev* __restrict__ shells,
                   int beg, int n, int nshell, double* Qtab, PairDev* pairsOut) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const PairDev P = pairs[beg + k];
  const ShellDev A = shells[P.shA], B = shells[P.shB];
  const int la = A.l, lb = B.l;
  const int nca = ncart(la), ncb = ncart(lb);
  const int na = A.pure ? nsph(la) : nca, nb = B.pure ? nsph(lb) : ncb;
  const double* TA = sph + sphOff[la];
  const double* TB = sph + sphOff[lb];
  double diag[ncart(LMAX)][ncart(LMAX)];
  for (int i = 0; i < na; i++)
    for (int j = 0; j < nb; j++) diag[i][j] = 0.0;
  double col[RtBounds<LMAX>::NAB];
  // (mu nu|mu nu) = sum_{abcd} T_a,mu T_b,nu T_c,mu T_d,nu (ab|cd)
  for (int c = 0; c < nca; c++)
    for (int d = 0; d < ncb; d++) {
      eri_column_rt<double, LMAX>(la, lb, la, lb, c, d, P, P, pp, boys, col);
      for (int mu = 0; mu < na; mu++) {
        const double tc = A.pure ? TA[c * nsph(la) + mu] : (c == mu ? 1.0 : 0.0);
        if (tc == 0.0) continue;
        for (int nu = 0; nu < nb; nu++) {
          const double td = B.pure ? TB[d * nsph(lb) + nu] : (d == nu ? 1.0 : 0.0);
          if (td == 0.0) continue;
          double s = 0.0;
          for (int ia = 0; ia < nca; ia++) {
            const double ta = A.pure ? TA[ia * nsph(la) + mu] : (ia == mu ? 1.0 : 0.0);
            if (ta == 0.0) continue;
            for (int ib = 0; ib < ncb; ib++) {
              const double tb = B.pure ? TB[ib * nsph(lb) + nu] : (ib == nu ? 1.0 : 0.0);
              s += ta * tb * col[ia * ncb + ib];
            }
          }
          diag[mu][nu] += tc * td * s;
        }
      }
    }
  // rows are the functions of s1 (the reference's first shell)
  const bool swp = P.shA != P.s1;
  double mx = 0.0;
  if (!swp) {
    for (int i = 0; i < na; i++) {
      double r = 0.0;
      for (int j = 0; j < nb; j++) r += fabs(diag[i][j]);
      mx = fmax(mx, r);
    }
  } else {
    for (int j = 0; j < nb; j++) {
      double r = 0.0;
      for (int i = 0; i < na; i++) r += fabs(diag[i][j]);
      mx = fmax(mx, r);
    }
  }
  const double q = sqrt(mx);
  pairsOut[beg + k].Q = q;
  Qtab[P.s1 + (size_t)P.s2 * nshell] = q;
  Qtab[P.s2 + (size_t)P.s1 * nshell] = q;
}

}  // namespace cqf
