// Shared device-side definitions of the direct J/K build (sm_100a).
//
// Data layout in HBM (one cqf_basis):
//   ShellDev[nshell]       shell metadata (l, pure, primitive/AO offsets, centre)
//   PairDev[npair]         significant shell pairs (ShellPairData semantics,
//                          src/basisset/basisset.cxx:652-706), grouped into
//                          angular-momentum classes (lA >= lB), inside each
//                          class sorted by primitive-pair count, then by
//                          Schwarz bound (both descending)
//   PrimPairDev[nprimpair] primitive-pair data (p, K/p, 1/2p, P, PA, PB,
//                          primitive indices), 112 B each, contiguous per
//                          shell pair in descending order of the primitive
//                          Schwarz bound (ppQ[nprimpair]); the same
//                          data tile-interleaved (field-major runs of 128
//                          kets) for the class kernels' per-lane ket loads
//   bra groups             per class a bra order by first shell, cut into
//                          groups (grouped class kernels)
//   boys tables            per angular sum L and grid point T_j = j*0.1 one
//                          row {F_L..F_{L+8}(T_j), exp(-T_j)}: 80 B, 16-B
//                          aligned, read with five 128-bit loads (FP64); FP32
//                          rows {F_L..F_{L+5}, exp(-T_j), 0}: 32 B.  The
//                          29 KB (FP64) / 11.6 KB (FP32) of one L are read
//                          through L1; one copy per device for all bases.
//   Cartesian-AO densities / accumulators, nMat x ncart x ncart
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace cqf {

constexpr int LMAX = 3;            // highest shell angular momentum (f)
constexpr double SPEED_OF_LIGHT = 137.035999074;  // atomic units (include/physcon.hpp:40)
constexpr int BOYS_MMAX = 40;      // orders of the host-side generation
constexpr double BOYS_DT = 0.1;    // grid spacing of the Taylor tables
constexpr double BOYS_TMAX = 36.0; // above: F0 = sqrt(pi/T)/2 + upward recursion
constexpr int BOYS_NPTS = 362;     // grid points 0 .. TMAX/DT (+ margin)
constexpr int BOYS_LTAB = 24;      // per-L rows exist for L = 0..BOYS_LTAB
constexpr int BOYS_K64 = 8;        // FP64 Taylor terms k = 0..8, |dT| <= 0.05:
                                   // remainder <= 0.05^9/9! = 5e-18 relative
constexpr int BOYS_K32 = 5;        // FP32 Taylor terms k = 0..5 (2e-11 relative)
constexpr int BOYS_ROW64 = 10;     // FP64 row: F_L..F_{L+8}, exp(-T_j)  (80 B)
constexpr int BOYS_ROW32 = 8;      // FP32 row: F_L..F_{L+5}, exp(-T_j), 0 (32 B)
// bytes of the rows of one L (what a block stages in shared memory)
constexpr int BOYS_LBYTES64 = BOYS_NPTS * BOYS_ROW64 * 8;
constexpr int BOYS_LBYTES32 = BOYS_NPTS * BOYS_ROW32 * 4;

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int nsph(int l) { return 2 * l + 1; }
// number of Hermite functions with t+u+v <= L
__host__ __device__ constexpr int nherm(int L) {
  return L < 0 ? 0 : (L + 1) * (L + 2) * (L + 3) / 6;
}
// compact Hermite index: blocks of equal t+u+v, inside a block t descending,
// then u descending (v ascending)
__host__ __device__ constexpr int hidx(int t, int u, int v) {
  return nherm(t + u + v - 1) + (u + v) * (u + v + 1) / 2 + v;
}
// Cartesian exponents of component i of an l shell (libint / CCA order):
// i = a (a + 1) / 2 + b runs over a = 0 .. l, b = 0 .. a with
// (lx, ly, lz) = (l - a, a - b, b).  The row a of i by comparisons with the
// triangular numbers (components of l <= 8).
__host__ __device__ constexpr int cart_row(int i) {
  return (i >= 1) + (i >= 3) + (i >= 6) + (i >= 10) + (i >= 15) + (i >= 21) + (i >= 28) +
         (i >= 36);
}
__host__ __device__ constexpr int cart_lz(int l, int i) {
  return i - cart_row(i) * (cart_row(i) + 1) / 2;
}
__host__ __device__ constexpr int cart_lx(int l, int i) { return l - cart_row(i); }
__host__ __device__ constexpr int cart_ly(int l, int i) { return cart_row(i) - cart_lz(l, i); }

struct __align__(16) ShellDev {
  int l, pure, nprim, prim_off;
  int cart_off, sph_off, pad0, pad1;
  double O[3];
};

// One significant shell pair.  (shA, shB) is the order the ERI kernels use
// (l(shA) >= l(shB)); (s1, s2) is the reference loop order (s1 >= s2).
struct __align__(16) PairDev {
  int shA, shB, s1, s2;
  int cA, cB;        // Cartesian AO offsets of shA / shB
  int lex;           // rank of (s1, s2) in the reference loop order
  int pp_off;        // first primitive pair
  int npp;           // number of primitive pairs
  int cls;           // class id (lA, lB)
  double Q;          // Schwarz bound sqrt(||(ab|ab) diag||_inf)
};

struct __align__(16) PrimPairDev {
  double p, Kp;      // exponent sum; c_a c_b exp(-mu |AB|^2) / p
  double P[3], PA[3], PB[3];
  double o2p;        // 1 / (2p)
  int ia, ib;        // primitive indices within shells shA and shB
};

// FP32 copy of a primitive pair's data for the FP32 class kernels.
struct __align__(16) PrimPair32 {
  float p, Kp;
  float P[3], PA[3], PB[3];
  float o2p;
};

// FP32 range guard of the mixed path.  The Hermite recursion starts from
// R^(n)_000 = (-2 alpha)^n F_n(T), n <= L, so its intermediates reach
// (2 alpha)^L; alpha = pq / (p + q) <= min(p, q).  Tight primitives (core
// shells of heavy atoms, exponents 1e4 .. 1e8) push that past FP32's 2^128
// at moderate L, and F_n underflows at the same time (inf * 0 = NaN), while
// FP64's range holds.  A quartet may run in FP32 only when
//   L log2(2 min(p, q))                                 <= 100, and
//   that + log2 max|Kp| + log2 max|Kq| + 2 dP log2(2p) + 2 dQ log2(2q) <= 110
// with p, q the pairs' largest primitive exponent sums and dP, dQ = 1 for a
// pair carrying the two derivative factors of a small-component bra or ket
// (each up to 2p).  r.x = log2(2 max p), r.y = log2(max |Kp|) per pair.
__device__ __forceinline__ bool fp32_range_ok(float2 rP, float2 rQ, int L, int dP, int dQ) {
  const float lr = (float)L * fmaxf(fminf(rP.x, rQ.x), 0.f);
  const float ld = 2.f * ((float)dP * fmaxf(rP.x, 0.f) + (float)dQ * fmaxf(rQ.x, 0.f));
  return lr <= 100.f && lr + rP.y + rQ.y + ld <= 110.f;
}

// ----------------------------------------------------------------- Boys
// F_0..F_L at T.  Taylor expansion of F_L about the nearest grid point
// (F_m' = -F_{m+1}), downward recursion F_m = (2T F_{m+1} + e^-T)/(2m+1);
// for T >= TMAX, F_0 = sqrt(pi/T)/2 and upward recursion keeping e^-T --
// evaluated in FP64 by both precisions (boys_f32 rounds the result).
// `rows` points at the rows of this L (global or shared memory).
template <int L>
__device__ __forceinline__ void boys_f64(double T, double* F, const double* __restrict__ rows) {
  if (T < BOYS_TMAX) {
    const int j = __double2int_rn(T * (1.0 / BOYS_DT));
    const double dT = j * BOYS_DT - T;
    const double2* row = reinterpret_cast<const double2*>(rows + j * BOYS_ROW64);
    const double2 r0 = row[0], r1 = row[1], r2 = row[2], r3 = row[3], r4 = row[4];
    // Taylor of F_L about T_j (F_m' = -F_{m+1}), terms k = 0..8
    double s = r4.x;
    s = r3.y + s * dT * (1.0 / 8);
    s = r3.x + s * dT * (1.0 / 7);
    s = r2.y + s * dT * (1.0 / 6);
    s = r2.x + s * dT * (1.0 / 5);
    s = r1.y + s * dT * (1.0 / 4);
    s = r1.x + s * dT * (1.0 / 3);
    s = r0.y + s * dT * (1.0 / 2);
    s = r0.x + s * dT;
    F[L] = s;
    if (L > 0) {
      // exp(-T) = exp(-T_j) exp(dT), |dT| <= DT/2, Taylor to dT^9
      double e = 1.0 + dT * (1.0 / 9);
#pragma unroll
      for (int k = 8; k >= 1; k--) e = 1.0 + dT * e * (1.0 / k);
      e *= r4.y;
      const double t2 = 2.0 * T;
#pragma unroll
      for (int m = L - 1; m >= 0; m--) F[m] = (t2 * F[m + 1] + e) * (1.0 / (2 * m + 1));
    }
  } else {
    double rT = rsqrt(T);
    F[0] = 0.88622692545275801365 * rT;  // sqrt(pi)/2
    if (L > 0) {
      double e = exp(-T), h = 0.5 * rT * rT;
#pragma unroll
      for (int m = 0; m < L; m++) F[m + 1] = ((2 * m + 1) * F[m] - e) * h;
    }
  }
}

template <int L>
__device__ __forceinline__ void boys_f32(float T, float* F, const float* __restrict__ rows) {
  if (T < (float)BOYS_TMAX) {
    const int j = __float2int_rn(T * (float)(1.0 / BOYS_DT));
    const float dT = j * (float)BOYS_DT - T;
    const float4* row = reinterpret_cast<const float4*>(rows + j * BOYS_ROW32);
    const float4 r0 = row[0], r1 = row[1];
    float s = r1.y;
    s = r1.x + s * dT * (1.0f / 5);
    s = r0.w + s * dT * (1.0f / 4);
    s = r0.z + s * dT * (1.0f / 3);
    s = r0.y + s * dT * (1.0f / 2);
    s = r0.x + s * dT;
    F[L] = s;
    if (L > 0) {
      const float e =
          r1.z * (1.0f + dT * (1.0f + dT * (0.5f + dT * ((1.0f / 6) + dT * (1.0f / 24)))));
      const float t2 = 2.0f * T;
#pragma unroll
      for (int m = L - 1; m >= 0; m--) F[m] = (t2 * F[m + 1] + e) * (1.0f / (2 * m + 1));
    }
  } else {
    // large arguments in FP64 (the asymptotic form and its upward recursion
    // lose accuracy in FP32 as (2m+1)/(2T) factors accumulate), then rounded;
    // e^-T <= 2.3e-16 enters the recursion only as a correction, so its FP32
    // value (relative error ~1e-7) is exact enough
    const double Td = (double)T;
    const double rT = rsqrt(Td);
    double f = 0.88622692545275801365 * rT;  // sqrt(pi)/2
    F[0] = (float)f;
    if (L > 0) {
      const double e = (double)__expf(-T), h = 0.5 * rT * rT;
#pragma unroll
      for (int m = 0; m < L; m++) {
        f = ((2 * m + 1) * f - e) * h;
        F[m + 1] = (float)f;
      }
    }
  }
}

// -------------------------------------------------- Hermite coefficients
// E^{ij}_t for one axis (McMurchie-Davidson; Helgaker eq. 9.5.6) without the
// Gaussian-product factor.  E[i][j][t], t <= i + j.
template <typename R, int LA, int LB>
__device__ __forceinline__ void hermite_E(R o2p, R PA, R PB, R (&E)[LA + 1][LB + 1][LA + LB + 1]) {
#pragma unroll
  for (int i = 0; i <= LA; i++)
#pragma unroll
    for (int j = 0; j <= LB; j++)
#pragma unroll
      for (int t = 0; t <= LA + LB; t++) E[i][j][t] = R(0);
  E[0][0][0] = R(1);
#pragma unroll
  for (int i = 1; i <= LA; i++)
#pragma unroll
    for (int t = 0; t <= i; t++) {
      R v = PA * (t <= i - 1 ? E[i - 1][0][t] : R(0));
      if (t >= 1) v += o2p * E[i - 1][0][t - 1];
      if (t + 1 <= i - 1) v += R(t + 1) * E[i - 1][0][t + 1];
      E[i][0][t] = v;
    }
#pragma unroll
  for (int i = 0; i <= LA; i++)
#pragma unroll
    for (int j = 1; j <= LB; j++)
#pragma unroll
      for (int t = 0; t <= i + j; t++) {
        R v = PB * (t <= i + j - 1 ? E[i][j - 1][t] : R(0));
        if (t >= 1) v += o2p * E[i][j - 1][t - 1];
        if (t + 1 <= i + j - 1) v += R(t + 1) * E[i][j - 1][t + 1];
        E[i][j][t] = v;
      }
}

// -------------------------------------------------- Hermite integrals R_tuv
// In-place downward sweep over the auxiliary index n (see hidx ordering):
// R^{(n)}_{t+1,u,v} = t R^{(n+1)}_{t-1,u,v} + X_PQ R^{(n+1)}_{t,u,v}, etc.
// On entry F[0..L] holds the Boys values; on exit R[hidx(t,u,v)] = R^{(0)}_tuv.
template <typename R, int L>
__device__ __forceinline__ void hermite_R(R alpha, R X, R Y, R Z, const R* F, R* Rv) {
  R m2a = R(-2) * alpha;
  R f[L + 1];
  f[0] = R(1);
#pragma unroll
  for (int n = 1; n <= L; n++) f[n] = f[n - 1] * m2a;
  Rv[0] = f[L] * F[L];
#pragma unroll
  for (int n = L - 1; n >= 0; n--) {
#pragma unroll
    for (int tot = L - n; tot >= 1; tot--) {
#pragma unroll
      for (int t = tot; t >= 0; t--) {
#pragma unroll
        for (int u = tot - t; u >= 0; u--) {
          const int v = tot - t - u;
          R val;
          if (t > 0) {
            val = X * Rv[hidx(t - 1, u, v)];
            if (t > 1) val += R(t - 1) * Rv[hidx(t - 2, u, v)];
          } else if (u > 0) {
            val = Y * Rv[hidx(0, u - 1, v)];
            if (u > 1) val += R(u - 1) * Rv[hidx(0, u - 2, v)];
          } else {
            val = Z * Rv[hidx(0, 0, v - 1)];
            if (v > 1) val += R(v - 1) * Rv[hidx(0, 0, v - 2)];
          }
          Rv[hidx(t, u, v)] = val;
        }
      }
    }
    Rv[0] = f[n] * F[n];
  }
}

}  // namespace cqf
