// Contracted Cartesian shell-quartet ERIs by McMurchie-Davidson with runtime
// angular momenta (any class up to LMAX), one thread per quartet.  Replaces
// libint2::Engine::compute2<coulomb,xx_xx,0>
// (include/particleintegrals/contract/direct.hpp:1811-1820) on the device for
// every class; the hot classes of the closed-shell build have generated
// straight-line kernels instead (cqf_gen_*.cuh).
//
// The Cartesian-to-spherical transform is not done per quartet: densities are
// taken to the Cartesian AO basis once per build and the accumulated J/K are
// transformed back (cqf_api.cu), which is exact linear algebra.
//
// Work is done one ket component pair (c, d) at a time, so per-thread storage
// is E tables + R + one column of the block, bounded for every class.
#pragma once

#include "cqf_common.cuh"

namespace cqf {

// Hermite E tables of one primitive pair for runtime (la, lb):
// E[((i*(lb+1) + j)*(la+lb+1) + t)] per axis.
template <typename T, int LM>
__device__ __forceinline__ void hermite_E_rt(int la, int lb, T o2p, T PA, T PB, T* E) {
  const int L1 = la + lb + 1;
#pragma unroll 1
  for (int k = 0; k < (la + 1) * (lb + 1) * L1; k++) E[k] = T(0);
  E[0] = T(1);
#pragma unroll 1
  for (int i = 0; i <= la; i++)
#pragma unroll 1
    for (int j = 0; j <= lb; j++) {
      if (i == 0 && j == 0) continue;
      const bool up = (j == 0);
      const int pi = up ? i - 1 : i, pj = up ? j : j - 1;
      const T* Ep = E + (pi * (lb + 1) + pj) * L1;
      T* Eo = E + (i * (lb + 1) + j) * L1;
      const T X = up ? PA : PB;
      const int top = pi + pj;
#pragma unroll 1
      for (int t = 0; t <= i + j; t++) {
        T v = (t <= top) ? X * Ep[t] : T(0);
        if (t >= 1) v += o2p * Ep[t - 1];
        if (t + 1 <= top) v += T(t + 1) * Ep[t + 1];
        Eo[t] = v;
      }
    }
}

// R^{(0)}_tuv for t+u+v <= L into Rv (compact hidx order), in place.
template <typename T>
__device__ __forceinline__ void hermite_R_rt(int L, T alpha, T X, T Y, T Z, const T* F, T* Rv) {
  const T m2a = T(-2) * alpha;
  T fn = T(1);
#pragma unroll 1
  for (int n = 0; n < L; n++) fn *= m2a;
  Rv[0] = fn * F[L];
#pragma unroll 1
  for (int n = L - 1; n >= 0; n--) {
#pragma unroll 1
    for (int tot = L - n; tot >= 1; tot--) {
#pragma unroll 1
      for (int t = tot; t >= 0; t--) {
#pragma unroll 1
        for (int u = tot - t; u >= 0; u--) {
          const int v = tot - t - u;
          T val;
          if (t > 0) {
            val = X * Rv[hidx(t - 1, u, v)];
            if (t > 1) val += T(t - 1) * Rv[hidx(t - 2, u, v)];
          } else if (u > 0) {
            val = Y * Rv[hidx(0, u - 1, v)];
            if (u > 1) val += T(u - 1) * Rv[hidx(0, u - 2, v)];
          } else {
            val = Z * Rv[hidx(0, 0, v - 1)];
            if (v > 1) val += T(v - 1) * Rv[hidx(0, 0, v - 2)];
          }
          Rv[hidx(t, u, v)] = val;
        }
      }
    }
    fn = (n == 0) ? T(1) : fn / m2a;
    Rv[0] = fn * F[n];
  }
}

template <typename T>
__device__ __forceinline__ void boys_rt(int L, T Targ, T* F, const T* tab);

template <>
__device__ __forceinline__ void boys_rt<double>(int L, double T, double* F, const double* tab) {
  if (T < BOYS_TMAX) {
    int j = __double2int_rn(T * (1.0 / BOYS_DT));
    double dT = j * BOYS_DT - T;
    const double* row = tab + ((size_t)L * BOYS_NPTS + j) * BOYS_ROW64;
    double s = __ldg(row + BOYS_K64);
#pragma unroll
    for (int k = BOYS_K64 - 1; k >= 0; k--) s = __ldg(row + k) + s * dT * (1.0 / (k + 1));
    F[L] = s;
    double e = exp(-T), t2 = 2.0 * T;
#pragma unroll 1
    for (int m = L - 1; m >= 0; m--) F[m] = (t2 * F[m + 1] + e) / (2 * m + 1);
  } else {
    double rT = rsqrt(T);
    F[0] = 0.88622692545275801365 * rT;
    double e = exp(-T), h = 0.5 * rT * rT;
#pragma unroll 1
    for (int m = 0; m < L; m++) F[m + 1] = ((2 * m + 1) * F[m] - e) * h;
  }
}

template <>
__device__ __forceinline__ void boys_rt<float>(int L, float T, float* F, const float* tab) {
  if (T < (float)BOYS_TMAX) {
    int j = __float2int_rn(T * (float)(1.0 / BOYS_DT));
    float dT = j * (float)BOYS_DT - T;
    const float* row = tab + ((size_t)L * BOYS_NPTS + j) * BOYS_ROW32;
    float s = __ldg(row + BOYS_K32);
#pragma unroll
    for (int k = BOYS_K32 - 1; k >= 0; k--) s = __ldg(row + k) + s * dT * (1.0f / (k + 1));
    F[L] = s;
    float e = __expf(-T), t2 = 2.0f * T;
#pragma unroll 1
    for (int m = L - 1; m >= 0; m--) F[m] = (t2 * F[m + 1] + e) / (2 * m + 1);
  } else {
    // large arguments in FP64, as boys_f32 does: sqrt(pi / T) / 2 and the
    // upward recursion, with e^-T from the FP32 exponential (below 2e-16 here)
    const double Td = (double)T, rT = rsqrt(Td), h = 0.5 * rT * rT;
    const double e = (double)__expf(-T);
    double f = 0.88622692545275801365 * rT;
    F[0] = (float)f;
#pragma unroll 1
    for (int m = 0; m < L; m++) {
      f = ((2 * m + 1) * f - e) * h;
      F[m + 1] = (float)f;
    }
  }
}

// F_0 .. F_L spread over the lanes of one warp: below TMAX every order from
// its own table row (the Taylor sum boys_rt uses for F_L), above it lane 0
// runs boys_rt's upward recursion.  All 32 lanes call it; F is shared memory.
template <typename T>
__device__ __forceinline__ void boys_lanes(int L, T Targ, T* F, const T* tab, int lane);

template <>
__device__ __forceinline__ void boys_lanes<double>(int L, double T, double* F, const double* tab,
                                                   int lane) {
  if (T < BOYS_TMAX) {
    const int j = __double2int_rn(T * (1.0 / BOYS_DT));
    const double dT = j * BOYS_DT - T;
#pragma unroll 1
    for (int m = lane; m <= L; m += 32) {
      const double* row = tab + ((size_t)m * BOYS_NPTS + j) * BOYS_ROW64;
      double s = __ldg(row + BOYS_K64);
#pragma unroll
      for (int k = BOYS_K64 - 1; k >= 0; k--) s = __ldg(row + k) + s * dT * (1.0 / (k + 1));
      F[m] = s;
    }
  } else if (lane == 0) {
    boys_rt<double>(L, T, F, tab);
  }
  __syncwarp();
}

template <>
__device__ __forceinline__ void boys_lanes<float>(int L, float T, float* F, const float* tab,
                                                  int lane) {
  if (T < (float)BOYS_TMAX) {
    const int j = __float2int_rn(T * (float)(1.0 / BOYS_DT));
    const float dT = j * (float)BOYS_DT - T;
#pragma unroll 1
    for (int m = lane; m <= L; m += 32) {
      const float* row = tab + ((size_t)m * BOYS_NPTS + j) * BOYS_ROW32;
      float s = __ldg(row + BOYS_K32);
#pragma unroll
      for (int k = BOYS_K32 - 1; k >= 0; k--) s = __ldg(row + k) + s * dT * (1.0f / (k + 1));
      F[m] = s;
    }
  } else if (lane == 0) {
    boys_rt<float>(L, T, F, tab);
  }
  __syncwarp();
}

// sum_k f[k] H[hidx(t, u, v + k)] for k < n, the Hermite index stepped
// incrementally: hidx(t, u, v + 1) - hidx(t, u, v) = (s + 1)(s + 2) / 2 +
// (u + v) + 2 with s = t + u + v, and that step grows by s + 3 per k.
template <typename T>
__device__ __forceinline__ T hdot_v(const T* f, int n, const T* H, int t, int u, int v) {
  const int s = t + u + v;
  int idx = hidx(t, u, v);
  int inc = (s + 1) * (s + 2) / 2 + (u + v) + 2;
  T acc = T(0);
#pragma unroll 1
  for (int k = 0; k < n; k++) {
    acc += f[k] * H[idx];
    idx += inc;
    inc += s + k + 3;
  }
  return acc;
}

// Storage bounds for angular momenta up to LM per shell.
template <int LM>
struct RtBounds {
  static constexpr int E1 = (LM + 1) * (LM + 1) * (2 * LM + 1);  // one axis, one pair
  static constexpr int HL = nherm(4 * LM);
  static constexpr int HAB = nherm(2 * LM);
  static constexpr int NAB = ncart(LM) * ncart(LM);
};

// col[a*nb + b] = (ab|cd) for one ket component pair (c, d) of the canonical
// quartet (shA shB | shC shD).  T is the primitive arithmetic type (double,
// or float on the mixed path); the primitive sum is kept in double.
template <typename T, int LM>
__device__ void eri_column_rt(int la, int lb, int lc, int ld, int c, int d, const PairDev& P,
                              const PairDev& Q, const PrimPairDev* __restrict__ pp,
                              const T* __restrict__ boys, double* __restrict__ col) {
  using Bd = RtBounds<LM>;
  const int lab = la + lb, lcd = lc + ld, L = lab + lcd;
  const int na = ncart(la), nb = ncart(lb);
  const int cx = cart_lx(lc, c), cy = cart_ly(lc, c), cz = cart_lz(lc, c);
  const int dx = cart_lx(ld, d), dy = cart_ly(ld, d), dz = cart_lz(ld, d);
  const int Lcd1 = lcd + 1, Lab1 = lab + 1;
  const T PI52x2 = T(34.986836655249725693);  // 2 pi^(5/2)
#pragma unroll 1
  for (int i = 0; i < na * nb; i++) col[i] = 0.0;

  T Ea[3][Bd::E1], Ec[3][Bd::E1];
  T G[Bd::HAB];
  T Rv[Bd::HL];
  T F[4 * LM + 1];
#pragma unroll 1
  for (int ip = 0; ip < P.npp; ip++) {
    const PrimPairDev& A = pp[P.pp_off + ip];
    const T p = T(A.p), o2p = T(0.5) / p;
#pragma unroll 1
    for (int x = 0; x < 3; x++) hermite_E_rt<T, LM>(la, lb, o2p, T(A.PA[x]), T(A.PB[x]), Ea[x]);
    const int HAB = nherm(lab);
#pragma unroll 1
    for (int h = 0; h < HAB; h++) G[h] = T(0);
#pragma unroll 1
    for (int iq = 0; iq < Q.npp; iq++) {
      const PrimPairDev& B = pp[Q.pp_off + iq];
      const T q = T(B.p), o2q = T(0.5) / q;
#pragma unroll 1
      for (int x = 0; x < 3; x++) hermite_E_rt<T, LM>(lc, ld, o2q, T(B.PA[x]), T(B.PB[x]), Ec[x]);
      const T X = T(A.P[0]) - T(B.P[0]), Y = T(A.P[1]) - T(B.P[1]), Z = T(A.P[2]) - T(B.P[2]);
      const T pq = p + q, alpha = p * q / pq;
      const T Targ = alpha * (X * X + Y * Y + Z * Z);
      const T pref = PI52x2 / sqrt(pq) * T(A.Kp) * T(B.Kp);
      boys_rt<T>(L, Targ, F, boys);
      hermite_R_rt<T>(L, alpha, X, Y, Z, F, Rv);
      const T* ex = Ec[0] + (cx * (ld + 1) + dx) * Lcd1;
      const T* ey = Ec[1] + (cy * (ld + 1) + dy) * Lcd1;
      const T* ez = Ec[2] + (cz * (ld + 1) + dz) * Lcd1;
      // the ket's (-1)^(tau + nu + phi): phi's in ezs, tau's and nu's in exy
      T ezs[2 * LM + 1];
#pragma unroll 1
      for (int ph = 0; ph <= cz + dz; ph++) ezs[ph] = (ph & 1) ? -ez[ph] : ez[ph];
#pragma unroll 1
      for (int t = 0; t <= lab; t++)
#pragma unroll 1
        for (int u = 0; u <= lab - t; u++)
#pragma unroll 1
          for (int v = 0; v <= lab - t - u; v++) {
            T s = T(0);
#pragma unroll 1
            for (int ta = 0; ta <= cx + dx; ta++)
#pragma unroll 1
              for (int nu = 0; nu <= cy + dy; nu++) {
                const T exy = ((ta + nu) & 1) ? -(ex[ta] * ey[nu]) : ex[ta] * ey[nu];
                s += exy * hdot_v(ezs, cz + dz + 1, Rv, t + ta, u + nu, v);
              }
            G[hidx(t, u, v)] += pref * s;
          }
    }
#pragma unroll 1
    for (int a = 0; a < na; a++) {
      const int ax = cart_lx(la, a), ay = cart_ly(la, a), az = cart_lz(la, a);
#pragma unroll 1
      for (int b = 0; b < nb; b++) {
        const int bx = cart_lx(lb, b), by = cart_ly(lb, b), bz = cart_lz(lb, b);
        const T* fx = Ea[0] + (ax * (lb + 1) + bx) * Lab1;
        const T* fy = Ea[1] + (ay * (lb + 1) + by) * Lab1;
        const T* fz = Ea[2] + (az * (lb + 1) + bz) * Lab1;
        T s = T(0);
#pragma unroll 1
        for (int t = 0; t <= ax + bx; t++)
#pragma unroll 1
          for (int u = 0; u <= ay + by; u++)
            s += fx[t] * fy[u] * hdot_v(fz, az + bz + 1, G, t, u, 0);
        col[a * nb + b] += double(s);
      }
    }
  }
}

}  // namespace cqf
