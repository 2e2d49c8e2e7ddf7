// Derivative ERI building blocks shared by the four-component kernels
// (cqf_rel.cu) and the nuclear-gradient contraction (cqf_grad.cu):
// McMurchie-Davidson over a primitive pair's Hermite tables raised by one on
// both centres, with d/dx on either centre of each pair,
//     d/dx [x^i e^{-a x^2}] = i x^{i-1} e^{-a x^2} - 2a x^{i+1} e^{-a x^2}.
#pragma once

#include "cqf_eri.cuh"

namespace cqf {

// ------------------------------------------------------- derivative ERIs
// One Cartesian axis of a primitive pair as a Hermite expansion, with d/dx
// on the first centre (type bit 0) and / or the second (bit 1).  E is the
// pair's table raised by one on both centres when a derivative is taken:
// E[(i * (l2r + 1) + j) * Lr + t].  Returns the length (t = 0 .. n-1).
template <typename T>
__device__ __forceinline__ int axis_factor(const T* E, int l2r, int Lr, int i, int j, int type,
                                           T a2, T b2, T* f) {
  const int dA = type & 1, dB = (type >> 1) & 1;
  const int n = i + j + dA + dB + 1;
  auto e = [&](int ii, int jj, int t) -> T {
    return (ii < 0 || jj < 0 || t > ii + jj) ? T(0) : E[(ii * (l2r + 1) + jj) * Lr + t];
  };
#pragma unroll 1
  for (int t = 0; t < n; t++) {
    T v;
    if (type == 0) v = e(i, j, t);
    else if (type == 1) v = T(i) * e(i - 1, j, t) - a2 * e(i + 1, j, t);
    else if (type == 2) v = T(j) * e(i, j - 1, t) - b2 * e(i, j + 1, t);
    else
      v = T(i * j) * e(i - 1, j - 1, t) - b2 * T(i) * e(i - 1, j + 1, t) -
          a2 * T(j) * e(i + 1, j - 1, t) + a2 * b2 * e(i + 1, j + 1, t);
    f[t] = v;
  }
  return n;
}

// G[tuv] += s * sum f_x[tau] f_y[nu] f_z[phi] R_{t+tau+sx,u+nu+sy,v+phi+sz}
// for t+u+v <= Lb; the ket factors carry the (-1)^(tau+nu+phi) sign
// already; (sx, sy, sz): the Hermite shift of an operator derivative.
template <typename T>
__device__ __forceinline__ void ket_add(T* G, T s, const T* fx, int nx, const T* fy, int ny,
                                        const T* fz, int nz, int Lb, const T* Rv, int sx = 0,
                                        int sy = 0, int sz = 0) {
#pragma unroll 1
  for (int t = 0; t <= Lb; t++)
#pragma unroll 1
    for (int u = 0; u <= Lb - t; u++)
#pragma unroll 1
      for (int v = 0; v <= Lb - t - u; v++) {
        T acc = T(0);
#pragma unroll 1
        for (int a = 0; a < nx; a++) {
          const T fa = fx[a];
          if (fa == T(0)) continue;
#pragma unroll 1
          for (int b = 0; b < ny; b++) {
            const T fab = fa * fy[b];
            if (fab == T(0)) continue;
            acc += fab * hdot_v(fz, nz, Rv, t + a + sx, u + b + sy, v + sz);
          }
        }
        G[hidx(t, u, v)] += s * acc;
      }
}

template <typename T>
__device__ __forceinline__ T bra_dot(const T* gx, int nx, const T* gy, int ny, const T* gz,
                                     int nz, const T* G) {
  T s = T(0);
#pragma unroll 1
  for (int t = 0; t < nx; t++) {
    if (gx[t] == T(0)) continue;
#pragma unroll 1
    for (int u = 0; u < ny; u++) {
      const T gxy = gx[t] * gy[u];
      if (gxy == T(0)) continue;
      s += gxy * hdot_v(gz, nz, G, t, u, 0);
    }
  }
  return s;
}

// operator component of the derivative pair (mu on the first centre, nu on
// the second): dot (0) or cross x / y / z (1..3), with its sign
__device__ __forceinline__ void op_of(int mu, int nu, int& op, double& sg) {
  if (mu == nu) {
    op = 0;
    sg = 1.0;
  } else {
    op = 3 - mu - nu + 1;
    sg = (nu == (mu + 1) % 3) ? 1.0 : -1.0;
  }
}

// exponents of the two primitives of primitive pair r (its primitive
// indices within shells SA and SB)
__device__ __forceinline__ void pair_exps(const ShellDev& SA, const ShellDev& SB,
                                          const double* __restrict__ prim,
                                          const PrimPairDev& r, double& ea, double& eb) {
  ea = __ldg(prim + SA.prim_off + r.ia);
  eb = __ldg(prim + SB.prim_off + r.ib);
}

constexpr double PI52X2 = 34.986836655249725693;  // 2 pi^(5/2)

// the symmetric operator-derivative pairs (i, i'), i <= i': xx, xy, xz, yy,
// yz, zz
__host__ __device__ __forceinline__ void op_pair(int k, int& i, int& ip) {
  i = (k >= 3) + (k >= 5);
  ip = k - (i == 0 ? 0 : (i == 1 ? 2 : 3));
}

// The kernel r12 in place of 1 / r12: the Hermite integrals are the
// R = P - Q derivatives of the Coulomb prefactor / (2 alpha) times
// f(T) = e^-T + (1 + 2T) F_0(T) (the mean of |r| under the Gaussian of the
// pair product), f' = F_0 - F_1, f^(n) = (-1)^(n-1) (F_(n-1) - F_n); the
// McMurchie-Davidson recursion then runs on Ft_0 = f, Ft_n = F_n - F_(n-1)
// (replaces F_0..F_L in place).  An operator derivative d_i d_j r12
// (derivatives in r = r1 - r2) shifts the Hermite index by e_i + e_j.
__device__ __forceinline__ void r12_aux(int L, double T, double* F) {
#pragma unroll 1
  for (int n = L; n >= 1; n--) F[n] -= F[n - 1];
  F[0] = exp(-T) + (1.0 + 2.0 * T) * F[0];
}

}  // namespace cqf
