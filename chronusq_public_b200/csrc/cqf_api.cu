// C ABI of the direct J/K build: basis set-up on the device and the
// contraction driver (GTODirectTPIContraction::twoBodyContract replacement).
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <map>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cqf_internal.hpp"
#include "cqf_jk_fast.cuh"
#include "cqf_jk_kernels.cuh"

using namespace cqf;

namespace {

thread_local std::string g_err;

}  // namespace

namespace cqf {
cqf_status fail(cqf_status s, const std::string& msg) {
  g_err = msg;
  return s;
}
}  // namespace cqf

namespace {

#define CQF_CUDA(call)                                                                 \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(e_ == cudaErrorMemoryAllocation ? CQF_ENOMEM : CQF_ECUDA,            \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                 \
  } while (0)

#define CQF_TRY(expr)              \
  do {                             \
    cqf_status s_ = (expr);        \
    if (s_ != CQF_OK) return s_;   \
  } while (0)

// ------------------------------------------------------------ host tables
// Boys table F_m(j*DT), m = 0..BOYS_MMAX, by the convergent series in long
// double followed by downward recursion (the table scheme of
// RealGTOIntEngine::generateFmTTable, src/particleintegrals/aointegrals/
// aointegrals_onee_inhouse.cxx:79-116, with a tighter series tolerance).
void make_boys_table(std::vector<double>& t64, std::vector<float>& t32) {
  const int M = BOYS_MMAX;
  t64.assign((size_t)(BOYS_LTAB + 1) * BOYS_NPTS * BOYS_ROW64, 0.0);
  t32.assign((size_t)(BOYS_LTAB + 1) * BOYS_NPTS * BOYS_ROW32, 0.0f);
  std::vector<long double> col(M + 1);
  for (int j = 0; j < BOYS_NPTS; j++) {
    long double T = (long double)j * BOYS_DT;
    long double term = 1.0L / (2 * M + 1), sum = term;
    for (int k = 1; k < 10000; k++) {
      term *= 2.0L * T / (2 * M + 2 * k + 1);
      sum += term;
      if (term < sum * 1e-21L) break;
    }
    long double eT = expl(-T);
    col[M] = eT * sum;
    for (int m = M - 1; m >= 0; m--) col[m] = (2.0L * T * col[m + 1] + eT) / (2 * m + 1);
    for (int L = 0; L <= BOYS_LTAB; L++) {
      double* r64 = &t64[((size_t)L * BOYS_NPTS + j) * BOYS_ROW64];
      float* r32 = &t32[((size_t)L * BOYS_NPTS + j) * BOYS_ROW32];
      for (int k = 0; k <= BOYS_K64; k++) r64[k] = (double)col[L + k];
      r64[BOYS_K64 + 1] = (double)eT;
      for (int k = 0; k <= BOYS_K32; k++) r32[k] = (float)col[L + k];
      r32[BOYS_K32 + 1] = (float)eT;
    }
  }
}

double fact(int n) {
  double r = 1;
  for (int i = 2; i <= n; i++) r *= i;
  return r;
}
double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1;
  for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
  return r;
}

// Real solid harmonics over Cartesian components (Helgaker, Jorgensen &
// Olsen eq. 6.4.47-6.4.50), m = -l..l; T[ic * (2l+1) + (m+l)].
std::vector<double> solid_harmonics(int l) {
  int nc = ncart(l), ns = 2 * l + 1;
  std::vector<double> T(nc * ns, 0.0);
  for (int m = -l; m <= l; m++) {
    int am = std::abs(m), vm2 = (m >= 0) ? 0 : 1;
    double N = 1.0 / (std::pow(2.0, am) * fact(l)) *
               std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
    for (int t = 0; t <= (l - am) / 2; t++)
      for (int u = 0; u <= t; u++) {
        int vmax2 = 2 * (int)std::floor(am / 2.0 - vm2 / 2.0) + vm2;
        for (int v2 = vm2; v2 <= vmax2; v2 += 2) {
          int sg = t + (v2 - vm2) / 2;
          double C = ((sg % 2) ? -1.0 : 1.0) * std::pow(0.25, t) * binom(l, t) *
                     binom(l - t, am + t) * binom(t, u) * binom(am, v2);
          int ex = 2 * t + am - (2 * u + v2), ey = 2 * u + v2, ez = l - 2 * t - am;
          for (int i = 0; i < nc; i++)
            if (cart_lx(l, i) == ex && cart_ly(l, i) == ey && cart_lz(l, i) == ez)
              T[i * ns + (m + l)] += N * C;
        }
      }
  }
  return T;
}

// ------------------------------------------------------------ set-up kernels
// Cartesian overlap and kinetic blocks of two contracted shells from the 1D
// Hermite coefficients E^{ij}_0 (McMurchie-Davidson); kinetic by
// T_ij = -2b^2 S_{i,j+2} + b(2j+1) S_{ij} - j(j-1)/2 S_{i,j-2} per axis.
__device__ void shell_pair_1e(const ShellDev& A, const ShellDev& B, const double* __restrict__ prim,
                              int nprimTot, double (*S)[ncart(LMAX)], double (*T)[ncart(LMAX)]) {
  double AB2 = 0.0;
  for (int x = 0; x < 3; x++) AB2 += (A.O[x] - B.O[x]) * (A.O[x] - B.O[x]);
  const int na = ncart(A.l), nb = ncart(B.l);
  for (int i = 0; i < na; i++)
    for (int j = 0; j < nb; j++) {
      S[i][j] = 0.0;
      if (T) T[i][j] = 0.0;
    }
  const int lb2 = B.l + 2;
  for (int ia = 0; ia < A.nprim; ia++)
    for (int jb = 0; jb < B.nprim; jb++) {
      const double a = prim[A.prim_off + ia], b = prim[B.prim_off + jb];
      const double ca = prim[nprimTot + A.prim_off + ia], cb = prim[nprimTot + B.prim_off + jb];
      const double p = a + b, mu = a * b / p;
      const double K = ca * cb * exp(-mu * AB2) * pow(M_PI / p, 1.5);
      double s1d[3][LMAX + 1][LMAX + 3];
      for (int x = 0; x < 3; x++) {
        const double P = (a * A.O[x] + b * B.O[x]) / p;
        const double PA = P - A.O[x], PB = P - B.O[x], o2p = 0.5 / p;
        double E[LMAX + 1][LMAX + 3][2 * LMAX + 3];
        for (int i = 0; i <= A.l; i++)
          for (int j = 0; j <= lb2; j++)
            for (int t = 0; t <= i + j; t++) E[i][j][t] = 0.0;
        E[0][0][0] = 1.0;
        for (int i = 0; i <= A.l; i++)
          for (int j = 0; j <= lb2; j++) {
            if (i == 0 && j == 0) continue;
            const bool up = (j == 0);
            const int pi = up ? i - 1 : i, pj = up ? j : j - 1, top = pi + pj;
            const double X = up ? PA : PB;
            for (int t = 0; t <= i + j; t++) {
              double v = (t <= top) ? X * E[pi][pj][t] : 0.0;
              if (t > 0) v += o2p * E[pi][pj][t - 1];
              if (t + 1 <= top) v += (t + 1) * E[pi][pj][t + 1];
              E[i][j][t] = v;
            }
          }
        for (int i = 0; i <= A.l; i++)
          for (int j = 0; j <= lb2; j++) s1d[x][i][j] = E[i][j][0];
      }
      for (int u = 0; u < na; u++)
        for (int v = 0; v < nb; v++) {
          const int ia3[3] = {cart_lx(A.l, u), cart_ly(A.l, u), cart_lz(A.l, u)};
          const int jb3[3] = {cart_lx(B.l, v), cart_ly(B.l, v), cart_lz(B.l, v)};
          double s[3], t[3];
          for (int x = 0; x < 3; x++) {
            const int i = ia3[x], j = jb3[x];
            s[x] = s1d[x][i][j];
            t[x] = -2.0 * b * b * s1d[x][i][j + 2] + b * (2 * j + 1) * s1d[x][i][j] -
                   (j >= 2 ? 0.5 * j * (j - 1) * s1d[x][i][j - 2] : 0.0);
          }
          S[u][v] += K * s[0] * s[1] * s[2];
          if (T) T[u][v] += K * (t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2]);
        }
    }
}

// Spherical (where pure) element (mu, nu) of a Cartesian block.
__device__ double sph_elem(const ShellDev& A, const ShellDev& B, const double* __restrict__ sph,
                           const int* __restrict__ sphOff, double (*M)[ncart(LMAX)], int mu,
                           int nu) {
  const int na = ncart(A.l), nb = ncart(B.l);
  const double* TA = sph + sphOff[A.l];
  const double* TB = sph + sphOff[B.l];
  double s = 0.0;
  for (int u = 0; u < na; u++) {
    const double ta = A.pure ? TA[u * nsph(A.l) + mu] : (u == mu);
    if (ta == 0.0) continue;
    for (int v = 0; v < nb; v++) {
      const double tb = B.pure ? TB[v * nsph(B.l) + nu] : (v == nu);
      s += ta * tb * M[u][v];
    }
  }
  return s;
}

// Significant shell pairs: same centre (1e-5 Bohr per coordinate), or the
// 2-norm of the overlap block >= 1e-12 (basisset.cxx:146-156, :652-706).
__global__ void sig_pairs_kernel(const ShellDev* __restrict__ sh, const double* __restrict__ prim,
                                 const double* __restrict__ sph, const int* __restrict__ sphOff,
                                 int nshell, int nprimTot, unsigned char* flags) {
  long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long npair = (long long)nshell * (nshell + 1) / 2;
  if (k >= npair) return;
  int s1 = (int)((sqrt(8.0 * k + 1.0) - 1.0) / 2.0);
  while ((long long)s1 * (s1 + 1) / 2 > k) s1--;
  while ((long long)(s1 + 1) * (s1 + 2) / 2 <= k) s1++;
  int s2 = (int)(k - (long long)s1 * (s1 + 1) / 2);
  const ShellDev A = sh[s1], B = sh[s2];
  bool same = fabs(A.O[0] - B.O[0]) < 1e-5 && fabs(A.O[1] - B.O[1]) < 1e-5 &&
              fabs(A.O[2] - B.O[2]) < 1e-5;
  if (same) { flags[k] = 1; return; }
  double S[ncart(LMAX)][ncart(LMAX)];
  shell_pair_1e(A, B, prim, nprimTot, S, nullptr);
  const int ma = A.pure ? nsph(A.l) : ncart(A.l), mb = B.pure ? nsph(B.l) : ncart(B.l);
  double n2 = 0.0;
  for (int mu = 0; mu < ma; mu++)
    for (int nu = 0; nu < mb; nu++) {
      const double s = sph_elem(A, B, sph, sphOff, S, mu, nu);
      n2 += s * s;
    }
  flags[k] = sqrt(n2) >= 1e-12 ? 1 : 0;
}

// Full overlap and kinetic matrices (column-major N x N), one thread per
// shell pair block.
__global__ void one_electron_kernel(const ShellDev* __restrict__ sh, const double* __restrict__ prim,
                                    const double* __restrict__ sph, const int* __restrict__ sphOff,
                                    int nshell, int nprimTot, int N, double* Smat, double* Tmat) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nshell * nshell) return;
  const int s1 = k % nshell, s2 = k / nshell;
  const ShellDev A = sh[s1], B = sh[s2];
  double S[ncart(LMAX)][ncart(LMAX)], T[ncart(LMAX)][ncart(LMAX)];
  shell_pair_1e(A, B, prim, nprimTot, S, T);
  const int ma = A.pure ? nsph(A.l) : ncart(A.l), mb = B.pure ? nsph(B.l) : ncart(B.l);
  for (int mu = 0; mu < ma; mu++)
    for (int nu = 0; nu < mb; nu++) {
      const size_t e = (size_t)(A.sph_off + mu) + (size_t)(B.sph_off + nu) * N;
      Smat[e] = sph_elem(A, B, sph, sphOff, S, mu, nu);
      Tmat[e] = sph_elem(A, B, sph, sphOff, T, mu, nu);
    }
}

// Nuclear-attraction matrix (column-major N x N), one thread per shell-pair
// block: V_ab = -sum_C Z_C (2 pi / p) f sum_tuv E^x_t E^y_u E^z_v R_tuv(a', P - C)
// per primitive pair (McMurchie-Davidson); point nucleus a' = p, f = 1;
// Gaussian charge of exponent zeta a' = p zeta / (p + zeta),
// f = sqrt(zeta / (p + zeta)).  nuc[5 c ..] = {Z, x, y, z, zeta}.
__global__ void nuclear_kernel(const ShellDev* __restrict__ sh, const double* __restrict__ prim,
                               const double* __restrict__ sph, const int* __restrict__ sphOff,
                               int nshell, int nprimTot, int N, int natom,
                               const double* __restrict__ nuc, const double* __restrict__ boys,
                               double* Vmat) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nshell * nshell) return;
  const int s1 = k % nshell, s2 = k / nshell;
  const ShellDev A = sh[s1], B = sh[s2];
  const int la = A.l, lb = B.l, L = la + lb, L1 = L + 1;
  const int na = ncart(la), nb = ncart(lb);
  constexpr int E1 = (LMAX + 1) * (LMAX + 1) * (2 * LMAX + 1);
  double V[ncart(LMAX)][ncart(LMAX)];
  for (int i = 0; i < na; i++)
    for (int j = 0; j < nb; j++) V[i][j] = 0.0;
  double AB2 = 0.0;
  for (int x = 0; x < 3; x++) AB2 += (A.O[x] - B.O[x]) * (A.O[x] - B.O[x]);
  double E[3][E1], F[2 * LMAX + 1], R[nherm(2 * LMAX)];
  for (int ia = 0; ia < A.nprim; ia++)
    for (int jb = 0; jb < B.nprim; jb++) {
      const double a = prim[A.prim_off + ia], b = prim[B.prim_off + jb];
      const double ca = prim[nprimTot + A.prim_off + ia], cb = prim[nprimTot + B.prim_off + jb];
      const double p = a + b, K = ca * cb * exp(-a * b / p * AB2);
      double P[3];
      for (int x = 0; x < 3; x++) {
        P[x] = (a * A.O[x] + b * B.O[x]) / p;
        hermite_E_rt<double, LMAX>(la, lb, 0.5 / p, P[x] - A.O[x], P[x] - B.O[x], E[x]);
      }
      for (int c = 0; c < natom; c++) {
        const double Z = nuc[5 * c], zeta = nuc[5 * c + 4];
        const double X = P[0] - nuc[5 * c + 1], Y = P[1] - nuc[5 * c + 2],
                     W = P[2] - nuc[5 * c + 3];
        const double al = zeta > 0.0 ? p * zeta / (p + zeta) : p;
        const double f = zeta > 0.0 ? sqrt(zeta / (p + zeta)) : 1.0;
        boys_rt<double>(L, al * (X * X + Y * Y + W * W), F, boys);
        hermite_R_rt<double>(L, al, X, Y, W, F, R);
        const double pref = -Z * K * 2.0 * M_PI / p * f;
        for (int u = 0; u < na; u++) {
          const int ax = cart_lx(la, u), ay = cart_ly(la, u), az = cart_lz(la, u);
          for (int v = 0; v < nb; v++) {
            const int bx = cart_lx(lb, v), by = cart_ly(lb, v), bz = cart_lz(lb, v);
            const double* ex = E[0] + (ax * (lb + 1) + bx) * L1;
            const double* ey = E[1] + (ay * (lb + 1) + by) * L1;
            const double* ez = E[2] + (az * (lb + 1) + bz) * L1;
            double sum = 0.0;
            for (int t = 0; t <= ax + bx; t++)
              for (int w = 0; w <= ay + by; w++)
                for (int z = 0; z <= az + bz; z++) sum += ex[t] * ey[w] * ez[z] * R[hidx(t, w, z)];
            V[u][v] += pref * sum;
          }
        }
      }
    }
  const int ma = A.pure ? nsph(A.l) : ncart(A.l), mb = B.pure ? nsph(B.l) : ncart(B.l);
  for (int mu = 0; mu < ma; mu++)
    for (int nu = 0; nu < mb; nu++)
      Vmat[(size_t)(A.sph_off + mu) + (size_t)(B.sph_off + nu) * N] =
          sph_elem(A, B, sph, sphOff, V, mu, nu);
}

// Derivative nuclear-attraction matrices of the four-component core
// Hamiltonian, one thread per shell-pair block: with D_{mu nu} = <d_mu a| V
// |d_nu b> (electron-coordinate gradients; d_x x^i e = i x^{i-1} e -
// 2 a x^{i+1} e, so each D is a sum of plain nuclear-attraction integrals of
// l +- 1 on each side, from Hermite tables of (la + 1, lb + 1)),
// W0 = pV.p = sum_mu D_{mu mu} and W_k = (pV x p)_k = D_{ij} - D_{ji}
// ((i, j, k) cyclic); out: 4 consecutive N x N column-major matrices.
__global__ void nuclear_pvp_kernel(const ShellDev* __restrict__ sh,
                                   const double* __restrict__ prim,
                                   const double* __restrict__ sph, const int* __restrict__ sphOff,
                                   int nshell, int nprimTot, int N, int natom,
                                   const double* __restrict__ nuc, const double* __restrict__ boys,
                                   double* Wmat) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nshell * nshell) return;
  const int s1 = k % nshell, s2 = k / nshell;
  const ShellDev A = sh[s1], B = sh[s2];
  const int la = A.l, lb = B.l, La = la + 1, Lb = lb + 1, L = La + Lb, L1 = L + 1;
  const int na = ncart(la), nb = ncart(lb);
  constexpr int E1 = (LMAX + 2) * (LMAX + 2) * (2 * LMAX + 3);
  double W[4][ncart(LMAX)][ncart(LMAX)];
  for (int q = 0; q < 4; q++)
    for (int i = 0; i < na; i++)
      for (int j = 0; j < nb; j++) W[q][i][j] = 0.0;
  double AB2 = 0.0;
  for (int x = 0; x < 3; x++) AB2 += (A.O[x] - B.O[x]) * (A.O[x] - B.O[x]);
  double E[3][E1], F[2 * LMAX + 3], R[nherm(2 * LMAX + 2)];
  for (int ia = 0; ia < A.nprim; ia++)
    for (int jb = 0; jb < B.nprim; jb++) {
      const double a = prim[A.prim_off + ia], b = prim[B.prim_off + jb];
      const double ca = prim[nprimTot + A.prim_off + ia], cb = prim[nprimTot + B.prim_off + jb];
      const double p = a + b, K = ca * cb * exp(-a * b / p * AB2);
      double P[3];
      for (int x = 0; x < 3; x++) {
        P[x] = (a * A.O[x] + b * B.O[x]) / p;
        hermite_E_rt<double, LMAX + 1>(La, Lb, 0.5 / p, P[x] - A.O[x], P[x] - B.O[x], E[x]);
      }
      for (int c = 0; c < natom; c++) {
        const double Z = nuc[5 * c], zeta = nuc[5 * c + 4];
        const double X = P[0] - nuc[5 * c + 1], Y = P[1] - nuc[5 * c + 2],
                     Wz = P[2] - nuc[5 * c + 3];
        const double al = zeta > 0.0 ? p * zeta / (p + zeta) : p;
        const double f = zeta > 0.0 ? sqrt(zeta / (p + zeta)) : 1.0;
        boys_rt<double>(L, al * (X * X + Y * Y + Wz * Wz), F, boys);
        hermite_R_rt<double>(L, al, X, Y, Wz, F, R);
        const double pref = -Z * K * 2.0 * M_PI / p * f;
        // plain integral of Cartesian exponents (i0, i1, i2 | j0, j1, j2)
        auto vint = [&](int i0, int i1, int i2, int j0, int j1, int j2) {
          if (i0 < 0 || i1 < 0 || i2 < 0 || j0 < 0 || j1 < 0 || j2 < 0) return 0.0;
          const double* ex = E[0] + (i0 * (Lb + 1) + j0) * L1;
          const double* ey = E[1] + (i1 * (Lb + 1) + j1) * L1;
          const double* ez = E[2] + (i2 * (Lb + 1) + j2) * L1;
          double sum = 0.0;
          for (int t = 0; t <= i0 + j0; t++)
            for (int w = 0; w <= i1 + j1; w++)
              for (int z = 0; z <= i2 + j2; z++) sum += ex[t] * ey[w] * ez[z] * R[hidx(t, w, z)];
          return sum;
        };
        for (int u = 0; u < na; u++) {
          const int a0[3] = {cart_lx(la, u), cart_ly(la, u), cart_lz(la, u)};
          for (int v = 0; v < nb; v++) {
            const int b0[3] = {cart_lx(lb, v), cart_ly(lb, v), cart_lz(lb, v)};
            double D[3][3];
            for (int m = 0; m < 3; m++)
              for (int n = 0; n < 3; n++) {
                double d = 0.0;
                for (int sa = -1; sa <= 1; sa += 2)
                  for (int sb = -1; sb <= 1; sb += 2) {
                    const double fa = sa < 0 ? (double)a0[m] : -2.0 * a;
                    const double fb = sb < 0 ? (double)b0[n] : -2.0 * b;
                    if (fa == 0.0 || fb == 0.0) continue;
                    int ii[3] = {a0[0], a0[1], a0[2]}, jj[3] = {b0[0], b0[1], b0[2]};
                    ii[m] += sa;
                    jj[n] += sb;
                    d += fa * fb * vint(ii[0], ii[1], ii[2], jj[0], jj[1], jj[2]);
                  }
                D[m][n] = pref * d;
              }
            W[0][u][v] += D[0][0] + D[1][1] + D[2][2];
            W[1][u][v] += D[1][2] - D[2][1];
            W[2][u][v] += D[2][0] - D[0][2];
            W[3][u][v] += D[0][1] - D[1][0];
          }
        }
      }
    }
  const int ma = A.pure ? nsph(A.l) : ncart(A.l), mb = B.pure ? nsph(B.l) : ncart(B.l);
  const size_t NN = (size_t)N * N;
  for (int q = 0; q < 4; q++)
    for (int mu = 0; mu < ma; mu++)
      for (int nu = 0; nu < mb; nu++)
        Wmat[q * NN + (size_t)(A.sph_off + mu) + (size_t)(B.sph_off + nu) * N] =
            sph_elem(A, B, sph, sphOff, W[q], mu, nu);
}

__global__ void prim_pairs_kernel(const ShellDev* __restrict__ sh, const double* __restrict__ prim,
                                  int nprimTot, const PairDev* __restrict__ pairs, int npair,
                                  PrimPairDev* pp) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npair) return;
  const PairDev P = pairs[k];
  const ShellDev A = sh[P.shA], B = sh[P.shB];
  double AB2 = 0.0;
  for (int x = 0; x < 3; x++) AB2 += (A.O[x] - B.O[x]) * (A.O[x] - B.O[x]);
  int idx = P.pp_off;
  for (int ia = 0; ia < A.nprim; ia++)
    for (int jb = 0; jb < B.nprim; jb++, idx++) {
      double a = prim[A.prim_off + ia], b = prim[B.prim_off + jb];
      double ca = prim[nprimTot + A.prim_off + ia], cb = prim[nprimTot + B.prim_off + jb];
      PrimPairDev r;
      r.p = a + b;
      r.Kp = ca * cb * exp(-a * b / r.p * AB2) / r.p;
      for (int x = 0; x < 3; x++) {
        r.P[x] = (a * A.O[x] + b * B.O[x]) / r.p;
        r.PA[x] = r.P[x] - A.O[x];
        r.PB[x] = r.P[x] - B.O[x];
      }
      r.o2p = 0.5 / r.p;
      r.ia = ia;
      r.ib = jb;
      pp[idx] = r;
    }
}

// Sort key of a pair: class, then primitive-pair count (descending: pairs
// of one contraction length sit together, so a warp's lanes run primitive
// loops of one length), then Schwarz bound (descending).
__global__ void sort_keys_kernel(const PairDev* pairs, int n, unsigned long long* keys, int* vals) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  unsigned long long qb = (unsigned long long)__double_as_longlong(pairs[k].Q);  // Q >= 0
  const unsigned long long np = 255u - (unsigned)min(pairs[k].npp, 255);
  keys[k] = ((unsigned long long)pairs[k].cls << 56) | (np << 48) |
            ((~qb >> 16) & ((1ull << 48) - 1));
  vals[k] = k;
}

__global__ void gather_pairs_kernel(const PairDev* in, const int* idx, int n, PairDev* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) out[k] = in[idx[k]];
}

// Primitive pairs of pair i moved from src[i] to pairs[i].pp_off (the order
// of the sorted pair list); one thread per pair.
__global__ void reorder_pp_kernel(const PrimPairDev* __restrict__ in, const PairDev* pairs,
                                  const long long* __restrict__ src, int n,
                                  PrimPairDev* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const PairDev P = pairs[i];
  for (int k = 0; k < P.npp; k++) out[P.pp_off + k] = in[src[i] + k];
}

__global__ void fill_kernel(double* __restrict__ x, long long n, double v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    x[i] = v;
}

// FP32 copy of the primitive-pair records.
__global__ void pp32_kernel(const PrimPairDev* __restrict__ pp, long long n, PrimPair32* out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const PrimPairDev r = pp[i];
    PrimPair32 o;
    o.p = (float)r.p;
    o.Kp = (float)r.Kp;
    o.o2p = (float)r.o2p;
    for (int x = 0; x < 3; x++) {
      o.P[x] = (float)r.P[x];
      o.PA[x] = (float)r.PA[x];
      o.PB[x] = (float)r.PB[x];
    }
    out[i] = o;
  }
}

// Each pair's primitive pairs in descending order of their primitive
// Schwarz bound (insertion sort, one thread per pair), so that the class
// kernels' primitive loops can stop at the first pair below the screen.
__global__ void sort_pp_kernel(const PairDev* __restrict__ pairs, int n, PrimPairDev* pp,
                               double* ppQ) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const PairDev P = pairs[i];
  PrimPairDev* r = pp + P.pp_off;
  double* q = ppQ + P.pp_off;
  for (int k = 1; k < P.npp; k++) {
    const PrimPairDev rk = r[k];
    const double qk = q[k];
    int j = k - 1;
    while (j >= 0 && q[j] < qk) {
      r[j + 1] = r[j];
      q[j + 1] = q[j];
      j--;
    }
    r[j + 1] = rk;
    q[j + 1] = qk;
  }
}

// FP32 range data of each pair: log2 of 2 max p and of max |Kp| over its
// primitive pairs (fp32_range_ok).
__global__ void pair_range_kernel(const PrimPairDev* __restrict__ pp, const PairDev* pairs,
                                  int n, float2* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const PairDev P = pairs[i];
  double pm = 0.0, km = 0.0;
  for (int k = 0; k < P.npp; k++) {
    pm = fmax(pm, pp[P.pp_off + k].p);
    km = fmax(km, fabs(pp[P.pp_off + k].Kp));
  }
  out[i] = make_float2((float)log2(fmax(2.0 * pm, 1e-30)), (float)log2(fmax(km, 1e-60)));
}

// Tile-interleaved ket data: one block per ket tile (KETT_TILE consecutive
// pairs of a class starting at pair tileFirst[t], tileCnt[t] of them), lane
// l = thread; field f of primitive iq of lane l at
// out[tileOff[t] + (iq * KETT_NF + f) * KETT_TILE + l], zero past the pair's
// primitives, for iq below the tile's largest primitive count.
__global__ void ket_tiles_kernel(const PrimPairDev* __restrict__ pp,
                                 const double* __restrict__ ppQ, const PairDev* pairs,
                                 const int* __restrict__ tileFirst,
                                 const int* __restrict__ tileCnt,
                                 const long long* __restrict__ tileOff, double* out,
                                 float* out32) {
  const int t = blockIdx.x, l = threadIdx.x;
  const long long base = tileOff[t];
  const int mx = (int)((tileOff[t + 1] - base) / (KETT_NF * KETT_TILE));
  const bool have = l < tileCnt[t];
  int npp = 0, off = 0;
  if (have) {
    const PairDev P = pairs[tileFirst[t] + l];
    npp = P.npp;
    off = P.pp_off;
  }
  for (int iq = 0; iq < mx; iq++) {
    double f[KETT_NF];
    if (iq < npp) {
      const PrimPairDev r = pp[off + iq];
      f[0] = r.p; f[1] = r.Kp; f[2] = r.o2p;
      for (int x = 0; x < 3; x++) {
        f[3 + x] = r.P[x];
        f[6 + x] = r.PA[x];
        f[9 + x] = r.PB[x];
      }
      f[12] = ppQ[off + iq];
    } else {
      for (int k = 0; k < KETT_NF; k++) f[k] = 0.0;
    }
    for (int k = 0; k < KETT_NF; k++) {
      const long long o = base + ((long long)iq * KETT_NF + k) * KETT_TILE + l;
      out[o] = f[k];
      out32[o] = (float)f[k];
    }
  }
}

// ------------------------------------------------------------ build kernels
// Shell-block infinity norms (ShellBlockNorm, direct.hpp:73-90): one thread
// per (s1, s2) block, max over rows of the absolute row sums.
__global__ void block_norms_kernel(const double* __restrict__ X, int cplx, int N,
                                   const ShellDev* __restrict__ sh, int ns, double* out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns * ns) return;
  int s1 = k % ns, s2 = k / ns;
  const ShellDev A = sh[s1], B = sh[s2];
  int n1 = A.pure ? nsph(A.l) : ncart(A.l), n2 = B.pure ? nsph(B.l) : ncart(B.l);
  double mx = 0.0;
  for (int i = 0; i < n1; i++) {
    double r = 0.0;
    for (int j = 0; j < n2; j++) {
      size_t e = (size_t)(A.sph_off + i) + (size_t)(B.sph_off + j) * N;
      r += cplx ? hypot(X[2 * e], X[2 * e + 1]) : fabs(X[e]);
    }
    mx = fmax(mx, r);
  }
  out[k] = mx;
}

// symmetrise the norms of non-Hermitian matrices (direct.hpp:1533-1542)
__global__ void sym_norms_kernel(double* nm, int ns) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ns * ns) return;
  int a = k % ns, b = k / ns;
  if (a <= b) return;
  double m = fmax(nm[a + (size_t)b * ns], nm[b + (size_t)a * ns]);
  nm[a + (size_t)b * ns] = m;
  nm[b + (size_t)a * ns] = m;
}

__global__ void max_norms_kernel(const double* __restrict__ nm, int nMat, size_t ns2,
                                 double* out, unsigned long long* gmax) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  double m = 0.0;
  if (k < ns2) {
    for (int i = 0; i < nMat; i++) m = fmax(m, nm[i * ns2 + k]);
    out[k] = m;
  }
  // block max, then one atomic (non-negative doubles order as their bits)
  __shared__ double red[256];
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    atomicMax(gmax, (unsigned long long)__double_as_longlong(red[0]));
}

// transpose of the max-norm table and the norm of each pair's own block
__global__ void norms_aux_kernel(const double* __restrict__ nm, int ns,
                                 const PairDev* __restrict__ pairs, int npair, double* nmT,
                                 double* pn) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t ns2 = (size_t)ns * ns;
  if (k < ns2) {
    const int r = (int)(k % ns), c = (int)(k / ns);
    nmT[k] = nm[c + (size_t)r * ns];
  }
  if (k < (size_t)npair) {
    const PairDev P = pairs[k];
    pn[k] = nm[P.s1 + (size_t)P.s2 * ns];
  }
}

// Xc = T X T^T per matrix (T: block-diagonal Cartesian -> AO transform).
__global__ void to_cart_kernel(const double* __restrict__ X, int cplx, int N, int nc,
                               const ShellDev* __restrict__ sh, const int* __restrict__ c2s,
                               const double* __restrict__ sph, const int* __restrict__ sphOff,
                               double* Xc) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= (size_t)nc * nc) return;
  int ci = (int)(k % nc), cj = (int)(k / nc);
  const ShellDev A = sh[c2s[ci]], B = sh[c2s[cj]];
  int a = ci - A.cart_off, b = cj - B.cart_off;
  int na = A.pure ? nsph(A.l) : ncart(A.l), nb = B.pure ? nsph(B.l) : ncart(B.l);
  const double* TA = sph + sphOff[A.l];
  const double* TB = sph + sphOff[B.l];
  double re = 0.0, im = 0.0;
  for (int mu = 0; mu < na; mu++) {
    double ta = A.pure ? TA[a * nsph(A.l) + mu] : (a == mu);
    if (ta == 0.0) continue;
    for (int nu = 0; nu < nb; nu++) {
      double tb = B.pure ? TB[b * nsph(B.l) + nu] : (b == nu);
      if (tb == 0.0) continue;
      size_t e = (size_t)(A.sph_off + mu) + (size_t)(B.sph_off + nu) * N;
      if (cplx) {
        re += ta * tb * X[2 * e];
        im += ta * tb * X[2 * e + 1];
      } else {
        re += ta * tb * X[e];
      }
    }
  }
  if (cplx) {
    Xc[2 * k] = re;
    Xc[2 * k + 1] = im;
  } else {
    Xc[k] = re;
  }
}

// AX += 1/2 (B + B^H) (Hermitian) or AX += 1/2 B, B = T^T Ac T
// (direct.hpp:2036-2066).
__global__ void from_cart_kernel(const double* __restrict__ Ac, int cplx, int her, int N, int nc,
                                 const ShellDev* __restrict__ sh, const int* __restrict__ ao2s,
                                 const double* __restrict__ sph, const int* __restrict__ sphOff,
                                 double* AX) {
  size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= (size_t)N * N) return;
  int i = (int)(k % N), j = (int)(k / N);
  auto bval = [&](int r, int c, double& bre, double& bim) {
    const ShellDev A = sh[ao2s[r]], B = sh[ao2s[c]];
    int mu = r - A.sph_off, nu = c - B.sph_off;
    int na = ncart(A.l), nb = ncart(B.l);
    const double* TA = sph + sphOff[A.l];
    const double* TB = sph + sphOff[B.l];
    bre = 0.0;
    bim = 0.0;
    for (int a = 0; a < na; a++) {
      double ta = A.pure ? TA[a * nsph(A.l) + mu] : (a == mu);
      if (ta == 0.0) continue;
      for (int b = 0; b < nb; b++) {
        double tb = B.pure ? TB[b * nsph(B.l) + nu] : (b == nu);
        if (tb == 0.0) continue;
        size_t e = (size_t)(A.cart_off + a) + (size_t)(B.cart_off + b) * nc;
        if (cplx) {
          bre += ta * tb * Ac[2 * e];
          bim += ta * tb * Ac[2 * e + 1];
        } else {
          bre += ta * tb * Ac[e];
        }
      }
    }
  };
  double r1, i1;
  bval(i, j, r1, i1);
  double outr, outi;
  if (her == 2) {  // real antisymmetric density: exchange stored transposed
    double r2, i2;
    bval(j, i, r2, i2);
    outr = 0.5 * (r2 - r1);
    outi = 0.0;
  } else if (her) {
    double r2, i2;
    bval(j, i, r2, i2);
    outr = 0.5 * (r1 + r2);
    outi = 0.5 * (i1 - i2);
  } else {
    outr = 0.5 * r1;
    outi = 0.5 * i1;
  }
  if (cplx) {
    AX[2 * k] += outr;
    AX[2 * k + 1] += outi;
  } else {
    AX[k] += outr;
  }
}

unsigned grid1(size_t n, int b) { return (unsigned)((n + b - 1) / b); }

// Real and imaginary parts of an interleaved complex matrix (n entries).
__global__ void to_float_kernel(const double* __restrict__ x, size_t n, float* y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

__global__ void split_complex_kernel(const double* __restrict__ Xc, size_t n, double* re,
                                     double* im) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  re[k] = Xc[2 * k];
  if (im) im[k] = Xc[2 * k + 1];
}

// AXc += re + i im (interleaved complex; im may be null).
__global__ void add_complex_kernel(double* AXc, size_t n, const double* __restrict__ re,
                                   const double* __restrict__ im) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n) return;
  AXc[2 * k] += re[k];
  if (im) AXc[2 * k + 1] += im[k];
}

// X <- (X + X^T) / 2 in place (n x n, column-major); each unordered pair
// (i < j) belongs to one thread.
__global__ void symmetrize_kernel(double* X, int n) {
  const size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= (size_t)n * n) return;
  const int i = (int)(k % n), j = (int)(k / n);
  if (i >= j) return;
  double* a = X + i + (size_t)j * n;
  double* b = X + j + (size_t)i * n;
  const double v = 0.5 * (*a + *b);
  *a = v;
  *b = v;
}

// Basis-owned device memory is stream-ordered on the basis' stream
// (cudaMallocAsync / cudaFreeAsync): creating, growing or destroying one
// basis never waits for the work of other bases (no device-wide sync).  The
// stream is synchronised before a new buffer is used from another stream.
cqf_status ensure_ws(cqf_basis* B, size_t bytes) {
  if (bytes <= B->ws_bytes) return CQF_OK;
  if (B->d_ws) CQF_CUDA(cudaFreeAsync(B->d_ws, B->stream));
  B->d_ws = nullptr;
  B->ws_bytes = 0;
  CQF_CUDA(cudaMallocAsync(&B->d_ws, bytes, B->stream));
  CQF_CUDA(cudaStreamSynchronize(B->stream));
  B->ws_bytes = bytes;
  return CQF_OK;
}

void aux_release(int device, cudaStream_t s);

void free_basis(cqf_basis* B) {
  if (!B) return;
  cudaSetDevice(B->device);
  if (B->stream) {
    cudaStream_t st = B->stream;
    for (void* p : {(void*)B->d_shells, (void*)B->d_prim, (void*)B->d_pairs, (void*)B->d_pp,
                    (void*)B->d_ppQ, (void*)B->d_qWin, (void*)B->d_pp32, (void*)B->d_ketT32,
                    (void*)B->d_ketT, (void*)B->d_tileOff, (void*)B->d_pairRange,
                    (void*)B->d_schwarz,
                    (void*)B->d_sph, (void*)B->d_sphOff, (void*)B->d_ao2shell,
                    (void*)B->d_cart2shell, (void*)B->d_ws, (void*)B->d_counters,
                    (void*)B->d_flags, (void*)B->d_qLL, (void*)B->d_qSS, (void*)B->d_qG, (void*)B->d_qB,
                    (void*)B->d_relws})
      if (p) cudaFreeAsync(p, st);
    cudaStreamSynchronize(st);
  }
  if (B->ev0) cudaEventDestroy(B->ev0);
  if (B->ev1) cudaEventDestroy(B->ev1);
  if (B->evFork) cudaEventDestroy(B->evFork);
  for (cudaEvent_t e : B->evStage)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t e : B->tune_ev)
    if (e) cudaEventDestroy(e);
  for (int i = 0; i < NAUX; i++) {
    if (B->evJoin[i]) cudaEventDestroy(B->evJoin[i]);
    aux_release(B->device, B->aux[i]);
  }
  if (B->stream) cudaStreamDestroy(B->stream);
  delete B;
}

template <typename T>
cqf_status upload(T** dst, const std::vector<T>& src, cudaStream_t st) {
  CQF_CUDA(cudaMallocAsync((void**)dst, std::max<size_t>(1, src.size()) * sizeof(T), st));
  // pageable source: the copy is staged before the call returns
  if (!src.empty())
    CQF_CUDA(cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice,
                             st));
  return CQF_OK;
}

// Auxiliary streams of the class-quartet launches: a per-device free list.
// A basis takes NAUX streams when it is created and gives them back when it
// is destroyed, so no two live bases share one (a stream being captured into
// a graph for one basis is never used by another) and a server that creates
// and destroys a basis per request reuses streams instead of creating them
// (stream creation showed in the set-up latency).  Streams are kept until
// the process exits.
struct AuxPool {
  std::mutex mu;
  std::vector<std::vector<cudaStream_t>> free;
};
AuxPool& aux_pool() {
  static AuxPool p;
  return p;
}

cqf_status aux_stream(int device, cudaStream_t* out) {
  AuxPool& P = aux_pool();
  {
    std::lock_guard<std::mutex> lk(P.mu);
    if ((int)P.free.size() <= device) P.free.resize(device + 1);
    if (!P.free[device].empty()) {
      *out = P.free[device].back();
      P.free[device].pop_back();
      return CQF_OK;
    }
  }
  CQF_CUDA(cudaStreamCreateWithFlags(out, cudaStreamNonBlocking));
  return CQF_OK;
}

void aux_release(int device, cudaStream_t s) {
  if (!s) return;
  AuxPool& P = aux_pool();
  std::lock_guard<std::mutex> lk(P.mu);
  if ((int)P.free.size() <= device) P.free.resize(device + 1);
  P.free[device].push_back(s);
}

// Boys tables: computed once per process, one device copy per device (held
// until exit, shared by every basis on the device).
cqf_status boys_tables(int device, cudaStream_t st, double** d64, float** d32) {
  static std::mutex mu;
  static std::vector<double> h64;
  static std::vector<float> h32;
  static std::vector<double*> dev64;
  static std::vector<float*> dev32;
  std::lock_guard<std::mutex> lk(mu);
  if (h64.empty()) make_boys_table(h64, h32);
  if ((int)dev64.size() <= device) {
    dev64.resize(device + 1, nullptr);
    dev32.resize(device + 1, nullptr);
  }
  if (!dev64[device]) {
    // the basis and workspace buffers are stream-ordered allocations from
    // the device's default pool; with its default release threshold (0) every
    // stream synchronisation hands the freed memory back to the driver, and
    // concurrent set-ups (a server) then serialise on re-mapping it.  Keep
    // freed memory in the pool for reuse (a process-local setting of this
    // process's pool, gone at exit).
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      unsigned long long keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    double* p64 = nullptr;
    float* p32 = nullptr;
    CQF_CUDA(cudaMalloc(&p64, h64.size() * sizeof(double)));
    CQF_CUDA(cudaMalloc(&p32, h32.size() * sizeof(float)));
    CQF_CUDA(cudaMemcpyAsync(p64, h64.data(), h64.size() * sizeof(double),
                             cudaMemcpyHostToDevice, st));
    CQF_CUDA(cudaMemcpyAsync(p32, h32.data(), h32.size() * sizeof(float), cudaMemcpyHostToDevice,
                             st));
    CQF_CUDA(cudaStreamSynchronize(st));
    dev64[device] = p64;
    dev32[device] = p32;
  }
  *d64 = dev64[device];
  *d32 = dev32[device];
  return CQF_OK;
}

cqf_status basis_create(const cqf_shell* shells, int nshell, double thresh, int device,
                        cqf_basis* B) {
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return fail(CQF_ENODEV, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(CQF_EINVAL, "bad device ordinal");
  B->device = device;
  for (int i = 0; i < NCLS; i++)
    for (int j = 0; j < NCLS; j++) B->blocks_per_sm[i][j] = 8;
  CQF_CUDA(cudaSetDevice(device));
  noalloc_prepare(device);
  CQF_CUDA(cudaDeviceGetAttribute(&B->nsm, cudaDevAttrMultiProcessorCount, device));
  CQF_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
  CQF_CUDA(cudaEventCreate(&B->ev0));
  CQF_CUDA(cudaEventCreate(&B->ev1));
  CQF_CUDA(cudaEventCreateWithFlags(&B->evFork, cudaEventDisableTiming));
  for (cudaEvent_t& e : B->evStage) CQF_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (int i = 0; i < NAUX; i++) {
    CQF_TRY(aux_stream(device, &B->aux[i]));
    CQF_CUDA(cudaEventCreateWithFlags(&B->evJoin[i], cudaEventDisableTiming));
  }
  B->thresh = thresh;
  B->nshell = nshell;

  // shells, primitive data
  std::vector<double> alpha, coef;
  int sphOff = 0, cartOff = 0;
  for (int s = 0; s < nshell; s++) {
    const cqf_shell& c = shells[s];
    if (c.l < 0 || c.l > LMAX) return fail(CQF_EINVAL, "shell angular momentum above LMAX");
    if (c.nprim <= 0 || !c.alpha || !c.coeff) return fail(CQF_EINVAL, "empty shell");
    ShellDev d{};
    d.l = c.l;
    d.pure = c.pure ? 1 : 0;
    d.nprim = c.nprim;
    d.prim_off = (int)alpha.size();
    d.cart_off = cartOff;
    d.sph_off = sphOff;
    for (int x = 0; x < 3; x++) d.O[x] = c.origin[x];
    for (int i = 0; i < c.nprim; i++) {
      alpha.push_back(c.alpha[i]);
      coef.push_back(c.coeff[i]);
    }
    sphOff += d.pure ? nsph(d.l) : ncart(d.l);
    cartOff += ncart(d.l);
    B->maxL = std::max(B->maxL, d.l);
    B->maxPrim = std::max(B->maxPrim, d.nprim);
    B->h_shells.push_back(d);
  }
  B->nbasis = sphOff;
  B->ncart = cartOff;
  const int nprimTot = (int)alpha.size();
  std::vector<double> prim(alpha);
  prim.insert(prim.end(), coef.begin(), coef.end());
  CQF_TRY(upload(&B->d_shells, B->h_shells, B->stream));
  CQF_TRY(upload(&B->d_prim, prim, B->stream));

  std::vector<int> ao2s, c2s;
  for (int s = 0; s < nshell; s++) {
    const ShellDev& d = B->h_shells[s];
    for (int i = 0; i < (d.pure ? nsph(d.l) : ncart(d.l)); i++) ao2s.push_back(s);
    for (int i = 0; i < ncart(d.l); i++) c2s.push_back(s);
  }
  CQF_TRY(upload(&B->d_ao2shell, ao2s, B->stream));
  CQF_TRY(upload(&B->d_cart2shell, c2s, B->stream));

  std::vector<double> sph;
  std::vector<int> sphO;
  for (int l = 0; l <= LMAX; l++) {
    sphO.push_back((int)sph.size());
    auto T = solid_harmonics(l);
    sph.insert(sph.end(), T.begin(), T.end());
  }
  CQF_TRY(upload(&B->d_sph, sph, B->stream));
  CQF_TRY(upload(&B->d_sphOff, sphO, B->stream));

  CQF_TRY(boys_tables(device, B->stream, &B->d_boys64, &B->d_boys32));

  // significant pairs on the device
  long long nlt = (long long)nshell * (nshell + 1) / 2;
  unsigned char* d_flags8 = nullptr;
  CQF_CUDA(cudaMallocAsync(&d_flags8, std::max<long long>(1, nlt), B->stream));
  sig_pairs_kernel<<<grid1(nlt, 128), 128, 0, B->stream>>>(B->d_shells, B->d_prim, B->d_sph,
                                                           B->d_sphOff, nshell, nprimTot, d_flags8);
  std::vector<unsigned char> f8(nlt);
  CQF_CUDA(cudaMemcpyAsync(f8.data(), d_flags8, nlt, cudaMemcpyDeviceToHost, B->stream));
  CQF_CUDA(cudaStreamSynchronize(B->stream));
  cudaFreeAsync(d_flags8, B->stream);

  // pair list in the reference loop order, then grouped by class (stable)
  std::vector<PairDev> lexPairs;
  for (int s1 = 0, k = 0; s1 < nshell; s1++)
    for (int s2 = 0; s2 <= s1; s2++, k++) {
      if (!f8[k]) continue;
      PairDev p{};
      p.s1 = s1;
      p.s2 = s2;
      const ShellDev &A = B->h_shells[s1], &Bs = B->h_shells[s2];
      if (A.l >= Bs.l) { p.shA = s1; p.shB = s2; }
      else { p.shA = s2; p.shB = s1; }
      p.cA = B->h_shells[p.shA].cart_off;
      p.cB = B->h_shells[p.shB].cart_off;
      p.lex = (int)lexPairs.size();
      p.cls = class_id(B->h_shells[p.shA].l, B->h_shells[p.shB].l);
      p.npp = B->h_shells[p.shA].nprim * B->h_shells[p.shB].nprim;
      lexPairs.push_back(p);
    }
  std::vector<PairDev> pairs;
  for (int c = 0; c < NCLS; c++) {
    B->cls_beg[c] = (int)pairs.size();
    for (auto& p : lexPairs)
      if (p.cls == c) pairs.push_back(p);
    B->cls_cnt[c] = (int)pairs.size() - B->cls_beg[c];
  }
  long long ppoff = 0;
  for (auto& p : pairs) {
    p.pp_off = (int)ppoff;
    ppoff += p.npp;
  }
  B->npair = (int)pairs.size();
  B->nprimpair = ppoff;
  PairDev* d_tmp = nullptr;
  CQF_TRY(upload(&d_tmp, pairs, B->stream));
  CQF_CUDA(cudaMallocAsync(&B->d_pp, std::max<long long>(1, ppoff) * sizeof(PrimPairDev), B->stream));
  prim_pairs_kernel<<<grid1(B->npair, 128), 128, 0, B->stream>>>(B->d_shells, B->d_prim, nprimTot,
                                                                 d_tmp, B->npair, B->d_pp);
  CQF_CUDA(cudaMallocAsync(&B->d_schwarz, (size_t)nshell * nshell * sizeof(double), B->stream));
  CQF_CUDA(cudaMemsetAsync(B->d_schwarz, 0, (size_t)nshell * nshell * sizeof(double), B->stream));
  double* d_diag = nullptr;
  CQF_CUDA(cudaMallocAsync(&d_diag, std::max(1, B->npair) * 36 * sizeof(double), B->stream));
  for (int c = 0; c < NCLS; c++) {
    if (B->cls_cnt[c] <= 0) continue;
    int la, lb;
    class_ls(c, la, lb);
    if (!launch_schwarz_fast(la, lb, d_tmp, B->d_pp, B->d_boys64, B->d_sph, B->d_sphOff,
                             B->d_shells, B->cls_beg[c], B->cls_cnt[c], nshell, B->d_schwarz,
                             d_tmp, d_diag + (size_t)B->cls_beg[c] * 36, B->stream))
      schwarz_kernel<<<grid1(B->cls_cnt[c], 64), 64, 0, B->stream>>>(
          d_tmp, B->d_pp, B->d_boys64, B->d_sph, B->d_sphOff, B->d_shells, B->cls_beg[c],
          B->cls_cnt[c], nshell, B->d_schwarz, d_tmp);
  }
  CQF_CUDA(cudaGetLastError());

  // sort each class by Schwarz bound, descending (stable: ties stay in
  // reference loop order)
  unsigned long long *kin = nullptr, *kout = nullptr;
  int *vin = nullptr, *vout = nullptr;
  int n = std::max(1, B->npair);
  CQF_CUDA(cudaMallocAsync(&kin, n * sizeof(unsigned long long), B->stream));
  CQF_CUDA(cudaMallocAsync(&kout, n * sizeof(unsigned long long), B->stream));
  CQF_CUDA(cudaMallocAsync(&vin, n * sizeof(int), B->stream));
  CQF_CUDA(cudaMallocAsync(&vout, n * sizeof(int), B->stream));
  sort_keys_kernel<<<grid1(B->npair, 128), 128, 0, B->stream>>>(d_tmp, B->npair, kin, vin);
  size_t tmpBytes = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, tmpBytes, kin, kout, vin, vout, B->npair, 0, 64,
                                  B->stream);
  void* d_cub = nullptr;
  CQF_CUDA(cudaMallocAsync(&d_cub, std::max<size_t>(1, tmpBytes), B->stream));
  CQF_CUDA(cub::DeviceRadixSort::SortPairs(d_cub, tmpBytes, kin, kout, vin, vout, B->npair, 0,
                                           64, B->stream));
  CQF_CUDA(cudaMallocAsync(&B->d_pairs, n * sizeof(PairDev), B->stream));
  gather_pairs_kernel<<<grid1(B->npair, 128), 128, 0, B->stream>>>(d_tmp, vout, B->npair,
                                                                   B->d_pairs);
  CQF_CUDA(cudaGetLastError());
  B->h_pairs.resize(B->npair);
  CQF_CUDA(cudaMemcpyAsync(B->h_pairs.data(), B->d_pairs, B->npair * sizeof(PairDev),
                           cudaMemcpyDeviceToHost, B->stream));
  CQF_CUDA(cudaStreamSynchronize(B->stream));
  {
    // largest Schwarz bound over each window of WTILE pairs starting at a
    // pair, inside its class: the tile-level screens' bound (pairs are not
    // in Schwarz order across contraction lengths)
    std::vector<double> qw(std::max(1, B->npair));
    for (int i = B->npair - 1; i >= 0; i--) {
      double m = B->h_pairs[i].Q;
      for (int j = i + 1; j < std::min(B->npair, i + WTILE); j++)
        if (B->h_pairs[j].cls == B->h_pairs[i].cls) m = std::max(m, B->h_pairs[j].Q);
      qw[i] = m;
    }
    CQF_TRY(upload(&B->d_qWin, qw, B->stream));
  }
  // primitive pairs in the same order as the sorted pairs: the primitives of
  // consecutive kets of a tile are one contiguous run (moved on the device;
  // only the per-pair offsets cross to the host and back)
  {
    std::vector<long long> src(std::max(1, B->npair));
    long long off2 = 0;
    for (int i = 0; i < B->npair; i++) {
      src[i] = B->h_pairs[i].pp_off;
      B->h_pairs[i].pp_off = (int)off2;
      off2 += B->h_pairs[i].npp;
    }
    CQF_CUDA(cudaMemcpyAsync(B->d_pairs, B->h_pairs.data(), B->npair * sizeof(PairDev),
                             cudaMemcpyHostToDevice, B->stream));
    long long* d_src = nullptr;
    CQF_TRY(upload(&d_src, src, B->stream));
    PrimPairDev* d_pp2 = nullptr;
    CQF_CUDA(cudaMallocAsync(&d_pp2, std::max<long long>(1, ppoff) * sizeof(PrimPairDev),
                             B->stream));
    reorder_pp_kernel<<<grid1(B->npair, 128), 128, 0, B->stream>>>(B->d_pp, B->d_pairs, d_src,
                                                                   B->npair, d_pp2);
    cudaFreeAsync(B->d_pp, B->stream);
    cudaFreeAsync(d_src, B->stream);
    B->d_pp = d_pp2;
    // primitive Schwarz bounds (the generated classes; others keep an
    // unscreened bound), then each pair's primitive pairs sorted by them
    CQF_CUDA(cudaMallocAsync(&B->d_ppQ, std::max<long long>(1, ppoff) * sizeof(double),
                             B->stream));
    fill_kernel<<<(unsigned)std::min<long long>(grid1(std::max<long long>(1, ppoff), 256), 4096),
                  256, 0, B->stream>>>(B->d_ppQ, std::max<long long>(1, ppoff), 1e300);
    for (int c = 0; c < NCLS; c++) {
      int la, lb;
      class_ls(c, la, lb);
      if (la <= 2)
        launch_prim_schwarz(la, lb, B->d_pairs, B->d_pp, B->d_boys64, B->cls_beg[c],
                            B->cls_cnt[c], B->d_ppQ, B->stream);
    }
    sort_pp_kernel<<<grid1(B->npair, 128), 128, 0, B->stream>>>(B->d_pairs, B->npair, B->d_pp,
                                                                B->d_ppQ);
    CQF_CUDA(cudaMallocAsync(&B->d_pp32, std::max<long long>(1, ppoff) * sizeof(PrimPair32),
                             B->stream));
    pp32_kernel<<<(unsigned)std::min<long long>(grid1(std::max<long long>(1, ppoff), 256), 4096),
                  256, 0, B->stream>>>(B->d_pp, ppoff, B->d_pp32);
    CQF_CUDA(cudaGetLastError());
    // the same data tile-interleaved for the class kernels' kets: per ket
    // tile (KETT_TILE consecutive pairs of a class), field-major runs of
    // KETT_TILE values for each primitive (zero past a pair's npp)
    std::vector<long long> toff;
    std::vector<int> tfirst, tcnt;
    long long ktn = 0;
    for (int c = 0; c < NCLS; c++) {
      B->cls_tile_beg[c] = (int)toff.size();
      const int cnt = B->cls_cnt[c];
      for (int t0 = 0; t0 < cnt; t0 += KETT_TILE) {
        int mx = 0;
        const int n = std::min(KETT_TILE, cnt - t0);
        for (int l = 0; l < n; l++) mx = std::max(mx, B->h_pairs[B->cls_beg[c] + t0 + l].npp);
        toff.push_back(ktn);
        tfirst.push_back(B->cls_beg[c] + t0);
        tcnt.push_back(n);
        ktn += (long long)mx * KETT_NF * KETT_TILE;
      }
    }
    const int ntile = (int)toff.size();
    toff.push_back(ktn);
    CQF_CUDA(cudaMallocAsync(&B->d_ketT, (size_t)(ktn + 1) * sizeof(double), B->stream));
    CQF_CUDA(cudaMemsetAsync(B->d_ketT + ktn, 0, sizeof(double), B->stream));
    CQF_CUDA(cudaMallocAsync(&B->d_ketT32, (size_t)(ktn + 1) * sizeof(float), B->stream));
    CQF_CUDA(cudaMemsetAsync(B->d_ketT32 + ktn, 0, sizeof(float), B->stream));
    CQF_TRY(upload(&B->d_tileOff, toff, B->stream));
    if (ntile > 0) {
      int *d_tf = nullptr, *d_tc = nullptr;
      CQF_TRY(upload(&d_tf, tfirst, B->stream));
      CQF_TRY(upload(&d_tc, tcnt, B->stream));
      ket_tiles_kernel<<<ntile, KETT_TILE, 0, B->stream>>>(B->d_pp, B->d_ppQ, B->d_pairs, d_tf,
                                                           d_tc, B->d_tileOff, B->d_ketT,
                                                           B->d_ketT32);
      cudaFreeAsync(d_tf, B->stream);
      cudaFreeAsync(d_tc, B->stream);
    }
    CQF_CUDA(cudaMallocAsync(&B->d_pairRange, std::max(1, B->npair) * sizeof(float2),
                             B->stream));
    pair_range_kernel<<<grid1(B->npair, 128), 128, 0, B->stream>>>(B->d_pp, B->d_pairs,
                                                                   B->npair, B->d_pairRange);
    CQF_CUDA(cudaGetLastError());
  }
  B->h_schwarz.resize((size_t)nshell * nshell);
  CQF_CUDA(cudaMemcpyAsync(B->h_schwarz.data(), B->d_schwarz,
                           (size_t)nshell * nshell * sizeof(double), cudaMemcpyDeviceToHost,
                           B->stream));
  CQF_CUDA(cudaStreamSynchronize(B->stream));
  cudaFreeAsync(kin, B->stream);
  cudaFreeAsync(kout, B->stream);
  cudaFreeAsync(vin, B->stream);
  cudaFreeAsync(vout, B->stream);
  cudaFreeAsync(d_cub, B->stream);
  cudaFreeAsync(d_tmp, B->stream);
  cudaFreeAsync(d_diag, B->stream);
  CQF_CUDA(cudaMallocAsync(&B->d_counters, 8 * sizeof(unsigned long long), B->stream));
  CQF_CUDA(cudaMallocAsync(&B->d_flags, MAXMAT * sizeof(int), B->stream));
  B->h_flags.assign(MAXMAT, 0);
  CQF_CUDA(cudaStreamSynchronize(B->stream));
  return CQF_OK;
}

}  // namespace

extern "C" {

void cqf_opts_default(cqf_opts* o) {
  if (!o) return;
  o->is_complex = 0;
  o->screen = 1;
  o->device_pointers = 0;
  o->precision = CQF_FP64;
  o->fp32_cutoff = 0.0;
  o->stream = nullptr;
  o->shard_index = 0;
  o->shard_count = 1;
}

const char* cqf_last_error(void) { return g_err.c_str(); }

cqf_status cqf_basis_create(const cqf_shell* shells, int nshell, double thresh_schwarz,
                            int device, cqf_basis** out) {
  g_err.clear();
  if (!out || !shells || nshell <= 0) return fail(CQF_EINVAL, "cqf_basis_create: bad argument");
  *out = nullptr;
  auto* B = new cqf_basis();
  cqf_status s = basis_create(shells, nshell, thresh_schwarz, device, B);
  if (s != CQF_OK) {
    std::string keep = g_err;
    free_basis(B);
    g_err = keep;
    return s;
  }
  *out = B;
  return CQF_OK;
}

cqf_status cqf_basis_destroy(cqf_basis* basis) {
  free_basis(basis);
  return CQF_OK;
}

cqf_status cqf_basis_info(const cqf_basis* B, int* nbasis, int* nshell, int* npair) {
  if (!B) return fail(CQF_EINVAL, "null basis");
  if (nbasis) *nbasis = B->nbasis;
  if (nshell) *nshell = B->nshell;
  if (npair) *npair = B->npair;
  return CQF_OK;
}

cqf_status cqf_basis_schwarz(const cqf_basis* B, double* Q) {
  if (!B || !Q) return fail(CQF_EINVAL, "null argument");
  std::copy(B->h_schwarz.begin(), B->h_schwarz.end(), Q);
  return CQF_OK;
}

cqf_status cqf_basis_one_electron(cqf_basis* B, double* S, double* T) {
  g_err.clear();
  if (!B || !S || !T) return fail(CQF_EINVAL, "null argument");
  std::lock_guard<std::mutex> lk(B->mu);
  CQF_CUDA(cudaSetDevice(B->device));
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  CQF_TRY(ensure_ws(B, 2 * NN * sizeof(double)));
  double* d = static_cast<double*>(B->d_ws);
  int nprimTot = 0;
  for (auto& sh : B->h_shells) nprimTot += sh.nprim;
  one_electron_kernel<<<grid1((size_t)B->nshell * B->nshell, 64), 64, 0, B->stream>>>(
      B->d_shells, B->d_prim, B->d_sph, B->d_sphOff, B->nshell, nprimTot, B->nbasis, d, d + NN);
  CQF_CUDA(cudaGetLastError());
  CQF_CUDA(cudaMemcpyAsync(S, d, NN * sizeof(double), cudaMemcpyDeviceToHost, B->stream));
  CQF_CUDA(cudaMemcpyAsync(T, d + NN, NN * sizeof(double), cudaMemcpyDeviceToHost, B->stream));
  CQF_CUDA(cudaStreamSynchronize(B->stream));
  return CQF_OK;
}

cqf_status cqf_basis_nuclear(cqf_basis* B, int natom, const double* nuclei, double* V) {
  g_err.clear();
  if (!B || !V || natom < 0 || (natom > 0 && !nuclei))
    return fail(CQF_EINVAL, "cqf_basis_nuclear: bad argument");
  std::lock_guard<std::mutex> lk(B->mu);
  CQF_CUDA(cudaSetDevice(B->device));
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  CQF_TRY(ensure_ws(B, (NN + 5 * (size_t)std::max(1, natom)) * sizeof(double)));
  double* d = static_cast<double*>(B->d_ws);
  double* dn = d + NN;
  if (natom > 0)
    CQF_CUDA(cudaMemcpyAsync(dn, nuclei, 5 * (size_t)natom * sizeof(double),
                             cudaMemcpyHostToDevice, B->stream));
  int nprimTot = 0;
  for (auto& sh : B->h_shells) nprimTot += sh.nprim;
  nuclear_kernel<<<grid1((size_t)B->nshell * B->nshell, 64), 64, 0, B->stream>>>(
      B->d_shells, B->d_prim, B->d_sph, B->d_sphOff, B->nshell, nprimTot, B->nbasis, natom, dn,
      B->d_boys64, d);
  CQF_CUDA(cudaGetLastError());
  CQF_CUDA(cudaMemcpyAsync(V, d, NN * sizeof(double), cudaMemcpyDeviceToHost, B->stream));
  CQF_CUDA(cudaStreamSynchronize(B->stream));
  return CQF_OK;
}

cqf_status cqf_basis_nuclear_pvp(cqf_basis* B, int natom, const double* nuclei, double* W) {
  g_err.clear();
  if (!B || !W || natom < 0 || (natom > 0 && !nuclei))
    return fail(CQF_EINVAL, "cqf_basis_nuclear_pvp: bad argument");
  std::lock_guard<std::mutex> lk(B->mu);
  CQF_CUDA(cudaSetDevice(B->device));
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  CQF_TRY(ensure_ws(B, (4 * NN + 5 * (size_t)std::max(1, natom)) * sizeof(double)));
  double* d = static_cast<double*>(B->d_ws);
  double* dn = d + 4 * NN;
  if (natom > 0)
    CQF_CUDA(cudaMemcpyAsync(dn, nuclei, 5 * (size_t)natom * sizeof(double),
                             cudaMemcpyHostToDevice, B->stream));
  int nprimTot = 0;
  for (auto& sh : B->h_shells) nprimTot += sh.nprim;
  nuclear_pvp_kernel<<<grid1((size_t)B->nshell * B->nshell, 64), 64, 0, B->stream>>>(
      B->d_shells, B->d_prim, B->d_sph, B->d_sphOff, B->nshell, nprimTot, B->nbasis, natom, dn,
      B->d_boys64, d);
  CQF_CUDA(cudaGetLastError());
  CQF_CUDA(cudaMemcpyAsync(W, d, 4 * NN * sizeof(double), cudaMemcpyDeviceToHost, B->stream));
  CQF_CUDA(cudaStreamSynchronize(B->stream));
  return CQF_OK;
}

cqf_status cqf_four_comp_core_hamiltonian(cqf_basis* B, int natom, const double* nuclei,
                                          void* const* H) {
  if (!B || !H) return fail(CQF_EINVAL, "cqf_four_comp_core_hamiltonian: null argument");
  for (int c = 0; c < 4; c++)
    if (!H[c]) return fail(CQF_EINVAL, "cqf_four_comp_core_hamiltonian: null component");
  const int N = B->nbasis;
  const size_t NN = (size_t)N * N;
  std::vector<double> S(NN), T(NN), V(NN), W(4 * NN);
  CQF_TRY(cqf_basis_one_electron(B, S.data(), T.data()));
  CQF_TRY(cqf_basis_nuclear(B, natom, nuclei, V.data()));
  CQF_TRY(cqf_basis_nuclear_pvp(B, natom, nuclei, W.data()));
  const double C2 = 1.0 / (4.0 * SPEED_OF_LIGHT * SPEED_OF_LIGHT);
  const size_t M = 2 * (size_t)N;  // 4C dimension
  for (int c = 0; c < 4; c++) std::fill_n(static_cast<double*>(H[c]), 2 * M * M, 0.0);
  // element (r, col) of component c: interleaved complex, column-major
  auto at = [&](int c, size_t r, size_t col) { return static_cast<double*>(H[c]) + 2 * (r + col * M); };
  for (int j = 0; j < N; j++)
    for (int i = 0; i < N; i++) {
      const size_t e = (size_t)i + (size_t)j * N;
      at(0, i, j)[0] = 2.0 * V[e];
      at(0, i, N + j)[0] = 2.0 * T[e];
      at(0, N + i, j)[0] = 2.0 * T[e];
      at(0, N + i, N + j)[0] = 2.0 * (C2 * W[e] - T[e]);
      for (int k = 1; k < 4; k++) at(k, N + i, N + j)[1] = 2.0 * C2 * W[k * NN + e];
    }
  return CQF_OK;
}

}  // extern "C"

namespace cqf {

void launch_block_norms(const cqf_basis* B, const double* X, int cplx, double* out,
                        cudaStream_t st) {
  const size_t ns2 = (size_t)B->nshell * B->nshell;
  block_norms_kernel<<<grid1(ns2, 128), 128, 0, st>>>(X, cplx, B->nbasis, B->d_shells, B->nshell,
                                                      out);
}

void launch_max_norms(const double* nm, int nMat, size_t ns2, double* out,
                      unsigned long long* gmax, cudaStream_t st) {
  max_norms_kernel<<<grid1(ns2, 256), 256, 0, st>>>(nm, nMat, ns2, out, gmax);
}

void launch_from_cart(const cqf_basis* B, const double* Ac, int cplx, int her, double* AX,
                      cudaStream_t st) {
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  from_cart_kernel<<<grid1(NN, 256), 256, 0, st>>>(Ac, cplx, her, B->nbasis, B->ncart,
                                                   B->d_shells, B->d_ao2shell, B->d_sph,
                                                   B->d_sphOff, AX);
}

void launch_to_cart(const cqf_basis* B, const double* X, int cplx, double* Xc, cudaStream_t st) {
  const size_t nc2 = (size_t)B->ncart * B->ncart;
  to_cart_kernel<<<grid1(nc2, 256), 256, 0, st>>>(X, cplx, B->nbasis, B->ncart, B->d_shells,
                                                  B->d_cart2shell, B->d_sph, B->d_sphOff, Xc);
}

cqf_status basis_workspace(cqf_basis* B, size_t bytes) { return ensure_ws(B, bytes); }

WsLayout ws_layout(const cqf_basis* B, int nMat, const cqf_opts& opts) {
  const int cw = opts.is_complex ? 2 : 1;
  const size_t matN = (size_t)B->nbasis * B->nbasis * cw;
  const size_t matC = (size_t)B->ncart * B->ncart * cw;
  const size_t ns2 = (size_t)B->nshell * B->nshell;
  WsLayout L{};
  size_t off = 0;
  auto take = [&](size_t doubles) {
    size_t o = off;
    off += (doubles + 31) / 32 * 32;
    return o;
  };
  const bool host = !opts.device_pointers;
  L.oX = host ? take(matN * nMat) : 0;
  L.oAX = host ? take(matN * nMat) : 0;
  L.oXc = take(matC * nMat);
  L.oAc = take(matC * nMat);
  L.oNm = take(ns2);
  L.oNmM = take(ns2 * nMat);
  L.oG = take(4);
  L.oNmT = take(ns2);
  L.oPN = take((size_t)std::max(1, B->npair));
  L.oWork = take((NWORK + 1) / 2);
  // FP32 copy of the Cartesian densities (mixed real builds)
  const bool mixed = opts.precision == CQF_MIXED && opts.fp32_cutoff > 0.0 && !opts.is_complex;
  L.oXc32 = take(mixed ? (matC * nMat + 1) / 2 : 0);
  // quartet masks of the fast class kernels: one region per launch stream,
  // as many mask words as the largest class pair needs (either orientation)
  // up to MASK_CAP_WORDS, and at least one bra row of the widest class;
  // larger class pairs run in slabs of bra pairs
  size_t need = 0, row = 1;
  for (int cb = 0; cb < NCLS; cb++) {
    row = std::max<size_t>(row, ((size_t)B->cls_cnt[cb] + WTILE - 1) / WTILE);
    for (int ck = 0; ck <= cb; ck++) {
      if (opts.is_complex || !B->cls_cnt[cb] || !B->cls_cnt[ck]) continue;
      const size_t nb = B->cls_cnt[cb], nk = B->cls_cnt[ck];
      need = std::max(need, std::max(nb * ((nk + WTILE - 1) / WTILE),
                                     nk * ((nb + WTILE - 1) / WTILE)));
    }
  }
  L.maskWords = need == 0 ? 0 : std::max(row, std::min(need, MASK_CAP_WORDS));
  // per word: the uint2 mask and one entry in each of the two word lists
  L.oMask = take(std::max<size_t>(2 * L.maskWords * (NAUX + 1), 1));
  L.total = off;
  return L;
}

cqf_status check_contract_args(const cqf_basis* B, const cqf_contraction* list, int nMat) {
  if (!B || !list || nMat <= 0) return fail(CQF_EINVAL, "cqf_two_body_contract: bad argument");
  if (nMat > MAXMAT) return fail(CQF_EINVAL, "too many contractions in one call");
  for (int m = 0; m < nMat; m++) {
    if (!list[m].X || !list[m].AX) return fail(CQF_EINVAL, "null X or AX");
    if (list[m].type != CQF_COULOMB && list[m].type != CQF_EXCHANGE)
      return fail(CQF_EINVAL, "unknown contraction type");
  }
  return CQF_OK;
}

cqf_status contract_core(cqf_basis* B, const cqf_contraction* list, int nMat,
                         const cqf_opts& opts, cqf_stats* stats, double* ws, bool capture,
                         const int* d_flags_pre, const double* const* normSrc,
                         double* pinned);

struct PinnedBuf {
  double* p;
  size_t bytes;
  bool busy;
};
static std::mutex g_pinned_mu;
static std::vector<PinnedBuf> g_pinned;

cqf_status pinned_acquire(size_t bytes, double** out) {
  std::lock_guard<std::mutex> lk(g_pinned_mu);
  PinnedBuf* best = nullptr;
  for (auto& b : g_pinned)
    if (!b.busy && b.bytes >= bytes && (!best || b.bytes < best->bytes)) best = &b;
  if (!best) {
    void* p = nullptr;
    if (cudaHostAlloc(&p, bytes, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();
      return fail(CQF_ENOMEM, "page-locked host staging allocation failed");
    }
    g_pinned.push_back({static_cast<double*>(p), bytes, false});
    best = &g_pinned.back();
  }
  best->busy = true;
  *out = best->p;
  return CQF_OK;
}

void pinned_release(double* p) {
  std::lock_guard<std::mutex> lk(g_pinned_mu);
  for (auto& b : g_pinned)
    if (b.p == p) b.busy = false;
}

// Complex Hermitian densities on the real fast kernels: with X = S + iA (S
// real symmetric, A real antisymmetric), J[X] = J[S] and K[X] = K[S] + i K[A],
// so one real contraction -- J on S, K on S and K on A (flagged
// antisymmetric) -- gives every result; the screen uses the norms of the
// complex X, as the reference's does.  The classes with f shells run on the
// real generic kernel, the others on the fast ones (split_eligible).

bool split_eligible(const cqf_basis* B, const cqf_contraction* list, int nMat,
                    const cqf_opts& opts) {
  if (!opts.is_complex || B->maxL > LMAX) return false;
  int nReal = 0;
  for (int m = 0; m < nMat; m++) {
    if (!list[m].hermitian) return false;
    nReal += list[m].type == CQF_EXCHANGE ? 2 : 1;
  }
  return nReal <= MAXMAT;
}

// The real contraction list of a split, in order: per complex entry its real
// part, and for exchange its imaginary part (hermitian = -1) after it.
int split_real_count(const cqf_contraction* list, int nMat) {
  int n = 0;
  for (int m = 0; m < nMat; m++) n += list[m].type == CQF_EXCHANGE ? 2 : 1;
  return n;
}
void split_flags(const cqf_contraction* list, int nMat, int* fl) {
  int r = 0;
  for (int m = 0; m < nMat; m++) {
    cqf_contraction c{nullptr, nullptr, 1, list[m].type};
    fl[r++] = contraction_flags(c, false);
    if (list[m].type == CQF_EXCHANGE) {
      c.hermitian = -1;
      fl[r++] = contraction_flags(c, false);
    }
  }
}

// Workspace (doubles) of split_core: the real contraction's | real X | real AX.
size_t split_ws_doubles(const cqf_basis* B, int nReal, const cqf_opts& opts) {
  cqf_opts ro = opts;
  ro.is_complex = 0;
  ro.device_pointers = 1;
  const size_t blk = ((size_t)B->nbasis * B->nbasis + 31) / 32 * 32;
  return ws_layout(B, nReal, ro).total + 2 * blk * nReal;
}

// The split on device pointers and a caller-provided workspace; with
// `capture` it only enqueues (stream capture), like contract_core.
cqf_status split_core(cqf_basis* B, const cqf_contraction* list, int nMat, const cqf_opts& opts,
                      cqf_stats* stats, double* ws, bool capture, const int* d_flags_pre) {
  cudaStream_t st = opts.stream ? (cudaStream_t)opts.stream : B->stream;
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  const size_t blk = (NN + 31) / 32 * 32;
  const int nReal = split_real_count(list, nMat);
  cqf_opts ro = opts;
  ro.is_complex = 0;
  ro.device_pointers = 1;
  double* rX = ws + ws_layout(B, nReal, ro).total;
  double* rA = rX + blk * nReal;
  std::vector<cqf_contraction> rl;
  std::vector<const double*> src;
  for (int m = 0; m < nMat; m++) {
    const bool k = list[m].type == CQF_EXCHANGE;
    const double* X = static_cast<const double*>(list[m].X);
    double* re = rX + blk * rl.size();
    split_complex_kernel<<<grid1(NN, 256), 256, 0, st>>>(X, NN, re, k ? re + blk : nullptr);
    rl.push_back({re, rA + blk * rl.size(), 1, list[m].type});
    src.push_back(X);
    if (k) {
      rl.push_back({re + blk, rA + blk * rl.size(), -1, CQF_EXCHANGE});
      src.push_back(X);
    }
  }
  CQF_CUDA(cudaMemsetAsync(rA, 0, blk * nReal * sizeof(double), st));
  CQF_CUDA(cudaGetLastError());
  CQF_TRY(contract_core(B, rl.data(), nReal, ro, stats, ws, capture, d_flags_pre, src.data()));
  for (int m = 0, r = 0; m < nMat; m++) {
    const bool k = list[m].type == CQF_EXCHANGE;
    add_complex_kernel<<<grid1(NN, 256), 256, 0, st>>>(
        static_cast<double*>(list[m].AX), NN, static_cast<const double*>(rl[r].AX),
        k ? static_cast<const double*>(rl[r + 1].AX) : nullptr);
    r += k ? 2 : 1;
  }
  CQF_CUDA(cudaGetLastError());
  return CQF_OK;
}

std::vector<cqf_contraction> normalized_list(const cqf_contraction* list, int nMat,
                                             bool* allHer) {
  std::vector<cqf_contraction> out(list, list + nMat);
  bool all = true;
  for (auto& c : out) {
    c.hermitian = c.hermitian ? 1 : 0;
    all = all && c.hermitian;
  }
  if (allHer) *allHer = all;
  return out;
}

// Workspace of contract_complex_split_on: [split workspace | complex X, AX
// staging (host pointers only)].
size_t complex_split_ws_doubles(const cqf_basis* B, const cqf_contraction* list, int nMat,
                                const cqf_opts& opts) {
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  const size_t blk = (NN + 31) / 32 * 32;
  const size_t inner = split_ws_doubles(B, split_real_count(list, nMat), opts);
  return inner + (opts.device_pointers ? 0 : 4 * blk * nMat);
}

// The split with host pointers staged on the device.  Caller holds B->mu,
// device current.
cqf_status contract_complex_split_on(cqf_basis* B, const cqf_contraction* list, int nMat,
                                     const cqf_opts& opts, cqf_stats* stats, double* ws) {
  cudaStream_t st = opts.stream ? (cudaStream_t)opts.stream : B->stream;
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  const size_t blk = (NN + 31) / 32 * 32;
  const bool host = !opts.device_pointers;
  const size_t inner = split_ws_doubles(B, split_real_count(list, nMat), opts);
  std::vector<cqf_contraction> dl(list, list + nMat);
  if (host) {
    for (int m = 0; m < nMat; m++) {
      double* x = ws + inner + 4 * blk * m;
      double* ax = x + 2 * blk;
      CQF_CUDA(cudaMemcpyAsync(x, list[m].X, 2 * NN * sizeof(double), cudaMemcpyHostToDevice,
                               st));
      CQF_CUDA(cudaMemcpyAsync(ax, list[m].AX, 2 * NN * sizeof(double), cudaMemcpyHostToDevice,
                               st));
      dl[m].X = x;
      dl[m].AX = ax;
    }
  }
  cqf_opts dopts = opts;
  dopts.device_pointers = 1;
  CQF_TRY(split_core(B, dl.data(), nMat, dopts, stats, ws, false, nullptr));
  if (host)
    for (int m = 0; m < nMat; m++)
      CQF_CUDA(cudaMemcpyAsync(list[m].AX, dl[m].AX, 2 * NN * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
  CQF_CUDA(cudaStreamSynchronize(st));
  return CQF_OK;
}

// The contraction pipeline on a caller-provided workspace `ws` of at least
// ws_layout(...).total doubles (device memory).  Caller holds B->mu and has
// made B's device current.
cqf_status contract_core(cqf_basis* B, const cqf_contraction* list, int nMat,
                         const cqf_opts& opts, cqf_stats* stats, double* ws, bool capture,
                         const int* d_flags_pre, const double* const* normSrc,
                         double* pinned) {
  if (opts.shard_count < 1 || opts.shard_index < 0 || opts.shard_index >= opts.shard_count)
    return fail(CQF_EINVAL, "shard_index must lie in [0, shard_count)");
  cudaStream_t st = opts.stream ? (cudaStream_t)opts.stream : B->stream;
  const int N = B->nbasis, nc = B->ncart, ns = B->nshell;
  const int cw = opts.is_complex ? 2 : 1;
  const size_t matN = (size_t)N * N * cw, matC = (size_t)nc * nc * cw;
  const size_t ns2 = (size_t)ns * ns;
  const WsLayout Lw = ws_layout(B, nMat, opts);
  const bool host = !opts.device_pointers;
  const size_t oX = Lw.oX, oAX = Lw.oAX, oXc = Lw.oXc, oAc = Lw.oAc, oNm = Lw.oNm,
               oNmM = Lw.oNmM, oG = Lw.oG;
  if (!capture) CQF_CUDA(cudaEventRecord(B->ev0, st));
  std::vector<const double*> Xd(nMat);
  std::vector<double*> AXd(nMat);
  for (int m = 0; m < nMat; m++) {
    if (host && pinned && !capture) {
      Xd[m] = ws + oX + m * matN;
      AXd[m] = ws + oAX + m * matN;
      CQF_CUDA(cudaMemsetAsync(AXd[m], 0, matN * sizeof(double), st));
      // J and K of one density share X (formRawGDInBatches passes the same
      // onePDM to both): one upload serves every entry with that pointer
      int same = -1;
      for (int k = 0; k < m && same < 0; k++)
        if (list[k].X == list[m].X) same = k;
      if (same >= 0) {
        Xd[m] = Xd[same];
        continue;
      }
      // in pieces: the host copy of one piece overlaps the upload of the last
      const size_t piece = (matN + NSTAGE - 1) / NSTAGE;
      for (size_t o = 0; o < matN; o += piece) {
        const size_t n = std::min(piece, matN - o);
        std::memcpy(pinned + m * matN + o, static_cast<const double*>(list[m].X) + o,
                    n * sizeof(double));
        CQF_CUDA(cudaMemcpyAsync((void*)(Xd[m] + o), pinned + m * matN + o, n * sizeof(double),
                                 cudaMemcpyHostToDevice, st));
      }
    } else if (host) {
      Xd[m] = ws + oX + m * matN;
      AXd[m] = ws + oAX + m * matN;
      CQF_CUDA(cudaMemcpyAsync((void*)Xd[m], list[m].X, matN * sizeof(double),
                               cudaMemcpyHostToDevice, st));
      CQF_CUDA(cudaMemcpyAsync(AXd[m], list[m].AX, matN * sizeof(double), cudaMemcpyHostToDevice,
                               st));
    } else {
      Xd[m] = static_cast<const double*>(list[m].X);
      AXd[m] = static_cast<double*>(list[m].AX);
    }
  }
  // per-matrix flags: uploaded here through pinned staging (every earlier
  // call on this basis has synchronised), or already on the device (graphs)
  const int* d_flags = d_flags_pre;
  if (!d_flags) {
    for (int m = 0; m < nMat; m++) B->h_flags[m] = contraction_flags(list[m], opts.is_complex != 0);
    CQF_CUDA(cudaMemcpyAsync(B->d_flags, B->h_flags.data(), nMat * sizeof(int), cudaMemcpyHostToDevice,
                             st));
    d_flags = B->d_flags;
  }
  CQF_CUDA(cudaMemsetAsync(B->d_counters, 0, 8 * sizeof(unsigned long long), st));
  CQF_CUDA(cudaMemsetAsync(ws + oG, 0, 4 * sizeof(double), st));
  unsigned int* work = reinterpret_cast<unsigned int*>(ws + Lw.oWork);
  CQF_CUDA(cudaMemsetAsync(work, 0, NWORK * sizeof(unsigned int), st));

  // shell-block norms (per matrix, symmetrised when non-Hermitian), max
  for (int m = 0; m < nMat; m++) {
    double* nm = ws + oNmM + m * ns2;
    block_norms_kernel<<<grid1(ns2, 128), 128, 0, st>>>(
        normSrc ? normSrc[m] : Xd[m], normSrc ? 1 : opts.is_complex, N, B->d_shells, ns, nm);
    if (!list[m].hermitian) sym_norms_kernel<<<grid1(ns2, 128), 128, 0, st>>>(nm, ns);
  }
  max_norms_kernel<<<grid1(ns2, 256), 256, 0, st>>>(ws + oNmM, nMat, ns2, ws + oNm,
                                                    reinterpret_cast<unsigned long long*>(ws + oG));
  norms_aux_kernel<<<grid1(std::max(ns2, (size_t)B->npair), 256), 256, 0, st>>>(
      ws + oNm, ns, B->d_pairs, B->npair, ws + Lw.oNmT, ws + Lw.oPN);
  // densities to the Cartesian AO basis, zero accumulators
  for (int m = 0; m < nMat; m++) {
    to_cart_kernel<<<grid1((size_t)nc * nc, 256), 256, 0, st>>>(
        Xd[m], opts.is_complex, N, nc, B->d_shells, B->d_cart2shell, B->d_sph, B->d_sphOff,
        ws + oXc + m * matC);
    if (!list[m].hermitian && hermitian_eff(list[m], opts.is_complex != 0))
      symmetrize_kernel<<<grid1((size_t)nc * nc, 256), 256, 0, st>>>(ws + oXc + m * matC, nc);
  }
  CQF_CUDA(cudaMemsetAsync(ws + oAc, 0, matC * nMat * sizeof(double), st));
  float* Xc32 = reinterpret_cast<float*>(ws + Lw.oXc32);
  const bool mixedReal =
      opts.precision == CQF_MIXED && opts.fp32_cutoff > 0.0 && !opts.is_complex;
  if (mixedReal)
    to_float_kernel<<<(unsigned)std::min<size_t>(grid1(matC * nMat, 256), 4096), 256, 0, st>>>(
        ws + oXc, matC * nMat, Xc32);
  CQF_CUDA(cudaGetLastError());

  JKLaunch a{};
  a.shardIdx = opts.shard_index;
  a.shardCnt = std::max(1, opts.shard_count);
  a.pairs = B->d_pairs;
  a.pp = B->d_pp;
  a.ppQ = B->d_ppQ;
  a.qWin = B->d_qWin;
  a.primK4 = std::pow((double)B->maxPrim, 4);
  a.boys64 = B->d_boys64;
  a.boys32 = B->d_boys32;
  a.screen = opts.screen;
  a.thresh = B->thresh;
  a.norms = ws + oNm;
  a.normsMat = ws + oNmM;
  a.maxNorm = ws + oG;
  a.normsT = ws + Lw.oNmT;
  a.pairNorm = ws + Lw.oPN;
  a.pairRange = B->d_pairRange;
  a.nShell = ns;
  a.nMat = nMat;
  a.cplx = opts.is_complex;
  a.ncart = nc;
  a.flags = d_flags;
  a.Xc = ws + oXc;
  a.Xc32 = mixedReal ? Xc32 : nullptr;
  a.Ac = ws + oAc;
  a.precision = opts.precision;
  a.fp32_cut = opts.fp32_cutoff;
  a.counters = B->d_counters;
  a.ketT = B->d_ketT;
  a.ketT32 = B->d_ketT32;
  a.pp32 = B->d_pp32;
  a.tileOff = B->d_tileOff;
  // closed-shell fast path: real matrices flagged Hermitian (symmetric)
  bool fastOK = !opts.is_complex;
  for (int m = 0; m < nMat; m++) fastOK = fastOK && hermitian_eff(list[m], false);
  // the class kernels go round-robin onto st and the NAUX auxiliary streams
  // (they only add into Ac and the counters: order-free), so each persistent
  // launch's tail overlaps the next one's start; fork here, join after the
  // loop
  CQF_CUDA(cudaEventRecord(B->evFork, st));
  for (int i = 0; i < NAUX; i++) CQF_CUDA(cudaStreamWaitEvent(B->aux[i], B->evFork, 0));
  cudaStream_t lanes[NAUX + 1] = {st};
  for (int i = 0; i < NAUX; i++) lanes[1 + i] = B->aux[i];
  int nlaunch = 0;
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
      a.braTileBeg = B->cls_tile_beg[cb];
      a.ketTileBeg = B->cls_tile_beg[ck];
      const int lm = std::max(std::max(la, lb), std::max(lc, ld));
      // autotuning times each class alone, on st, between two events
      const bool tune = B->tuning && !capture;
      const int li = tune ? 0 : nlaunch++ % (NAUX + 1);
      const cudaStream_t ls = lanes[li];
      if (tune) CQF_CUDA(cudaEventRecord(B->tune_ev[2 * (cb * NCLS + ck)], st));
      uint2* masks = reinterpret_cast<uint2*>(ws + Lw.oMask) + 2 * Lw.maskWords * li;
      a.braOff = 0;
      if (!(fastOK && lm <= 2 &&
            launch_jk_fast(a, la, lb, lc, ld, masks, (long long)Lw.maskWords, work + 4 * li,
                           B->nsm, ls, B->blocks_per_sm[cb][ck])))
        launch_jk_generic(a, la, lb, lc, ld, ls);
      if (tune) CQF_CUDA(cudaEventRecord(B->tune_ev[2 * (cb * NCLS + ck) + 1], st));
    }
  for (int i = 0; i < NAUX; i++) {
    CQF_CUDA(cudaEventRecord(B->evJoin[i], B->aux[i]));
    CQF_CUDA(cudaStreamWaitEvent(st, B->evJoin[i], 0));
  }
  CQF_CUDA(cudaGetLastError());
  for (int m = 0; m < nMat; m++)
    from_cart_kernel<<<grid1((size_t)N * N, 256), 256, 0, st>>>(
        ws + oAc + m * matC, opts.is_complex,
        list[m].hermitian < 0 ? 2 : (hermitian_eff(list[m], opts.is_complex != 0) ? 1 : 0),
        N, nc, B->d_shells,
        B->d_ao2shell, B->d_sph, B->d_sphOff, AXd[m]);
  CQF_CUDA(cudaGetLastError());
  const bool staged = host && pinned && !capture;
  // staged downloads go in NSTAGE pieces over all matrices, an event after
  // each, so that AX += G[X] on the host runs behind the transfer
  const size_t allN = (size_t)nMat * matN, piece = (allN + NSTAGE - 1) / NSTAGE;
  if (staged) {  // AXd[m] = ws + oAX + m matN: one contiguous range
    int i = 0;
    for (size_t o = 0; o < allN; o += piece, i++) {
      CQF_CUDA(cudaMemcpyAsync(pinned + allN + o, ws + oAX + o,
                               std::min(piece, allN - o) * sizeof(double),
                               cudaMemcpyDeviceToHost, st));
      CQF_CUDA(cudaEventRecord(B->evStage[i], st));
    }
  } else if (host) {
    for (int m = 0; m < nMat; m++)
      CQF_CUDA(cudaMemcpyAsync(list[m].AX, AXd[m], matN * sizeof(double), cudaMemcpyDeviceToHost,
                               st));
  }
  if (capture) return CQF_OK;
  CQF_CUDA(cudaEventRecord(B->ev1, st));
  unsigned long long cnt[4] = {0, 0, 0, 0};
  CQF_CUDA(cudaMemcpyAsync(cnt, B->d_counters, 4 * sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, st));
  if (staged) {  // AX += G[X] on the host, each piece once it has landed
    int i = 0;
    for (size_t o = 0; o < allN; o += piece, i++) {
      CQF_CUDA(cudaEventSynchronize(B->evStage[i]));
      const size_t end = std::min(o + piece, allN);
      for (size_t e = o; e < end;) {
        const size_t m = e / matN, off = e % matN, n = std::min(end - e, matN - off);
        double* ax = static_cast<double*>(list[m].AX) + off;
        const double* g = pinned + allN + e;
        for (size_t k = 0; k < n; k++) ax[k] += g[k];
        e += n;
      }
    }
  }
  CQF_CUDA(cudaStreamSynchronize(st));
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


}  // namespace cqf

extern "C" {

cqf_status cqf_autotune(cqf_basis* B, const cqf_contraction* listIn, int nMat,
                        const cqf_opts* optsIn, const char* cache_path, int* from_cache) {
  g_err.clear();
  CQF_TRY(check_contract_args(B, listIn, nMat));
  cqf_opts opts;
  cqf_opts_default(&opts);
  if (optsIn) opts = *optsIn;
  if (from_cache) *from_cache = 0;
  bool allHer = true;
  std::vector<cqf_contraction> list = normalized_list(listIn, nMat, &allHer);
  // which kernels the contraction runs: only the persistent fast kernels
  // (real Hermitian-effective matrices, l <= 2; complex Hermitian densities
  // through their real split) have launch shapes to tune
  const bool csplit = opts.is_complex && allHer && split_eligible(B, list.data(), nMat, opts);
  bool fast = !opts.is_complex;
  for (int m = 0; m < nMat && fast; m++) fast = hermitian_eff(list[m], false);
  if (!(fast || csplit)) return CQF_OK;  // generic kernels only: nothing to tune
  std::lock_guard<std::mutex> lk(B->mu);
  CQF_CUDA(cudaSetDevice(B->device));
  cudaDeviceProp prop;
  CQF_CUDA(cudaGetDeviceProperties(&prop, B->device));
  std::string gpu = prop.name;
  for (char& c : gpu)
    if (c == ' ') c = '_';
  const char* kind = csplit ? "csplit" : "real";
  // key of a class pair: GPU, contraction kind, angular momenta, size bucket
  // log2(nBra nKet), precision
  auto key = [&](int cb, int ck) {
    int la, lb, lc, ld;
    class_ls(cb, la, lb);
    class_ls(ck, lc, ld);
    const double n = std::max(1.0, (double)B->cls_cnt[cb] * B->cls_cnt[ck]);
    return gpu + " " + kind + " " + std::to_string(la) + std::to_string(lb) +
           std::to_string(lc) + std::to_string(ld) + " " + std::to_string((int)std::log2(n)) +
           " " + (opts.precision == CQF_MIXED && opts.fp32_cutoff > 0.0 ? "mixed" : "fp64");
  };
  auto valid_shape = [](int v) { return v == 2 || v == 4 || v == 8 || v == 16; };
  std::vector<std::pair<int, int>> pairs;
  for (int cb = 0; cb < NCLS; cb++)
    for (int ck = 0; ck <= cb; ck++)
      if (B->cls_cnt[cb] && B->cls_cnt[ck]) pairs.push_back({cb, ck});
  // cached choices (values other than the candidates are ignored: the class
  // pair is measured again)
  std::map<std::string, int> cache;
  if (cache_path) {
    if (FILE* f = std::fopen(cache_path, "r")) {
      char k1[256], k2[64], k3[64], k4[64], k5[64];
      int v;
      while (std::fscanf(f, "%255s %63s %63s %63s %63s %d", k1, k2, k3, k4, k5, &v) == 6)
        if (valid_shape(v))
          cache[std::string(k1) + " " + k2 + " " + k3 + " " + k4 + " " + k5] = v;
      std::fclose(f);
    }
  }
  bool all = !pairs.empty();
  for (auto& p : pairs) all = all && cache.count(key(p.first, p.second));
  if (all) {
    for (auto& p : pairs) B->blocks_per_sm[p.first][p.second] = cache[key(p.first, p.second)];
    if (from_cache) *from_cache = 1;
    return CQF_OK;
  }
  // measure: every candidate on the real contraction that runs, each class
  // timed alone; the shapes in use are restored if anything fails
  int saved[NCLS][NCLS];
  std::memcpy(saved, B->blocks_per_sm, sizeof saved);
  const size_t NN = (size_t)B->nbasis * B->nbasis;
  std::vector<double*> buf;
  std::vector<cqf_contraction> tl;
  auto release = [&](bool restore) {
    for (double* p : buf) cudaFree(p);
    B->tuning = false;
    if (restore) std::memcpy(B->blocks_per_sm, saved, sizeof saved);
  };
  auto dev_alloc = [&](size_t doubles) -> double* {
    double* p = nullptr;
    if (cudaMalloc(&p, doubles * sizeof(double)) != cudaSuccess) return nullptr;
    buf.push_back(p);
    return p;
  };
  for (int m = 0; m < nMat; m++) {
    const size_t cw = opts.is_complex ? 2 : 1;
    double* x = dev_alloc(cw * NN);
    if (!x || cudaMemcpy(x, list[m].X, cw * NN * sizeof(double), cudaMemcpyDefault) !=
                  cudaSuccess) {
      release(true);
      return fail(CQF_ENOMEM, "cqf_autotune: scratch allocation / copy");
    }
    if (!csplit) {
      double* ax = dev_alloc(NN);
      if (!ax) {
        release(true);
        return fail(CQF_ENOMEM, "cqf_autotune: scratch allocation");
      }
      tl.push_back({x, ax, list[m].hermitian, list[m].type});
      continue;
    }
    // the split of a complex Hermitian density: its real part, and for
    // exchange its imaginary part (antisymmetric) as a second real entry
    const bool k = list[m].type == CQF_EXCHANGE;
    double* re = dev_alloc(NN);
    double* im = k ? dev_alloc(NN) : nullptr;
    double* ax = dev_alloc(NN);
    double* ax2 = k ? dev_alloc(NN) : nullptr;
    if (!re || !ax || (k && (!im || !ax2))) {
      release(true);
      return fail(CQF_ENOMEM, "cqf_autotune: scratch allocation");
    }
    split_complex_kernel<<<grid1(NN, 256), 256, 0, B->stream>>>(x, NN, re, im);
    tl.push_back({re, ax, 1, list[m].type});
    if (k) tl.push_back({im, ax2, -1, CQF_EXCHANGE});
  }
  if (cudaStreamSynchronize(B->stream) != cudaSuccess || (int)tl.size() > MAXMAT) {
    release(true);
    return fail(CQF_ECUDA, "cqf_autotune: preparing the real contraction");
  }
  const int nT = (int)tl.size();
  cqf_opts to = opts;
  to.device_pointers = 1;
  to.is_complex = 0;
  to.stream = nullptr;
  if (B->tune_ev.empty()) {
    B->tune_ev.assign(2 * NCLS * NCLS, nullptr);
    for (auto& e : B->tune_ev)
      if (cudaEventCreate(&e) != cudaSuccess) {
        release(true);
        return fail(CQF_ECUDA, "cqf_autotune: event creation");
      }
  }
  if (ensure_ws(B, ws_layout(B, nT, to).total * sizeof(double)) != CQF_OK) {
    release(true);
    return CQF_ENOMEM;
  }
  const int cand[4] = {2, 4, 8, 16};
  std::vector<float> best(NCLS * NCLS, 1e30f);
  std::vector<int> choice(NCLS * NCLS, 8);
  B->tuning = true;
  for (int c : cand) {
    for (auto& p : pairs) B->blocks_per_sm[p.first][p.second] = c;
    for (int rep = 0; rep < 2; rep++) {  // the first run loads and warms
      cqf_status st = contract_core(B, tl.data(), nT, to, nullptr,
                                    static_cast<double*>(B->d_ws), false, nullptr);
      if (st != CQF_OK) {
        release(true);
        return st;
      }
    }
    for (auto& p : pairs) {
      const int k = p.first * NCLS + p.second;
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, B->tune_ev[2 * k], B->tune_ev[2 * k + 1]) == cudaSuccess &&
          ms < best[k]) {
        best[k] = ms;
        choice[k] = c;
      }
    }
  }
  release(false);
  for (auto& p : pairs) B->blocks_per_sm[p.first][p.second] = choice[p.first * NCLS + p.second];
  if (cache_path) {
    if (FILE* f = std::fopen(cache_path, "a")) {
      for (auto& p : pairs) {
        const std::string k = key(p.first, p.second);
        if (!cache.count(k))
          std::fprintf(f, "%s %d\n", k.c_str(), choice[p.first * NCLS + p.second]);
      }
      std::fclose(f);
    } else {
      return fail(CQF_EINVAL, std::string("cqf_autotune: cannot write ") + cache_path);
    }
  }
  return CQF_OK;
}

cqf_status cqf_two_body_contract(cqf_basis* B, const cqf_contraction* listIn, int nMat,
                                 const cqf_opts* optsIn, cqf_stats* stats) {
  g_err.clear();
  CQF_TRY(check_contract_args(B, listIn, nMat));
  cqf_opts opts;
  cqf_opts_default(&opts);
  if (optsIn) opts = *optsIn;
  bool allHer = true;
  std::vector<cqf_contraction> list = normalized_list(listIn, nMat, &allHer);
  std::lock_guard<std::mutex> lk(B->mu);
  CQF_CUDA(cudaSetDevice(B->device));
  if (allHer && split_eligible(B, list.data(), nMat, opts)) {
    CQF_TRY(ensure_ws(B, complex_split_ws_doubles(B, list.data(), nMat, opts) * sizeof(double)));
    return contract_complex_split_on(B, list.data(), nMat, opts, stats,
                                     static_cast<double*>(B->d_ws));
  }
  CQF_TRY(ensure_ws(B, ws_layout(B, nMat, opts).total * sizeof(double)));
  if (opts.device_pointers)
    return contract_core(B, list.data(), nMat, opts, stats, static_cast<double*>(B->d_ws),
                         false, nullptr);
  // host pointers: X up and the result down through a pooled page-locked
  // buffer (contract_core synchronises before returning)
  const size_t matN = (size_t)B->nbasis * B->nbasis * (opts.is_complex ? 2 : 1);
  double* pinned = nullptr;
  CQF_TRY(pinned_acquire(2 * nMat * matN * sizeof(double), &pinned));
  const cqf_status s = contract_core(B, list.data(), nMat, opts, stats,
                                     static_cast<double*>(B->d_ws), false, nullptr, nullptr,
                                     pinned);
  pinned_release(pinned);
  return s;
}

}  // extern "C"
