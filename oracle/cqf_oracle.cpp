// CPU oracle for the direct two-electron (J/K) contraction.
//
// TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
// product and the timed CPU baseline ("port" of the reference loop).  Only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
// may load the library built from it.  Nothing in chronusq_public_b200/ links
// or calls it.
//
// What it restates (file:line in xsligroup/chronusq_public):
//   * GTODirectTPIContraction::directScaffoldNew
//       include/particleintegrals/contract/direct.hpp:1412-2123
//     - shell-block infinity norms            direct.hpp:73-105, :1518-1561
//     - 8-fold quartet loop + round robin     direct.hpp:1642-1730
//     - Schwarz x density screen, per matrix  direct.hpp:1733-1786
//     - degeneracy, 0.5*deg buffer scaling    direct.hpp:1791-1803, :1849-1850
//     - J/K digestion (4 code branches)       direct.hpp:1858-2002
//     - thread reduction + Hermitisation      direct.hpp:2036-2066
//   * DirectTPI::computeSchwarz
//       src/particleintegrals/aointegrals/aointegrals_utilities.cxx:53-162
//   * ShellPairData::computeShellPairs (significant pairs)
//       src/basisset/basisset.cxx:652-706
//   * Boys function: Taylor table with dT = 0.025 and 6 correction terms plus
//     downward recursion, the scheme of RealGTOIntEngine::computeFmTTaylor
//     (src/particleintegrals/aointegrals/aointegrals_onee_inhouse.cxx:79-170;
//     Obara & Saika, JCP 84, 3963).  The table is generated here in long
//     double by the convergent series; above T = 36 the value is
//     F_0 = sqrt(pi/T)/2 with upward recursion that keeps the exp(-T) term.
//
// The reference's ERIs come from libint2 (libint-cq 2.7.0-beta.6), which is
// not present; this oracle computes them by the McMurchie-Davidson scheme
// (McMurchie & Davidson, J. Comput. Phys. 26, 218 (1978); Helgaker,
// Jorgensen & Olsen ch. 9) restated from the mathematics.  libint's own
// primitive screening (precision >= machine epsilon) drops terms below
// ~1e-15 relative and is not mimicked.
//
// Build: see oracle/Makefile (g++ -O3 -march=native -fopenmp -shared).

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include <omp.h>

namespace {

using dcomplex = std::complex<double>;

// ---------------------------------------------------------------- utilities
inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

double dfact(int n) {  // n!!, (-1)!! = 1
  double r = 1.0;
  while (n > 1) { r *= n; n -= 2; }
  return r;
}

double binom(int n, int k) {
  if (k < 0 || k > n) return 0.0;
  double r = 1.0;
  for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
  return r;
}

double fact(int n) { double r = 1; for (int i = 2; i <= n; i++) r *= i; return r; }

// Cartesian exponents in libint/CCA order.
void cart_list(int l, std::vector<int>& lx, std::vector<int>& ly,
               std::vector<int>& lz) {
  lx.clear(); ly.clear(); lz.clear();
  for (int i = 0; i <= l; i++)
    for (int j = 0; j <= i; j++) {
      lx.push_back(l - i); ly.push_back(i - j); lz.push_back(j);
    }
}

// Real solid harmonics, Helgaker/Jorgensen/Olsen eq. 6.4.47-6.4.50.
// Returns T[i_cart * nsph + (m + l)].
std::vector<double> solid_harmonics(int l) {
  std::vector<int> lx, ly, lz;
  cart_list(l, lx, ly, lz);
  int nc = ncart(l), ns = 2 * l + 1;
  std::vector<double> T(nc * ns, 0.0);
  for (int m = -l; m <= l; m++) {
    int am = std::abs(m);
    // v runs over integers (m >= 0) or half-integers (m < 0); use 2v.
    int vm2 = (m >= 0) ? 0 : 1;
    double N = 1.0 / (std::pow(2.0, am) * fact(l)) *
               std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
    for (int t = 0; t <= (l - am) / 2; t++)
      for (int u = 0; u <= t; u++) {
        // v from v_m to floor(|m|/2 - v_m) + v_m
        int vmax2 = 2 * (int)std::floor(am / 2.0 - vm2 / 2.0) + vm2;
        for (int v2 = vm2; v2 <= vmax2; v2 += 2) {
          int sgn_exp = t + (v2 - vm2) / 2;
          double C = ((sgn_exp % 2) ? -1.0 : 1.0) * std::pow(0.25, t) *
                     binom(l, t) * binom(l - t, am + t) * binom(t, u) *
                     binom(am, v2);
          int ex = 2 * t + am - (2 * u + v2);
          int ey = 2 * u + v2;
          int ez = l - 2 * t - am;
          for (int i = 0; i < nc; i++)
            if (lx[i] == ex && ly[i] == ey && lz[i] == ez)
              T[i * ns + (m + l)] += N * C;
        }
      }
  }
  return T;
}

// ---------------------------------------------------------------- Boys
struct BoysTable {
  static constexpr int MMAX = 48;   // orders tabulated (need m + 6)
  static constexpr double DT = 0.025;
  static constexpr double TCRIT = 36.0;
  int npts;
  std::vector<double> tab;  // [i][m]
  BoysTable() {
    npts = (int)(TCRIT / DT) + 8;
    tab.assign((size_t)npts * (MMAX + 1), 0.0);
    for (int i = 0; i < npts; i++) {
      long double T = (long double)i * DT;
      // series: F_M(T) = e^{-T} sum_k (2T)^k / ((2M+1)(2M+3)...(2M+2k+1))
      long double term = 1.0L / (2 * MMAX + 1), sum = term;
      for (int k = 1; k < 4000; k++) {
        term *= 2.0L * T / (2 * MMAX + 2 * k + 1);
        sum += term;
        if (term < sum * 1e-22L) break;
      }
      long double eT = std::exp(-T);
      long double F = eT * sum;
      tab[(size_t)i * (MMAX + 1) + MMAX] = (double)F;
      for (int m = MMAX - 1; m >= 0; m--) {
        F = (2.0L * T * F + eT) / (2 * m + 1);
        tab[(size_t)i * (MMAX + 1) + m] = (double)F;
      }
    }
  }
  // F_0..F_mmax at T
  void eval(int mmax, double T, double* F) const {
    if (T > TCRIT) {
      double eT = std::exp(-T);
      F[0] = 0.5 * std::sqrt(M_PI / T) * std::erf(std::sqrt(T));
      for (int m = 0; m < mmax; m++) F[m + 1] = ((2 * m + 1) * F[m] - eT) / (2.0 * T);
      return;
    }
    int j = (int)(T / DT + 0.5);
    double dT = j * DT - T;  // expand about the nearest grid point
    const double* row = &tab[(size_t)j * (MMAX + 1)];
    double sum = row[mmax], tmp = 1.0;
    for (int i = 1; i <= 6; i++) {
      tmp *= dT / i;
      sum += tmp * row[mmax + i];
    }
    F[mmax] = sum;
    double eT = std::exp(-T), twoT = 2.0 * T;
    for (int m = mmax - 1; m >= 0; m--) F[m] = (twoT * F[m + 1] + eT) / (2 * m + 1);
  }
};

const BoysTable& boys() {
  static BoysTable t;
  return t;
}

// ---------------------------------------------------------------- basis
struct Shell {
  int l;
  bool pure;
  std::vector<double> alpha, coef;  // normalised (libint convention)
  double O[3];
  int size() const { return pure ? 2 * l + 1 : ncart(l); }
};

std::vector<double> normalize(int l, const std::vector<double>& a,
                              const std::vector<double>& c0) {
  int n = (int)a.size();
  double df = dfact(2 * l - 1);
  std::vector<double> c(n);
  for (int i = 0; i < n; i++)
    c[i] = c0[i] * std::sqrt(std::pow(2.0 * a[i] / M_PI, 1.5) *
                             std::pow(4.0 * a[i], l) / df);
  double norm = 0.0;
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) {
      double ab = a[i] + a[j];
      norm += c[i] * c[j] * df / std::pow(2.0 * ab, l) * std::pow(M_PI / ab, 1.5);
    }
  for (auto& x : c) x /= std::sqrt(norm);
  return c;
}

// Hermite expansion coefficients E^{ij}_t (Helgaker eq. 9.5.6), one axis,
// without the exp(-mu X_AB^2) factor.  E[(i*(lb+1)+j)*(la+lb+1)+t].
void hermite_E(int la, int lb, double p, double PA, double PB,
               std::vector<double>& E) {
  int L = la + lb + 1;
  E.assign((size_t)(la + 1) * (lb + 1) * L, 0.0);
  auto at = [&](int i, int j, int t) -> double& {
    return E[((size_t)i * (lb + 1) + j) * L + t];
  };
  auto get = [&](int i, int j, int t) -> double {
    if (t < 0 || t > i + j) return 0.0;
    return E[((size_t)i * (lb + 1) + j) * L + t];
  };
  double o2p = 0.5 / p;
  at(0, 0, 0) = 1.0;
  for (int i = 0; i <= la; i++)
    for (int j = 0; j <= lb; j++) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; t++) {
        if (j == 0) {
          at(i, j, t) = o2p * get(i - 1, j, t - 1) + PA * get(i - 1, j, t) +
                        (t + 1) * get(i - 1, j, t + 1);
        } else {
          at(i, j, t) = o2p * get(i, j - 1, t - 1) + PB * get(i, j - 1, t) +
                        (t + 1) * get(i, j - 1, t + 1);
        }
      }
    }
}

// Primitive pair data (a cached "shell pair", cf. libint2::ShellPair).
struct PrimPair {
  double p, P[3], K;                 // K = ca*cb*exp(-mu AB^2)
  std::vector<double> Ex, Ey, Ez;
};
struct PairData {
  int la, lb;
  std::vector<PrimPair> prims;
};

PairData make_pair(const Shell& A, const Shell& B) {
  PairData pd;
  pd.la = A.l; pd.lb = B.l;
  double AB2 = 0;
  for (int x = 0; x < 3; x++) AB2 += (A.O[x] - B.O[x]) * (A.O[x] - B.O[x]);
  for (size_t i = 0; i < A.alpha.size(); i++)
    for (size_t j = 0; j < B.alpha.size(); j++) {
      PrimPair pp;
      double a = A.alpha[i], b = B.alpha[j];
      pp.p = a + b;
      double mu = a * b / pp.p;
      for (int x = 0; x < 3; x++) pp.P[x] = (a * A.O[x] + b * B.O[x]) / pp.p;
      pp.K = A.coef[i] * B.coef[j] * std::exp(-mu * AB2);
      hermite_E(A.l, B.l, pp.p, pp.P[0] - A.O[0], pp.P[0] - B.O[0], pp.Ex);
      hermite_E(A.l, B.l, pp.p, pp.P[1] - A.O[1], pp.P[1] - B.O[1], pp.Ey);
      hermite_E(A.l, B.l, pp.p, pp.P[2] - A.O[2], pp.P[2] - B.O[2], pp.Ez);
      pd.prims.push_back(std::move(pp));
    }
  return pd;
}

struct Basis {
  std::vector<Shell> shells;
  std::vector<int> off;  // first AO of each shell
  int nbasis = 0, maxL = 0, maxPrim = 0;
  std::vector<std::vector<double>> sph;  // solid harmonics per l
  std::vector<std::vector<int>> cx, cy, cz;
  // significant pairs: sig[s1] = sorted s2 <= s1 (basisset.cxx:652-706)
  std::vector<std::vector<int>> sig;
  std::vector<double> schwarz;  // nShell x nShell (col-major, symmetric)
  bool have_schwarz = false;
  std::vector<PairData> pairs;  // lower-triangle index s1*(s1+1)/2+s2 (s1>=s2)

  const PairData& pair(int s1, int s2) const {
    return pairs[(size_t)s1 * (s1 + 1) / 2 + s2];
  }
};

// ---------------------------------------------------------------- 1e ints
// Overlap / kinetic of two primitive-contracted shells, Cartesian, via E.
void cart_overlap_kinetic(const Shell& A, const Shell& B, const Basis& bs,
                          std::vector<double>& S, std::vector<double>& T) {
  int na = ncart(A.l), nb = ncart(B.l);
  S.assign(na * nb, 0.0);
  T.assign(na * nb, 0.0);
  double AB2 = 0;
  for (int x = 0; x < 3; x++) AB2 += (A.O[x] - B.O[x]) * (A.O[x] - B.O[x]);
  const auto &ax = bs.cx[A.l], &ay = bs.cy[A.l], &az = bs.cz[A.l];
  const auto &bx = bs.cx[B.l], &by = bs.cy[B.l], &bz = bs.cz[B.l];
  for (size_t i = 0; i < A.alpha.size(); i++)
    for (size_t j = 0; j < B.alpha.size(); j++) {
      double a = A.alpha[i], b = B.alpha[j], p = a + b, mu = a * b / p;
      double P[3];
      for (int x = 0; x < 3; x++) P[x] = (a * A.O[x] + b * B.O[x]) / p;
      double K = A.coef[i] * B.coef[j] * std::exp(-mu * AB2);
      // 1D overlaps S^x_{ij} for i <= la, j <= lb+2 (for kinetic)
      std::vector<double> E[3];
      int lb2 = B.l + 2;
      hermite_E(A.l, lb2, p, P[0] - A.O[0], P[0] - B.O[0], E[0]);
      hermite_E(A.l, lb2, p, P[1] - A.O[1], P[1] - B.O[1], E[1]);
      hermite_E(A.l, lb2, p, P[2] - A.O[2], P[2] - B.O[2], E[2]);
      int L = A.l + lb2 + 1;
      double sq = std::sqrt(M_PI / p);
      auto s1d = [&](int x, int ii, int jj) -> double {
        if (jj < 0) return 0.0;
        return E[x][((size_t)ii * (lb2 + 1) + jj) * L + 0] * sq;
      };
      for (int u = 0; u < na; u++)
        for (int v = 0; v < nb; v++) {
          int ia[3] = {ax[u], ay[u], az[u]};
          int jb[3] = {bx[v], by[v], bz[v]};
          double s[3], t[3];
          for (int x = 0; x < 3; x++) {
            s[x] = s1d(x, ia[x], jb[x]);
            int l = jb[x];
            t[x] = -2.0 * b * b * s1d(x, ia[x], l + 2) + b * (2 * l + 1) * s1d(x, ia[x], l) -
                   0.5 * l * (l - 1) * s1d(x, ia[x], l - 2);
          }
          S[u * nb + v] += K * s[0] * s[1] * s[2];
          T[u * nb + v] += K * (t[0] * s[1] * s[2] + s[0] * t[1] * s[2] + s[0] * s[1] * t[2]);
        }
    }
}

// Transform a row-major block with Cartesian index dims to the shells' AO
// dims (spherical where pure).  dims[k] = ncart of index k; sh[k] shell.
void cart_to_sph_block(const Basis& bs, const Shell* const* sh, int nidx,
                       std::vector<double>& buf) {
  std::vector<int> dims(nidx);
  for (int k = 0; k < nidx; k++) dims[k] = ncart(sh[k]->l);
  for (int k = 0; k < nidx; k++) {
    if (!sh[k]->pure) continue;
    int nc = ncart(sh[k]->l), ns = 2 * sh[k]->l + 1;
    const double* Tm = bs.sph[sh[k]->l].data();
    size_t outer = 1, inner = 1;
    for (int q = 0; q < k; q++) outer *= dims[q];
    for (int q = k + 1; q < nidx; q++) inner *= dims[q];
    std::vector<double> out(outer * ns * inner, 0.0);
    for (size_t o = 0; o < outer; o++)
      for (int c = 0; c < nc; c++)
        for (int m = 0; m < ns; m++) {
          double t = Tm[c * ns + m];
          if (t == 0.0) continue;
          const double* src = &buf[(o * nc + c) * inner];
          double* dst = &out[(o * ns + m) * inner];
          for (size_t i = 0; i < inner; i++) dst[i] += t * src[i];
        }
    buf.swap(out);
    dims[k] = ns;
  }
}

// ---------------------------------------------------------------- ERIs
// Contracted (s1 s2 | s3 s4) in AO order i,j,k,l row-major (as libint).
void eri_quartet(const Basis& bs, int s1, int s2, int s3, int s4,
                 std::vector<double>& out, std::vector<double>& scratch) {
  const Shell &A = bs.shells[s1], &B = bs.shells[s2], &C = bs.shells[s3],
              &D = bs.shells[s4];
  // pair data is cached for s1 >= s2 only; build on the fly otherwise.
  PairData tmpab, tmpcd;
  const PairData* ab;
  const PairData* cd;
  if (s1 >= s2 && !bs.pairs.empty()) ab = &bs.pair(s1, s2);
  else { tmpab = make_pair(A, B); ab = &tmpab; }
  if (s3 >= s4 && !bs.pairs.empty()) cd = &bs.pair(s3, s4);
  else { tmpcd = make_pair(C, D); cd = &tmpcd; }

  int la = A.l, lb = B.l, lc = C.l, ld = D.l;
  int lab = la + lb, lcd = lc + ld, L = lab + lcd;
  int na = ncart(la), nb = ncart(lb), nc = ncart(lc), nd = ncart(ld);
  size_t nabcd = (size_t)na * nb * nc * nd;
  out.assign(nabcd, 0.0);
  const auto &ax = bs.cx[la], &ay = bs.cy[la], &az = bs.cz[la];
  const auto &bx = bs.cx[lb], &by = bs.cy[lb], &bz = bs.cz[lb];
  const auto &cx = bs.cx[lc], &cy = bs.cy[lc], &cz = bs.cz[lc];
  const auto &dx = bs.cx[ld], &dy = bs.cy[ld], &dz = bs.cz[ld];
  int L1 = L + 1;
  // R[t][u][v] for t+u+v <= L, stored densely (L+1)^3
  std::vector<double>& R = scratch;
  size_t RS = (size_t)L1 * L1 * L1;
  R.assign(RS * (L + 1), 0.0);
  auto Ridx = [&](int n, int t, int u, int v) -> size_t {
    return (((size_t)n * L1 + t) * L1 + u) * L1 + v;
  };
  double F[64];
  // intermediate G[cd][t][u][v] over bra Hermite indices (t+u+v <= lab)
  int Lb1 = lab + 1;
  std::vector<double> G((size_t)nc * nd * Lb1 * Lb1 * Lb1);
  const int Lab1 = lab + 1, Lcd1 = lcd + 1;
  for (const auto& pq1 : ab->prims) {
    std::fill(G.begin(), G.end(), 0.0);
    for (const auto& pq2 : cd->prims) {
      double p = pq1.p, q = pq2.p, alpha = p * q / (p + q);
      double PQ[3] = {pq1.P[0] - pq2.P[0], pq1.P[1] - pq2.P[1], pq1.P[2] - pq2.P[2]};
      double T = alpha * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
      double pref = 2.0 * std::pow(M_PI, 2.5) / (p * q * std::sqrt(p + q)) * pq1.K * pq2.K;
      boys().eval(L, T, F);
      // R^{(n)}_{000}
      double m2a = -2.0 * alpha, f = 1.0;
      for (int n = 0; n <= L; n++) { R[Ridx(n, 0, 0, 0)] = f * F[n]; f *= m2a; }
      for (int n = L - 1; n >= 0; n--) {
        int top = L - n;
        for (int t = 0; t <= top; t++)
          for (int u = 0; u <= top - t; u++)
            for (int v = 0; v <= top - t - u; v++) {
              if (t + u + v == 0) continue;
              double val;
              if (t > 0) {
                val = PQ[0] * R[Ridx(n + 1, t - 1, u, v)];
                if (t > 1) val += (t - 1) * R[Ridx(n + 1, t - 2, u, v)];
              } else if (u > 0) {
                val = PQ[1] * R[Ridx(n + 1, t, u - 1, v)];
                if (u > 1) val += (u - 1) * R[Ridx(n + 1, t, u - 2, v)];
              } else {
                val = PQ[2] * R[Ridx(n + 1, t, u, v - 1)];
                if (v > 1) val += (v - 1) * R[Ridx(n + 1, t, u, v - 2)];
              }
              R[Ridx(n, t, u, v)] = val;
            }
      }
      // G[cd][tuv] += pref * sum_{tau nu phi} (-1)^{..} E^cd R_{t+tau,...}
      for (int c = 0; c < nc; c++)
        for (int d = 0; d < nd; d++) {
          int ic[3] = {cx[c], cy[c], cz[c]}, id[3] = {dx[d], dy[d], dz[d]};
          const double* Ecx = &pq2.Ex[((size_t)ic[0] * (ld + 1) + id[0]) * Lcd1];
          const double* Ecy = &pq2.Ey[((size_t)ic[1] * (ld + 1) + id[1]) * Lcd1];
          const double* Ecz = &pq2.Ez[((size_t)ic[2] * (ld + 1) + id[2]) * Lcd1];
          double* g = &G[((size_t)c * nd + d) * Lb1 * Lb1 * Lb1];
          for (int t = 0; t <= lab; t++)
            for (int u = 0; u <= lab - t; u++)
              for (int v = 0; v <= lab - t - u; v++) {
                double s = 0.0;
                for (int ta = 0; ta <= ic[0] + id[0]; ta++)
                  for (int nu = 0; nu <= ic[1] + id[1]; nu++)
                    for (int ph = 0; ph <= ic[2] + id[2]; ph++) {
                      double e = Ecx[ta] * Ecy[nu] * Ecz[ph];
                      if ((ta + nu + ph) & 1) e = -e;
                      s += e * R[Ridx(0, t + ta, u + nu, v + ph)];
                    }
                g[(t * Lb1 + u) * Lb1 + v] += pref * s;
              }
        }
    }
    // (ab|cd) += sum_tuv E^ab_tuv G[cd][tuv]
    for (int a = 0; a < na; a++)
      for (int b = 0; b < nb; b++) {
        int ia[3] = {ax[a], ay[a], az[a]}, ib[3] = {bx[b], by[b], bz[b]};
        const double* Ex = &pq1.Ex[((size_t)ia[0] * (lb + 1) + ib[0]) * Lab1];
        const double* Ey = &pq1.Ey[((size_t)ia[1] * (lb + 1) + ib[1]) * Lab1];
        const double* Ez = &pq1.Ez[((size_t)ia[2] * (lb + 1) + ib[2]) * Lab1];
        for (int cdi = 0; cdi < nc * nd; cdi++) {
          const double* g = &G[(size_t)cdi * Lb1 * Lb1 * Lb1];
          double s = 0.0;
          for (int t = 0; t <= ia[0] + ib[0]; t++)
            for (int u = 0; u <= ia[1] + ib[1]; u++)
              for (int v = 0; v <= ia[2] + ib[2]; v++)
                s += Ex[t] * Ey[u] * Ez[v] * g[(t * Lb1 + u) * Lb1 + v];
          out[((size_t)a * nb + b) * nc * nd + cdi] += s;
        }
      }
  }
  const Shell* sh[4] = {&A, &B, &C, &D};
  cart_to_sph_block(bs, sh, 4, out);
}

void build_pairs(Basis& bs) {
  int ns = (int)bs.shells.size();
  bs.pairs.resize((size_t)ns * (ns + 1) / 2);
#pragma omp parallel for schedule(dynamic)
  for (int s1 = 0; s1 < ns; s1++)
    for (int s2 = 0; s2 <= s1; s2++)
      bs.pairs[(size_t)s1 * (s1 + 1) / 2 + s2] = make_pair(bs.shells[s1], bs.shells[s2]);
}

// Overlap block (spherical where pure), row-major n1 x n2.
void overlap_block(const Basis& bs, int s1, int s2, std::vector<double>& S) {
  std::vector<double> T;
  cart_overlap_kinetic(bs.shells[s1], bs.shells[s2], bs, S, T);
  const Shell* sh[2] = {&bs.shells[s1], &bs.shells[s2]};
  cart_to_sph_block(bs, sh, 2, S);
}

// Significant shell pairs: same centre, or ||S_ab||_2 >= 1e-12
// (ShellPairData::computeShellPairs, basisset.cxx:652-706; centres compared
// with the 1e-5 Bohr tolerance of BasisSet::update, basisset.cxx:146-156).
void build_sig_pairs(Basis& bs) {
  int ns = (int)bs.shells.size();
  bs.sig.assign(ns, {});
  std::vector<double> S;
  for (int s1 = 0; s1 < ns; s1++) {
    for (int s2 = 0; s2 <= s1; s2++) {
      const Shell &A = bs.shells[s1], &B = bs.shells[s2];
      bool same = std::abs(A.O[0] - B.O[0]) < 1e-5 && std::abs(A.O[1] - B.O[1]) < 1e-5 &&
                  std::abs(A.O[2] - B.O[2]) < 1e-5;
      bool significant = same;
      if (!same) {
        overlap_block(bs, s1, s2, S);
        double n2 = 0;
        for (double x : S) n2 += x * x;
        significant = std::sqrt(n2) >= 1e-12;
      }
      if (significant) bs.sig[s1].push_back(s2);
    }
  }
}

// DirectTPI::computeSchwarz (aointegrals_utilities.cxx:53-162):
// Q(s1,s2) = sqrt( || diag block ||_inf ) where diag(i,j) = (ij|ij),
// infinity norm = max row sum over i of sum_j |(ij|ij)|.
void compute_schwarz(Basis& bs) {
  int ns = (int)bs.shells.size();
  bs.schwarz.assign((size_t)ns * ns, 0.0);
#pragma omp parallel
  {
    std::vector<double> buf, scr;
#pragma omp for schedule(dynamic)
    for (int s1 = 0; s1 < ns; s1++)
      for (int s2 = 0; s2 <= s1; s2++) {
        int n1 = bs.shells[s1].size(), n2 = bs.shells[s2].size();
        eri_quartet(bs, s1, s2, s1, s2, buf, scr);
        double mx = 0.0;
        for (int i = 0; i < n1; i++) {
          double row = 0.0;
          for (int j = 0; j < n2; j++) {
            size_t ij = (size_t)i * n2 + j;
            row += std::abs(buf[ij * n1 * n2 + ij]);
          }
          mx = std::max(mx, row);
        }
        double q = std::sqrt(mx);
        bs.schwarz[s1 + (size_t)s2 * ns] = q;
        bs.schwarz[s2 + (size_t)s1 * ns] = q;
      }
  }
  bs.have_schwarz = true;
}

template <typename T> inline T sconj(const T& x) { return x; }
template <> inline dcomplex sconj(const dcomplex& x) { return std::conj(x); }
inline double re(double x) { return x; }
inline double re(const dcomplex& x) { return x.real(); }

// ShellBlockNorm (direct.hpp:73-90): infinity norm of each shell block.
template <typename T>
void shell_block_norm(const Basis& bs, const T* X, int N, double* out) {
  int ns = (int)bs.shells.size();
  for (int s1 = 0; s1 < ns; s1++)
    for (int s2 = 0; s2 < ns; s2++) {
      int n1 = bs.shells[s1].size(), n2 = bs.shells[s2].size();
      double mx = 0.0;
      for (int i = 0; i < n1; i++) {
        double row = 0.0;
        for (int j = 0; j < n2; j++)
          row += std::abs(X[(bs.off[s1] + i) + (size_t)(bs.off[s2] + j) * N]);
        mx = std::max(mx, row);
      }
      out[s1 + (size_t)s2 * ns] = mx;
    }
}

enum { COULOMB = 0, EXCHANGE = 1 };

struct Stats {
  int64_t quartets_total = 0, quartets_screened = 0, quartets_computed = 0;
};

// GTODirectTPIContraction::directScaffoldNew, one basis (basisSet_ ==
// basisSet2_), screen = true.  AX is accumulated as with >1 thread
// (direct.hpp:2047-2058): AX += 1/2 (A + A^H) (HER) or AX += 1/2 A.
// mpiRank / mpiSize: the reference's MPI split, contiguous chunks of the
// significant-pair counter s12 of (nshell (nshell + 1) / 2) / mpiSize pairs,
// the last rank taking the rest (direct.hpp:1600-1604, :1655-1656); the
// ranks' AX sum to the whole contraction (MPIReduce, :2085-2107).
template <typename T>
void direct_scaffold(Basis& bs, int nMat, const int* her, const int* type,
                     const T* const* X, T* const* AX, double thresh, int nThreads,
                     bool screen, Stats* stats, int mpiRank = 0, int mpiSize = 1) {
  int ns = (int)bs.shells.size();
  int N = bs.nbasis;
  if (!bs.have_schwarz) compute_schwarz(bs);
  const double* schwarz = bs.schwarz.data();
  if (nThreads <= 0) nThreads = omp_get_max_threads();

  // shell block norms per matrix, symmetrised for non-Hermitian
  // (direct.hpp:1518-1561); elementwise max over matrices when nMat > 1.
  size_t ns2 = (size_t)ns * ns;
  std::vector<double> normsMat((size_t)nMat * ns2), norms(ns2, 0.0);
  for (int m = 0; m < nMat; m++) {
    double* nm = &normsMat[m * ns2];
    shell_block_norm(bs, X[m], N, nm);
    if (!her[m])
      for (int k = 0; k < ns; k++)
        for (int l = 0; l < k; l++) {
          double mx = std::max(nm[k + (size_t)l * ns], nm[l + (size_t)k * ns]);
          nm[k + (size_t)l * ns] = mx;
          nm[l + (size_t)k * ns] = mx;
        }
  }
  const double* shblk;
  if (nMat == 1) shblk = normsMat.data();
  else {
    for (size_t i = 0; i < ns2; i++)
      for (int m = 0; m < nMat; m++) norms[i] = std::max(norms[i], normsMat[m * ns2 + i]);
    shblk = norms.data();
  }

  std::vector<T> AXraw((size_t)nThreads * nMat * N * N, T(0.0));
  std::vector<int64_t> nTot(nThreads, 0), nSkip(nThreads, 0);
  const size_t npairMax = (size_t)ns * (ns + 1) / 2;
  const size_t mpiChunks = npairMax / (size_t)mpiSize;
  const size_t mpiS12St = (size_t)mpiRank * mpiChunks;
  const size_t mpiS12End = (mpiRank == mpiSize - 1) ? npairMax : (size_t)(mpiRank + 1) * mpiChunks;

#pragma omp parallel num_threads(nThreads)
  {
    int tid = omp_get_thread_num();
    T* AXloc = &AXraw[(size_t)tid * nMat * N * N];
    std::vector<double> buf, scr, ibuf;
    std::vector<int> conMat(nMat);
    std::vector<double> shMax123Mat(nMat);
    size_t s12 = 0;
    for (int s1 = 0; s1 < ns; s1++) {
      int n1 = bs.shells[s1].size(), bf1s = bs.off[s1];
      for (int s2 : bs.sig[s1]) {
        int n2 = bs.shells[s2].size(), bf2s = bs.off[s2];
        if (s12 < mpiS12St || s12 >= mpiS12End) {
          s12++;
          continue;
        }
        if ((s12++) % nThreads != (size_t)tid) continue;
        double s12deg = (s1 == s2) ? 1.0 : 2.0;
        double shz12 = 0, shMax12 = 0;
        if (screen) {
          shz12 = schwarz[s1 + (size_t)s2 * ns];
          shMax12 = shblk[s1 + (size_t)s2 * ns];
        }
        for (int s3 = 0; s3 <= s1; s3++) {
          int n3 = bs.shells[s3].size(), bf3s = bs.off[s3];
          double shMax123 = 0;
          if (screen) {
            shMax123 = std::max(shblk[s1 + (size_t)s3 * ns], shblk[s2 + (size_t)s3 * ns]);
            shMax123 = std::max(shMax123, shMax12);
            if (nMat != 1)
              for (int m = 0; m < nMat; m++) {
                const double* nm = &normsMat[m * ns2];
                shMax123Mat[m] = std::max(nm[s1 + (size_t)s2 * ns],
                                          std::max(nm[s1 + (size_t)s3 * ns], nm[s2 + (size_t)s3 * ns]));
              }
          }
          int s4max = (s1 == s3) ? s2 : s3;
          for (int s4 : bs.sig[s3]) {
            if (s4 > s4max) break;
            int n4 = bs.shells[s4].size(), bf4s = bs.off[s4];
            nTot[tid]++;
            int nCon = nMat;
            for (int m = 0; m < nMat; m++) conMat[m] = m;
            if (screen) {
              double shMax = shblk[s3 + (size_t)s4 * ns];
              shMax = std::max(shMax, std::max(shblk[s1 + (size_t)s4 * ns], shblk[s2 + (size_t)s4 * ns]));
              shMax = std::max(shMax, shMax123);
              if (shMax * shz12 * schwarz[s3 + (size_t)s4 * ns] < thresh) {
                nSkip[tid]++;
                continue;
              }
              if (nMat != 1) {
                nCon = 0;
                for (int m = 0; m < nMat; m++) {
                  const double* nm = &normsMat[m * ns2];
                  double sm = nm[s3 + (size_t)s4 * ns];
                  sm = std::max(sm, std::max(nm[s1 + (size_t)s4 * ns], nm[s2 + (size_t)s4 * ns]));
                  sm = std::max(sm, shMax123Mat[m]);
                  if (!(sm * shz12 * schwarz[s3 + (size_t)s4 * ns] < thresh)) conMat[nCon++] = m;
                }
              }
            }
            double s34deg = (s3 == s4) ? 1.0 : 2.0;
            double s1234deg = (s1 == s3) ? (s2 == s4 ? 1.0 : 2.0) : 2.0;
            double deg = s12deg * s34deg * s1234deg;
            eri_quartet(bs, s1, s2, s3, s4, buf, scr);
            size_t nq = (size_t)n1 * n2 * n3 * n4;
            ibuf.resize(nq);
            for (size_t i = 0; i < nq; i++) ibuf[i] = buf[i] * 0.5 * deg;
            const double* I = ibuf.data();
            for (int ic = 0; ic < nCon; ic++) {
              int m = conMat[ic];
              const T* Xm = X[m];
              T* A = AXloc + (size_t)m * N * N;
              if (her[m]) {
                if (type[m] == COULOMB) {
                  size_t ijkl = 0;
                  for (int i = 0, bf1 = bf1s; i < n1; i++, bf1++)
                    for (int j = 0, bf2 = bf2s; j < n2; j++, bf2++) {
                      size_t b1 = bf1 + (size_t)N * bf2;
                      double X1 = re(Xm[b1]);
                      double* Xp1 = reinterpret_cast<double*>(A + b1);
                      for (int k = 0, bf3 = bf3s; k < n3; k++, bf3++)
                        for (int l = 0, bf4 = bf4s; l < n4; l++, bf4++, ijkl++) {
                          *Xp1 += re(Xm[bf4 + (size_t)bf3 * N]) * I[ijkl];
                          *reinterpret_cast<double*>(A + bf4 + (size_t)bf3 * N) += X1 * I[ijkl];
                        }
                    }
                } else {
                  size_t ijkl = 0;
                  for (int i = 0, bf1 = bf1s; i < n1; i++, bf1++)
                    for (int j = 0, bf2 = bf2s; j < n2; j++, bf2++)
                      for (int k = 0, bf3 = bf3s; k < n3; k++, bf3++) {
                        size_t b1 = bf1 + (size_t)bf3 * N, b2 = bf2 + (size_t)bf3 * N;
                        T T1 = 0.5 * sconj(Xm[b1]);
                        T T2 = 0.5 * sconj(Xm[b2]);
                        for (int l = 0, bf4 = bf4s; l < n4; l++, bf4++, ijkl++) {
                          A[b1] += 0.5 * sconj(Xm[bf4 + (size_t)N * bf2]) * I[ijkl];
                          A[bf4 + (size_t)bf2 * N] += T1 * I[ijkl];
                          A[bf4 + (size_t)bf1 * N] += T2 * I[ijkl];
                          A[b2] += 0.5 * sconj(Xm[bf4 + (size_t)N * bf1]) * I[ijkl];
                        }
                      }
                }
              } else {
                if (type[m] == COULOMB) {
                  size_t ijkl = 0;
                  for (int i = 0, bf1 = bf1s; i < n1; i++, bf1++)
                    for (int j = 0, bf2 = bf2s; j < n2; j++, bf2++) {
                      size_t b1 = bf1 + (size_t)N * bf2, b2 = bf2 + (size_t)N * bf1;
                      T T1 = Xm[b1], T2 = Xm[b2];
                      for (int k = 0, bf3 = bf3s; k < n3; k++, bf3++)
                        for (int l = 0, bf4 = bf4s; l < n4; l++, bf4++, ijkl++) {
                          T x34 = 0.5 * (Xm[bf4 + (size_t)bf3 * N] + Xm[bf3 + (size_t)bf4 * N]);
                          A[b1] += x34 * I[ijkl];
                          A[bf3 + (size_t)bf4 * N] += 0.5 * (T2 + T1) * I[ijkl];
                          A[b2] += x34 * I[ijkl];
                          A[bf4 + (size_t)bf3 * N] += 0.5 * (T2 + T1) * I[ijkl];
                        }
                    }
                } else {
                  size_t ijkl = 0;
                  for (int i = 0, bf1 = bf1s; i < n1; i++, bf1++)
                    for (int j = 0, bf2 = bf2s; j < n2; j++, bf2++)
                      for (int k = 0, bf3 = bf3s; k < n3; k++, bf3++) {
                        size_t b1 = bf1 + (size_t)bf3 * N, b2 = bf2 + (size_t)bf3 * N;
                        size_t b3 = bf3 + (size_t)bf1 * N, b4 = bf3 + (size_t)bf2 * N;
                        T T1 = 0.5 * Xm[b1], T2 = 0.5 * Xm[b2];
                        T T3 = 0.5 * Xm[b3], T4 = 0.5 * Xm[b4];
                        for (int l = 0, bf4 = bf4s; l < n4; l++, bf4++, ijkl++) {
                          double v = I[ijkl];
                          A[b3] += 0.5 * Xm[bf4 + (size_t)N * bf2] * v;
                          A[bf4 + (size_t)bf2 * N] += T3 * v;
                          A[bf4 + (size_t)bf1 * N] += T4 * v;
                          A[b4] += 0.5 * Xm[bf4 + (size_t)N * bf1] * v;
                          A[b1] += 0.5 * Xm[bf2 + (size_t)N * bf4] * v;
                          A[bf2 + (size_t)bf4 * N] += T1 * v;
                          A[bf1 + (size_t)bf4 * N] += T2 * v;
                          A[b2] += 0.5 * Xm[bf1 + (size_t)N * bf4] * v;
                        }
                      }
                }
              }
            }
          }
        }
      }
    }
  }
  // Reduction + Hermitisation (direct.hpp:2036-2066), nThreads != 1 form.
  for (int m = 0; m < nMat; m++) {
    T* out = AX[m];
    for (int t = 0; t < nThreads; t++) {
      const T* A = &AXraw[((size_t)t * nMat + m) * N * N];
      if (her[m]) {
        for (int j = 0; j < N; j++)
          for (int i = 0; i < N; i++)
            out[i + (size_t)j * N] += 0.5 * A[i + (size_t)j * N] + 0.5 * sconj(A[j + (size_t)i * N]);
      } else {
        for (size_t i = 0; i < (size_t)N * N; i++) out[i] += 0.5 * A[i];
      }
    }
  }
  if (stats) {
    for (int t = 0; t < nThreads; t++) {
      stats->quartets_total += nTot[t];
      stats->quartets_screened += nSkip[t];
    }
    stats->quartets_computed = stats->quartets_total - stats->quartets_screened;
  }
}

// ------------------------------------------------ algorithmic FLOP model
// Per primitive quartet with l_ab, l_cd, L, H(n) = (n+1)(n+2)(n+3)/6,
// c(l) = (l+1)(l+2)/2 (the frozen McMurchie-Davidson count):
//  20 + 3L + 3 sum_{n=0..L} H(L-n) + 2 H(lab) H(lcd) c(lc)c(ld)
//  + 2 c(la)c(lb) H(lab) c(lc)c(ld) + 3 [c(la)c(lb)H(lab) + c(lc)c(ld)H(lcd)]
// plus per contracted quartet the Cartesian-to-spherical transform and a
// digestion of 12 n1n2n3n4 per density.
double H3(int n) { return (n + 1.0) * (n + 2.0) * (n + 3.0) / 6.0; }
double flop_prim(int la, int lb, int lc, int ld) {
  int lab = la + lb, lcd = lc + ld, L = lab + lcd;
  double c_a = ncart(la), c_b = ncart(lb), c_c = ncart(lc), c_d = ncart(ld);
  double s = 0;
  for (int n = 0; n <= L; n++) s += H3(L - n);
  return 20 + 3.0 * L + 3.0 * s + 2.0 * H3(lab) * H3(lcd) * c_c * c_d +
         2.0 * c_a * c_b * H3(lab) * c_c * c_d + 3.0 * (c_a * c_b * H3(lab) + c_c * c_d * H3(lcd));
}
double flop_sph(const Basis& bs, int s1, int s2, int s3, int s4) {
  // 2 * sum over centres of n_sph * n_cart * (remaining dims)
  const Shell* sh[4] = {&bs.shells[s1], &bs.shells[s2], &bs.shells[s3], &bs.shells[s4]};
  double dims[4];
  for (int k = 0; k < 4; k++) dims[k] = ncart(sh[k]->l);
  double f = 0;
  for (int k = 0; k < 4; k++) {
    if (!sh[k]->pure) continue;
    double rest = 1;
    for (int q = 0; q < 4; q++) if (q != k) rest *= dims[q];
    f += 2.0 * (2 * sh[k]->l + 1) * ncart(sh[k]->l) * rest;
    dims[k] = 2 * sh[k]->l + 1;
  }
  return f;
}

}  // namespace

// ===================================================================== C API
extern "C" {

void* orc_basis_new(int nshell, const int* l, const int* pure, const int* nprim,
                    const double* alpha, const double* coef, const double* origin,
                    int coef_is_raw) {
  auto* bs = new Basis();
  size_t off = 0;
  int bf = 0;
  for (int s = 0; s < nshell; s++) {
    Shell sh;
    sh.l = l[s];
    sh.pure = pure[s] != 0;
    sh.alpha.assign(alpha + off, alpha + off + nprim[s]);
    std::vector<double> c(coef + off, coef + off + nprim[s]);
    sh.coef = coef_is_raw ? normalize(sh.l, sh.alpha, c) : c;
    for (int x = 0; x < 3; x++) sh.O[x] = origin[3 * s + x];
    off += nprim[s];
    bs->off.push_back(bf);
    bf += sh.size();
    bs->maxL = std::max(bs->maxL, sh.l);
    bs->maxPrim = std::max(bs->maxPrim, (int)sh.alpha.size());
    bs->shells.push_back(std::move(sh));
  }
  bs->nbasis = bf;
  bs->sph.resize(bs->maxL + 8);
  bs->cx.resize(bs->maxL + 8);
  bs->cy.resize(bs->maxL + 8);
  bs->cz.resize(bs->maxL + 8);
  for (int L = 0; L < bs->maxL + 8; L++) {
    bs->sph[L] = solid_harmonics(L);
    cart_list(L, bs->cx[L], bs->cy[L], bs->cz[L]);
  }
  build_pairs(*bs);
  build_sig_pairs(*bs);
  return bs;
}

void orc_basis_free(void* b) { delete static_cast<Basis*>(b); }
int orc_nbasis(void* b) { return static_cast<Basis*>(b)->nbasis; }

void orc_coefs(void* b, double* out) {
  auto* bs = static_cast<Basis*>(b);
  size_t k = 0;
  for (auto& sh : bs->shells)
    for (double c : sh.coef) out[k++] = c;
}

double orc_boys(int m, double T) {
  double F[64];
  boys().eval(m, T, F);
  return F[m];
}

// Overlap and kinetic matrices (column-major N x N).
void orc_overlap_kinetic(void* b, double* S, double* Tk) {
  auto* bs = static_cast<Basis*>(b);
  int ns = (int)bs->shells.size(), N = bs->nbasis;
  for (int s1 = 0; s1 < ns; s1++)
    for (int s2 = 0; s2 < ns; s2++) {
      std::vector<double> Sb, Tb;
      cart_overlap_kinetic(bs->shells[s1], bs->shells[s2], *bs, Sb, Tb);
      const Shell* sh[2] = {&bs->shells[s1], &bs->shells[s2]};
      cart_to_sph_block(*bs, sh, 2, Sb);
      cart_to_sph_block(*bs, sh, 2, Tb);
      int n1 = bs->shells[s1].size(), n2 = bs->shells[s2].size();
      for (int i = 0; i < n1; i++)
        for (int j = 0; j < n2; j++) {
          size_t idx = (bs->off[s1] + i) + (size_t)(bs->off[s2] + j) * N;
          if (S) S[idx] = Sb[i * n2 + j];
          if (Tk) Tk[idx] = Tb[i * n2 + j];
        }
    }
}

// Nuclear-attraction matrix V (column-major N x N): V_ab = -sum_C Z_C
// (a| |r - C|^-1 |b) for point nuclei (the libint2::Operator::nuclear engine
// with charges -Z at the atoms, src/particleintegrals/aointegrals/
// aointegrals_onee_drivers.cxx:139-145), or the potential of a Gaussian
// nuclear charge Z (zeta/pi)^{3/2} exp(-zeta |r - C|^2) (finiteWidthNuc;
// Molecule::computeCDist, src/molecule/molecule.cxx:197-226).  McMurchie-
// Davidson: for a primitive pair (p, P) and nucleus C,
//   (2 pi / p) f sum_tuv E^x_t E^y_u E^z_v R_tuv(a', P - C),
// point: a' = p, f = 1; Gaussian: a' = p zeta / (p + zeta),
// f = sqrt(zeta / (p + zeta)).  nuc[5 i ..] = {Z, x, y, z, zeta (0: point)}.
void orc_nuclear(void* b, int natom, const double* nuc, double* V) {
  auto* bs = static_cast<Basis*>(b);
  int ns = (int)bs->shells.size(), N = bs->nbasis;
  for (int s1 = 0; s1 < ns; s1++)
    for (int s2 = 0; s2 < ns; s2++) {
      const Shell &A = bs->shells[s1], &B = bs->shells[s2];
      const int la = A.l, lb = B.l, L = la + lb, L1 = L + 1;
      const int na = ncart(la), nb = ncart(lb);
      std::vector<double> Vb((size_t)na * nb, 0.0);
      double AB2 = 0;
      for (int x = 0; x < 3; x++) AB2 += (A.O[x] - B.O[x]) * (A.O[x] - B.O[x]);
      const auto &ax = bs->cx[la], &ay = bs->cy[la], &az = bs->cz[la];
      const auto &bx = bs->cx[lb], &by = bs->cy[lb], &bz = bs->cz[lb];
      std::vector<double> R((size_t)(L + 1) * L1 * L1 * L1);
      auto Ridx = [&](int n, int t, int u, int v) -> size_t {
        return (((size_t)n * L1 + t) * L1 + u) * L1 + v;
      };
      for (size_t i = 0; i < A.alpha.size(); i++)
        for (size_t j = 0; j < B.alpha.size(); j++) {
          const double a = A.alpha[i], bb = B.alpha[j], p = a + bb, mu = a * bb / p;
          double P[3];
          for (int x = 0; x < 3; x++) P[x] = (a * A.O[x] + bb * B.O[x]) / p;
          const double K = A.coef[i] * B.coef[j] * std::exp(-mu * AB2);
          std::vector<double> E[3];
          for (int x = 0; x < 3; x++) hermite_E(la, lb, p, P[x] - A.O[x], P[x] - B.O[x], E[x]);
          auto e = [&](int x, int ii, int jj, int t) {
            return E[x][((size_t)ii * (lb + 1) + jj) * L1 + t];
          };
          for (int c = 0; c < natom; c++) {
            const double Z = nuc[5 * c], zeta = nuc[5 * c + 4];
            const double PC[3] = {P[0] - nuc[5 * c + 1], P[1] - nuc[5 * c + 2],
                                  P[2] - nuc[5 * c + 3]};
            const double al = zeta > 0.0 ? p * zeta / (p + zeta) : p;
            const double f = zeta > 0.0 ? std::sqrt(zeta / (p + zeta)) : 1.0;
            const double T = al * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
            double F[64];
            boys().eval(L, T, F);
            double m2a = -2.0 * al, fn = 1.0;
            for (int n = 0; n <= L; n++) { R[Ridx(n, 0, 0, 0)] = fn * F[n]; fn *= m2a; }
            for (int n = L - 1; n >= 0; n--) {
              const int top = L - n;
              for (int t = 0; t <= top; t++)
                for (int u = 0; u <= top - t; u++)
                  for (int v = 0; v <= top - t - u; v++) {
                    if (t + u + v == 0) continue;
                    double val;
                    if (t > 0) {
                      val = PC[0] * R[Ridx(n + 1, t - 1, u, v)];
                      if (t > 1) val += (t - 1) * R[Ridx(n + 1, t - 2, u, v)];
                    } else if (u > 0) {
                      val = PC[1] * R[Ridx(n + 1, t, u - 1, v)];
                      if (u > 1) val += (u - 1) * R[Ridx(n + 1, t, u - 2, v)];
                    } else {
                      val = PC[2] * R[Ridx(n + 1, t, u, v - 1)];
                      if (v > 1) val += (v - 1) * R[Ridx(n + 1, t, u, v - 2)];
                    }
                    R[Ridx(n, t, u, v)] = val;
                  }
            }
            const double pref = -Z * K * 2.0 * M_PI / p * f;
            for (int u = 0; u < na; u++)
              for (int v = 0; v < nb; v++) {
                double sum = 0.0;
                for (int t = 0; t <= ax[u] + bx[v]; t++)
                  for (int w = 0; w <= ay[u] + by[v]; w++)
                    for (int z = 0; z <= az[u] + bz[v]; z++)
                      sum += e(0, ax[u], bx[v], t) * e(1, ay[u], by[v], w) *
                             e(2, az[u], bz[v], z) * R[Ridx(0, t, w, z)];
                Vb[u * nb + v] += pref * sum;
              }
          }
        }
      const Shell* sh[2] = {&A, &B};
      cart_to_sph_block(*bs, sh, 2, Vb);
      const int n1 = A.size(), n2 = B.size();
      for (int i = 0; i < n1; i++)
        for (int j = 0; j < n2; j++)
          V[(bs->off[s1] + i) + (size_t)(bs->off[s2] + j) * N] = Vb[i * n2 + j];
    }
}

// Derivative nuclear-attraction matrices of the four-component core
// Hamiltonian: D_{mu nu}(a, b) = <d_mu a| V |d_nu b> (d = gradient with
// respect to the electron coordinate, V = -sum_C Z_C / |r - C| or its
// Gaussian-nucleus form as in orc_nuclear), and
//   W[0] = pV.p   = sum_mu D_{mu mu},
//   W[1..3] = (pV x p)_k = D_{ij} - D_{ji}, (i, j, k) cyclic,
// each N x N column-major (the OnePRelInts scalar / SOX / SOY / SOZ
// components, include/particleintegrals/onepints/relativisticints.hpp;
// src/particleintegrals/spatialtospinor.cxx:205-230).  d_x x^i e^{-a x^2} =
// i x^{i-1} e^{..} - 2 a x^{i+1} e^{..}, so every D is a sum of plain
// nuclear-attraction integrals with l raised or lowered by one on each side,
// from Hermite tables of (la + 1, lb + 1).
void orc_nuclear_pvp(void* b, int natom, const double* nuc, double* W) {
  auto* bs = static_cast<Basis*>(b);
  int ns = (int)bs->shells.size(), N = bs->nbasis;
  for (int s1 = 0; s1 < ns; s1++)
    for (int s2 = 0; s2 < ns; s2++) {
      const Shell &A = bs->shells[s1], &B = bs->shells[s2];
      const int la = A.l, lb = B.l, La = la + 1, Lb = lb + 1, L = La + Lb, L1 = L + 1;
      const int na = ncart(la), nb = ncart(lb);
      std::vector<double> Dm((size_t)9 * na * nb, 0.0);
      double AB2 = 0;
      for (int x = 0; x < 3; x++) AB2 += (A.O[x] - B.O[x]) * (A.O[x] - B.O[x]);
      const auto &ax = bs->cx[la], &ay = bs->cy[la], &az = bs->cz[la];
      const auto &bx = bs->cx[lb], &by = bs->cy[lb], &bz = bs->cz[lb];
      std::vector<double> R((size_t)(L + 1) * L1 * L1 * L1);
      auto Ridx = [&](int n, int t, int u, int v) -> size_t {
        return (((size_t)n * L1 + t) * L1 + u) * L1 + v;
      };
      for (size_t i = 0; i < A.alpha.size(); i++)
        for (size_t j = 0; j < B.alpha.size(); j++) {
          const double a = A.alpha[i], bb = B.alpha[j], p = a + bb, mu = a * bb / p;
          double P[3];
          for (int x = 0; x < 3; x++) P[x] = (a * A.O[x] + bb * B.O[x]) / p;
          const double K = A.coef[i] * B.coef[j] * std::exp(-mu * AB2);
          std::vector<double> E[3];
          for (int x = 0; x < 3; x++) hermite_E(La, Lb, p, P[x] - A.O[x], P[x] - B.O[x], E[x]);
          auto e = [&](int x, int ii, int jj, int t) {
            if (ii < 0 || jj < 0 || t > ii + jj) return 0.0;
            return E[x][((size_t)ii * (Lb + 1) + jj) * L1 + t];
          };
          for (int c = 0; c < natom; c++) {
            const double Z = nuc[5 * c], zeta = nuc[5 * c + 4];
            const double PC[3] = {P[0] - nuc[5 * c + 1], P[1] - nuc[5 * c + 2],
                                  P[2] - nuc[5 * c + 3]};
            const double al = zeta > 0.0 ? p * zeta / (p + zeta) : p;
            const double f = zeta > 0.0 ? std::sqrt(zeta / (p + zeta)) : 1.0;
            const double T = al * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
            double F[64];
            boys().eval(L, T, F);
            double m2a = -2.0 * al, fn = 1.0;
            for (int n = 0; n <= L; n++) { R[Ridx(n, 0, 0, 0)] = fn * F[n]; fn *= m2a; }
            for (int n = L - 1; n >= 0; n--) {
              const int top = L - n;
              for (int t = 0; t <= top; t++)
                for (int u = 0; u <= top - t; u++)
                  for (int v = 0; v <= top - t - u; v++) {
                    if (t + u + v == 0) continue;
                    double val;
                    if (t > 0) {
                      val = PC[0] * R[Ridx(n + 1, t - 1, u, v)];
                      if (t > 1) val += (t - 1) * R[Ridx(n + 1, t - 2, u, v)];
                    } else if (u > 0) {
                      val = PC[1] * R[Ridx(n + 1, t, u - 1, v)];
                      if (u > 1) val += (u - 1) * R[Ridx(n + 1, t, u - 2, v)];
                    } else {
                      val = PC[2] * R[Ridx(n + 1, t, u, v - 1)];
                      if (v > 1) val += (v - 1) * R[Ridx(n + 1, t, u, v - 2)];
                    }
                    R[Ridx(n, t, u, v)] = val;
                  }
            }
            const double pref = -Z * K * 2.0 * M_PI / p * f;
            // plain integral of Cartesian exponents ia[3], ib[3]
            auto vint = [&](const int* ia, const int* ib) {
              for (int x = 0; x < 3; x++)
                if (ia[x] < 0 || ib[x] < 0) return 0.0;
              double sum = 0.0;
              for (int t = 0; t <= ia[0] + ib[0]; t++)
                for (int w = 0; w <= ia[1] + ib[1]; w++)
                  for (int z = 0; z <= ia[2] + ib[2]; z++)
                    sum += e(0, ia[0], ib[0], t) * e(1, ia[1], ib[1], w) *
                           e(2, ia[2], ib[2], z) * R[Ridx(0, t, w, z)];
              return sum;
            };
            for (int u = 0; u < na; u++)
              for (int v = 0; v < nb; v++) {
                const int a0[3] = {ax[u], ay[u], az[u]}, b0[3] = {bx[v], by[v], bz[v]};
                for (int m = 0; m < 3; m++)
                  for (int nn = 0; nn < 3; nn++) {
                    double d = 0.0;
                    for (int sa = -1; sa <= 1; sa += 2)
                      for (int sb = -1; sb <= 1; sb += 2) {
                        const double fa = sa < 0 ? a0[m] : -2.0 * a;
                        const double fb = sb < 0 ? b0[nn] : -2.0 * bb;
                        if (fa == 0.0 || fb == 0.0) continue;
                        int ia[3] = {a0[0], a0[1], a0[2]}, ib[3] = {b0[0], b0[1], b0[2]};
                        ia[m] += sa;
                        ib[nn] += sb;
                        d += fa * fb * vint(ia, ib);
                      }
                    Dm[((size_t)(m * 3 + nn) * na + u) * nb + v] += pref * d;
                  }
              }
          }
        }
      std::vector<double> Wb[4];
      for (int k = 0; k < 4; k++) Wb[k].assign((size_t)na * nb, 0.0);
      auto D = [&](int m, int nn, int u, int v) { return Dm[((size_t)(m * 3 + nn) * na + u) * nb + v]; };
      for (int u = 0; u < na; u++)
        for (int v = 0; v < nb; v++) {
          const size_t q = (size_t)u * nb + v;
          Wb[0][q] = D(0, 0, u, v) + D(1, 1, u, v) + D(2, 2, u, v);
          Wb[1][q] = D(1, 2, u, v) - D(2, 1, u, v);
          Wb[2][q] = D(2, 0, u, v) - D(0, 2, u, v);
          Wb[3][q] = D(0, 1, u, v) - D(1, 0, u, v);
        }
      const Shell* sh[2] = {&A, &B};
      const int n1 = A.size(), n2 = B.size();
      for (int k = 0; k < 4; k++) {
        cart_to_sph_block(*bs, sh, 2, Wb[k]);
        for (int i = 0; i < n1; i++)
          for (int j = 0; j < n2; j++)
            W[(size_t)k * N * N + (bs->off[s1] + i) + (size_t)(bs->off[s2] + j) * N] =
                Wb[k][i * n2 + j];
      }
    }
}

// Contracted shell quartet in AO order (row-major i,j,k,l).
int orc_eri_quartet(void* b, int s1, int s2, int s3, int s4, double* out) {
  auto* bs = static_cast<Basis*>(b);
  std::vector<double> buf, scr;
  eri_quartet(*bs, s1, s2, s3, s4, buf, scr);
  std::copy(buf.begin(), buf.end(), out);
  return (int)buf.size();
}

void orc_schwarz(void* b, double* Q) {
  auto* bs = static_cast<Basis*>(b);
  if (!bs->have_schwarz) compute_schwarz(*bs);
  std::copy(bs->schwarz.begin(), bs->schwarz.end(), Q);
}

// Number of significant pairs and the (s1, s2) list in loop order.
int orc_sig_pairs(void* b, int* s1out, int* s2out) {
  auto* bs = static_cast<Basis*>(b);
  int k = 0;
  for (size_t s1 = 0; s1 < bs->sig.size(); s1++)
    for (int s2 : bs->sig[s1]) {
      if (s1out) { s1out[k] = (int)s1; s2out[k] = s2; }
      k++;
    }
  return k;
}

// directScaffoldNew restated.  X/AX: arrays of nMat pointers to column-major
// N x N buffers (double or interleaved complex).  AX is accumulated.
int orc_contract_part(void* b, int nMat, int is_complex, const int* her, const int* type,
                      const void* const* X, void* const* AX, double thresh, int nthreads,
                      int screen, long long* stats_out, int mpi_rank, int mpi_size) {
  auto* bs = static_cast<Basis*>(b);
  Stats st;
  if (mpi_size < 1 || mpi_rank < 0 || mpi_rank >= mpi_size) return 1;
  if (is_complex)
    direct_scaffold<dcomplex>(*bs, nMat, her, type, reinterpret_cast<const dcomplex* const*>(X),
                              reinterpret_cast<dcomplex* const*>(AX), thresh, nthreads,
                              screen != 0, &st, mpi_rank, mpi_size);
  else
    direct_scaffold<double>(*bs, nMat, her, type, reinterpret_cast<const double* const*>(X),
                            reinterpret_cast<double* const*>(AX), thresh, nthreads, screen != 0,
                            &st, mpi_rank, mpi_size);
  if (stats_out) {
    stats_out[0] = st.quartets_total;
    stats_out[1] = st.quartets_screened;
    stats_out[2] = st.quartets_computed;
  }
  return 0;
}

int orc_contract(void* b, int nMat, int is_complex, const int* her, const int* type,
                 const void* const* X, void* const* AX, double thresh, int nthreads,
                 int screen, long long* stats_out) {
  return orc_contract_part(b, nMat, is_complex, her, type, X, AX, thresh, nthreads, screen,
                           stats_out, 0, 1);
}

// Algorithmic FLOP count of one build under the frozen count model, over the
// quartets that survive the reference screen for the given densities.
// Per quartet the FLOPs go to fp32 when bound*shMax < fp32_cut (else fp64);
// fp32_cut <= 0 puts everything in fp64.  out[0]=F64, out[1]=F32,
// out[2]=#quartets kept, out[3]=#fp32 quartets.
void orc_flops(void* b, int nMat, const double* const* X, double thresh, double fp32_cut,
               double* out) {
  auto* bs = static_cast<Basis*>(b);
  int ns = (int)bs->shells.size(), N = bs->nbasis;
  if (!bs->have_schwarz) compute_schwarz(*bs);
  size_t ns2 = (size_t)ns * ns;
  std::vector<double> norms(ns2, 0.0), tmp(ns2);
  for (int m = 0; m < nMat; m++) {
    shell_block_norm(*bs, X[m], N, tmp.data());
    for (size_t i = 0; i < ns2; i++) norms[i] = std::max(norms[i], tmp[i]);
  }
  const double* Q = bs->schwarz.data();
  double f64 = 0, f32 = 0, nk = 0, n32 = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : f64, f32, nk, n32)
  for (int s1 = 0; s1 < ns; s1++)
    for (int s2 : bs->sig[s1])
      for (int s3 = 0; s3 <= s1; s3++) {
        int s4max = (s1 == s3) ? s2 : s3;
        for (int s4 : bs->sig[s3]) {
          if (s4 > s4max) break;
          double shMax = std::max({norms[s3 + (size_t)s4 * ns], norms[s1 + (size_t)s4 * ns],
                                   norms[s2 + (size_t)s4 * ns], norms[s1 + (size_t)s3 * ns],
                                   norms[s2 + (size_t)s3 * ns], norms[s1 + (size_t)s2 * ns]});
          double bound = shMax * Q[s1 + (size_t)s2 * ns] * Q[s3 + (size_t)s4 * ns];
          if (bound < thresh) continue;
          const Shell &A = bs->shells[s1], &B = bs->shells[s2], &C = bs->shells[s3],
                      &D = bs->shells[s4];
          double np = (double)A.alpha.size() * B.alpha.size() * C.alpha.size() * D.alpha.size();
          double f = np * flop_prim(A.l, B.l, C.l, D.l) + flop_sph(*bs, s1, s2, s3, s4) +
                     12.0 * nMat * A.size() * B.size() * C.size() * D.size();
          nk += 1;
          if (fp32_cut > 0 && bound < fp32_cut) { f32 += f; n32 += 1; }
          else f64 += f;
        }
      }
  out[0] = f64; out[1] = f32; out[2] = nk; out[3] = n32;
}

}  // extern "C"

// ======================================================================
// Four-component Dirac-Coulomb (test infrastructure, same rules as above).
//
// Restates GTODirectRelERIContraction::directScaffoldLibcint
// (include/particleintegrals/contract/direct4C_libcint.hpp):
//   * Schwarz tables (:341-481): Q^LL = sqrt(max |(ab|ab)|) over the whole
//     block, Q^SS = C2 sqrt(max |(dA dB ab|dA dB ab)|) over the 81 components;
//   * BARE_COULOMB (LL|LL) (:514-790), LLSS (:810-1441), SSSS (:1841-2832):
//     loop order, screens, degeneracy factors, update sites and conditions;
//   * and FourCompFock::formGDDirect (include/fockbuilder/fourcompfock/
//     impl.hpp:3752-4636): LL/SS/LS blocks, the 2C2 / -C2 / 2C4 / -C4
//     weights, LS -> SL, G = twoeH - xHFX K.
// The component formulas of the reference are products of spin operators:
// a differentiated pair (m, n) acts as P_mn = dm.dn + i sigma.(dm x dn) on
// the electron's spin; exchange updates are -P D P' (SSSS) or -D P (LS),
// Coulomb updates P Re Tr[P' D]/2.  They are evaluated here through that
// algebra (own formulation; the reference writes each component out).
// Derivative ERIs (libcint int2e_ipvip1 / int2e_ipvip1ipvip2 in the
// reference, v5.1.2, not present) are computed by McMurchie-Davidson over
// the raised/lowered Cartesian functions: d/dx x^a e^{-a x^2} =
// a x^{a-1} e - 2 alpha x^{a+1} e.
// ======================================================================
namespace {

// Primitive-contracted Cartesian ERIs over all exponent tuples with total
// <= lmax of each centre (dense table), then derivative blocks from it.
struct RaisedTable {
  int lm[4];
  std::vector<std::array<int, 3>> tup[4];  // tuples per centre
  std::vector<int> idx[4];                 // (ax,ay,az) -> position
  std::vector<double> v;                   // [a][b][c][d]
  int n[4];
  int pos(int c, int x, int y, int z) const {
    int L = lm[c] + 1;
    if (x < 0 || y < 0 || z < 0 || x + y + z > lm[c]) return -1;
    return idx[c][(x * L + y) * L + z];
  }
};

void build_tuples(RaisedTable& T, int c, int lmax) {
  T.lm[c] = lmax;
  int L = lmax + 1;
  T.idx[c].assign(L * L * L, -1);
  T.tup[c].clear();
  for (int l = 0; l <= lmax; l++)
    for (int i = 0; i <= l; i++)
      for (int j = 0; j <= i; j++) {
        std::array<int, 3> t = {l - i, i - j, j};
        T.idx[c][(t[0] * L + t[1]) * L + t[2]] = (int)T.tup[c].size();
        T.tup[c].push_back(t);
      }
  T.n[c] = (int)T.tup[c].size();
}

// Uncontracted primitive table for exponents (a,b,c,d) on centres (A..D).
// Kernel: 1 / r12 (op == nullptr), or d_i d_j r12 (op = {i, j}, each 0..2 or
// -1 for none; derivatives in r = r1 - r2).  For r12 the Hermite integrals
// are the derivatives in R = P - Q of the s-type integral, which is the
// Coulomb prefactor / (2 alpha) times f(T) = e^-T + (1 + 2T) F_0(T) (the
// mean of |r| under the Gaussian of width 1 / (2 alpha) centred at R, with
// T = alpha R^2); its T-derivatives are f' = F_0 - F_1 and
// f^(n) = (-1)^(n-1) (F_(n-1) - F_n), so the McMurchie-Davidson recursion
// runs unchanged on Ft_0 = f, Ft_n = F_n - F_(n-1), and the operator
// derivatives d_i d_j shift the Hermite index by e_i + e_j.
void prim_table(double a, const double* A, double b, const double* B, double c, const double* C,
                double d, const double* D, RaisedTable& T, const int* op = nullptr) {
  int l1 = T.lm[0], l2 = T.lm[1], l3 = T.lm[2], l4 = T.lm[3];
  int lab = l1 + l2, lcd = l3 + l4;
  int sh[3] = {0, 0, 0};
  if (op)
    for (int k = 0; k < 2; k++)
      if (op[k] >= 0) sh[op[k]]++;
  const int L = lab + lcd + sh[0] + sh[1] + sh[2];
  double p = a + b, q = c + d, alpha = p * q / (p + q);
  double P[3], Q[3], PQ[3];
  for (int x = 0; x < 3; x++) {
    P[x] = (a * A[x] + b * B[x]) / p;
    Q[x] = (c * C[x] + d * D[x]) / q;
    PQ[x] = P[x] - Q[x];
  }
  double AB2 = 0, CD2 = 0;
  for (int x = 0; x < 3; x++) {
    AB2 += (A[x] - B[x]) * (A[x] - B[x]);
    CD2 += (C[x] - D[x]) * (C[x] - D[x]);
  }
  double Kab = std::exp(-a * b / p * AB2), Kcd = std::exp(-c * d / q * CD2);
  double pref = 2.0 * std::pow(M_PI, 2.5) / (p * q * std::sqrt(p + q)) * Kab * Kcd;
  if (op) pref /= 2.0 * alpha;
  std::vector<double> Eb[3], Ek[3];
  for (int x = 0; x < 3; x++) {
    hermite_E(l1, l2, p, P[x] - A[x], P[x] - B[x], Eb[x]);
    hermite_E(l3, l4, q, Q[x] - C[x], Q[x] - D[x], Ek[x]);
  }
  int L1 = L + 1;
  std::vector<double> R((size_t)(L + 1) * L1 * L1 * L1, 0.0);
  auto Ridx = [&](int nn, int t, int u, int v) -> size_t {
    return (((size_t)nn * L1 + t) * L1 + u) * L1 + v;
  };
  double F[96];
  const double Targ = alpha * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
  boys().eval(L, Targ, F);
  if (op) {
    for (int nn = L; nn >= 1; nn--) F[nn] -= F[nn - 1];
    F[0] = std::exp(-Targ) + (1.0 + 2.0 * Targ) * F[0];
  }
  double f = 1.0;
  for (int nn = 0; nn <= L; nn++) { R[Ridx(nn, 0, 0, 0)] = f * F[nn]; f *= -2.0 * alpha; }
  for (int nn = L - 1; nn >= 0; nn--)
    for (int t = 0; t <= L - nn; t++)
      for (int u = 0; u <= L - nn - t; u++)
        for (int v = 0; v <= L - nn - t - u; v++) {
          if (t + u + v == 0) continue;
          double val;
          if (t > 0) {
            val = PQ[0] * R[Ridx(nn + 1, t - 1, u, v)];
            if (t > 1) val += (t - 1) * R[Ridx(nn + 1, t - 2, u, v)];
          } else if (u > 0) {
            val = PQ[1] * R[Ridx(nn + 1, t, u - 1, v)];
            if (u > 1) val += (u - 1) * R[Ridx(nn + 1, t, u - 2, v)];
          } else {
            val = PQ[2] * R[Ridx(nn + 1, t, u, v - 1)];
            if (v > 1) val += (v - 1) * R[Ridx(nn + 1, t, u, v - 2)];
          }
          R[Ridx(nn, t, u, v)] = val;
        }
  const int Lb1 = lab + 1, Lk1 = lcd + 1;
  // G[cd][tuv]
  int ncd = T.n[2] * T.n[3];
  std::vector<double> G((size_t)ncd * Lb1 * Lb1 * Lb1, 0.0);
  for (int ci = 0; ci < T.n[2]; ci++)
    for (int di = 0; di < T.n[3]; di++) {
      const auto &tc = T.tup[2][ci], &td = T.tup[3][di];
      double* g = &G[((size_t)ci * T.n[3] + di) * Lb1 * Lb1 * Lb1];
      const double* ex = &Ek[0][((size_t)tc[0] * (l4 + 1) + td[0]) * Lk1];
      const double* ey = &Ek[1][((size_t)tc[1] * (l4 + 1) + td[1]) * Lk1];
      const double* ez = &Ek[2][((size_t)tc[2] * (l4 + 1) + td[2]) * Lk1];
      for (int t = 0; t <= lab; t++)
        for (int u = 0; u <= lab - t; u++)
          for (int v = 0; v <= lab - t - u; v++) {
            double s = 0.0;
            for (int ta = 0; ta <= tc[0] + td[0]; ta++)
              for (int nu = 0; nu <= tc[1] + td[1]; nu++)
                for (int ph = 0; ph <= tc[2] + td[2]; ph++) {
                  double e = ex[ta] * ey[nu] * ez[ph];
                  if ((ta + nu + ph) & 1) e = -e;
                  s += e * R[Ridx(0, t + ta + sh[0], u + nu + sh[1], v + ph + sh[2])];
                }
            g[(t * Lb1 + u) * Lb1 + v] = pref * s;
          }
    }
  T.v.assign((size_t)T.n[0] * T.n[1] * ncd, 0.0);
  for (int ai = 0; ai < T.n[0]; ai++)
    for (int bi = 0; bi < T.n[1]; bi++) {
      const auto &ta = T.tup[0][ai], &tb = T.tup[1][bi];
      const double* ex = &Eb[0][((size_t)ta[0] * (l2 + 1) + tb[0]) * Lb1];
      const double* ey = &Eb[1][((size_t)ta[1] * (l2 + 1) + tb[1]) * Lb1];
      const double* ez = &Eb[2][((size_t)ta[2] * (l2 + 1) + tb[2]) * Lb1];
      for (int cd = 0; cd < ncd; cd++) {
        const double* g = &G[(size_t)cd * Lb1 * Lb1 * Lb1];
        double s = 0.0;
        for (int t = 0; t <= ta[0] + tb[0]; t++)
          for (int u = 0; u <= ta[1] + tb[1]; u++)
            for (int v = 0; v <= ta[2] + tb[2]; v++)
              s += ex[t] * ey[u] * ez[v] * g[(t * Lb1 + u) * Lb1 + v];
        T.v[((size_t)ai * T.n[1] + bi) * ncd + cd] = s;
      }
    }
}

// Derivative ERIs of a contracted quartet: comp-major blocks
// out[comp][i][j][k][l] over the AO functions of s1..s4 (spherical where
// pure), with derivatives (d/dr of the orbital) on the centres in dmask
// (bit 0..3 = s1..s4); comp = sum over differentiated centres, in order,
// of 3-digit indices (x, y, z), the last centre varying fastest.
void eri_deriv_quartet(const Basis& bs, int s1, int s2, int s3, int s4, int dmask,
                       std::vector<double>& out, const int* op = nullptr) {
  const int sh[4] = {s1, s2, s3, s4};
  const Shell* S[4] = {&bs.shells[s1], &bs.shells[s2], &bs.shells[s3], &bs.shells[s4]};
  int nd = 0;
  for (int c = 0; c < 4; c++) nd += (dmask >> c) & 1;
  int ncomp = 1;
  for (int k = 0; k < nd; k++) ncomp *= 3;
  int nc[4];
  for (int c = 0; c < 4; c++) nc[c] = ncart(S[c]->l);
  const size_t ncart4 = (size_t)nc[0] * nc[1] * nc[2] * nc[3];
  std::vector<double> cart((size_t)ncomp * ncart4, 0.0);
  RaisedTable T;
  for (int c = 0; c < 4; c++) build_tuples(T, c, S[c]->l + ((dmask >> c) & 1));
  for (size_t i = 0; i < S[0]->alpha.size(); i++)
    for (size_t j = 0; j < S[1]->alpha.size(); j++)
      for (size_t k = 0; k < S[2]->alpha.size(); k++)
        for (size_t l = 0; l < S[3]->alpha.size(); l++) {
          const double ex[4] = {S[0]->alpha[i], S[1]->alpha[j], S[2]->alpha[k], S[3]->alpha[l]};
          const double cf = S[0]->coef[i] * S[1]->coef[j] * S[2]->coef[k] * S[3]->coef[l];
          prim_table(ex[0], S[0]->O, ex[1], S[1]->O, ex[2], S[2]->O, ex[3], S[3]->O, T, op);
          const int nT2 = T.n[2] * T.n[3], nT1 = T.n[1];
          for (int a = 0; a < nc[0]; a++)
            for (int b = 0; b < nc[1]; b++)
              for (int c = 0; c < nc[2]; c++)
                for (int d = 0; d < nc[3]; d++) {
                  int base[4][3];
                  const int comps[4] = {a, b, c, d};
                  for (int q = 0; q < 4; q++) {
                    base[q][0] = bs.cx[S[q]->l][comps[q]];
                    base[q][1] = bs.cy[S[q]->l][comps[q]];
                    base[q][2] = bs.cz[S[q]->l][comps[q]];
                  }
                  const size_t cidx = (((size_t)a * nc[1] + b) * nc[2] + c) * nc[3] + d;
                  for (int comp = 0; comp < ncomp; comp++) {
                    // direction of each differentiated centre
                    int dir[4] = {-1, -1, -1, -1};
                    int rem = comp;
                    for (int q = 3; q >= 0; q--)
                      if ((dmask >> q) & 1) { dir[q] = rem % 3; rem /= 3; }
                    // sum over lowered (-) / raised (+) choices
                    double val = 0.0;
                    for (int sel = 0; sel < (1 << 4); sel++) {
                      bool ok = true;
                      double w = 1.0;
                      int tp[4][3];
                      for (int q = 0; q < 4 && ok; q++) {
                        for (int x = 0; x < 3; x++) tp[q][x] = base[q][x];
                        if (dir[q] < 0) {
                          if ((sel >> q) & 1) ok = false;
                          continue;
                        }
                        if ((sel >> q) & 1) {  // raised: -2 alpha
                          tp[q][dir[q]] += 1;
                          w *= -2.0 * ex[q];
                        } else {  // lowered: a_i
                          int ai = base[q][dir[q]];
                          if (ai == 0) { ok = false; continue; }
                          tp[q][dir[q]] -= 1;
                          w *= ai;
                        }
                      }
                      if (!ok) continue;
                      int p0 = T.pos(0, tp[0][0], tp[0][1], tp[0][2]);
                      int p1 = T.pos(1, tp[1][0], tp[1][1], tp[1][2]);
                      int p2 = T.pos(2, tp[2][0], tp[2][1], tp[2][2]);
                      int p3 = T.pos(3, tp[3][0], tp[3][1], tp[3][2]);
                      val += w * T.v[((size_t)p0 * nT1 + p1) * nT2 + (size_t)p2 * T.n[3] + p3];
                    }
                    cart[(size_t)comp * ncart4 + cidx] += cf * val;
                  }
                }
        }
  // spherical transform of every component block
  size_t nsph4 = 1;
  for (int c = 0; c < 4; c++) nsph4 *= S[c]->size();
  out.assign((size_t)ncomp * nsph4, 0.0);
  std::vector<double> blk;
  for (int comp = 0; comp < ncomp; comp++) {
    blk.assign(cart.begin() + comp * ncart4, cart.begin() + (comp + 1) * ncart4);
    cart_to_sph_block(bs, S, 4, blk);
    std::copy(blk.begin(), blk.end(), out.begin() + comp * nsph4);
  }
  (void)sh;
}

// DirectGradContraction::directScaffoldGrad (direct.hpp:2198-2571): for
// Hermitian real X, the contractions of the first derivatives of the ERIs
// with respect to the nuclear coordinates -- over the 8-fold quartet loop of
// significant pairs without screening (:2343-2398), the 12 derivatives of
// each quartet (3 per centre; d/dA = -d/dr of the orbital) scaled by
// 0.5 * degeneracy, each added into the matrices of gradient component
// atom(shell) * 3 + xyz with the COULOMB / EXCHANGE update sites
// (:2470-2520) -- then AX += 1/2 (A + A^T) per component and matrix
// (:2550-2560).  AX: [component][matrix], 3 * nAtom * nMat N x N arrays.
void grad_scaffold(const Basis& bs, const int* shellAtom, int nAtom, int nMat, const int* type,
                   const double* const* X, double* const* AX, int nThreads) {
  const int ns = (int)bs.shells.size(), N = bs.nbasis;
  const size_t NN = (size_t)N * N;
  const int nGrad = 3 * nAtom;
  if (nThreads <= 0) nThreads = omp_get_max_threads();
  std::vector<double> loc((size_t)nThreads * nGrad * nMat * NN, 0.0);
#pragma omp parallel num_threads(nThreads)
  {
    const int tid = omp_get_thread_num();
    double* A = &loc[(size_t)tid * nGrad * nMat * NN];
    auto at = [&](int g, int m, int r, int c) -> double& {
      return A[((size_t)g * nMat + m) * NN + r + (size_t)c * N];
    };
    std::vector<double> buf[4];
    size_t s12 = 0;
    for (int s1 = 0; s1 < ns; s1++)
      for (int s2 : bs.sig[s1]) {
        if ((s12++) % nThreads != (size_t)tid) continue;
        const double s12deg = (s1 == s2) ? 1.0 : 2.0;
        for (int s3 = 0; s3 <= s1; s3++) {
          const int s4max = (s1 == s3) ? s2 : s3;
          for (int s4 : bs.sig[s3]) {
            if (s4 > s4max) break;
            const double s34deg = (s3 == s4) ? 1.0 : 2.0;
            const double s1234deg = (s1 == s3) ? (s2 == s4 ? 1.0 : 2.0) : 2.0;
            const double f = -0.5 * s12deg * s34deg * s1234deg;  // d/dA = -d/dr
            const int sh[4] = {s1, s2, s3, s4};
            for (int c = 0; c < 4; c++) eri_deriv_quartet(bs, s1, s2, s3, s4, 1 << c, buf[c]);
            const int n1 = bs.shells[s1].size(), n2 = bs.shells[s2].size();
            const int n3 = bs.shells[s3].size(), n4 = bs.shells[s4].size();
            const size_t nq = (size_t)n1 * n2 * n3 * n4;
            for (int c = 0; c < 4; c++)
              for (int xyz = 0; xyz < 3; xyz++) {
                const int g = shellAtom[sh[c]] * 3 + xyz;
                const double* I = buf[c].data() + (size_t)xyz * nq;
                for (int i = 0; i < n1; i++)
                  for (int j = 0; j < n2; j++)
                    for (int k = 0; k < n3; k++)
                      for (int l = 0; l < n4; l++) {
                        const double v = f * I[(((size_t)i * n2 + j) * n3 + k) * n4 + l];
                        const int b1 = bs.off[s1] + i, b2 = bs.off[s2] + j;
                        const int b3 = bs.off[s3] + k, b4 = bs.off[s4] + l;
                        for (int m = 0; m < nMat; m++) {
                          const double* Xm = X[m];
                          auto x = [&](int r, int cc) { return Xm[r + (size_t)cc * N]; };
                          if (type[m] == 0) {  // COULOMB
                            at(g, m, b1, b2) += x(b4, b3) * v;
                            at(g, m, b4, b3) += x(b1, b2) * v;
                          } else {  // EXCHANGE
                            at(g, m, b1, b3) += 0.5 * x(b4, b2) * v;
                            at(g, m, b4, b2) += 0.5 * x(b3, b1) * v;
                            at(g, m, b4, b1) += 0.5 * x(b3, b2) * v;
                            at(g, m, b2, b3) += 0.5 * x(b4, b1) * v;
                          }
                        }
                      }
              }
          }
        }
      }
  }
  for (int g = 0; g < nGrad; g++)
    for (int m = 0; m < nMat; m++) {
      double* out = AX[(size_t)g * nMat + m];
      for (int t = 0; t < nThreads; t++) {
        const double* a = &loc[(((size_t)t * nGrad + g) * nMat + m) * NN];
        for (int c = 0; c < N; c++)
          for (int r = 0; r < N; r++)
            out[r + (size_t)c * N] += 0.5 * (a[r + (size_t)c * N] + a[c + (size_t)r * N]);
      }
    }
}

}  // namespace

namespace {

using cdbl = std::complex<double>;
const cdbl I1(0.0, 1.0);

// s + v.sigma (2x2 spin matrix in Pauli components)
struct Q4 {
  cdbl s, v[3];
};
Q4 qmul(const Q4& p, const Q4& q) {
  Q4 r;
  r.s = p.s * q.s + p.v[0] * q.v[0] + p.v[1] * q.v[1] + p.v[2] * q.v[2];
  for (int x = 0; x < 3; x++) {
    int y = (x + 1) % 3, z = (x + 2) % 3;
    r.v[x] = p.s * q.v[x] + q.s * p.v[x] + I1 * (p.v[y] * q.v[z] - p.v[z] * q.v[y]);
  }
  return r;
}
Q4 sigma(int a) {  // a = 0 (identity), 1..3 (x, y, z)
  Q4 r{0.0, {0.0, 0.0, 0.0}};
  if (a == 0) r.s = 1.0;
  else r.v[a - 1] = 1.0;
  return r;
}

// Index of the 17 (X, AX) pairs of a 4C contraction list
// (DIRAC_PAULI_SPINOR_COMP, direct4C_libcint.hpp:279-310).
enum { CLLMS, XLLMS, XLLMX, XLLMY, XLLMZ, CSSMS, CSSMX, CSSMY, CSSMZ, XSSMS, XSSMX, XSSMY,
       XSSMZ, XLSMS, XLSMX, XLSMY, XLSMZ, NREL };

// (i, j, sign) patterns of the dot (a = 0) and cross (a = 1..3) products of
// two derivative directions.
struct Pat { int i, j; double s; };
const std::vector<Pat>& pat(int a) {
  static const std::vector<Pat> P[4] = {
      {{0, 0, 1}, {1, 1, 1}, {2, 2, 1}},
      {{1, 2, 1}, {2, 1, -1}},
      {{2, 0, 1}, {0, 2, -1}},
      {{0, 1, 1}, {1, 0, -1}}};
  return P[a];
}

// Shell-block norms of one complex N x N matrix (direct.hpp:73-90).
void norms_c(const Basis& bs, const cdbl* X, std::vector<double>& out) {
  int ns = (int)bs.shells.size(), N = bs.nbasis;
  out.assign((size_t)ns * ns, 0.0);
  shell_block_norm(bs, X, N, out.data());
}

struct Schwarz4C {
  std::vector<double> LL, SS;  // nshell^2
};

// direct4C_libcint.hpp:341-481
void schwarz_4c(const Basis& bs, bool needLL, bool needSS, Schwarz4C& Q) {
  const int ns = (int)bs.shells.size();
  const double C2 = 1.0 / (4.0 * 137.035999074 * 137.035999074);
  if (needLL) Q.LL.assign((size_t)ns * ns, 0.0);
  if (needSS) Q.SS.assign((size_t)ns * ns, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int s1 = 0; s1 < ns; s1++) {
    std::vector<double> buf, scr;
    for (int s2 = 0; s2 <= s1; s2++) {
      if (needLL) {
        eri_quartet(bs, s1, s2, s1, s2, buf, scr);
        double mx = 0;
        for (double v : buf) mx = std::max(mx, std::abs(v));
        Q.LL[s1 + (size_t)s2 * ns] = Q.LL[s2 + (size_t)s1 * ns] = std::sqrt(mx);
      }
      if (needSS) {
        eri_deriv_quartet(bs, s1, s2, s1, s2, 15, buf);
        double mx = 0;
        for (double v : buf) mx = std::max(mx, std::abs(v));
        Q.SS[s1 + (size_t)s2 * ns] = Q.SS[s2 + (size_t)s1 * ns] = C2 * std::sqrt(mx);
      }
    }
  }
}

inline Q4 dens(const cdbl* const* X, int base, size_t e) {
  return Q4{X[base][e], {X[base + 1][e], X[base + 2][e], X[base + 3][e]}};
}

// One contraction type (0 BARE_COULOMB, 1 LLSS, 2 SSSS) of
// directScaffoldLibcint; AX (17 N x N complex) is zeroed first (:313-314).
void direct_4c(const Basis& bs, int type, const cdbl* const* X, cdbl* const* AX, double thresh,
               const Schwarz4C& Qs, bool exchange) {
  const int ns = (int)bs.shells.size(), N = bs.nbasis;
  const size_t NN = (size_t)N * N;
  for (int m = 0; m < NREL; m++) std::fill(AX[m], AX[m] + NN, cdbl(0.0));
  // max shell-block norms over the matrices each type screens with
  std::vector<int> mats;
  if (type == 0) mats = {CLLMS, XLLMS, XLLMX, XLLMY, XLLMZ};
  else if (type == 1) mats = {CLLMS, CSSMS, CSSMX, CSSMY, CSSMZ, XLSMS, XLSMX, XLSMY, XLSMZ};
  else mats = {CSSMS, CSSMX, CSSMY, CSSMZ};
  std::vector<double> nrm((size_t)ns * ns, 0.0), tmp;
  for (int m : mats) {
    norms_c(bs, X[m], tmp);
    for (size_t i = 0; i < nrm.size(); i++) nrm[i] = std::max(nrm[i], std::abs(tmp[i]));
  }
  auto B = [&](int a, int b) { return nrm[a + (size_t)b * ns]; };
  const double* Q12 = (type == 0) ? Qs.LL.data() : Qs.SS.data();
  const double* Q34 = (type == 2) ? Qs.SS.data() : Qs.LL.data();
  const int nth = omp_get_max_threads();
  std::vector<cdbl> loc((size_t)nth * NREL * NN, cdbl(0.0));
#pragma omp parallel
  {
    const int tid = omp_get_thread_num();
    cdbl* A[NREL];
    for (int m = 0; m < NREL; m++) A[m] = &loc[((size_t)tid * NREL + m) * NN];
    auto ix = [N](int r, int c) { return (size_t)r + (size_t)c * N; };
    std::vector<double> buf, scr;
    size_t s1234 = 0;
    for (int s1 = 0; s1 < ns; s1++)
      for (int s2 = 0; s2 <= s1; s2++) {
        const double shMax12 = B(s1, s2);
        const int s3max = (type == 1) ? ns - 1 : s1;
        for (int s3 = 0; s3 <= s3max; s3++) {
          const double shMax123 = std::max(std::max(B(s1, s3), B(s2, s3)), shMax12);
          const int s4max = (type == 1) ? s3 : ((s1 == s3) ? s2 : s3);
          for (int s4 = 0; s4 <= s4max; s4++, s1234++) {
            if (s1234 % nth != (size_t)tid) continue;
            double shMax = std::max(B(s1, s4), std::max(B(s2, s4), B(s3, s4)));
            shMax = std::max(shMax, shMax123);
            if (shMax * Q12[s1 + (size_t)s2 * ns] * Q34[s3 + (size_t)s4 * ns] < thresh) continue;
            const int n1 = bs.shells[s1].size(), n2 = bs.shells[s2].size();
            const int n3 = bs.shells[s3].size(), n4 = bs.shells[s4].size();
            const int o1 = bs.off[s1], o2 = bs.off[s2], o3 = bs.off[s3], o4 = bs.off[s4];
            const double s12d = (s1 == s2) ? 1.0 : 2.0, s34d = (s3 == s4) ? 1.0 : 2.0;
            const size_t nq = (size_t)n1 * n2 * n3 * n4;
            if (type == 0) {
              eri_quartet(bs, s1, s2, s3, s4, buf, scr);
              const double deg = s12d * s34d * ((s1 == s3) ? (s2 == s4 ? 1.0 : 2.0) : 2.0);
              for (int i = 0; i < n1; i++)
                for (int j = 0; j < n2; j++)
                  for (int k = 0; k < n3; k++)
                    for (int l = 0; l < n4; l++) {
                      const int b1 = o1 + i, b2 = o2 + j, b3 = o3 + k, b4 = o4 + l;
                      double v = buf[(((size_t)i * n2 + j) * n3 + k) * n4 + l] * 0.5 * deg;
                      A[CLLMS][ix(b1, b2)] += v * X[CLLMS][ix(b4, b3)].real();
                      A[CLLMS][ix(b3, b4)] += v * X[CLLMS][ix(b2, b1)].real();
                      v *= 0.5;
                      for (int c = 0; c < 4; c++) {
                        A[XLLMS + c][ix(b1, b4)] += v * X[XLLMS + c][ix(b2, b3)];
                        A[XLLMS + c][ix(b1, b3)] += v * X[XLLMS + c][ix(b2, b4)];
                        A[XLLMS + c][ix(b2, b4)] += v * X[XLLMS + c][ix(b1, b3)];
                        A[XLLMS + c][ix(b2, b3)] += v * X[XLLMS + c][ix(b1, b4)];
                      }
                    }
              continue;
            }
            // derivative integrals: LLSS on (s1 s2), SSSS on all four
            eri_deriv_quartet(bs, s1, s2, s3, s4, type == 1 ? 3 : 15, buf);
            for (int i = 0; i < n1; i++)
              for (int j = 0; j < n2; j++)
                for (int k = 0; k < n3; k++)
                  for (int l = 0; l < n4; l++) {
                    const int b1 = o1 + i, b2 = o2 + j, b3 = o3 + k, b4 = o4 + l;
                    const size_t q = (((size_t)i * n2 + j) * n3 + k) * n4 + l;
                    if (type == 1) {
                      // operator components of the (1 2) pair
                      double M[4];
                      for (int a = 0; a < 4; a++) {
                        M[a] = 0.0;
                        for (const auto& p : pat(a)) M[a] += p.s * buf[(size_t)(3 * p.i + p.j) * nq + q];
                      }
                      // Coulomb: LL(3,4) from the SS density, SS(1,2) from LL
                      if (b3 >= b4) {
                        const Q4 d = dens(X, CSSMS, ix(b2, b1));
                        double r = M[0] * d.s.real();
                        for (int x = 0; x < 3; x++) r -= M[x + 1] * d.v[x].imag();
                        A[CLLMS][ix(b3, b4)] += s12d * r;
                      }
                      if (b1 >= b2) {
                        const double rho = X[CLLMS][ix(b4, b3)].real();
                        for (int a = 0; a < 4; a++) A[CSSMS + a][ix(b1, b2)] += s34d * M[a] * rho;
                      }
                      if (!exchange) continue;
                      // exchange LS blocks: -D P (P12 or P21)
                      auto ls = [&](int t1, int t2, int d1, int d2, double flip) {
                        const Q4 d = dens(X, XLSMS, ix(d1, d2));
                        Q4 r{0.0, {0.0, 0.0, 0.0}};
                        for (int a = 0; a < 4; a++) {
                          const cdbl c = (a == 0) ? cdbl(M[0]) : I1 * (flip * M[a]);
                          const Q4 t = qmul(d, sigma(a));
                          r.s += c * t.s;
                          for (int x = 0; x < 3; x++) r.v[x] += c * t.v[x];
                        }
                        A[XLSMS][ix(t1, t2)] -= r.s;
                        for (int x = 0; x < 3; x++) A[XLSMX + x][ix(t1, t2)] -= r.v[x];
                      };
                      ls(b3, b2, b4, b1, 1.0);
                      if (s1 != s2) ls(b3, b1, b4, b2, -1.0);
                      if (s3 != s4) {
                        ls(b4, b2, b3, b1, 1.0);
                        if (s1 != s2) ls(b4, b1, b3, b2, -1.0);
                      }
                    } else {
                      // combined operator components M[a][b] of (12)(34)
                      double M[4][4];
                      for (int a = 0; a < 4; a++)
                        for (int b = 0; b < 4; b++) {
                          double s = 0.0;
                          for (const auto& p : pat(a))
                            for (const auto& r : pat(b))
                              s += p.s * r.s * buf[(size_t)(27 * p.i + 9 * p.j + 3 * r.i + r.j) * nq + q];
                          M[a][b] = s;
                        }
                      // Coulomb: SS(t) = P_t rho, rho = Re Tr[P_o D(o2,o1)]/2
                      auto coul = [&](int t1, int t2, int d1, int d2, bool swap, double sd) {
                        const Q4 d = dens(X, CSSMS, ix(d1, d2));
                        const double rv[4] = {d.s.real(), -d.v[0].imag(), -d.v[1].imag(),
                                              -d.v[2].imag()};
                        for (int a = 0; a < 4; a++) {
                          double s = 0.0;
                          for (int b = 0; b < 4; b++) s += (swap ? M[b][a] : M[a][b]) * rv[b];
                          A[CSSMS + a][ix(t1, t2)] += sd * s;
                        }
                      };
                      if (b1 >= b2) coul(b1, b2, b4, b3, false, s34d);
                      if ((s1 != s3 || s2 != s4) && b3 >= b4) coul(b3, b4, b2, b1, true, s12d);
                      if (!exchange) continue;
                      // exchange SS: -P_first D P_second (fl: orientation signs)
                      auto ex = [&](int t1, int t2, int d1, int d2, bool swap, double f1, double f2) {
                        const Q4 d = dens(X, XSSMS, ix(d1, d2));
                        Q4 r{0.0, {0.0, 0.0, 0.0}};
                        for (int a = 0; a < 4; a++)
                          for (int b = 0; b < 4; b++) {
                            const double m = swap ? M[b][a] : M[a][b];
                            if (m == 0.0) continue;
                            cdbl c = m;
                            if (a > 0) c *= I1 * f1;
                            if (b > 0) c *= I1 * f2;
                            const Q4 t = qmul(qmul(sigma(a), d), sigma(b));
                            r.s += c * t.s;
                            for (int x = 0; x < 3; x++) r.v[x] += c * t.v[x];
                          }
                        A[XSSMS][ix(t1, t2)] -= r.s;
                        for (int x = 0; x < 3; x++) A[XSSMX + x][ix(t1, t2)] -= r.v[x];
                      };
                      if (b1 >= b4) ex(b1, b4, b2, b3, false, 1, 1);
                      if (s3 != s4 && b1 >= b3) ex(b1, b3, b2, b4, false, 1, -1);
                      if (s1 != s2) {
                        if (b2 >= b4) ex(b2, b4, b1, b3, false, -1, 1);
                        if (s3 != s4 && b2 >= b3) ex(b2, b3, b1, b4, false, -1, -1);
                      }
                      if (s1 != s3 || s2 != s4) {
                        if (b3 >= b2) ex(b3, b2, b4, b1, true, 1, 1);
                        if (s1 != s2 && b3 >= b1) ex(b3, b1, b4, b2, true, 1, -1);
                        if (s3 != s4 && b4 >= b2) {
                          ex(b4, b2, b3, b1, true, -1, 1);
                          if (s1 != s2 && b4 >= b1) ex(b4, b1, b3, b2, true, -1, -1);
                        }
                      }
                    }
                  }
          }
        }
      }
  }
  // thread reduction and the per-type epilogues
  std::vector<cdbl> red((size_t)NREL * NN, cdbl(0.0));
  for (int t = 0; t < nth; t++)
    for (size_t e = 0; e < (size_t)NREL * NN; e++) red[e] += loc[(size_t)t * NREL * NN + e];
  auto R = [&](int m) { return &red[(size_t)m * NN]; };
  if (type == 0) {
    for (int m = CLLMS; m <= XLLMZ; m++)
      for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++)
          AX[m][i + (size_t)j * N] += 0.5 * R(m)[i + (size_t)j * N] + 0.5 * std::conj(R(m)[j + (size_t)i * N]);
    return;
  }
  std::vector<int> her;
  for (int m = 0; m < NREL; m++) {
    cdbl f = (m == CSSMX || m == CSSMY || m == CSSMZ) ? I1 : cdbl(1.0);
    for (size_t e = 0; e < NN; e++) AX[m][e] += f * R(m)[e];
  }
  if (type == 1) her = {CLLMS, CSSMS, CSSMX, CSSMY, CSSMZ};
  else her = {CSSMS, CSSMX, CSSMY, CSSMZ, XSSMS, XSSMX, XSSMY, XSSMZ};
  for (int m : her)
    for (int i = 0; i < N; i++)
      for (int j = 0; j < i; j++) AX[m][j + (size_t)i * N] = std::conj(AX[m][i + (size_t)j * N]);
}

// ---------------------------------------------------------------- Gaunt
// The Gaunt term -alpha_1.alpha_2 / r12 (direct4C_libcint.hpp:2833-3907).
// Its 29-entry list continues DIRAC_PAULI_SPINOR_COMP with the LS Coulomb,
// SL Coulomb and SL exchange entries (:279-310).
enum { CLSMS = NREL, CLSMX, CLSMY, CLSMZ, CSLMS, CSLMX, CSLMY, CSLMZ, XSLMS, XSLMX, XSLMY, XSLMZ,
       NGAUNT };

// The 3 x 3 derivative block T[j][l] = (m d_j n | d_l k l) of one element,
// d/dr of the orbital on the second and third function, as the invariants
// the spin algebra needs: t = tr T, the cross vector tau = (T_yz - T_zy,
// T_zx - T_xz, T_xy - T_yx) and S' = T + T^T - t I.  The transposed block
// T^T has the same t and S' and -tau.
struct GT {
  double T[3][3], t, tau[3], Sp[3][3];
};
GT gt_of(const double* v, bool transpose) {
  GT g;
  for (int j = 0; j < 3; j++)
    for (int l = 0; l < 3; l++) g.T[j][l] = transpose ? v[3 * l + j] : v[3 * j + l];
  g.t = g.T[0][0] + g.T[1][1] + g.T[2][2];
  g.tau[0] = g.T[1][2] - g.T[2][1];
  g.tau[1] = g.T[2][0] - g.T[0][2];
  g.tau[2] = g.T[0][1] - g.T[1][0];
  for (int j = 0; j < 3; j++)
    for (int l = 0; l < 3; l++) g.Sp[j][l] = g.T[j][l] + g.T[l][j] - (j == l ? g.t : 0.0);
  return g;
}

// Spin algebra of the four update kinds.  With two-spinor charge densities
// rho^k_LS = (-i/2c) sum_j (s_k s_j) chi d_j chi, rho^k_SL its adjoint, and
// the identities sum_k s_k X s_k = 2 tr(X) - X and
// sum_jl T_jl s_j (d0 + d.s) s_l = d0 t - i d.tau + (i d0 tau + S' d).s,
// every update is a fixed 4 x 4 complex map of Pauli components (storage
// scale S = 2 d0 etc. carries through, the maps being linear):
//   LL exchange from the SS density  (:3436-3480):  3 (d0 t - i d.tau), -(i d0 tau + S' d)
//   SS exchange from the LL density  (:3487-3535):  3 d0 t - i d.tau, -3 i d0 tau - S' d
//   LS Coulomb from SL (1) and LS (2) (:3541-3610): (d1_0 - d2_0) t + i (d1 + d2).tau,
//                                       i (d2_0 - d1_0) tau + (T^T - t)(d1 + d2)
//   LS exchange from the SL density  (:3613-3680):  d0 t - i d.tau, i d0 tau + S' d - 4 T^T d
Q4 g_ll(const GT& g, const Q4& d) {
  Q4 r;
  cdbl dt = d.v[0] * g.tau[0] + d.v[1] * g.tau[1] + d.v[2] * g.tau[2];
  r.s = 3.0 * (d.s * g.t - I1 * dt);
  for (int x = 0; x < 3; x++)
    r.v[x] = -(I1 * d.s * g.tau[x] + g.Sp[x][0] * d.v[0] + g.Sp[x][1] * d.v[1] + g.Sp[x][2] * d.v[2]);
  return r;
}
Q4 g_ss(const GT& g, const Q4& d) {
  Q4 r;
  cdbl dt = d.v[0] * g.tau[0] + d.v[1] * g.tau[1] + d.v[2] * g.tau[2];
  r.s = 3.0 * d.s * g.t - I1 * dt;
  for (int x = 0; x < 3; x++)
    r.v[x] = -3.0 * I1 * d.s * g.tau[x] -
             (g.Sp[x][0] * d.v[0] + g.Sp[x][1] * d.v[1] + g.Sp[x][2] * d.v[2]);
  return r;
}
Q4 g_cls(const GT& g, const Q4& d1, const Q4& d2) {
  Q4 r;
  cdbl e[3];
  for (int x = 0; x < 3; x++) e[x] = d1.v[x] + d2.v[x];
  r.s = (d1.s - d2.s) * g.t + I1 * (e[0] * g.tau[0] + e[1] * g.tau[1] + e[2] * g.tau[2]);
  for (int x = 0; x < 3; x++)
    r.v[x] = I1 * (d2.s - d1.s) * g.tau[x] + g.T[0][x] * e[0] + g.T[1][x] * e[1] +
             g.T[2][x] * e[2] - g.t * e[x];
  return r;
}
Q4 g_xls(const GT& g, const Q4& d) {
  Q4 r;
  cdbl dt = d.v[0] * g.tau[0] + d.v[1] * g.tau[1] + d.v[2] * g.tau[2];
  r.s = d.s * g.t - I1 * dt;
  for (int x = 0; x < 3; x++) {
    r.v[x] = I1 * d.s * g.tau[x];
    for (int y = 0; y < 3; y++) r.v[x] += (g.Sp[x][y] - 4.0 * g.T[y][x]) * d.v[y];
  }
  return r;
}

// SchwarzGaunt (:2910-2955): Q^G(s1, s2) = C1 sqrt(max |(d s1 s2 | d s1 s2)|)
// over the 9 components and the block, derivatives on the first function of
// each pair, C1 = 1 / 2c; not symmetric in (s1, s2).
void schwarz_gaunt(const Basis& bs, std::vector<double>& QG) {
  const int ns = (int)bs.shells.size();
  const double C1 = 1.0 / (2.0 * 137.035999074);
  QG.assign((size_t)ns * ns, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int s1 = 0; s1 < ns; s1++) {
    std::vector<double> buf;
    for (int s2 = 0; s2 < ns; s2++) {
      eri_deriv_quartet(bs, s1, s2, s1, s2, 5, buf);
      double mx = 0;
      for (double v : buf) mx = std::max(mx, std::abs(v));
      QG[s1 + (size_t)s2 * ns] = C1 * std::sqrt(mx);
    }
  }
}

// The Gaunt contraction on the 29 (X, AX) entries; AX is zeroed first.
// Quartets (:2996-3160): s1, s2 over all shells, s3 <= s2, s4 <= (s2 == s3 ?
// s1 : last) -- every unordered pair of (differentiated, other) shell pairs
// (s2, s1), (s3, s4) once -- screened by max shell-block norm of the 16
// exchange densities times Q^G(s3, s4) Q^G(s2, s1).  Per element (m n | k l)
// the reference's update sites and conditions (:3436-3680), with T and, for
// the image (l k | n m), T^T; then LL and SS exchange get their upper
// triangles from the lower ones (:3833-3858).
void direct_gaunt(const Basis& bs, const cdbl* const* X, cdbl* const* AX, double thresh,
                  const std::vector<double>& QG, bool exchange) {
  const int ns = (int)bs.shells.size(), N = bs.nbasis;
  const size_t NN = (size_t)N * N;
  for (int m = 0; m < NGAUNT; m++) std::fill(AX[m], AX[m] + NN, cdbl(0.0));
  std::vector<double> nrm((size_t)ns * ns, 0.0), tmp;
  for (int base : {(int)XLSMS, (int)XSLMS, (int)XLLMS, (int)XSSMS})
    for (int c = 0; c < 4; c++) {
      norms_c(bs, X[base + c], tmp);
      for (size_t i = 0; i < nrm.size(); i++) nrm[i] = std::max(nrm[i], std::abs(tmp[i]));
    }
  auto B = [&](int a, int b) { return nrm[a + (size_t)b * ns]; };
  const int nth = omp_get_max_threads();
  std::vector<cdbl> loc((size_t)nth * NGAUNT * NN, cdbl(0.0));
#pragma omp parallel
  {
    const int tid = omp_get_thread_num();
    cdbl* A[NGAUNT];
    for (int m = 0; m < NGAUNT; m++) A[m] = &loc[((size_t)tid * NGAUNT + m) * NN];
    auto ix = [N](int r, int c) { return (size_t)r + (size_t)c * N; };
    auto put = [&](int base, size_t e, const Q4& q) {
      A[base][e] += q.s;
      for (int x = 0; x < 3; x++) A[base + 1 + x][e] += q.v[x];
    };
    std::vector<double> buf;
    size_t s1234 = 0;
    for (int s1 = 0; s1 < ns; s1++)
      for (int s2 = 0; s2 < ns; s2++) {
        const double shMax12 = B(s2, s1);
        for (int s3 = 0; s3 <= s2; s3++) {
          const double shMax123 = std::max(std::max(B(s1, s3), B(s2, s3)), shMax12);
          const int s4max = (s2 == s3) ? s1 : ns - 1;
          for (int s4 = 0; s4 <= s4max; s4++, s1234++) {
            if (s1234 % nth != (size_t)tid) continue;
            double shMax = std::max(B(s1, s4), std::max(B(s2, s4), B(s3, s4)));
            shMax = std::max(shMax, shMax123);
            if (shMax * QG[s3 + (size_t)s4 * ns] * QG[s2 + (size_t)s1 * ns] < thresh) continue;
            eri_deriv_quartet(bs, s1, s2, s3, s4, 6, buf);
            const int n1 = bs.shells[s1].size(), n2 = bs.shells[s2].size();
            const int n3 = bs.shells[s3].size(), n4 = bs.shells[s4].size();
            const size_t nq = (size_t)n1 * n2 * n3 * n4;
            const bool img = (s1 != s4) || (s2 != s3);
            for (int i = 0; i < n1; i++)
              for (int j = 0; j < n2; j++)
                for (int k = 0; k < n3; k++)
                  for (int l = 0; l < n4; l++) {
                    const int m1 = bs.off[s1] + i, m2 = bs.off[s2] + j;
                    const int m3 = bs.off[s3] + k, m4 = bs.off[s4] + l;
                    const size_t q = (((size_t)i * n2 + j) * n3 + k) * n4 + l;
                    double v[9];
                    for (int c = 0; c < 9; c++) v[c] = buf[(size_t)c * nq + q];
                    const GT T = gt_of(v, false), Tt = gt_of(v, true);
                    if (exchange) {
                      if (s1 >= s4) put(XLLMS, ix(m1, m4), g_ll(T, dens(X, XSSMS, ix(m2, m3))));
                      if (s1 < s4 || (s1 == s4 && s2 != s3))
                        put(XLLMS, ix(m4, m1), g_ll(Tt, dens(X, XSSMS, ix(m3, m2))));
                      put(XSSMS, ix(m2, m3), g_ss(Tt, dens(X, XLLMS, ix(m1, m4))));
                      if (s1 != s4 && s2 == s3)
                        put(XSSMS, ix(m3, m2), g_ss(T, dens(X, XLLMS, ix(m4, m1))));
                    }
                    put(CLSMS, ix(m1, m2),
                        g_cls(T, dens(X, CSLMS, ix(m3, m4)), dens(X, CLSMS, ix(m4, m3))));
                    if (img)
                      put(CLSMS, ix(m4, m3),
                          g_cls(Tt, dens(X, CSLMS, ix(m2, m1)), dens(X, CLSMS, ix(m1, m2))));
                    if (exchange) {
                      put(XLSMS, ix(m1, m3), g_xls(T, dens(X, XSLMS, ix(m2, m4))));
                      if (img) put(XLSMS, ix(m4, m2), g_xls(Tt, dens(X, XSLMS, ix(m3, m1))));
                    }
                  }
          }
        }
      }
  }
  for (int t = 0; t < nth; t++)
    for (int m = 0; m < NGAUNT; m++)
      for (size_t e = 0; e < NN; e++) AX[m][e] += loc[((size_t)t * NGAUNT + m) * NN + e];
  if (!exchange) return;
  for (int m : {XLLMS, XLLMX, XLLMY, XLLMZ, XSSMS, XSSMX, XSSMY, XSSMZ})
    for (int i = 0; i < N; i++)
      for (int j = 0; j < i; j++) AX[m][j + (size_t)i * N] = std::conj(AX[m][i + (size_t)j * N]);
}


// ---------------------------------------------------------------- Gauge
// The gauge part of the Breit interaction (direct4C_libcint.hpp:3908-5160):
// the GAUNT list and update sites with the kernel -r_i r_i' / r12^3 of
// (alpha_1 . r12)(alpha_2 . r12) / r12^3 in place of Gaunt's
// -delta_ii' / r12 (the build then halves the Gaunt weight, so that the sum
// is the Breit term).  Per element the integrals are
//   V[i][i'][j][l] = (m d_j n | -r_i r_i' / r^3 | d_l k l)
//                  = -delta_ii' T[j][l] + (m d_j n | d_i d_i' r12 | d_l k l),
// using r_i r_i' / r^3 = delta_ii' / r - d_i d_i' r (derivatives in
// r = r1 - r2).  With sigma_i sigma_j = Q_ij and general V the four update
// kinds are
//   LL exchange from SS:  -sum V^{ii'}_{jl} Q_ij D Q_li'
//   SS exchange from LL:  -sum V^{ii'}_{jl} Q_ji D Q_i'l
//   LS Coulomb from SL (1), LS (2):
//                  1/2 sum V^{ii'}_{jl} Q_ij (tr[Q_li' D2] - tr[Q_i'l D1])
//   LS exchange from SL:   sum V^{ii'}_{jl} Q_ij D Q_i'l
// (for V = -delta T they reduce to the Gaunt maps); the image (l k | n m)
// takes V with j and l exchanged (the kernel is even in r12).
struct GV {
  double v[3][3][3][3];  // [i][i'][j][l]
};
Q4 qij(int i, int j) {  // sigma_i sigma_j = delta_ij + i eps_ijm sigma_m
  Q4 r{0.0, {0.0, 0.0, 0.0}};
  if (i == j) r.s = 1.0;
  else {
    const int m = 3 - i - j;
    r.v[m] = (j == (i + 1) % 3) ? I1 : -I1;
  }
  return r;
}
cdbl qtr(const Q4& q) { return 2.0 * q.s; }  // trace of the 2 x 2 matrix
Q4 qscale(const Q4& q, cdbl f) {
  Q4 r{q.s * f, {q.v[0] * f, q.v[1] * f, q.v[2] * f}};
  return r;
}
void qacc(Q4& a, const Q4& b) {
  a.s += b.s;
  for (int x = 0; x < 3; x++) a.v[x] += b.v[x];
}
GV gv_of(const double* T, const double* const* U, size_t q, size_t nq, bool img) {
  // T: 9 Coulomb components [j][l]; U[6]: d_i d_i' r12 for (i, i') = xx, xy,
  // xz, yy, yz, zz, each 9 components [j][l]
  static const int sym[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  GV g;
  for (int i = 0; i < 3; i++)
    for (int ip = 0; ip < 3; ip++)
      for (int j = 0; j < 3; j++)
        for (int l = 0; l < 3; l++) {
          const int jj = img ? l : j, ll = img ? j : l;
          double v = U[sym[i][ip]][(size_t)(3 * jj + ll) * nq + q];
          if (i == ip) v -= T[(size_t)(3 * jj + ll) * nq + q];
          g.v[i][ip][j][l] = v;
        }
  return g;
}
Q4 gg_ll(const GV& g, const Q4& d) {
  Q4 r{0.0, {0.0, 0.0, 0.0}};
  for (int i = 0; i < 3; i++)
    for (int ip = 0; ip < 3; ip++)
      for (int j = 0; j < 3; j++)
        for (int l = 0; l < 3; l++)
          if (g.v[i][ip][j][l] != 0.0)
            qacc(r, qscale(qmul(qmul(qij(i, j), d), qij(l, ip)), -g.v[i][ip][j][l]));
  return r;
}
Q4 gg_ss(const GV& g, const Q4& d) {
  Q4 r{0.0, {0.0, 0.0, 0.0}};
  for (int i = 0; i < 3; i++)
    for (int ip = 0; ip < 3; ip++)
      for (int j = 0; j < 3; j++)
        for (int l = 0; l < 3; l++)
          if (g.v[i][ip][j][l] != 0.0)
            qacc(r, qscale(qmul(qmul(qij(j, i), d), qij(ip, l)), -g.v[i][ip][j][l]));
  return r;
}
Q4 gg_cls(const GV& g, const Q4& d1, const Q4& d2) {
  Q4 r{0.0, {0.0, 0.0, 0.0}};
  for (int i = 0; i < 3; i++)
    for (int ip = 0; ip < 3; ip++)
      for (int j = 0; j < 3; j++)
        for (int l = 0; l < 3; l++)
          if (g.v[i][ip][j][l] != 0.0) {
            const cdbl w = 0.5 * g.v[i][ip][j][l] *
                           (qtr(qmul(qij(l, ip), d2)) - qtr(qmul(qij(ip, l), d1)));
            qacc(r, qscale(qij(i, j), w));
          }
  return r;
}
Q4 gg_xls(const GV& g, const Q4& d) {
  Q4 r{0.0, {0.0, 0.0, 0.0}};
  for (int i = 0; i < 3; i++)
    for (int ip = 0; ip < 3; ip++)
      for (int j = 0; j < 3; j++)
        for (int l = 0; l < 3; l++)
          if (g.v[i][ip][j][l] != 0.0)
            qacc(r, qscale(qmul(qmul(qij(i, j), d), qij(ip, l)), g.v[i][ip][j][l]));
  return r;
}

// The V blocks of one contracted quartet: T (Coulomb, 9 components) and the
// six d_i d_i' r12 blocks, derivatives on the centres in dmask.
void gauge_blocks(const Basis& bs, int s1, int s2, int s3, int s4, int dmask,
                  std::vector<double>& T, std::vector<double> (&U)[6]) {
  static const int ops[6][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}};
  eri_deriv_quartet(bs, s1, s2, s3, s4, dmask, T);
  for (int k = 0; k < 6; k++) eri_deriv_quartet(bs, s1, s2, s3, s4, dmask, U[k], ops[k]);
}

// SchwarzGauge (:3960-4005): Q(o, d) = C1 sqrt(max |V|) over the block
// (o d_j d | o d_l d) and its components, derivatives on the second
// function of each pair, indexed [o + d * nshell].  The reference maxes over
// libcint's 16 spin components of the same operator; here over the 81
// spatial components of V.
void schwarz_gauge(const Basis& bs, std::vector<double>& QB) {
  const int ns = (int)bs.shells.size();
  const double C1 = 1.0 / (2.0 * 137.035999074);
  QB.assign((size_t)ns * ns, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int o = 0; o < ns; o++) {
    std::vector<double> T, U[6];
    for (int d = 0; d < ns; d++) {
      gauge_blocks(bs, o, d, o, d, 10, T, U);
      const size_t nq = T.size() / 9;
      const double* Up[6];
      for (int k = 0; k < 6; k++) Up[k] = U[k].data();
      double mx = 0.0;
      for (size_t q = 0; q < nq; q++) {
        const GV g = gv_of(T.data(), Up, q, nq, false);
        for (int a = 0; a < 81; a++) mx = std::max(mx, std::abs((&g.v[0][0][0][0])[a]));
      }
      QB[o + (size_t)d * ns] = C1 * std::sqrt(mx);
    }
  }
}

// The GAUGE contraction on the 29 (X, AX) entries; AX is zeroed first.
// Quartets and sites as direct_gaunt (:4170-4215, :4400-5100), screened by
// shMax Q(s1, s2) Q(s4, s3) (:4213).
void direct_gauge(const Basis& bs, const cdbl* const* X, cdbl* const* AX, double thresh,
                  const std::vector<double>& QB, bool exchange) {
  const int ns = (int)bs.shells.size(), N = bs.nbasis;
  const size_t NN = (size_t)N * N;
  for (int m = 0; m < NGAUNT; m++) std::fill(AX[m], AX[m] + NN, cdbl(0.0));
  std::vector<double> nrm((size_t)ns * ns, 0.0), tmp;
  for (int base : {(int)XLSMS, (int)XSLMS, (int)XLLMS, (int)XSSMS})
    for (int c = 0; c < 4; c++) {
      norms_c(bs, X[base + c], tmp);
      for (size_t i = 0; i < nrm.size(); i++) nrm[i] = std::max(nrm[i], std::abs(tmp[i]));
    }
  auto B = [&](int a, int b) { return nrm[a + (size_t)b * ns]; };
  const int nth = omp_get_max_threads();
  std::vector<cdbl> loc((size_t)nth * NGAUNT * NN, cdbl(0.0));
#pragma omp parallel
  {
    const int tid = omp_get_thread_num();
    cdbl* A[NGAUNT];
    for (int m = 0; m < NGAUNT; m++) A[m] = &loc[((size_t)tid * NGAUNT + m) * NN];
    auto ix = [N](int r, int c) { return (size_t)r + (size_t)c * N; };
    auto put = [&](int base, size_t e, const Q4& q) {
      A[base][e] += q.s;
      for (int x = 0; x < 3; x++) A[base + 1 + x][e] += q.v[x];
    };
    std::vector<double> T, U[6];
    size_t s1234 = 0;
    for (int s1 = 0; s1 < ns; s1++)
      for (int s2 = 0; s2 < ns; s2++) {
        const double shMax12 = B(s2, s1);
        for (int s3 = 0; s3 <= s2; s3++) {
          const double shMax123 = std::max(std::max(B(s1, s3), B(s2, s3)), shMax12);
          const int s4max = (s2 == s3) ? s1 : ns - 1;
          for (int s4 = 0; s4 <= s4max; s4++, s1234++) {
            if (s1234 % nth != (size_t)tid) continue;
            double shMax = std::max(B(s1, s4), std::max(B(s2, s4), B(s3, s4)));
            shMax = std::max(shMax, shMax123);
            if (shMax * QB[s1 + (size_t)s2 * ns] * QB[s4 + (size_t)s3 * ns] < thresh) continue;
            gauge_blocks(bs, s1, s2, s3, s4, 6, T, U);
            const double* Up[6];
            for (int k = 0; k < 6; k++) Up[k] = U[k].data();
            const int n1 = bs.shells[s1].size(), n2 = bs.shells[s2].size();
            const int n3 = bs.shells[s3].size(), n4 = bs.shells[s4].size();
            const size_t nq = (size_t)n1 * n2 * n3 * n4;
            const bool img = (s1 != s4) || (s2 != s3);
            for (int i = 0; i < n1; i++)
              for (int j = 0; j < n2; j++)
                for (int k = 0; k < n3; k++)
                  for (int l = 0; l < n4; l++) {
                    const int m1 = bs.off[s1] + i, m2 = bs.off[s2] + j;
                    const int m3 = bs.off[s3] + k, m4 = bs.off[s4] + l;
                    const size_t q = (((size_t)i * n2 + j) * n3 + k) * n4 + l;
                    const GV V = gv_of(T.data(), Up, q, nq, false);
                    const GV Vt = gv_of(T.data(), Up, q, nq, true);
                    if (exchange) {
                      if (s1 >= s4) put(XLLMS, ix(m1, m4), gg_ll(V, dens(X, XSSMS, ix(m2, m3))));
                      if (s1 < s4 || (s1 == s4 && s2 != s3))
                        put(XLLMS, ix(m4, m1), gg_ll(Vt, dens(X, XSSMS, ix(m3, m2))));
                      put(XSSMS, ix(m2, m3), gg_ss(V, dens(X, XLLMS, ix(m1, m4))));
                      if (s1 != s4 && s2 == s3)
                        put(XSSMS, ix(m3, m2), gg_ss(Vt, dens(X, XLLMS, ix(m4, m1))));
                    }
                    put(CLSMS, ix(m1, m2),
                        gg_cls(V, dens(X, CSLMS, ix(m3, m4)), dens(X, CLSMS, ix(m4, m3))));
                    if (img)
                      put(CLSMS, ix(m4, m3),
                          gg_cls(Vt, dens(X, CSLMS, ix(m2, m1)), dens(X, CLSMS, ix(m1, m2))));
                    if (exchange) {
                      put(XLSMS, ix(m1, m3), gg_xls(V, dens(X, XSLMS, ix(m2, m4))));
                      if (img) put(XLSMS, ix(m4, m2), gg_xls(Vt, dens(X, XSLMS, ix(m3, m1))));
                    }
                  }
          }
        }
      }
  }
  for (int t = 0; t < nth; t++)
    for (int m = 0; m < NGAUNT; m++)
      for (size_t e = 0; e < NN; e++) AX[m][e] += loc[((size_t)t * NGAUNT + m) * NN + e];
  if (!exchange) return;
  for (int m : {XLLMS, XLLMX, XLLMY, XLLMZ, XSSMS, XSSMX, XSSMY, XSSMZ})
    for (int i = 0; i < N; i++)
      for (int j = 0; j < i; j++) AX[m][j + (size_t)i * N] = std::conj(AX[m][i + (size_t)j * N]);
}

}  // namespace

extern "C" {

// FourCompFock::formGDDirect (fourcompfock/impl.hpp:3752-4636) with
// BareCoulomb / DiracCoulomb / DiracCoulombSSSS switches.  D and G: 4 Pauli
// components (S, X, Y, Z) of 2N x 2N complex column-major matrices; G gets
// twoeH - xHFX * K.
// libcint selects the reference's bare-Coulomb branch: with libcint the
// 17-entry BARE_COULOMB contraction and twoeH_LL = 2 CLLMS
// (fourcompfock/impl.hpp:3901-3933), without it the 1C J/K contraction and
// twoeH_LL = J (:3934-3969).
int orc_dirac_coulomb(void* b, const void* const* Dv, void* const* Gv, int bare, int dc,
                      int ssss, double xHFX, double thresh, int libcint, int gaunt, int gauge) {
  auto* bs = static_cast<Basis*>(b);
  const int N = bs->nbasis, N2 = 2 * N;
  const cdbl* const* D = reinterpret_cast<const cdbl* const*>(Dv);
  cdbl* const* G = reinterpret_cast<cdbl* const*>(Gv);
  const double c = 137.035999074, C2 = 1.0 / (4 * c * c), C4 = 1.0 / (16 * c * c * c * c);
  const bool exch = std::abs(xHFX) >= 1e-12;
  const size_t NN = (size_t)N * N, NN2 = (size_t)N2 * N2;
  // blocks LL, SS, LS, SL of each Pauli component
  std::vector<cdbl> blk[4][4];
  const int bro[4] = {0, N, 0, N}, bco[4] = {0, N, N, 0};
  for (int cmp = 0; cmp < 4; cmp++)
    for (int k = 0; k < 4; k++) {
      blk[k][cmp].assign(NN, 0.0);
      for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++)
          blk[k][cmp][i + (size_t)j * N] = D[cmp][(bro[k] + i) + (size_t)(bco[k] + j) * N2];
    }
  std::vector<cdbl> ax((size_t)NGAUNT * NN);
  const cdbl* X[NGAUNT];
  cdbl* AX[NGAUNT];
  for (int m = 0; m < NGAUNT; m++) AX[m] = &ax[(size_t)m * NN];
  X[CLLMS] = blk[0][0].data();
  for (int c4 = 0; c4 < 4; c4++) {
    X[XLLMS + c4] = blk[0][c4].data();
    X[CSSMS + c4] = blk[1][c4].data();
    X[XSSMS + c4] = blk[1][c4].data();
    X[XLSMS + c4] = blk[2][c4].data();
    X[CLSMS + c4] = blk[2][c4].data();
    X[CSLMS + c4] = blk[3][c4].data();
    X[XSLMS + c4] = blk[3][c4].data();
  }
  std::vector<cdbl> twoeH[4], K[4];
  for (int c4 = 0; c4 < 4; c4++) {
    twoeH[c4].assign(NN2, 0.0);
    K[c4].assign(NN2, 0.0);
  }
  auto add = [&](std::vector<cdbl>& dst, int ro, int co, const cdbl* src, cdbl f) {
    for (int j = 0; j < N; j++)
      for (int i = 0; i < N; i++) dst[(ro + i) + (size_t)(co + j) * N2] += f * src[i + (size_t)j * N];
  };
  Schwarz4C Qs;
  schwarz_4c(*bs, bare || dc, dc || ssss, Qs);
  if (bare) {
    direct_4c(*bs, 0, X, AX, thresh, Qs, exch);
    add(twoeH[0], 0, 0, AX[CLLMS], libcint ? 2.0 : 1.0);
    if (exch)
      for (int c4 = 0; c4 < 4; c4++) add(K[c4], 0, 0, AX[XLLMS + c4], 1.0);
  }
  if (dc) {
    direct_4c(*bs, 1, X, AX, thresh, Qs, exch);
    add(twoeH[0], 0, 0, AX[CLLMS], 2.0 * C2);
    for (int c4 = 0; c4 < 4; c4++) add(twoeH[c4], N, N, AX[CSSMS + c4], 2.0 * C2);
    if (exch)
      for (int c4 = 0; c4 < 4; c4++) add(K[c4], 0, N, AX[XLSMS + c4], -C2);
  }
  if (ssss) {
    direct_4c(*bs, 2, X, AX, thresh, Qs, exch);
    for (int c4 = 0; c4 < 4; c4++) add(twoeH[c4], N, N, AX[CSSMS + c4], 2.0 * C4);
    if (exch)
      for (int c4 = 0; c4 < 4; c4++) add(K[c4], N, N, AX[XSSMS + c4], -C4);
  }
  // Gaunt and Gauge (impl.hpp:4228-4540): with the gauge term both are
  // weighted C2 / 2 (their sum is the Breit term)
  const double C2b = gauge ? 0.5 * C2 : C2;
  auto breit_add = [&]() {
    for (int c4 = 0; c4 < 4; c4++) add(twoeH[c4], 0, N, AX[CLSMS + c4], 2.0 * C2b);
    if (exch)
      for (int c4 = 0; c4 < 4; c4++) {
        add(K[c4], 0, 0, AX[XLLMS + c4], -C2b);
        add(K[c4], N, N, AX[XSSMS + c4], -C2b);
        add(K[c4], 0, N, AX[XLSMS + c4], -C2b);
      }
  };
  if (gaunt) {
    std::vector<double> QG;
    schwarz_gaunt(*bs, QG);
    direct_gaunt(*bs, X, AX, thresh, QG, exch);
    breit_add();
  }
  if (gauge) {
    std::vector<double> QB;
    schwarz_gauge(*bs, QB);
    direct_gauge(*bs, X, AX, thresh, QB, exch);
    breit_add();
  }
  // LS -> SL as the conjugate transpose, then G = twoeH - xHFX K
  for (int c4 = 0; c4 < 4; c4++) {
    for (auto* M : {&twoeH[c4], &K[c4]})
      for (int j = 0; j < N; j++)
        for (int i = 0; i < N; i++)
          (*M)[(N + j) + (size_t)i * N2] = std::conj((*M)[i + (size_t)(N + j) * N2]);
    for (size_t e = 0; e < NN2; e++) G[c4][e] = twoeH[c4][e] - (exch ? xHFX * K[c4][e] : 0.0);
  }
  return 0;
}

// One contraction type (0 BARE_COULOMB, 1 LLSS, 2 SSSS, 3 GAUNT, 4 GAUGE) of
// GTODirectRelERIContraction::twoBodyContract on the N x N complex (X, AX)
// entries in DIRAC_PAULI_SPINOR_COMP order (17, or 29 for GAUNT and GAUGE);
// AX is zeroed first (direct4C_libcint.hpp:313-314).
// Derivative ERIs of one contracted shell quartet (eri_deriv_quartet):
// comp-major blocks over the AO functions of s1..s4, derivatives (d/dr of
// the orbital) on the centres in dmask (bit 0..3 = s1..s4); returns the
// number of values written.
int orc_eri_deriv_quartet(void* b, int s1, int s2, int s3, int s4, int dmask, double* out) {
  const auto* bs = static_cast<const Basis*>(b);
  std::vector<double> buf;
  eri_deriv_quartet(*bs, s1, s2, s3, s4, dmask, buf);
  std::copy(buf.begin(), buf.end(), out);
  return (int)buf.size();
}

// As orc_eri_deriv_quartet with the kernel d_i d_j r12 (i, j = 0..2, -1 for
// none; derivatives in r = r1 - r2) in place of 1 / r12.
int orc_r12_deriv_quartet(void* b, int s1, int s2, int s3, int s4, int dmask, int i, int j,
                          double* out) {
  const auto* bs = static_cast<const Basis*>(b);
  const int op[2] = {i, j};
  std::vector<double> buf;
  eri_deriv_quartet(*bs, s1, s2, s3, s4, dmask, buf, op);
  std::copy(buf.begin(), buf.end(), out);
  return (int)buf.size();
}

int orc_rel_contract(void* b, int type, const void* const* Xv, void* const* AXv, double thresh,
                     int exchange) {
  auto* bs = static_cast<Basis*>(b);
  const cdbl* const* X = reinterpret_cast<const cdbl* const*>(Xv);
  cdbl* const* AX = reinterpret_cast<cdbl* const*>(AXv);
  if (type == 3) {
    std::vector<double> QG;
    schwarz_gaunt(*bs, QG);
    direct_gaunt(*bs, X, AX, thresh, QG, exchange != 0);
    return 0;
  }
  if (type == 4) {
    std::vector<double> QB;
    schwarz_gauge(*bs, QB);
    direct_gauge(*bs, X, AX, thresh, QB, exchange != 0);
    return 0;
  }
  Schwarz4C Qs;
  schwarz_4c(*bs, type <= 1, type >= 1, Qs);
  direct_4c(*bs, type, X, AX, thresh, Qs, exchange != 0);
  return 0;
}

// DirectGradContraction::directScaffoldGrad on real Hermitian X
// (grad_scaffold); AX: 3 * natom * nMat arrays, component-major.
int orc_grad_contract(void* b, const int* shell_atom, int natom, int nMat, const int* type,
                      const double* const* X, double* const* AX, int nthreads) {
  grad_scaffold(*static_cast<Basis*>(b), shell_atom, natom, nMat, type, X, AX, nthreads);
  return 0;
}


}  // extern "C"
