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
template <typename T>
void direct_scaffold(Basis& bs, int nMat, const int* her, const int* type,
                     const T* const* X, T* const* AX, double thresh, int nThreads,
                     bool screen, Stats* stats) {
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
int orc_contract(void* b, int nMat, int is_complex, const int* her, const int* type,
                 const void* const* X, void* const* AX, double thresh, int nthreads,
                 int screen, long long* stats_out) {
  auto* bs = static_cast<Basis*>(b);
  Stats st;
  if (is_complex)
    direct_scaffold<dcomplex>(*bs, nMat, her, type, reinterpret_cast<const dcomplex* const*>(X),
                              reinterpret_cast<dcomplex* const*>(AX), thresh, nthreads,
                              screen != 0, &st);
  else
    direct_scaffold<double>(*bs, nMat, her, type, reinterpret_cast<const double* const*>(X),
                            reinterpret_cast<double* const*>(AX), thresh, nthreads, screen != 0,
                            &st);
  if (stats_out) {
    stats_out[0] = st.quartets_total;
    stats_out[1] = st.quartets_screened;
    stats_out[2] = st.quartets_computed;
  }
  return 0;
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
