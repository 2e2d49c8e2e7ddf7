// Nuclear-gradient contraction on the device.
//
// Replaces DirectGradContraction::gradTwoBodyContract (include/
// particleintegrals/gradints.hpp:278-283) -> directScaffoldGrad
// (include/particleintegrals/contract/direct.hpp:2198-2571): for Hermitian
// real densities X, the J- and K-type contractions of the first derivatives
// of the ERIs with respect to every nuclear coordinate,
//   AX[atom, xyz] += 1/2 (A + A^T),  A = sum over quartets of
//   d(12|34)/dR_{atom,xyz} at the COULOMB / EXCHANGE update sites,
// over the reference's quartet set (unordered pairs of significant shell
// pairs, no screening: the reference's loop has none) with its degeneracy
// factors.  The derivative of a quartet with respect to the centre of one of
// its shells is minus the d/dr of that shell's functions; each of the 12
// (4 centres x 3 axes) goes to the component of the shell's atom.
//
// One thread per unique shell quartet and ket Cartesian component pair:
// per bra primitive pair the Hermite tables raised by one on both centres,
// the ket-contracted Hermite sums of the plain ket and of its six
// derivatives (on C or D, x / y / z), and for every bra component pair the
// 12 derivative integrals -- six from differentiated bra factors against the
// plain ket sums, six from plain bra factors against the differentiated
// ones.  Accumulators are Cartesian, FP64 atomics, one per (component,
// matrix); the back transform symmetrises.  FP64.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "cqf_deriv.cuh"
#include "cqf_internal.hpp"

namespace cqf {
namespace {

#define CQF_GCUDA(call)                                                                    \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(e_ == cudaErrorMemoryAllocation ? CQF_ENOMEM : CQF_ECUDA,                \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                     \
  } while (0)

constexpr int GRAD_THREADS = 64;
constexpr int GRAD_MAXMAT = 8;  // matrices per call

struct GradLaunch {
  const PairDev* pairs;
  const PrimPairDev* pp;
  const ShellDev* shells;
  const double* prim;
  const double* boys;
  int braBeg, nBra, ketBeg, nKet, same;
  int ncart, nMat;
  int type[GRAD_MAXMAT];  // COULOMB / EXCHANGE
  const int* shellAtom;   // per shell (device)
  const double* Xc;       // nMat Cartesian real densities
  double* Ac;             // (3 natom) x nMat Cartesian accumulators
  int shardIdx, shardCnt;
  unsigned long long* counters;
};

template <int LM>
__global__ void __launch_bounds__(GRAD_THREADS)
    grad_kernel(const GradLaunch a, int la, int lb, int lc, int ld, int nsplit) {
  const int ib = blockIdx.x;
  if (!in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) return;  // another shard's bra
  const int split = blockIdx.y % nsplit;
  const int jk = (blockIdx.y / nsplit) * GRAD_THREADS + threadIdx.x;
  const bool visited = jk < a.nKet && !(a.same && jk > ib);
  if (split == 0) {
    const unsigned mask = __activemask();
    const unsigned bv = __ballot_sync(mask, visited);
    if ((int)(threadIdx.x & 31) == __ffs(mask) - 1 && bv) {
      atomicAdd(a.counters + 0, (unsigned long long)__popc(bv));
      atomicAdd(a.counters + 3, (unsigned long long)__popc(bv));
    }
  }
  if (!visited) return;
  const PairDev P = a.pairs[a.braBeg + ib];
  const PairDev Q = a.pairs[a.ketBeg + jk];

  constexpr int NCL = ncart(LM);
  constexpr int E1 = (LM + 2) * (LM + 2) * (2 * LM + 3);
  constexpr int HB = nherm(2 * LM + 1);
  constexpr int HL = nherm(4 * LM + 1);
  constexpr int FL = 2 * LM + 3;
  const int na = ncart(la), nb = ncart(lb), ncc = ncart(lc), nd = ncart(ld);
  const int nab = na * nb;
  const ShellDev SA = a.shells[P.shA], SB = a.shells[P.shB];
  const ShellDev SC = a.shells[Q.shA], SD = a.shells[Q.shB];
  const int Lb = la + lb + 1, Lk = lc + ld + 1, L = la + lb + lc + ld + 1;
  // the reference's orientation: (s1 s2 | s3 s4) with (s1, s2) the pair
  // later in its loop order; its degeneracy (direct.hpp:2365-2398), and
  // d/dA = -d/dr
  const bool pRef = P.lex >= Q.lex;
  const PairDev& R12 = pRef ? P : Q;
  const PairDev& R34 = pRef ? Q : P;
  const double deg = (R12.s1 == R12.s2 ? 1.0 : 2.0) * (R34.s1 == R34.s2 ? 1.0 : 2.0) *
                     ((R12.s1 == R34.s1) ? (R12.s2 == R34.s2 ? 1.0 : 2.0) : 2.0);
  const double f = -0.5 * deg;
  // atom of each differentiated centre: A, B, C, D
  const int atom[4] = {__ldg(a.shellAtom + P.shA), __ldg(a.shellAtom + P.shB),
                       __ldg(a.shellAtom + Q.shA), __ldg(a.shellAtom + Q.shB)};
  const size_t nc = a.ncart, nc2 = nc * nc;

  double Ea[3][E1], Ec[3][E1];
  double G[7][HB];  // plain ket, then d/dC x y z, d/dD x y z
  double Rv[HL];
  double F[4 * LM + 3];
  double acc[NCL * NCL * 12];  // [ab][centre * 3 + xyz]
  double fa[3][3][FL], fc[3][3][FL];
  int nfa[3][3], nfc[3][3];

#pragma unroll 1
  for (int cd = split; cd < ncc * nd; cd += nsplit) {
    const int c = cd / nd, d = cd % nd;
    const int ci[3] = {cart_lx(lc, c), cart_ly(lc, c), cart_lz(lc, c)};
    const int di[3] = {cart_lx(ld, d), cart_ly(ld, d), cart_lz(ld, d)};
#pragma unroll 1
    for (int k = 0; k < nab * 12; k++) acc[k] = 0.0;
#pragma unroll 1
    for (int ip = 0; ip < P.npp; ip++) {
      const PrimPairDev& A = a.pp[P.pp_off + ip];
      double ea, eb;
      pair_exps(SA, SB, a.prim, A, ea, eb);
#pragma unroll 1
      for (int x = 0; x < 3; x++)
        hermite_E_rt<double, LM + 1>(la + 1, lb + 1, A.o2p, A.PA[x], A.PB[x], Ea[x]);
#pragma unroll 1
      for (int k = 0; k < 7; k++)
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
        const double pref = PI52X2 / sqrt(pq) * A.Kp * Bq.Kp;
        boys_rt<double>(L, alpha * (X * X + Y * Y + Z * Z), F, a.boys);
        hermite_R_rt<double>(L, alpha, X, Y, Z, F, Rv);
#pragma unroll 1
        for (int x = 0; x < 3; x++)
#pragma unroll 1
          for (int ty = 0; ty < 3; ty++) {
            nfc[x][ty] = axis_factor<double>(Ec[x], ld + 1, lc + ld + 3, ci[x], di[x], ty,
                                             2.0 * ec, 2.0 * ed, fc[x][ty]);
#pragma unroll 1
            for (int t = 1; t < nfc[x][ty]; t += 2) fc[x][ty][t] = -fc[x][ty][t];
          }
        // plain ket (the bra derivatives need only Lb - 1 < Lb Hermite orders)
        ket_add<double>(G[0], pref, fc[0][0], nfc[0][0], fc[1][0], nfc[1][0], fc[2][0],
                        nfc[2][0], Lb, Rv);
#pragma unroll 1
        for (int k = 0; k < 6; k++) {
          const int side = k / 3, dir = k % 3;  // 0: C, 1: D
          const int tx = dir == 0 ? 1 + side : 0, ty = dir == 1 ? 1 + side : 0,
                    tz = dir == 2 ? 1 + side : 0;
          ket_add<double>(G[1 + k], pref, fc[0][tx], nfc[0][tx], fc[1][ty], nfc[1][ty],
                          fc[2][tz], nfc[2][tz], Lb - 1, Rv);
        }
      }
#pragma unroll 1
      for (int ab = 0; ab < nab; ab++) {
        const int ai = ab / nb, bi = ab % nb;
        const int ax[3] = {cart_lx(la, ai), cart_ly(la, ai), cart_lz(la, ai)};
        const int bx[3] = {cart_lx(lb, bi), cart_ly(lb, bi), cart_lz(lb, bi)};
#pragma unroll 1
        for (int x = 0; x < 3; x++)
#pragma unroll 1
          for (int ty = 0; ty < 3; ty++)
            nfa[x][ty] = axis_factor<double>(Ea[x], lb + 1, la + lb + 3, ax[x], bx[x], ty,
                                             2.0 * ea, 2.0 * eb, fa[x][ty]);
        double* m = acc + ab * 12;
#pragma unroll 1
        for (int k = 0; k < 6; k++) {  // d/dr on A or B against the plain ket
          const int side = k / 3, dir = k % 3;
          const int tx = dir == 0 ? 1 + side : 0, ty = dir == 1 ? 1 + side : 0,
                    tz = dir == 2 ? 1 + side : 0;
          m[k] += bra_dot<double>(fa[0][tx], nfa[0][tx], fa[1][ty], nfa[1][ty], fa[2][tz],
                                  nfa[2][tz], G[0]);
        }
#pragma unroll 1
        for (int k = 0; k < 6; k++)  // plain bra against d/dr on C or D
          m[6 + k] += bra_dot<double>(fa[0][0], nfa[0][0], fa[1][0], nfa[1][0], fa[2][0],
                                      nfa[2][0], G[1 + k]);
      }
    }
    // digestion at the reference's update sites (direct.hpp:2470-2520)
    const int gC = Q.cA + c, gD = Q.cB + d;
#pragma unroll 1
    for (int ab = 0; ab < nab; ab++) {
      const int gA = P.cA + ab / nb, gB = P.cB + ab % nb;
      // Cartesian AO index of the function of shells s1..s4 (a pair with
      // s1 == s2 maps shA to s1)
      const int pa1 = (P.s1 == P.shA) ? gA : gB, pa2 = (P.s1 == P.shA) ? gB : gA;
      const int qa1 = (Q.s1 == Q.shA) ? gC : gD, qa2 = (Q.s1 == Q.shA) ? gD : gC;
      const int b1 = pRef ? pa1 : qa1, b2 = pRef ? pa2 : qa2;
      const int b3 = pRef ? qa1 : pa1, b4 = pRef ? qa2 : pa2;
      const double* m = acc + ab * 12;
#pragma unroll 1
      for (int k = 0; k < 12; k++) {
        const double v = f * m[k];
        if (v == 0.0) continue;
        const int g = atom[k / 3] * 3 + k % 3;
#pragma unroll 1
        for (int mt = 0; mt < a.nMat; mt++) {
          const double* X = a.Xc + (size_t)mt * nc2;
          double* A = a.Ac + ((size_t)g * a.nMat + mt) * nc2;
          auto x = [&](int r, int cc) { return __ldg(X + r + (size_t)cc * nc); };
          if (a.type[mt] == CQF_COULOMB) {
            atomicAdd(A + b1 + (size_t)b2 * nc, x(b4, b3) * v);
            atomicAdd(A + b4 + (size_t)b3 * nc, x(b1, b2) * v);
          } else {
            atomicAdd(A + b1 + (size_t)b3 * nc, 0.5 * x(b4, b2) * v);
            atomicAdd(A + b4 + (size_t)b2 * nc, 0.5 * x(b3, b1) * v);
            atomicAdd(A + b4 + (size_t)b1 * nc, 0.5 * x(b3, b2) * v);
            atomicAdd(A + b2 + (size_t)b3 * nc, 0.5 * x(b4, b1) * v);
          }
        }
      }
    }
  }
}

void launch_grad(const GradLaunch& a, int la, int lb, int lc, int ld, cudaStream_t st) {
  if (a.nBra == 0 || a.nKet == 0) return;
  const int tiles = (a.nKet + GRAD_THREADS - 1) / GRAD_THREADS;
  const long long quartets = (long long)a.nBra * a.nKet;
  const int ncd = ncart(lc) * ncart(ld);
  int nsplit = (int)std::min<long long>(ncd, std::max<long long>(1, (1 << 18) / quartets));
  nsplit = std::max(1, std::min(nsplit, 65535 / tiles));
  dim3 grid(a.nBra, tiles * nsplit);
  const int lm = std::max(std::max(la, lb), std::max(lc, ld));
  if (lm <= 1) grad_kernel<1><<<grid, GRAD_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit);
  else if (lm == 2) grad_kernel<2><<<grid, GRAD_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit);
  else grad_kernel<3><<<grid, GRAD_THREADS, 0, st>>>(a, la, lb, lc, ld, nsplit);
}

}  // namespace
}  // namespace cqf

using namespace cqf;

extern "C" {

cqf_status cqf_grad_two_body_contract(cqf_basis* B, const int* shell_atom, int natom,
                                      const cqf_contraction* list, int nMat, void* const* AX,
                                      const cqf_opts* optsIn, cqf_stats* stats) {
  if (!B || !shell_atom || !list || !AX || natom < 1 || nMat < 1)
    return fail(CQF_EINVAL, "cqf_grad_two_body_contract: null or empty argument");
  if (nMat > GRAD_MAXMAT)
    return fail(CQF_EINVAL, "cqf_grad_two_body_contract: at most 8 matrices per call");
  cqf_opts o;
  cqf_opts_default(&o);
  if (optsIn) o = *optsIn;
  if (o.is_complex)
    return fail(CQF_EINVAL, "cqf_grad_two_body_contract: complex densities are not built");
  if (o.shard_count < 1 || o.shard_index < 0 || o.shard_index >= o.shard_count)
    return fail(CQF_EINVAL, "shard_index must lie in [0, shard_count)");
  for (int m = 0; m < nMat; m++) {
    if (!list[m].X) return fail(CQF_EINVAL, "cqf_grad_two_body_contract: null X");
    // the reference stops on non-Hermitian gradient contractions (:2539-2541)
    if (!list[m].hermitian)
      return fail(CQF_EINVAL, "cqf_grad_two_body_contract: non-Hermitian X is not built");
    if (list[m].type != CQF_COULOMB && list[m].type != CQF_EXCHANGE)
      return fail(CQF_EINVAL, "cqf_grad_two_body_contract: COULOMB or EXCHANGE only");
  }
  const int nGrad = 3 * natom;
  for (int k = 0; k < nGrad * nMat; k++)
    if (!AX[k]) return fail(CQF_EINVAL, "cqf_grad_two_body_contract: null AX");
  for (int s = 0; s < B->nshell; s++)
    if (shell_atom[s] < 0 || shell_atom[s] >= natom)
      return fail(CQF_EINVAL, "cqf_grad_two_body_contract: shell_atom outside [0, natom)");
  std::lock_guard<std::mutex> lk(B->mu);
  CQF_GCUDA(cudaSetDevice(B->device));
  cudaStream_t st = o.stream ? (cudaStream_t)o.stream : B->stream;
  const int N = B->nbasis, nc = B->ncart;
  const size_t NN = (size_t)N * N, nc2 = (size_t)nc * nc;
  // scratch (stream-ordered): shell atoms | Cartesian X | Cartesian
  // accumulators | host staging of X and AX
  const size_t host = o.device_pointers ? 0 : (size_t)nMat * NN + (size_t)nGrad * nMat * NN;
  const size_t doubles = (size_t)nMat * nc2 + (size_t)nGrad * nMat * nc2 + host;
  double* ws = nullptr;
  int* dAtom = nullptr;
  CQF_GCUDA(cudaMallocAsync(&ws, doubles * sizeof(double), st));
  CQF_GCUDA(cudaMallocAsync(&dAtom, (size_t)B->nshell * sizeof(int), st));
  double* Xc = ws;
  double* Ac = Xc + (size_t)nMat * nc2;
  double* hX = Ac + (size_t)nGrad * nMat * nc2;
  double* hAX = hX + (size_t)nMat * NN;
  CQF_GCUDA(cudaMemcpyAsync(dAtom, shell_atom, (size_t)B->nshell * sizeof(int),
                            cudaMemcpyHostToDevice, st));
  for (int m = 0; m < nMat; m++) {
    const double* X = static_cast<const double*>(list[m].X);
    if (!o.device_pointers) {
      CQF_GCUDA(cudaMemcpyAsync(hX + (size_t)m * NN, X, NN * sizeof(double),
                                cudaMemcpyHostToDevice, st));
      X = hX + (size_t)m * NN;
    }
    launch_to_cart(B, X, 0, Xc + (size_t)m * nc2, st);
  }
  CQF_GCUDA(cudaMemsetAsync(Ac, 0, (size_t)nGrad * nMat * nc2 * sizeof(double), st));
  CQF_GCUDA(cudaMemsetAsync(B->d_counters, 0, 4 * sizeof(unsigned long long), st));
  CQF_GCUDA(cudaEventRecord(B->ev0, st));

  GradLaunch a{};
  a.pairs = B->d_pairs;
  a.pp = B->d_pp;
  a.shells = B->d_shells;
  a.prim = B->d_prim;
  a.boys = B->d_boys64;
  a.ncart = nc;
  a.nMat = nMat;
  for (int m = 0; m < nMat; m++) a.type[m] = list[m].type;
  a.shellAtom = dAtom;
  a.Xc = Xc;
  a.Ac = Ac;
  a.shardIdx = o.shard_index;
  a.shardCnt = o.shard_count;
  a.counters = B->d_counters;
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
      launch_grad(a, la, lb, lc, ld, st);
    }
  CQF_GCUDA(cudaGetLastError());
  // AX += 1/2 (A + A^T) per component and matrix (:2550-2560)
  for (int k = 0; k < nGrad * nMat; k++) {
    double* dst = static_cast<double*>(AX[k]);
    if (!o.device_pointers) {
      dst = hAX + (size_t)k * NN;
      CQF_GCUDA(cudaMemcpyAsync(dst, AX[k], NN * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    launch_from_cart(B, Ac + (size_t)k * nc2, 0, 1, dst, st);
  }
  CQF_GCUDA(cudaGetLastError());
  CQF_GCUDA(cudaEventRecord(B->ev1, st));
  if (!o.device_pointers)
    for (int k = 0; k < nGrad * nMat; k++)
      CQF_GCUDA(cudaMemcpyAsync(AX[k], hAX + (size_t)k * NN, NN * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
  unsigned long long h[4];
  CQF_GCUDA(cudaMemcpyAsync(h, B->d_counters, sizeof(h), cudaMemcpyDeviceToHost, st));
  cudaFreeAsync(ws, st);
  cudaFreeAsync(dAtom, st);
  CQF_GCUDA(cudaStreamSynchronize(st));
  if (stats) {
    stats->quartets_total = (long long)h[0];
    stats->quartets_screened = 0;
    stats->quartets_fp32 = 0;
    stats->quartets_fp64 = (long long)h[3];
    float ms = 0.f;
    cudaEventElapsedTime(&ms, B->ev0, B->ev1);
    stats->device_ms = ms;
  }
  return CQF_OK;
}

}  // extern "C"
