// Host-side internals shared by the translation units of libcqfock.so.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "../../include/cqfock.h"
#include "cqf_common.cuh"

namespace cqf {

constexpr int NCLS = (LMAX + 1) * (LMAX + 2) / 2;  // pair classes (lA >= lB)
inline int class_id(int la, int lb) { return la * (la + 1) / 2 + lb; }
inline void class_ls(int c, int& la, int& lb) {
  la = 0;
  while ((la + 1) * (la + 2) / 2 <= c) la++;
  lb = c - la * (la + 1) / 2;
}

// Per-matrix flags packed for the kernels: bit0 HER, bit1 EXCHANGE.
constexpr int MAXMAT = 512;

// Tile-interleaved ket primitive data: fields p, Kp, o2p, P[3], PA[3], PB[3],
// Qp (primitive Schwarz bound) of KETT_TILE consecutive kets of a class.
constexpr int NAUX = 2;           // auxiliary streams of the class-quartet launches
constexpr int NSTAGE = 8;         // pieces of a host-pointer download (one event each)
constexpr int KETT_NF = 13;
constexpr int KETT_TILE = 128;
constexpr int WTILE = 32;         // kets per mask word of the class kernels

// Arguments of one class-quartet J/K launch.
struct JKLaunch {
  const PairDev* pairs;
  const PrimPairDev* pp;
  const double* boys64;
  const float* boys32;
  int braBeg, nBra, ketBeg, nKet, same;
  int screen;
  double thresh;
  const double* norms;      // max over matrices, nshell x nshell (col-major)
  const double* normsMat;   // nMat x nshell x nshell (only read when nMat > 1)
  const double* maxNorm;    // device scalar: max of norms (tile-level screen)
  const double* normsT;     // transpose of norms
  const double* pairNorm;   // per pair (pair order): norms(s1, s2)
  const float2* pairRange;  // per pair: FP32 range data (fp32_range_ok)
  int nShell;
  int nMat, cplx, ncart;
  const int* flags;         // nMat flags (device)
  const double* Xc;         // nMat x ncart x ncart (complex: interleaved)
  double* Ac;               // same shape, accumulated
  // ket primitive pairs, tile-interleaved (structure of arrays): field f of
  // primitive iq of the ket at tile position l is
  // ketT[tileOff[ketTileBeg + tile] + (iq * KETT_NF + f) * KETT_TILE + l]
  const double* ketT;
  const float* ketT32;      // FP32 copy of ketT (same offsets)
  const PrimPair32* pp32;   // FP32 copy of pp
  const long long* tileOff;
  int braTileBeg, ketTileBeg;
  const float* Xc32;        // FP32 copy of Xc (mixed builds, FP32 class kernels)
  const double* ppQ;        // primitive Schwarz bound of each primitive pair
  const double* qWin;       // per pair: largest Q of the WTILE pairs from it (same class)
  double primK4;            // (largest contraction length)^4 of the basis
  int lsum;                 // la + lb + lc + ld of the launch's class
  int braOff;               // position of the launch's first bra pair in its class (slabs)
  int precision;            // 0 FP64, 1 mixed
  double fp32_cut;          // mixed: bound < cut -> FP32 ERIs
  int shardIdx, shardCnt;   // bra pairs p with p % shardCnt == shardIdx only
  unsigned long long* counters;  // [0] visited, [1] screened, [2] fp32, [3] fp64
};

// Whether bra pair p (position in the pair list) belongs to this call's
// shard of the work (cqf_opts::shard_index / shard_count).
__host__ __device__ inline bool in_shard(int p, int idx, int cnt) {
  return cnt <= 1 || p % cnt == idx;
}

// Sets the thread's last-error text and returns s (cqf_api.cu).
cqf_status fail(cqf_status s, const std::string& msg);

// Workspace layout of one contraction (in doubles, each part 256-B aligned):
// [X copies | AX copies] (host pointers only) | Xc | Ac | norms | normsMat |
// gmax | norms^T | pair norms | work counters | Xc in FP32 (mixed real
// builds) | quartet masks of the fast class kernels (per launch stream a
// region of maskWords uint2 masks, one per bra pair and ket tile, then the
// two lists of non-empty words)
// class-kernel work counters / list lengths: four per launch stream
constexpr int NWORK = 4 * (NAUX + 1);
// mask words a launch stream's region holds at most (16 B per word: the
// uint2 mask and two list entries); class pairs with more run in slabs
constexpr size_t MASK_CAP_WORDS = size_t(1) << 18;
struct WsLayout {
  size_t oX, oAX, oXc, oAc, oNm, oNmM, oG, oNmT, oPN, oWork, oXc32, oMask, total;
  size_t maskWords;  // mask words of each launch stream's region
};
WsLayout ws_layout(const cqf_basis* B, int nMat, const cqf_opts& opts);
cqf_status check_contract_args(const cqf_basis* B, const cqf_contraction* list, int nMat);
// The contraction on a caller-provided device workspace of ws_layout().total
// doubles; the caller holds B->mu and has made B's device current.
// With capture = true nothing synchronises or reads back (stream capture);
// d_flags_pre: per-matrix flags already on the device (else uploaded here).
// A real Coulomb contraction of a non-Hermitian X equals that of its
// symmetric part (J[X] = J[(X + X^T)/2], as (ab|cd) = (ab|dc); the
// reference's non-Hermitian J branch, direct.hpp:1920-1950, symmetrises the
// same way), so it runs as a Hermitian one on the symmetrised Cartesian
// density; the screen keeps the norms of X as given.
inline bool hermitian_eff(const cqf_contraction& c, bool cplx) {
  return c.hermitian || (!cplx && c.type == CQF_COULOMB);
}
// per-matrix kernel flags: bit 0 Hermitian (effective), bit 1 exchange,
// bit 2 real antisymmetric (hermitian = -1: only the library's own split of
// a complex Hermitian density makes such entries)
inline int contraction_flags(const cqf_contraction& c, bool cplx) {
  return (hermitian_eff(c, cplx) ? 1 : 0) | (c.type == CQF_EXCHANGE ? 2 : 0) |
         (c.hermitian < 0 ? 4 : 0);
}

// The caller's contraction list with TwoBodyContraction::HER as the bool it
// is in the reference (twopints.hpp:59-75): any nonzero value becomes 1, so
// a caller's "true" never reaches the library's internal -1 flag (the
// antisymmetric part of a complex split).  *allHer: every entry Hermitian.
std::vector<cqf_contraction> normalized_list(const cqf_contraction* list, int nMat,
                                             bool* allHer);

// Complex Hermitian contractions on the real fast kernels (cqf_api.cu):
// eligibility, real-entry count and flags, workspace, and the pipeline on
// device pointers and a caller-provided workspace (capture-able).
bool split_eligible(const cqf_basis* B, const cqf_contraction* list, int nMat,
                    const cqf_opts& opts);
int split_real_count(const cqf_contraction* list, int nMat);
void split_flags(const cqf_contraction* list, int nMat, int* fl);
size_t split_ws_doubles(const cqf_basis* B, int nReal, const cqf_opts& opts);
cqf_status split_core(cqf_basis* B, const cqf_contraction* list, int nMat, const cqf_opts& opts,
                      cqf_stats* stats, double* ws, bool capture, const int* d_flags_pre);

// The split for device or host pointers on a caller-provided workspace of
// complex_split_ws_doubles() doubles (host pointers are staged in it);
// synchronises before returning.  Caller holds B->mu, device current.
size_t complex_split_ws_doubles(const cqf_basis* B, const cqf_contraction* list, int nMat,
                                const cqf_opts& opts);
cqf_status contract_complex_split_on(cqf_basis* B, const cqf_contraction* list, int nMat,
                                     const cqf_opts& opts, cqf_stats* stats, double* ws);

// normSrc (optional, device pointers): per entry, the complex matrix whose
// shell-block norms screen it in place of its own X (the split of a complex
// Hermitian density keeps the reference's complex screen).
// pinned (host pointers, optional): page-locked host buffer of 2 nMat
// matrices; X goes to the device through it and the contraction's result
// comes back through it and is added to the caller's AX on the host (no
// upload of AX).  Without it the host matrices are copied directly.
cqf_status contract_core(cqf_basis* B, const cqf_contraction* list, int nMat,
                         const cqf_opts& opts, cqf_stats* stats, double* ws, bool capture,
                         const int* d_flags_pre, const double* const* normSrc = nullptr,
                         double* pinned = nullptr);
// Page-locked host staging buffers of host-pointer contractions, shared by
// every basis of the process: acquire returns a buffer of at least `bytes`
// that no other call holds (allocating one only when none fits), release
// returns it.  They are kept until the process exits -- freeing page-locked
// memory synchronises the whole device, which would stall the concurrent
// requests of a server.
cqf_status pinned_acquire(size_t bytes, double** out);
void pinned_release(double* p);

// Resolves the no-alloc scratch array's device address on `device` (current)
// during basis creation (cqf_noalloc.cu).
void noalloc_prepare(int device);

// Launch helpers shared with the four-component path (cqf_api.cu).
// Shell-block infinity norms of one N x N matrix (complex: |z|).
void launch_block_norms(const cqf_basis* B, const double* X, int cplx, double* out,
                        cudaStream_t st);
// out = elementwise max over nMat norm tables; *gmax = max of out (bits).
void launch_max_norms(const double* nm, int nMat, size_t ns2, double* out,
                      unsigned long long* gmax, cudaStream_t st);
// Xc = T X T^T (spherical -> Cartesian AO), real or complex interleaved.
void launch_to_cart(const cqf_basis* B, const double* X, int cplx, double* Xc, cudaStream_t st);
// AX (N x N) += the back transform of the Cartesian accumulator Ac:
// 1/2 (B + B^H) with her = 1, 1/2 B with her = 0 (B = T^T Ac T).
void launch_from_cart(const cqf_basis* B, const double* Ac, int cplx, int her, double* AX,
                      cudaStream_t st);
// Grows the basis' contraction workspace (B->d_ws) to at least `bytes`.
cqf_status basis_workspace(cqf_basis* B, size_t bytes);

}  // namespace cqf

struct cqf_basis {
  int device = 0;
  int nsm = 148;
  cudaStream_t stream = nullptr;
  int nshell = 0, nbasis = 0, ncart = 0, npair = 0, maxL = 0, maxPrim = 0;
  long long nprimpair = 0;
  double thresh = 1e-12;
  std::vector<cqf::ShellDev> h_shells;
  std::vector<cqf::PairDev> h_pairs;     // final (class, npp, Q) order
  int cls_beg[cqf::NCLS] = {0}, cls_cnt[cqf::NCLS] = {0};
  // launch shape of each class pair's persistent kernel: resident blocks per
  // SM requested (8 by default; cqf_autotune measures and sets it)
  int blocks_per_sm[cqf::NCLS][cqf::NCLS];
  // autotuning: when set, contract_core launches the class kernels on one
  // stream with an event pair around each (tune_ev[2 (cb NCLS + ck) + 0/1])
  bool tuning = false;
  std::vector<cudaEvent_t> tune_ev;
  int cls_tile_beg[cqf::NCLS] = {0};    // first ket tile of each class
  std::vector<double> h_schwarz;         // nshell^2
  // device-resident basis data
  cqf::ShellDev* d_shells = nullptr;
  double* d_prim = nullptr;              // alpha | coeff
  cqf::PairDev* d_pairs = nullptr;
  cqf::PrimPairDev* d_pp = nullptr;
  double* d_ppQ = nullptr;               // primitive Schwarz bounds (pp order)
  double* d_qWin = nullptr;              // per pair: window maximum of Q (tile screens)
  double* d_ketT = nullptr;              // tile-interleaved ket primitive data
  float* d_ketT32 = nullptr;             // its FP32 copy (FP32 class kernels)
  cqf::PrimPair32* d_pp32 = nullptr;     // FP32 copy of d_pp
  long long* d_tileOff = nullptr;        // per tile: offset into d_ketT
  float2* d_pairRange = nullptr;         // per pair: FP32 range data
  double* d_boys64 = nullptr;
  float* d_boys32 = nullptr;
  double* d_schwarz = nullptr;
  double* d_sph = nullptr;               // solid-harmonic matrices, all l
  int* d_sphOff = nullptr;               // offset of l's matrix in d_sph
  int* d_ao2shell = nullptr;             // AO (spherical) -> shell
  int* d_cart2shell = nullptr;           // Cartesian AO -> shell
  // per-call workspace (grown on demand)
  size_t ws_bytes = 0;
  void* d_ws = nullptr;
  unsigned long long* d_counters = nullptr;
  int* d_flags = nullptr;                // MAXMAT per-matrix flags
  std::vector<int> h_flags;              // host staging of the flags
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t evStage[cqf::NSTAGE] = {};  // host-pointer downloads, piece by piece
  // class-quartet kernels are spread over the call's stream and these NAUX
  // (fork / join by events) so that each persistent launch's tail overlaps
  // the next one's start; the streams come from a per-device pool
  cudaStream_t aux[cqf::NAUX] = {};
  cudaEvent_t evFork = nullptr, evJoin[cqf::NAUX] = {};
  // four-component path: Schwarz tables (computed on first use, nshell^2
  // each, zero for pairs outside the significant-pair list) and workspace
  double* d_qLL = nullptr;
  double* d_qSS = nullptr;
  double* d_qG = nullptr;  // Gaunt: qG[d + o * nshell], derivative on shell d
  double* d_qB = nullptr;  // gauge, the same layout
  bool rel_qLL = false, rel_qSS = false, rel_qG = false, rel_qB = false;
  void* d_relws = nullptr;
  size_t relws_bytes = 0;
  std::mutex mu;
};
