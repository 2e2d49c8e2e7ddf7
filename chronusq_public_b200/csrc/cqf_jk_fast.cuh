// Closed-shell fast path: real densities flagged Hermitian (symmetric), every
// shell l <= 2.  One thread per unique quartet, generated straight-line
// McMurchie-Davidson code per class (gen/cqf_gen_jk.cuh), FP64 or FP32
// primitive arithmetic chosen per launch, FP64 accumulation.
//
// Screening, unique-quartet set and degeneracy are those of the generic
// kernel (cqf_jk_kernels.cuh); the digestion uses the canonical quartet order
// instead of the reference's shell roles, which gives the same J and K after
// the final 1/2 (A + A^T) when X is symmetric.
#pragma once

#include "cqf_jk_kernels.cuh"
#include "gen/cqf_gen_jk.cuh"

#include <algorithm>

namespace cqf {

static_assert(JK_THREADS == KETT_TILE, "a ket tile is one block of kets");

template <int N>
__device__ __forceinline__ void warp_sum(double (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N; i++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
  }
}

// Ket primitive-pair data of one quartet for the generated eri():
// KetAoS reads the PrimPairDev records of the pair (any pair order);
// KetSoA reads the tile-interleaved copy, where the 128 kets of a tile have
// each field of primitive iq contiguous (a warp's load is one coalesced run).
struct KetAoS {
  const PrimPairDev* b;
  __device__ __forceinline__ double p(int iq) const { return b[iq].p; }
  __device__ __forceinline__ double Kp(int iq) const { return b[iq].Kp; }
  __device__ __forceinline__ double o2p(int iq) const { return b[iq].o2p; }
  __device__ __forceinline__ double P(int iq, int x) const { return b[iq].P[x]; }
  __device__ __forceinline__ double PA(int iq, int x) const { return b[iq].PA[x]; }
  __device__ __forceinline__ double PB(int iq, int x) const { return b[iq].PB[x]; }
};
struct KetSoA {
  const double* q;  // tile base + lane
  __device__ __forceinline__ double f(int iq, int k) const {
    return __ldg(q + (iq * KETT_NF + k) * KETT_TILE);
  }
  __device__ __forceinline__ double p(int iq) const { return f(iq, 0); }
  __device__ __forceinline__ double Kp(int iq) const { return f(iq, 1); }
  __device__ __forceinline__ double o2p(int iq) const { return f(iq, 2); }
  __device__ __forceinline__ double P(int iq, int x) const { return f(iq, 3 + x); }
  __device__ __forceinline__ double PA(int iq, int x) const { return f(iq, 6 + x); }
  __device__ __forceinline__ double PB(int iq, int x) const { return f(iq, 9 + x); }
};

// Rows of the Boys tables for angular sum L (global memory).
template <typename T>
__device__ __forceinline__ const T* boys_rows(const JKLaunch& a, int L);
template <>
__device__ __forceinline__ const double* boys_rows<double>(const JKLaunch& a, int L) {
  return a.boys64 + (size_t)L * BOYS_NPTS * BOYS_ROW64;
}
template <>
__device__ __forceinline__ const float* boys_rows<float>(const JKLaunch& a, int L) {
  return a.boys32 + (size_t)L * BOYS_NPTS * BOYS_ROW32;
}

// Persistent class kernel.  Every warp independently takes work items (bra
// pair, chunk, ket tile of 32) from a device counter until none are left --
// no block barriers.  The Boys rows of the class's angular sum (29 KB FP64,
// 12 KB FP32) are read from global memory through L1: staging them in shared
// memory capped residency at 6 blocks per SM and measured slower.  On the mixed path a warp computes its
// quartets in FP32 when every surviving quartet's bound is below the cut
// and in FP64 otherwise (kets are sorted by Schwarz bound, so the warps of
// a bra row switch from FP64 to FP32 once), in one traversal.
constexpr int WTILE = 32;  // kets per work item (one warp)

// Shell-block norm maximum of a quartet in the reference's roles
// (direct.hpp:1693-1736), with the warp-uniform bra pair P: the pair norms
// come from the per-pair array, and the four cross terms are read from the
// column of a bra shell (normsT holds the transpose), so a warp's lanes read
// one column instead of 32 scattered ones.
__device__ __forceinline__ double sh_max_bra(const JKLaunch& a, const PairDev& P,
                                             const PairDev& Q, double nP, double nQ,
                                             bool pRef) {
  const int ns = a.nShell;
  double m;
  if (pRef) {  // rows from P (uniform): B(r, c) = normsT[c + r ns]
    const double* c1 = a.normsT + (size_t)P.s1 * ns;
    const double* c2 = a.normsT + (size_t)P.s2 * ns;
    m = fmax(fmax(__ldg(c1 + Q.s1), __ldg(c2 + Q.s1)), fmax(__ldg(c1 + Q.s2), __ldg(c2 + Q.s2)));
  } else {     // rows from Q, columns from P (uniform): B(r, c) = norms[r + c ns]
    const double* c1 = a.norms + (size_t)P.s1 * ns;
    const double* c2 = a.norms + (size_t)P.s2 * ns;
    m = fmax(fmax(__ldg(c1 + Q.s1), __ldg(c1 + Q.s2)), fmax(__ldg(c2 + Q.s1), __ldg(c2 + Q.s2)));
  }
  return fmax(m, fmax(nP, nQ));
}

template <class G64, class G32, bool MIXED>
__global__ void __launch_bounds__(JK_THREADS, G64::MINB)
    jk_fast_kernel(const JKLaunch a, unsigned int* __restrict__ work) {
  static_assert(G64::NCHUNK == G32::NCHUNK && G64::NI == G32::NI, "shared chunking");
  constexpr int NA = ncart(G64::LA), NB = ncart(G64::LB);
  constexpr int NCH = G64::NCHUNK;
  constexpr int LSUM = G64::LA + G64::LB + G64::LC + G64::LD;
  const double cut = MIXED ? a.fp32_cut : 0.0;
  constexpr bool mixed = MIXED;
  const double* boys64 = boys_rows<double>(a, LSUM);
  const float* boys32 = boys_rows<float>(a, LSUM);
  const int lane = threadIdx.x & 31;
  const int ketTiles = (a.nKet + WTILE - 1) / WTILE;
  const long long perBra = (long long)ketTiles * NCH;
  const long long total = (long long)a.nBra * perBra;
  const size_t nc = a.ncart;
  const size_t matStride = (size_t)a.ncart * a.ncart;
  // quartet counts of this warp, flushed once at exit
  unsigned long long cVis = 0, cScr = 0, c32 = 0, c64 = 0;

  for (;;) {
    unsigned int itemU = 0;
    if (lane == 0) itemU = atomicAdd(work, 1u);
    const long long item = (long long)__shfl_sync(0xffffffffu, itemU, 0);
    if (item >= total) break;
    const int ib = (int)(item / perBra);
    const int rem = (int)(item % perBra);
    const int ch = rem / ketTiles, tile = rem % ketTiles;
    // same class: each unordered pair {P, Q} once, as ket position <= bra
    // position (roles still follow the lex order)
    if (a.same && tile * WTILE > ib) continue;
    const int jk = tile * WTILE + lane;
    const PairDev P = a.pairs[a.braBeg + ib];
    bool visited = false, screened = false, w64 = false, w32 = false;
    PairDev Q;
    if (jk < a.nKet && !(a.same && jk > ib)) {
      Q = a.pairs[a.ketBeg + jk];
      visited = true;
    }
    const bool counter = ch == 0;  // one count per quartet
    const double tileMax = __ldg(a.maxNorm) * P.Q * a.pairs[a.ketBeg + tile * WTILE].Q;
    if (a.screen && tileMax < a.thresh) {
      if (counter) {
        const unsigned bv = __ballot_sync(0xffffffffu, visited);
        cVis += __popc(bv);
        cScr += __popc(bv);
      }
      continue;
    }
    int s1 = 0, s2 = 0, s3 = 0, s4 = 0;
    if (visited) {
      const bool pRef = P.lex >= Q.lex;
      const PairDev& R12 = pRef ? P : Q;
      const PairDev& R34 = pRef ? Q : P;
      s1 = R12.s1; s2 = R12.s2; s3 = R34.s1; s4 = R34.s2;
      double bound = 1e300;
      if (a.screen) {
        bound = sh_max_bra(a, P, Q, __ldg(a.pairNorm + a.braBeg + ib),
                           __ldg(a.pairNorm + a.ketBeg + jk), pRef) * P.Q * Q.Q;
        screened = bound < a.thresh;
      }
      w64 = !screened;
      w32 = w64 && mixed && bound < cut &&
            fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib), __ldg(a.pairRange + a.ketBeg + jk),
                          LSUM, 0, 0);
    }
    // one precision per warp: FP32 only when every surviving quartet of the
    // warp is below the cut (no divergent FP64 / FP32 code in a warp)
    if (__any_sync(0xffffffffu, w64 && !w32)) {
      w32 = false;
    } else {
      w64 = w64 && !w32;
    }
    const unsigned b64 = __ballot_sync(0xffffffffu, w64);
    const unsigned b32 = __ballot_sync(0xffffffffu, w32);
    if (counter) {
      cVis += __popc(__ballot_sync(0xffffffffu, visited));
      cScr += __popc(__ballot_sync(0xffffffffu, screened));
      c64 += __popc(b64);
      c32 += __popc(b32);
    }
    if (!(b64 | b32)) continue;
    const bool work_ = w64 || w32;

    const double deg = ((s1 == s2) ? 1.0 : 2.0) * ((s3 == s4) ? 1.0 : 2.0) *
                       ((s1 == s3 && s2 == s4) ? 1.0 : 2.0);
    const double sJ = work_ ? 0.5 * deg : 0.0, sK = work_ ? 0.25 * deg : 0.0;
    double I[G64::NI];
    const KetSoA kq{a.ketT + __ldg(a.tileOff + a.ketTileBeg + jk / KETT_TILE) + jk % KETT_TILE};
    if (w64) {
      G64::template eri<double>(P, Q, a.pp, kq, boys64, ch, I);
    } else if (MIXED && w32) {
      G32::template eri<float>(P, Q, a.pp, kq, boys32, ch, I);
    } else {
#pragma unroll
      for (int i = 0; i < G64::NI; i++) I[i] = 0.0;
    }
#pragma unroll 1
    for (int m = 0; m < a.nMat; m++) {
      const int fl = __ldg(a.flags + m);
      const bool doJ = !(fl & 2), doK = (fl & 2);
      double jab[NA * NB];
#pragma unroll
      for (int i = 0; i < NA * NB; i++) jab[i] = 0.0;
      const double* X = a.Xc + m * matStride;
      double* A = a.Ac + m * matStride;
      G64::digest(I, ch, X, A, nc, P.cA, P.cB, Q.cA, Q.cB, sJ, sK, (fl & 4) ? -sK : sK,
                  doJ && work_, doK && work_,
                  jab);
      if (doJ) {
        // every lane of the warp shares the bra pair: reduce, one atomic each
#pragma unroll
        for (int i = 0; i < NA * NB; i++) jab[i] *= sJ;
        warp_sum(jab);
        if (lane == 0) {
#pragma unroll
          for (int i = 0; i < NA * NB; i++)
            if (jab[i] != 0.0)
              atomicAdd(A + (size_t)(P.cA + i / NB) + (size_t)(P.cB + i % NB) * nc, jab[i]);
        }
      }
    }
  }
  if (lane == 0) {
    if (cVis) atomicAdd(a.counters + 0, cVis);
    if (cScr) atomicAdd(a.counters + 1, cScr);
    if (c32) atomicAdd(a.counters + 2, c32);
    if (c64) atomicAdd(a.counters + 3, c64);
  }
}

// Grouped variant for the light single-chunk classes (G64::GROUPED): a work
// item is (bra group, ket tile of 32); the group's bra pairs share their
// first shell A, so each lane's updates J_cd, K_ac and K_ad (targets fixed by
// its ket pair and by A) are summed in registers over the whole group and
// flushed once -- fewer atomics than one flush per quartet.  Launched when
// the call has one J and one K matrix (else jk_fast_kernel runs; the
// per-matrix flush below keeps the kernel correct for any matrix list).
// Quartet set, screens, roles, degeneracy and precision choice are those of
// jk_fast_kernel.
template <class G64, class G32, bool MIXED>
__global__ void __launch_bounds__(JK_THREADS, G64::MINB)
    jk_group_kernel(const JKLaunch a, unsigned int* __restrict__ work) {
  static_assert(G64::NCHUNK == 1 && G32::NCHUNK == 1, "single-chunk classes");
  constexpr int NA = ncart(G64::LA), NB = ncart(G64::LB);
  constexpr int NC = ncart(G64::LC), ND = ncart(G64::LD);
  constexpr int LSUM = G64::LA + G64::LB + G64::LC + G64::LD;
  const double cut = MIXED ? a.fp32_cut : 0.0;
  const double* boys64 = boys_rows<double>(a, LSUM);
  const float* boys32 = boys_rows<float>(a, LSUM);
  const int lane = threadIdx.x & 31;
  const int ketTiles = (a.nKet + WTILE - 1) / WTILE;
  const long long total = (long long)a.braNGroups * ketTiles;
  const size_t nc = a.ncart;
  const size_t matStride = (size_t)a.ncart * a.ncart;
  const bool grouped = a.jmat >= 0;
  unsigned long long cVis = 0, cScr = 0, c32 = 0, c64 = 0;

  for (;;) {
    unsigned int itemU = 0;
    if (lane == 0) itemU = atomicAdd(work, 1u);
    const long long item = (long long)__shfl_sync(0xffffffffu, itemU, 0);
    if (item >= total) break;
    const int g = (int)(item / ketTiles), tile = (int)(item % ketTiles);
    const int2 gr = __ldg(a.groups + a.braGroupBeg + g);
    const int jk = tile * WTILE + lane;
    const bool qvalid = jk < a.nKet;
    PairDev Q;
    if (qvalid) Q = a.pairs[a.ketBeg + jk];
    const double tileQ = a.pairs[a.ketBeg + tile * WTILE].Q;
    double jcd[G64::NJCD], kac[G64::NKAC], kad[G64::NKAD];
#pragma unroll
    for (int i = 0; i < G64::NJCD; i++) jcd[i] = 0.0;
#pragma unroll
    for (int i = 0; i < G64::NKAC; i++) kac[i] = 0.0;
#pragma unroll
    for (int i = 0; i < G64::NKAD; i++) kad[i] = 0.0;
    int cAgrp = 0;
    bool any = false;

#pragma unroll 1
    for (int mm = 0; mm < gr.y; mm++) {
      const int ib = __ldg(a.braPerm + a.braBeg + gr.x + mm);  // position in the class
      if (a.same && tile * WTILE > ib) continue;  // warp-uniform
      const PairDev P = a.pairs[a.braBeg + ib];
      const bool visited = qvalid && !(a.same && jk > ib);
      if (a.screen && __ldg(a.maxNorm) * P.Q * tileQ < a.thresh) {
        const unsigned bv = __ballot_sync(0xffffffffu, visited);
        cVis += __popc(bv);
        cScr += __popc(bv);
        continue;
      }
      bool screened = false, w64 = false, w32 = false;
      int s1 = 0, s2 = 0, s3 = 0, s4 = 0;
      if (visited) {
        const bool pRef = P.lex >= Q.lex;
        const PairDev& R12 = pRef ? P : Q;
        const PairDev& R34 = pRef ? Q : P;
        s1 = R12.s1; s2 = R12.s2; s3 = R34.s1; s4 = R34.s2;
        double bound = 1e300;
        if (a.screen) {
          bound = sh_max_bra(a, P, Q, __ldg(a.pairNorm + a.braBeg + ib),
                             __ldg(a.pairNorm + a.ketBeg + jk), pRef) * P.Q * Q.Q;
          screened = bound < a.thresh;
        }
        w64 = !screened;
        w32 = w64 && MIXED && bound < cut &&
              fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib),
                            __ldg(a.pairRange + a.ketBeg + jk), LSUM, 0, 0);
      }
      if (__any_sync(0xffffffffu, w64 && !w32)) w32 = false;
      else w64 = w64 && !w32;
      const unsigned b64 = __ballot_sync(0xffffffffu, w64);
      const unsigned b32 = __ballot_sync(0xffffffffu, w32);
      cVis += __popc(__ballot_sync(0xffffffffu, visited));
      cScr += __popc(__ballot_sync(0xffffffffu, screened));
      c64 += __popc(b64);
      c32 += __popc(b32);
      if (!(b64 | b32)) continue;
      const bool work_ = w64 || w32;
      cAgrp = P.cA;
      any = any || work_;
      const double deg = ((s1 == s2) ? 1.0 : 2.0) * ((s3 == s4) ? 1.0 : 2.0) *
                         ((s1 == s3 && s2 == s4) ? 1.0 : 2.0);
      const double sJ = work_ ? 0.5 * deg : 0.0, sK = work_ ? 0.25 * deg : 0.0;
      double I[G64::NI];
      if (w64) {
        const KetSoA kq{a.ketT + __ldg(a.tileOff + a.ketTileBeg + jk / KETT_TILE) + jk % KETT_TILE};
        G64::template eri<double>(P, Q, a.pp, kq, boys64, 0, I);
      } else if (MIXED && w32) {
        const KetSoA kq{a.ketT + __ldg(a.tileOff + a.ketTileBeg + jk / KETT_TILE) + jk % KETT_TILE};
        G32::template eri<float>(P, Q, a.pp, kq, boys32, 0, I);
      } else {
#pragma unroll
        for (int i = 0; i < G64::NI; i++) I[i] = 0.0;
      }
#pragma unroll 1
      for (int m = 0; m < a.nMat; m++) {
        const int fl = __ldg(a.flags + m);
        const bool doJ = !(fl & 2), doK = (fl & 2);
        double jab[NA * NB];
#pragma unroll
        for (int i = 0; i < NA * NB; i++) jab[i] = 0.0;
        const double* X = a.Xc + m * matStride;
        double* A = a.Ac + m * matStride;
        G64::digest_g(I, X, A, nc, P.cA, P.cB, Q.cA, Q.cB, sJ, sK, (fl & 4) ? -sK : sK,
                      doJ && work_, doK && work_,
                      jab, jcd, kac, kad);
        if (!grouped && work_) {  // flush this matrix's sums now
#pragma unroll
          for (int k = 0; k < G64::NJCD; k++) {
            if (jcd[k] != 0.0)
              atomicAdd(A + (size_t)(Q.cA + k / ND) + (size_t)(Q.cB + k % ND) * nc, jcd[k]);
            jcd[k] = 0.0;
          }
#pragma unroll
          for (int k = 0; k < G64::NKAC; k++) {
            if (kac[k] != 0.0)
              atomicAdd(A + (size_t)(Q.cA + k % NC) + (size_t)(P.cA + k / NC) * nc, kac[k]);
            kac[k] = 0.0;
          }
#pragma unroll
          for (int k = 0; k < G64::NKAD; k++) {
            if (kad[k] != 0.0)
              atomicAdd(A + (size_t)(Q.cB + k % ND) + (size_t)(P.cA + k / ND) * nc, kad[k]);
            kad[k] = 0.0;
          }
        }
        if (doJ) {
#pragma unroll
          for (int i = 0; i < NA * NB; i++) jab[i] *= sJ;
          warp_sum(jab);
          if (lane == 0) {
#pragma unroll
            for (int i = 0; i < NA * NB; i++)
              if (jab[i] != 0.0)
                atomicAdd(A + (size_t)(P.cA + i / NB) + (size_t)(P.cB + i % NB) * nc, jab[i]);
          }
        }
      }
    }
    if (grouped && any) {
      double* AJ = a.Ac + a.jmat * matStride;
      double* AK = a.Ac + a.kmat * matStride;
#pragma unroll
      for (int k = 0; k < G64::NJCD; k++)
        if (jcd[k] != 0.0)
          atomicAdd(AJ + (size_t)(Q.cA + k / ND) + (size_t)(Q.cB + k % ND) * nc, jcd[k]);
#pragma unroll
      for (int k = 0; k < G64::NKAC; k++)
        if (kac[k] != 0.0)
          atomicAdd(AK + (size_t)(Q.cA + k % NC) + (size_t)(cAgrp + k / NC) * nc, kac[k]);
#pragma unroll
      for (int k = 0; k < G64::NKAD; k++)
        if (kad[k] != 0.0)
          atomicAdd(AK + (size_t)(Q.cB + k % ND) + (size_t)(cAgrp + k / ND) * nc, kad[k]);
    }
  }
  if (lane == 0) {
    if (cVis) atomicAdd(a.counters + 0, cVis);
    if (cScr) atomicAdd(a.counters + 1, cScr);
    if (c32) atomicAdd(a.counters + 2, c32);
    if (c64) atomicAdd(a.counters + 3, c64);
  }
}

// Launches the generated kernels of the class (la lb | lc ld) (either
// orientation); returns false when the class has no generated kernel.
// work: two zeroed device counters for this class (FP64, FP32 launch).
inline bool launch_jk_fast(JKLaunch a, int la, int lb, int lc, int ld, unsigned int* work,
                           int nsm, cudaStream_t st, int blocksPerSm = 8) {
  if (a.nBra == 0 || a.nKet == 0) return true;
  bool done = false;
  auto go = [&](auto tag64, auto tag32, bool swap) {
    using G64 = decltype(tag64);
    using G32 = decltype(tag32);
    JKLaunch b = a;
    if (swap) {
      b.braBeg = a.ketBeg; b.nBra = a.nKet;
      b.ketBeg = a.braBeg; b.nKet = a.nBra;
      b.braTileBeg = a.ketTileBeg; b.ketTileBeg = a.braTileBeg;
      b.braGroupBeg = a.ketGroupBeg; b.braNGroups = a.ketNGroups;
      b.ketGroupBeg = a.braGroupBeg; b.ketNGroups = a.braNGroups;
    }
    const long long tiles = (long long)((b.nKet + WTILE - 1) / WTILE);
    // bra groups pay off when one J and one K matrix share the sums;
    // many-density launches use the per-quartet kernel
    const bool useGroups = G64::GROUPED && b.jmat >= 0;
    const long long items = useGroups ? (long long)b.braNGroups * tiles
                                      : (long long)b.nBra * tiles * G64::NCHUNK;
    // persistent blocks: enough for full residency on every SM (extra blocks
    // queue and find the counter exhausted); one work item per warp at a time
    constexpr int WPB = JK_THREADS / 32;
    const unsigned g =
        (unsigned)std::min<long long>((items + WPB - 1) / WPB, (long long)nsm * blocksPerSm);
    const bool mixed = b.precision == 1 && b.fp32_cut > 0.0;
    if constexpr (G64::GROUPED) {
      if (useGroups) {
        if (mixed)
          jk_group_kernel<G64, G32, true><<<g, JK_THREADS, 0, st>>>(b, work);
        else
          jk_group_kernel<G64, G32, false><<<g, JK_THREADS, 0, st>>>(b, work);
      } else {
        if (mixed)
          jk_fast_kernel<G64, G32, true><<<g, JK_THREADS, 0, st>>>(b, work);
        else
          jk_fast_kernel<G64, G32, false><<<g, JK_THREADS, 0, st>>>(b, work);
      }
    } else {
      if (mixed)
        jk_fast_kernel<G64, G32, true><<<g, JK_THREADS, 0, st>>>(b, work);
      else
        jk_fast_kernel<G64, G32, false><<<g, JK_THREADS, 0, st>>>(b, work);
    }
    done = true;
  };
#define CQF_TRY_CLASS(A_, B_, C_, D_, N64, N32)                                          \
  if (!done && la == A_ && lb == B_ && lc == C_ && ld == D_) go(N64{}, N32{}, false);    \
  if (!done && la == C_ && lb == D_ && lc == A_ && ld == B_) go(N64{}, N32{}, true);
  CQF_GEN_JK_CLASSES(CQF_TRY_CLASS)
#undef CQF_TRY_CLASS
  return done;
}

// ----------------------------------------------------------- Schwarz (fast)
// Diagonal (mu nu|mu nu) of the pairs of one class (LA, LB) with LA, LB <= 2
// from the generated (ab|ab) code, one thread per (pair, chunk); the chunk's
// share of each spherical diagonal element is added into diag[pair][mu][nu].
template <class GC>
__global__ void __launch_bounds__(JK_THREADS)
    schwarz_diag_kernel(const PairDev* __restrict__ pairs, const PrimPairDev* __restrict__ pp,
                        const double* __restrict__ boys, const double* __restrict__ sph,
                        const int* __restrict__ sphOff, const ShellDev* __restrict__ shells,
                        int beg, int n, double* diag) {
  constexpr int NA = ncart(GC::LA), NB = ncart(GC::LB), NCH = GC::NCHUNK;
  constexpr int CS = GC::NI / (NA * NB);
  const long long item = (long long)blockIdx.x * JK_THREADS + threadIdx.x;
  if (item >= (long long)n * NCH) return;
  const int k = (int)(item / NCH), ch = (int)(item % NCH);
  const PairDev P = pairs[beg + k];
  const ShellDev A = shells[P.shA], B = shells[P.shB];
  const int na = A.pure ? nsph(GC::LA) : NA, nb = B.pure ? nsph(GC::LB) : NB;
  const double* TA = sph + sphOff[GC::LA];
  const double* TB = sph + sphOff[GC::LB];
  auto ta = [&](int c, int mu) { return A.pure ? TA[c * nsph(GC::LA) + mu] : (c == mu ? 1.0 : 0.0); };
  auto tb = [&](int c, int nu) { return B.pure ? TB[c * nsph(GC::LB) + nu] : (c == nu ? 1.0 : 0.0); };
  double I[GC::NI];
  GC::template eri<double>(P, P, pp, KetAoS{pp + P.pp_off},
                           boys + (size_t)(2 * (GC::LA + GC::LB)) * BOYS_NPTS * BOYS_ROW64, ch, I);
  for (int mu = 0; mu < na; mu++)
    for (int nu = 0; nu < nb; nu++) {
      double s = 0.0;
      for (int kk = 0; kk < CS; kk++) {
        const int cd = ch * CS + kk;
        if (cd >= NA * NB) break;
        const double tcd = ta(cd / NB, mu) * tb(cd % NB, nu);
        if (tcd == 0.0) continue;
        double sab = 0.0;
        for (int a = 0; a < NA; a++) {
          const double t1 = ta(a, mu);
          if (t1 == 0.0) continue;
          for (int b = 0; b < NB; b++) sab += t1 * tb(b, nu) * I[(a * NB + b) * CS + kk];
        }
        s += tcd * sab;
      }
      if (s != 0.0) atomicAdd(diag + (size_t)k * 36 + mu * 6 + nu, s);
    }
}

// Q = sqrt(max row sum |diag|) with rows the functions of s1
// (aointegrals_utilities.cxx:78-104); writes the pair and the table.
__global__ void schwarz_finish_kernel(const PairDev* __restrict__ pairs,
                                      const ShellDev* __restrict__ shells, int beg, int n,
                                      int nshell, const double* __restrict__ diag, double* Qtab,
                                      PairDev* pairsOut) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const PairDev P = pairs[beg + k];
  const ShellDev A = shells[P.shA], B = shells[P.shB];
  const int na = A.pure ? nsph(A.l) : ncart(A.l), nb = B.pure ? nsph(B.l) : ncart(B.l);
  const double* d = diag + (size_t)k * 36;
  const bool swp = P.shA != P.s1;
  double mx = 0.0;
  if (!swp) {
    for (int i = 0; i < na; i++) {
      double r = 0.0;
      for (int j = 0; j < nb; j++) r += fabs(d[i * 6 + j]);
      mx = fmax(mx, r);
    }
  } else {
    for (int j = 0; j < nb; j++) {
      double r = 0.0;
      for (int i = 0; i < na; i++) r += fabs(d[i * 6 + j]);
      mx = fmax(mx, r);
    }
  }
  const double q = sqrt(mx);
  pairsOut[beg + k].Q = q;
  Qtab[P.s1 + (size_t)P.s2 * nshell] = q;
  Qtab[P.s2 + (size_t)P.s1 * nshell] = q;
}

// Schwarz bounds of one class with the generated code; false if the class
// has none.  diag: n x 36 doubles (6 x 6 per pair), zeroed here.
inline bool launch_schwarz_fast(int la, int lb, const PairDev* pairs, const PrimPairDev* pp,
                                const double* boys, const double* sph, const int* sphOff,
                                const ShellDev* shells, int beg, int n, int nshell, double* Qtab,
                                PairDev* pairsOut, double* diag, cudaStream_t st) {
  if (n <= 0) return true;
  bool done = false;
  auto go = [&](auto tag64) {
    using G = decltype(tag64);
    cudaMemsetAsync(diag, 0, (size_t)n * 36 * sizeof(double), st);
    const long long items = (long long)n * G::NCHUNK;
    schwarz_diag_kernel<G><<<(unsigned)((items + JK_THREADS - 1) / JK_THREADS), JK_THREADS, 0,
                             st>>>(pairs, pp, boys, sph, sphOff, shells, beg, n, diag);
    schwarz_finish_kernel<<<(n + 127) / 128, 128, 0, st>>>(pairs, shells, beg, n, nshell, diag,
                                                          Qtab, pairsOut);
    done = true;
  };
#define CQF_TRY_SCHWARZ(A_, B_, C_, D_, N64, N32) \
  if (!done && A_ == la && B_ == lb && C_ == la && D_ == lb) go(N64{});
  CQF_GEN_JK_CLASSES(CQF_TRY_SCHWARZ)
#undef CQF_TRY_SCHWARZ
  return done;
}

}  // namespace cqf
