// Closed-shell fast path: real densities flagged Hermitian (symmetric), every
// shell l <= 2.  One thread per unique quartet, generated straight-line
// McMurchie-Davidson code per class and precision (gen/cqf_gen_jk.cuh): a
// planning pass names each quartet's precision, then an FP64 and (mixed
// builds) an FP32 kernel per class compute their quartets; FP64
// accumulation.
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

template <typename T, int N>
__device__ __forceinline__ void warp_sum(T (&v)[N]) {
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
  const double* q;  // primitive Schwarz bounds of the same pairs (read only when screening)
  __device__ __forceinline__ double Qp(int iq) const { return q[iq]; }
  __device__ __forceinline__ double p(int iq) const { return b[iq].p; }
  __device__ __forceinline__ double Kp(int iq) const { return b[iq].Kp; }
  __device__ __forceinline__ double o2p(int iq) const { return b[iq].o2p; }
  __device__ __forceinline__ double P(int iq, int x) const { return b[iq].P[x]; }
  __device__ __forceinline__ double PA(int iq, int x) const { return b[iq].PA[x]; }
  __device__ __forceinline__ double PB(int iq, int x) const { return b[iq].PB[x]; }
};
template <typename E>  // element type: double, or float for the FP32 copy
struct KetSoAT {
  const E* q;  // tile base + lane
  __device__ __forceinline__ E f(int iq, int k) const {
    return __ldg(q + (iq * KETT_NF + k) * KETT_TILE);
  }
  __device__ __forceinline__ E p(int iq) const { return f(iq, 0); }
  __device__ __forceinline__ E Kp(int iq) const { return f(iq, 1); }
  __device__ __forceinline__ E o2p(int iq) const { return f(iq, 2); }
  __device__ __forceinline__ E P(int iq, int x) const { return f(iq, 3 + x); }
  __device__ __forceinline__ E PA(int iq, int x) const { return f(iq, 6 + x); }
  __device__ __forceinline__ E PB(int iq, int x) const { return f(iq, 9 + x); }
  __device__ __forceinline__ double Qp(int iq) const { return (double)f(iq, 12); }
};
using KetSoA = KetSoAT<double>;

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

// Planning pass of one class pair: for every (bra pair, tile of 32 kets) the
// quartets that survive the Schwarz x density screen, split by precision --
// mask.x: lanes computed in FP64, mask.y: lanes computed in FP32 (mixed
// builds: screening bound below the cut and inside the FP32 range guard).
// Quartet set, screens and counts are those of the reference's loop
// (direct.hpp:1642-1805); in the same class a ket sits at or before its bra
// (each unordered pair of pairs once).  The masks form one row-major
// sequence of words (bra pair, ket tile); a warp takes runs of 32
// consecutive words and appends the indices of its non-empty words to one
// list per precision (lengths in lcount[0 / 1]), so the class kernels visit
// only words that name quartets of their precision.
constexpr int PLAN_RUN = 32;
template <bool MIXED>
__global__ void __launch_bounds__(256)
    jk_plan_kernel(const JKLaunch a, uint2* __restrict__ masks, int* __restrict__ list64,
                   int* __restrict__ list32, unsigned int* __restrict__ lcount) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int nTiles = (a.nKet + WTILE - 1) / WTILE;
  const int nWords = a.nBra * nTiles;
  const int nRuns = (nWords + PLAN_RUN - 1) / PLAN_RUN;
  const double cut = MIXED ? a.fp32_cut : 0.0;
  unsigned long long cVis = 0, cScr = 0, c32 = 0, c64 = 0;
  for (int run = gw; run < nRuns; run += nw) {
    int my64 = -1, my32 = -1, n64 = 0, n32 = 0;
    const int wEnd = min((run + 1) * PLAN_RUN, nWords);
    for (int word = run * PLAN_RUN; word < wEnd; word++) {
      const int ib = word / nTiles, tile = word - ib * nTiles;
      unsigned b64 = 0u, b32 = 0u;
      const int ibc = ib + a.braOff;  // the bra's position in its class
      // else: no quartet in this word (above the diagonal, or another shard's bra)
      if (!(a.same && tile * WTILE > ibc) && in_shard(a.braBeg + ib, a.shardIdx, a.shardCnt)) {
        const int jk = tile * WTILE + lane;
        const PairDev P = a.pairs[a.braBeg + ib];
        const bool visited = jk < a.nKet && !(a.same && jk > ibc);
        const double tileMax = __ldg(a.maxNorm) * P.Q * __ldg(a.qWin + a.ketBeg + tile * WTILE);
        bool screened = false, w32 = false;
        if (a.screen && tileMax < a.thresh) {
          screened = true;
        } else if (visited && a.screen) {
          const PairDev Q = a.pairs[a.ketBeg + jk];
          const bool pRef = P.lex >= Q.lex;
          const double bound = sh_max_bra(a, P, Q, __ldg(a.pairNorm + a.braBeg + ib),
                                          __ldg(a.pairNorm + a.ketBeg + jk), pRef) * P.Q * Q.Q;
          screened = bound < a.thresh;
          w32 = MIXED && !screened && bound < cut &&
                fp32_range_ok(__ldg(a.pairRange + a.braBeg + ib),
                              __ldg(a.pairRange + a.ketBeg + jk), a.lsum, 0, 0);
        }  // without the screen every quartet runs in FP64
        const unsigned bv = __ballot_sync(0xffffffffu, visited);
        const unsigned bs = __ballot_sync(0xffffffffu, visited && screened);
        b32 = __ballot_sync(0xffffffffu, visited && !screened && w32);
        b64 = bv & ~bs & ~b32;
        cVis += __popc(bv);
        cScr += __popc(bs);
        c32 += __popc(b32);
        c64 += __popc(b64);
      }
      if (lane == 0) masks[word] = make_uint2(b64, b32);
      if (b64) {
        if (lane == n64) my64 = word;
        n64++;
      }
      if (b32) {
        if (lane == n32) my32 = word;
        n32++;
      }
    }
    unsigned int base64 = 0, base32 = 0;
    if (lane == 0) {
      if (n64) base64 = atomicAdd(lcount + 0, (unsigned)n64);
      if (n32) base32 = atomicAdd(lcount + 1, (unsigned)n32);
    }
    base64 = __shfl_sync(0xffffffffu, base64, 0);
    base32 = __shfl_sync(0xffffffffu, base32, 0);
    if (lane < n64) list64[base64 + lane] = my64;
    if (lane < n32) list32[base32 + lane] = my32;
  }
  if (lane == 0) {
    if (cVis) atomicAdd(a.counters + 0, cVis);
    if (cScr) atomicAdd(a.counters + 1, cScr);
    if (c32) atomicAdd(a.counters + 2, c32);
    if (c64) atomicAdd(a.counters + 3, c64);
  }
}

// Position of the n-th (0-based) set bit of m (n < popc(m)).
__device__ __forceinline__ int nth_set_bit(unsigned m, int n) {
  int pos = 0;
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    const unsigned lo = m & ((1u << w) - 1u);
    const int c = __popc(lo);
    if (n >= c) {
      n -= c;
      m >>= w;
      pos += w;
    } else {
      m = lo;
    }
  }
  return pos;
}

// Class kernel of one shell-quartet class in one precision (G = GenJK64_x
// or GenJK32_x; FP32 = which mask half and word list it uses).  A work item
// is (run of consecutive entries of the precision's word list -- sized from
// the list's length, at most entriesPerItem -- ket component chunk), handed
// out by a device counter.  A warp walks
// its run's words and packs the quartets they name into batches of 32 lanes
// (nth_set_bit), so every lane of a batch computes a surviving quartet; a
// batch may span two bra pairs.  The batch's integrals of the chunk come
// from generated straight-line McMurchie-Davidson code and are digested per
// density: J_ab warp-reduced when the batch has one bra pair (per lane
// otherwise), J_cd and the four exchange blocks with FP64 atomics.  The FP32
// kernel forms integrals and products in FP32 from the FP32 copy of the
// Cartesian densities; accumulation is FP64 in both.
template <class G, bool FP32>
__global__ void __launch_bounds__(JK_THREADS, G::MINB)
    jk_class_kernel(const JKLaunch a, const uint2* __restrict__ masks,
                    const int* __restrict__ list, const unsigned int* __restrict__ lcount,
                    int entriesPerItem, unsigned int* __restrict__ counter) {
  using T = typename G::T;
  constexpr int NA = ncart(G::LA), NB = ncart(G::LB);
  constexpr int NCH = G::NCHUNK;
  constexpr int LSUM = G::LA + G::LB + G::LC + G::LD;
  const T* boys = boys_rows<T>(a, LSUM);
  const T* Xbase = FP32 ? reinterpret_cast<const T*>(a.Xc32) : reinterpret_cast<const T*>(a.Xc);
  const int lane = threadIdx.x & 31;
  const int nTiles = (a.nKet + WTILE - 1) / WTILE;
  const int nEntries = (int)*lcount;  // written by the planning pass
  // entries per item from the list's actual length: about four items per
  // warp of the grid, at most entriesPerItem entries
  const int gridWarps = (int)(gridDim.x * (blockDim.x / 32));
  const int epi = max(1, min(entriesPerItem, (int)((long long)nEntries * NCH /
                                                   (4LL * gridWarps))));
  const int nItems = (nEntries + epi - 1) / epi * NCH;
  const size_t nc = a.ncart;
  const size_t matStride = (size_t)a.ncart * a.ncart;
  // primitive screen threshold: libint's engine precision as the reference
  // sets it, max(eps_double, tau / (max shell-block norm x K^4)), K the
  // largest contraction length (direct.hpp:1563-1589)
  const double peps =
      a.screen ? fmax(2.220446049250313e-16, a.thresh / (__ldg(a.maxNorm) * a.primK4)) : 0.0;
  // entry e of the list: (word index, this precision's mask of it)
  auto entry = [&](int e) {
    const int w = __ldg(list + e);
    return make_int2(w, (int)(FP32 ? __ldg(&masks[w].y) : __ldg(&masks[w].x)));
  };

  for (;;) {
    unsigned int itemU = 0;
    if (lane == 0) itemU = atomicAdd(counter, 1u);
    const int item = (int)__shfl_sync(0xffffffffu, itemU, 0);
    if (item >= nItems) break;
    const int run = item / NCH, ch = item - run * NCH;
    int e = run * epi;
    const int eEnd = min(e + epi, nEntries);
    int2 wm = entry(e);
    unsigned m = (unsigned)wm.y;
    for (;;) {
      // pack the next (up to) 32 named quartets of the run into the lanes
      int fill = 0, myW = -1, myBit = 0;
      while (fill < 32 && e < eEnd) {
        const int c = __popc(m);
        const int take = min(c, 32 - fill);
        const int r = lane - fill;
        if (r >= 0 && r < take) {
          myW = wm.x;
          myBit = nth_set_bit(m, r);
        }
        fill += take;
        if (take == c) {
          if (++e < eEnd) {
            wm = entry(e);
            m = (unsigned)wm.y;
          }
        } else {
          m &= ~((2u << nth_set_bit(m, take - 1)) - 1u);  // drop the bits taken
        }
      }
      if (fill == 0) break;
      const bool work_ = myW >= 0;
      // lane 0 always holds a quartet; idle lanes take its bra pair
      const int w0 = __shfl_sync(0xffffffffu, myW, 0);
      const int wl = work_ ? myW : w0;
      const int ib = wl / nTiles;
      const int jk = (wl - ib * nTiles) * WTILE + myBit;
      const bool oneBra = __all_sync(0xffffffffu, ib == w0 / nTiles);
      const PairDev P = a.pairs[a.braBeg + ib];
      PairDev Q{};  // idle lanes: npp = 0, no primitive loop
      if (work_) Q = a.pairs[a.ketBeg + jk];
      const bool pRef = P.lex >= Q.lex;
      const int s1 = pRef ? P.s1 : Q.s1, s2 = pRef ? P.s2 : Q.s2;
      const int s3 = pRef ? Q.s1 : P.s1, s4 = pRef ? Q.s2 : P.s2;
      const T deg = T(((s1 == s2) ? 1 : 2) * ((s3 == s4) ? 1 : 2) *
                      ((s1 == s3 && s2 == s4) ? 1 : 2));
      const T sJ = work_ ? T(0.5) * deg : T(0), sK = work_ ? T(0.25) * deg : T(0);
      const int jkc = work_ ? jk : 0;
      const long long ko = __ldg(a.tileOff + a.ketTileBeg + jkc / KETT_TILE) + jkc % KETT_TILE;
      T I[G::NI];
      if constexpr (FP32)  // FP32 copies of the pair data: half the load bytes
        G::eri(P, Q, a.pp32, KetSoAT<float>{a.ketT32 + ko}, boys, ch, I, a.ppQ, peps);
      else
        G::eri(P, Q, a.pp, KetSoA{a.ketT + ko}, boys, ch, I, a.ppQ, peps);
#pragma unroll 1
      for (int mt = 0; mt < a.nMat; mt++) {
        const int fl = __ldg(a.flags + mt);
        const bool doJ = !(fl & 2), doK = (fl & 2);
        T jab[NA * NB];
#pragma unroll
        for (int i = 0; i < NA * NB; i++) jab[i] = T(0);
        double* A = a.Ac + mt * matStride;
        G::digest(I, ch, Xbase + mt * matStride, A, nc, P.cA, P.cB, Q.cA, Q.cB, sJ, sK,
                  (fl & 4) ? -sK : sK, doJ && work_, doK && work_, jab);
        if (doJ) {
#pragma unroll
          for (int i = 0; i < NA * NB; i++) jab[i] *= sJ;
          if (oneBra) {  // the lanes share the bra pair: reduce, one atomic each
            warp_sum(jab);
            if (lane == 0) {
#pragma unroll
              for (int i = 0; i < NA * NB; i++)
                if (jab[i] != T(0))
                  atomicAdd(A + (size_t)(P.cA + i / NB) + (size_t)(P.cB + i % NB) * nc,
                            double(jab[i]));
            }
          } else if (work_) {
#pragma unroll
            for (int i = 0; i < NA * NB; i++)
              if (jab[i] != T(0))
                atomicAdd(A + (size_t)(P.cA + i / NB) + (size_t)(P.cB + i % NB) * nc,
                          double(jab[i]));
          }
        }
      }
    }
  }
}

// Upper limit of word-list entries per work item of a class kernel (the
// kernel sizes its items from the list's actual length).
inline int entries_per_item(long long nWords, int nchunk, int nsm) {
  const long long per = nWords * nchunk / ((long long)nsm * 256);
  return (int)std::min<long long>(64, std::max<long long>(4, per));
}

// Launches the planning pass and the generated class kernels of the class
// (la lb | lc ld) (either orientation); false when the class has no
// generated kernel.  masks: the launch stream's region of maskWords uint2
// (mask words of a slab of bra pairs x ceil(nKet / 32) ket tiles, then its
// two word lists); work: the stream's four counters (FP64 / FP32 class
// kernel items, FP64 / FP32 list lengths), zeroed here before each slab.
inline bool launch_jk_fast(JKLaunch a, int la, int lb, int lc, int ld, uint2* masks,
                           long long maskWords, unsigned int* work, int nsm, cudaStream_t st,
                           int blocksPerSm = 8) {
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
    }
    b.lsum = la + lb + lc + ld;
    const bool mixed = b.precision == 1 && b.fp32_cut > 0.0;
    const int nTiles = (b.nKet + WTILE - 1) / WTILE;
    // slabs of bra pairs whose mask words fit the stream's region; each
    // reuses the region and the stream's counters after the last one's
    // kernels (stream order)
    const int slab = (int)std::max<long long>(1, maskWords / nTiles);
    for (int ib0 = 0; ib0 < b.nBra; ib0 += slab) {
      JKLaunch c = b;
      c.braBeg = b.braBeg + ib0;
      c.nBra = std::min(slab, b.nBra - ib0);
      c.braOff = b.braOff + ib0;
      cudaMemsetAsync(work, 0, 4 * sizeof(unsigned int), st);
      const long long nWords = (long long)c.nBra * nTiles;
      const long long nRuns = (nWords + PLAN_RUN - 1) / PLAN_RUN;
      const unsigned gp = (unsigned)std::min<long long>((nRuns + 7) / 8, (long long)nsm * 8);
      // word lists: FP64 then FP32, nWords entries each; counts in work[2..3]
      int* list64 = reinterpret_cast<int*>(masks + nWords);
      int* list32 = list64 + nWords;
      if (mixed)
        jk_plan_kernel<true><<<gp, 256, 0, st>>>(c, masks, list64, list32, work + 2);
      else
        jk_plan_kernel<false><<<gp, 256, 0, st>>>(c, masks, list64, list32, work + 2);
      constexpr int WPB = JK_THREADS / 32;
      auto grid = [&](long long items) {
        return (unsigned)std::max<long long>(
            1, std::min<long long>((items + WPB - 1) / WPB, (long long)nsm * blocksPerSm));
      };
      const int e64 = entries_per_item(nWords, G64::NCHUNK, nsm);
      jk_class_kernel<G64, false><<<grid((nWords + e64 - 1) / e64 * G64::NCHUNK), JK_THREADS,
                                    0, st>>>(c, masks, list64, work + 2, e64, work);
      if (mixed) {
        const int e32 = entries_per_item(nWords, G32::NCHUNK, nsm);
        jk_class_kernel<G32, true><<<grid((nWords + e32 - 1) / e32 * G32::NCHUNK), JK_THREADS,
                                     0, st>>>(c, masks, list32, work + 3, e32, work + 1);
      }
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
  GC::eri(P, P, pp, KetAoS{pp + P.pp_off, nullptr},
                           boys + (size_t)(2 * (GC::LA + GC::LB)) * BOYS_NPTS * BOYS_ROW64, ch, I, nullptr, 0.0);
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

// Primitive Schwarz bounds of the pairs of one class (LA, LB <= 2):
// Qp = sqrt(max over Cartesian components |(ab|ab)|) of each primitive pair
// alone (contraction coefficients included; the integrals the class kernels
// form), one thread per pair.  They bound each primitive quartet's integrals
// by Qp_ab Qp_cd (Cauchy-Schwarz), the primitive screen's estimate.
template <class GC>
__global__ void prim_schwarz_kernel(const PairDev* __restrict__ pairs,
                                    const PrimPairDev* __restrict__ pp,
                                    const double* __restrict__ boys, int beg, int n,
                                    double* __restrict__ ppQ) {
  constexpr int NA = ncart(GC::LA), NB = ncart(GC::LB), NCH = GC::NCHUNK;
  constexpr int CS = GC::NI / (NA * NB);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const PairDev P = pairs[beg + k];
  for (int ip = 0; ip < P.npp; ip++) {
    PairDev P1 = P;
    P1.npp = 1;
    P1.pp_off = P.pp_off + ip;
    double mx = 0.0;
    for (int ch = 0; ch < NCH; ch++) {
      double I[GC::NI];
      GC::eri(P1, P1, pp, KetAoS{pp + P1.pp_off, nullptr},
              boys + (size_t)(2 * (GC::LA + GC::LB)) * BOYS_NPTS * BOYS_ROW64, ch, I, nullptr,
              0.0);
      for (int kk = 0; kk < CS; kk++) {
        const int cd = ch * CS + kk;  // the diagonal element (ab | ab), ab = cd
        if (cd < NA * NB) mx = fmax(mx, fabs(I[cd * CS + kk]));
      }
    }
    ppQ[P.pp_off + ip] = sqrt(mx);
  }
}

// Primitive Schwarz bounds of one class with the generated code; false if
// the class has none.
inline bool launch_prim_schwarz(int la, int lb, const PairDev* pairs, const PrimPairDev* pp,
                                const double* boys, int beg, int n, double* ppQ,
                                cudaStream_t st) {
  if (n <= 0) return true;
  bool done = false;
  auto go = [&](auto tag64) {
    using G = decltype(tag64);
    prim_schwarz_kernel<G><<<(n + 63) / 64, 64, 0, st>>>(pairs, pp, boys, beg, n, ppQ);
    done = true;
  };
#define CQF_TRY_PRIM(A_, B_, C_, D_, N64, N32) \
  if (!done && A_ == la && B_ == lb && C_ == la && D_ == lb) go(N64{});
  CQF_GEN_JK_CLASSES(CQF_TRY_PRIM)
#undef CQF_TRY_PRIM
  return done;
}

}  // namespace cqf
