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

namespace cqf {

template <int N>
__device__ __forceinline__ void warp_sum(double (&v)[N]) {
#pragma unroll
  for (int i = 0; i < N; i++) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
  }
}

// FP64 launch: quartets with bound >= cut (all when cut <= 0); FP32 launch:
// quartets with thresh <= bound < cut.  The FP64 launch also counts the
// visited / screened quartets.
template <class GC, typename T>
__global__ void __launch_bounds__(JK_THREADS)
    jk_fast_kernel(const JKLaunch a) {
  constexpr int NA = ncart(GC::LA), NB = ncart(GC::LB);
  constexpr bool IS64 = sizeof(T) == 8;
  const int ib = blockIdx.x;
  const int jk = blockIdx.y * JK_THREADS + threadIdx.x;
  const PairDev P = a.pairs[a.braBeg + ib];
  const int ns = a.nShell;
  const double cut = (a.precision == 1) ? a.fp32_cut : 0.0;

  bool visited = false, screened = false, work = false;
  PairDev Q;
  if (jk < a.nKet) {
    Q = a.pairs[a.ketBeg + jk];
    visited = !(a.same && Q.lex > P.lex);
  }
  const double tileMax =
      __ldg(a.maxNorm) * P.Q * a.pairs[a.ketBeg + blockIdx.y * JK_THREADS].Q;
  const bool tileDead = a.screen && tileMax < a.thresh;
  if (tileDead || (!IS64 && cut <= 0.0)) {
    if (IS64) count_block(a.counters, visited, visited, false, false);
    return;
  }
  int s1 = 0, s2 = 0, s3 = 0, s4 = 0;
  if (visited) {
    const bool pRef = P.lex >= Q.lex;
    const PairDev& R12 = pRef ? P : Q;
    const PairDev& R34 = pRef ? Q : P;
    s1 = R12.s1; s2 = R12.s2; s3 = R34.s1; s4 = R34.s2;
    double bound = 1e300;
    if (a.screen) {
      bound = sh_max(a.norms, s1, s2, s3, s4, ns) * P.Q * Q.Q;
      screened = bound < a.thresh;
    }
    const bool lo = bound < cut;
    work = !screened && (IS64 ? !lo : lo);
  }
  if (IS64)
    count_block(a.counters, visited, screened, false, work);
  else
    count_block(a.counters, false, false, work, false);
  if (!__syncthreads_or(work)) return;

  const double deg = ((s1 == s2) ? 1.0 : 2.0) * ((s3 == s4) ? 1.0 : 2.0) *
                     ((s1 == s3 && s2 == s4) ? 1.0 : 2.0);
  const double sJ = work ? 0.5 * deg : 0.0, sK = work ? 0.25 * deg : 0.0;
  const size_t nc = a.ncart;
  const size_t matStride = (size_t)a.ncart * a.ncart;
  const T* boys = IS64 ? reinterpret_cast<const T*>(a.boys64)
                       : reinterpret_cast<const T*>(a.boys32);
#pragma unroll 1
  for (int ch = 0; ch < GC::NCHUNK; ch++) {
    double I[GC::NI];
    if (work) {
      GC::template eri<T>(P, Q, a.pp, boys, ch, I);
    } else {
#pragma unroll
      for (int i = 0; i < GC::NI; i++) I[i] = 0.0;
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
      GC::digest(I, ch, X, A, nc, P.cA, P.cB, Q.cA, Q.cB, sJ, sK, doJ && work, doK && work, jab);
      if (doJ) {
        // every lane of the warp shares the bra pair: reduce, one atomic each
#pragma unroll
        for (int i = 0; i < NA * NB; i++) jab[i] *= sJ;
        warp_sum(jab);
        if ((threadIdx.x & 31) == 0) {
#pragma unroll
          for (int i = 0; i < NA * NB; i++)
            if (jab[i] != 0.0)
              atomicAdd(A + (size_t)(P.cA + i / NB) + (size_t)(P.cB + i % NB) * nc, jab[i]);
        }
      }
    }
  }
}

// Launches the generated kernel of the class (bra bucket cb, ket bucket ck);
// returns false when the class has no generated kernel.
inline bool launch_jk_fast(JKLaunch a, int la, int lb, int lc, int ld, cudaStream_t st) {
  if (a.nBra == 0 || a.nKet == 0) return true;
  bool done = false;
  auto go = [&](auto tag, bool swap) {
    using GC = decltype(tag);
    JKLaunch b = a;
    if (swap) {
      b.braBeg = a.ketBeg; b.nBra = a.nKet;
      b.ketBeg = a.braBeg; b.nKet = a.nBra;
    }
    dim3 grid(b.nBra, (b.nKet + JK_THREADS - 1) / JK_THREADS);
    jk_fast_kernel<GC, double><<<grid, JK_THREADS, 0, st>>>(b);
    if (b.precision == 1 && b.fp32_cut > 0.0)
      jk_fast_kernel<GC, float><<<grid, JK_THREADS, 0, st>>>(b);
    done = true;
  };
#define CQF_TRY_CLASS(A_, B_, C_, D_, NAME)                                   \
  if (!done && la == A_ && lb == B_ && lc == C_ && ld == D_) go(NAME{}, false); \
  if (!done && la == C_ && lb == D_ && lc == A_ && ld == B_) go(NAME{}, true);
  CQF_GEN_JK_CLASSES(CQF_TRY_CLASS)
#undef CQF_TRY_CLASS
  return done;
}

}  // namespace cqf
