// CUDA-graph form of the contraction, for builds repeated on the same device
// buffers (RT-TDDFT steps, response right-hand sides, SCF iterations with
// many densities): the whole contraction -- block norms, Cartesian
// transforms, every class-quartet kernel, back transform -- is captured once
// and replayed with one cudaGraphLaunch.  The graph owns its workspace, so
// later calls on the same basis cannot move it.
#include <vector>

#include "cqf_internal.hpp"

struct cqf_graph {
  cqf_basis* B = nullptr;
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  double* ws = nullptr;
  int* d_flags = nullptr;
};

namespace {

#define CQF_GCUDA(call)                                                                    \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return cqf::fail(e_ == cudaErrorMemoryAllocation ? CQF_ENOMEM : CQF_ECUDA,           \
                       std::string(#call) + ": " + cudaGetErrorString(e_));               \
  } while (0)

void release(cqf_graph* G) {
  if (!G) return;
  if (G->ge) cudaGraphExecDestroy(G->ge);
  if (G->g) cudaGraphDestroy(G->g);
  cudaFree(G->ws);
  cudaFree(G->d_flags);
  delete G;
}

cqf_status create(cqf_basis* B, const cqf_contraction* list, int nMat, const cqf_opts& opts,
                  cqf_graph* G) {
  G->B = B;
  // complex Hermitian densities on an s..d basis: the real split
  const bool split = cqf::split_eligible(B, list, nMat, opts);
  const int nFlags = split ? cqf::split_real_count(list, nMat) : nMat;
  const size_t wsd = split ? cqf::split_ws_doubles(B, nFlags, opts)
                           : cqf::ws_layout(B, nMat, opts).total;
  CQF_GCUDA(cudaMalloc(&G->ws, wsd * sizeof(double)));
  CQF_GCUDA(cudaMalloc(&G->d_flags, nFlags * sizeof(int)));
  std::vector<int> fl(nFlags);
  if (split)
    cqf::split_flags(list, nMat, fl.data());
  else
    for (int m = 0; m < nMat; m++) fl[m] = cqf::contraction_flags(list[m], opts.is_complex != 0);
  CQF_GCUDA(cudaMemcpy(G->d_flags, fl.data(), nFlags * sizeof(int), cudaMemcpyHostToDevice));
  auto run = [&](const cqf_contraction* l, const cqf_opts& o, bool capture) {
    return split ? cqf::split_core(B, l, nMat, o, nullptr, G->ws, capture, G->d_flags)
                 : cqf::contract_core(B, l, nMat, o, nullptr, G->ws, capture, G->d_flags);
  };
  // warm-up into throw-away outputs, so every kernel of the graph is loaded
  // before capture starts
  const size_t matN = (size_t)B->nbasis * B->nbasis * (opts.is_complex ? 2 : 1);
  double* tmp = nullptr;
  CQF_GCUDA(cudaMalloc(&tmp, matN * nMat * sizeof(double)));
  std::vector<cqf_contraction> warm(list, list + nMat);
  for (int m = 0; m < nMat; m++) warm[m].AX = tmp + m * matN;
  cqf_opts wo = opts;
  wo.stream = B->stream;
  cqf_status s = run(warm.data(), wo, false);
  cudaStreamSynchronize(B->stream);
  cudaFree(tmp);
  if (s != CQF_OK) return s;
  // capture on the basis' private stream
  CQF_GCUDA(cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal));
  s = run(list, wo, true);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(B->stream, &g);
  if (s != CQF_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess)
    return cqf::fail(CQF_ECUDA, std::string("stream capture: ") + cudaGetErrorString(e));
  G->g = g;
  CQF_GCUDA(cudaGraphInstantiate(&G->ge, g, 0));
  return CQF_OK;
}

}  // namespace

extern "C" {

cqf_status cqf_graph_create(cqf_basis* B, const cqf_contraction* list, int nMat,
                            const cqf_opts* optsIn, cqf_graph** out) {
  cqf::fail(CQF_OK, "");
  if (!out) return cqf::fail(CQF_EINVAL, "cqf_graph_create: null output");
  *out = nullptr;
  cqf_status s = cqf::check_contract_args(B, list, nMat);
  if (s != CQF_OK) return s;
  cqf_opts opts;
  cqf_opts_default(&opts);
  if (optsIn) opts = *optsIn;
  if (!opts.device_pointers)
    return cqf::fail(CQF_EINVAL, "cqf_graph_create: graphs need device pointers");
  std::lock_guard<std::mutex> lk(B->mu);
  if (cudaSetDevice(B->device) != cudaSuccess) return cqf::fail(CQF_ECUDA, "cudaSetDevice");
  auto* G = new cqf_graph();
  s = create(B, list, nMat, opts, G);
  if (s != CQF_OK) {
    release(G);
    return s;
  }
  *out = G;
  return CQF_OK;
}

cqf_status cqf_graph_launch(cqf_graph* G, void* stream) {
  if (!G || !G->ge) return cqf::fail(CQF_EINVAL, "cqf_graph_launch: null graph");
  cudaStream_t st = stream ? (cudaStream_t)stream : G->B->stream;
  cudaError_t e = cudaGraphLaunch(G->ge, st);
  if (e != cudaSuccess)
    return cqf::fail(CQF_ECUDA, std::string("cudaGraphLaunch: ") + cudaGetErrorString(e));
  return CQF_OK;
}

cqf_status cqf_graph_destroy(cqf_graph* G) {
  if (G) {
    cudaSetDevice(G->B->device);
    release(G);
  }
  return CQF_OK;
}

}  // extern "C"
