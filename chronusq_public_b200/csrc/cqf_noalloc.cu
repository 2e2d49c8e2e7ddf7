// cqf_two_body_contract_noalloc: the direct J/K contraction for callers that
// must not allocate device memory during the call.
//
// Who cannot allocate: host code that runs inside a framework that owns the
// whole device memory pool and forbids side allocations (e.g. a serving
// engine that has reserved HBM up front), and latency-critical loops that
// cannot afford the implicit device synchronisation of cudaFree.
// cqf_two_body_contract grows a per-basis workspace with cudaMalloc on first
// use; this entry point instead uses one fixed array compiled into the
// library.
//
// The scratch is a file-scope __device__ array of CQF_NOALLOC_SCRATCH_BYTES
// (32 MiB).  Every GPU that loads the library holds it until the process
// exits.  Calls whose workspace (Cartesian densities and accumulators, shell
// block norms, and for host pointers the device copies of X and AX) exceeds
// it are rejected with CQF_EINVAL.  All calls share the one array and it keeps
// the last call's contents; everything that must start at zero is cleared by
// the call itself.  Two calls that overlap on the GPU (different streams or
// host threads with different bases) race on the array: serialise them.
// The array's device address is resolved by cqf_basis_create (see
// noalloc_prepare), so the calls themselves map nothing.
#include <cstdio>
#include <mutex>
#include <vector>

#include "cqf_internal.hpp"

namespace {

constexpr size_t kScratchDoubles = CQF_NOALLOC_SCRATCH_BYTES / sizeof(double);

// The scratch array.  In host code its name is a host-side stand-in, not a
// device address: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
double* g_addr[kMaxDevices] = {nullptr};

// Device address of the scratch array on `device`, resolved once per device
// with that device current (the caller has made it current).
cqf_status scratch_address(int device, double** out) {
  if (device < 0 || device >= kMaxDevices)
    return cqf::fail(CQF_EINVAL, "cqf_two_body_contract_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return cqf::fail(CQF_ECUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                      cudaGetErrorString(e));
    g_addr[device] = static_cast<double*>(p);
  }
  *out = g_addr[device];
  return CQF_OK;
}

}  // namespace

namespace cqf {

// Called by cqf_basis_create with `device` current.  CUDA loads this file's
// module -- and with it maps the scratch array on the device -- lazily, on
// the first use of one of its symbols; resolving the address here puts that
// mapping inside basis creation, which allocates anyway, so that the no-alloc
// entry point's own calls never do.  A failure here is not fatal to the
// basis: the no-alloc call retries and reports it.
void noalloc_prepare(int device) {
  double* p = nullptr;
  if (scratch_address(device, &p) != CQF_OK) cudaGetLastError();
}

}  // namespace cqf

extern "C" cqf_status cqf_two_body_contract_noalloc(cqf_basis* B, const cqf_contraction* listIn,
                                                    int nMat, const cqf_opts* optsIn,
                                                    cqf_stats* stats) {
  cqf::fail(CQF_OK, "");
  cqf_status s = cqf::check_contract_args(B, listIn, nMat);
  if (s != CQF_OK) return s;
  cqf_opts opts;
  cqf_opts_default(&opts);
  if (optsIn) opts = *optsIn;
  // the same normalisation and kernel choice as cqf_two_body_contract:
  // HER is a bool, and complex Hermitian densities run on the real fast
  // kernels through their symmetric / antisymmetric split
  bool allHer = true;
  std::vector<cqf_contraction> list = cqf::normalized_list(listIn, nMat, &allHer);
  const bool split = allHer && cqf::split_eligible(B, list.data(), nMat, opts);
  const size_t need = split ? cqf::complex_split_ws_doubles(B, list.data(), nMat, opts)
                            : cqf::ws_layout(B, nMat, opts).total;
  if (need > kScratchDoubles) {
    char msg[256];
    std::snprintf(msg, sizeof msg,
                  "cqf_two_body_contract_noalloc: this call needs %zu bytes of scratch, the "
                  "fixed scratch array holds %zu bytes (use cqf_two_body_contract)",
                  need * sizeof(double), (size_t)CQF_NOALLOC_SCRATCH_BYTES);
    return cqf::fail(CQF_EINVAL, msg);
  }
  std::lock_guard<std::mutex> lk(B->mu);
  cudaError_t e = cudaSetDevice(B->device);
  if (e != cudaSuccess)
    return cqf::fail(CQF_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  double* ws = nullptr;
  s = scratch_address(B->device, &ws);
  if (s != CQF_OK) return s;
  if (split) return cqf::contract_complex_split_on(B, list.data(), nMat, opts, stats, ws);
  return cqf::contract_core(B, list.data(), nMat, opts, stats, ws, false, nullptr);
}
