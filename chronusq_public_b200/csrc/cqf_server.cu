// Fock-build server: continuous batching of closed-shell Fock builds of any
// basis size on one GPU (cqf_server_* in cqfock.h).
//
// Requests wait in one FIFO queue.  `slots` worker threads each take the
// queue's head when it is admissible -- its device-memory footprint fits in
// the budget left by the running requests and the idle cached bases (idle
// bases are evicted, least recently used first, to make room; a request alone
// on the GPU is always admitted) -- run it (basis set-up unless its geometry
// is cached, then J and K on the basis' own stream, then G = 2J - xHFX K) and
// put its basis into the cache.  Only host threads and the C ABI's own calls
// are used here; the device work is cqf_basis_create / cqf_two_body_contract.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cqf_internal.hpp"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

int nfunc(int l, int pure) { return pure ? 2 * l + 1 : (l + 1) * (l + 2) / 2; }

struct Request {
  long long id = 0;
  std::vector<cqf_shell> shells;
  std::vector<double> prim;  // alpha and coeff storage of the copied shells
  double thresh = 1e-12;
  std::vector<double> D;
  double* G = nullptr;
  double xHFX = 1.0;
  int precision = CQF_FP64;
  double cutoff = 0.0;
  int N = 0;
  unsigned long long footprint = 0;
  std::string key;  // exact geometry + basis key of the basis cache
  Clock::time_point t_submit, t_admit, t_setup, t_done;
  bool done = false;
  cqf_status status = CQF_OK;
  std::string err;
};

struct CacheEntry {
  cqf_basis* basis;
  unsigned long long mem;
};

}  // namespace

struct cqf_server {
  cqf_server_opts opts{};
  std::mutex mu;
  std::condition_variable cv_work;  // workers: queue changed or memory freed
  std::condition_variable cv_done;  // waiters: a request completed
  std::deque<std::shared_ptr<Request>> queue;
  std::unordered_map<long long, std::shared_ptr<Request>> reqs;
  // idle cached bases, most recently used at the back
  std::list<std::pair<std::string, CacheEntry>> cache;
  unsigned long long cache_mem = 0, in_use = 0;
  int inflight = 0, peak_inflight = 0;
  long long next_id = 1, submitted = 0, completed = 0, failed = 0;
  std::vector<double> latencies;
  bool stop = false;
  std::vector<std::thread> workers;

  // Under mu: true when the queue's head may start now; evicted bases are
  // appended to `drop` (destroyed by the caller outside the lock).
  bool admissible(std::vector<cqf_basis*>& drop) {
    if (queue.empty()) return false;
    const Request& r = *queue.front();
    unsigned long long cached = 0;
    for (auto& e : cache)
      if (e.first == r.key) cached = e.second.mem;
    auto free_now = [&] {
      const unsigned long long used = in_use + cache_mem;
      return used >= opts.mem_budget ? 0ull : opts.mem_budget - used;
    };
    const unsigned long long need = r.footprint > cached ? r.footprint - cached : 0;
    while (free_now() < need) {
      auto it = std::find_if(cache.begin(), cache.end(),
                             [&](const std::pair<std::string, CacheEntry>& e) {
                               return e.first != r.key;
                             });
      if (it == cache.end()) break;
      cache_mem -= it->second.mem;
      drop.push_back(it->second.basis);
      cache.erase(it);
    }
    return free_now() >= need || inflight == 0;
  }

  void worker() {
    for (;;) {
      std::shared_ptr<Request> r;
      cqf_basis* B = nullptr;
      std::vector<cqf_basis*> drop;
      {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
          if (admissible(drop)) break;
          if (stop && queue.empty()) break;
          if (!drop.empty()) {
            lk.unlock();
            for (cqf_basis* b : drop) cqf_basis_destroy(b);
            drop.clear();
            lk.lock();
            continue;
          }
          cv_work.wait(lk);
        }
        if (queue.empty()) {  // stopping
          lk.unlock();
          for (cqf_basis* b : drop) cqf_basis_destroy(b);
          return;
        }
        r = queue.front();
        queue.pop_front();
        for (auto it = cache.begin(); it != cache.end(); ++it)
          if (it->first == r->key) {
            B = it->second.basis;
            cache_mem -= it->second.mem;
            cache.erase(it);
            break;
          }
        in_use += r->footprint;
        inflight++;
        peak_inflight = std::max(peak_inflight, inflight);
        r->t_admit = Clock::now();
      }
      for (cqf_basis* b : drop) cqf_basis_destroy(b);
      run(*r, B);
    }
  }

  void run(Request& r, cqf_basis* B) {
    cqf_status st = CQF_OK;
    std::string err;
    if (!B) {
      st = cqf_basis_create(r.shells.data(), (int)r.shells.size(), r.thresh, opts.device, &B);
      if (st != CQF_OK) err = cqf_last_error();
    }
    r.t_setup = Clock::now();
    if (st == CQF_OK) {
      const size_t NN = (size_t)r.N * r.N;
      std::vector<double> J(NN, 0.0), K(NN, 0.0);
      cqf_contraction list[2];
      list[0] = {r.D.data(), J.data(), 1, CQF_COULOMB};
      list[1] = {r.D.data(), K.data(), 1, CQF_EXCHANGE};
      cqf_opts o;
      cqf_opts_default(&o);
      o.precision = r.precision;
      o.fp32_cutoff = r.cutoff;
      st = cqf_two_body_contract(B, list, 2, &o, nullptr);
      if (st != CQF_OK) {
        err = cqf_last_error();
      } else {
        for (size_t i = 0; i < NN; i++) r.G[i] = 2.0 * J[i] - r.xHFX * K[i];
      }
    }
    std::vector<cqf_basis*> drop;
    {
      std::lock_guard<std::mutex> lk(mu);
      r.t_done = Clock::now();
      r.status = st;
      r.err = err;
      r.done = true;
      in_use -= r.footprint;
      inflight--;
      if (st == CQF_OK) {
        completed++;
        latencies.push_back(ms_between(r.t_submit, r.t_done));
      } else {
        failed++;
      }
      if (B) {
        // keep the basis (one entry per geometry), most recent last
        bool dup = false;
        for (auto& e : cache) dup |= e.first == r.key;
        if (dup || st != CQF_OK || opts.cache_entries <= 0) {
          drop.push_back(B);
        } else {
          cache.push_back({r.key, CacheEntry{B, r.footprint}});
          cache_mem += r.footprint;
          while ((int)cache.size() > opts.cache_entries) {
            cache_mem -= cache.front().second.mem;
            drop.push_back(cache.front().second.basis);
            cache.pop_front();
          }
        }
      }
    }
    for (cqf_basis* b : drop) cqf_basis_destroy(b);
    cv_done.notify_all();
    cv_work.notify_all();
  }
};

extern "C" {

void cqf_server_opts_default(cqf_server_opts* o) {
  if (!o) return;
  o->device = 0;
  o->slots = 8;
  o->mem_budget = 8ull << 30;
  o->cache_entries = 16;
}

unsigned long long cqf_fock_footprint(const cqf_shell* shells, int nshell) {
  if (!shells || nshell <= 0) return 0;
  unsigned long long N = 0, nc = 0, maxp = 0;
  for (int s = 0; s < nshell; s++) {
    N += nfunc(shells[s].l, shells[s].pure);
    nc += (unsigned long long)(shells[s].l + 1) * (shells[s].l + 2) / 2;
    maxp = std::max<unsigned long long>(maxp, (unsigned long long)std::max(0, shells[s].nprim));
  }
  const unsigned long long ns = nshell, npair = ns * (ns + 1) / 2, nmat = 2;
  // per pair: its record and window bound; per primitive pair: the record
  // (112 B) and its FP32 copy (48 B), its Schwarz bound and the
  // tile-interleaved ket copy (13 doubles + 13 floats)
  const unsigned long long pairs =
      npair * (72 + (112 + 48 + 8 + 104 + 52) * maxp * maxp) + ns * ns * 8 + 300000;
  // workspace: densities and accumulators (spherical, Cartesian, FP32
  // copy), norms, and the class kernels' quartet masks and word lists
  // (16 B per mask word -- 32 quartets of a bra pair and a ket tile -- in
  // each of the three launch streams' regions, at most 2^18 words each)
  const unsigned long long maskw = std::min<unsigned long long>(
      npair * ((npair + 31) / 32), 1ull << 18);
  const unsigned long long masks = 3 * 16 * maskw;
  const unsigned long long ws =
      8 * (2 * nmat * N * N + 2 * nmat * nc * nc + (nmat + 1) * ns * ns) + 4 * nmat * nc * nc +
      masks;
  return pairs + ws;
}

cqf_status cqf_server_create(const cqf_server_opts* opts, cqf_server** out) {
  if (!out) return cqf::fail(CQF_EINVAL, "cqf_server_create: null argument");
  *out = nullptr;
  cqf_server_opts o;
  cqf_server_opts_default(&o);
  if (opts) o = *opts;
  if (o.slots <= 0) return cqf::fail(CQF_EINVAL, "cqf_server_create: slots must be positive");
  auto* S = new cqf_server();
  S->opts = o;
  for (int i = 0; i < o.slots; i++) S->workers.emplace_back([S] { S->worker(); });
  *out = S;
  return CQF_OK;
}

cqf_status cqf_server_submit(cqf_server* S, const cqf_fock_request* q, long long* id) {
  if (!S || !q || !id || !q->shells || q->nshell <= 0 || !q->D || !q->G)
    return cqf::fail(CQF_EINVAL, "cqf_server_submit: null argument");
  auto r = std::make_shared<Request>();
  size_t nprim = 0;
  for (int s = 0; s < q->nshell; s++) {
    const cqf_shell& c = q->shells[s];
    if (c.nprim <= 0 || !c.alpha || !c.coeff)
      return cqf::fail(CQF_EINVAL, "cqf_server_submit: empty shell");
    nprim += c.nprim;
    r->N += nfunc(c.l, c.pure);
  }
  // copy the shells: [alpha | coeff] per shell, in order
  r->prim.resize(2 * nprim);
  r->shells.assign(q->shells, q->shells + q->nshell);
  size_t off = 0;
  std::string key;
  key.reserve(q->nshell * 48 + nprim * 16 + 8);
  auto put = [&](const void* p, size_t n) { key.append(static_cast<const char*>(p), n); };
  put(&q->thresh_schwarz, sizeof(double));
  for (int s = 0; s < q->nshell; s++) {
    cqf_shell& c = r->shells[s];
    std::copy(c.alpha, c.alpha + c.nprim, r->prim.begin() + off);
    std::copy(c.coeff, c.coeff + c.nprim, r->prim.begin() + off + c.nprim);
    c.alpha = r->prim.data() + off;
    c.coeff = r->prim.data() + off + c.nprim;
    off += 2 * c.nprim;
    put(&c.l, sizeof(int));
    put(&c.pure, sizeof(int));
    put(&c.nprim, sizeof(int));
    put(c.origin, 3 * sizeof(double));
    put(c.alpha, c.nprim * sizeof(double));
    put(c.coeff, c.nprim * sizeof(double));
  }
  r->key = std::move(key);
  r->thresh = q->thresh_schwarz;
  r->D.assign(q->D, q->D + (size_t)r->N * r->N);
  r->G = q->G;
  r->xHFX = q->xHFX;
  r->precision = q->precision;
  r->cutoff = q->fp32_cutoff;
  r->footprint = cqf_fock_footprint(q->shells, q->nshell);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return cqf::fail(CQF_EINVAL, "cqf_server_submit: server is shutting down");
    r->id = S->next_id++;
    r->t_submit = Clock::now();
    S->reqs[r->id] = r;
    S->queue.push_back(r);
    S->submitted++;
    *id = r->id;
  }
  S->cv_work.notify_all();
  return CQF_OK;
}

cqf_status cqf_server_wait(cqf_server* S, long long id, double timeout_s, cqf_request_info* info) {
  if (!S) return cqf::fail(CQF_EINVAL, "cqf_server_wait: null server");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  if (it == S->reqs.end()) return cqf::fail(CQF_EINVAL, "cqf_server_wait: unknown request id");
  std::shared_ptr<Request> r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_s < 0) {
    S->cv_done.wait(lk, ready);
  } else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    return cqf::fail(CQF_ETIMEDOUT, "cqf_server_wait: request still running");
  }
  if (info) {
    info->status = r->status;
    info->queue_ms = ms_between(r->t_submit, r->t_admit);
    info->setup_ms = ms_between(r->t_admit, r->t_setup);
    info->build_ms = ms_between(r->t_setup, r->t_done);
    info->latency_ms = ms_between(r->t_submit, r->t_done);
  }
  S->reqs.erase(id);
  if (r->status != CQF_OK) return cqf::fail(r->status, r->err);
  return CQF_OK;
}

cqf_status cqf_server_get_stats(cqf_server* S, cqf_server_stats* st) {
  if (!S || !st) return cqf::fail(CQF_EINVAL, "cqf_server_get_stats: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  st->submitted = S->submitted;
  st->completed = S->completed;
  st->failed = S->failed;
  st->peak_inflight = S->peak_inflight;
  st->p50_ms = st->p99_ms = st->mean_ms = 0.0;
  std::vector<double> v = S->latencies;
  if (!v.empty()) {
    std::sort(v.begin(), v.end());
    // linear interpolation between closest ranks
    auto pct = [&](double p) {
      const double x = p / 100.0 * (double)(v.size() - 1);
      const size_t i = (size_t)x;
      const double f = x - (double)i;
      return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
    };
    st->p50_ms = pct(50.0);
    st->p99_ms = pct(99.0);
    double s = 0.0;
    for (double x : v) s += x;
    st->mean_ms = s / (double)v.size();
  }
  return CQF_OK;
}

cqf_status cqf_server_destroy(cqf_server* S) {
  if (!S) return CQF_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->workers) t.join();
  for (auto& e : S->cache) cqf_basis_destroy(e.second.basis);
  delete S;
  return CQF_OK;
}

}  // extern "C"
