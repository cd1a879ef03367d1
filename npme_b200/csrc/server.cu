// Native serving queue: npme_gpu_submit / npme_gpu_poll / npme_gpu_wait.
//
// A server owns one device.  Requests (parameters, geometry, charges and the
// caller's output buffer) are admitted in arrival order while the estimated
// device bytes of the requests in flight stay under the budget; set-up
// threads take the admitted requests (up to setup_batch at a time), give
// each a pooled handle (an idle handle whose buffers fit, given the new
// parameters with npme_gpu_set_params where they differ, else a new one),
// set them all up in one pass of the set-up kernels and upload their
// charges; one dispatch thread runs every set-up request it finds as one
// batched CalcV (npme_gpu_calcv_batch) and hands the batch to a completion
// thread, which copies each result into the caller's buffer, returns the
// handles to the pool and completes the tickets.  Set-up of the next
// requests and the copies of the last batch's results overlap the batch on
// the GPU.  All state is guarded by one mutex; the GPU work itself runs
// outside it.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "internal.h"

bool npme::step_trace_on() {
  static const bool on = std::getenv("NPME_SERVER_TRACE") != nullptr;
  return on;
}

npme::StepTimer::~StepTimer() {
  if (!on) return;
  const double ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  if (ms > 5.0) std::fprintf(stderr, "npme server: %s took %.1f ms (%zu)\n", name, ms, count);
}

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  unsigned long long id = 0;
  npme_params p;
  size_t n = 0;
  const double *coord = nullptr;
  const double *charge = nullptr;
  double *V = nullptr;
  size_t footprint = 0;
  int state = NPME_TICKET_QUEUED;
  int status = NPME_OK;
  std::string err;
  npme_handle *h = nullptr;
  double t_submit = 0, t_admit = 0, t_ready = 0, t_done = 0;
  int batch_size = 0;
};

using Key = std::tuple<int, int, int, int, double, double, double, double, long, long, long, int>;

Key key_of(const npme_params &p) {
  return Key(p.funcType, p.EwaldSplit, p.BnOrder, p.nDeriv, p.Rdir, p.alpha, p.k0_r, p.k0_i,
             p.N1, p.N2, p.N3, p.precision);
}

bool complex_kernel(const npme_params &p) { return p.funcType == NPME_FUNC_HELMHOLTZ; }

// Device bytes a request holds while it is in flight: the spread grid and
// spectrum, the kernel transform and its construction scratch, the per-point
// records of the spreading and of the direct sum, charges and results.
size_t footprint(const npme_params &p, size_t n) {
  const size_t s = p.precision == NPME_PREC_FP32 ? 4 : 8;
  const size_t cx = complex_kernel(p) ? 2 : 1;
  const size_t N = (size_t)p.N1 * p.N2 * p.N3;
  const size_t M = (size_t)(p.N1 / 2 + 1) * (p.N2 / 2 + 1) * (p.N3 / 2 + 1);
  size_t grid = N * s * cx;
  if (cx == 1) grid += (size_t)p.N1 * p.N2 * (p.N3 / 2 + 1) * 2 * s;
  return grid + M * (s * cx + 32) + n * (260 + 40 * cx);
}

}  // namespace

struct npme_server {
  npme_server_config cfg;
  Clock::time_point t0;
  npme_batch *batch = nullptr;
  cudaStream_t stream = nullptr;

  std::mutex mu;
  std::condition_variable cv_setup, cv_ready, cv_done;
  bool stopping = false;
  unsigned long long next_id = 1;
  std::unordered_map<unsigned long long, Request *> tickets;
  std::deque<Request *> waiting, admitted, ready;
  size_t in_flight = 0;
  std::vector<npme_handle *> idle;  // idle handles, any parameters
  size_t idle_bytes = 0;             // device bytes they hold
  npme_server_stats stats;
  std::vector<std::thread> workers;
  std::thread dispatcher, copier;
  // batches run by the dispatch thread whose results the completion thread
  // copies back
  struct Finished {
    std::vector<Request *> rs;
    int rc = NPME_OK;
    std::string msg;
  };
  std::deque<Finished> finished;
  std::condition_variable cv_copy;
  bool dispatch_done = false;
  cudaStream_t copy_stream = nullptr;
  bool reserved = false;  // holds a reservation of the device pool

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  // Moves waiting requests to the set-up queue while the budget allows (a
  // request larger than the budget runs alone).  Caller holds mu.
  void admit() {
    bool any = false;
    while (!waiting.empty()) {
      Request *r = waiting.front();
      if (in_flight != 0 && in_flight + r->footprint > cfg.hbm_budget) break;
      waiting.pop_front();
      in_flight += r->footprint;
      r->t_admit = now();
      admitted.push_back(r);
      any = true;
    }
    if (any) cv_setup.notify_all();
  }

  // An idle handle for a request with parameters p and estimated device
  // bytes `bytes`, among the idle handles of p's precision: one with the same
  // parameters that already holds enough device memory, else the smallest
  // that holds enough (its buffers need not grow), else one with the same
  // parameters, else the largest.  Parameters rarely repeat exactly (the FFT
  // box follows each system's extent), so the fit of the buffers decides.
  // *exact: same parameters.  Caller holds mu.
  npme_handle *take_idle(const npme_params &p, size_t bytes, bool *exact) {
    const Key k = key_of(p);
    long best = -1;
    int best_rank = 4;
    size_t best_bytes = 0;
    for (size_t i = 0; i < idle.size(); i++) {
      const npme_handle *h = idle[i];
      if (h->p.precision != p.precision) continue;
      const bool fits = h->dev_bytes >= bytes, same = key_of(h->p) == k;
      const int rank = same && fits ? 0 : fits ? 1 : same ? 2 : 3;
      const bool better = rank < best_rank ||
                          (rank == best_rank &&
                           (fits ? h->dev_bytes < best_bytes : h->dev_bytes > best_bytes));
      if (better) best = (long)i, best_rank = rank, best_bytes = h->dev_bytes;
    }
    if (best < 0) return nullptr;
    npme_handle *h = idle[best];
    idle[best] = idle.back();
    idle.pop_back();
    idle_bytes -= h->dev_bytes;
    *exact = key_of(h->p) == k;
    return h;
  }

  // Keeps h for reuse; with the pool full (pool_capacity handles, or idle
  // device bytes up to pool_bytes), the smallest of the pool and h is let
  // go.  Caller holds mu; returns the handle to destroy outside the lock,
  // if any.
  npme_handle *give_back(npme_handle *h) {
    if (!h) return nullptr;
    if ((int)idle.size() < cfg.pool_capacity && idle_bytes + h->dev_bytes <= cfg.pool_bytes) {
      idle.push_back(h);
      idle_bytes += h->dev_bytes;
      return nullptr;
    }
    stats.handles_dropped++;
    if (idle.empty()) return h;
    size_t small = 0;
    for (size_t i = 1; i < idle.size(); i++)
      if (idle[i]->dev_bytes < idle[small]->dev_bytes) small = i;
    const size_t swapped = idle_bytes - idle[small]->dev_bytes + h->dev_bytes;
    if (idle[small]->dev_bytes >= h->dev_bytes || swapped > cfg.pool_bytes) return h;
    idle_bytes = swapped;
    std::swap(idle[small], h);
    return h;
  }

  // Completes a request.  Caller holds mu.
  void finish(Request *r, int status, const std::string &msg) {
    r->status = status;
    r->err = msg;
    r->state = status == NPME_OK ? NPME_TICKET_DONE : NPME_TICKET_FAILED;
    r->t_done = now();
    in_flight -= r->footprint;
    if (status == NPME_OK) stats.completed++;
    else stats.failed++;
    admit();
    cv_done.notify_all();
    if (stopping) cv_ready.notify_all();  // the dispatch thread may be done
  }

  void setup_loop();
  void dispatch_loop();
  void copy_loop();
};

void npme_server::setup_loop() {
  cudaSetDevice(cfg.device);
  std::vector<Request *> rs;
  std::vector<npme_handle *> hs, sh;
  std::vector<char> exact;
  std::vector<int> rcs, st;
  std::vector<std::string> msgs;
  std::vector<size_t> sn, si;
  std::vector<const double *> sc;
  for (;;) {
    rs.clear(), hs.clear(), exact.clear();
    {
      std::unique_lock<std::mutex> lk(mu);
      // on shutdown, stay until every request has been admitted and set up
      // a set-up thread runs at most one full batch ahead of the dispatch
      // thread, so handles return to the pool instead of piling up in the
      // ready queue
      cv_setup.wait(lk, [&] {
        return (!admitted.empty() && (int)ready.size() < cfg.max_batch) ||
               (stopping && waiting.empty());
      });
      if (admitted.empty()) return;
      // every admitted request up to setup_batch: one pass of the set-up
      // kernels serves them all
      while (!admitted.empty() && (int)rs.size() < cfg.setup_batch) {
        Request *r = admitted.front();
        admitted.pop_front();
        r->state = NPME_TICKET_SETUP;
        bool ex = false;
        npme_handle *h = take_idle(r->p, r->footprint, &ex);
        if (!h) stats.handles_created++;
        else if (!ex) stats.handles_retuned++;
        rs.push_back(r), hs.push_back(h), exact.push_back(ex);
      }
    }
    const size_t m = rs.size();
    rcs.assign(m, NPME_OK);
    msgs.assign(m, std::string());
    for (size_t k = 0; k < m; k++) {
      npme::StepTimer t("set-up thread: create or retune a handle", 1);
      if (!hs[k]) {
        rcs[k] = npme_gpu_create(&rs[k]->p, &hs[k]);
        if (rcs[k]) {
          char buf[512];
          npme_gpu_last_error(nullptr, buf, sizeof buf);
          msgs[k] = buf;
          hs[k] = nullptr;
        }
      } else if (!exact[k]) {
        rcs[k] = npme_gpu_set_params(hs[k], &rs[k]->p);
        if (rcs[k]) msgs[k] = hs[k]->err;
      }
    }
    sh.clear(), sn.clear(), sc.clear(), si.clear();
    for (size_t k = 0; k < m; k++)
      if (!rcs[k]) sh.push_back(hs[k]), sn.push_back(rs[k]->n), sc.push_back(rs[k]->coord),
            si.push_back(k);
    if (!sh.empty()) {
      npme::StepTimer t("set-up thread: setup_many", sh.size());
      st.assign(sh.size(), NPME_OK);
      npme::setup_many(sh.data(), (int)sh.size(), sn.data(), sc.data(), st.data());
      for (size_t j = 0; j < sh.size(); j++)
        if (st[j]) rcs[si[j]] = st[j], msgs[si[j]] = sh[j]->err;
    }
    // charges: every upload enqueued, then one wait per stream
    npme::StepTimer t_up("set-up thread: charge uploads and waits", m);
    for (size_t k = 0; k < m; k++) {
      if (rcs[k]) continue;
      const size_t words = (complex_kernel(rs[k]->p) ? 2 : 1) * rs[k]->n;
      const cudaError_t e = cudaMemcpyAsync(hs[k]->d_q_in, rs[k]->charge, sizeof(double) * words,
                                            cudaMemcpyHostToDevice, hs[k]->stream);
      if (e != cudaSuccess)
        rcs[k] = NPME_ECUDA, msgs[k] = std::string("charge upload: ") + cudaGetErrorString(e);
    }
    for (size_t k = 0; k < m; k++) {
      if (rcs[k]) continue;
      const cudaError_t e = cudaStreamSynchronize(hs[k]->stream);
      if (e != cudaSuccess)
        rcs[k] = NPME_ECUDA, msgs[k] = std::string("charge upload: ") + cudaGetErrorString(e);
    }
    std::vector<npme_handle *> drop;
    {
      std::lock_guard<std::mutex> lk(mu);
      bool any = false;
      for (size_t k = 0; k < m; k++) {
        Request *r = rs[k];
        if (rcs[k]) {
          if (npme_handle *d = give_back(hs[k])) drop.push_back(d);
          finish(r, rcs[k], msgs[k]);
        } else {
          r->h = hs[k];
          r->t_ready = now();
          r->state = NPME_TICKET_READY;
          ready.push_back(r);
          any = true;
        }
      }
      if (any) cv_ready.notify_one();
    }
    for (npme_handle *d : drop) {
      npme::StepTimer t("set-up thread: destroy a handle", 1);
      npme_gpu_destroy(d);
    }
  }
}

void npme_server::dispatch_loop() {
  cudaSetDevice(cfg.device);
  std::vector<Request *> rs;
  std::vector<npme_handle *> hs;
  std::vector<double *> dV;
  std::vector<const double *> dq;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_ready.wait(lk, [&] {
        return !ready.empty() ||
               (stopping && waiting.empty() && admitted.empty() && in_flight == 0);
      });
      if (ready.empty()) {
        dispatch_done = true;
        cv_copy.notify_all();
        return;
      }
      rs.clear();
      while (!ready.empty() && (int)rs.size() < cfg.max_batch) {
        rs.push_back(ready.front());
        ready.pop_front();
      }
      for (Request *r : rs) r->state = NPME_TICKET_RUNNING;
      if (!admitted.empty()) cv_setup.notify_all();
    }
    hs.clear(), dV.clear(), dq.clear();
    for (Request *r : rs) {
      hs.push_back(r->h);
      dV.push_back(r->h->d_V);
      dq.push_back(r->h->d_q_in);
    }
    int rc;
    {
      npme::StepTimer t("dispatch: batched CalcV enqueue", hs.size());
      rc = npme_gpu_calcv_batch(batch, hs.data(), (int)hs.size(), dV.data(), dq.data(), stream);
    }
    if (!rc) {
      npme::StepTimer t("dispatch: batched CalcV wait", hs.size());
      rc = npme_gpu_batch_sync(batch);
    }
    std::string msg;
    if (rc) {
      char buf[512];
      npme_gpu_batch_last_error(batch, buf, sizeof buf);
      msg = buf;
    }
    // results go back on the completion thread, so their copies overlap
    // the next batch
    {
      std::lock_guard<std::mutex> lk(mu);
      stats.batches++;
      stats.batched_requests += rs.size();
      for (Request *r : rs) r->batch_size = (int)rs.size();
      finished.push_back(Finished{rs, rc, msg});
    }
    cv_copy.notify_one();
  }
}

void npme_server::copy_loop() {
  cudaSetDevice(cfg.device);
  for (;;) {
    Finished f;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv_copy.wait(lk, [&] { return !finished.empty() || dispatch_done; });
      if (finished.empty()) return;
      f = std::move(finished.front());
      finished.pop_front();
    }
    std::vector<int> rcs(f.rs.size(), f.rc);
    std::string msg = f.msg;
    if (!f.rc) {
      npme::StepTimer t("completion: result copies", f.rs.size());
      for (size_t i = 0; i < f.rs.size(); i++) {
        Request *r = f.rs[i];
        const size_t words = (complex_kernel(r->p) ? 8 : 4) * r->n;
        cudaError_t e = cudaMemcpyAsync(r->V, r->h->d_V, sizeof(double) * words,
                                        cudaMemcpyDeviceToHost, copy_stream);
        if (e != cudaSuccess) rcs[i] = NPME_ECUDA;
      }
      cudaError_t e = cudaStreamSynchronize(copy_stream);
      if (e != cudaSuccess) {
        std::fill(rcs.begin(), rcs.end(), (int)NPME_ECUDA);
        msg = std::string("result copy: ") + cudaGetErrorString(e);
      }
    }
    std::vector<npme_handle *> drop;
    {
      std::lock_guard<std::mutex> lk(mu);
      for (size_t i = 0; i < f.rs.size(); i++) {
        Request *r = f.rs[i];
        if (npme_handle *d = give_back(r->h)) drop.push_back(d);
        r->h = nullptr;
        finish(r, rcs[i], rcs[i] ? (msg.empty() ? std::string("result copy failed") : msg) : "");
      }
    }
    for (npme_handle *d : drop) {
      npme::StepTimer t("completion: destroy a handle", 1);
      npme_gpu_destroy(d);
    }
  }
}

extern "C" {

void npme_gpu_server_default_config(npme_server_config *c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->device = 0;
  c->setup_threads = 8;
  c->max_batch = 64;
  c->hbm_budget = 0;
  c->pool_capacity = 256;
  c->setup_batch = 4;
  c->pool_bytes = 0;
}

int npme_gpu_server_create(const npme_server_config *cfg, npme_server **out) {
  if (!cfg || !out) return NPME_EINVAL;
  *out = nullptr;
  if (cfg->setup_threads < 1 || cfg->setup_threads > 256 || cfg->max_batch < 1 ||
      cfg->pool_capacity < 0 || cfg->setup_batch < 1 || cfg->setup_batch > 1024)
    return NPME_EINVAL;
  npme_server *s = new (std::nothrow) npme_server;
  if (!s) return NPME_ENOMEM;
  s->cfg = *cfg;
  s->t0 = Clock::now();
  memset(&s->stats, 0, sizeof(s->stats));
  cudaError_t e = cudaSetDevice(cfg->device);
  if (e == cudaSuccess && (s->cfg.hbm_budget == 0 || s->cfg.pool_bytes == 0)) {
    size_t fr = 0, tot = 0;
    e = cudaMemGetInfo(&fr, &tot);
    if (s->cfg.hbm_budget == 0) s->cfg.hbm_budget = fr / 2;
    if (s->cfg.pool_bytes == 0) s->cfg.pool_bytes = fr / 2;
  }
  // the idle pool's budget reserved in the device pool now, so that serving
  // never waits for the pool to grow
  if (e == cudaSuccess && npme::pool_reserve(cfg->device, s->cfg.pool_bytes) == NPME_OK)
    s->reserved = true;
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    if (s->stream) cudaStreamDestroy(s->stream);
    if (s->reserved) npme::pool_unreserve(cfg->device);
    delete s;
    return NPME_ECUDA;
  }
  int rc = npme_gpu_batch_create(cfg->device, &s->batch);
  if (rc) {
    cudaStreamDestroy(s->stream);
    cudaStreamDestroy(s->copy_stream);
    if (s->reserved) npme::pool_unreserve(cfg->device);
    delete s;
    return rc;
  }
  for (int i = 0; i < cfg->setup_threads; i++) s->workers.emplace_back([s] { s->setup_loop(); });
  s->dispatcher = std::thread([s] { s->dispatch_loop(); });
  s->copier = std::thread([s] { s->copy_loop(); });
  *out = s;
  return NPME_OK;
}

int npme_gpu_submit(npme_server *s, const npme_params *p, size_t n, const double *coord,
                    const double *charge, double *V, unsigned long long *ticket) {
  if (!s || !p || !coord || !charge || !V || !ticket || n == 0) return NPME_EINVAL;
  if (p->device != s->cfg.device) return NPME_EINVAL;
  Request *r = new (std::nothrow) Request;
  if (!r) return NPME_ENOMEM;
  r->p = *p;
  r->n = n;
  r->coord = coord, r->charge = charge, r->V = V;
  r->footprint = footprint(*p, n);
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stopping) {
    delete r;
    return NPME_ESTATE;
  }
  r->id = s->next_id++;
  r->t_submit = s->now();
  s->tickets[r->id] = r;
  s->waiting.push_back(r);
  s->stats.submitted++;
  s->admit();
  *ticket = r->id;
  return NPME_OK;
}

int npme_gpu_poll(npme_server *s, unsigned long long ticket, int *state) {
  if (!s || !state) return NPME_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return NPME_EINVAL;
  *state = it->second->state;
  return NPME_OK;
}

int npme_gpu_wait(npme_server *s, unsigned long long ticket, double timeout_s) {
  if (!s) return NPME_EINVAL;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return NPME_EINVAL;
  Request *r = it->second;
  auto done = [&] { return r->state == NPME_TICKET_DONE || r->state == NPME_TICKET_FAILED; };
  if (timeout_s < 0) s->cv_done.wait(lk, done);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done))
    return NPME_ETIMEOUT;
  return r->status;
}

int npme_gpu_ticket_info(npme_server *s, unsigned long long ticket, npme_ticket_info *info) {
  if (!s || !info) return NPME_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return NPME_EINVAL;
  const Request *r = it->second;
  info->state = r->state;
  info->status = r->status;
  info->t_submit = r->t_submit;
  info->t_admit = r->t_admit;
  info->t_ready = r->t_ready;
  info->t_done = r->t_done;
  info->batch_size = r->batch_size;
  info->footprint = r->footprint;
  strncpy(info->error, r->err.c_str(), sizeof(info->error) - 1);
  info->error[sizeof(info->error) - 1] = 0;
  return NPME_OK;
}

int npme_gpu_release_ticket(npme_server *s, unsigned long long ticket) {
  if (!s) return NPME_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return NPME_EINVAL;
  Request *r = it->second;
  if (r->state != NPME_TICKET_DONE && r->state != NPME_TICKET_FAILED) return NPME_ESTATE;
  s->tickets.erase(it);
  delete r;
  return NPME_OK;
}

int npme_gpu_server_stats(npme_server *s, npme_server_stats *st) {
  if (!s || !st) return NPME_EINVAL;
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->stats;
  st->idle_handles = (int)s->idle.size();
  st->in_flight_bytes = s->in_flight;
  st->hbm_budget = s->cfg.hbm_budget;
  st->clock_s = s->now();
  st->idle_bytes = s->idle_bytes;
  st->pool_bytes = s->cfg.pool_bytes;
  return NPME_OK;
}

int npme_gpu_server_destroy(npme_server *s) {
  if (!s) return NPME_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_setup.notify_all();
  s->cv_ready.notify_all();
  // requests still waiting for admission are admitted as the ones in flight
  // complete; every submitted request completes before the threads end
  for (;;) {
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->waiting.empty() && s->admitted.empty() && s->ready.empty() && s->in_flight == 0) break;
    s->cv_done.wait_for(lk, std::chrono::milliseconds(10));
  }
  s->cv_setup.notify_all();
  s->cv_ready.notify_all();
  for (auto &t : s->workers) t.join();
  s->dispatcher.join();
  s->copier.join();
  for (npme_handle *h : s->idle) npme_gpu_destroy(h);
  for (auto &kv : s->tickets) delete kv.second;
  npme_gpu_batch_destroy(s->batch);
  cudaStreamDestroy(s->stream);
  cudaStreamDestroy(s->copy_stream);
  if (s->reserved) npme::pool_unreserve(s->cfg.device);
  delete s;
  return NPME_OK;
}

}  // extern "C"
