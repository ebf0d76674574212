// Serving loop over the batched solver: continuous batching of independent FMM solves.
//
// Requests (bodies + expansion order) are copied in at submit and queued; each takes the
// opening angle set for its order (fmm_b200_server_set_theta; else the configuration's), so
// that every order can be held to the same accuracy.  A scheduler thread forms batches from
// whatever is pending whenever a worker is free: the oldest request decides the order P (and
// angle), later requests of the same P and angle join in arrival order while the
// batch fits the free part of the device-memory budget, the batch-size limit and
// kBatchBodies bodies (a larger request rides alone).  Each
// worker owns a CUDA stream and one solver handle per order, so batches on different
// workers overlap on the GPU; requests that arrive while batches run are admitted into the
// next batch as soon as a worker and budget free up.  A request's result does not depend on
// which batch it rode in (fmm_b200_solve_batch_*: every solve is computed as it is alone).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/exafmm_b200.h"

namespace {

using Clock = std::chrono::steady_clock;

// Bodies per batch (unless one request alone is larger).  A batch of this size fills the
// GPU; the cap keeps the batches, and so each worker's pinned staging and its handles'
// device arrays, within sizes reached in the first passes, so that later passes do not
// stop to allocate (a pinned allocation of a few hundred MB takes tens of ms).
constexpr size_t kBatchBodies = (size_t)1 << 21;

struct Request {
  long long id = 0;
  int n = 0, P = 0;
  double theta = 0;  // opening angle of the request's order when it was submitted
  std::vector<double> x, q, p, f;
  size_t bytes = 0;
  int status = FMM_OK;
  bool done = false;
  Clock::time_point t_submit, t_start, t_done;
};

struct Worker {
  int index = 0;
  cudaStream_t stream = nullptr;
  std::map<std::pair<int, double>, fmm_b200_solver*> handles;  // per (order, theta)
  std::vector<std::shared_ptr<Request>> batch;
  bool busy = false;
  std::thread thread;
  // pinned staging for the batch's inputs / outputs; staging it has grown out of is kept
  // until the worker exits (cudaFreeHost synchronises the device, stalling the other workers)
  double* pin = nullptr;
  size_t pin_cap = 0;
  std::vector<double*> pin_retired;
};

}  // namespace

struct fmm_b200_server {
  fmm_b200_config cfg;
  size_t budget = 0, in_flight = 0;
  int max_batch = 256;
  std::mutex mu;
  std::condition_variable cv;   // scheduler wakes on submit / worker done
  std::condition_variable done_cv;
  std::deque<std::shared_ptr<Request>> pending;
  std::unordered_map<long long, std::shared_ptr<Request>> all;
  std::vector<std::unique_ptr<Worker>> workers;
  std::thread scheduler;
  bool stop = false;
  bool paused = false;  // fmm_b200_server_trim holds new batches back while it frees
  long long next_id = 1;
  long long completed = 0, bodies_done = 0, batches = 0;
  // worker seconds spent staging inputs, in the batched solve, and copying results out
  double t_stage = 0, t_solve = 0, t_unstage = 0;
  std::string err;
  std::map<int, double> theta_of;  // per-order opening angle (fmm_b200_server_set_theta)
};

namespace {

// Host copies of request data (into the worker's pinned staging and out of it), split over
// a few threads when they are large: a burst of 7 M bodies moves ~0.5 GB through them, which
// one thread copies at ~10 GB/s.
struct CopyJob {
  void* dst;
  const void* src;
  size_t bytes;
};

void copy_jobs(const std::vector<CopyJob>& jobs) {
  size_t total = 0;
  for (const auto& j : jobs) total += j.bytes;
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = (int)std::min<size_t>(std::min(8u, hw), total >> 22);  // >= 4 MB a thread
  auto run = [&](size_t lo, size_t hi) {  // the byte range [lo, hi) of the concatenated jobs
    size_t base = 0;
    for (const auto& j : jobs) {
      const size_t a = std::max(lo, base), b = std::min(hi, base + j.bytes);
      if (a < b)
        std::memcpy(static_cast<char*>(j.dst) + (a - base),
                    static_cast<const char*>(j.src) + (a - base), b - a);
      base += j.bytes;
    }
  };
  if (nt <= 1) {
    run(0, total);
    return;
  }
  std::vector<std::thread> ts;
  const size_t per = (total + nt - 1) / nt;
  for (int t = 1; t < nt; t++) ts.emplace_back(run, t * per, std::min(total, (t + 1) * per));
  run(0, std::min(total, per));
  for (auto& t : ts) t.join();
}

// device memory of one solve in the batched solver (bodies, sort scratch, tree, expansions,
// interaction lists), an upper-end estimate used for admission
size_t estimate_bytes(const fmm_b200_config& c, int n, int P) {
  const size_t ncoef = c.basis == FMM_SPHERICAL ? (size_t)P * (P + 1) : (size_t)P * (P + 1) * (P + 2) / 6;
  const size_t real = c.precision == FMM_FP64 ? 8 : 4;
  const size_t cells = 2 * (size_t)n / std::max(1, c.ncrit) + 64;
  return (size_t)n * (8 * real + 48) + cells * (2 * ncoef * real + 160) + cells * 400 * 8;
}

// A new handle solves two synthetic batches of kBatchBodies bodies before its first
// request: one Plummer sphere (a deep tree) and 256 cubes of equal size (many shallow trees,
// the most cells and list entries per body), so that its device arrays reach the sizes of
// a full batch now rather than one growth at a time during later passes.  Deterministic
// (a 64-bit linear congruential generator); uses the worker's pinned staging.
void presize(fmm_b200_solver* h, double* pin) {
  const int n = (int)kBatchBodies;
  double *x = pin, *q = x + 3 * (size_t)n, *p = q + n, *f = p + n;
  unsigned long long st = 0x9e3779b97f4a7c15ULL;
  auto uni = [&st]() {  // [0, 1)
    st = st * 6364136223846793005ULL + 1442695040888963407ULL;
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int i = 0; i < n; i++) {  // Plummer, a = 1, radii clipped at 10
    double r;
    do {
      const double u = uni();
      r = u > 0 ? 1.0 / std::sqrt(std::pow(u, -2.0 / 3.0) - 1.0) : 1e9;
    } while (!(r < 10.0));
    const double ct = 2 * uni() - 1, ph = 2 * 3.141592653589793 * uni();
    const double st2 = std::sqrt(1 - ct * ct);
    x[3 * i] = r * st2 * std::cos(ph);
    x[3 * i + 1] = r * st2 * std::sin(ph);
    x[3 * i + 2] = r * ct;
    q[i] = 1.0 / n;
  }
  int one = n;
  if (fmm_b200_solve_batch_host(h, 1, &one, x, q, p, f) != FMM_OK) return;
  std::vector<int> counts(256, n / 256);
  for (int i = 0; i < n; i++) {
    for (int d = 0; d < 3; d++) x[3 * i + d] = 2 * uni() - 1;
    q[i] = 2 * uni() - 1;
  }
  fmm_b200_solve_batch_host(h, 256, counts.data(), x, q, p, f);
}

void worker_loop(fmm_b200_server* S, Worker* W) {
  cudaSetDevice(S->cfg.device);
  cudaStreamCreateWithFlags(&W->stream, cudaStreamNonBlocking);
  // staging for a full batch (x, q, p, f: 8 doubles a body), allocated before any request
  if (cudaMallocHost((void**)&W->pin, 8 * kBatchBodies * sizeof(double)) == cudaSuccess)
    W->pin_cap = 8 * kBatchBodies;
  else
    W->pin = nullptr;
  for (;;) {
    std::vector<std::shared_ptr<Request>> batch;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv.wait(lk, [&] { return S->stop || !W->batch.empty(); });
      if (W->batch.empty() && S->stop) break;
      batch.swap(W->batch);
    }
    const int P = batch.front()->P;
    const double theta = batch.front()->theta;
    int rc = FMM_OK;
    fmm_b200_solver*& h = W->handles[{P, theta}];
    if (!h) {
      fmm_b200_config c = S->cfg;
      c.P = P;
      c.theta = theta;
      rc = fmm_b200_create(&c, &h);
      if (rc == FMM_OK) rc = fmm_b200_set_stream(h, W->stream);
      if (rc != FMM_OK) h = nullptr;
      if (h && W->pin && W->pin_cap >= 8 * kBatchBodies) presize(h, W->pin);
    }
    std::vector<int> counts;
    size_t n = 0;
    for (auto& r : batch) {
      counts.push_back(r->n);
      n += r->n;
    }
    if (rc == FMM_OK) {
      if (W->pin_cap < 8 * n) {
        if (W->pin) W->pin_retired.push_back(W->pin);
        W->pin_cap = 12 * n + 1024;  // 1.5x the need: fewer growths
        if (cudaMallocHost((void**)&W->pin, W->pin_cap * sizeof(double)) != cudaSuccess) {
          W->pin = nullptr;
          W->pin_cap = 0;
          rc = FMM_ERR_NO_MEMORY;
        }
      }
    }
    const auto t_start = Clock::now();
    auto t_a = t_start, t_b = t_start;
    if (rc == FMM_OK) {
      double *x = W->pin, *q = x + 3 * n, *p = q + n, *f = p + n;
      std::vector<CopyJob> jobs;
      size_t o = 0;
      for (auto& r : batch) {
        jobs.push_back({x + 3 * o, r->x.data(), sizeof(double) * 3 * r->n});
        jobs.push_back({q + o, r->q.data(), sizeof(double) * r->n});
        o += r->n;
      }
      copy_jobs(jobs);
      t_a = Clock::now();
      rc = fmm_b200_solve_batch_host(h, (int)counts.size(), counts.data(), x, q, p, f);
      t_b = Clock::now();
      if (rc == FMM_OK) {
        jobs.clear();
        o = 0;
        for (auto& r : batch) {
          r->p.resize(r->n);
          r->f.resize(3 * (size_t)r->n);
          jobs.push_back({r->p.data(), p + o, sizeof(double) * r->n});
          jobs.push_back({r->f.data(), f + 3 * o, sizeof(double) * 3 * r->n});
          o += r->n;
        }
        copy_jobs(jobs);
      }
    }
    const auto t_done = Clock::now();
    {
      std::lock_guard<std::mutex> lk(S->mu);
      for (auto& r : batch) {
        r->status = rc;
        r->done = true;
        r->t_start = t_start;
        r->t_done = t_done;
        S->in_flight -= r->bytes;
        S->completed++;
        S->bodies_done += r->n;
      }
      S->batches++;
      S->t_stage += std::chrono::duration<double>(t_a - t_start).count();
      S->t_solve += std::chrono::duration<double>(t_b - t_a).count();
      S->t_unstage += std::chrono::duration<double>(t_done - t_b).count();
      W->busy = false;
      if (rc != FMM_OK && h) S->err = fmm_b200_last_error(h);
    }
    S->cv.notify_all();
    S->done_cv.notify_all();
  }
  for (auto& kv : W->handles)
    if (kv.second) fmm_b200_destroy(kv.second);
  if (W->pin) cudaFreeHost(W->pin);
  for (double* q : W->pin_retired) cudaFreeHost(q);
  cudaStreamDestroy(W->stream);
}

void scheduler_loop(fmm_b200_server* S) {
  std::unique_lock<std::mutex> lk(S->mu);
  for (;;) {
    Worker* free_w = nullptr;
    S->cv.wait(lk, [&] {
      if (S->stop) return true;
      if (S->pending.empty() || S->paused) return false;
      free_w = nullptr;
      for (auto& w : S->workers)
        if (!w->busy) {
          free_w = w.get();
          break;
        }
      return free_w && S->in_flight + S->pending.front()->bytes <= S->budget;
    });
    if (S->stop) break;
    // batch: the oldest request's order (and opening angle), later ones of the same order
    // and angle in arrival order
    const int P = S->pending.front()->P;
    const double theta = S->pending.front()->theta;
    std::vector<std::shared_ptr<Request>> batch;
    size_t bodies = 0;
    for (auto it = S->pending.begin(); it != S->pending.end() && (int)batch.size() < S->max_batch;) {
      if ((*it)->P == P && (*it)->theta == theta && S->in_flight + (*it)->bytes <= S->budget &&
          (batch.empty() || bodies + (size_t)(*it)->n <= kBatchBodies)) {
        S->in_flight += (*it)->bytes;
        bodies += (size_t)(*it)->n;
        batch.push_back(*it);
        it = S->pending.erase(it);
      } else {
        ++it;
      }
    }
    free_w->busy = true;
    free_w->batch = std::move(batch);
    S->cv.notify_all();
  }
}

}  // namespace

extern "C" {

int fmm_b200_server_create(const fmm_b200_config* cfg, double hbm_budget_bytes, int nworkers,
                           int max_batch, fmm_b200_server** out) {
  if (!cfg || !out || nworkers < 1 || max_batch < 1 || !(hbm_budget_bytes > 0))
    return FMM_ERR_INVALID;
  // validate the configuration (and the device) once up front; the order comes with each
  // request, so the probe takes one the basis is compiled for if cfg->P is not
  fmm_b200_config pc = *cfg;
  int ords[64];
  const int nord = std::min(fmm_b200_supported_orders(pc.basis, ords, 64), 64);
  if (nord > 0 && std::find(ords, ords + nord, pc.P) == ords + nord) pc.P = ords[0];
  fmm_b200_solver* probe = nullptr;
  int rc = fmm_b200_create(&pc, &probe);
  if (rc != FMM_OK) return rc;
  fmm_b200_destroy(probe);
  fmm_b200_server* S = new fmm_b200_server();
  S->cfg = *cfg;
  S->budget = (size_t)hbm_budget_bytes;
  S->max_batch = max_batch;
  for (int i = 0; i < nworkers; i++) {
    S->workers.emplace_back(new Worker());
    S->workers.back()->index = i;
  }
  for (auto& w : S->workers) w->thread = std::thread(worker_loop, S, w.get());
  S->scheduler = std::thread(scheduler_loop, S);
  *out = S;
  return FMM_OK;
}

int fmm_b200_server_submit(fmm_b200_server* S, int n, const double* x, const double* q, int P,
                           long long* id) {
  if (!S || n < 1 || !x || !q || !id) return FMM_ERR_INVALID;
  auto r = std::make_shared<Request>();
  r->n = n;
  r->P = P;
  r->bytes = estimate_bytes(S->cfg, n, P);
  if (r->bytes > S->budget) return FMM_ERR_NO_MEMORY;  // never fits: reject, do not queue
  int buf[64];
  const int nord = fmm_b200_supported_orders(S->cfg.basis, buf, 64);
  if (std::find(buf, buf + std::min(nord, 64), P) == buf + std::min(nord, 64)) return FMM_ERR_INVALID;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto th = S->theta_of.find(P);
    r->theta = th == S->theta_of.end() ? S->cfg.theta : th->second;
  }
  r->x.resize(3 * (size_t)n);
  r->q.resize(n);
  copy_jobs({{r->x.data(), x, sizeof(double) * 3 * n}, {r->q.data(), q, sizeof(double) * n}});
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return FMM_ERR_STATE;
    r->id = S->next_id++;
    S->pending.push_back(r);
    S->all[r->id] = r;
    *id = r->id;
  }
  S->cv.notify_all();
  return FMM_OK;
}

int fmm_b200_server_set_theta(fmm_b200_server* S, int P, double theta) {
  if (!S || !(theta > 0) || !(theta < 1)) return FMM_ERR_INVALID;
  int buf[64];
  const int nord = std::min(fmm_b200_supported_orders(S->cfg.basis, buf, 64), 64);
  if (std::find(buf, buf + nord, P) == buf + nord) return FMM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  S->theta_of[P] = theta;
  return FMM_OK;
}

int fmm_b200_server_poll(fmm_b200_server* S, long long id, int* done) {
  if (!S || !done) return FMM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->all.find(id);
  if (it == S->all.end()) return FMM_ERR_INVALID;
  *done = it->second->done ? 1 : 0;
  return FMM_OK;
}

int fmm_b200_server_wait(fmm_b200_server* S, long long id, double* p, double* f,
                         double* latency_s, double* queue_s) {
  if (!S) return FMM_ERR_INVALID;
  std::shared_ptr<Request> r;
  {
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return FMM_ERR_INVALID;
    r = it->second;
    S->done_cv.wait(lk, [&] { return r->done; });
    S->all.erase(it);
  }
  if (r->status != FMM_OK) return r->status;
  std::vector<CopyJob> out;
  if (p) out.push_back({p, r->p.data(), sizeof(double) * r->n});
  if (f) out.push_back({f, r->f.data(), sizeof(double) * 3 * r->n});
  copy_jobs(out);
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  if (queue_s) *queue_s = std::chrono::duration<double>(r->t_start - r->t_submit).count();
  return FMM_OK;
}

int fmm_b200_server_stats(fmm_b200_server* S, long long* completed, long long* bodies,
                          long long* batches, int* pending) {
  if (!S) return FMM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  if (completed) *completed = S->completed;
  if (bodies) *bodies = S->bodies_done;
  if (batches) *batches = S->batches;
  if (pending) *pending = (int)S->pending.size();
  return FMM_OK;
}

int fmm_b200_server_profile(fmm_b200_server* S, double* stage_s, double* solve_s,
                            double* unstage_s) {
  if (!S) return FMM_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->mu);
  if (stage_s) *stage_s = S->t_stage;
  if (solve_s) *solve_s = S->t_solve;
  if (unstage_s) *unstage_s = S->t_unstage;
  return FMM_OK;
}

int fmm_b200_server_trim(fmm_b200_server* S) {
  if (!S) return FMM_ERR_INVALID;
  std::unique_lock<std::mutex> lk(S->mu);
  S->done_cv.wait(lk, [&] {  // no batch running; new ones wait until the trim is done
    for (auto& w : S->workers)
      if (w->busy) return false;
    return true;
  });
  S->paused = true;
  lk.unlock();
  int rc = FMM_OK;
  for (auto& w : S->workers)
    for (auto& kv : w->handles)
      if (kv.second && fmm_b200_trim(kv.second) != FMM_OK) rc = FMM_ERR_CUDA;
  lk.lock();
  S->paused = false;
  lk.unlock();
  S->cv.notify_all();
  return rc;
}

int fmm_b200_server_destroy(fmm_b200_server* S) {
  if (!S) return FMM_ERR_INVALID;
  {
    // drain: let queued requests finish first
    std::unique_lock<std::mutex> lk(S->mu);
    S->done_cv.wait(lk, [&] {
      if (!S->pending.empty()) return false;
      for (auto& w : S->workers)
        if (w->busy) return false;
      return true;
    });
    S->stop = true;
  }
  S->cv.notify_all();
  S->scheduler.join();
  for (auto& w : S->workers) w->thread.join();
  delete S;
  return FMM_OK;
}

}  // extern "C"
