// Request loop over one batch: a worker thread admits queued solves by free
// device memory and slots, advances every resident system with chunked graph
// launches (b200la_batch_run) and harvests the finished ones.  Host code
// only; all device work goes through the b200la_batch_* entry points on the
// context's stream, from the worker thread.
//
// No reference counterpart: the reference solves one system per CG<LAD>
// call (linear_solver/cg.h:87-246).  The per-system recurrence is the
// batch's; this file only decides what is resident and when.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.cuh"

using namespace b200la;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
  int64_t id = 0;
  bool q1 = false;
  int dim = 0, cells = 0;
  uint64_t seed = 0;
  double sigma = 0.0;
  std::vector<int> rowptr, col;
  std::vector<double> val, rhs, x0;
  int n = 0;
  int64_t nnz = 0;
  int64_t bytes = 0;  // admission charge
  int slot = -1;
  int status = B200LA_OK;  // non-zero: failed at admission (or the server failed)
  std::string error;
  bool done = false;
  b200la_sys_result res{};
  std::vector<double> x;
  Clock::time_point t_submit, t_admit, t_done;
};

}  // namespace

struct b200la_server_s {
  b200la_ctx ctx = nullptr;
  b200la_batch batch = nullptr;
  b200la_server_params prm{};
  int capacity = 0;
  int chunk = 32;
  int max_skips = 8;
  bool mixed = true;

  std::mutex mu;
  std::condition_variable cv_work;  // worker: something queued or stop
  std::condition_variable cv_done;  // clients: a request finished
  std::deque<Request *> queue;
  std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
  std::vector<Request *> slot_req;  // worker-owned: request resident in each slot
  int64_t next_id = 1;
  int running = 0;  // admitted and not yet harvested
  int head_skips = 0;
  int64_t in_use = 0, peak = 0;
  bool stop = false;
  int fatal = B200LA_OK;
  std::string fatal_msg;

  // statistics
  int64_t submitted = 0, completed = 0, failed = 0, launches = 0, passes = 0;
  std::vector<double> lat_ms;
  bool have_first = false;
  Clock::time_point t_first, t_last;

  std::thread worker;
};

namespace {

using Server = b200la_server;

// Admission charge: the slot's resident bytes, plus the per-cell coefficient
// buffer that device assembly holds while it runs (sigma > 0).
int64_t charge_q1(int dim, int cells, double sigma, bool mixed) {
  const int64_t n = q1_rows(dim, cells), nnz = q1_nnz(dim, cells);
  int64_t bytes = 0;
  const int ell = cells >= 2 ? (dim == 2 ? 9 : 27) : (dim == 2 ? 4 : 8);
  b200la_batch_slot_bytes(n, nnz, ell, mixed ? 1 : 0, &bytes);
  if (sigma > 0.0) bytes += 8 * (dim == 2 ? (int64_t)cells * cells : (int64_t)cells * cells * cells);
  return bytes;
}

// Marks a request finished (under the lock) and records its latency.
void finish_locked(Server S, Request *r, Clock::time_point now) {
  r->done = true;
  r->t_done = now;
  if (r->status == B200LA_OK) {
    S->completed++;
    S->lat_ms.push_back(ms_between(r->t_submit, now));
  } else {
    S->failed++;
  }
  S->t_last = now;
}

// A CUDA error in the worker ends the server: every queued and resident
// request fails with that status.
void fail_all_locked(Server S, int status, const std::string &msg) {
  S->fatal = status;
  S->fatal_msg = msg;
  const auto now = Clock::now();
  for (Request *r : S->queue) {
    r->status = status;
    r->error = msg;
    finish_locked(S, r, now);
  }
  S->queue.clear();
  for (Request *&r : S->slot_req) {
    if (!r) continue;
    r->status = status;
    r->error = msg;
    finish_locked(S, r, now);
    r = nullptr;
  }
  S->running = 0;
  S->in_use = 0;
  S->cv_done.notify_all();
}

// Picks queued requests to admit: first fit in FIFO order while slots and
// budget last; once the head has been passed over max_skips times nothing
// behind it is admitted until it fits.
void pick_locked(Server S, std::vector<Request *> &out) {
  int free_slots = S->capacity - S->running;
  const int64_t budget = S->prm.hbm_budget;
  bool head = true;
  for (auto it = S->queue.begin(); it != S->queue.end() && free_slots > 0;) {
    Request *r = *it;
    if (S->in_use + r->bytes <= budget) {
      out.push_back(r);
      S->in_use += r->bytes;
      S->peak = std::max(S->peak, S->in_use);
      S->running++;
      free_slots--;
      if (head) S->head_skips = 0;
      it = S->queue.erase(it);
      continue;
    }
    if (head) {
      head = false;
      if (++S->head_skips > S->max_skips) break;
    }
    ++it;
  }
}

}  // namespace

namespace {

// Uploads (or assembles) one admitted request into a free slot.
int admit_one(Server S, Request *r) {
  int slot = -1;
  int rc;
  if (r->q1) {
    rc = b200la_batch_add_q1(S->batch, r->dim, r->cells, r->seed, r->sigma, &slot);
  } else {
    rc = b200la_batch_add(S->batch, r->n, r->nnz, r->rowptr.data(), r->col.data(), r->val.data(), r->rhs.data(),
                          r->x0.empty() ? nullptr : r->x0.data(), &slot);
  }
  if (rc != B200LA_OK) return rc;
  r->slot = slot;
  r->t_admit = Clock::now();
  S->slot_req[slot] = r;
  return B200LA_OK;
}

// Copies each finished system's result and solution to its request and
// frees the slot.
int harvest(Server S) {
  for (int slot = 0; slot < S->capacity; ++slot) {
    Request *r = S->slot_req[slot];
    if (!r) continue;
    b200la_sys_result res;
    B_TRY(b200la_batch_result(S->batch, slot, nullptr, &res));
    if (!res.phase_done) continue;
    std::vector<double> x((size_t)r->n);
    B_TRY(b200la_batch_result(S->batch, slot, x.data(), &res));
    B_TRY(b200la_batch_remove(S->batch, slot));
    S->slot_req[slot] = nullptr;
    std::lock_guard<std::mutex> lk(S->mu);
    r->res = res;
    r->x.swap(x);
    S->in_use -= r->bytes;
    S->running--;
    finish_locked(S, r, Clock::now());
    S->cv_done.notify_all();
  }
  return B200LA_OK;
}

void worker_main(Server S) {
  if (cudaSetDevice(S->ctx->device) != cudaSuccess) {
    std::lock_guard<std::mutex> lk(S->mu);
    fail_all_locked(S, B200LA_ERR_CUDA, "server worker: cudaSetDevice failed");
    return;
  }
  std::vector<Request *> admit;
  for (;;) {
    admit.clear();
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stop || S->running > 0 || !S->queue.empty(); });
      if (S->stop || S->fatal != B200LA_OK) return;
      pick_locked(S, admit);
    }
    for (Request *r : admit) {
      const int rc = admit_one(S, r);
      if (rc != B200LA_OK) {
        // the request fails on its own (e.g. the allocation failed); the
        // server keeps serving the rest
        std::lock_guard<std::mutex> lk(S->mu);
        r->status = rc;
        r->error = b200la_last_error();
        S->in_use -= r->bytes;
        S->running--;
        finish_locked(S, r, Clock::now());
        S->cv_done.notify_all();
      }
    }
    bool any = false;
    for (Request *r : S->slot_req) any = any || r;
    if (!any) continue;
    int active = 0;
    int rc = b200la_batch_run(S->batch, S->chunk, &active);
    int taken = 0;
    if (rc == B200LA_OK) rc = b200la_batch_last_run(S->batch, &taken, nullptr);
    if (rc == B200LA_OK) {
      // the host copies of admitted systems are no longer needed
      for (Request *r : admit) {
        std::vector<int>().swap(r->rowptr);
        std::vector<int>().swap(r->col);
        std::vector<double>().swap(r->val);
        std::vector<double>().swap(r->rhs);
        std::vector<double>().swap(r->x0);
      }
      rc = harvest(S);
    }
    std::lock_guard<std::mutex> lk(S->mu);
    S->launches++;
    S->passes += taken;
    if (rc != B200LA_OK) {
      fail_all_locked(S, rc, b200la_last_error());
      return;
    }
  }
}

Request *find_locked(Server S, int64_t id) {
  auto it = S->reqs.find(id);
  return it == S->reqs.end() ? nullptr : it->second.get();
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  // nearest rank
  size_t k = (size_t)std::ceil(q * (double)v.size());
  k = std::min(std::max<size_t>(k, 1), v.size()) - 1;
  std::nth_element(v.begin(), v.begin() + (ptrdiff_t)k, v.end());
  return v[k];
}

// Enqueues a request (the caller filled its problem fields and charge).
int enqueue(Server S, std::unique_ptr<Request> r, int64_t *id) {
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->fatal != B200LA_OK) return fail(S->fatal, "server: stopped after an error: %s", S->fatal_msg.c_str());
  B_CHECK(!S->stop, B200LA_ERR_INVALID, "server: stopping");
  r->id = S->next_id++;
  r->t_submit = Clock::now();
  if (!S->have_first) {
    S->have_first = true;
    S->t_first = r->t_submit;
  }
  S->submitted++;
  *id = r->id;
  S->queue.push_back(r.get());
  S->reqs.emplace(r->id, std::move(r));
  S->cv_work.notify_one();
  return B200LA_OK;
}

}  // namespace

extern "C" {

int b200la_server_start(b200la_ctx ctx, const b200la_server_params *p, b200la_server *out) {
  B_CHECK(ctx && p && out, B200LA_ERR_INVALID, "server_start: null argument");
  B_CHECK(p->hbm_budget >= 0 && p->chunk_passes >= 0 && p->max_skips >= 0, B200LA_ERR_INVALID,
          "server_start: negative budget, chunk or skip count");
  B_CUDA(cudaSetDevice(ctx->device));
  std::unique_ptr<b200la_server_s> S(new b200la_server_s());
  S->ctx = ctx;
  S->prm = *p;
  S->capacity = p->batch.capacity;
  S->chunk = p->chunk_passes ? p->chunk_passes : 32;
  S->max_skips = p->max_skips ? p->max_skips : 8;
  S->mixed = p->batch.mixed != 0;
  B_TRY(b200la_batch_create(ctx, &p->batch, &S->batch));
  if (S->prm.hbm_budget == 0) {
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
      b200la_batch_destroy(S->batch);
      return fail(B200LA_ERR_CUDA, "server_start: cudaMemGetInfo failed");
    }
    S->prm.hbm_budget = (int64_t)(0.9 * (double)free_b);
  }
  S->slot_req.assign((size_t)S->capacity, nullptr);
  b200la_server_s *raw = S.get();
  try {
    S->worker = std::thread(worker_main, raw);
  } catch (...) {
    b200la_batch_destroy(S->batch);
    return fail(B200LA_ERR_INVALID, "server_start: could not start the worker thread");
  }
  *out = S.release();
  return B200LA_OK;
}

int b200la_server_stop(b200la_server S) {
  if (!S) return B200LA_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  // the worker has exited: this thread may use the context now
  cudaSetDevice(S->ctx->device);
  const int rc = b200la_batch_destroy(S->batch);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->cv_done.notify_all();
  }
  delete S;
  return rc;
}

int b200la_server_submit_csr(b200la_server S, int n, int64_t nnz, const int *rowptr, const int *col,
                             const double *val, const double *rhs, const double *x0, int64_t *id) {
  B_CHECK(S && id && rhs, B200LA_ERR_INVALID, "server_submit_csr: null argument");
  B_CHECK(n > 0, B200LA_ERR_INVALID, "server_submit_csr: empty system");
  int max_row = 0;
  B_TRY(validate_csr(n, n, nnz, rowptr, col, &max_row));
  B_CHECK(nnz == 0 || val, B200LA_ERR_MATRIX, "server_submit_csr: val is NULL");
  int64_t bytes = 0;
  B_TRY(b200la_batch_slot_bytes(n, nnz, std::max(max_row, 1), S->mixed ? 1 : 0, &bytes));
  B_CHECK(bytes <= S->prm.hbm_budget, B200LA_ERR_NOMEM,
          "server_submit_csr: system needs %lld device bytes, the budget is %lld", (long long)bytes,
          (long long)S->prm.hbm_budget);
  std::unique_ptr<Request> r(new Request());
  r->n = n;
  r->nnz = nnz;
  r->bytes = bytes;
  r->rowptr.assign(rowptr, rowptr + n + 1);
  r->col.assign(col, col + nnz);
  r->val.assign(val, val + nnz);
  r->rhs.assign(rhs, rhs + n);
  if (x0) r->x0.assign(x0, x0 + n);
  return enqueue(S, std::move(r), id);
}

int b200la_server_submit_q1(b200la_server S, int dim, int cells, uint64_t seed, double sigma, int64_t *id) {
  B_CHECK(S && id, B200LA_ERR_INVALID, "server_submit_q1: null argument");
  B_CHECK((dim == 2 || dim == 3) && cells >= 1 && sigma >= 0.0, B200LA_ERR_INVALID,
          "server_submit_q1: dim %d cells %d sigma %g", dim, cells, sigma);
  B_CHECK(q1_nnz(dim, cells) < (int64_t)INT32_MAX, B200LA_ERR_UNSUPPORTED,
          "server_submit_q1: nnz exceeds int32 indexing");
  const int64_t bytes = charge_q1(dim, cells, sigma, S->mixed);
  B_CHECK(bytes <= S->prm.hbm_budget, B200LA_ERR_NOMEM,
          "server_submit_q1: system needs %lld device bytes, the budget is %lld", (long long)bytes,
          (long long)S->prm.hbm_budget);
  std::unique_ptr<Request> r(new Request());
  r->q1 = true;
  r->dim = dim;
  r->cells = cells;
  r->seed = seed;
  r->sigma = sigma;
  r->n = (int)q1_rows(dim, cells);
  r->nnz = q1_nnz(dim, cells);
  r->bytes = bytes;
  return enqueue(S, std::move(r), id);
}

int b200la_server_poll(b200la_server S, int64_t id, int *done, double *x, b200la_sys_result *result,
                       double *latency_ms) {
  B_CHECK(S && done, B200LA_ERR_INVALID, "server_poll: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  Request *r = find_locked(S, id);
  B_CHECK(r, B200LA_ERR_INVALID, "server_poll: unknown request %lld", (long long)id);
  *done = r->done ? 1 : 0;
  if (!r->done) return B200LA_OK;
  if (r->status != B200LA_OK)
    return fail(r->status, "server: request %lld failed: %s", (long long)id, r->error.c_str());
  if (result) *result = r->res;
  if (latency_ms) *latency_ms = ms_between(r->t_submit, r->t_done);
  if (x) {
    B_CHECK(!r->x.empty() || r->n == 0, B200LA_ERR_INVALID, "server_poll: request %lld was released",
            (long long)id);
    std::memcpy(x, r->x.data(), sizeof(double) * (size_t)r->n);
  }
  return B200LA_OK;
}

int b200la_server_wait(b200la_server S, int64_t id, double timeout_s, int *done) {
  B_CHECK(S && done && timeout_s >= 0, B200LA_ERR_INVALID, "server_wait: bad argument");
  std::unique_lock<std::mutex> lk(S->mu);
  Request *r = find_locked(S, id);
  B_CHECK(r, B200LA_ERR_INVALID, "server_wait: unknown request %lld", (long long)id);
  S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] { return r->done; });
  *done = r->done ? 1 : 0;
  return B200LA_OK;
}

int b200la_server_release(b200la_server S, int64_t id) {
  B_CHECK(S, B200LA_ERR_INVALID, "server_release: null server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(id);
  B_CHECK(it != S->reqs.end(), B200LA_ERR_INVALID, "server_release: unknown request %lld", (long long)id);
  B_CHECK(it->second->done, B200LA_ERR_INVALID, "server_release: request %lld is not done", (long long)id);
  S->reqs.erase(it);
  return B200LA_OK;
}

int b200la_server_drain(b200la_server S, double timeout_s) {
  B_CHECK(S && timeout_s >= 0, B200LA_ERR_INVALID, "server_drain: bad argument");
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                      [&] { return S->queue.empty() && S->running == 0; });
  if (S->fatal != B200LA_OK) return fail(S->fatal, "server: stopped after an error: %s", S->fatal_msg.c_str());
  B_CHECK(ok, B200LA_ERR_TIMEOUT, "server_drain: %zu queued and %d running after %.1f s", S->queue.size(),
          S->running, timeout_s);
  return B200LA_OK;
}

int b200la_server_get_stats(b200la_server S, b200la_server_stats *st) {
  B_CHECK(S && st, B200LA_ERR_INVALID, "server_get_stats: null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  memset(st, 0, sizeof(*st));
  st->submitted = S->submitted;
  st->completed = S->completed;
  st->failed = S->failed;
  st->running = S->running;
  st->queued = (int64_t)S->queue.size();
  st->hbm_in_use = S->in_use;
  st->hbm_peak = S->peak;
  st->hbm_budget = S->prm.hbm_budget;
  st->launches = S->launches;
  st->passes = S->passes;
  if (!S->lat_ms.empty()) {
    double sum = 0.0, mx = 0.0;
    for (double v : S->lat_ms) {
      sum += v;
      mx = std::max(mx, v);
    }
    st->mean_ms = sum / (double)S->lat_ms.size();
    st->max_ms = mx;
    st->p50_ms = percentile(S->lat_ms, 0.50);
    st->p99_ms = percentile(S->lat_ms, 0.99);
  }
  if (S->have_first && S->completed + S->failed > 0) {
    st->wall_s = std::chrono::duration<double>(S->t_last - S->t_first).count();
    if (st->wall_s > 0) st->solves_per_s = (double)S->completed / st->wall_s;
  }
  return B200LA_OK;
}

int b200la_server_reset_stats(b200la_server S) {
  B_CHECK(S, B200LA_ERR_INVALID, "server_reset_stats: null server");
  std::lock_guard<std::mutex> lk(S->mu);
  S->submitted = (int64_t)S->queue.size() + S->running;
  S->completed = S->failed = S->launches = S->passes = 0;
  S->lat_ms.clear();
  S->peak = S->in_use;
  S->have_first = false;
  return B200LA_OK;
}

}  // extern "C"
