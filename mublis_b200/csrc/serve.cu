// serve.cu -- continuous-batching request server for Level-3 calls.
//
// The reference is thread-safe (pthread_once context, mutex-guarded pool:
// frame/base/safe_dispatch.c:6,64, frame/base/pool.c:233-318) but every call
// runs alone on its host thread.  On one B200 that leaves the device idle
// between small calls and serialises large ones behind each other's
// synchronisation.  The server turns calls from many host threads into
// device work that overlaps:
//
//   * clients: when a server is attached (mublis_b200_server_attach), every
//     cblas_* / mublis_* call whose operands are all device-resident becomes a
//     request; the calling thread blocks until its request completes, so the
//     BLAS call stays synchronous;
//   * operands stay on the device behind handles allocated through the
//     server (mublis_b200_server_alloc), counted against an HBM budget;
//   * one scheduler thread drains the queue continuously: small plain GEMMs
//     (max(m, n, k) <= small_max_dim) and small left TRSMs (order <= 256)
//     that are waiting together are coalesced per precision into ONE grouped
//     persistent launch (grouped.cu); everything else is admitted when its
//     scratch estimate fits the HBM budget and a stream slot is free, and is
//     issued asynchronously on a pool of streams so large calls overlap;
//   * completion is signalled from the stream itself (cudaLaunchHostFunc),
//     which wakes the waiting client and feeds the latency statistics
//     (p50 / p99) and the throughput counter.
// Requests arriving while others execute are admitted as soon as a slot and
// memory free up: that is the continuous batching.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "../../include/mublis_b200.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Req {
  int kind = 0;  // 0 L3 product, 1 left TRSM
  b200_l3_desc_t l3;
  b200_trsm_desc_t tr;
  int dtype = 0;
  bool small = false;
  double flops = 0;
  size_t scratch = 0;
  double t_submit = 0, t_done = 0;
  int status = 0;
  bool done = false;
  int stream = -1;
};

}  // namespace

struct mublis_b200_server {
  mublis_b200_server_config_t cfg;
  int device = 0;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req *> queue;
  std::vector<cudaStream_t> streams;
  std::vector<int> inflight;
  std::unordered_map<void *, size_t> handles;
  size_t hbm_handles = 0, hbm_scratch = 0;
  bool stop = false;
  std::thread sched;
  std::vector<double> lat;
  double flops = 0, t_first = -1, t_last = 0;
  unsigned long long completed = 0, batches = 0, batched = 0;
};

namespace {

std::atomic<mublis_b200_server *> g_attached{nullptr};

struct Batch {
  mublis_b200_server *srv;
  std::vector<Req *> reqs;
  int stream;
};

void finish_locked(mublis_b200_server *S, Req *r, int status) {
  r->status = status;
  r->t_done = now_s();
  r->done = true;
  if (status == B200_OK) {
    S->lat.push_back(r->t_done - r->t_submit);
    S->flops += r->flops;
    S->t_last = std::max(S->t_last, r->t_done);
    S->completed++;
  }
  if (!r->small) S->hbm_scratch -= r->scratch;
}

void CUDART_CB on_batch_done(void *p) {
  Batch *b = static_cast<Batch *>(p);
  mublis_b200_server *S = b->srv;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (Req *r : b->reqs) finish_locked(S, r, B200_OK);
    S->inflight[b->stream]--;
  }
  S->cv_done.notify_all();
  S->cv_work.notify_one();
  delete b;
}

// Scratch a non-batched request will draw from the pool (packed panels).
size_t scratch_estimate(const Req &r) {
  const size_t elt = r.dtype == B200_F64 ? 8 : 4;
  if (r.kind == 1) return (size_t)(r.tr.m + r.tr.n) * r.tr.m * elt;
  const b200_l3_desc_t &d = r.l3;
  size_t mp = b200_round_up(d.m, 256), np = b200_round_up(d.n, 256);
  size_t kp = b200_round_up((long)d.k * d.npairs, 128);
  int f = d.form;
  if (f == B200_FORM_POLICY) f = r.dtype == B200_F64 ? B200_FORM_OZAKI2 : B200_FORM_BF16X6;
  if (f == B200_FORM_BF16X6) return 3 * (mp + np) * kp * 2;
  if (f == B200_FORM_BF16X3 || f == B200_FORM_FP16X3) return 2 * (mp + np) * kp * 2 + 8 * (mp + np);
  if (f == B200_FORM_OZAKI) return 12 * (mp + np) * kp + 148 * 256 * 256 * 8;
  if (f == B200_FORM_OZAKI2) return 16 * (mp + np) * kp + 148 * 16 * 256 * 256;
  return (mp + np) * kp * elt;
}

int pick_stream(mublis_b200_server *S) {
  int best = 0;
  for (int i = 1; i < (int)S->streams.size(); ++i)
    if (S->inflight[i] < S->inflight[best]) best = i;
  return best;
}

void dispatch_batch(mublis_b200_server *S, std::vector<Req *> &reqs, int dtype, int kind) {
  if (reqs.empty()) return;
  int si;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    si = pick_stream(S);
    S->inflight[si]++;
    S->batches++;
    S->batched += reqs.size();
  }
  cudaStream_t s = S->streams[si];
  int st;
  if (kind == 0) {
    std::vector<const b200_l3_desc_t *> d;
    for (Req *r : reqs) d.push_back(&r->l3);
    st = b200_grouped_gemm_async(dtype, d.data(), (int)d.size(), s);
  } else {
    std::vector<const b200_trsm_desc_t *> d;
    for (Req *r : reqs) d.push_back(&r->tr);
    st = b200_grouped_trsm_async(dtype, d.data(), (int)d.size(), s);
  }
  Batch *b = new Batch{S, reqs, si};
  if (st == B200_OK && cudaLaunchHostFunc(s, on_batch_done, b) == cudaSuccess) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (Req *r : reqs) finish_locked(S, r, st ? st : B200_ECUDA);
    S->inflight[si]--;
  }
  delete b;
  S->cv_done.notify_all();
}

struct Single {
  mublis_b200_server *srv;
  Req *r;
  int stream;
};

void CUDART_CB on_single_done(void *p) {
  Single *x = static_cast<Single *>(p);
  mublis_b200_server *S = x->srv;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    finish_locked(S, x->r, B200_OK);
    S->inflight[x->stream]--;
  }
  S->cv_done.notify_all();
  S->cv_work.notify_one();
  delete x;
}

void dispatch_single(mublis_b200_server *S, Req *r) {
  const int si = r->stream;
  cudaStream_t s = S->streams[si];
  b200_set_thread_stream((void *)s);
  int st = r->kind == 0 ? b200_l3_run(&r->l3) : b200_trsm_run(&r->tr);
  Single *x = new Single{S, r, si};
  if (st == B200_OK && cudaLaunchHostFunc(s, on_single_done, x) == cudaSuccess) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    finish_locked(S, r, st ? st : B200_ECUDA);
    S->inflight[si]--;
  }
  delete x;
  S->cv_done.notify_all();
}

void scheduler(mublis_b200_server *S) {
  cudaSetDevice(S->device);
  const int depth = 2;  // requests in flight per stream
  while (true) {
    std::vector<Req *> gemm[2], trsm[2], large;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
      if (S->stop && S->queue.empty()) break;
      if (S->cfg.batch_window_us > 0) {
        // Give small arrivals a short window to coalesce while only small
        // requests are waiting.
        auto deadline = std::chrono::steady_clock::now() +
                        std::chrono::microseconds(S->cfg.batch_window_us);
        while (!S->stop && (int)S->queue.size() < S->cfg.max_batch &&
               std::all_of(S->queue.begin(), S->queue.end(), [](Req *r) { return r->small; }) &&
               S->cv_work.wait_until(lk, deadline) != std::cv_status::timeout) {
        }
      }
      for (auto it = S->queue.begin(); it != S->queue.end();) {
        Req *r = *it;
        if (r->small) {
          auto &v = r->kind == 0 ? gemm[r->dtype] : trsm[r->dtype];
          if ((int)v.size() < S->cfg.max_batch) {
            v.push_back(r);
            it = S->queue.erase(it);
            continue;
          }
          ++it;
          continue;
        }
        // admission: HBM budget and a free stream slot
        int si = pick_stream(S);
        bool fits = S->hbm_handles + S->hbm_scratch + r->scratch <= S->cfg.hbm_budget_bytes ||
                    (S->hbm_scratch == 0 && large.empty());
        if (S->inflight[si] < depth && fits) {
          S->hbm_scratch += r->scratch;
          S->inflight[si]++;
          r->stream = si;
          large.push_back(r);
          it = S->queue.erase(it);
          continue;
        }
        ++it;
      }
      if (gemm[0].empty() && gemm[1].empty() && trsm[0].empty() && trsm[1].empty() &&
          large.empty()) {
        // Nothing admissible now: wait for a completion to free a slot.
        S->cv_work.wait_for(lk, std::chrono::milliseconds(1));
        continue;
      }
    }
    for (int dt = 0; dt < 2; ++dt) {
      dispatch_batch(S, gemm[dt], dt, 0);
      dispatch_batch(S, trsm[dt], dt, 1);
    }
    for (Req *r : large) dispatch_single(S, r);
  }
}

int submit_and_wait(mublis_b200_server *S, Req &r) {
  r.t_submit = now_s();
  {
    std::unique_lock<std::mutex> lk(S->mu);
    if (S->t_first < 0) S->t_first = r.t_submit;
    S->queue.push_back(&r);
    S->cv_work.notify_one();
    S->cv_done.wait(lk, [&] { return r.done; });
  }
  if (r.status != B200_OK) return r.status;
  if (int e = b200_take_device_error())
    return b200_set_error(e, "a device-side bounded wait timed out (kernel aborted)");
  return B200_OK;
}

double l3_flops(const b200_l3_desc_t &d) {
  double m = d.m, n = d.n, k = (double)d.k * d.npairs;
  if (d.product.domain.ji != MUBLIS_L3_ALL) return m * (m + 1) * k;  // SYRK / SYR2K
  return 2.0 * m * n * k;
}

}  // namespace

extern "C" int b200_serve_attached(void) { return g_attached.load() != nullptr; }

extern "C" int b200_serve_l3(const b200_l3_desc_t *d) {
  mublis_b200_server *S = g_attached.load();
  if (!S) return b200_l3_run(d);
  Req r;
  r.kind = 0;
  r.l3 = *d;
  r.dtype = d->dtype;
  r.flops = l3_flops(*d);
  const int mx = std::max(d->m, std::max(d->n, d->k));
  r.small = b200_l3_is_plain_gemm(d) && mx <= S->cfg.small_max_dim;
  if (!r.small && r.l3.form == B200_FORM_AUTO) {
    int slices = 0;
    int f = b200_parse_form(d->dtype == B200_F64 ? S->cfg.dform : S->cfg.sform, &slices, nullptr);
    r.l3.form = f;
    if (slices) r.l3.slices = slices;
  }
  r.scratch = r.small ? 0 : scratch_estimate(r);
  return submit_and_wait(S, r);
}

extern "C" int b200_serve_trsm(const b200_trsm_desc_t *d) {
  mublis_b200_server *S = g_attached.load();
  if (!S) return b200_trsm_run(d);
  Req r;
  r.kind = 1;
  r.tr = *d;
  r.dtype = d->dtype;
  r.flops = (double)d->m * d->m * d->n;
  r.small = d->m <= 256 && d->alpha != 0.0;
  if (!r.small && r.tr.form == B200_FORM_AUTO) {
    int slices = 0;
    r.tr.form = b200_parse_form(d->dtype == B200_F64 ? S->cfg.dform : S->cfg.sform, &slices, nullptr);
    if (slices) r.tr.slices = slices;
  }
  r.scratch = r.small ? 0 : scratch_estimate(r);
  return submit_and_wait(S, r);
}

extern "C" {

int mublis_b200_server_create(const mublis_b200_server_config_t *cfg, mublis_b200_server_t **out) {
  if (!out) return b200_set_error(B200_EINVAL, "server: null output");
  *out = nullptr;
  B200_TRY(b200_init());
  auto *S = new mublis_b200_server;
  memset(&S->cfg, 0, sizeof S->cfg);
  if (cfg) S->cfg = *cfg;
  if (!S->cfg.hbm_budget_bytes) S->cfg.hbm_budget_bytes = 64ull << 30;
  if (S->cfg.streams <= 0) S->cfg.streams = 4;
  if (S->cfg.small_max_dim <= 0) S->cfg.small_max_dim = 512;
  if (S->cfg.max_batch <= 0) S->cfg.max_batch = 4096;
  cudaGetDevice(&S->device);
  S->streams.resize(S->cfg.streams);
  S->inflight.assign(S->cfg.streams, 0);
  for (auto &s : S->streams) {
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
      delete S;
      return b200_set_error(B200_ECUDA, "server: stream creation failed");
    }
  }
  // Reserve the HBM budget in the stream-ordered pool now (at most half of
  // the free memory): handles and request scratch are both carved from the
  // pool, and admission keeps their sum within the budget, so the pool need
  // not grow while serving.  Growing it maps new memory inside
  // cudaMallocAsync, on the scheduler thread, which stalls every later
  // dispatch (measured: up to 119 ms per allocation; with half the budget
  // reserved and handles outside the pool, some runs of the served mix lost
  // 2-3x of their throughput this way).  The pool keeps freed memory (its
  // release threshold is raised at initialisation).
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
    const size_t reserve = std::min<size_t>(S->cfg.hbm_budget_bytes, free_b / 2);
    void *p = nullptr;
    if (reserve > 0 && cudaMallocAsync(&p, reserve, S->streams[0]) == cudaSuccess)
      cudaFreeAsync(p, S->streams[0]);
    cudaStreamSynchronize(S->streams[0]);
    cudaGetLastError();  // a failed reservation only costs speed
  }
  S->sched = std::thread(scheduler, S);
  *out = S;
  return B200_OK;
}

int mublis_b200_server_destroy(mublis_b200_server_t *S) {
  if (!S) return B200_OK;
  mublis_b200_server *expected = S;
  g_attached.compare_exchange_strong(expected, nullptr);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->sched.joinable()) S->sched.join();
  cudaDeviceSynchronize();
  for (auto &h : S->handles) cudaFreeAsync(h.first, S->streams[0]);
  for (auto &s : S->streams) {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
  delete S;
  return B200_OK;
}

int mublis_b200_server_attach(mublis_b200_server_t *S) {
  g_attached.store(S);
  return B200_OK;
}

int mublis_b200_server_alloc(mublis_b200_server_t *S, size_t bytes, void **dptr) {
  if (!S || !dptr) return b200_set_error(B200_EINVAL, "server_alloc: bad arguments");
  *dptr = nullptr;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->hbm_handles + bytes > S->cfg.hbm_budget_bytes)
      return b200_set_error(B200_ENOMEM, "server_alloc: HBM budget exceeded");
    S->hbm_handles += bytes;
  }
  // From the pool reserved at creation; usable on every stream once the
  // allocating stream has synchronised.
  cudaError_t e = cudaMallocAsync(dptr, bytes ? bytes : 256, S->streams[0]);
  if (e == cudaSuccess) e = cudaStreamSynchronize(S->streams[0]);
  std::lock_guard<std::mutex> lk(S->mu);
  if (e != cudaSuccess) {
    S->hbm_handles -= bytes;
    *dptr = nullptr;
    return b200_set_error(B200_ENOMEM, "server_alloc: allocation failed");
  }
  S->handles[*dptr] = bytes;
  return B200_OK;
}

int mublis_b200_server_free(mublis_b200_server_t *S, void *dptr) {
  if (!S) return b200_set_error(B200_EINVAL, "server_free: null server");
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->handles.find(dptr);
  if (it == S->handles.end()) return b200_set_error(B200_EINVAL, "server_free: unknown handle");
  S->hbm_handles -= it->second;
  S->handles.erase(it);
  // The device-wide wait cudaFree implied: no queued work still reads it.
  cudaDeviceSynchronize();
  cudaFreeAsync(dptr, S->streams[0]);
  cudaStreamSynchronize(S->streams[0]);
  return B200_OK;
}

int mublis_b200_server_stats(mublis_b200_server_t *S, mublis_b200_server_stats_t *out) {
  if (!S || !out) return b200_set_error(B200_EINVAL, "server_stats: bad arguments");
  std::lock_guard<std::mutex> lk(S->mu);
  memset(out, 0, sizeof *out);
  out->completed = S->completed;
  out->batches = S->batches;
  out->batched_requests = S->batched;
  out->queue_depth = S->queue.size();
  out->hbm_in_use = S->hbm_handles + S->hbm_scratch;
  std::vector<double> l = S->lat;
  if (!l.empty()) {
    std::sort(l.begin(), l.end());
    auto pct = [&](double q) { return l[std::min(l.size() - 1, (size_t)(q * (l.size() - 1) + 0.5))]; };
    out->p50_latency_s = pct(0.50);
    out->p99_latency_s = pct(0.99);
    double sum = 0;
    for (double x : l) sum += x;
    out->mean_latency_s = sum / l.size();
  }
  if (S->t_first >= 0 && S->t_last > S->t_first) {
    out->elapsed_s = S->t_last - S->t_first;
    out->tflops = S->flops / out->elapsed_s / 1e12;
  }
  return B200_OK;
}

int mublis_b200_server_reset_stats(mublis_b200_server_t *S) {
  if (!S) return b200_set_error(B200_EINVAL, "server_reset_stats: null server");
  std::lock_guard<std::mutex> lk(S->mu);
  S->lat.clear();
  S->flops = 0;
  S->t_first = -1;
  S->t_last = 0;
  S->completed = S->batches = S->batched = 0;
  return B200_OK;
}

}  // extern "C"
