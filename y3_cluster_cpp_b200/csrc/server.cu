// server.cu -- continuous-batching request server over one engine.
//
// A running sampler submits likelihood-evaluation requests (1..N parameter
// points each, every point with its own HMF / distance / Sigma_crit tables)
// as they arrive and waits for each one's counts (and DeltaSigma).  One
// worker thread owns the engine and the device:
//   * admission (planner.h): a request's tables are copied once into a
//     device-resident table pool, on a copy stream, when the pool has a
//     contiguous run of free slots for it; the pool size is bounded by the
//     HBM budget;
//   * launches: each launch gathers up to max_batch points from all admitted
//     requests (oldest first; a large request is split across launches) and
//     evaluates them in one engine call, points addressing their tables by
//     pool slot.  Up to max_inflight launches are queued on the compute
//     stream, so requests that arrive while one runs are already in the next
//     and the device does not idle between launches;
//   * completion: when a launch's event has fired, its results are scattered
//     into the requests' output buffers; a request whose points have all
//     returned is complete and its slots go back to the pool.
// The reference evaluates one point per CosmoSIS execute() call and has no
// request server; this is the serving form of the same integrals.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "engine_internal.h"
#include "host_common.h"
#include "planner.h"

using y3b::DevBuf;
using y3b::PlanChunk;

namespace {

double
now_s()
{
  using namespace std::chrono;
  return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
  int n;
  const y3b_point* pts;
  const double* tables;
  double* counts;
  double* shear;
  double t_submit = 0.0, t_done = 0.0;
  int status = Y3B_OK;
  std::string message;
  bool done = false;
  bool cancelled = false;
  cudaEvent_t copied = nullptr;  // tables are in the pool once this fires
  nvtxRangeId_t range = 0;       // NVTX range from submission to completion
};

struct Launch {
  DevBuf<y3b_point> pts;
  DevBuf<int> slot;
  DevBuf<double> counts, shear;
  y3b_point* h_pts = nullptr;  // pinned
  int* h_slot = nullptr;
  double* h_counts = nullptr;
  double* h_shear = nullptr;
  int* h_status = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<PlanChunk> chunks;
  int n = 0;
};

}  // namespace

struct y3b_server {
  y3b_engine* e = nullptr;
  y3b_server_config cfg{};
  y3b::EngineInfo info{};
  int device = 0;
  y3b::Planner* planner = nullptr;
  DevBuf<double> pool;
  std::vector<std::unique_ptr<Launch>> launches;
  std::vector<int> free_launch;
  std::deque<int> inflight;
  cudaStream_t cs = nullptr, xs = nullptr;  // compute, copy
  std::unordered_map<long long, Request> reqs;
  long long next_id = 1;
  std::mutex m;
  std::condition_variable cv_work, cv_done;
  bool stop = false;
  std::thread worker;
  y3b_server_stats st{};
  size_t fixed_bytes = 0;  // engine + launch buffers
  ~y3b_server()
  {
    for (auto& Lp : launches) {
      Launch& L = *Lp;
      if (L.h_pts) cudaFreeHost(L.h_pts);
      if (L.h_slot) cudaFreeHost(L.h_slot);
      if (L.h_counts) cudaFreeHost(L.h_counts);
      if (L.h_shear) cudaFreeHost(L.h_shear);
      if (L.h_status) cudaFreeHost(L.h_status);
      if (L.done) cudaEventDestroy(L.done);
    }
    for (auto& kv : reqs)
      if (kv.second.copied) cudaEventDestroy(kv.second.copied);
    if (cs) cudaStreamDestroy(cs);
    if (xs) cudaStreamDestroy(xs);
    delete planner;
  }
};

namespace {

using y3b::set_error;

// Enqueues one launch: its points and slots, the engine evaluation, the
// result and status copies back, and the completion event.
int
enqueue_launch(y3b_server* S, Launch& L, const std::vector<cudaEvent_t>& waits)
{
  const int n = L.n, nB = S->info.n_bins, nR = S->info.n_R;
  const bool shear = S->cfg.with_shear != 0;
  for (cudaEvent_t ev : waits) Y3B_CUDA(cudaStreamWaitEvent(S->cs, ev, 0));
  Y3B_CUDA(cudaMemcpyAsync(L.pts.get(), L.h_pts, n * sizeof(y3b_point), cudaMemcpyHostToDevice,
                           S->cs));
  Y3B_CUDA(
    cudaMemcpyAsync(L.slot.get(), L.h_slot, n * sizeof(int), cudaMemcpyHostToDevice, S->cs));
  Y3B_TRY(y3b_engine_eval_pooled(S->e, S->cfg.precision, n, L.pts.get(), S->pool.get(),
                                 L.slot.get(), L.counts.get(), shear ? L.shear.get() : nullptr,
                                 S->cs));
  Y3B_TRY(y3b::engine_status_to_host(S->e, L.h_status, S->cs));
  Y3B_CUDA(cudaMemcpyAsync(L.h_counts, L.counts.get(), (size_t)n * nB * sizeof(double),
                           cudaMemcpyDeviceToHost, S->cs));
  if (shear)
    Y3B_CUDA(cudaMemcpyAsync(L.h_shear, L.shear.get(), (size_t)n * nB * nR * sizeof(double),
                             cudaMemcpyDeviceToHost, S->cs));
  Y3B_CUDA(cudaEventRecord(L.done, S->cs));
  return Y3B_OK;
}

// A request whose points are all back (or that was cancelled with none out):
// complete it (lock held).
void
mark_done(y3b_server* S, Request& r, double t)
{
  r.done = true;
  r.t_done = t;
  if (r.copied) cudaEventDestroy(r.copied);
  r.copied = nullptr;
  nvtxRangeEnd(r.range);
  if (r.cancelled)
    ++S->st.requests_cancelled;
  else
    ++S->st.requests_done;
}

// Scatters a finished launch into its requests (lock held).
void
finish_launch(y3b_server* S, Launch& L, int status, const char* msg)
{
  const int nB = S->info.n_bins, nR = S->info.n_R;
  int k = 0;
  const double t = now_s();
  for (const PlanChunk& c : L.chunks) {
    Request& r = S->reqs[c.id];
    if (status == Y3B_OK && r.status == Y3B_OK) {
      std::memcpy(r.counts + (size_t)c.first * nB, L.h_counts + (size_t)k * nB,
                  (size_t)c.count * nB * sizeof(double));
      if (r.shear && S->cfg.with_shear)
        std::memcpy(r.shear + (size_t)c.first * nB * nR, L.h_shear + (size_t)k * nB * nR,
                    (size_t)c.count * nB * nR * sizeof(double));
    } else if (r.status == Y3B_OK) {
      r.status = status;
      r.message = msg ? msg : "";
    }
    k += c.count;
    if (S->planner->complete(c.id, c.count) == 1) mark_done(S, r, t);
  }
  S->st.points_done += L.n;
  ++S->st.launches;
  if (L.n > S->st.max_launch_points) S->st.max_launch_points = L.n;
  S->cv_done.notify_all();
}


void
worker_main(y3b_server* S)
{
  cudaSetDevice(S->device);
  const size_t stride = S->info.stride;
  std::unique_lock<std::mutex> lk(S->m);
  for (;;) {
    bool progressed = false;
    // 1. admission: copy the tables of newly admitted requests into the pool
    std::vector<std::pair<long long, int>> adm;
    S->planner->admit(&adm);
    for (auto& a : adm) {
      Request& r = S->reqs[a.first];
      const double* src = r.tables;
      const int n = r.n;
      double* dst = S->pool.get() + (size_t)a.second * stride;
      cudaEvent_t ev = nullptr;
      lk.unlock();
      cudaError_t ce = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(dst, src, (size_t)n * stride * sizeof(double),
                             cudaMemcpyHostToDevice, S->xs);
      if (ce == cudaSuccess) ce = cudaEventRecord(ev, S->xs);
      lk.lock();
      r.copied = ev;
      if (ce != cudaSuccess) {
        // Nothing of the request may be launched from its unfilled slots:
        // it leaves the planner (nothing of it was scheduled yet) with the
        // upload error as its status.
        r.status = Y3B_ERR_CUDA;
        r.message = std::string("table upload: ") + cudaGetErrorString(ce);
        if (S->planner->cancel(a.first) == 1) mark_done(S, r, now_s());
      }
      progressed = true;
    }
    // 2. launches, up to max_inflight queued on the device
    while (!S->free_launch.empty()) {
      const int b = S->free_launch.back();
      Launch& L = *S->launches[b];
      L.chunks.clear();
      const int n = S->planner->next_batch(&L.chunks);
      if (n == 0) break;
      S->free_launch.pop_back();
      L.n = n;
      std::vector<cudaEvent_t> waits;
      int k = 0;
      for (const PlanChunk& c : L.chunks) {
        Request& r = S->reqs[c.id];
        std::memcpy(L.h_pts + k, r.pts + c.first, (size_t)c.count * sizeof(y3b_point));
        for (int j = 0; j < c.count; ++j) L.h_slot[k + j] = c.slot + j;
        k += c.count;
        if (r.copied) waits.push_back(r.copied);
      }
      lk.unlock();
      const int rc = enqueue_launch(S, L, waits);
      std::string msg = rc ? y3b_last_error() : "";
      lk.lock();
      if (rc) {
        // nothing of this launch reached the device in a usable state
        cudaStreamSynchronize(S->cs);
        finish_launch(S, L, rc, msg.c_str());
        S->free_launch.push_back(b);
      } else {
        S->inflight.push_back(b);
      }
      progressed = true;
    }
    // 3. completion of the oldest launch
    if (!S->inflight.empty()) {
      const int b = S->inflight.front();
      Launch& L = *S->launches[b];
      const cudaError_t q = cudaEventQuery(L.done);
      if (q == cudaSuccess || q != cudaErrorNotReady) {
        int status = Y3B_OK;
        std::string msg;
        if (q != cudaSuccess) {
          status = Y3B_ERR_CUDA;
          msg = std::string("launch: ") + cudaGetErrorString(q);
        } else if (*L.h_status != 0) {  // a device-side error code (0 = ok)
          status = y3b::device_status_rc(*L.h_status);  // device code -> y3b_status
          msg = y3b_last_error();
        }
        finish_launch(S, L, status, msg.c_str());
        S->inflight.pop_front();
        S->free_launch.push_back(b);
        progressed = true;
      }
    }
    if (S->stop && S->inflight.empty() && S->planner->idle()) break;
    if (progressed) continue;
    if (!S->inflight.empty())
      S->cv_work.wait_for(lk, std::chrono::microseconds(20));
    else
      S->cv_work.wait(lk);
  }
}

}  // namespace

extern "C" int
y3b_server_create(y3b_engine* e, const y3b_server_config* cfg_in, y3b_server** out)
{
  using namespace y3b;
  clear_error();
  if (!e || !cfg_in || !out) {
    set_error("y3b_server_create: null argument");
    return Y3B_ERR_INVALID;
  }
  *out = nullptr;
  Y3B_TRY(require_device());
  y3b_server_config cfg = *cfg_in;
  EngineInfo info;
  engine_info(e, &info);
  if (cfg.max_batch == 0) cfg.max_batch = info.max_points;
  if (cfg.max_inflight == 0) cfg.max_inflight = 2;
  if (cfg.hbm_budget == 0) cfg.hbm_budget = (size_t)150 << 30;
  if (cfg.max_batch < 1 || cfg.max_batch > info.max_points || cfg.max_inflight < 1 ||
      cfg.max_inflight > 4 || cfg.pool_points < 0 ||
      (cfg.precision != Y3B_FP64 && cfg.precision != Y3B_MIXED) ||
      (cfg.with_shear && !info.with_shear)) {
    set_error("y3b_server_create: need 1 <= max_batch <= the engine's max_points, "
              "1 <= max_inflight <= 4, a valid precision, and an engine built with_shear "
              "for with_shear");
    return Y3B_ERR_INVALID;
  }
  const size_t slot_bytes = info.stride * sizeof(double);
  const size_t per_launch =
    (size_t)cfg.max_batch * (sizeof(y3b_point) + sizeof(int) +
                             info.n_bins * sizeof(double) * (1 + (cfg.with_shear ? info.n_R : 0)));
  const size_t fixed = info.device_bytes + cfg.max_inflight * per_launch;
  if (fixed >= cfg.hbm_budget) {
    set_error("y3b_server_create: the engine and launch buffers (%zu bytes) exceed the HBM "
              "budget (%zu bytes)", fixed, cfg.hbm_budget);
    return Y3B_ERR_BUDGET;
  }
  const size_t fit = (cfg.hbm_budget - fixed) / slot_bytes;
  if (cfg.pool_points == 0) cfg.pool_points = (int)std::min<size_t>(fit, 65536);
  if ((size_t)cfg.pool_points > fit || cfg.pool_points < 1) {
    set_error("y3b_server_create: a pool of %d points (%zu bytes each) does not fit the HBM "
              "budget (%zu points fit)", cfg.pool_points, slot_bytes, fit);
    return Y3B_ERR_BUDGET;
  }
  y3b_server* S = new (std::nothrow) y3b_server;
  if (!S) return Y3B_ERR_NOMEM;
  int rc0;
  // Launch sizes vary from launch to launch, so captured graphs would rarely
  // be replayed: the server's launches go straight to the stream.
  if ((rc0 = y3b_engine_set_graphs(e, 0))) {
    delete S;
    return rc0;
  }
  S->e = e;
  S->cfg = cfg;
  S->info = info;
  cudaGetDevice(&S->device);
  auto fail = [&](int rc) {
    delete S;
    return rc;
  };
  int rc = Y3B_OK;
  auto cu = [&](cudaError_t ce, const char* what) {
    if (rc == Y3B_OK) rc = cuda_status(ce, what);
  };
  cu(cudaStreamCreateWithFlags(&S->cs, cudaStreamNonBlocking), "cudaStreamCreate");
  cu(cudaStreamCreateWithFlags(&S->xs, cudaStreamNonBlocking), "cudaStreamCreate");
  if (rc) return fail(rc);
  S->planner = new (std::nothrow) Planner(cfg.pool_points, cfg.max_batch);
  if (!S->planner) return fail(Y3B_ERR_NOMEM);
  if ((rc = S->pool.alloc((size_t)cfg.pool_points * info.stride))) return fail(rc);
  for (int i = 0; i < cfg.max_inflight; ++i) {
    S->launches.emplace_back(new (std::nothrow) Launch);
    if (!S->launches.back()) return fail(Y3B_ERR_NOMEM);
  }
  const int nB = info.n_bins, nR = info.n_R, B = cfg.max_batch;
  for (int i = 0; i < cfg.max_inflight; ++i) {
    Launch& L = *S->launches[i];
    if ((rc = L.pts.alloc(B)) || (rc = L.slot.alloc(B)) || (rc = L.counts.alloc((size_t)B * nB)))
      return fail(rc);
    if (cfg.with_shear && (rc = L.shear.alloc((size_t)B * nB * nR))) return fail(rc);
    cu(cudaHostAlloc((void**)&L.h_pts, B * sizeof(y3b_point), cudaHostAllocDefault), "cudaHostAlloc");
    cu(cudaHostAlloc((void**)&L.h_slot, B * sizeof(int), cudaHostAllocDefault), "cudaHostAlloc");
    cu(cudaHostAlloc((void**)&L.h_counts, (size_t)B * nB * sizeof(double), cudaHostAllocDefault),
       "cudaHostAlloc");
    if (cfg.with_shear)
      cu(cudaHostAlloc((void**)&L.h_shear, (size_t)B * nB * nR * sizeof(double),
                       cudaHostAllocDefault),
         "cudaHostAlloc");
    cu(cudaHostAlloc((void**)&L.h_status, sizeof(int), cudaHostAllocDefault), "cudaHostAlloc");
    cu(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming), "cudaEventCreate");
    if (rc) return fail(rc);
    S->free_launch.push_back(i);
  }
  S->st.pool_points = cfg.pool_points;
  S->fixed_bytes = fixed;
  S->worker = std::thread(worker_main, S);
  *out = S;
  return Y3B_OK;
}

extern "C" int
y3b_server_submit(y3b_server* S, int n, const y3b_point* pts, const double* tables,
                  double* counts, double* shear, long long* ticket)
{
  using namespace y3b;
  const double t0 = now_s();
  clear_error();
  if (!S || n < 1 || !pts || !tables || !counts || !ticket ||
      (S->cfg.with_shear && !shear)) {
    set_error("y3b_server_submit: invalid arguments (n >= 1; pts, tables, counts, ticket and, "
              "with shear, shear are required)");
    return Y3B_ERR_INVALID;
  }
  int mask = 0;
  Y3B_TRY(engine_check_points(S->e, n, pts, &mask));
  Y3B_TRY(engine_check_tables(S->e, n, pts, tables));
  std::lock_guard<std::mutex> lk(S->m);
  if (S->stop) {
    set_error("y3b_server_submit: the server is shutting down");
    return Y3B_ERR_INVALID;
  }
  const long long id = S->next_id++;
  if (S->planner->submit(id, n)) {
    set_error("y3b_server_submit: a request of %d points can never fit the table pool of %d "
              "points", n, S->planner->capacity());
    return Y3B_ERR_BUDGET;
  }
  Request r;
  r.n = n;
  r.pts = pts;
  r.tables = tables;
  r.counts = counts;
  r.shear = S->cfg.with_shear ? shear : nullptr;
  r.t_submit = t0;
  char label[64];
  std::snprintf(label, sizeof label, "y3b request %lld (%d points)", id, n);
  r.range = nvtxRangeStartA(label);
  S->reqs.emplace(id, std::move(r));
  *ticket = id;
  S->cv_work.notify_one();
  return Y3B_OK;
}

extern "C" int
y3b_server_wait(y3b_server* S, long long ticket, double timeout_s, double* latency_s)
{
  using namespace y3b;
  clear_error();
  if (!S) return Y3B_ERR_INVALID;
  std::unique_lock<std::mutex> lk(S->m);
  if (!S->reqs.count(ticket)) {
    set_error("y3b_server_wait: unknown ticket %lld (never issued or already collected)", ticket);
    return Y3B_ERR_INVALID;
  }
  auto ready = [&] {
    auto it = S->reqs.find(ticket);
    return it == S->reqs.end() || it->second.done;
  };
  if (timeout_s < 0) {
    S->cv_done.wait(lk, ready);
  } else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    set_error("y3b_server_wait: request %lld still running after %.3f s", ticket, timeout_s);
    return Y3B_ERR_TIMEOUT;
  }
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) {
    set_error("y3b_server_wait: ticket %lld collected by another thread", ticket);
    return Y3B_ERR_INVALID;
  }
  const Request& r = it->second;
  const int status = r.status;
  if (latency_s) *latency_s = r.t_done - r.t_submit;
  if (status != Y3B_OK) set_error("y3b server: %s", r.message.c_str());
  S->reqs.erase(it);
  return status;
}

extern "C" int
y3b_server_stats_read(y3b_server* S, y3b_server_stats* out)
{
  y3b::clear_error();
  if (!S || !out) return Y3B_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->m);
  *out = S->st;
  out->pool_free_points = S->planner->free_slots();
  out->waiting = S->planner->waiting();
  out->unscheduled = S->planner->unscheduled();
  const size_t slot_bytes = S->info.stride * sizeof(double);
  out->device_bytes = S->fixed_bytes + (size_t)S->cfg.pool_points * slot_bytes;
  out->pool_bytes_in_use = (size_t)(S->cfg.pool_points - out->pool_free_points) * slot_bytes;
  return Y3B_OK;
}

extern "C" int
y3b_server_cancel(y3b_server* S, long long ticket)
{
  y3b::clear_error();
  if (!S) return Y3B_ERR_INVALID;
  std::lock_guard<std::mutex> lk(S->m);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) {
    y3b::set_error("y3b_server_cancel: unknown ticket %lld (never issued or already collected)",
                   ticket);
    return Y3B_ERR_INVALID;
  }
  Request& r = it->second;
  if (r.done || r.cancelled) return Y3B_OK;
  r.cancelled = true;
  if (r.status == Y3B_OK) {
    r.status = Y3B_ERR_CANCELLED;
    r.message = "request cancelled";
  }
  if (S->planner->cancel(ticket) == 1) {
    mark_done(S, r, now_s());
    S->cv_done.notify_all();
  }
  S->cv_work.notify_one();
  return Y3B_OK;
}

extern "C" void
y3b_server_destroy(y3b_server* S)
{
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->m);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->worker.joinable()) S->worker.join();
  cudaStreamSynchronize(S->cs);
  cudaStreamSynchronize(S->xs);
  delete S;
}

/* The planner alone, for capacity planning and for tests of the policy. */
struct y3b_planner {
  y3b::Planner p;
  y3b_planner(int a, int b) : p(a, b) {}
};

extern "C" int
y3b_planner_create(int pool_points, int max_batch, y3b_planner** out)
{
  y3b::clear_error();
  if (!out || pool_points < 1 || max_batch < 1) {
    y3b::set_error("y3b_planner_create: pool_points and max_batch must be >= 1");
    return Y3B_ERR_INVALID;
  }
  *out = new (std::nothrow) y3b_planner(pool_points, max_batch);
  return *out ? Y3B_OK : Y3B_ERR_NOMEM;
}

extern "C" void
y3b_planner_destroy(y3b_planner* p)
{
  delete p;
}

extern "C" int
y3b_planner_submit(y3b_planner* p, long long id, int n_points)
{
  y3b::clear_error();
  if (!p) return Y3B_ERR_INVALID;
  if (p->p.submit(id, n_points)) {
    y3b::set_error("y3b_planner_submit: request %lld of %d points is a duplicate or exceeds "
                   "the pool of %d", id, n_points, p->p.capacity());
    return Y3B_ERR_BUDGET;
  }
  return Y3B_OK;
}

extern "C" int
y3b_planner_admit(y3b_planner* p, long long* ids, int* slot0, int cap, int* n_out)
{
  y3b::clear_error();
  if (!p || !ids || !slot0 || !n_out || cap < 0) return Y3B_ERR_INVALID;
  std::vector<std::pair<long long, int>> adm;
  p->p.admit(&adm);
  if ((int)adm.size() > cap) {
    y3b::set_error("y3b_planner_admit: %zu admissions exceed the output capacity %d",
                   adm.size(), cap);
    return Y3B_ERR_INVALID;
  }
  for (size_t i = 0; i < adm.size(); ++i) {
    ids[i] = adm[i].first;
    slot0[i] = adm[i].second;
  }
  *n_out = (int)adm.size();
  return Y3B_OK;
}

extern "C" int
y3b_planner_next_batch(y3b_planner* p, long long* ids, int* first, int* count, int* slot,
                       int cap, int* n_chunks, int* n_points)
{
  y3b::clear_error();
  if (!p || !ids || !first || !count || !slot || !n_chunks || !n_points || cap < 1)
    return Y3B_ERR_INVALID;
  std::vector<PlanChunk> ch;
  *n_points = p->p.next_batch(&ch, cap);
  for (size_t i = 0; i < ch.size(); ++i) {
    ids[i] = ch[i].id;
    first[i] = ch[i].first;
    count[i] = ch[i].count;
    slot[i] = ch[i].slot;
  }
  *n_chunks = (int)ch.size();
  return Y3B_OK;
}

extern "C" int
y3b_planner_complete(y3b_planner* p, long long id, int count, int* finished)
{
  y3b::clear_error();
  if (!p || !finished) return Y3B_ERR_INVALID;
  const int r = p->p.complete(id, count);
  if (r < 0) {
    y3b::set_error("y3b_planner_complete: request %lld has fewer than %d points out", id, count);
    return Y3B_ERR_INVALID;
  }
  *finished = r;
  return Y3B_OK;
}

extern "C" int
y3b_planner_cancel(y3b_planner* p, long long id, int* finished)
{
  y3b::clear_error();
  if (!p || !finished) return Y3B_ERR_INVALID;
  const int r = p->p.cancel(id);
  if (r < 0) {
    y3b::set_error("y3b_planner_cancel: unknown request %lld", id);
    return Y3B_ERR_INVALID;
  }
  *finished = r;
  return Y3B_OK;
}

extern "C" int
y3b_planner_free_points(const y3b_planner* p)
{
  return p ? p->p.free_slots() : -1;
}
