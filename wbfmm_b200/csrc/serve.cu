// Served form: continuous batching of independent FMM solves on one GPU.
//
// A server owns S slots.  Each slot is a host thread with its own CUDA
// stream and a reusable solver per precision whose buffers come from the
// server's stream-ordered pool.  Requests wait in an arrival-ordered queue;
// a slot that falls free takes the oldest request whose arrival time has
// passed, provided the device-memory footprints of the solves in flight plus
// its own stay within the budget (first come, first served: a request that
// does not fit yet holds back the ones behind it), or, with the
// largest-first order, the largest of the requests that have arrived (a
// batch submitted at once then runs its big solves first and its small ones
// fill the tail).  A slot queues the whole
// solve -- tree build, passes, evaluation, copy-back -- on its stream with no
// host wait, then sleeps on a blocking event until the stream drains, so
// up to S solves run on the device at once and their kernels overlap.
// The order-only operator tables (rotations, shift phases, Laplace coaxial
// tables) are shared between slots through a TableCache; each Helmholtz
// solve builds its own coaxial tables (they depend on its k).
//
// Callers keep a request's input and output arrays alive until the request
// has completed (wbfmm_b200_server_wait / _poll).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "solver.h"

using namespace wbfmm;

namespace {

double now_s() {
  using clk = std::chrono::steady_clock;
  return std::chrono::duration<double>(clk::now().time_since_epoch()).count();
}

struct Req {
  int64_t id = 0;
  wbfmm_b200_request_t r;
  int64_t footprint = 0;
  double t_arrival = 0, t_start = 0, t_queued = 0, t_end = 0;   // server clock
  int state = 0;                                   // 0 queued, 1 running, 2 done
  int64_t launches = 0;                            // kernels its solve launched
  int status = 0;
  char error[256] = "";
};

// pinned host staging that only grows, at least doubling (each regrowth's
// cudaFreeHost synchronises the device, stalling every slot)
struct Pinned {
  double* p = nullptr;
  size_t n = 0;
  // outgrown buffers, freed with the server: cudaFreeHost synchronises the
  // device, which would stall every slot's work; growth is geometric, so
  // they hold less than the current buffer
  std::vector<double*> retired;
  ~Pinned() {
    if (p) cudaFreeHost(p);
    for (double* r : retired) cudaFreeHost(r);
  }
  int reserve(size_t count) {
    if (count <= n) return 0;
    const size_t want = std::max(count + count / 4, 2 * n);
    double* q = nullptr;
    if (cudaMallocHost(&q, sizeof(double) * want) != cudaSuccess) {
      cudaGetLastError();
      return set_error(WBFMM_B200_E_NOMEM, "pinned host allocation failed");
    }
    if (p) retired.push_back(p);   // idle: each solve ends with the slot's event wait
    p = q;
    n = want;
    return 0;
  }
};

}  // namespace

struct wbfmm_b200_server {
  struct Slot {
    std::thread th;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    Solver<float>* s32 = nullptr;
    Solver<double>* s64 = nullptr;
    Pinned in, out;
  };

  int device = 0;
  int largest_first = 0;    // among arrived requests, the largest footprint first
  int64_t budget = 0;       // for the footprints of the solves in flight
  int64_t keep = 0;         // work buffers a slot may keep between solves
  cudaMemPool_t pool = nullptr;   // the solves' device memory
  double epoch = 0;
  TableCache cache;
  std::vector<Slot*> slots;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> queue;                     // ordered by arrival time
  std::unordered_map<int64_t, Req*> reqs;
  int64_t next_id = 1, inflight = 0, peak_inflight = 0, completed = 0;
  int64_t launches = 0;                       // kernels of completed solves
  int running = 0, peak_running = 0;
  bool stop = false;

  double clock() const { return now_s() - epoch; }

  ~wbfmm_b200_server() {
    {
      std::lock_guard<std::mutex> lk(mu);
      stop = true;
    }
    cv_work.notify_all();
    for (Slot* s : slots)
      if (s->th.joinable()) s->th.join();
    cudaSetDevice(device);
    for (Slot* s : slots) {
      delete s->s32;
      delete s->s64;
      if (s->done) cudaEventDestroy(s->done);
      if (s->stream) cudaStreamDestroy(s->stream);
      delete s;
    }
    for (auto& e : reqs) delete e.second;
    cache.clear();
    if (pool) cudaMemPoolDestroy(pool);
  }

  template <typename T>
  int make_solver(Slot* s, const wbfmm_b200_config_t* c, Solver<T>** out) {
    if (!*out) {
      auto* x = new Solver<T>();
      x->cache = &cache;
      x->async_checks = true;
      int rc = x->init(c, (void*)s->stream);
      if (rc) { delete x; return rc; }
      cudaMemPool_t pl = pool;
      x->each_buf([pl](auto& b) { b.pool = pl; });
      *out = x;
    }
    return (*out)->reset(c);
  }

  // one solve on the slot's stream; fields land in the caller's arrays
  // (host arrays through the slot's pinned staging, or device arrays)
  template <typename T>
  int execute(Slot* s, Solver<T>* sv, const wbfmm_b200_request_t& r, double* t_queued) {
    const int w = r.cfg.problem == WBFMM_B200_HELMHOLTZ ? 2 : 1;
    const size_t ns = (size_t)r.nsrc, nt = (size_t)r.ntgt;
    const bool same = r.xt == r.xs && r.ntgt == r.nsrc;
    const size_t np = r.pot ? w * nt : 0, ng = r.grad ? 3 * w * nt : 0;
    if (r.on_device) {
      WBFMM_TRY(sv->set_sources((int)ns, r.xs, 3, r.normals, 3, 1));
      WBFMM_TRY(sv->set_strengths(r.q, w, r.dipoles, w, 1));
      WBFMM_TRY(sv->set_targets((int)nt, r.xt, 3, 1));
      WBFMM_TRY(sv->run_async());
      WBFMM_TRY(sv->fetch_async(r.pot, r.grad, cudaMemcpyDeviceToDevice));
      WBFMM_CUDA(cudaEventRecord(s->done, s->stream));
      *t_queued = clock();
      WBFMM_CUDA(cudaEventSynchronize(s->done));
      return sv->check_flags();
    }
    size_t need = 3 * ns + (r.q ? w * ns : 0) + (r.normals ? 3 * ns : 0) +
                  (r.dipoles ? w * ns : 0) + (same ? 0 : 3 * nt);
    WBFMM_TRY(s->in.reserve(need));
    double* p = s->in.p;
    auto stage = [&](const double* src, size_t n) -> const double* {
      if (!src) return nullptr;
      memcpy(p, src, sizeof(double) * n);
      const double* q = p;
      p += n;
      return q;
    };
    const double* xs = stage(r.xs, 3 * ns);
    const double* q = stage(r.q, w * ns);
    const double* nrm = stage(r.normals, 3 * ns);
    const double* dip = stage(r.dipoles, w * ns);
    const double* xt = same ? xs : stage(r.xt, 3 * nt);
    WBFMM_TRY(s->out.reserve(np + ng));
    WBFMM_TRY(sv->set_sources((int)ns, xs, 3, nrm, 3, 0));
    WBFMM_TRY(sv->set_strengths(q, w, dip, w, 0));
    WBFMM_TRY(sv->set_targets((int)nt, xt, 3, 0));
    WBFMM_TRY(sv->run_async());
    WBFMM_TRY(sv->fetch_async(np ? s->out.p : nullptr, ng ? s->out.p + np : nullptr,
                              cudaMemcpyDeviceToHost));
    WBFMM_CUDA(cudaEventRecord(s->done, s->stream));
    *t_queued = clock();
    WBFMM_CUDA(cudaEventSynchronize(s->done));
    WBFMM_TRY(sv->check_flags());
    if (np) memcpy(r.pot, s->out.p, sizeof(double) * np);
    if (ng) memcpy(r.grad, s->out.p + np, sizeof(double) * ng);
    return 0;
  }

  int run_one(Slot* s, Req* q) {
    const wbfmm_b200_request_t& r = q->r;
    int rc;
    const int64_t l0 = (s->s32 ? s->s32->launches : 0) + (s->s64 ? s->s64->launches : 0);
    if (r.cfg.precision == WBFMM_B200_FP32) {
      rc = make_solver(s, &r.cfg, &s->s32);
      if (!rc) rc = execute(s, s->s32, r, &q->t_queued);
    } else {
      rc = make_solver(s, &r.cfg, &s->s64);
      if (!rc) rc = execute(s, s->s64, r, &q->t_queued);
    }
    q->launches = (s->s32 ? s->s32->launches : 0) + (s->s64 ? s->s64->launches : 0) - l0;
    if (rc) {
      // drain whatever was queued before the failure
      cudaStreamSynchronize(s->stream);
      cudaGetLastError();
    }
    // a slot keeps its work buffers for the next solve (no allocation then)
    // while they stay within its allowance; a failed solve releases them
    if (s->s32) {
      if (rc || (int64_t)s->s32->buffer_bytes() > keep) s->s32->release_buffers();
    }
    if (s->s64) {
      if (rc || (int64_t)s->s64->buffer_bytes() > keep) s->s64->release_buffers();
    }
    return rc;
  }

  void slot_main(Slot* s) {
    cudaSetDevice(device);
    for (;;) {
      Req* q = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
          if (stop && queue.empty()) return;
          if (!queue.empty()) {
            auto hi = queue.begin();
            double t = clock();
            if ((*hi)->t_arrival > t) {
              cv_work.wait_for(lk, std::chrono::duration<double>((*hi)->t_arrival - t));
              continue;
            }
            if (largest_first)   // the largest of the requests that have arrived
              for (auto it = queue.begin(); it != queue.end() && (*it)->t_arrival <= t; ++it)
                if ((*it)->footprint > (*hi)->footprint) hi = it;
            Req* h = *hi;
            if (inflight + h->footprint <= budget || running == 0) {
              queue.erase(hi);
              q = h;
              inflight += q->footprint;
              peak_inflight = std::max(peak_inflight, inflight);
              running++;
              peak_running = std::max(peak_running, running);
              q->state = 1;
              break;
            }
          }
          cv_work.wait(lk);
        }
      }
      q->t_start = clock();
      int rc = run_one(s, q);
      q->t_end = clock();
      {
        std::lock_guard<std::mutex> lk(mu);
        q->status = rc;
        if (rc) snprintf(q->error, sizeof(q->error), "%s", wbfmm::last_error());
        q->state = 2;
        inflight -= q->footprint;
        running--;
        completed++;
        launches += q->launches;
      }
      cv_done.notify_all();
      cv_work.notify_all();
    }
  }
};

extern "C" {

int wbfmm_b200_server_create(wbfmm_b200_server_t** out, int nslots,
                             int64_t hbm_budget) {
  if (!out || nslots < 1 || nslots > 256 || hbm_budget <= 0)
    return set_error(WBFMM_B200_E_ARG, "server: bad arguments");
  *out = nullptr;
  if (wbfmm_b200_device_count() < 1)
    return set_error(WBFMM_B200_E_NOGPU, "no CUDA device is available");
  auto* srv = new wbfmm_b200_server();
  if (cudaGetDevice(&srv->device) != cudaSuccess) {
    delete srv;
    return set_error(WBFMM_B200_E_NOGPU, "no current CUDA device");
  }
  // each slot may keep up to a quarter of its share of the budget (at most
  // 4 GB) of work buffers between solves; admission counts the rest
  srv->keep = std::min<int64_t>(hbm_budget / (4 * (int64_t)nslots), (int64_t)4 << 30);
  srv->budget = hbm_budget - srv->keep * nslots;
  srv->epoch = now_s();
  // A pool of the server's own: freed memory stays cached (solves
  // reallocate cheaply) and is reused only once its free has completed, so
  // the pool never makes one slot's stream wait for another's.
  cudaMemPoolProps props;
  memset(&props, 0, sizeof(props));
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = srv->device;
  if (cudaMemPoolCreate(&srv->pool, &props) != cudaSuccess) {
    cudaGetLastError();
    delete srv;
    return set_error(WBFMM_B200_E_NOMEM, "server: memory pool creation failed");
  }
  srv->cache.pool = srv->pool;
  uint64_t thr = UINT64_MAX;
  int off = 0;
  cudaMemPoolSetAttribute(srv->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  cudaMemPoolSetAttribute(srv->pool, cudaMemPoolReuseAllowInternalDependencies, &off);
  for (int i = 0; i < nslots; i++) {
    auto* s = new wbfmm_b200_server::Slot();
    srv->slots.push_back(s);
    if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&s->done, cudaEventBlockingSync | cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      delete srv;
      return set_error(WBFMM_B200_E_NOMEM, "server: stream creation failed");
    }
  }
  for (auto* s : srv->slots) s->th = std::thread([srv, s] { srv->slot_main(s); });
  *out = srv;
  return 0;
}

int wbfmm_b200_server_destroy(wbfmm_b200_server_t* srv) {
  delete srv;
  return 0;
}

double wbfmm_b200_server_clock(wbfmm_b200_server_t* srv) {
  return srv ? srv->clock() : 0.0;
}

int wbfmm_b200_server_submit(wbfmm_b200_server_t* srv,
                             const wbfmm_b200_request_t* r, int64_t* ticket) {
  if (!srv || !r || !ticket) return set_error(WBFMM_B200_E_ARG, "null argument");
  if (r->nsrc <= 0 || r->ntgt <= 0 || !r->xs || !r->xt || (!r->q && !r->dipoles))
    return set_error(WBFMM_B200_E_ARG, "request needs sources, strengths and targets");
  if (r->dipoles && !r->normals)
    return set_error(WBFMM_B200_E_ARG, "dipole strengths need normals");
  if (r->cfg.precision != WBFMM_B200_FP32 && r->cfg.precision != WBFMM_B200_FP64)
    return set_error(WBFMM_B200_E_ARG, "precision must be FP64 (0) or FP32 (1)");
  if (r->cfg.sparse)
    return set_error(WBFMM_B200_E_ARG, "served requests use dense level storage (sparse storage sizes its arrays with a host wait)");
  auto* q = new Req();
  q->r = *r;
  q->footprint = wbfmm_b200_footprint(&r->cfg, r->nsrc, r->ntgt);
  if (q->footprint > srv->budget) {
    delete q;
    return set_error(WBFMM_B200_E_ADMISSION, "request footprint exceeds the server's device-memory budget");
  }
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    q->id = srv->next_id++;
    double t = srv->clock();
    q->t_arrival = r->arrival > t ? r->arrival : t;
    auto it = srv->queue.end();
    while (it != srv->queue.begin() && (*(it - 1))->t_arrival > q->t_arrival) --it;
    srv->queue.insert(it, q);
    srv->reqs[q->id] = q;
    *ticket = q->id;
  }
  srv->cv_work.notify_all();
  return 0;
}

int wbfmm_b200_server_set_order(wbfmm_b200_server_t* srv, int largest_first) {
  if (!srv) return set_error(WBFMM_B200_E_ARG, "null server");
  std::lock_guard<std::mutex> lk(srv->mu);
  srv->largest_first = largest_first != 0;
  return 0;
}

int wbfmm_b200_server_poll(wbfmm_b200_server_t* srv, int64_t ticket) {
  if (!srv) return set_error(WBFMM_B200_E_ARG, "null server");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(ticket);
  if (it == srv->reqs.end()) return set_error(WBFMM_B200_E_ARG, "unknown ticket");
  return it->second->state == 2 ? 1 : 0;
}

int wbfmm_b200_server_wait(wbfmm_b200_server_t* srv, int64_t ticket) {
  if (!srv) return set_error(WBFMM_B200_E_ARG, "null server");
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(ticket);
  if (it == srv->reqs.end()) return set_error(WBFMM_B200_E_ARG, "unknown ticket");
  Req* q = it->second;
  srv->cv_done.wait(lk, [q] { return q->state == 2; });
  if (q->status) return set_error(q->status, q->error);
  return 0;
}

int wbfmm_b200_server_times(wbfmm_b200_server_t* srv, int64_t ticket,
                            double* t4) {
  if (!srv || !t4) return set_error(WBFMM_B200_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(ticket);
  if (it == srv->reqs.end()) return set_error(WBFMM_B200_E_ARG, "unknown ticket");
  // a running request's slot writes its times without the lock; they are
  // read only once its completion (written under the lock) is seen
  const Req* q = it->second;
  if (q->state != 2) return set_error(WBFMM_B200_E_STATE, "request not complete");
  t4[0] = q->t_arrival;
  t4[1] = q->t_start;
  t4[2] = q->t_queued;
  t4[3] = q->t_end;
  return 0;
}

int wbfmm_b200_server_forget(wbfmm_b200_server_t* srv, int64_t ticket) {
  if (!srv) return set_error(WBFMM_B200_E_ARG, "null server");
  std::lock_guard<std::mutex> lk(srv->mu);
  auto it = srv->reqs.find(ticket);
  if (it == srv->reqs.end()) return set_error(WBFMM_B200_E_ARG, "unknown ticket");
  if (it->second->state != 2) return set_error(WBFMM_B200_E_STATE, "request not complete");
  delete it->second;
  srv->reqs.erase(it);
  return 0;
}

int wbfmm_b200_server_drain(wbfmm_b200_server_t* srv) {
  if (!srv) return set_error(WBFMM_B200_E_ARG, "null server");
  std::unique_lock<std::mutex> lk(srv->mu);
  srv->cv_done.wait(lk, [srv] { return srv->queue.empty() && srv->running == 0; });
  return 0;
}

int wbfmm_b200_server_stats(wbfmm_b200_server_t* srv, int64_t* out7) {
  if (!srv || !out7) return set_error(WBFMM_B200_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(srv->mu);
  std::lock_guard<std::mutex> lc(srv->cache.mu);
  out7[0] = srv->completed;
  out7[1] = srv->peak_inflight;
  out7[2] = srv->peak_running;
  out7[3] = srv->cache.hits;
  out7[4] = srv->cache.misses;
  out7[5] = (int64_t)srv->cache.bytes;
  out7[6] = srv->launches;
  return 0;
}

}  // extern "C"
