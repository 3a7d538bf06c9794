// Operator tables shared by the solves of a server (included by solver.h).
//
// Rotation tables, per-shift angles and phases and the Laplace coaxial
// tables depend only on the expansion order, so one set, built for the
// largest order seen so far, serves every solve; a request of higher order
// builds a larger set (earlier sets stay alive for the solves using them).
// Helmholtz coaxial tables depend on (k * box width, order): they are kept
// per key, reference-counted while a solve uses them, and the least
// recently used unreferenced ones are released above a byte cap.
// Entries are written on the stream of the solve that first needs them; an
// event marks them ready and other streams wait on it.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <condition_variable>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/wbfmm_b200.h"
#include "engine.h"
#include "fmm_math.cuh"
#include "kernels.h"
#include "tables.h"

namespace wbfmm {

// Host per-shift tables for phases up to order L (L + 1 entries per shift):
// rotation index, list-4 distance index, distance, (cos, sin)(m ph) and
// (cos, sin)(m ch) (src/shift.c:587-724 tabulates the same angles).
inline void shift_op_tables(const ShiftGeometry& geom, int L,
                            std::vector<int>& ith, std::vector<int>& dist,
                            std::vector<double>& r, std::vector<double>& ph,
                            std::vector<double>& ch) {
  ith.assign(kNumOps, 0);
  dist.assign(kNumOps, 0);
  r.assign(kNumOps, 0.0);
  ph.assign((size_t)kNumOps * (L + 1) * 2, 0.0);
  ch.assign((size_t)kNumOps * (L + 1) * 2, 0.0);
  for (int op = 0; op < kNumOps; op++) {
    const ShiftAngles& a = op < kOpM2M ? geom.offset[op]
                          : op < kOpL2L ? geom.child_to_parent[op - kOpM2M]
                                        : geom.parent_to_child[op - kOpL2L];
    ith[op] = a.ith < 0 ? 0 : a.ith;
    dist[op] = op < kOpM2M ? std::max(0, list_dist_index(a.idist)) : 0;
    r[op] = a.r;
    for (int m = 0; m <= L; m++) {
      ph[((size_t)op * (L + 1) + m) * 2 + 0] = cos(m * a.ph);
      ph[((size_t)op * (L + 1) + m) * 2 + 1] = sin(m * a.ph);
      ch[((size_t)op * (L + 1) + m) * 2 + 0] = cos(m * a.ch);
      ch[((size_t)op * (L + 1) + m) * 2 + 1] = sin(m * a.ch);
    }
  }
}

template <typename T>
__global__ void k_cache_narrow(const double* __restrict__ a, T* __restrict__ b,
                               int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (T)a[i];
}

struct TableCache {
  // order-only tables, FP64 masters and FP32 copies
  struct Geo {
    int L = 0;                  // phases and rotations cover degrees < L
    int64_t hstride = 0;
    int nth = 0;
    double* H64 = nullptr; float* H32 = nullptr;
    int* op_ith = nullptr; int* op_dist = nullptr;
    double* r64 = nullptr; float* r32 = nullptr;
    double* ph64 = nullptr; float* ph32 = nullptr;
    double* ch64 = nullptr; float* ch32 = nullptr;
    double* lap64[3] = {nullptr, nullptr, nullptr};
    float* lap32[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t ready = nullptr;
  };
  // Helmholtz coaxial table for one (kind, k w bits, order)
  struct Coax {
    double* d64 = nullptr; float* d32 = nullptr;
    int64_t count = 0;           // doubles
    cudaEvent_t ready = nullptr;
    int refs = 0;
    uint64_t last = 0;
    int state = 1;               // 0 being built, 1 ready, -1 build failed
  };
  using Key = std::tuple<int, uint64_t, int>;

  std::mutex mu;
  std::condition_variable built;  // a coaxial entry left the "being built" state
  cudaMemPool_t pool = nullptr;   // stream-ordered allocations when set
  std::vector<Geo*> geos;
  std::map<Key, Coax*> coax;
  size_t coax_bytes = 0, coax_cap = (size_t)4 << 30;
  uint64_t tick = 0;
  int64_t hits = 0, misses = 0;

  ~TableCache() { clear(); }

  // release every table (no solve may be using them)
  void clear() {
    for (Geo* g : geos) {
      void* ps[] = {g->H64, g->H32, g->op_ith, g->op_dist, g->r64, g->r32,
                    g->ph64, g->ph32, g->ch64, g->ch32, g->lap64[0], g->lap64[1],
                    g->lap64[2], g->lap32[0], g->lap32[1], g->lap32[2]};
      for (void* p : ps) cudaFree(p);
      if (g->ready) cudaEventDestroy(g->ready);
      delete g;
    }
    geos.clear();
    for (auto& e : coax) drop(e.second, nullptr);
    coax.clear();
    coax_bytes = 0;
  }

  // frees stream-ordered on s when given (the entry is unreferenced, so no
  // queued work reads it), else synchronously
  void drop(Coax* c, cudaStream_t s) {
    free_tables(c, s);
    delete c;
  }
  void free_tables(Coax* c, cudaStream_t s) {
    if (s) {
      if (c->d64) cudaFreeAsync(c->d64, s);
      if (c->d32) cudaFreeAsync(c->d32, s);
    } else {
      cudaFree(c->d64);
      cudaFree(c->d32);
    }
    if (c->ready) cudaEventDestroy(c->ready);
    c->d64 = nullptr; c->d32 = nullptr; c->ready = nullptr;
  }

  template <typename X>
  int dalloc(X** p, size_t n, cudaStream_t s) {
    cudaError_t e = pool ? cudaMallocFromPoolAsync((void**)p, sizeof(X) * (n ? n : 1), pool, s)
                         : cudaMalloc(p, sizeof(X) * (n ? n : 1));
    if (e != cudaSuccess) {
      cudaGetLastError();
      *p = nullptr;
      return set_error(WBFMM_B200_E_NOMEM, "table cache allocation failed");
    }
    return 0;
  }

  static int narrow(const double* a, float* b, int64_t n, cudaStream_t s) {
    if (n <= 0) return 0;
    k_cache_narrow<float><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, b, n);
    WBFMM_CUDA(cudaGetLastError());
    return 0;
  }

#define WBFMM_CACHE_TRY(call)        \
  do {                               \
    int rc_ = (call);                \
    if (rc_ != 0) return rc_;        \
  } while (0)

  // release a Geo's tables and event (stream-ordered on s for pool memory)
  // and the Geo
  void drop_geo(Geo* g, cudaStream_t s) {
    void* ps[] = {g->H64, g->H32, g->op_ith, g->op_dist, g->r64, g->r32,
                  g->ph64, g->ph32, g->ch64, g->ch32, g->lap64[0], g->lap64[1],
                  g->lap64[2], g->lap32[0], g->lap32[1], g->lap32[2]};
    for (void* p : ps)
      if (p) {
        if (pool) cudaFreeAsync(p, s);
        else cudaFree(p);
      }
    if (g->ready) cudaEventDestroy(g->ready);
    delete g;
  }

  // build the order-only tables for phases up to L (caller holds mu); a
  // failure part way releases what was allocated
  int build_geo(int L, cudaStream_t s, Geo** out) {
    Geo* g = new Geo();
    const int rc = fill_geo(g, L, s);
    if (rc) {
      cudaGetLastError();
      drop_geo(g, s);
      return rc;
    }
    geos.push_back(g);
    *out = g;
    return 0;
  }

  int fill_geo(Geo* g, int L, cudaStream_t s) {
    g->L = L;
    ShiftGeometry geom;
    build_shift_geometry(&geom);
    std::vector<int> ith, dist;
    std::vector<double> r, ph, ch;
    shift_op_tables(geom, L, ith, dist, r, ph, ch);
    const size_t nph = ph.size();
    WBFMM_CACHE_TRY(dalloc(&g->op_ith, kNumOps, s));
    WBFMM_CACHE_TRY(dalloc(&g->op_dist, kNumOps, s));
    WBFMM_CACHE_TRY(dalloc(&g->r64, kNumOps, s));
    WBFMM_CACHE_TRY(dalloc(&g->r32, kNumOps, s));
    WBFMM_CACHE_TRY(dalloc(&g->ph64, nph, s));
    WBFMM_CACHE_TRY(dalloc(&g->ph32, nph, s));
    WBFMM_CACHE_TRY(dalloc(&g->ch64, nph, s));
    WBFMM_CACHE_TRY(dalloc(&g->ch32, nph, s));
    WBFMM_CUDA(cudaMemcpyAsync(g->op_ith, ith.data(), sizeof(int) * kNumOps, cudaMemcpyHostToDevice, s));
    WBFMM_CUDA(cudaMemcpyAsync(g->op_dist, dist.data(), sizeof(int) * kNumOps, cudaMemcpyHostToDevice, s));
    WBFMM_CUDA(cudaMemcpyAsync(g->r64, r.data(), sizeof(double) * kNumOps, cudaMemcpyHostToDevice, s));
    WBFMM_CUDA(cudaMemcpyAsync(g->ph64, ph.data(), sizeof(double) * nph, cudaMemcpyHostToDevice, s));
    WBFMM_CUDA(cudaMemcpyAsync(g->ch64, ch.data(), sizeof(double) * nph, cudaMemcpyHostToDevice, s));
    WBFMM_CACHE_TRY(narrow(g->r64, g->r32, kNumOps, s));
    WBFMM_CACHE_TRY(narrow(g->ph64, g->ph32, (int64_t)nph, s));
    WBFMM_CACHE_TRY(narrow(g->ch64, g->ch32, (int64_t)nph, s));
    g->hstride = rot_count(L) + 8;
    g->nth = (int)geom.thetas.size();
    const size_t nh = (size_t)g->hstride * g->nth;
    WBFMM_CACHE_TRY(dalloc(&g->H64, nh, s));
    WBFMM_CACHE_TRY(dalloc(&g->H32, nh, s));
    WBFMM_CACHE_TRY(generate_rotation_tables(geom.thetas, L, g->H64, g->hstride, s));
    WBFMM_CACHE_TRY(narrow(g->H64, g->H32, (int64_t)nh, s));
    const size_t n3 = (size_t)(L + 1) * (L + 1) * (L + 1);
    for (int i = 0; i < 3; i++) {
      WBFMM_CACHE_TRY(dalloc(&g->lap64[i], n3, s));
      WBFMM_CACHE_TRY(dalloc(&g->lap32[i], n3, s));
    }
    WBFMM_CACHE_TRY(generate_laplace_tables(L, g->lap64[0], g->lap64[1], g->lap64[2], s));
    for (int i = 0; i < 3; i++) WBFMM_CACHE_TRY(narrow(g->lap64[i], g->lap32[i], (int64_t)n3, s));
    WBFMM_CUDA(cudaEventCreateWithFlags(&g->ready, cudaEventDisableTiming));
    WBFMM_CUDA(cudaEventRecord(g->ready, s));
    return 0;
  }

  // Order-only tables covering phases up to L, ready on stream s.
  template <typename T>
  int geometry(int L, cudaStream_t s, OpTables<T>* t) {
    Geo* g = nullptr;
    {
      std::lock_guard<std::mutex> lk(mu);
      for (Geo* c : geos)
        if (c->L >= L && (!g || c->L < g->L)) g = c;
      if (!g) {
        int Lb = L < 24 ? 24 : ((L + 7) / 8) * 8;   // headroom: fewer rebuilds
        WBFMM_CACHE_TRY(build_geo(Lb, s, &g));
      } else {
        WBFMM_CUDA(cudaStreamWaitEvent(s, g->ready, 0));
      }
    }
    const bool f32 = sizeof(T) == 4;
    t->H = f32 ? (const T*)g->H32 : (const T*)g->H64;
    t->hstride = g->hstride;
    t->op_ith = g->op_ith;
    t->op_dist = g->op_dist;
    t->op_r = f32 ? (const T*)g->r32 : (const T*)g->r64;
    t->ph = f32 ? (const T*)g->ph32 : (const T*)g->ph64;
    t->ch = f32 ? (const T*)g->ch32 : (const T*)g->ch64;
    t->lmax = g->L;
    t->lapSS = f32 ? (const T*)g->lap32[0] : (const T*)g->lap64[0];
    t->lapRR = f32 ? (const T*)g->lap32[1] : (const T*)g->lap64[1];
    t->lapSR = f32 ? (const T*)g->lap32[2] : (const T*)g->lap64[2];
    t->lt = g->L;
    return 0;
  }

  // Helmholtz coaxial table: kind 0 = (S|R) at the 15 list-4 distances
  // k w sqrt(d2) (complex, stride 2 (coax_count(L) + 1) per distance);
  // kind 1 = (R|R) at k w sqrt(3)/2 (real).  Returns a referenced entry.
  // The (kind, k w, L) coaxial table, shared: a hit waits (on the stream)
  // for the table's build; a miss builds it outside the cache's lock, so
  // solves building different tables (every Helmholtz request of a served
  // stream has its own k) do not queue behind each other.
  template <typename T>
  int coaxial(int kind, double kw, int L, cudaStream_t s, const T** out,
              Coax** ref) {
    uint64_t bits;
    memcpy(&bits, &kw, sizeof(bits));
    Key key(kind, bits, L);
    std::unique_lock<std::mutex> lk(mu);
    Coax* c = nullptr;
    auto it = coax.find(key);
    if (it != coax.end()) {
      c = it->second;
      hits++;
      c->refs++;
      c->last = ++tick;
      built.wait(lk, [c] { return c->state != 0; });
      if (c->state < 0) {
        if (--c->refs == 0) delete c;
        return set_error(WBFMM_B200_E_NOMEM, "coaxial table build failed");
      }
      cudaEvent_t ev = c->ready;
      lk.unlock();
      const cudaError_t e = cudaStreamWaitEvent(s, ev, 0);
      if (e != cudaSuccess) {
        lk.lock();
        c->refs--;
        return set_cuda_error(e, __FILE__, __LINE__);
      }
    } else {
      misses++;
      c = new Coax();
      c->state = 0;
      c->refs = 1;
      c->last = ++tick;
      coax[key] = c;
      lk.unlock();
      const int64_t per = (int64_t)(L + 1) * (L + 2) * (L + 3) / 6 + 1;
      std::vector<double> krs;
      int nc;
      if (kind == 0) {
        for (int i = 0; i < 15; i++) krs.push_back(kw * sqrt((double)kListDist2[i]));
        nc = 2;
      } else {
        krs.push_back(kw * 0.5 * sqrt(3.0));
        nc = 1;
      }
      c->count = per * nc * (int64_t)krs.size();
      int rc = dalloc(&c->d64, (size_t)c->count, s);
      if (!rc) rc = dalloc(&c->d32, (size_t)c->count, s);
      if (!rc) rc = generate_coaxial_tables(krs, L, nc, c->d64, per * nc, s);
      if (!rc) rc = narrow(c->d64, c->d32, c->count, s);
      cudaError_t e = cudaSuccess;
      if (!rc) e = cudaEventCreateWithFlags(&c->ready, cudaEventDisableTiming);
      if (!rc && e == cudaSuccess) e = cudaEventRecord(c->ready, s);
      if (!rc && e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
      lk.lock();
      if (rc) {
        coax.erase(key);
        free_tables(c, s);
        c->state = -1;
        built.notify_all();
        if (--c->refs == 0) delete c;    // else the last waiter deletes it
        return rc;
      }
      c->state = 1;
      coax_bytes += (size_t)c->count * 12;
      built.notify_all();
      evict(s);
    }
    *out = sizeof(T) == 4 ? (const T*)c->d32 : (const T*)c->d64;
    *ref = c;
    return 0;
  }

  void release(Coax* c) {
    std::lock_guard<std::mutex> lk(mu);
    if (c->refs > 0) c->refs--;
  }

  // drop least recently used unreferenced entries above the cap (mu held)
  void evict(cudaStream_t s) {
    while (coax_bytes > coax_cap) {
      auto victim = coax.end();
      for (auto it = coax.begin(); it != coax.end(); ++it)
        if (it->second->refs == 0 &&
            (victim == coax.end() || it->second->last < victim->second->last))
          victim = it;
      if (victim == coax.end()) return;
      coax_bytes -= (size_t)victim->second->count * 12;
      drop(victim->second, s);
      coax.erase(victim);
    }
  }
#undef WBFMM_CACHE_TRY
};

}  // namespace wbfmm
