// Operator tables shared by the solves of a server (included by solver.h).
//
// Rotation tables, per-shift angles and phases and the Laplace coaxial
// tables depend only on the expansion order, so one set, built for the
// largest order seen so far, serves every solve; a request of higher order
// builds a larger set (earlier sets stay alive for the solves using them).
// A set is written on the stream of the solve that first needs it; an
// event marks it ready and other streams wait on it.  (Helmholtz coaxial
// tables depend on k times the box width, which differs from request to
// request; each solve builds its own, Solver::helm_coaxial_set.)
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <mutex>
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
    size_t nbytes = 0;
  };

  std::mutex mu;
  cudaMemPool_t pool = nullptr;   // stream-ordered allocations when set
  std::vector<Geo*> geos;
  size_t bytes = 0;               // device bytes of the sets
  int64_t hits = 0, misses = 0;   // lookups served by an existing set / building one

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
    bytes = 0;
  }

  template <typename X>
  int dalloc(Geo* g, X** p, size_t n, cudaStream_t s) {
    g->nbytes += sizeof(X) * (n ? n : 1);
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
    bytes += g->nbytes;
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
    WBFMM_CACHE_TRY(dalloc(g, &g->op_ith, kNumOps, s));
    WBFMM_CACHE_TRY(dalloc(g, &g->op_dist, kNumOps, s));
    WBFMM_CACHE_TRY(dalloc(g, &g->r64, kNumOps, s));
    WBFMM_CACHE_TRY(dalloc(g, &g->r32, kNumOps, s));
    WBFMM_CACHE_TRY(dalloc(g, &g->ph64, nph, s));
    WBFMM_CACHE_TRY(dalloc(g, &g->ph32, nph, s));
    WBFMM_CACHE_TRY(dalloc(g, &g->ch64, nph, s));
    WBFMM_CACHE_TRY(dalloc(g, &g->ch32, nph, s));
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
    WBFMM_CACHE_TRY(dalloc(g, &g->H64, nh, s));
    WBFMM_CACHE_TRY(dalloc(g, &g->H32, nh, s));
    WBFMM_CACHE_TRY(generate_rotation_tables(geom.thetas, L, g->H64, g->hstride, s));
    WBFMM_CACHE_TRY(narrow(g->H64, g->H32, (int64_t)nh, s));
    const size_t n3 = (size_t)(L + 1) * (L + 1) * (L + 1);
    for (int i = 0; i < 3; i++) {
      WBFMM_CACHE_TRY(dalloc(g, &g->lap64[i], n3, s));
      WBFMM_CACHE_TRY(dalloc(g, &g->lap32[i], n3, s));
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
        misses++;
      } else {
        WBFMM_CUDA(cudaStreamWaitEvent(s, g->ready, 0));
        hits++;
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

#undef WBFMM_CACHE_TRY
};

}  // namespace wbfmm
