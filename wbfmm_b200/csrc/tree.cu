// Tree build on the GPU: Morton keys, a stable LSD radix sort, and the
// level-by-level box ranges of wbfmm_tree_refine, all bit-exact with the
// reference (src/boxes.c:93-339, src/indexing.c:68-178).
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include "engine.h"

namespace wbfmm {

// ----------------------------------------------------------------- errors
static thread_local char g_err[512] = "";

int set_cuda_error(cudaError_t e, const char* file, int line) {
  snprintf(g_err, sizeof(g_err), "CUDA error %d (%s) at %s:%d", (int)e,
           cudaGetErrorString(e), file, line);
  return -(int)e - 1000;
}
int set_error(int code, const char* msg) {
  snprintf(g_err, sizeof(g_err), "%s", msg);
  return code;
}
const char* last_error() { return g_err; }

// ------------------------------------------------------------------- keys
// (x - c)/D*2^20 truncated per axis: the division comes first and the
// scaling by 2^20 is exact, so this is bit-identical to the host formula
// With f32, the single-precision build's arithmetic (src/boxes.c:324-339
// compiled with WBFMM_REAL = gfloat): coordinates, origin and width are
// FP32 values (held exactly in the FP64 inputs) and every step rounds to
// FP32.
__device__ __forceinline__ uint32_t key_coord(double x, double x0, double D, bool f32) {
  if (f32)
    return (uint32_t)__fmul_rn(__fdiv_rn(__fsub_rn((float)x, (float)x0), (float)D), 1048576.0f);
  return (uint32_t)(__ddiv_rn(__dsub_rn(x, x0), D) * 1048576.0);
}

__global__ void k_point_keys(const double* __restrict__ pts, int64_t pstr,
                             int n, double x0, double y0, double z0, double D,
                             uint64_t* __restrict__ keys,
                             uint32_t* __restrict__ vals, bool f32) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = pts + (int64_t)i * pstr;
  uint32_t xi = key_coord(p[0], x0, D, f32);
  uint32_t yi = key_coord(p[1], y0, D, f32);
  uint32_t zi = key_coord(p[2], z0, D, f32);
  // Points strictly inside the cube give 20-bit coordinates.  Anything else
  // (rejected by the domain check, which the served form reads back only
  // after the solve) is clamped so every key stays below 2^60 and every box
  // index derived from it inside its level's array.
  const uint32_t top = (1u << 20) - 1;
  xi = xi < top ? xi : top; yi = yi < top ? yi : top; zi = zi < top ? zi : top;
  keys[i] = morton(xi, yi, zi);
  vals[i] = (uint32_t)i;
}

void launch_point_keys(const double* pts, int64_t pstr, int n,
                       const double* x0, double D, uint64_t* keys,
                       uint32_t* vals, cudaStream_t s, bool f32) {
  if (n <= 0) return;
  k_point_keys<<<(n + 255) / 256, 256, 0, s>>>(pts, pstr, n, x0[0], x0[1],
                                               x0[2], D, keys, vals, f32);
}

// wbfmm_point_box (src/boxes.c:585-634); with f32 in FP32 arithmetic
__device__ __forceinline__ bool outside_closed(double x, double x0, double D, bool f32) {
  if (f32) {
    const float xf = (float)x, x0f = (float)x0;
    return xf < x0f || xf > __fadd_rn(x0f, (float)D);
  }
  return x < x0 || x > x0 + D;
}
__device__ __forceinline__ uint32_t box_coord(double x, double x0, double D, int level, bool f32) {
  if (f32) {
    const float wb = __fdiv_rn((float)D, (float)(1u << level));
    return (uint32_t)floorf(__fdiv_rn(__fsub_rn((float)x, (float)x0), wb));
  }
  const double wb = __ddiv_rn(D, (double)(1u << level));
  return (uint32_t)floor(__ddiv_rn(__dsub_rn(x, x0), wb));
}

__global__ void k_target_keys(const double* __restrict__ pts, int64_t pstr,
                              int n, double x0, double y0, double z0, double D,
                              int level, uint64_t* __restrict__ keys,
                              uint32_t* __restrict__ vals, int* bad, bool f32) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = pts + (int64_t)i * pstr;
  double x = p[0], y = p[1], z = p[2];
  if (outside_closed(x, x0, D, f32) || outside_closed(y, y0, D, f32) ||
      outside_closed(z, z0, D, f32)) {
    *bad = 1;
    keys[i] = 0;
    vals[i] = (uint32_t)i;
    return;
  }
  uint32_t a = box_coord(x, x0, D, level, f32);
  uint32_t b = box_coord(y, y0, D, level, f32);
  uint32_t c = box_coord(z, z0, D, level, f32);
  // a point on the upper face gives 2^level; the reference then indexes
  // out of its box array, here the index is clamped into the last box
  uint32_t nb = 1u << level;
  a = a < nb ? a : nb - 1; b = b < nb ? b : nb - 1; c = c < nb ? c : nb - 1;
  keys[i] = morton(a, b, c);
  vals[i] = (uint32_t)i;
}

// *a = va and, when b is given, *b = vb: device-side initialisation of
// flags and roots, so that no pageable host->device copy (which may wait for
// the stream to drain) sits in the middle of a solve
__global__ void k_set_words(uint32_t* a, uint32_t va, uint32_t* b, uint32_t vb) {
  *a = va;
  if (b) *b = vb;
}

void launch_set_words(uint32_t* a, uint32_t va, uint32_t* b, uint32_t vb,
                      cudaStream_t s) {
  k_set_words<<<1, 1, 0, s>>>(a, va, b, vb);
}

void launch_target_keys(const double* pts, int64_t pstr, int n,
                        const double* x0, double D, int level,
                        uint64_t* keys, uint32_t* vals, int* bad,
                        cudaStream_t s, bool f32) {
  if (n <= 0) return;
  k_target_keys<<<(n + 255) / 256, 256, 0, s>>>(pts, pstr, n, x0[0], x0[1],
                                                x0[2], D, level, keys, vals,
                                                bad, f32);
}

// strict interior (src/boxes.c:148-153); with f32 in FP32 arithmetic
__device__ __forceinline__ bool outside_open(double x, double x0, double D, bool f32) {
  if (f32) {
    const float xf = (float)x, x0f = (float)x0;
    return xf <= x0f || xf >= __fadd_rn(x0f, (float)D);
  }
  return x <= x0 || x >= x0 + D;
}

__global__ void k_domain_check(const double* __restrict__ pts, int64_t pstr,
                               int n, double x0, double y0, double z0,
                               double D, int* bad, bool f32) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* p = pts + (int64_t)i * pstr;
  if (outside_open(p[0], x0, D, f32) || outside_open(p[1], y0, D, f32) ||
      outside_open(p[2], z0, D, f32))
    atomicMin(bad, i);
}

void launch_domain_check(const double* pts, int64_t pstr, int n,
                         const double* x0, double D, int* bad, cudaStream_t s,
                         bool f32) {
  if (n <= 0) return;
  k_domain_check<<<(n + 255) / 256, 256, 0, s>>>(pts, pstr, n, x0[0], x0[1],
                                                 x0[2], D, bad, f32);
}

// ------------------------------------------------------------ radix sort
// Stable LSD radix sort, 8-bit digits.  Each pass: per-tile digit
// histograms (digit-major), one exclusive scan, then a scatter in which
// every tile ranks its elements round by round (warp match + per-warp
// digit counts), which keeps equal digits in input order.
constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;

__global__ void k_radix_hist(const uint64_t* __restrict__ keys, int n, int shift,
                             int ntiles, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * kSortTile;
  for (int r = 0; r < kSortItems; r++) {
    int i = base + r * kSortThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(keys[i] >> shift) & 0xff], 1u);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// exclusive scan of m entries by one block of 1024 threads
__global__ void k_scan_exclusive(uint32_t* data, int m) {
  __shared__ uint32_t sums[1024];
  int t = threadIdx.x;
  int per = (m + 1023) / 1024;
  int lo = t * per, hi = min(lo + per, m);
  uint32_t s = 0;
  for (int i = lo; i < hi; i++) s += data[i];
  sums[t] = s;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    uint32_t v = t >= off ? sums[t - off] : 0;
    __syncthreads();
    sums[t] += v;
    __syncthreads();
  }
  uint32_t run = t > 0 ? sums[t - 1] : 0;
  for (int i = lo; i < hi; i++) {
    uint32_t v = data[i];
    data[i] = run;
    run += v;
  }
}

__global__ void k_radix_scatter(const uint64_t* __restrict__ keys,
                                const uint32_t* __restrict__ vals, int n,
                                int shift, int ntiles,
                                const uint32_t* __restrict__ offs,
                                uint64_t* __restrict__ okeys,
                                uint32_t* __restrict__ ovals) {
  __shared__ uint32_t base[256];
  __shared__ uint32_t wcnt[kSortThreads / 32][256];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  base[t] = offs[t * ntiles + blockIdx.x];
  int tile0 = blockIdx.x * kSortTile;
  for (int r = 0; r < kSortItems; r++) {
    for (int w = 0; w < kSortThreads / 32; w++) wcnt[w][t] = 0;
    __syncthreads();
    int i = tile0 + r * kSortThreads + t;
    bool valid = i < n;
    uint64_t key = valid ? keys[i] : 0;
    uint32_t d = valid ? (uint32_t)((key >> shift) & 0xff) : 256u + lane;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int rank = __popc(peers & ((1u << lane) - 1));
    if (valid && rank == 0) wcnt[warp][d] = __popc(peers);
    __syncthreads();
    {  // per digit: prefix over warps, advance the digit base
      uint32_t run = base[t];
      for (int w = 0; w < kSortThreads / 32; w++) {
        uint32_t c = wcnt[w][t];
        wcnt[w][t] = run;
        run += c;
      }
      base[t] = run;
    }
    __syncthreads();
    if (valid) {
      uint32_t pos = wcnt[warp][d] + rank;
      okeys[pos] = key;
      ovals[pos] = vals[i];
    }
    __syncthreads();
  }
}

cudaMemPool_t library_pool();   // solver.cu

// Growth of the sort's scratch, stream-ordered from the library's pool: a
// solver that meets a larger point count (a serving slot, say) does not
// synchronise the device as cudaFree / cudaMalloc would.
template <typename X>
static cudaError_t scratch_regrow(X** p, size_t count, cudaStream_t s) {
  if (*p) cudaFreeAsync(*p, s);
  *p = nullptr;
  cudaMemPool_t pl = library_pool();
  return pl ? cudaMallocFromPoolAsync((void**)p, sizeof(X) * count, pl, s)
            : cudaMallocAsync((void**)p, sizeof(X) * count, s);
}

int radix_sort_pairs(uint64_t* keys, uint32_t* vals, int n, int bits,
                     RadixScratch* scr, cudaStream_t s, int lo) {
  if (n <= 1) return 0;
  int ntiles = (n + kSortTile - 1) / kSortTile;
  if (scr->cap < (size_t)n) {
    scr->cap = 0;
    WBFMM_CUDA(scratch_regrow(&scr->keys_alt, (size_t)n, s));
    WBFMM_CUDA(scratch_regrow(&scr->vals_alt, (size_t)n, s));
    scr->cap = n;
  }
  if (scr->hist_cap < (size_t)ntiles * 256) {
    scr->hist_cap = 0;
    WBFMM_CUDA(scratch_regrow(&scr->hist, (size_t)256 * ntiles, s));
    scr->hist_cap = (size_t)ntiles * 256;
  }
  int passes = (bits + 7) / 8;
  uint64_t *ki = keys, *ko = scr->keys_alt;
  uint32_t *vi = vals, *vo = scr->vals_alt;
  for (int p = 0; p < passes; p++) {
    int shift = lo + 8 * p;
    k_radix_hist<<<ntiles, kSortThreads, 0, s>>>(ki, n, shift, ntiles, scr->hist);
    k_scan_exclusive<<<1, 1024, 0, s>>>(scr->hist, 256 * ntiles);
    k_radix_scatter<<<ntiles, kSortThreads, 0, s>>>(ki, vi, n, shift, ntiles,
                                                    scr->hist, ko, vo);
    uint64_t* tk = ki; ki = ko; ko = tk;
    uint32_t* tv = vi; vi = vo; vo = tv;
  }
  if (ki != keys) {
    WBFMM_CUDA(cudaMemcpyAsync(keys, ki, sizeof(uint64_t) * n,
                               cudaMemcpyDeviceToDevice, s));
    WBFMM_CUDA(cudaMemcpyAsync(vals, vi, sizeof(uint32_t) * n,
                               cudaMemcpyDeviceToDevice, s));
  }
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

void radix_scratch_free(RadixScratch* scr) {
  cudaFree(scr->keys_alt); cudaFree(scr->vals_alt); cudaFree(scr->hist);
  *scr = RadixScratch();
}

// ----------------------------------------------------------------- refine
// first sorted position whose level-`level` box id is >= c
__device__ __forceinline__ uint32_t lower_bound_box(const uint64_t* keys,
                                                    int n, int shift,
                                                    uint64_t c) {
  uint32_t lo = 0, hi = (uint32_t)n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if ((keys[mid] >> shift) < c) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Child c of parent P (level `level` boxes):
//   n = number of points in c;
//   i = P.i (before refinement) for the first child; for the others, the
//       sorted position of c's first point when the reference's scan
//       reaches c (i.e. c is not past the parent's last point), else 0.
__global__ void k_refine_children(const uint64_t* __restrict__ keys, int npts,
                                  int level, const uint32_t* __restrict__ pi,
                                  uint32_t* __restrict__ ci,
                                  uint32_t* __restrict__ cn) {
  int64_t nb = (int64_t)1 << (3 * level);
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nb) return;
  int shift = 3 * (20 - level);
  uint32_t lb = lower_bound_box(keys, npts, shift, (uint64_t)c);
  uint32_t ub = lower_bound_box(keys, npts, shift, (uint64_t)c + 1);
  uint32_t pend = lower_bound_box(keys, npts, shift, (uint64_t)((c | 7) + 1));
  cn[c] = ub - lb;
  if ((c & 7) == 0) ci[c] = pi[c >> 3];
  else ci[c] = lb < pend ? lb : 0u;
}

__global__ void k_refine_parents(int64_t np, uint32_t* __restrict__ pi,
                                 const uint32_t* __restrict__ pn) {
  int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < np) pi[p] += pn[p];
}

void launch_refine_children(const uint64_t* sorted_keys, int npts, int level,
                            const uint32_t* parent_i, uint32_t* child_i,
                            uint32_t* child_n, cudaStream_t s) {
  int64_t nb = (int64_t)1 << (3 * level);
  k_refine_children<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(
      sorted_keys, npts, level, parent_i, child_i, child_n);
}

void launch_refine_parents(int level, uint32_t* parent_i,
                           const uint32_t* parent_n, cudaStream_t s) {
  int64_t np = (int64_t)1 << (3 * level);
  k_refine_parents<<<(unsigned)((np + 255) / 256), 256, 0, s>>>(np, parent_i,
                                                                parent_n);
}

__global__ void k_box_ranges(const uint64_t* __restrict__ ids, int n,
                             int64_t nb, uint32_t* __restrict__ start,
                             uint32_t* __restrict__ count) {
  int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nb) return;
  uint32_t lb = lower_bound_box(ids, n, 0, (uint64_t)c);
  uint32_t ub = lower_bound_box(ids, n, 0, (uint64_t)c + 1);
  start[c] = lb;
  count[c] = ub - lb;
}

void launch_box_ranges(const uint64_t* sorted_ids, int n, int level,
                       uint32_t* start, uint32_t* count, cudaStream_t s) {
  int64_t nb = (int64_t)1 << (3 * level);
  k_box_ranges<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(sorted_ids, n, nb,
                                                            start, count);
}

// ----------------------------------------------------------------- gathers
__global__ void k_gather_points(const double* __restrict__ pts, int64_t pstr,
                                const uint32_t* __restrict__ ip, int n,
                                double* __restrict__ x, double* __restrict__ y,
                                double* __restrict__ z) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double* p = pts + (int64_t)ip[j] * pstr;
  x[j] = p[0]; y[j] = p[1]; z[j] = p[2];
}

void launch_gather_points(const double* pts, int64_t pstr, const uint32_t* ip,
                          int n, double* x, double* y, double* z,
                          cudaStream_t s) {
  if (n <= 0) return;
  k_gather_points<<<(n + 255) / 256, 256, 0, s>>>(pts, pstr, ip, n, x, y, z);
}

template <typename T>
__global__ void k_gather_real(const double* __restrict__ src, int64_t sstr,
                              const uint32_t* __restrict__ ip, int n, int ncomp,
                              T* __restrict__ dst) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double* p = src + (int64_t)ip[j] * sstr;
  for (int c = 0; c < ncomp; c++) dst[(int64_t)j * ncomp + c] = (T)p[c];
}

void launch_gather_real(const double* src, int64_t sstr, const uint32_t* ip,
                        int n, int ncomp, double* dst, cudaStream_t s) {
  if (n <= 0) return;
  k_gather_real<double><<<(n + 255) / 256, 256, 0, s>>>(src, sstr, ip, n, ncomp, dst);
}

void launch_gather_real_f32(const double* src, int64_t sstr, const uint32_t* ip,
                            int n, int ncomp, float* dst, cudaStream_t s) {
  if (n <= 0) return;
  k_gather_real<float><<<(n + 255) / 256, 256, 0, s>>>(src, sstr, ip, n, ncomp, dst);
}

}  // namespace wbfmm
