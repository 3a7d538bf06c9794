// Internal C++ interface of the B200 FMM engine: device buffers, kernel
// launchers and the per-solve state shared by the .cu translation units.
// The public boundary is the C ABI in include/wbfmm_b200.h.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <atomic>
#include <vector>

#include "fmm_math.cuh"

namespace wbfmm {

constexpr int kMaxDepth = 16;       // WBFMM_TREE_MAX_DEPTH (src/wbfmm.h:77)
constexpr int kMaxOrder = 62;       // per-point scratch arrays hold <= 64

#define WBFMM_CUDA(call)                                                  \
  do {                                                                    \
    cudaError_t e_ = (call);                                              \
    if (e_ != cudaSuccess) return wbfmm::set_cuda_error(e_, __FILE__, __LINE__); \
  } while (0)

int set_cuda_error(cudaError_t e, const char* file, int line);
int set_error(int code, const char* msg);
const char* last_error();

// Raise kernel K's dynamic shared-memory limit on the current device to at
// least `bytes`, calling the runtime only when a larger size is first needed
// (cudaFuncSetAttribute takes the driver's locks: issued before every
// launch it serialised the host threads of concurrent solves).
template <auto K>
int ensure_smem(size_t bytes) {
  static std::atomic<int> done[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    dev = -1;
  }
  int cur = dev >= 0 ? done[dev].load(std::memory_order_relaxed) : 0;
  if (dev >= 0 && (int)bytes <= cur) return 0;
  WBFMM_CUDA(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  if (dev >= 0)
    while (cur < (int)bytes && !done[dev].compare_exchange_weak(cur, (int)bytes)) {
    }
  return 0;
}
// WBFMM_SMEM(bytes, kernel): ensure_smem, returning its status on failure
// (the kernel last: its template arguments hold commas)
#define WBFMM_SMEM(bytes, ...)                                            \
  do {                                                                    \
    const int rc_ = wbfmm::ensure_smem<__VA_ARGS__>((size_t)(bytes));     \
    if (rc_) return rc_;                                                  \
  } while (0)

// ------------------------------------------------------------------ tree
// *a = va and, when b is non-null, *b = vb (one thread, on stream s)
void launch_set_words(uint32_t* a, uint32_t va, uint32_t* b, uint32_t vb,
                      cudaStream_t s);
// keys[i] = Morton key of point i (src/boxes.c:324-339); vals[i] = i.
// f32: in FP32 arithmetic, as the single-precision build (the *_f API), on
// coordinates, origin and width that are FP32 values
void launch_point_keys(const double* pts, int64_t pstr, int n,
                       const double* x0, double D, uint64_t* keys,
                       uint32_t* vals, cudaStream_t s, bool f32 = false);
// target leaf boxes by floor((x-x0)/wb) (src/boxes.c:585-634); vals[i] = i;
// points outside the closed cube set *bad (host-visible flag) to 1
void launch_target_keys(const double* pts, int64_t pstr, int n,
                        const double* x0, double D, int level,
                        uint64_t* keys, uint32_t* vals, int* bad,
                        cudaStream_t s, bool f32 = false);
// strict-interior domain check of sources (src/boxes.c:148-153)
void launch_domain_check(const double* pts, int64_t pstr, int n,
                         const double* x0, double D, int* bad, cudaStream_t s,
                         bool f32 = false);

struct RadixScratch {
  uint64_t* keys_alt = nullptr;
  uint32_t* vals_alt = nullptr;
  uint32_t* hist = nullptr;
  size_t cap = 0, hist_cap = 0;
};
// stable LSD radix sort of (keys, vals) on key bits [lo, lo + bits);
// result in keys/vals (ping-pong through scratch)
int radix_sort_pairs(uint64_t* keys, uint32_t* vals, int n, int bits,
                     RadixScratch* scr, cudaStream_t s, int lo = 0);
void radix_scratch_free(RadixScratch* scr);

// curl[3 nt] from the gradients g[3][3 nt] of the three potential components
int launch_curl_combine(const double* g, int nt, double* curl, cudaStream_t s);

// box {i, n} of one level from the sorted keys, reproducing
// wbfmm_tree_refine (src/boxes.c:208-277); parent_i is read before the
// parents' .i advance, which launch_refine_parents then applies.
void launch_refine_children(const uint64_t* sorted_keys, int npts,
                            int level, const uint32_t* parent_i,
                            uint32_t* child_i, uint32_t* child_n,
                            cudaStream_t s);
void launch_refine_parents(int level, uint32_t* parent_i,
                           const uint32_t* parent_n, cudaStream_t s);
// per-box start / count of sorted box ids (plain lower bounds; used for
// the target bins)
void launch_box_ranges(const uint64_t* sorted_ids, int n, int level,
                       uint32_t* start, uint32_t* count, cudaStream_t s);

// gathers into sorted order
void launch_gather_points(const double* pts, int64_t pstr, const uint32_t* ip,
                          int n, double* x, double* y, double* z,
                          cudaStream_t s);
void launch_gather_real(const double* src, int64_t sstr, const uint32_t* ip,
                        int n, int ncomp, double* dst, cudaStream_t s);
void launch_gather_real_f32(const double* src, int64_t sstr, const uint32_t* ip,
                            int n, int ncomp, float* dst, cudaStream_t s);

}  // namespace wbfmm
