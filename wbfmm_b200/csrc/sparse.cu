// Sparse level storage: the coefficient arrays of a level hold only the
// groups of eight sibling boxes whose parent holds sources or targets.
//
// The reference stores every one of the 8^l boxes of a level
// (src/boxes.c:518-583, src/tree.c:57-72); for clustered points almost all
// of them are empty.  Here a level l keeps, per group g (a box of level
// l - 1), a slot gmap[g] (kNoGroup when the group is not stored), the
// stored groups at consecutive slots in Morton order (glist[slot] = g), and
// the coefficients of slot s at compact box indices 8 s + child, each
// group in the reference's Layout L.  The maps come from the per-level box
// counts of the sources and the target masks by a flag / exclusive scan /
// scatter per level.
#include <cub/cub.cuh>

#include "../../include/wbfmm_b200.h"
#include "engine.h"
#include "fmm_math.cuh"
#include "kernels.h"

namespace wbfmm {

namespace {

// flag[g] = group g of the next level is stored: box g holds sources or
// targets
__global__ void k_group_flags(const uint32_t* __restrict__ box_n,
                              const uint8_t* __restrict__ tmask, int64_t n,
                              uint32_t* __restrict__ flag) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  flag[g] = (box_n[g] != 0 || (tmask && tmask[g] != 0)) ? 1u : 0u;
}

// gmap holds the exclusive scan of flag: the count of stored groups (read
// by the last group's thread before it writes), then kNoGroup for the
// groups not stored
__global__ void k_group_finish(const uint32_t* __restrict__ flag, int64_t n,
                               uint32_t* __restrict__ gmap, uint32_t* __restrict__ count) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const uint32_t f = flag[g];
  if (g == n - 1) *count = gmap[g] + f;
  if (!f) gmap[g] = kNoGroup;
}

__global__ void k_group_list(const uint32_t* __restrict__ gmap, int64_t n,
                             uint32_t* __restrict__ glist) {
  const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= n) return;
  const uint32_t s = gmap[g];
  if (s != kNoGroup) glist[s] = (uint32_t)g;
}

// dense[glist[s] * glen + i] = compact[s * glen + i] (a group's Layout L
// block is contiguous in both)
template <typename T>
__global__ void k_expand_groups(const T* __restrict__ compact, const uint32_t* __restrict__ glist,
                                int64_t groups, int64_t glen, T* __restrict__ dense) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= groups * glen) return;
  const int64_t s = e / glen, i = e - s * glen;
  dense[(int64_t)glist[s] * glen + i] = compact[e];
}

}  // namespace

size_t sparse_scan_scratch(int64_t n) {
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                (int)n);
  return bytes + 16;
}

int sparse_group_map(const uint32_t* box_n, const uint8_t* tmask, int64_t n, uint32_t* flag,
                     uint32_t* gmap, uint32_t* count, void* scratch, size_t scratch_bytes,
                     cudaStream_t s) {
  if (n <= 0 || n > 0x7fffffffLL)
    return set_error(WBFMM_B200_E_ARG, "sparse storage: group count out of range");
  const unsigned blocks = (unsigned)((n + 255) / 256);
  k_group_flags<<<blocks, 256, 0, s>>>(box_n, tmask, n, flag);
  WBFMM_CUDA(cudaGetLastError());
  size_t bytes = scratch_bytes;
  WBFMM_CUDA(cub::DeviceScan::ExclusiveSum(scratch, bytes, (const uint32_t*)flag, gmap, (int)n, s));
  k_group_finish<<<blocks, 256, 0, s>>>(flag, n, gmap, count);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

int sparse_group_list(const uint32_t* gmap, int64_t n, uint32_t* glist, cudaStream_t s) {
  if (n <= 0) return 0;
  k_group_list<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(gmap, n, glist);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

template <typename T>
int sparse_expand(const T* compact, const uint32_t* glist, int64_t groups, int64_t glen,
                  T* dense, int64_t dense_len, cudaStream_t s) {
  WBFMM_CUDA(cudaMemsetAsync(dense, 0, sizeof(T) * dense_len, s));
  const int64_t tot = groups * glen;
  if (tot <= 0) return 0;
  k_expand_groups<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(compact, glist, groups, glen,
                                                                    dense);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}
template int sparse_expand<float>(const float*, const uint32_t*, int64_t, int64_t, float*,
                                  int64_t, cudaStream_t);
template int sparse_expand<double>(const double*, const uint32_t*, int64_t, int64_t, double*,
                                   int64_t, cudaStream_t);

}  // namespace wbfmm
