// Allocation-free variant of the tree-build sort: Morton keys plus the
// stable Morton permutation of device-resident points, with the radix
// sort's scratch held in a file-scope device array instead of memory from
// cudaMalloc.
//
// Some callers of this library cannot allocate device memory at the point
// where they need the sort: latency-critical serving loops that must not
// take cudaMalloc's implicit device-wide synchronisation, and processes
// whose device memory is owned by another allocator (a framework's caching
// allocator that has reserved the GPU).  They pass their own input and
// output buffers; everything else this entry point needs lives in
// g_noalloc_scratch below, a fixed-size array that every GPU which loads
// the library holds until the process exits.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/wbfmm_b200.h"
#include "engine.h"

namespace wbfmm {

// Scratch of the LSD radix sort for up to kNoAllocMaxPoints points: the
// ping-pong key and value buffers and the per-tile digit histograms, plus
// one int for the domain check.  The tile size (2048 elements) matches
// radix_sort_pairs in tree.cu.
constexpr int kNoAllocMaxPoints = WBFMM_B200_NOALLOC_MAX_POINTS;
constexpr int kNoAllocTiles = (kNoAllocMaxPoints + 2047) / 2048;
constexpr size_t kNaKeysOff = 0;
constexpr size_t kNaValsOff = kNaKeysOff + sizeof(uint64_t) * (size_t)kNoAllocMaxPoints;
constexpr size_t kNaHistOff = kNaValsOff + sizeof(uint32_t) * (size_t)kNoAllocMaxPoints;
constexpr size_t kNaFlagOff = kNaHistOff + sizeof(uint32_t) * 256 * (size_t)kNoAllocTiles;
constexpr size_t kNaBytes = kNaFlagOff + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

// device address of g_noalloc_scratch, looked up once per device with that
// device current (host code may not use the symbol itself as an address).
// The address stays valid while the device's primary context lives, so a
// process must not reset the device (cudaDeviceReset) and then call again.
static unsigned char* g_na_addr[64] = {nullptr};
static std::mutex g_na_mutex;

static int noalloc_scratch(unsigned char** out) {
  int dev = 0;
  WBFMM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64)
    return set_error(WBFMM_B200_E_ARG, "device index out of range for the no-allocation scratch table");
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return set_cuda_error(e, __FILE__, __LINE__);
    g_na_addr[dev] = (unsigned char*)p;
  }
  *out = g_na_addr[dev];
  return 0;
}

}  // namespace wbfmm

using namespace wbfmm;

extern "C" int wbfmm_b200_morton_sort_noalloc(int n, const double* pts,
                                              int pstr, const double* x0,
                                              double D, uint64_t* keys,
                                              uint32_t* ip, void* stream) {
  if (n <= 0 || !pts || !x0 || !keys || !ip || pstr < 3 || !(D > 0.0))
    return set_error(WBFMM_B200_E_ARG, "morton_sort_noalloc: bad arguments");
  if (n > kNoAllocMaxPoints)
    return set_error(WBFMM_B200_E_ARG,
                     "morton_sort_noalloc: more points than the fixed scratch holds "
                     "(WBFMM_B200_NOALLOC_MAX_POINTS); use wbfmm_b200_set_sources");
  unsigned char* base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  int* flag = (int*)(base + kNaFlagOff);
  // strict-interior domain check (src/boxes.c:148-153): the flag keeps the
  // last call's value, so a kernel on the caller's stream resets it first
  launch_set_words((uint32_t*)flag, 0x7fffffffu, nullptr, 0, s);
  launch_domain_check(pts, pstr, n, x0, D, flag, s);
  launch_point_keys(pts, pstr, n, x0, D, keys, ip, s);
  RadixScratch scr;
  scr.keys_alt = (uint64_t*)(base + kNaKeysOff);
  scr.vals_alt = (uint32_t*)(base + kNaValsOff);
  scr.hist = (uint32_t*)(base + kNaHistOff);
  scr.cap = (size_t)kNoAllocMaxPoints;
  scr.hist_cap = (size_t)256 * kNoAllocTiles;
  // with cap and hist_cap covering n, radix_sort_pairs allocates nothing;
  // the histograms are fully rewritten by every pass
  rc = radix_sort_pairs(keys, ip, n, 60, &scr, s);
  if (rc) return rc;
  int bad = 0;
  WBFMM_CUDA(cudaMemcpyAsync(&bad, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
  WBFMM_CUDA(cudaStreamSynchronize(s));
  if (bad != 0x7fffffff)
    return set_error(WBFMM_B200_E_DOMAIN,
                     "morton_sort_noalloc: a point does not lie strictly inside the cube");
  return 0;
}
