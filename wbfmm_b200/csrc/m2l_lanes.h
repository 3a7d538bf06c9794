// Lane-per-pair M2L (m2l_lanes.cu): parameters and launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace wbfmm {

constexpr int kLanesMaxHelm = 8;    // orders instantiated for Helmholtz
constexpr int kLanesMaxLap = 12;    // and for Laplace

template <typename T>
struct LanesParams {
  int level;            // target level
  int N;                // expansion order (singular = regular)
  int nsplit;           // CTAs sharing the 189 offsets of a target tile
  const void* lin_raw;  // transposed singular expansions (complex, padded grid)
  T* cout;              // regular expansions of the level (Layout L), added to
  const T* coax;        // Helmholtz (S|R) tables of the level
  int64_t coax_stride;
  T width;              // box width of the level
  const uint8_t* tmask; // targets to compute, or null for all
  void* partial_raw;    // [nsplit][8][V][np] complex when nsplit > 1
};

template <typename T, bool HELM>
bool lanes_supported(int Ns, int Nr);
template <typename T, bool HELM>
int lanes_to_lin(const T* arr, int level, int N, void* lin, cudaStream_t s);
size_t lanes_lin_bytes(int level, int N, bool helm, size_t tsize);
template <typename T, bool HELM>
int launch_m2l_lanes(const LanesParams<T>& p, const OpTables<T>& t,
                     cudaStream_t s);

}  // namespace wbfmm
