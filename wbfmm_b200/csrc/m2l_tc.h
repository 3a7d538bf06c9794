// Laplace M2L on the tensor cores (m2l_tc.cu): parameters and launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace wbfmm {

// per-degree scale factors of a level of width w: sources enter as
// w^-n M_n, results leave as w^-(n+1) (That M)_n
struct LapTcScales {
  float in[32];
  float out[32];
};

struct LapTcParams {
  int level, P;              // target level, order (singular = regular)
  int KS, MT, KP;            // k-steps of 8, M tiles of 128, padded K
  int nsplit;                // CTAs sharing the 189 offsets of a target tile
  const float* ops;          // dense operators, TF32 hi / lo tiles per shift slot
  const int* slot;           // shift code -> operator slot (-1: near field)
  const int* offsets;        // [8][189] packed list-4 offsets (build_offset_table)
  const float* lin;          // [8][padded grid][KS][16] scaled sources, TF32 hi / lo per 8-K chunk
  float* cout;               // regular expansions of the level (Layout L), added to
  float* partial;            // [nsplit][8][C][np] when nsplit > 1
  const int* act;            // sparse targets: [8][np] parents per child type, or null
  const int* act_n;          // [8] list lengths (device)
  const uint8_t* smask;      // [8][padded grid]: source box holds sources, or null
  const uint8_t* tmask;      // targets to write in the split reduction, or null
  int* err;                  // set to 1 when a wait ran out
  LapTcScales sc;
};

// orders the tensor-core M2L handles (equal orders, (p+1)^2 <= 256)
bool tc_lap_supported(int Ns, int Nr);
// bytes of the scaled source copy of a level
size_t tc_lin_bytes(int level, int P);
// the order's dense operators (built on first use per device from FP64
// tables at unit width, and kept for the process); fills ops, slot,
// offsets, KS, MT
int tc_lap_ops(int P, cudaStream_t s, LapTcParams* p);
// the M2L of a level: scaled source copy into `lin`, the product, and the
// split reduction when nsplit > 1 (partial must then hold
// nsplit * 8 * (P+1)^2 * 8^(level-1) floats)
int launch_m2l_tc(LapTcParams p, const float* mps, void* lin, cudaStream_t s);

}  // namespace wbfmm
