// Lane-per-pair M2L (m2l_lanes.cu): parameters and launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "kernels.h"

namespace wbfmm {

constexpr int kLanesMaxHelm = 8;    // orders instantiated for Helmholtz
constexpr int kLanesMaxLap = 16;    // and for Laplace

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
  int lap_e;            // Laplace: degree l of lin_raw is scaled by 2^(lap_e l)
  int helm_e;           // Helmholtz tiles (helm_m2l_exp): degree l of lin_raw is
                        // scaled by 2^(helm_e l), coax by 2^(-helm_e (n + l)),
                        // and output degree n by 2^(helm_e n)
  const void* lapsr;    // Laplace: [kNumOps][(P+1)^3] scaled S|R per shift (build_lap_sr_ops)
  const void* hcx;      // Helmholtz tiles: the level's coaxial rows (build_helm_coax_rows)
  const int* act;       // sparse targets: [8][np] parents per child type, or null
  const int* act_n;     // [8] list lengths (device)
  const uint8_t* smask; // [8][padded grid]: source box holds sources, or null (all)
  int boxmajor;         // lin_raw is [8][padded grid][V] (lanes_to_lin), not [8][V][grid]
  void* partial_raw;    // [nsplit][8][V][np] complex when nsplit > 1
  // sparse storage: lin_raw is [8][V][lin_stride] (box-major:
  // [8][lin_stride][V]) over the source slots (lanes_to_lin_groups), pmap
  // maps the padded parent grid to a slot (lin_stride - 1, a zero column,
  // where no group is stored), gmap the target groups to their slots; null
  // for dense storage
  const uint32_t* pmap;
  const uint32_t* gmap;
  int64_t lin_stride;
};

// The 189 list-4 offsets seen by a target of child type tau, packed as
// op | sigma << 9 | (dx+1) << 12 | (dy+1) << 14 | (dz+1) << 16 with op the
// shift code (dx+3)*49+(dy+3)*7+dz+3 of src/indexing.c:330-377, sigma the
// source's child type and (dx, dy, dz) the source parent's offset from the
// target's parent (each in [-1, 1]).
inline void build_offset_table(int* tab) {
  for (int tau = 0; tau < 8; tau++) {
    int ta[3] = {tau & 1, (tau >> 1) & 1, (tau >> 2) & 1};
    int j = 0;
    for (int dx = -2 - ta[0]; dx <= 3 - ta[0]; dx++)
      for (int dy = -2 - ta[1]; dy <= 3 - ta[1]; dy++)
        for (int dz = -2 - ta[2]; dz <= 3 - ta[2]; dz++) {
          if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1)
            continue;
          int d[3] = {dx, dy, dz}, sg = 0, Dl[3];
          for (int a = 0; a < 3; a++) {
            int s = ta[a] + d[a];
            sg |= (s & 1) << a;
            Dl[a] = s >> 1;   // floor division (s in [-2, 4])
          }
          int op = (dx + 3) * 49 + (dy + 3) * 7 + dz + 3;
          tab[tau * 189 + j] = op | (sg << 9) | ((Dl[0] + 1) << 12) |
                               ((Dl[1] + 1) << 14) | ((Dl[2] + 1) << 16);
          j++;
        }
  }
}

template <typename T, bool HELM>
bool lanes_supported(int Ns, int Nr);
// sum of the split partial results (split order) into the level array
template <typename T, bool HELM>
int launch_lanes_reduce(const LanesParams<T>& p, cudaStream_t s);

// offset-major target tiles (m2l_tiles.cu), any order up to a shared-memory
// limit
template <typename T, bool HELM>
bool tiles_supported(int Ns, int Nr);
template <typename T, bool HELM>
int launch_m2l_tiles(const LanesParams<T>& p, const OpTables<T>& t,
                     cudaStream_t s);
// targets per CTA of the tile kernel at order N (0: unsupported); *dense
// (if given): whether it reads the level's Helmholtz coaxial rows; sparse:
// the launch on sparse level storage (LanesParams::pmap set)
template <typename T, bool HELM>
int tiles_per_cta(int N, bool* dense = nullptr, bool sparse = false);
// the tile kernel's Helmholtz coaxial rows of a level (15 distances, rows
// of (S|R) pairs with signs folded in) from its (S|R) table, into
// helm_coax_rows_count(P) values
template <typename T>
int build_helm_coax_rows(const T* raw, int64_t raw_stride, int P, T* out, cudaStream_t s);
size_t helm_coax_rows_count(int P);
// smask[sg][padded parent] = the level's box of child type sg under that
// parent holds sources (0 on the padding), from the level's box counts
int build_source_mask(const uint32_t* src_n, int level, uint8_t* smask, cudaStream_t s);
size_t source_mask_bytes(int level);
// degree l scaled by 2^(scale_e l) (the Laplace or Helmholtz M2L exponent)
template <typename T, bool HELM>
int lanes_to_lin(const T* arr, int level, int N, int scale_e, void* lin, cudaStream_t s,
                 bool boxmajor = false);
size_t lanes_lin_bytes(int level, int N, bool helm, size_t tsize);
// sparse storage: a level's compact array (groups slots, Layout L per
// group) -> lin[tau][c][slot] (boxmajor: lin[tau][slot][c]) over groups + 1
// slots (the last zero), degree n scaled by 2^(scale_e n); bytes:
// lanes_lin_groups_bytes
template <typename T, bool HELM>
int lanes_to_lin_groups(const T* arr, int64_t groups, int N, int scale_e, void* lin,
                        cudaStream_t s, bool boxmajor = false);
size_t lanes_lin_groups_bytes(int64_t groups, int N, bool helm, size_t tsize);
// pmap[pp] = slot of the parent at padded-grid position pp (gmap of the
// level), or `groups` (the zero column) on the padding and for parents
// whose group is not stored; source_mask_bytes(level) / 8 entries
int build_parent_slot_map(const uint32_t* gmap, int level, uint32_t groups, uint32_t* pmap,
                          cudaStream_t s);

// Active-target lists of a level for the lane and tile M2L: for each child
// type tau, the parents (linear index, x fastest) whose child of type tau
// has tmask set, ascending, in act[tau * np ...], with the lengths in
// act_n[8].  act holds 8^level ints; scratch active_list_scratch(level) ints.
size_t active_list_scratch(int level);

// Laplace M2L operators of one level for the lane kernel, per shift code:
// out[op][(n (P+1) + nd) (P+1) + m] = S|R(n, nd, m) / (t^(n+1) (2^e t)^nd),
// t = width |d_op| (the scaled form of lap_scale_exp)
template <typename T>
int build_lap_sr_ops(const OpTables<T>& t, int P, T width, int lap_e, T* out,
                     cudaStream_t s);
int build_active_lists(const uint8_t* tmask, int level, int* act, int* act_n,
                       int* scratch, cudaStream_t s);
template <typename T, bool HELM>
int launch_m2l_lanes(const LanesParams<T>& p, const OpTables<T>& t,
                     cudaStream_t s);

}  // namespace wbfmm
