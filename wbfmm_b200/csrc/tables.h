// Operator tables of the engine (see tables.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "engine.h"

namespace wbfmm {

struct ShiftAngles {
  double th = 0, ph = 0, ch = 0, r = 0;  // angles and distance (unit width)
  int ith = -1;                          // index into ShiftGeometry::thetas
  int idist = 0;                         // |d|^2 for list-4 offsets
};

struct ShiftGeometry {
  ShiftAngles offset[343];          // (dx+3)*49+(dy+3)*7+dz+3, d = src - tgt
  ShiftAngles child_to_parent[8];   // M2M, unit = child width
  ShiftAngles parent_to_child[8];   // L2L, unit = child width
  std::vector<double> thetas;       // distinct rotation angles
};

void build_shift_geometry(ShiftGeometry* g);

// H tables for every theta: rot_count(N) doubles each at stride hstride
int generate_rotation_tables(const std::vector<double>& thetas, int N,
                             double* dH, int64_t hstride, cudaStream_t s);
// coaxial tables for each kr: nc=2 complex (S|R), nc=1 real (R|R)
int generate_coaxial_tables(const std::vector<double>& krs, int L, int nc,
                            double* dout, int64_t ostride, cudaStream_t s);
// any set of coaxial tables in one launch pair: table i at dout + out_off
constexpr int kMaxCoaxJobs = 160;
struct CoaxJob {
  double kr;
  int L, nc;         // order; 2 complex (S|R), 1 real (R|R)
  int64_t out_off;   // doubles
  int64_t scr_off;   // the recursion's scratch (set by generate_coaxial_set)
};
struct CoaxJobs { CoaxJob j[kMaxCoaxJobs]; };   // kernel argument (5 KB)
int generate_coaxial_set(const CoaxJob* jobs, int njobs, double* dout, cudaStream_t s);
// FP32 copies of ntables complex (S|R) tables of order L, entry (l, m, n)
// scaled by 2^(-e (l + n)) (the Helmholtz FP32 M2L's scaled form)
int narrow_coax_scaled(const double* src, float* dst, int L, int64_t stride, int ntables,
                       int e, cudaStream_t s);
// Laplace dense [n][nd][m] tables, n, nd, m <= Lt
int generate_laplace_tables(int Lt, double* SS, double* RR, double* SR,
                            cudaStream_t s);

// the 15 list-4 distances |d|^2 (src/shift.c:709-723)
static const int kListDist2[15] = {4, 5, 6, 8, 9, 10, 11, 12, 13, 14,
                                   17, 18, 19, 22, 27};
inline int list_dist_index(int d2) {
  for (int i = 0; i < 15; i++)
    if (kListDist2[i] == d2) return i;
  return -1;
}

}  // namespace wbfmm
