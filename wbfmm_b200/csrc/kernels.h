// Launch parameters of the FMM pass kernels (kernels.cu).
#pragma once

#include <cmath>

#include <cuda_runtime.h>
#include <stdint.h>

namespace wbfmm {

// number of shift operators: 343 list-4 offsets, 8 child->parent (M2M),
// 8 parent->child (L2L)
constexpr int kOpM2M = 343;
constexpr int kOpL2L = 351;
constexpr int kNumOps = 359;

// Device tables shared by a solve (all T = coefficient precision).
template <typename T>
struct OpTables {
  const T* H = nullptr;          // rotation tables, one per theta
  int64_t hstride = 0;
  const int* op_ith = nullptr;   // [kNumOps] theta index
  const int* op_dist = nullptr;  // [kNumOps] list-4 distance index (0..14)
  const T* op_r = nullptr;       // [kNumOps] distance in box widths
  const T* ph = nullptr;         // [kNumOps][lmax+1] (cos, sin)(m ph)
  const T* ch = nullptr;         // [kNumOps][lmax+1] (cos, sin)(m ch)
  int lmax = 0;
  // Laplace dense coaxial tables [n][nd][m], dimension lt+1
  const T* lapSS = nullptr;
  const T* lapRR = nullptr;
  const T* lapSR = nullptr;
  int lt = 0;
};

template <typename T>
struct P2MParams {
  int64_t nbox;       // boxes at the leaf level
  int level, N;
  double x0, y0, z0, wb;
  T k;
  const uint32_t* box_i;
  const uint32_t* box_n;
  const double* x; const double* y; const double* z;  // sorted sources
  const T* q;         // Laplace [n]; Helmholtz [2n]; may be null
  const T* dip;       // dipole strengths (same layout), may be null
  const T* nx; const T* ny; const T* nz;   // sorted normals (dipoles)
  T* mps;             // leaf level, Layout L
  int accumulate;     // 1: add to the existing coefficients
  // sparse storage: slot -> group (parent box) of the leaf level; boxes are
  // then the compact indices 8 slot + child (nbox = 8 x slots), or null
  const uint32_t* glist = nullptr;
};

template <typename T>
struct EvalParams {
  int ntgt;
  int level, N;
  double x0, y0, z0, wb;
  T k;
  const double* tx; const double* ty; const double* tz;  // leaf-box order
  const uint32_t* tperm;                   // sorted target -> original index
  const uint32_t* tbox;                    // sorted target -> leaf box
  const uint32_t* tstart; const uint32_t* tcount;  // per leaf box
  const uint32_t* box_i; const uint32_t* box_n;    // source leaf ranges
  const double* x; const double* y; const double* z;  // sorted sources
  const T* q; const T* dip;
  const T* nx; const T* ny; const T* nz;
  const T* mpr;                             // leaf regular expansions
  T* pot;    // [ntgt] or [2 ntgt] (original order), may be null
  T* grad;   // [3 ntgt] or [6 ntgt], may be null
  int64_t nbox;
  const uint32_t* gmap = nullptr;   // sparse storage: leaf group -> slot, or null
};

template <typename T>
struct XlateParams {
  int level;          // level of the boxes that receive the result
  int64_t nbox;       // M2L: boxes at `level`; M2M/L2L: parents
  int Nin, Nout;      // orders of input and output expansions
  const T* cin;       // input level array (Layout L)
  T* cout;            // output level array (Layout L)
  const uint32_t* src_n;   // M2L: source box counts (skip empty), or null
  const T* coax;           // Helmholtz coaxial table(s) for this level
  int64_t coax_stride;     // per distance (complex S|R)
  T width;                 // box width of the translation's distance unit
  T k;
  int nsplit;              // M2L: CTAs per target box
  T* partial;              // M2L split: [nsplit][nbox][2*ncout]
  const uint8_t* tmask;    // M2L: only targets with tmask[b] != 0, or null
  int lap_e;               // Laplace M2L scale exponent (lap_scale_exp)
  // sparse storage (M2M, L2L): one CTA per slot of the child level
  // (nbox = its slots), glist its slot -> group (the parent box), gmap the
  // parent level's group -> slot; both null for dense storage
  const uint32_t* glist;
  const uint32_t* gmap;
};

// Laplace M2L scale exponent of a level of box width w: e = -ilogb(w), so
// 2^e w is in [1, 2).  M2L kernels scale degree l of the singular
// expansions by 2^(e l) and apply S|R(n,l,m) / (t^(n+1) (2^e t)^l): every
// factor stays near the size of the expansions themselves, where the plain
// S|R / t^(n+l+1) (t = |d| w, n + l up to 2p) leaves the FP32 range at
// deep levels (t = 2/256 at level 8 gives 128^21 ~ 1.8e44 for p = 10).
inline int lap_scale_exp(double w) { return -std::ilogb(w); }

// Helmholtz FP32 M2L scale exponent of a level (0: none needed).  With
// x = 2 k w the nearest list-4 distance, the level's (S|R) coefficients of
// degrees n, l <= P grow like (2(n+l)-1)!! / x^(n+l+1) (G&D (4.79) seeded
// by h_l(x)), beyond the FP32 range at small k w and high order.  The M2L
// then works on sources whose degree l is scaled by 2^(e l), on the table
// scaled by 2^(-e (n + l)), and scales degree n of its results back by
// 2^(e n): with 2^-e about the (2P)-th root of x^(2P+1) / (4P-1)!!, the
// largest scaled coefficient (n = l = P) is of order one and the smallest
// ((n, l) = (0, 0), h_0(x) ~ 1/x) unchanged; the scaled sources stay below
// ((sqrt 3 / 4) x 2^e)^l / (2l+1)!! per unit strength.  Exact (powers of
// two); the stored expansions are not scaled.
inline int helm_m2l_exp(double k, double w, int P) {
  const double x = 2.0 * k * w;
  double lf = 0.0;                       // log10 (4P-1)!!
  for (int i = 4 * P - 1; i > 1; i -= 2) lf += std::log10((double)i);
  if (lf - (2 * P + 1) * std::log10(x) <= 30.0) return 0;
  const double log2s = ((2 * P + 1) * std::log10(x) - lf) / (2.0 * P) / std::log10(2.0);
  return -(int)std::floor(log2s + 0.5);
}

template <typename T, bool HELM>
int launch_p2m(const P2MParams<T>& p, cudaStream_t s);
template <typename T, bool HELM>
int launch_m2m(const XlateParams<T>& p, const OpTables<T>& t, cudaStream_t s);
template <typename T, bool HELM>
int launch_m2l(const XlateParams<T>& p, const OpTables<T>& t, cudaStream_t s);
template <typename T, bool HELM>
int launch_l2l(const XlateParams<T>& p, const OpTables<T>& t, cudaStream_t s);
template <typename T, bool HELM>
int launch_l2p(const EvalParams<T>& p, cudaStream_t s);
template <typename T, bool HELM>
int launch_p2p(const EvalParams<T>& p, cudaStream_t s);
// Laplace second derivatives (hessian.cu): the coefficients of d/dx, d/dy,
// d/dz (degree N - 1) of each box's regular expansion L (degree N >= 1);
// hess[9 t + 3 a + b] = g[a][3 t + b] (g null: zeros); the near-field
// second derivatives of the monopoles of the 27 neighbour boxes added into
// hess; out[12 t] = curl and its gradient from the components' gradients
// g[3][3 nt] and Hessians h[3][9 nt]
template <typename T>
int launch_laplace_deriv(const T* L, int N, int64_t nbox, T* Dx, T* Dy, T* Dz,
                         cudaStream_t s);
template <typename T>
int launch_hess_gather(const T* g, int nt, double* hess, cudaStream_t s);
template <typename T>
int launch_p2p_hessian(const EvalParams<T>& p, double* hess, cudaStream_t s);
int launch_curl_gradient_combine(const double* g, const double* h, int nt, double* out,
                                 cudaStream_t s);
// precomputed target bases (target_bases.cu): pair offsets of the targets'
// near fields; the CSR sources, monopole and (wd non-null) dipole weights
// and the coefficient-major regular-expansion bases; the potential from them
template <typename T>
int tl_offsets(const EvalParams<T>& p, int64_t* off, int64_t* npairs, cudaStream_t s);
template <typename T, bool HELM>
int tl_fill(const EvalParams<T>& p, const int64_t* off, uint32_t* src, T* wq, T* wd, T* basis,
            cudaStream_t s);
template <typename T, bool HELM>
int tl_apply(const EvalParams<T>& p, const T* basis, const int64_t* off, const uint32_t* src,
             const T* wq, const T* wd, cudaStream_t s);
// FP32 copies of FP64 arrays, and FP32 results added into FP64 ones
int launch_narrow(const double* src, float* dst, int64_t n, cudaStream_t s);
int launch_add_widened(double* dst, const float* src, int64_t n, cudaStream_t s);
// self-test of the FP32 near-field sine/cosine (kernels.cu)
int sincos_near_errors(double xmax, int n, double* host_err);
// sparse level storage (sparse.cu): the group map of a level from the n
// boxes of the level above (stored: box_n != 0 or tmask set; tmask may be
// null): gmap[g] = slot or kNoGroup, *count = stored groups (device);
// scratch of sparse_scan_scratch(n) bytes; then the slot -> group list, and
// a compact array expanded to the dense Layout L array (zeros elsewhere)
size_t sparse_scan_scratch(int64_t n);
int sparse_group_map(const uint32_t* box_n, const uint8_t* tmask, int64_t n, uint32_t* flag,
                     uint32_t* gmap, uint32_t* count, void* scratch, size_t scratch_bytes,
                     cudaStream_t s);
int sparse_group_list(const uint32_t* gmap, int64_t n, uint32_t* glist, cudaStream_t s);
template <typename T>
int sparse_expand(const T* compact, const uint32_t* glist, int64_t groups, int64_t glen,
                  T* dense, int64_t dense_len, cudaStream_t s);

}  // namespace wbfmm
