// M2L, lane-per-pair form for expansion orders known at compile time.
//
// The list-4 interactions of a level are regrouped by target child type tau
// (the target's position inside its parent): all targets of one type see
// the same 189 offsets d = source - target (src/indexing.c:330-377), each
// with one rotate / coaxial / rotate-back operator.  A CTA takes 128 target
// parents of one type; its 4 warps x 32 lanes each own one target.  The CTA
// walks the 189 offsets in a fixed order; for each it stages the offset's
// operator in shared memory (rotation block H_n^{nu,m}(theta) for n <= P,
// the phases e^{i m ph}, e^{i m ch}, and the coaxial coefficients), and every
// lane applies it to its own source vector (shared-memory broadcast of the
// operator, per-lane vectors).  Degree and order loops are unrolled for the
// compile-time order P, so each lane's inner work is straight-line FMA code.
//
// Sources are read from a transposed copy of the level's singular
// expansions: per child type, per coefficient, a parent grid padded by one
// empty parent on every side (so list-4 sources outside the domain read
// zeros, exactly the reference's clipping), consecutive lanes reading
// consecutive parents.
#include <cuda_runtime.h>

#include "engine.h"
#include "kernels.h"
#include "m2l_lanes.h"
#include "translate.cuh"

namespace wbfmm {

template <typename T> struct V2t;
template <> struct V2t<float> { typedef float2 t; };
template <> struct V2t<double> { typedef double2 t; };

// per target type: 189 packed offsets (op | sigma << 9 | (dx+1) << 12 |
// (dy+1) << 14 | (dz+1) << 16), dx.. = parent offset of the source
__constant__ int c_offsets[8][189];
static bool g_offsets_ready[64] = {false};

static int ensure_offsets() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && g_offsets_ready[dev]) return 0;
  int tab[8 * 189];
  build_offset_table(tab);
  WBFMM_CUDA(cudaMemcpyToSymbol(c_offsets, tab, sizeof(tab)));
  if (dev < 64) g_offsets_ready[dev] = true;
  return 0;
}

// ----------------------------------------------------------- transpose
// Layout L level array -> lin[tau][c][pp] (complex), pp on the padded
// parent grid (nx+2)^3, degree n scaled by 2^(scale_e n); the halo must be
// zero beforehand
template <typename T, bool HELM>
__global__ void k_to_lin(const T* __restrict__ arr, int level, int N, int scale_e, bool boxmajor,
                         typename V2t<T>::t* __restrict__ lin) {
  typedef typename V2t<T>::t T2;
  const int V = HELM ? (N + 1) * (N + 1) : (N + 1) * (N + 2) / 2;
  const int nc = (N + 1) * (N + 1);
  const int nx = 1 << (level - 1), npx = nx + 2;
  const int64_t npp = (int64_t)npx * npx * npx;
  const int64_t np = (int64_t)nx * nx * nx;
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np * V * 8) return;
  const int tau = (int)(e & 7);
  const int c = (int)((e >> 3) % V);
  const int64_t P = (e >> 3) / V;        // parent Morton index
  uint32_t px, py, pz;
  demorton((uint64_t)P, &px, &py, &pz);
  const int64_t pp = (px + 1) + npx * ((int64_t)(py + 1) + npx * (int64_t)(pz + 1));
  const int64_t b = (P << 3) | tau;
  T2 v;
  if (HELM) {
    int64_t o = layout_off(b, c, nc);
    v.x = arr[2 * o]; v.y = arr[2 * o + 1];
    if (scale_e) {
      const int n = full_degree(c);
      v.x = scale2(v.x, scale_e * n);
      v.y = scale2(v.y, scale_e * n);
    }
  } else {
    int n = half_degree(c), m = c - n * (n + 1) / 2;
    if (m == 0) {
      v.x = arr[layout_off(b, n * n, nc)]; v.y = T(0);
    } else {
      int id = lidx(n, m);
      v.x = arr[layout_off(b, id, nc)]; v.y = arr[layout_off(b, id + 1, nc)];
    }
    v.x = scale2(v.x, scale_e * n);
    v.y = scale2(v.y, scale_e * n);
  }
  if (boxmajor) lin[((int64_t)tau * npp + pp) * V + c] = v;
  else lin[((int64_t)tau * V + c) * npp + pp] = v;
}

// sparse storage: compact level array -> lin[tau][c][slot] (box-major:
// lin[tau][slot][c]), slot in [0, groups] (slot `groups` zero), degree n
// scaled by 2^(scale_e n)
template <typename T, bool HELM>
__global__ void k_to_lin_groups(const T* __restrict__ arr, int64_t groups, int N, int scale_e,
                                bool boxmajor, typename V2t<T>::t* __restrict__ lin) {
  typedef typename V2t<T>::t T2;
  const int V = HELM ? (N + 1) * (N + 1) : (N + 1) * (N + 2) / 2;
  const int nc = (N + 1) * (N + 1);
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (groups + 1) * V * 8) return;
  const int tau = (int)(e & 7);
  const int c = (int)((e >> 3) % V);
  const int64_t slot = (e >> 3) / V;
  T2 v;
  v.x = T(0); v.y = T(0);
  if (slot < groups) {
    const int64_t b = (slot << 3) | tau;
    int n;
    if (HELM) {
      const int64_t o = layout_off(b, c, nc);
      v.x = arr[2 * o]; v.y = arr[2 * o + 1];
      n = full_degree(c);
    } else {
      n = half_degree(c);
      const int m = c - n * (n + 1) / 2;
      if (m == 0) {
        v.x = arr[layout_off(b, n * n, nc)];
      } else {
        const int id = lidx(n, m);
        v.x = arr[layout_off(b, id, nc)]; v.y = arr[layout_off(b, id + 1, nc)];
      }
    }
    if (scale_e) {
      v.x = scale2(v.x, scale_e * n);
      v.y = scale2(v.y, scale_e * n);
    }
  }
  if (boxmajor) lin[((int64_t)tau * (groups + 1) + slot) * V + c] = v;
  else lin[((int64_t)tau * V + c) * (groups + 1) + slot] = v;
}

// pmap[pp]: slot of the padded-grid parent pp, `groups` on the padding and
// where the parent's group is not stored
__global__ void k_parent_slot_map(const uint32_t* __restrict__ gmap, int nx, int64_t npp,
                                  uint32_t groups, uint32_t* __restrict__ pmap) {
  const int64_t pp = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (pp >= npp) return;
  const int npx = nx + 2;
  const int px = (int)(pp % npx) - 1, py = (int)((pp / npx) % npx) - 1,
            pz = (int)(pp / ((int64_t)npx * npx)) - 1;
  uint32_t v = groups;
  if (px >= 0 && px < nx && py >= 0 && py < nx && pz >= 0 && pz < nx) {
    const uint32_t g = gmap[morton(px, py, pz)];
    if (g != kNoGroup) v = g;
  }
  pmap[pp] = v;
}

// --------------------------------------------------------------- kernel
// compiler-only memory fence: keeps the unrolled per-degree blocks from
// being hoisted into one another (bounds register live ranges)
__device__ __forceinline__ void cfence() { asm volatile("" ::: "memory"); }

template <typename T2, typename T>
__device__ __forceinline__ T2 cm(T2 a, T er, T ei) {
  T2 r;
  r.x = a.x * er - a.y * ei;
  r.y = a.x * ei + a.y * er;
  return r;
}


// asynchronous global -> shared copies of one element (Ampere-style
// cp.async, completion by group)
__device__ __forceinline__ void cp_async_t(float* dst, const float* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_t(double* dst, const double* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::);
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

template <int P>
struct LaneDims {
  static constexpr int VF = (P + 1) * (P + 1);                 // full vector
  static constexpr int VH = (P + 1) * (P + 2) / 2;             // half vector
  static constexpr int NH = (P + 1) * (P + 2) * (4 * P + 3) / 6;  // H, n <= P
  static constexpr int NC = (P + 1) * (P + 2) * (P + 3) / 6;   // coaxial
  static constexpr int NL = (P + 1) * (P + 1) * (P + 1);       // Laplace S|R
};

// whether a lane keeps its working vector in registers (about 100 of them at
// most); otherwise it is a shared-memory column like the accumulator
// (WBFMM_LANES_NO_REGISTER_VECTOR builds every order the second way, to
// compare the two)
template <typename T, bool HELM, int P>
struct LaneReg {
  static constexpr int V = HELM ? LaneDims<P>::VF : LaneDims<P>::VH;
#ifdef WBFMM_LANES_NO_REGISTER_VECTOR
  static constexpr bool value = false;
#else
  static constexpr bool value = 2 * V * (int)(sizeof(T) / 4) <= 100;
#endif
};

// CTAs per SM that the register-resident variant is compiled for (it caps
// the registers per thread at 65536 / (128 * this)).  Measured on B200, FP32,
// level-5/6 M2L (ms for caps 3 / 4 / none): Helmholtz p = 6 11.96 / 13.85 /
// 10.51 (no cap: ILP of the unrolled body beats occupancy), p = 5 0.914 /
// 0.986 / 0.943; Laplace p = 6 0.863 / 0.756 / 1.048, p = 8 1.694 / 1.837 /
// 1.781.  WBFMM_LANES_REG_CTAS overrides the table.
template <typename T, bool HELM, int P>
struct LaneRegCtas {
#ifdef WBFMM_LANES_REG_CTAS
  static constexpr int value = WBFMM_LANES_REG_CTAS;
#else
  static constexpr int value = (sizeof(T) == 4 && HELM && P == 6) ? 1
                             : (sizeof(T) == 4 && !HELM && P == 6) ? 4 : 3;
#endif
};

// a lane's working vector: registers, or a shared-memory column of stride 32
template <typename T2, int V, bool REG>
struct WVec {
  T2* p;
  __device__ explicit WVec(T2* q) : p(q) {}
  __device__ __forceinline__ T2& operator[](int i) { return p[i * 32]; }
};
template <typename T2, int V>
struct WVec<T2, V, true> {
  T2 r[V];
  __device__ explicit WVec(T2*) {}
  __device__ __forceinline__ T2& operator[](int i) { return r[i]; }
};

// shared memory layout, in units of T: [H: NH][eph: 2(P+1)][ech: 2(P+1)]
// [coax: Helmholtz 2 NC | Laplace NL] then per warp the accumulator column
// and, unless the working vector is in registers, its column; as many
// warps (<= 4) as fit in 200 KB
template <typename T, bool HELM, int P>
struct LaneSmem {
  static constexpr int ncols = LaneReg<T, HELM, P>::value ? 1 : 2;
  static constexpr size_t col_bytes =
      ncols * sizeof(T) * 2 * (size_t)(HELM ? LaneDims<P>::VF : LaneDims<P>::VH) * 32;
  static constexpr int off_eph = LaneDims<P>::NH;
  static constexpr int off_ech = off_eph + 2 * (P + 1);
  static constexpr int off_cx = off_ech + 2 * (P + 1);
  static constexpr int ops = off_cx + (HELM ? 2 * LaneDims<P>::NC : LaneDims<P>::NL);
  static constexpr int ops_pad = (ops + 3) & ~3;   // one operator buffer
  // Laplace stages the next offset's operator while the lanes apply the
  // current one (two buffers); Helmholtz stages between barriers (one)
  static constexpr bool DB = !HELM;
  static constexpr size_t ops_bytes = sizeof(T) * (size_t)((DB ? 2 : 1) * ops_pad);
  static constexpr size_t cap = 220 * 1024;
  static constexpr int W = ops_bytes + col_bytes * 4 <= cap ? 4
                         : ops_bytes + col_bytes * 2 <= cap ? 2 : 1;
  static constexpr bool fits = ops_bytes + col_bytes * W <= cap;
  static constexpr int CTA = 32 * W;
  static constexpr int V = HELM ? LaneDims<P>::VF : LaneDims<P>::VH;
  // per-lane columns (accumulator, working vector) per warp, T2 each
  static constexpr size_t bytes = ops_bytes + col_bytes * W;
};

template <typename T, bool HELM, int P>
__global__ void __launch_bounds__(LaneSmem<T, HELM, P>::CTA,
                                  LaneReg<T, HELM, P>::value ? LaneRegCtas<T, HELM, P>::value : 1)
k_m2l_lanes(LanesParams<T> p, OpTables<T> t) {
  typedef typename V2t<T>::t T2;
  typedef LaneSmem<T, HELM, P> SM;
  constexpr int kLanesCTA = SM::CTA;
  constexpr int V = SM::V;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* opsb = (T*)smraw;                         // operator buffer(s)
  T2* cols = (T2*)(smraw + SM::ops_bytes);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr bool REG = LaneReg<T, HELM, P>::value;
  T2* acc = cols + (size_t)warp * SM::ncols * V * 32 + lane;   // accumulator, stride 32
  WVec<T2, V, REG> w(acc + (size_t)V * 32);                      // working vector

  // the 8 child types of one parent tile are adjacent in the grid, so the
  // CTAs that read the same source neighbourhood run together (L2 reuse)
  const int tau = blockIdx.x & 7;
  const int split = blockIdx.z;
  const int nx = 1 << (p.level - 1), npx = nx + 2;
  const int64_t npp = (int64_t)npx * npx * npx;
  const int64_t np = (int64_t)nx * nx * nx;
  int64_t plin = (int64_t)(blockIdx.x >> 3) * kLanesCTA + threadIdx.x;
  bool active = plin < np;
  if (p.act) {
    // sparse targets: this CTA's slots of the child type's list
    const int na = p.act_n[tau];
    const int64_t slot0 = (int64_t)(blockIdx.x >> 3) * kLanesCTA;
    if (slot0 >= na) return;                  // the whole CTA, before any barrier
    active = plin < na;
    plin = active ? p.act[(int64_t)tau * np + plin] : 0;
  }
  int64_t pp = 0, pmort = 0;
  if (active) {
    int px = (int)(plin % nx), py = (int)((plin / nx) % nx), pz = (int)(plin / ((int64_t)nx * nx));
    pp = (px + 1) + npx * ((int64_t)(py + 1) + npx * (int64_t)(pz + 1));
    pmort = (int64_t)morton(px, py, pz);
    if (!p.act && p.tmask && !p.tmask[(pmort << 3) | tau]) active = false;
  }
#pragma unroll 1
  for (int c = 0; c < V; c++) { T2 z; z.x = T(0); z.y = T(0); acc[c * 32] = z; }

  // Staging of an offset's operator: the rotation block, both phase sets
  // and the coaxial coefficients (Helmholtz: the level's table of the
  // offset's distance; Laplace: the level's scaled S|R of the shift code).
  // Laplace double-buffers it: while the lanes apply offset j's operator
  // from one buffer, offset j + nsplit's streams into the other (cp.async),
  // so one barrier per offset both publishes a buffer and retires the other.
  auto copy = [&](T* d, const T* src) {
    if constexpr (SM::DB) cp_async_t(d, src); else *d = *src;
  };
  auto stage = [&](int j, T* dst) {
    const int op = c_offsets[tau][j] & 511;
    const T* H = t.H + (int64_t)t.op_ith[op] * t.hstride;
    for (int i = threadIdx.x; i < LaneDims<P>::NH; i += kLanesCTA) copy(dst + i, H + i);
    const T* eph = t.ph + (size_t)op * (t.lmax + 1) * 2;
    const T* ech = t.ch + (size_t)op * (t.lmax + 1) * 2;
    for (int i = threadIdx.x; i < 2 * (P + 1); i += kLanesCTA) {
      copy(dst + SM::off_eph + i, eph + i);
      copy(dst + SM::off_ech + i, ech + i);
    }
    if (HELM) {
      const T* cx = p.coax + (int64_t)t.op_dist[op] * p.coax_stride;
      for (int i = threadIdx.x; i < 2 * LaneDims<P>::NC; i += kLanesCTA)
        copy(dst + SM::off_cx + i, cx + i);
    } else {
      const T* cx = (const T*)p.lapsr + (int64_t)op * LaneDims<P>::NL;
      for (int i = threadIdx.x; i < LaneDims<P>::NL; i += kLanesCTA)
        copy(dst + SM::off_cx + i, cx + i);
    }
    if constexpr (SM::DB) cp_async_commit();
  };
  if (SM::DB && split < 189) stage(split, opsb);
  int buf = 0;
#pragma unroll 1
  for (int j = split; j < 189; j += p.nsplit) {
    const int code = c_offsets[tau][j];
    const int sg = (code >> 9) & 7;
    const int ddx = ((code >> 12) & 3) - 1, ddy = ((code >> 14) & 3) - 1,
              ddz = ((code >> 16) & 3) - 1;
    if constexpr (SM::DB) {
      cp_async_wait_all();
      __syncthreads();   // this offset's operator visible; the other buffer free
      if (j + p.nsplit < 189) stage(j + p.nsplit, opsb + (buf ^ 1) * SM::ops_pad);
    } else {
      __syncthreads();   // previous operator no longer in use
      stage(j, opsb);
      __syncthreads();
    }
    const T* ops = opsb + buf * SM::ops_pad;
    if constexpr (SM::DB) buf ^= 1;
    const T* sH = ops;
    const T* seph = ops + SM::off_eph;
    const T* sech = ops + SM::off_ech;
    const T* scx = ops + SM::off_cx;
    if (!active) continue;
    const int64_t spp = pp + ddx + npx * ((int64_t)ddy + npx * (int64_t)ddz);
    if (p.smask && !p.smask[(int64_t)sg * npp + spp]) continue;   // no sources there
    // a target list's lanes hold boxes that are not neighbours: each reads
    // its source's coefficients contiguously there (box-major copy); sparse
    // storage: the source parent's slot column (the zero column where none)
    const int64_t lstride = p.pmap ? p.lin_stride : npp;
    const int64_t col = p.pmap ? (int64_t)p.pmap[spp] : spp;
    const int64_t cs = p.boxmajor ? 1 : lstride;
    const T2* src = (const T2*)p.lin_raw + (int64_t)sg * V * lstride + (p.boxmajor ? col * V : col);
    if (HELM) {
      // stage A: copy the source into the lane's column with e^{i m ch}
#pragma unroll
      for (int n = 0; n <= P; n++) {
#pragma unroll
        for (int m = -n; m <= n; m++) {
          const int am = m < 0 ? -m : m;
          T2 v = __ldg(src + (int64_t)cidx(n, m) * cs);
          w[cidx(n, m)] = cm(v, sech[2 * am], m < 0 ? -sech[2 * am + 1] : sech[2 * am + 1]);
        }
        cfence();
      }
      // stage B: forward rotation per degree, in place, then e^{-i nu ph}
#pragma unroll
      for (int n = 0; n <= P; n++) {
        T2 in[2 * P + 1];
#pragma unroll
        for (int m = -n; m <= n; m++) in[m + n] = w[cidx(n, m)];
        const int hb = rot_idx(-n, 0, n);
#pragma unroll
        for (int nu = -n; nu <= n; nu++) {
          T sr = T(0), si = T(0);
#pragma unroll
          for (int m = -n; m <= n; m++) {
            const T h = m >= 0 ? sH[hb + (nu + n) * (n + 1) + m]
                               : sH[hb + (-nu + n) * (n + 1) - m];
            sr += h * in[m + n].x;
            si += h * in[m + n].y;
          }
          const int an = nu < 0 ? -nu : nu;
          T2 o; o.x = sr; o.y = si;
          w[cidx(n, nu)] = cm(o, seph[2 * an], nu < 0 ? seph[2 * an + 1] : -seph[2 * an + 1]);
        }
        cfence();
      }
      // stage C: coaxial (S|R) per order m, in place, then e^{i m ph}
#pragma unroll
      for (int m = -P; m <= P; m++) {
        const int am = m < 0 ? -m : m;
        T2 tv[P + 1];
#pragma unroll
        for (int l = am; l <= P; l++) tv[l] = w[cidx(l, m)];
#pragma unroll
        for (int n = am; n <= P; n++) {
          T sr = T(0), si = T(0);
#pragma unroll
          for (int l = am; l <= P; l++) {
            const int ic = l >= n ? coax_idx(l, am, n) : coax_idx(n, am, l);
            const T sgn = (l >= n || ((n + l) & 1) == 0) ? T(1) : T(-1);
            const T cr = sgn * scx[2 * ic], ci = sgn * scx[2 * ic + 1];
            sr += cr * tv[l].x - ci * tv[l].y;
            si += ci * tv[l].x + cr * tv[l].y;
          }
          T2 o; o.x = sr; o.y = si;
          w[cidx(n, m)] = cm(o, seph[2 * am], m < 0 ? -seph[2 * am + 1] : seph[2 * am + 1]);
        }
        cfence();
      }
      // stage D: back rotation, acc[n,nu] += e^{-i nu ch} sum_m H w[n,m]
#pragma unroll
      for (int n = 0; n <= P; n++) {
        T2 in[2 * P + 1];
#pragma unroll
        for (int m = -n; m <= n; m++) in[m + n] = w[cidx(n, m)];
        const int hb = rot_idx(-n, 0, n);
#pragma unroll
        for (int nu = -n; nu <= n; nu++) {
          T sr = T(0), si = T(0);
#pragma unroll
          for (int m = -n; m <= n; m++) {
            const T h = m >= 0 ? sH[hb + (nu + n) * (n + 1) + m]
                               : sH[hb + (-nu + n) * (n + 1) - m];
            sr += h * in[m + n].x;
            si += h * in[m + n].y;
          }
          const int an = nu < 0 ? -nu : nu;
          T2 o; o.x = sr; o.y = si;
          o = cm(o, sech[2 * an], nu < 0 ? sech[2 * an + 1] : -sech[2 * an + 1]);
          T2 a = acc[cidx(n, nu) * 32];
          a.x += o.x; a.y += o.y;
          acc[cidx(n, nu) * 32] = a;
        }
        cfence();
      }
    } else {
      // Laplace, half vectors (m >= 0; negative m are conjugates)
#pragma unroll
      for (int n = 0; n <= P; n++) {
#pragma unroll
        for (int m = 0; m <= n; m++) {
          T2 v = __ldg(src + (int64_t)hidx(n, m) * cs);
          w[hidx(n, m)] = cm(v, sech[2 * m], sech[2 * m + 1]);
        }
        cfence();
      }
#pragma unroll
      for (int n = 0; n <= P; n++) {
        T2 in[P + 1];
#pragma unroll
        for (int m = 0; m <= n; m++) in[m] = w[hidx(n, m)];
        const int hb = rot_idx(-n, 0, n);
#pragma unroll
        for (int nu = 0; nu <= n; nu++) {
          T tr = sH[hb + (nu + n) * (n + 1)] * in[0].x, ti = T(0);
#pragma unroll
          for (int m = 1; m <= n; m++) {
            const T hp = sH[hb + (nu + n) * (n + 1) + m];
            const T hm = sH[hb + (-nu + n) * (n + 1) + m];
            tr += (hp + hm) * in[m].x;
            ti += (hp - hm) * in[m].y;
          }
          const T er = seph[2 * nu], ei = seph[2 * nu + 1];
          T2 o;
          o.x = er * tr + ei * ti;
          o.y = nu == 0 ? T(0) : er * ti - ei * tr;
          w[hidx(n, nu)] = o;
        }
        cfence();
      }
#pragma unroll
      for (int m = 0; m <= P; m++) {
        T2 tv[P + 1];
#pragma unroll
        for (int nd = m; nd <= P; nd++) tv[nd] = w[hidx(nd, m)];
#pragma unroll
        for (int n = m; n <= P; n++) {
          T sr = T(0), si = T(0);
#pragma unroll
          for (int nd = m; nd <= P; nd++) {
            const T c = scx[(n * (P + 1) + nd) * (P + 1) + m];
            sr += c * tv[nd].x;
            si += c * tv[nd].y;
          }
          if (m == 0) si = T(0);
          T2 o; o.x = sr; o.y = si;
          w[hidx(n, m)] = cm(o, seph[2 * m], seph[2 * m + 1]);
        }
        cfence();
      }
#pragma unroll
      for (int n = 0; n <= P; n++) {
        T2 in[P + 1];
#pragma unroll
        for (int m = 0; m <= n; m++) in[m] = w[hidx(n, m)];
        const int hb = rot_idx(-n, 0, n);
#pragma unroll
        for (int nu = 0; nu <= n; nu++) {
          T tr = sH[hb + (nu + n) * (n + 1)] * in[0].x, ti = T(0);
#pragma unroll
          for (int m = 1; m <= n; m++) {
            const T hp = sH[hb + (nu + n) * (n + 1) + m];
            const T hm = sH[hb + (-nu + n) * (n + 1) + m];
            tr += (hp + hm) * in[m].x;
            ti += (hp - hm) * in[m].y;
          }
          const T er = sech[2 * nu], ei = sech[2 * nu + 1];
          T2 a = acc[hidx(n, nu) * 32];
          a.x += er * tr + ei * ti;
          if (nu != 0) a.y += er * ti - ei * tr;
          acc[hidx(n, nu) * 32] = a;
        }
        cfence();
      }
    }
  }
  if (!active) return;
  const int nc = (P + 1) * (P + 1);
  const int64_t g0 = compact_box(p.gmap, pmort << 3);   // storage index of the group
  if (g0 < 0) return;   // (targets lie in stored groups)
  const int64_t b = g0 | tau;
  if (p.nsplit == 1) {
    if (HELM) {
      for (int c = 0; c < V; c++) {
        T2 a = acc[c * 32];
        int64_t o = layout_off(b, c, nc);
        p.cout[2 * o] += a.x;
        p.cout[2 * o + 1] += a.y;
      }
    } else {
      for (int c = 0; c < V; c++) {
        T2 a = acc[c * 32];
        int n = half_degree(c), m = c - n * (n + 1) / 2;
        if (m == 0) {
          p.cout[layout_off(b, n * n, nc)] += a.x;
        } else {
          int id = lidx(n, m);
          p.cout[layout_off(b, id, nc)] += a.x;
          p.cout[layout_off(b, id + 1, nc)] += a.y;
        }
      }
    }
  } else {
    T2* part = (T2*)p.partial_raw + ((int64_t)split * 8 + tau) * V * np + plin;
    for (int c = 0; c < V; c++) part[(int64_t)c * np] = acc[c * 32];
  }
}

// sum the split partials (split order) into the Layout L output
template <typename T, bool HELM>
__global__ void k_lanes_reduce(LanesParams<T> p, int N) {
  typedef typename V2t<T>::t T2;
  const int V = HELM ? (N + 1) * (N + 1) : (N + 1) * (N + 2) / 2;
  const int nc = (N + 1) * (N + 1);
  const int nx = 1 << (p.level - 1);
  const int64_t np = (int64_t)nx * nx * nx;
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np * 8 * V) return;
  const int64_t plin = e % np;
  const int c = (int)((e / np) % V);
  const int tau = (int)(e / (np * V));
  int px = (int)(plin % nx), py = (int)((plin / nx) % nx), pz = (int)(plin / ((int64_t)nx * nx));
  const int64_t pm = (int64_t)morton(px, py, pz);
  if (p.tmask && !p.tmask[(pm << 3) | tau]) return;
  const int64_t g0 = compact_box(p.gmap, pm << 3);
  if (g0 < 0) return;
  const int64_t b = g0 | tau;   // storage index
  T sx = T(0), sy = T(0);
  for (int s = 0; s < p.nsplit; s++) {
    T2 v = ((const T2*)p.partial_raw)[(((int64_t)s * 8 + tau) * V + c) * np + plin];
    sx += v.x; sy += v.y;
  }
  if (HELM) {
    int64_t o = layout_off(b, c, nc);
    p.cout[2 * o] += sx; p.cout[2 * o + 1] += sy;
  } else {
    int n = half_degree(c), m = c - n * (n + 1) / 2;
    if (m == 0) {
      p.cout[layout_off(b, n * n, nc)] += sx;
    } else {
      int id = lidx(n, m);
      p.cout[layout_off(b, id, nc)] += sx;
      p.cout[layout_off(b, id + 1, nc)] += sy;
    }
  }
}

// ------------------------------------------------- Laplace operators
template <typename T>
__global__ void k_lap_sr_ops(OpTables<T> t, int P, T width, int lap_e, T* out) {
  const int P1 = P + 1, NL = P1 * P1 * P1;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (int64_t)kNumOps * NL) return;
  const int op = (int)(i / NL), e = (int)(i % NL);
  const int m = e % P1, nd = (e / P1) % P1, n = e / (P1 * P1);
  const T r = width * t.op_r[op];
  if (!(r > T(0))) { out[i] = T(0); return; }   // shift codes that are not list-4
  const T rinv = T(1) / r, qinv = T(1) / scale2(r, lap_e);
  const int Dm = t.lt + 1;
  const T v = t.lapSR[((int64_t)n * Dm + nd) * Dm + m];
  T sc = rinv, q = T(1);
  for (int k = 0; k < n; k++) sc *= rinv;
  for (int k = 0; k < nd; k++) q *= qinv;
  out[i] = (v * q) * sc;
}

template <typename T>
int build_lap_sr_ops(const OpTables<T>& t, int P, T width, int lap_e, T* out,
                     cudaStream_t s) {
  const int64_t tot = (int64_t)kNumOps * (P + 1) * (P + 1) * (P + 1);
  k_lap_sr_ops<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(t, P, width, lap_e, out);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}
template int build_lap_sr_ops<float>(const OpTables<float>&, int, float, int, float*, cudaStream_t);
template int build_lap_sr_ops<double>(const OpTables<double>&, int, double, int, double*, cudaStream_t);

// ------------------------------------------------------- active lists
constexpr int kActBlock = 256;

__device__ __forceinline__ bool act_flag(const uint8_t* tmask, int nx, int64_t np,
                                         int64_t plin, int tau) {
  if (plin >= np) return false;
  const int px = (int)(plin % nx), py = (int)((plin / nx) % nx),
            pz = (int)(plin / ((int64_t)nx * nx));
  return tmask[((int64_t)morton(px, py, pz) << 3) | tau] != 0;
}

// bcnt[tau][block] = active parents of the block
__global__ void k_act_count(const uint8_t* __restrict__ tmask, int nx, int64_t np,
                            int nblk, int* __restrict__ bcnt) {
  const int tau = blockIdx.y;
  const int64_t plin = (int64_t)blockIdx.x * kActBlock + threadIdx.x;
  const int c = __syncthreads_count(act_flag(tmask, nx, np, plin, tau));
  if (threadIdx.x == 0) bcnt[(int64_t)tau * nblk + blockIdx.x] = c;
}

// exclusive scan of bcnt[tau][*] in place, one CTA per tau; act_n[tau] = total
__global__ void k_act_scan(int* __restrict__ bcnt, int nblk, int* __restrict__ act_n) {
  __shared__ int s[1024];
  const int tau = blockIdx.x, tid = threadIdx.x;
  int* b = bcnt + (int64_t)tau * nblk;
  int carry = 0;
  for (int base = 0; base < nblk; base += 1024) {
    const int v = base + tid < nblk ? b[base + tid] : 0;
    s[tid] = v;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
      const int u = tid >= d ? s[tid - d] : 0;
      __syncthreads();
      s[tid] += u;
      __syncthreads();
    }
    if (base + tid < nblk) b[base + tid] = carry + s[tid] - v;
    carry += s[1023];
    __syncthreads();
  }
  if (tid == 0) act_n[tau] = carry;
}

// act[tau][offset of the block + rank in the block] = plin
__global__ void k_act_scatter(const uint8_t* __restrict__ tmask, int nx, int64_t np,
                              int nblk, const int* __restrict__ bcnt, int* __restrict__ act) {
  __shared__ int wsum[kActBlock / 32];
  const int tau = blockIdx.y, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t plin = (int64_t)blockIdx.x * kActBlock + threadIdx.x;
  const bool f = act_flag(tmask, nx, np, plin, tau);
  const unsigned bal = __ballot_sync(0xffffffffu, f);
  if (lane == 0) wsum[warp] = __popc(bal);
  __syncthreads();
  int off = bcnt[(int64_t)tau * nblk + blockIdx.x];
  for (int w = 0; w < warp; w++) off += wsum[w];
  off += __popc(bal & ((1u << lane) - 1u));
  if (f) act[(int64_t)tau * np + off] = (int)plin;
}

size_t active_list_scratch(int level) {
  const int64_t np = (int64_t)1 << (3 * (level - 1));
  return (size_t)8 * ((np + kActBlock - 1) / kActBlock);
}

int build_active_lists(const uint8_t* tmask, int level, int* act, int* act_n,
                       int* scratch, cudaStream_t s) {
  const int nx = 1 << (level - 1);
  const int64_t np = (int64_t)nx * nx * nx;
  const int nblk = (int)((np + kActBlock - 1) / kActBlock);
  dim3 grid((unsigned)nblk, 8);
  k_act_count<<<grid, kActBlock, 0, s>>>(tmask, nx, np, nblk, scratch);
  k_act_scan<<<8, 1024, 0, s>>>(scratch, nblk, act_n);
  k_act_scatter<<<grid, kActBlock, 0, s>>>(tmask, nx, np, nblk, scratch, act);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------- launchers
template <typename T, bool HELM>
int launch_lanes_reduce(const LanesParams<T>& p, cudaStream_t s) {
  const int N = p.N;
  const int V = HELM ? (N + 1) * (N + 1) : (N + 1) * (N + 2) / 2;
  const int64_t np = (int64_t)1 << (3 * (p.level - 1));
  const int64_t tot = np * 8 * V;
  k_lanes_reduce<T, HELM><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(p, N);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

template <typename T, bool HELM>
int lanes_to_lin(const T* arr, int level, int N, int scale_e, void* lin, cudaStream_t s,
                 bool boxmajor) {
  typedef typename V2t<T>::t T2;
  const int V = HELM ? (N + 1) * (N + 1) : (N + 1) * (N + 2) / 2;
  const int64_t nx = 1 << (level - 1), npx = nx + 2;
  WBFMM_CUDA(cudaMemsetAsync(lin, 0, sizeof(T2) * 8 * V * npx * npx * npx, s));
  const int64_t tot = nx * nx * nx * V * 8;
  k_to_lin<T, HELM><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(arr, level, N, scale_e,
                                                                   boxmajor, (T2*)lin);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

template <typename T, bool HELM>
int lanes_to_lin_groups(const T* arr, int64_t groups, int N, int scale_e, void* lin,
                        cudaStream_t s, bool boxmajor) {
  typedef typename V2t<T>::t T2;
  const int V = HELM ? (N + 1) * (N + 1) : (N + 1) * (N + 2) / 2;
  const int64_t tot = (groups + 1) * V * 8;
  k_to_lin_groups<T, HELM><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(arr, groups, N, scale_e,
                                                                         boxmajor, (T2*)lin);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

size_t lanes_lin_groups_bytes(int64_t groups, int N, bool helm, size_t tsize) {
  const size_t V = helm ? (N + 1) * (N + 1) : (N + 1) * (N + 2) / 2;
  return 2 * tsize * 8 * V * (size_t)(groups + 1);
}

int build_parent_slot_map(const uint32_t* gmap, int level, uint32_t groups, uint32_t* pmap,
                          cudaStream_t s) {
  const int nx = 1 << (level - 1);
  const int64_t npp = (int64_t)(nx + 2) * (nx + 2) * (nx + 2);
  k_parent_slot_map<<<(unsigned)((npp + 255) / 256), 256, 0, s>>>(gmap, nx, npp, groups, pmap);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

__global__ void k_source_mask(const uint32_t* __restrict__ src_n, int nx, int64_t npp,
                              uint8_t* __restrict__ smask) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 8 * npp) return;
  const int sg = (int)(e / npp);
  const int64_t pp = e - sg * npp;
  const int npx = nx + 2;
  const int px = (int)(pp % npx) - 1, py = (int)((pp / npx) % npx) - 1,
            pz = (int)(pp / ((int64_t)npx * npx)) - 1;
  uint8_t f = 0;
  if (px >= 0 && px < nx && py >= 0 && py < nx && pz >= 0 && pz < nx)
    f = src_n[((int64_t)morton(px, py, pz) << 3) | sg] != 0;
  smask[e] = f;
}

size_t source_mask_bytes(int level) {
  const size_t npx = (1u << (level - 1)) + 2;
  return 8 * npx * npx * npx;
}

int build_source_mask(const uint32_t* src_n, int level, uint8_t* smask, cudaStream_t s) {
  const int nx = 1 << (level - 1);
  const int64_t npp = (int64_t)(nx + 2) * (nx + 2) * (nx + 2);
  k_source_mask<<<(unsigned)((8 * npp + 255) / 256), 256, 0, s>>>(src_n, nx, npp, smask);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

size_t lanes_lin_bytes(int level, int N, bool helm, size_t tsize) {
  const size_t V = helm ? (N + 1) * (N + 1) : (N + 1) * (N + 2) / 2;
  const size_t npx = (1u << (level - 1)) + 2;
  return 2 * tsize * 8 * V * npx * npx * npx;
}

template <typename T, bool HELM, int P>
static int launch_lanes_P(const LanesParams<T>& p, const OpTables<T>& t,
                          cudaStream_t s) {
  typedef LaneSmem<T, HELM, P> SM;
  WBFMM_SMEM(SM::bytes, k_m2l_lanes<T, HELM, P>);
  const int64_t np = (int64_t)1 << (3 * (p.level - 1));
  dim3 grid((unsigned)(8 * ((np + SM::CTA - 1) / SM::CTA)), 1, p.nsplit);
  k_m2l_lanes<T, HELM, P><<<grid, SM::CTA, SM::bytes, s>>>(p, t);
  WBFMM_CUDA(cudaGetLastError());
  if (p.nsplit > 1) return launch_lanes_reduce<T, HELM>(p, s);
  return 0;
}

template <typename T, bool HELM>
bool lanes_supported(int Ns, int Nr) {
  if (Ns != Nr) return false;
  if (HELM ? (Ns < 2 || Ns > kLanesMaxHelm) : (Ns < 2 || Ns > kLanesMaxLap)) return false;
  // the instantiation's operator buffers and vector columns fit one CTA
  switch (Ns) {
#define WBFMM_LANES_FIT(PP) \
  case PP: return LaneSmem<T, HELM, PP>::fits;
    WBFMM_LANES_FIT(2) WBFMM_LANES_FIT(3) WBFMM_LANES_FIT(4) WBFMM_LANES_FIT(5)
    WBFMM_LANES_FIT(6) WBFMM_LANES_FIT(7) WBFMM_LANES_FIT(8) WBFMM_LANES_FIT(9)
    WBFMM_LANES_FIT(10) WBFMM_LANES_FIT(11) WBFMM_LANES_FIT(12) WBFMM_LANES_FIT(13)
    WBFMM_LANES_FIT(14) WBFMM_LANES_FIT(15) WBFMM_LANES_FIT(16)
#undef WBFMM_LANES_FIT
    default: return false;
  }
}

template <typename T, bool HELM>
int launch_m2l_lanes(const LanesParams<T>& p, const OpTables<T>& t,
                     cudaStream_t s) {
  {
    int rc = ensure_offsets();
    if (rc) return rc;
  }
  switch (p.N) {
#define WBFMM_LANES_CASE(PP) \
  case PP: return launch_lanes_P<T, HELM, PP>(p, t, s);
    WBFMM_LANES_CASE(2)
    WBFMM_LANES_CASE(3)
    WBFMM_LANES_CASE(4)
    WBFMM_LANES_CASE(5)
    WBFMM_LANES_CASE(6)
    WBFMM_LANES_CASE(7)
    WBFMM_LANES_CASE(8)
#undef WBFMM_LANES_CASE
    default: break;
  }
  if (!HELM) {
    switch (p.N) {
#define WBFMM_LANES_CASE(PP) \
  case PP: return launch_lanes_P<T, false, PP>(p, t, s);
      WBFMM_LANES_CASE(9)
      WBFMM_LANES_CASE(10)
      WBFMM_LANES_CASE(11)
      WBFMM_LANES_CASE(12)
      WBFMM_LANES_CASE(13)
      WBFMM_LANES_CASE(14)
      WBFMM_LANES_CASE(15)
      WBFMM_LANES_CASE(16)
#undef WBFMM_LANES_CASE
      default: break;
    }
  }
  return set_error(-3, "M2L lane kernel: order not instantiated");
}

#define WBFMM_LANES_INST(T, H)                                                   \
  template int lanes_to_lin<T, H>(const T*, int, int, int, void*, cudaStream_t, bool); \
  template int lanes_to_lin_groups<T, H>(const T*, int64_t, int, int, void*, cudaStream_t, bool); \
  template int launch_lanes_reduce<T, H>(const LanesParams<T>&, cudaStream_t);   \
  template bool lanes_supported<T, H>(int, int);                                 \
  template int launch_m2l_lanes<T, H>(const LanesParams<T>&, const OpTables<T>&, \
                                      cudaStream_t);
WBFMM_LANES_INST(double, true)
WBFMM_LANES_INST(double, false)
WBFMM_LANES_INST(float, true)
WBFMM_LANES_INST(float, false)

}  // namespace wbfmm
