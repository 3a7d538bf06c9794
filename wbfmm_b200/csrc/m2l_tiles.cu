// M2L for any expansion order: offset-major tiles of targets.
//
// As in the lane-per-pair kernel, the list-4 interactions of a level are
// regrouped by target child type tau, so that TC target boxes of one type
// (the tau-children of TC consecutive parents) see the same 189 offsets,
// each with one rotate / coaxial / rotate-back operator (src/pass.c:56-105:
// wbfmm_rotate_H, wbfmm_coaxial_translate_ref, rotate back).  Here a CTA of
// 256 threads applies each offset's operator to all TC source vectors at
// once, as three small matrix products staged through shared memory:
//
//   A  X[n,m][t]  = e^{i m ch} src_t[n,m]
//   B  Y[n,nu][t] = e^{-i nu ph} sum_m H_n^{nu,m} X[n,m][t]       (per degree)
//   C  Z[n,m][t]  = e^{i m ph} sum_l (S|R)_{l,n}^{|m|} Y[l,m][t]   (per order)
//   D  acc[n,nu][t] += e^{-i nu ch} sum_m H_n^{nu,m} Z[n,m][t]    (per degree)
//
// Each thread computes a register tile of 2 output rows x 4 targets, so an
// operator entry read from shared memory feeds 4 (complex) multiply-adds and
// a source value 2.  The order is a runtime parameter; TC (32, 16 or 8) is
// the largest whose three vector blocks fit beside the operator.  Laplace
// uses half vectors (m >= 0), as the reference's real-packed coefficients.
// Per offset: the column map (double-buffered, so that it is built while
// the previous offset's stage D still reads its own) and one barrier; the
// operator staging and stage A in one phase (A reads its phases from the
// table, not the staged copy), then B, C and D, four barriers in all.
#include <cuda_runtime.h>

#include "engine.h"
#include "kernels.h"
#include "m2l_lanes.h"
#include "translate.cuh"

namespace wbfmm {

namespace {

template <typename T> struct C2;
template <> struct C2<float> { typedef float2 t; };
template <> struct C2<double> { typedef double2 t; };

template <typename T>
struct __align__(16) R4 { T a, b, c, d; };

// Helmholtz coaxial rows for stage C: per distance, per order am >= 0, per
// row pair (n0 = am + 2k, n0 + 1), per l = am..P, the complex (S|R)
// coefficients of both rows with the sign of l < n folded in, as
// (re0, im0, re1, im1).  Offset of the pair's row, in entries:
__host__ __device__ inline int coax_row_base(int P, int am) {
  int b = 0;
  for (int m = 0; m < am; m++) b += ((P + 2 - m) / 2) * (P + 1 - m);
  return b;
}
__host__ __device__ inline int coax_rows(int P) { return coax_row_base(P, P + 1); }

template <typename T>
__global__ void k_helm_coax_rows(const T* __restrict__ raw, int64_t raw_stride, int P,
                                 T* __restrict__ out) {
  const int d = blockIdx.x, am = blockIdx.y;
  const int len = P + 1 - am, npair = (P + 2 - am) / 2;
  const T* cx = raw + (int64_t)d * raw_stride;
  T* o = out + ((int64_t)d * coax_rows(P) + coax_row_base(P, am)) * 4;
  for (int e = threadIdx.x; e < npair * len; e += blockDim.x) {
    const int k = e / len, l = am + e % len;
    T v[4] = {T(0), T(0), T(0), T(0)};
    for (int r = 0; r < 2; r++) {
      const int n = am + 2 * k + r;
      if (n > P) continue;
      const int ic = l >= n ? coax_idx(l, am, n) : coax_idx(n, am, l);
      const T sg = (l >= n || ((n + l) & 1) == 0) ? T(1) : T(-1);
      v[2 * r] = sg * cx[2 * ic];
      v[2 * r + 1] = sg * cx[2 * ic + 1];
    }
    for (int c = 0; c < 4; c++) o[4 * e + c] = v[c];
  }
}

__constant__ int c_tile_offsets[8][189];
bool g_tile_offsets_ready[64] = {false};

int ensure_tile_offsets() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && g_tile_offsets_ready[dev]) return 0;
  int tab[8 * 189];
  build_offset_table(tab);
  WBFMM_CUDA(cudaMemcpyToSymbol(c_tile_offsets, tab, sizeof(tab)));
  if (dev < 64) g_tile_offsets_ready[dev] = true;
  return 0;
}

constexpr int kTileThreads = 256;

// shared-memory plan of one launch (units: bytes)
struct TilePlan {
  int P, V, TC, NH, ncx, nB, nC, cx_off;
  bool dense;  // Helmholtz: stage C reads the level's coaxial rows (k_helm_coax_rows)
  bool sparse; // sparse level storage: each target's source column (s_src)
  size_t ops_bytes, desc_bytes, vec_bytes, total;
};

template <typename T, bool HELM>
__host__ __device__ TilePlan tile_plan(int P, int TC, bool dense, bool sparse) {
  TilePlan q;
  q.P = P;
  q.TC = TC;
  q.dense = HELM && dense;
  q.sparse = sparse;
  q.V = HELM ? (P + 1) * (P + 1) : (P + 1) * (P + 2) / 2;
  q.NH = (P + 1) * (P + 2) * (4 * P + 3) / 6;
  q.ncx = !HELM ? (P + 1) * (P + 1) * (P + 1)
          : q.dense ? 4 * coax_rows(P) : 2 * ((P + 1) * (P + 2) * (P + 3) / 6);
  q.nB = 0;
  for (int n = 0; n <= P; n++) q.nB += HELM ? n + 1 : (n + 2) / 2;
  q.nC = 0;
  for (int m = HELM ? -P : 0; m <= P; m++) {
    int am = m < 0 ? -m : m;
    q.nC += (P + 1 - am + 1) / 2;
  }
  // the coaxial table starts on a 4-value boundary (16-byte row loads)
  q.cx_off = (q.NH + 6 * (P + 1) + 3) & ~3;
  size_t ops = sizeof(T) * ((size_t)q.cx_off + q.ncx);
  q.ops_bytes = (ops + 15) & ~(size_t)15;
  q.desc_bytes = ((sizeof(int) * (size_t)(q.nB + (q.dense ? 2 : 1) * q.nC + q.V) +
                   (sparse ? 5 : 4) * sizeof(int) * TC) + 15) & ~(size_t)15;
  q.vec_bytes = 3 * sizeof(typename C2<T>::t) * (size_t)q.V * TC;
  q.total = q.ops_bytes + q.desc_bytes + q.vec_bytes;
  return q;
}

constexpr size_t kTileSmemCap = 220 * 1024;

// Targets per CTA: the tile kernel is latency-bound (one offset's stages are
// separated by barriers), so prefer the TC that keeps the most targets
// resident per SM (228 KB of shared memory, 1 KB reserved per CTA), and on a
// tie the smaller TC (more CTAs, more warps to switch between).  Helmholtz
// stage C reads the coaxial rows (twice the triangular table, no index
// arithmetic in the inner loop; about 10% faster at order 14) when they keep
// as many targets resident as the triangular table does.
struct TileChoice { int tc; bool dense; };

template <typename T, bool HELM>
TileChoice pick_tc(int P, bool sparse) {
  TileChoice best = {0, false};
  int best_score = 0;
  for (int dense = 0; dense <= (HELM ? 1 : 0); dense++)
    for (int tc = 32; tc >= 8; tc >>= 1) {
      const size_t bytes = tile_plan<T, HELM>(P, tc, dense, sparse).total;
      if (bytes > kTileSmemCap) continue;
      const int ctas = (int)((228 * 1024) / (bytes + 1024));
      const int score = ctas * tc;
      if (score > best_score ||
          (score == best_score && (tc < best.tc || (tc == best.tc && dense)))) {
        best.tc = tc; best.dense = dense; best_score = score;
      }
    }
  return best;
}

// the 4 consecutive columns of a thread's register tile (16-byte aligned:
// row offsets are multiples of TC and t0 of 4): two 16-byte loads for FP32
__device__ __forceinline__ void load_cols(const float2* p, float2 (&o)[4]) {
  const float4 a = reinterpret_cast<const float4*>(p)[0];
  const float4 b = reinterpret_cast<const float4*>(p)[1];
  o[0] = make_float2(a.x, a.y); o[1] = make_float2(a.z, a.w);
  o[2] = make_float2(b.x, b.y); o[3] = make_float2(b.z, b.w);
}
__device__ __forceinline__ void load_cols(const double2* p, double2 (&o)[4]) {
#pragma unroll
  for (int k = 0; k < 4; k++) o[k] = p[k];
}
__device__ __forceinline__ void store_cols(float2* p, const float2 (&v)[4]) {
  reinterpret_cast<float4*>(p)[0] = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
  reinterpret_cast<float4*>(p)[1] = make_float4(v[2].x, v[2].y, v[3].x, v[3].y);
}
__device__ __forceinline__ void store_cols(double2* p, const double2 (&v)[4]) {
#pragma unroll
  for (int k = 0; k < 4; k++) p[k] = v[k];
}

template <typename T2, typename T>
__device__ __forceinline__ T2 cmul(T2 a, T er, T ei) {
  T2 r;
  r.x = a.x * er - a.y * ei;
  r.y = a.x * ei + a.y * er;
  return r;
}

// resident CTAs the register budget is sized for: the shared-memory limit
// of the serving orders (FP32 Laplace 3 per SM at p = 14, the others 2)
template <typename T, bool HELM>
__global__ void __launch_bounds__(kTileThreads, (HELM || sizeof(T) == 8) ? 2 : 3)
k_m2l_tiles(LanesParams<T> p, OpTables<T> t, int TC, bool dense) {
  typedef typename C2<T>::t T2;
  extern __shared__ __align__(16) unsigned char smraw[];
  const TilePlan q = tile_plan<T, HELM>(p.N, TC, dense, p.pmap != nullptr);
  const int P = q.P, V = q.V;
  T* sH = (T*)smraw;
  T* seph = sH + q.NH;
  T* sech = seph + 2 * (P + 1);
  T* scx = sH + q.cx_off;
  int* dB = (int*)(smraw + q.ops_bytes);
  int* dC = dB + q.nB;
  int* s_nm = dC + q.nC;             // (n, m) of each vector entry
  int* s_pp = s_nm + V;              // padded-grid index of each target's parent
  int* s_act = s_pp + TC;            // 1 + parent linear index, 0: no target
  int* s_map = s_act + TC;           // the offset's columns: target of each (two buffers)
  int* s_src = s_map + 2 * TC;       // sparse: each target's source column in lin
  int* dCo = s_src + (q.sparse ? TC : 0);   // Helmholtz: row offset of each C row pair
  T2* X = (T2*)(smraw + q.ops_bytes + q.desc_bytes);
  T2* Y = X + (size_t)V * TC;
  T2* A = Y + (size_t)V * TC;
  const int tid = threadIdx.x;

  // child types of one target tile adjacent in the grid: shared sources
  const int tau = blockIdx.x & 7, split = blockIdx.z;
  const int nx = 1 << (p.level - 1), npx = nx + 2;
  const int64_t npp = (int64_t)npx * npx * npx;
  const int64_t np = (int64_t)nx * nx * nx;
  const int64_t lstride = p.pmap ? p.lin_stride : npp;   // lin columns per (tau, c)
  const int64_t base = (int64_t)(blockIdx.x >> 3) * TC;
  // sparse targets: this CTA's slots of the child type's list
  const int64_t nlist = p.act ? (int64_t)p.act_n[tau] : np;
  if (base >= nlist) return;                  // the whole CTA, before any barrier

  // stage descriptors: B/D rows (n, nu0) and C rows (m, n0), 2 rows each
  if (tid == 0) {
    int k = 0;
    for (int n = 0; n <= P; n++)
      for (int nu = HELM ? -n : 0; nu <= n; nu += 2) dB[k++] = n | ((nu + 64) << 8);
    k = 0;
    for (int m = HELM ? -P : 0; m <= P; m++) {
      int am = m < 0 ? -m : m;
      for (int n = am; n <= P; n += 2) {
        if (q.dense) dCo[k] = coax_row_base(P, am) + ((n - am) / 2) * (P + 1 - am);
        dC[k++] = n | ((m + 64) << 8);
      }
    }
  }
  for (int c = tid; c < V; c += kTileThreads) {
    const int n = HELM ? full_degree(c) : half_degree(c);
    const int m = HELM ? c - n * (n + 1) : c - n * (n + 1) / 2;
    s_nm[c] = n | ((m + 64) << 8);
  }
  for (int i = tid; i < TC; i += kTileThreads) {
    int64_t plin = base + i;
    int act = plin < nlist;
    int pp = 0;
    if (act) {
      if (p.act) plin = p.act[(int64_t)tau * np + plin];
      int px = (int)(plin % nx), py = (int)((plin / nx) % nx), pz = (int)(plin / ((int64_t)nx * nx));
      pp = (px + 1) + npx * ((py + 1) + npx * (pz + 1));
      if (!p.act && p.tmask && !p.tmask[((int64_t)morton(px, py, pz) << 3) | tau]) act = 0;
    }
    s_pp[i] = pp;
    s_act[i] = act ? (int)plin + 1 : 0;
  }
  for (int i = tid; i < V * TC; i += kTileThreads) { T2 z; z.x = T(0); z.y = T(0); A[i] = z; }
  __syncthreads();

#pragma unroll 1
  for (int j = split; j < 189; j += p.nsplit) {
    const int code = c_tile_offsets[tau][j];
    const int op = code & 511, sg = (code >> 9) & 7;
    const int ddx = ((code >> 12) & 3) - 1, ddy = ((code >> 14) & 3) - 1,
              ddz = ((code >> 16) & 3) - 1;
    const int64_t doff = ddx + npx * ((int64_t)ddy + npx * (int64_t)ddz);
    // the previous offset's operator and vectors are free.  Only the targets
    // whose source box of this offset lies in the grid (and holds sources,
    // with skip_empty) take a column: the stages run over ceil(cnt / 4)
    // groups of 4 columns, and an offset with none is skipped (the decision
    // is the CTA's)
    int f = 0;
    if (q.sparse && tid < TC) {
      // an active target's s_pp + doff stays on the padded grid (doff moves
      // one parent at most); a slot without a target is never read
      s_src[tid] = s_act[tid] ? (int)p.pmap[s_pp[tid] + doff] : 0;
    }
    if (tid < TC && s_act[tid]) {
      if (p.smask) {
        f = p.smask[(int64_t)sg * npp + s_pp[tid] + doff];
      } else {
        const int pp = s_pp[tid];
        const int sx = pp % npx + ddx, sy = (pp / npx) % npx + ddy, sz = pp / (npx * npx) + ddz;
        f = sx >= 1 && sx <= nx && sy >= 1 && sy <= nx && sz >= 1 && sz <= nx;
      }
    }
    // the columns (targets in warp 0: TC <= 32), into the buffer that the
    // offset before last read in its stage D (finished before the last
    // barrier); stage D of the previous offset reads the other one
    int* smap = s_map + ((j - split) / p.nsplit & 1) * TC;
    if (tid < 32) {
      const unsigned bal = __ballot_sync(0xffffffffu, f);
      if (f) smap[__popc(bal & ((1u << tid) - 1u))] = tid;
    }
    const int cnt = __syncthreads_count(f);
    if (cnt == 0) continue;
    const int TQ = (cnt + 3) / 4, TCc = 4 * TQ;
    // the operator into shared memory and (same phase, one barrier) stage A:
    // the TC source vectors with e^{i m ch}, the phases read from the table
    {
      const T* H = t.H + (int64_t)t.op_ith[op] * t.hstride;
      for (int i = tid; i < q.NH; i += kTileThreads) sH[i] = H[i];
      const T* eph = t.ph + (size_t)op * (t.lmax + 1) * 2;
      const T* ech = t.ch + (size_t)op * (t.lmax + 1) * 2;
      for (int i = tid; i < 2 * (P + 1); i += kTileThreads) {
        seph[i] = eph[i];
        sech[i] = ech[i];
      }
      if (HELM) {
        // the offset's distance: the level's coaxial rows (k_helm_coax_rows)
        // or its triangular (S|R) table
        const T* cx = q.dense ? (const T*)p.hcx + (int64_t)t.op_dist[op] * q.ncx
                              : p.coax + (int64_t)t.op_dist[op] * p.coax_stride;
        for (int i = tid; i < q.ncx; i += kTileThreads) scx[i] = cx[i];
      } else {
        // the level's S|R(n,nd,m) / (t^{n+1} (2^e t)^nd) of this shift code
        // (build_lap_sr_ops), on sources scaled by 2^(e nd)
        const T* cx = (const T*)p.lapsr + (int64_t)op * q.ncx;
        for (int i = tid; i < q.ncx; i += kTileThreads) scx[i] = cx[i];
      }
    }
    {
      const T* ech = t.ch + (size_t)op * (t.lmax + 1) * 2;
      const T2* src = (const T2*)p.lin_raw + (int64_t)sg * V * lstride + (q.sparse ? 0 : doff);
      const int* col = q.sparse ? s_src : s_pp;
      for (int i = tid; i < V * TCc; i += kTileThreads) {
        const int c = i / TCc, tt = i - c * TCc;
        T2 v;
        v.x = T(0); v.y = T(0);
        if (tt < cnt) {
          v = src[(int64_t)c * lstride + col[smap[tt]]];
          const int m = (s_nm[c] >> 8) - 64, am = m < 0 ? -m : m;
          const T er = __ldg(ech + 2 * am), ei = __ldg(ech + 2 * am + 1);
          v = cmul(v, er, m < 0 ? -ei : ei);
        }
        X[(size_t)c * TC + tt] = v;
      }
    }
    __syncthreads();
    // stage B: forward rotation per degree, then e^{-i nu ph}
    for (int w = tid; w < q.nB * TQ; w += kTileThreads) {
      const int d = dB[w / TQ], t0 = (w % TQ) * 4;
      const int n = d & 255, nu0 = (d >> 8) - 64;
      const bool two = nu0 + 1 <= n;
      const int hb = rot_idx(-n, 0, n);
      T2 a0[4], a1[4];
#pragma unroll
      for (int k = 0; k < 4; k++) { a0[k].x = a0[k].y = a1[k].x = a1[k].y = T(0); }
      if (HELM) {
        // rows nu0 and nu0 + 1 of the half-stored matrix: H(nu, m) for
        // m >= 0, H(-nu, -m) for m < 0, as two loops (without a second row,
        // a1 is not stored and reads the first row again)
        const T* rp0 = sH + hb + (nu0 + n) * (n + 1);
        const T* rn0 = sH + hb + (-nu0 + n) * (n + 1);
        const T* rp1 = two ? rp0 + (n + 1) : rp0;
        const T* rn1 = two ? rn0 - (n + 1) : rn0;
        const T2* xr = X + (size_t)cidx(n, -n) * TC + t0;
        for (int m = n; m > 0; m--, xr += TC) {
          const T h0 = rn0[m], h1 = rn1[m];
          T2 xv[4];
          load_cols(xr, xv);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 x = xv[k];
            a0[k].x += h0 * x.x; a0[k].y += h0 * x.y;
            a1[k].x += h1 * x.x; a1[k].y += h1 * x.y;
          }
        }
        for (int m = 0; m <= n; m++, xr += TC) {
          const T h0 = rp0[m], h1 = rp1[m];
          T2 xv[4];
          load_cols(xr, xv);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 x = xv[k];
            a0[k].x += h0 * x.x; a0[k].y += h0 * x.y;
            a1[k].x += h1 * x.x; a1[k].y += h1 * x.y;
          }
        }
        for (int r = 0; r < (two ? 2 : 1); r++) {
          const int nu = nu0 + r, an = nu < 0 ? -nu : nu;
          const T er = seph[2 * an], ei = nu < 0 ? seph[2 * an + 1] : -seph[2 * an + 1];
          T2* yr = Y + (size_t)cidx(n, nu) * TC + t0;
#pragma unroll
          for (int k = 0; k < 4; k++) yr[k] = cmul(r ? a1[k] : a0[k], er, ei);
        }
      } else {
        // a0/a1 hold (tr, ti) of rows nu0, nu0 + 1
        for (int m = 0; m <= n; m++) {
          const T2* xr = X + (size_t)hidx(n, m) * TC + t0;
          T p0, m0, p1 = T(0), m1 = T(0);
          p0 = sH[hb + (nu0 + n) * (n + 1) + m];
          m0 = sH[hb + (-nu0 + n) * (n + 1) + m];
          if (two) {
            p1 = sH[hb + (nu0 + 1 + n) * (n + 1) + m];
            m1 = sH[hb + (-nu0 - 1 + n) * (n + 1) + m];
          }
          if (m == 0) { m0 = T(0); m1 = T(0); }
          T2 xv[4];
          load_cols(xr, xv);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 x = xv[k];
            a0[k].x += (p0 + m0) * x.x; a0[k].y += (p0 - m0) * x.y;
            a1[k].x += (p1 + m1) * x.x; a1[k].y += (p1 - m1) * x.y;
          }
        }
        for (int r = 0; r < (two ? 2 : 1); r++) {
          const int nu = nu0 + r;
          const T er = seph[2 * nu], ei = seph[2 * nu + 1];
          T2* yr = Y + (size_t)hidx(n, nu) * TC + t0;
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 a = r ? a1[k] : a0[k];
            T2 o;
            o.x = er * a.x + ei * a.y;
            o.y = nu == 0 ? T(0) : er * a.y - ei * a.x;
            yr[k] = o;
          }
        }
      }
    }
    __syncthreads();
    // stage C: coaxial translation per order m, then e^{i m ph}; into X
    for (int w = tid; w < q.nC * TQ; w += kTileThreads) {
      const int d = dC[w / TQ], t0 = (w % TQ) * 4;
      const int n0 = d & 255, m = (d >> 8) - 64, am = m < 0 ? -m : m;
      const bool two = n0 + 1 <= P;
      T2 a0[4], a1[4];
#pragma unroll
      for (int k = 0; k < 4; k++) { a0[k].x = a0[k].y = a1[k].x = a1[k].y = T(0); }
      const R4<T>* crow = q.dense ? (const R4<T>*)scx + dCo[w / TQ] - am : nullptr;
      for (int l = am; l <= P; l++) {
        const T2* yr = Y + (size_t)(HELM ? cidx(l, m) : hidx(l, m)) * TC + t0;
        if (HELM) {
          T c0r, c0i, c1r = T(0), c1i = T(0);
          if (q.dense) {
            const R4<T> c = crow[l];
            c0r = c.a; c0i = c.b; c1r = c.c; c1i = c.d;
          } else {
            int ic = l >= n0 ? coax_idx(l, am, n0) : coax_idx(n0, am, l);
            const T sg0 = (l >= n0 || ((n0 + l) & 1) == 0) ? T(1) : T(-1);
            c0r = sg0 * scx[2 * ic];
            c0i = sg0 * scx[2 * ic + 1];
            if (two) {
              const int n1 = n0 + 1;
              ic = l >= n1 ? coax_idx(l, am, n1) : coax_idx(n1, am, l);
              const T sg1 = (l >= n1 || ((n1 + l) & 1) == 0) ? T(1) : T(-1);
              c1r = sg1 * scx[2 * ic];
              c1i = sg1 * scx[2 * ic + 1];
            }
          }
          T2 yv[4];
          load_cols(yr, yv);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 y = yv[k];
            a0[k].x += c0r * y.x - c0i * y.y; a0[k].y += c0i * y.x + c0r * y.y;
            a1[k].x += c1r * y.x - c1i * y.y; a1[k].y += c1i * y.x + c1r * y.y;
          }
        } else {
          const T c0 = scx[(n0 * (P + 1) + l) * (P + 1) + m];
          const T c1 = two ? scx[((n0 + 1) * (P + 1) + l) * (P + 1) + m] : T(0);
          T2 yv[4];
          load_cols(yr, yv);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 y = yv[k];
            a0[k].x += c0 * y.x; a0[k].y += c0 * y.y;
            a1[k].x += c1 * y.x; a1[k].y += c1 * y.y;
          }
        }
      }
      const T er = seph[2 * am], ei = m < 0 ? -seph[2 * am + 1] : seph[2 * am + 1];
      for (int r = 0; r < (two ? 2 : 1); r++) {
        const int n = n0 + r;
        T2* xr = X + (size_t)(HELM ? cidx(n, m) : hidx(n, m)) * TC + t0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          T2 a = r ? a1[k] : a0[k];
          if (!HELM && m == 0) a.y = T(0);
          xr[k] = cmul(a, er, ei);
        }
      }
    }
    __syncthreads();
    // stage D: back rotation per degree, e^{-i nu ch}, accumulate; when
    // every target has a column (the map is the identity) a thread's four
    // accumulator columns are updated with two 16-byte loads and stores
    const bool full = cnt == TC;
    for (int w = tid; w < q.nB * TQ; w += kTileThreads) {
      const int d = dB[w / TQ], t0 = (w % TQ) * 4;
      const int n = d & 255, nu0 = (d >> 8) - 64;
      const bool two = nu0 + 1 <= n;
      const int hb = rot_idx(-n, 0, n);
      T2 a0[4], a1[4];
#pragma unroll
      for (int k = 0; k < 4; k++) { a0[k].x = a0[k].y = a1[k].x = a1[k].y = T(0); }
      if (HELM) {
        // rows nu0 and nu0 + 1 of the half-stored matrix: H(nu, m) for
        // m >= 0, H(-nu, -m) for m < 0, as two loops (without a second row,
        // a1 is not stored and reads the first row again)
        const T* rp0 = sH + hb + (nu0 + n) * (n + 1);
        const T* rn0 = sH + hb + (-nu0 + n) * (n + 1);
        const T* rp1 = two ? rp0 + (n + 1) : rp0;
        const T* rn1 = two ? rn0 - (n + 1) : rn0;
        const T2* xr = X + (size_t)cidx(n, -n) * TC + t0;
        for (int m = n; m > 0; m--, xr += TC) {
          const T h0 = rn0[m], h1 = rn1[m];
          T2 xv[4];
          load_cols(xr, xv);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 x = xv[k];
            a0[k].x += h0 * x.x; a0[k].y += h0 * x.y;
            a1[k].x += h1 * x.x; a1[k].y += h1 * x.y;
          }
        }
        for (int m = 0; m <= n; m++, xr += TC) {
          const T h0 = rp0[m], h1 = rp1[m];
          T2 xv[4];
          load_cols(xr, xv);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 x = xv[k];
            a0[k].x += h0 * x.x; a0[k].y += h0 * x.y;
            a1[k].x += h1 * x.x; a1[k].y += h1 * x.y;
          }
        }
        for (int r = 0; r < (two ? 2 : 1); r++) {
          const int nu = nu0 + r, an = nu < 0 ? -nu : nu;
          const T er = sech[2 * an], ei = nu < 0 ? sech[2 * an + 1] : -sech[2 * an + 1];
          T2* ar = A + (size_t)cidx(n, nu) * TC;
          if (full) {
            T2 cur[4];
            load_cols(ar + t0, cur);
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const T2 o = cmul(r ? a1[k] : a0[k], er, ei);
              cur[k].x += o.x; cur[k].y += o.y;
            }
            store_cols(ar + t0, cur);
            continue;
          }
#pragma unroll
          for (int k = 0; k < 4; k++) {
            if (t0 + k >= cnt) break;
            const T2 o = cmul(r ? a1[k] : a0[k], er, ei);
            T2& a = ar[smap[t0 + k]];
            a.x += o.x; a.y += o.y;
          }
        }
      } else {
        for (int m = 0; m <= n; m++) {
          const T2* xr = X + (size_t)hidx(n, m) * TC + t0;
          T p0, m0, p1 = T(0), m1 = T(0);
          p0 = sH[hb + (nu0 + n) * (n + 1) + m];
          m0 = sH[hb + (-nu0 + n) * (n + 1) + m];
          if (two) {
            p1 = sH[hb + (nu0 + 1 + n) * (n + 1) + m];
            m1 = sH[hb + (-nu0 - 1 + n) * (n + 1) + m];
          }
          if (m == 0) { m0 = T(0); m1 = T(0); }
          T2 xv[4];
          load_cols(xr, xv);
#pragma unroll
          for (int k = 0; k < 4; k++) {
            const T2 x = xv[k];
            a0[k].x += (p0 + m0) * x.x; a0[k].y += (p0 - m0) * x.y;
            a1[k].x += (p1 + m1) * x.x; a1[k].y += (p1 - m1) * x.y;
          }
        }
        for (int r = 0; r < (two ? 2 : 1); r++) {
          const int nu = nu0 + r;
          const T er = sech[2 * nu], ei = sech[2 * nu + 1];
          T2* ar = A + (size_t)hidx(n, nu) * TC;
          if (full) {
            T2 cur[4];
            load_cols(ar + t0, cur);
#pragma unroll
            for (int k = 0; k < 4; k++) {
              const T2 a = r ? a1[k] : a0[k];
              cur[k].x += er * a.x + ei * a.y;
              if (nu != 0) cur[k].y += er * a.y - ei * a.x;
            }
            store_cols(ar + t0, cur);
            continue;
          }
#pragma unroll
          for (int k = 0; k < 4; k++) {
            if (t0 + k >= cnt) break;
            const T2 a = r ? a1[k] : a0[k];
            T2& o = ar[smap[t0 + k]];
            o.x += er * a.x + ei * a.y;
            if (nu != 0) o.y += er * a.y - ei * a.x;
          }
        }
      }
    }
  }
  __syncthreads();
  // results: add into the level array, or the split partials
  const int nc = (P + 1) * (P + 1);
  for (int i = tid; i < V * TC; i += kTileThreads) {
    const int c = i / TC, tt = i - c * TC;
    if (!s_act[tt]) continue;
    const int64_t plin = s_act[tt] - 1;
    T2 a = A[i];
    if (HELM && p.helm_e) {
      const int n = s_nm[c] & 255;
      a.x = scale2(a.x, p.helm_e * n);
      a.y = scale2(a.y, p.helm_e * n);
    }
    if (p.nsplit > 1) {
      ((T2*)p.partial_raw)[(((int64_t)split * 8 + tau) * V + c) * np + plin] = a;
      continue;
    }
    const int px = (int)(plin % nx), py = (int)((plin / nx) % nx), pz = (int)(plin / ((int64_t)nx * nx));
    const int64_t g0 = compact_box(p.gmap, (int64_t)morton(px, py, pz) << 3);
    if (g0 < 0) continue;   // (targets lie in stored groups)
    const int64_t b = g0 | tau;
    if (HELM) {
      const int64_t o = layout_off(b, c, nc);
      p.cout[2 * o] += a.x;
      p.cout[2 * o + 1] += a.y;
    } else {
      const int n = s_nm[c] & 255, m = (s_nm[c] >> 8) - 64;
      if (m == 0) {
        p.cout[layout_off(b, n * n, nc)] += a.x;
      } else {
        const int id = lidx(n, m);
        p.cout[layout_off(b, id, nc)] += a.x;
        p.cout[layout_off(b, id + 1, nc)] += a.y;
      }
    }
  }
}

}  // namespace

template <typename T, bool HELM>
bool tiles_supported(int Ns, int Nr) {
  return Ns == Nr && Ns >= 2 && Ns <= 60 && pick_tc<T, HELM>(Ns, false).tc > 0;
}

template <typename T, bool HELM>
int launch_m2l_tiles(const LanesParams<T>& p, const OpTables<T>& t,
                     cudaStream_t s) {
  {
    int rc = ensure_tile_offsets();
    if (rc) return rc;
  }
  const bool sparse = p.pmap != nullptr;
  const TileChoice c = pick_tc<T, HELM>(p.N, sparse);
  const int TC = c.tc;
  if (!TC) return set_error(-3, "M2L tiles: expansion order too large for shared memory");
  if (c.dense && !p.hcx) return set_error(-3, "M2L tiles: coaxial rows of the level missing");
  const TilePlan q = tile_plan<T, HELM>(p.N, TC, c.dense, sparse);
  WBFMM_SMEM(q.total, k_m2l_tiles<T, HELM>);
  const int64_t np = (int64_t)1 << (3 * (p.level - 1));
  dim3 grid((unsigned)(8 * ((np + TC - 1) / TC)), 1, p.nsplit);
  k_m2l_tiles<T, HELM><<<grid, kTileThreads, q.total, s>>>(p, t, TC, c.dense);
  WBFMM_CUDA(cudaGetLastError());
  if (p.nsplit > 1) return launch_lanes_reduce<T, HELM>(p, s);
  return 0;
}

template <typename T>
int build_helm_coax_rows(const T* raw, int64_t raw_stride, int P, T* out, cudaStream_t s) {
  k_helm_coax_rows<T><<<dim3(15, P + 1), 128, 0, s>>>(raw, raw_stride, P, out);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}
template int build_helm_coax_rows<float>(const float*, int64_t, int, float*, cudaStream_t);
template int build_helm_coax_rows<double>(const double*, int64_t, int, double*, cudaStream_t);
size_t helm_coax_rows_count(int P) { return (size_t)15 * 4 * coax_rows(P); }

template <typename T, bool HELM>
int tiles_per_cta(int N, bool* dense, bool sparse) {
  const TileChoice c = pick_tc<T, HELM>(N, sparse);
  if (dense) *dense = c.dense;
  return c.tc;
}

#define WBFMM_TILES_INST(T, H)                                                   \
  template bool tiles_supported<T, H>(int, int);                                 \
  template int launch_m2l_tiles<T, H>(const LanesParams<T>&, const OpTables<T>&, \
                                      cudaStream_t);                             \
  template int tiles_per_cta<T, H>(int, bool*, bool);
WBFMM_TILES_INST(double, true)
WBFMM_TILES_INST(double, false)
WBFMM_TILES_INST(float, true)
WBFMM_TILES_INST(float, false)

}  // namespace wbfmm
