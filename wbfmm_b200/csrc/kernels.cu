// FMM pass kernels: P2M, M2M, M2L, L2L, L2P and P2P.
//
//  P2M  one warp per leaf box; lanes take the box's sources 32 at a time and
//       every coefficient contribution is reduced across the warp in a fixed
//       order (deterministic), accumulating in shared memory.
//  M2M  one CTA per parent; warps take the eight children.
//  M2L  one CTA per target box (optionally split over several CTAs); warps
//       take the list-4 sources (src/indexing.c:330-377) and run the
//       rotate / coaxial / rotate-back sequence in shared memory,
//       accumulating per warp; the warps' partial sums are added in a
//       fixed order.
//  L2L  one CTA per parent; one warp per child.
//  L2P  one thread per target.
//  P2P  one warp per leaf box holding targets; lanes take the flattened
//       sources of the 27 neighbour boxes (src/indexing.c:250-286).
#include <cuda_runtime.h>

#include <type_traits>

#include "engine.h"
#include "expand.cuh"
#include "kernels.h"
#include "translate.cuh"

namespace wbfmm {

// |d|^2 of the 15 list-4 distances (src/shift.c:709-723), device copy
__constant__ int c_list_dist2[15] = {4, 5, 6, 8, 9, 10, 11, 12, 13, 14,
                                     17, 18, 19, 22, 27};

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sums over the warp of several values at once, by transposing while
// reducing: after the exchanges across lanes 16 (and 8) apart, each half
// (quarter) of the warp carries one value, whose sum the remaining steps
// form.  Two values: lanes 0-15 hold the sum of a, 16-31 of b (5 shuffles
// instead of 10); four: lanes 0-7, 8-15, 16-23, 24-31 hold those of a, b,
// c, d (6 shuffles instead of 20).
template <typename T>
__device__ __forceinline__ T warp_sum2(T a, T b, int lane) {
  const bool hi = lane & 16;
  T w = (hi ? b : a) + __shfl_xor_sync(0xffffffffu, hi ? a : b, 16);
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
  return w;
}
template <typename T>
__device__ __forceinline__ T warp_sum4(T a, T b, T c, T d, int lane) {
  const bool hi = lane & 16, q = lane & 8;
  const T u = (hi ? c : a) + __shfl_xor_sync(0xffffffffu, hi ? a : c, 16);
  const T v = (hi ? d : b) + __shfl_xor_sync(0xffffffffu, hi ? b : d, 16);
  T w = (q ? v : u) + __shfl_xor_sync(0xffffffffu, q ? u : v, 8);
#pragma unroll
  for (int o = 4; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
  return w;
}

// the P2M kernel's emitters: each emission summed over the warp's points
// (one per lane) into the warp's accumulator in shared memory; pairs of
// emissions reduced together (warp_sum2 / warp_sum4), their sums added by
// one lane of each half / quarter
template <typename T>
struct P2MEmitHelm {
  T* acc;
  int lane;
  __device__ __forceinline__ void operator()(int idx, T re, T im) const {
    re = warp_sum(re); im = warp_sum(im);
    if (lane == 0) { acc[2 * idx] += re; acc[2 * idx + 1] += im; }
  }
  __device__ __forceinline__ void pair(int i1, T r1, T m1, int i2, T r2, T m2) const {
    const T w = warp_sum4(r1, m1, r2, m2, lane);
    if ((lane & 7) == 0) acc[2 * ((lane & 16) ? i2 : i1) + ((lane & 8) ? 1 : 0)] += w;
  }
};
template <typename T>
struct P2MEmitLap {
  T* acc;
  int lane;
  __device__ __forceinline__ void operator()(int idx, T v) const {
    v = warp_sum(v);
    if (lane == 0) acc[idx] += v;
  }
  __device__ __forceinline__ void pair(int i1, T v1, int i2, T v2) const {
    const T w = warp_sum2(v1, v2, lane);
    if ((lane & 15) == 0) acc[(lane & 16) ? i2 : i1] += w;
  }
};

// box centre exactly as wbfmm_tree_box_centre (src/util.c:290-330)
__device__ __forceinline__ void box_centre(int64_t b, double x0, double y0,
                                           double z0, double wb, double* c) {
  uint32_t i, j, k;
  demorton((uint64_t)b, &i, &j, &k);
  c[0] = x0 + wb * i; c[1] = y0 + wb * j; c[2] = z0 + wb * k;
  c[0] += 0.5 * wb; c[1] += 0.5 * wb; c[2] += 0.5 * wb;
}

// ------------------------------------------------------------------- P2M
// shared-memory bytes of the Legendre constants of degrees <= N + 2
// (LegTab), or 0 where they would take more than 40 KB (then computed)
template <typename T>
static size_t leg_table_bytes(int N) {
  const size_t b = 4 * sizeof(T) * (size_t)(N + 3) * (N + 3);
  return b <= 40 * 1024 ? b : 0;
}

// shared-memory bytes of the per-thread recursion rows (expand.cuh) of a
// CTA of `threads` threads
template <typename T>
static size_t p2m_row_bytes(int N, int threads) {
  return sizeof(T) * (size_t)p2m_rows() * (N + kRowPad) * threads;
}
template <typename T>
static size_t l2p_row_bytes(int N, bool helm, bool grad, int threads) {
  return sizeof(T) * (size_t)l2p_rows(helm, grad) * (N + kRowPad) * threads;
}
// rows in shared memory up to this many bytes per CTA; above it (high
// orders, FP64) the rows stay in per-thread local arrays, where occupancy
// is worth more than the shorter latency
constexpr size_t kRowSmemMax = 48 * 1024;
constexpr int kL2PBoxes = 4;     // leaf boxes whose expansions an L2P CTA stages
constexpr int kFixedOrder = 14;   // P2M / L2P order with a compile-time instantiation
#define WBFMM_TRY_K(call)          \
  do {                             \
    const int rc_ = (call);        \
    if (rc_) return rc_;           \
  } while (0)

// SROWS: recursion rows in shared memory (else per-thread local arrays);
// NC > 0: the expansion order fixed at compile time (p.N == NC), the rows
// in a per-thread array whose every index the unrolled recursion knows, so
// that they stay in registers
template <typename T, bool HELM, bool SROWS, int NC = 0>
__global__ void k_p2m(P2MParams<T> p, int legt) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  // Legendre recursion constants of degrees <= N + 2, once per CTA
  const int LW = (NC > 0 ? NC : p.N) + 3;
  T* lt = (T*)smraw;
  if (legt) {
    leg_table_fill(lt, LW - 1, threadIdx.x, blockDim.x);
    __syncthreads();
  }
  // the box's storage index, and (sparse storage) its Morton index
  const int64_t cb = (int64_t)blockIdx.x * nw + warp;
  if (cb >= p.nbox) return;   // whole warp leaves; no block barriers below
  const int64_t b = p.glist ? (((int64_t)p.glist[cb >> 3] << 3) | (cb & 7)) : cb;
  const int N = NC > 0 ? NC : p.N;
  const int nc = ncoef(N);
  const int w = HELM ? 2 : 1;
  const int RL = N + kRowPad;
  T* rows = (T*)smraw + (legt ? 4 * LW * LW : 0);
  T loc[NC > 0 ? 2 * (NC + kRowPad) : (SROWS ? 1 : 2 * kPtMax)];
  const Scratch<T> sc = SROWS && NC == 0 ? Scratch<T>{rows + threadIdx.x, RL, (int)blockDim.x}
                                         : Scratch<T>{loc, RL, 1};
  T* acc = rows + (SROWS && NC == 0 ? p2m_rows() * RL * blockDim.x : 0) + (size_t)warp * nc * w;
  for (int c = lane; c < nc * w; c += 32) acc[c] = T(0);
  __syncwarp();
  const uint32_t cnt = p.box_n[b], start = p.box_i[b];
  if (cnt > 0) {
    double cd[3];
    box_centre(b, p.x0, p.y0, p.z0, p.wb, cd);
    // source position relative to the box centre, formed in FP64
    const T xc[3] = {T(0), T(0), T(0)};
    for (uint32_t base = 0; base < cnt; base += 32) {
      const uint32_t t = base + lane;
      const bool act = t < cnt;
      const uint32_t s = start + (act ? t : 0);
      T xs[3] = {act ? (T)(p.x[s] - cd[0]) : T(0),
                 act ? (T)(p.y[s] - cd[1]) : T(0),
                 act ? (T)(p.z[s] - cd[2]) : T(0)};
      auto expand = [&](const auto& leg) {
        if (HELM) {
          const P2MEmitHelm<T> emit{acc, lane};
          if (p.q) {
            T qr = act ? p.q[2 * s] : T(0), qi = act ? p.q[2 * s + 1] : T(0);
            p2m_helmholtz<T>(N, p.k, xc, xs, qr, qi, emit, leg, sc);
          }
          if (p.dip) {
            T dr = act ? p.dip[2 * s] : T(0), di = act ? p.dip[2 * s + 1] : T(0);
            T nrm[3] = {act ? p.nx[s] : T(0), act ? p.ny[s] : T(0),
                        act ? p.nz[s] : T(1)};
            p2m_helmholtz_dipole<T>(N, p.k, xc, xs, nrm, dr, di, emit, leg, sc);
          }
        } else {
          const P2MEmitLap<T> emit{acc, lane};
          if (p.q) {
            T qv = act ? p.q[s] : T(0);
            p2m_laplace<T>(N, xc, xs, qv, emit, leg, sc);
          }
          if (p.dip) {
            T dv = act ? p.dip[s] : T(0);
            T nrm[3] = {act ? p.nx[s] : T(0), act ? p.ny[s] : T(0),
                        act ? p.nz[s] : T(1)};
            p2m_laplace_dipole<T>(N, xc, xs, nrm, dv, emit, leg, sc);
          }
        }
      };
      if (legt) expand(LegTab<T>{lt, LW});
      else expand(LegDirect<T>());
    }
  }
  __syncwarp();
  for (int c = lane; c < nc; c += 32) {
    int64_t o = layout_off(cb, c, nc);
    if (HELM) {
      if (p.accumulate) {
        p.mps[2 * o] += acc[2 * c];
        p.mps[2 * o + 1] += acc[2 * c + 1];
      } else {
        p.mps[2 * o] = acc[2 * c];
        p.mps[2 * o + 1] = acc[2 * c + 1];
      }
    } else {
      if (p.accumulate) p.mps[o] += acc[c]; else p.mps[o] = acc[c];
    }
  }
}

template <typename T, bool HELM>
int launch_p2m(const P2MParams<T>& p, cudaStream_t s) {
  if (p.nbox <= 0) return 0;
  const int nw = 4;
  const size_t leg = leg_table_bytes<T>(p.N);
  const size_t rows = p2m_row_bytes<T>(p.N, nw * 32);
  const bool srows = rows <= kRowSmemMax;
  size_t smem = leg + (srows ? rows : 0) + sizeof(T) * (size_t)nw * ncoef(p.N) * (HELM ? 2 : 1);
  unsigned grid = (unsigned)((p.nbox + nw - 1) / nw);
  // the serving orders' leaf expansions: rows in registers (not for FP64
  // Helmholtz, whose unrolled recursion exceeds the register file)
  constexpr bool kFixedOk = !(HELM && sizeof(T) == 8);
  if (kFixedOk && p.N == kFixedOrder) {
    if constexpr (kFixedOk) {
      const size_t sm = leg + sizeof(T) * (size_t)nw * ncoef(p.N) * (HELM ? 2 : 1);
      if (sm > 48 * 1024) WBFMM_SMEM(sm, k_p2m<T, HELM, false, kFixedOrder>);
      k_p2m<T, HELM, false, kFixedOrder><<<grid, nw * 32, sm, s>>>(p, leg ? 1 : 0);
    }
  } else if (srows) {
    if (smem > 48 * 1024) WBFMM_SMEM(smem, k_p2m<T, HELM, true>);
    k_p2m<T, HELM, true><<<grid, nw * 32, smem, s>>>(p, leg ? 1 : 0);
  } else {
    if (smem > 48 * 1024) WBFMM_SMEM(smem, k_p2m<T, HELM, false>);
    k_p2m<T, HELM, false><<<grid, nw * 32, smem, s>>>(p, leg ? 1 : 0);
  }
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

// ----------------------------------------------------- translation core
// vector length (complex entries) for order N
template <bool HELM>
__host__ __device__ __forceinline__ int vlen(int N) {
  return HELM ? (N + 1) * (N + 1) : nhalf(N);
}

// load a Layout-L box vector into a shared complex vector
template <typename T, bool HELM>
__device__ __forceinline__ void load_vec(T* v, const T* arr, int64_t b, int N,
                                         int nc, int lane) {
  if (HELM) {
    for (int c = lane; c < (N + 1) * (N + 1); c += 32) {
      int64_t o = layout_off(b, c, nc);
      v[2 * c] = arr[2 * o]; v[2 * c + 1] = arr[2 * o + 1];
    }
  } else {
    for (int c = lane; c < nhalf(N); c += 32) {
      int n = half_degree(c), m = c - n * (n + 1) / 2;
      if (m == 0) {
        v[2 * c] = arr[layout_off(b, n * n, nc)];
        v[2 * c + 1] = T(0);
      } else {
        int id = lidx(n, m);
        v[2 * c] = arr[layout_off(b, id, nc)];
        v[2 * c + 1] = arr[layout_off(b, id + 1, nc)];
      }
    }
  }
}

// out[b] (+)= v  (Layout L), all lanes of the caller cooperate
template <typename T, bool HELM, bool ACC>
__device__ __forceinline__ void store_vec(T* arr, int64_t b, int N, int nc,
                                          const T* v, int tid, int nt) {
  if (HELM) {
    for (int c = tid; c < (N + 1) * (N + 1); c += nt) {
      int64_t o = layout_off(b, c, nc);
      if (ACC) { arr[2 * o] += v[2 * c]; arr[2 * o + 1] += v[2 * c + 1]; }
      else { arr[2 * o] = v[2 * c]; arr[2 * o + 1] = v[2 * c + 1]; }
    }
  } else {
    for (int c = tid; c < nhalf(N); c += nt) {
      int n = half_degree(c), m = c - n * (n + 1) / 2;
      if (m == 0) {
        int64_t o = layout_off(b, n * n, nc);
        if (ACC) arr[o] += v[2 * c]; else arr[o] = v[2 * c];
      } else {
        int id = lidx(n, m);
        int64_t o0 = layout_off(b, id, nc), o1 = layout_off(b, id + 1, nc);
        if (ACC) { arr[o0] += v[2 * c]; arr[o1] += v[2 * c + 1]; }
        else { arr[o0] = v[2 * c]; arr[o1] = v[2 * c + 1]; }
      }
    }
  }
}

// A holds the input vector (order Nin).  Runs rotate -> coaxial -> rotate
// back for shift operator `op`; result added to (ACC) or written into out.
// kind: Laplace coaxial kind (0 S|R, 1 S|S, 2 R|R); Helmholtz: CPLX table
// for M2L (S|R), real for M2M/L2L.
template <typename T, bool HELM, bool CPLX, bool ACC>
__device__ void shift_vec(T* A, T* B, T* out, int Nin, int Nout, int op,
                          const OpTables<T>& t, const T* coax, const T* tp,
                          int kind, int lane) {
  const T* H = t.H + (int64_t)t.op_ith[op] * t.hstride;
  const T* eph = t.ph + (size_t)op * (t.lmax + 1) * 2;
  const T* ech = t.ch + (size_t)op * (t.lmax + 1) * 2;
  if (HELM) {
    phase_full(A, Nin, ech, lane, 32);
    __syncwarp();
    hsum_full<T, T, false>(B, A, Nin, H, eph, lane, 32);
    __syncwarp();
    coax_full<T, T, CPLX>(A, B, Nout, Nin, coax, lane, 32);
    __syncwarp();
    phase_full(A, Nout, eph, lane, 32);
    __syncwarp();
    hsum_full<T, T, ACC>(out, A, Nout, H, ech, lane, 32);
    __syncwarp();
  } else {
    phase_half(A, Nin, ech, lane, 32);
    __syncwarp();
    hsum_half<T, T, false>(B, A, Nin, H, eph, lane, 32);
    __syncwarp();
    coax_half<T, T>(A, B, Nout, Nin,
                    kind == 0 ? t.lapSR : (kind == 1 ? t.lapSS : t.lapRR),
                    t.lt, tp, kind, lane, 32);
    __syncwarp();
    phase_half(A, Nout, eph, lane, 32);
    __syncwarp();
    hsum_half<T, T, ACC>(out, A, Nout, H, ech, lane, 32);
    __syncwarp();
  }
}

// shared memory per warp: three vectors of the larger order
template <bool HELM>
static size_t warp_smem_bytes(int Nmax, size_t tsize) {
  return tsize * 2 * 3 * (size_t)vlen<HELM>(Nmax);
}

// ------------------------------------------------------------------- M2L
template <typename T, bool HELM>
__global__ void k_m2l(XlateParams<T> p, OpTables<T> t) {
  extern __shared__ unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int Ns = p.Nin, Nr = p.Nout, Lm = Ns > Nr ? Ns : Nr;
  const int V = vlen<HELM>(Lm);
  T* A = (T*)smraw + (size_t)warp * 6 * V;
  T* B = A + 2 * V;
  T* acc = B + 2 * V;
  T* tpow = (T*)smraw + (size_t)nw * 6 * V;   // Laplace: [15][Ns+Nr+2] of (2^e t)^j
  const int tpn = Ns + Nr + 2;
  const int64_t tb = blockIdx.x / p.nsplit;
  const int split = blockIdx.x % p.nsplit;
  const int outlen = vlen<HELM>(Nr);
  for (int c = lane; c < 2 * outlen; c += 32) acc[c] = T(0);
  if (!HELM) {
    for (int di = threadIdx.x; di < 15; di += blockDim.x) {
      // sources enter scaled by 2^(e l) and results leave scaled by
      // 2^(e (n+1)), so S|R / (2^e t)^(n+l+1) stays in range
      T r = scale2(p.width * (T)sqrt((double)c_list_dist2[di]), p.lap_e);
      T* tp = tpow + di * tpn;
      tp[0] = T(1);
      for (int j = 1; j < tpn; j++) tp[j] = r * tp[j - 1];
    }
  }
  __syncthreads();
  const bool active = !(p.tmask && !p.tmask[tb]);
  if (active) {
    uint32_t i, j, k;
    demorton((uint64_t)tb, &i, &j, &k);
    const int nside = 1 << p.level;
    int i0 = (int)(i - i % 2), j0 = (int)(j - j % 2), k0 = (int)(k - k % 2);
    int i1 = min(i0 + 3, nside - 1), j1 = min(j0 + 3, nside - 1),
        k1 = min(k0 + 3, nside - 1);
    if (i0 > 0) i0 -= 2;
    if (j0 > 0) j0 -= 2;
    if (k0 > 0) k0 -= 2;
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1, nk = k1 - k0 + 1;
    const int total = ni * nj * nk;
    const int ncs = ncoef(Ns);
    for (int e = split * nw + warp; e < total; e += p.nsplit * nw) {
      int ii = i0 + e / (nj * nk), jj = j0 + (e / nk) % nj, kk = k0 + e % nk;
      int dx = ii - (int)i, dy = jj - (int)j, dz = kk - (int)k;
      if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1)
        continue;
      uint64_t s = morton((uint32_t)ii, (uint32_t)jj, (uint32_t)kk);
      if (p.src_n && p.src_n[s] == 0) continue;
      const int op = (dx + 3) * 49 + (dy + 3) * 7 + dz + 3;
      const int di = t.op_dist[op];
      load_vec<T, HELM>(A, p.cin, (int64_t)s, Ns, ncs, lane);
      if (!HELM) {
        for (int c = lane; c < nhalf(Ns); c += 32) {
          const int n = half_degree(c);
          A[2 * c] = scale2(A[2 * c], p.lap_e * n);
          A[2 * c + 1] = scale2(A[2 * c + 1], p.lap_e * n);
        }
      }
      __syncwarp();
      shift_vec<T, HELM, true, true>(A, B, acc, Ns, Nr, op, t,
                                     HELM ? p.coax + di * p.coax_stride : nullptr,
                                     HELM ? nullptr : tpow + di * tpn, 0, lane);
    }
  }
  __syncthreads();
  // fixed-order sum of the warps' partial results
  const T* acc0 = (T*)smraw + 4 * V;
  const int ncr = ncoef(Nr);
  if (p.nsplit == 1) {
    if (!active) return;
    T* red = A;   // reuse warp 0's first vector as the reduction buffer
    __syncthreads();
    for (int c = threadIdx.x; c < 2 * outlen; c += blockDim.x) {
      T v = acc0[c];
      for (int w = 1; w < nw; w++) v += acc0[(size_t)w * 6 * V + c];
      if (!HELM) v = scale2(v, p.lap_e * (half_degree(c >> 1) + 1));
      ((T*)smraw)[c] = v;
    }
    __syncthreads();
    store_vec<T, HELM, true>(p.cout, tb, Nr, ncr, (T*)smraw, threadIdx.x,
                             blockDim.x);
    (void)red;
  } else {
    T* part = p.partial + ((size_t)split * p.nbox + tb) * 2 * outlen;
    for (int c = threadIdx.x; c < 2 * outlen; c += blockDim.x) {
      T v = acc0[c];
      for (int w = 1; w < nw; w++) v += acc0[(size_t)w * 6 * V + c];
      if (!HELM) v = scale2(v, p.lap_e * (half_degree(c >> 1) + 1));
      part[c] = v;
    }
  }
}

// adds the split partial sums, in split order, into cout
template <typename T, bool HELM>
__global__ void k_m2l_reduce(XlateParams<T> p) {
  const int64_t tb = blockIdx.x;
  if (p.tmask && !p.tmask[tb]) return;
  extern __shared__ unsigned char smraw[];
  T* v = (T*)smraw;
  const int Nr = p.Nout, outlen = vlen<HELM>(Nr);
  for (int c = threadIdx.x; c < 2 * outlen; c += blockDim.x) {
    T s = T(0);
    for (int sp = 0; sp < p.nsplit; sp++)
      s += p.partial[((size_t)sp * p.nbox + tb) * 2 * outlen + c];
    v[c] = s;
  }
  __syncthreads();
  store_vec<T, HELM, true>(p.cout, tb, Nr, ncoef(Nr), v, threadIdx.x,
                           blockDim.x);
}

static int pick_warps(size_t per_warp, size_t extra, int want) {
  const size_t cap = 200 * 1024;
  int nw = want;
  while (nw > 1 && per_warp * nw + extra > cap) nw--;
  return nw;
}

template <typename T, bool HELM>
int launch_m2l(const XlateParams<T>& p, const OpTables<T>& t, cudaStream_t s) {
  const int Lm = p.Nin > p.Nout ? p.Nin : p.Nout;
  const size_t per = warp_smem_bytes<HELM>(Lm, sizeof(T));
  const size_t extra = HELM ? 0 : sizeof(T) * 15 * (p.Nin + p.Nout + 2);
  const int nw = pick_warps(per, extra, 4);
  const size_t smem = per * nw + extra;
  if (smem > 227 * 1024) return set_error(-3, "M2L: expansion order too large for shared memory");
  WBFMM_SMEM(smem, k_m2l<T, HELM>);
  unsigned grid = (unsigned)(p.nbox * p.nsplit);
  k_m2l<T, HELM><<<grid, nw * 32, smem, s>>>(p, t);
  WBFMM_CUDA(cudaGetLastError());
  if (p.nsplit > 1) {
    size_t rs = sizeof(T) * 2 * vlen<HELM>(p.Nout);
    if (rs > 48 * 1024)
      WBFMM_SMEM(rs, k_m2l_reduce<T, HELM>);
    k_m2l_reduce<T, HELM><<<(unsigned)p.nbox, 256, rs, s>>>(p);
    WBFMM_CUDA(cudaGetLastError());
  }
  return 0;
}

// ------------------------------------------------------------------- M2M
// parents at `level-1` receive the shifted expansions of their children at
// `level`; p.nbox = number of parents, p.width = child box width
template <typename T, bool HELM>
__global__ void k_m2m(XlateParams<T> p, OpTables<T> t) {
  extern __shared__ unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int Nc = p.Nin, Np = p.Nout, Lm = Nc > Np ? Nc : Np;
  const int V = vlen<HELM>(Lm);
  T* A = (T*)smraw + (size_t)warp * 6 * V;
  T* B = A + 2 * V;
  T* acc = B + 2 * V;
  T* tp = (T*)smraw + (size_t)nw * 6 * V;
  const int tpn = Nc + Np + 2;
  // the children's group (dense: the parent box); the parent's storage index
  const int64_t P = blockIdx.x;
  const int64_t Pout = p.glist ? compact_box(p.gmap, (int64_t)p.glist[P]) : P;
  if (Pout < 0) return;   // (a stored group's parent is stored) whole CTA, before any barrier
  const int outlen = vlen<HELM>(Np);
  for (int c = lane; c < 2 * outlen; c += 32) acc[c] = T(0);
  if (!HELM && threadIdx.x == 0) {
    T r = p.width * (T)t.op_r[kOpM2M];
    tp[0] = T(1);
    for (int j = 1; j < tpn; j++) tp[j] = r * tp[j - 1];
  }
  __syncthreads();
  const int ncc = ncoef(Nc);
  for (int ch = warp; ch < 8; ch += nw) {
    int64_t c = 8 * P + ch;
    load_vec<T, HELM>(A, p.cin, c, Nc, ncc, lane);
    __syncwarp();
    shift_vec<T, HELM, false, true>(A, B, acc, Nc, Np, kOpM2M + ch, t, p.coax,
                                    tp, 1, lane);
  }
  __syncthreads();
  const T* acc0 = (T*)smraw + 4 * V;
  T* red = (T*)smraw;
  for (int c = threadIdx.x; c < 2 * outlen; c += blockDim.x) {
    T v = acc0[c];
    for (int w = 1; w < nw; w++) v += acc0[(size_t)w * 6 * V + c];
    red[c] = v;   // entries c of warp 0's A are read only by this thread
  }
  __syncthreads();
  store_vec<T, HELM, false>(p.cout, Pout, Np, ncoef(Np), red, threadIdx.x,
                            blockDim.x);
}

template <typename T, bool HELM>
int launch_m2m(const XlateParams<T>& p, const OpTables<T>& t, cudaStream_t s) {
  const int Lm = p.Nin > p.Nout ? p.Nin : p.Nout;
  const size_t per = warp_smem_bytes<HELM>(Lm, sizeof(T));
  const size_t extra = sizeof(T) * (p.Nin + p.Nout + 2);
  const int nw = pick_warps(per, extra, 8);
  const size_t smem = per * nw + extra;
  if (smem > 227 * 1024) return set_error(-3, "M2M: expansion order too large for shared memory");
  WBFMM_SMEM(smem, k_m2m<T, HELM>);
  k_m2m<T, HELM><<<(unsigned)p.nbox, nw * 32, smem, s>>>(p, t);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------------- L2L
// children at `level+1` receive (overwrite) the shifted expansion of their
// parent at `level`; p.nbox = number of parents, p.width = child width
template <typename T, bool HELM>
__global__ void k_l2l(XlateParams<T> p, OpTables<T> t) {
  extern __shared__ unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = blockDim.x >> 5;
  const int Np = p.Nin, Nc = p.Nout, Lm = Nc > Np ? Nc : Np;
  const int V = vlen<HELM>(Lm);
  T* A = (T*)smraw + (size_t)warp * 6 * V;
  T* B = A + 2 * V;
  T* out = B + 2 * V;
  T* tp = (T*)smraw + (size_t)nw * 6 * V;
  const int tpn = Nc + Np + 2;
  // the children's group (dense: the parent box); the parent's storage index
  const int64_t P = blockIdx.x;
  const int64_t Pin = p.glist ? compact_box(p.gmap, (int64_t)p.glist[P]) : P;
  if (Pin < 0) return;    // (a stored group's parent is stored) whole CTA, before any barrier
  if (!HELM && threadIdx.x == 0) {
    T r = p.width * (T)t.op_r[kOpL2L];
    tp[0] = T(1);
    for (int j = 1; j < tpn; j++) tp[j] = r * tp[j - 1];
  }
  __syncthreads();
  const int ncp = ncoef(Np), ncc = ncoef(Nc);
  for (int ch = warp; ch < 8; ch += nw) {
    load_vec<T, HELM>(A, p.cin, Pin, Np, ncp, lane);
    __syncwarp();
    shift_vec<T, HELM, false, false>(A, B, out, Np, Nc, kOpL2L + ch, t, p.coax,
                                     tp, 2, lane);
    store_vec<T, HELM, false>(p.cout, 8 * P + ch, Nc, ncc, out, lane, 32);
    __syncwarp();
  }
}

template <typename T, bool HELM>
int launch_l2l(const XlateParams<T>& p, const OpTables<T>& t, cudaStream_t s) {
  const int Lm = p.Nin > p.Nout ? p.Nin : p.Nout;
  const size_t per = warp_smem_bytes<HELM>(Lm, sizeof(T));
  const size_t extra = sizeof(T) * (p.Nin + p.Nout + 2);
  const int nw = pick_warps(per, extra, 8);
  const size_t smem = per * nw + extra;
  if (smem > 227 * 1024) return set_error(-3, "L2L: expansion order too large for shared memory");
  WBFMM_SMEM(smem, k_l2l<T, HELM>);
  k_l2l<T, HELM><<<(unsigned)p.nbox, nw * 32, smem, s>>>(p, t);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------------- L2P
// recursion constants of the L2P gradients from shared-memory tables filled
// once per CTA (rows n = -1..N+1, columns m + M0)
template <typename T>
struct RecTab {
  const T* ta;   // rec_a(n, m): row n + 1, column m
  const T* tb;   // rec_b(n, m): row n, column m + M0
  int W, M0;
  __device__ T a(int n, int m) const { return ta[(n + 1) * W + (m < 0 ? -m : m)]; }
  __device__ T b(int n, int m) const { return tb[n * W + m + M0]; }
};
template <typename T>
struct LapRecTab {
  const T* t;    // (am, a0, ap) at ((n (N+1) + m) * 3
  int N1;
  __device__ void c(int n, int m, T* am, T* a0, T* ap) const {
    const T* e = t + (n * N1 + m) * 3;
    *am = e[0]; *a0 = e[1]; *ap = e[2];
  }
};

// shared-memory bytes of the L2P tables at order N (0: computed on the fly)
template <typename T, bool HELM>
__host__ __device__ inline size_t l2p_table_bytes(int N) {
  const size_t b = HELM ? 2 * (size_t)(N + 3) * (2 * N + 3) * sizeof(T)
                        : 3 * (size_t)(N + 1) * (N + 1) * sizeof(T);
  return b <= 40 * 1024 ? b : 0;
}

// one thread per target (sorted by box); potential and gradient in one sweep
// SROWS: recursion rows in shared memory, after the tables (else
// per-thread local arrays)
// stage: the CTA's leaf expansions copied to shared memory when its targets
// fall in at most kL2PBoxes leaf boxes (targets are sorted by box)
// NC > 0: the expansion order fixed at compile time (p.N == NC), the rows
// in a per-thread array whose every index the unrolled recursion knows
template <typename T, bool HELM, bool SROWS, bool STAGE, int NC = 0>
__global__ void k_l2p(EvalParams<T> p, int tab, int legt) {
  const int stage = STAGE ? 1 : 0;
  extern __shared__ __align__(16) unsigned char l2p_sm[];
  __shared__ unsigned s_bal[32];
  __shared__ int64_t s_box[kL2PBoxes];
  T* st = (T*)l2p_sm;
  const int N = NC > 0 ? NC : p.N;
  const int W = 2 * N + 3, M0 = N + 1;
  // Legendre constants (degrees <= N + 2) after the recursion tables
  const int LW = N + 3;
  T* lt = st + (tab ? l2p_table_bytes<T, HELM>(N) / sizeof(T) : 0);
  T* rows = lt + (legt ? 4 * LW * LW : 0);
  constexpr bool SR = SROWS && NC == 0;
  T* cst = rows + (SR ? (size_t)l2p_rows(HELM, p.grad != nullptr) * (N + kRowPad) * blockDim.x : 0);
  T loc[NC > 0 ? 3 * (NC + kRowPad) : (SROWS ? 1 : 3 * kPtMax)];
  const Scratch<T> sc = SR ? Scratch<T>{rows + threadIdx.x, N + kRowPad, (int)blockDim.x}
                           : Scratch<T>{loc, N + kRowPad, 1};
  if (legt) leg_table_fill(lt, N + 2, threadIdx.x, blockDim.x);
  if (tab) {
    if (HELM) {
      T* ta = st;
      T* tb = st + (N + 3) * W;
      for (int i = threadIdx.x; i < (N + 3) * W; i += blockDim.x) {
        const int row = i / W, col = i - row * W;
        ta[i] = rec_a<T>(row - 1, col);
        tb[i] = rec_b<T>(row, col - M0);
      }
    } else {
      const int N1 = N + 1;
      for (int i = threadIdx.x; i < N1 * N1; i += blockDim.x) {
        const int n = i / N1, m = i - n * N1;
        T* e = st + 3 * i;
        if (n >= 1 && m <= n) LapRecDirect<T>().c(n, m, &e[0], &e[1], &e[2]);
        else e[0] = e[1] = e[2] = T(0);
      }
    }
  }
  const int jt = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = ncoef(N), wc = HELM ? 2 : 1;
  int slot = -1;
  if (stage) {
    const int j0 = blockIdx.x * blockDim.x;
    const bool in = jt < p.ntgt;
    const bool first = in && (jt == j0 || p.tbox[jt] != p.tbox[jt - 1]);
    const int nb = __syncthreads_count(first);
    if (nb <= kL2PBoxes) {
      const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
      const unsigned bal = __ballot_sync(0xffffffffu, first);
      if (lane == 0) s_bal[warp] = bal;
      __syncthreads();
      int before = __popc(bal & ((1u << lane) - 1u));
      for (int w = 0; w < warp; w++) before += __popc(s_bal[w]);
      slot = before + (first ? 1 : 0) - 1;
      if (first) s_box[slot] = compact_box(p.gmap, (int64_t)p.tbox[jt]);
      __syncthreads();
      for (int i = threadIdx.x; i < nb * nc; i += blockDim.x) {
        const int k = i / nc, c = i - k * nc;
        if (s_box[k] < 0) {   // (targets lie in stored groups)
          for (int u = 0; u < wc; u++) cst[(size_t)i * wc + u] = T(0);
          continue;
        }
        const int64_t o = layout_off(s_box[k], c, nc);
        for (int u = 0; u < wc; u++) cst[(size_t)i * wc + u] = p.mpr[wc * o + u];
      }
      if (!in) slot = -1;
    }
  }
  if (tab || legt || stage) __syncthreads();
  if (jt >= p.ntgt) return;
  const int64_t b = p.tbox[jt];
  const int64_t cb = compact_box(p.gmap, b);   // storage index
  if (cb < 0) return;   // (targets lie in stored groups) no barriers below
  double cd[3];
  box_centre(b, p.x0, p.y0, p.z0, p.wb, cd);
  // target position relative to the box centre, formed in FP64
  const T xc[3] = {T(0), T(0), T(0)};
  const T xf[3] = {(T)(p.tx[jt] - cd[0]), (T)(p.ty[jt] - cd[1]),
                   (T)(p.tz[jt] - cd[2])};
  const uint32_t o = p.tperm[jt];
  // the staged copy, or (a CTA whose targets span more boxes) null
  const T* mine = STAGE && slot >= 0 ? cst + (size_t)slot * nc * wc : nullptr;
  if (HELM) {
    auto coef = [&](int idx, T* re, T* im) {
      if (STAGE && mine) { *re = mine[2 * idx]; *im = mine[2 * idx + 1]; return; }
      int64_t off = layout_off(cb, idx, nc);
      *re = p.mpr[2 * off]; *im = p.mpr[2 * off + 1];
    };
    auto eval = [&](const auto& leg) {
      if (p.grad) {
        T g[6] = {T(0), T(0), T(0), T(0), T(0), T(0)}, f[2] = {T(0), T(0)};
        T* fp = p.pot ? f : nullptr;
        if (tab) {
          RecTab<T> rt{st, st + (N + 3) * W, W, M0};
          l2p_helmholtz_grad<T>(N, p.k, xc, xf, coef, g, fp, rt, leg, sc);
        } else {
          l2p_helmholtz_grad<T>(N, p.k, xc, xf, coef, g, fp, RecDirect<T>(), leg, sc);
        }
        for (int c = 0; c < 6; c++) p.grad[6 * (size_t)o + c] = g[c];
        if (p.pot) { p.pot[2 * (size_t)o] = f[0]; p.pot[2 * (size_t)o + 1] = f[1]; }
      } else if (p.pot) {
        T fr = T(0), fi = T(0);
        l2p_helmholtz<T>(N, p.k, xc, xf, coef, &fr, &fi, leg, sc);
        p.pot[2 * (size_t)o] = fr; p.pot[2 * (size_t)o + 1] = fi;
      }
    };
    if (legt) eval(LegTab<T>{lt, LW}); else eval(LegDirect<T>());
  } else {
    auto coef = [&](int idx) -> T {
      return STAGE && mine ? mine[idx] : p.mpr[layout_off(cb, idx, nc)];
    };
    auto eval = [&](const auto& leg) {
      if (p.grad) {
        T g[3] = {T(0), T(0), T(0)}, f = T(0);
        T* fp = p.pot ? &f : nullptr;
        if (tab) {
          LapRecTab<T> rt{st, N + 1};
          l2p_laplace_grad<T>(N, xc, xf, coef, g, fp, rt, leg, sc);
        } else {
          l2p_laplace_grad<T>(N, xc, xf, coef, g, fp, LapRecDirect<T>(), leg, sc);
        }
        for (int c = 0; c < 3; c++) p.grad[3 * (size_t)o + c] = g[c];
        if (p.pot) p.pot[o] = f;
      } else if (p.pot) {
        p.pot[o] = l2p_laplace<T>(N, xc, xf, coef, leg, sc);
      }
    };
    if (legt) eval(LegTab<T>{lt, LW}); else eval(LegDirect<T>());
  }
}

template <typename T, bool HELM>
int launch_l2p(const EvalParams<T>& p, cudaStream_t s) {
  if (p.ntgt <= 0) return 0;
  const size_t sm = l2p_table_bytes<T, HELM>(p.N);
  const size_t lg = leg_table_bytes<T>(p.N);
  const size_t rows = l2p_row_bytes<T>(p.N, HELM, p.grad != nullptr, 128);
  const unsigned grid = (unsigned)((p.ntgt + 127) / 128);
  // staged leaf expansions: up to kL2PBoxes per CTA within 32 KB
  const size_t cb = (size_t)kL2PBoxes * ncoef(p.N) * (HELM ? 2 : 1) * sizeof(T);
  const int stage = cb <= 32 * 1024 ? 1 : 0;
  auto go = [&](auto srows, auto stg) -> int {
    constexpr bool SR = decltype(srows)::value, ST = decltype(stg)::value;
    const size_t bytes = sm + lg + (SR ? rows : 0) + (ST ? cb : 0);
    if (bytes > 48 * 1024) WBFMM_SMEM(bytes, k_l2p<T, HELM, SR, ST>);
    k_l2p<T, HELM, SR, ST><<<grid, 128, bytes, s>>>(p, sm ? 1 : 0, lg ? 1 : 0);
    return 0;
  };
  // the serving orders' Laplace leaf evaluation: rows in registers (the
  // Helmholtz one, unrolled, needs 170-255 registers and runs slower)
  constexpr bool kFixedOk = !HELM;
  if (kFixedOk && p.N == kFixedOrder) {
    if constexpr (kFixedOk) {
      auto fixed = [&](auto stg) -> int {
        constexpr bool ST = decltype(stg)::value;
        const size_t bytes = sm + lg + (ST ? cb : 0);
        if (bytes > 48 * 1024) WBFMM_SMEM(bytes, k_l2p<T, HELM, false, ST, kFixedOrder>);
        k_l2p<T, HELM, false, ST, kFixedOrder><<<grid, 128, bytes, s>>>(p, sm ? 1 : 0, lg ? 1 : 0);
        return 0;
      };
      WBFMM_TRY_K(stage ? fixed(std::true_type()) : fixed(std::false_type()));
    }
  } else if (rows <= kRowSmemMax) {
    WBFMM_TRY_K(stage ? go(std::true_type(), std::true_type()) : go(std::true_type(), std::false_type()));
  } else {
    WBFMM_TRY_K(stage ? go(std::false_type(), std::true_type()) : go(std::false_type(), std::false_type()));
  }
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

// ------------------------------------------------------------------- P2P
// One CTA per target leaf box.  The sources of the 27 neighbour boxes (a
// virtual list, box by box) are staged through shared memory in tiles of NT
// (the CTA's thread count: 128, or 32 for trees whose leaves hold a few
// points each, so that more boxes are resident per SM).  The box's targets
// are taken NT at a time, the m of a pass spread over all NT threads (NT/m
// or NT/m + 1 consecutive threads per target, so that no thread idles
// whatever m is): thread gl of a target's g takes tile entries gl, gl + g,
// ..., accumulating in FP64 registers in a fixed order, and the target's
// first thread adds its threads' sums in thread order.  The FP32
// form computes pair terms in FP32 from separations that keep FP64 accuracy
// (coordinates as float pairs hi + lo, the hi parts of neighbouring points
// subtracting exactly), sums each run of 8 of a thread's terms in FP32 and
// adds that into the FP64 sums.  Pair kernels and the r > 1e-6 cutoff follow
// src/local.c:32-262 and src/local-laplace.c:400-523, 1091-1227.
constexpr int kP2PRun = 8;     // FP32 terms summed before each FP64 add

template <typename T, bool HELM, int NT>
struct P2PTile {
  double x[NT], y[NT], z[NT];   // FP32 form: float hi[NT], lo[NT] in each
  T q[NT * (HELM ? 2 : 1)];
  T d[NT * (HELM ? 2 : 1)];
  T nx[NT], ny[NT], nz[NT];
};

// sin and cos of x >= 0 in FP32 for the near field: x = n pi/2 + r with
// |r| <= pi/4 by the two-constant reduction of Cody and Waite (FMA), the
// Taylor series of sin r to r^9 and of cos r to r^10 (truncation below 2e-9
// at |r| = pi/4), then the quadrant's swap and signs.  A few ulp for x up to
// about 1e4; the near field's k r stays far below that.
__device__ __forceinline__ void sincos_near(float x, float* sp, float* cp) {
  const float q = rintf(x * 0.636619772367581343f);            // 2/pi
  float r = fmaf(-q, 1.57079637050628662109375f, x);          // fl(pi/2)
  r = fmaf(-q, -4.37113900018624283e-8f, r);                  // pi/2 - fl(pi/2)
  const float r2 = r * r;
  float ps = fmaf(r2, 2.75573192239858907e-6f, -1.98412698412698413e-4f);
  ps = fmaf(r2, ps, 8.33333333333333333e-3f);
  ps = fmaf(r2, ps, -1.66666666666666667e-1f);
  const float sn = fmaf(r * r2, ps, r);
  float pc = fmaf(r2, -2.75573192239858907e-7f, 2.48015873015873016e-5f);
  pc = fmaf(r2, pc, -1.38888888888888889e-3f);
  pc = fmaf(r2, pc, 4.16666666666666667e-2f);
  pc = fmaf(r2, pc, -0.5f);
  const float cn = fmaf(r2, pc, 1.0f);
  const int n = (int)q;
  float so = (n & 1) ? cn : sn, co = (n & 1) ? sn : cn;
  if (n & 2) so = -so;
  if ((n + 1) & 2) co = -co;
  *sp = so;
  *cp = co;
}

// The terms of one (target, source) pair at separation r = (rx, ry, rz)
// (|r|^2 = r2) added to acc[0..] (Helmholtz: pot re, im, then grad x re,
// x im, y, z; Laplace: pot, grad x, y, z), without the kernels' constant
// factors, which the caller applies once per target (p2p_scale): 1/(4 pi)
// on the potential, -k/(4 pi) (Helmholtz) and 1/(4 pi) (Laplace) on the
// gradient.
// MASKED: a pair within the cutoff (r2 <= rc2) takes 1/r = 0, which makes
// each of its terms an exact zero, instead of being branched around (the
// pairs of a run then interleave without divergence)
// 1/sqrt(x) of a pair: in FP32 the MUFU approximation alone
// (rsqrt.approx.ftz: no subnormal handling, which a squared distance above
// the cutoff, at least 1e-12, never needs; for such normal arguments it is
// the approximation rsqrtf returns)
__device__ __forceinline__ float pair_rsqrt(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ double pair_rsqrt(double x) { return rsqrt(x); }

template <typename T, bool HELM, int NT, bool want_pot, bool want_grad, bool MASKED = false>
__device__ __forceinline__ void p2p_pair(const P2PTile<T, HELM, NT>& tl, int j, T rx, T ry, T rz,
                                         T r2, T k, T kinv, bool hd, T* acc, T rc2 = T(0)) {
  const T ir = MASKED ? (r2 > rc2 ? pair_rsqrt(r2) : T(0)) : pair_rsqrt(r2);
  if (HELM) {
    const T r = r2 * ir;
    T kr = k * r, ikr, sn, cs;
    if constexpr (sizeof(T) == 4) {
      ikr = ir * kinv;
      sincos_near(kr, &sn, &cs);
    } else {
      ikr = ir / k;
      sincos(kr, &sn, &cs);
    }
    // h0 = e^{ikr} / (i k r), h1 = h0 / (i k r) - ... (the first-order
    // spherical Hankel function), so that grad h0(kr) = -k h1 r / r
    const T h0r = sn * ikr, h0i = -cs * ikr;
    const T h1r = fma(h0r, ikr, h0i), h1i = fma(h0i, ikr, -h0r);
    const T qr = tl.q[2 * j], qi = tl.q[2 * j + 1];
    if (want_pot) {
      acc[0] = fma(h0r, qr, fma(-h0i, qi, acc[0]));
      acc[1] = fma(h0i, qr, fma(h0r, qi, acc[1]));
      if (hd) {
        const T nr = (rx * tl.nx[j] + ry * tl.ny[j] + rz * tl.nz[j]) * ir;
        const T dr = tl.d[2 * j] * nr, di = tl.d[2 * j + 1] * nr;
        acc[0] -= k * (h1r * dr - h1i * di);
        acc[1] -= k * (h1r * di + h1i * dr);
      }
    }
    if (want_grad) {
      const T ar = (h1r * qr - h1i * qi) * ir, ai = (h1r * qi + h1i * qr) * ir;
      acc[2] = fma(ar, rx, acc[2]); acc[3] = fma(ai, rx, acc[3]);
      acc[4] = fma(ar, ry, acc[4]); acc[5] = fma(ai, ry, acc[5]);
      acc[6] = fma(ar, rz, acc[6]); acc[7] = fma(ai, rz, acc[7]);
      if (hd) {
        const T nxs = tl.nx[j], nys = tl.ny[j], nzs = tl.nz[j];
        const T nr = rx * nxs + ry * nys + rz * nzs;
        const T dpr = h0r - T(2) * h1r * ikr, dpi = h0i - T(2) * h1i * ikr;
        const T dr = tl.d[2 * j], di = tl.d[2 * j + 1];
        const T rv[3] = {rx, ry, rz}, nv[3] = {nxs, nys, nzs};
        const T ir2 = ir * ir;
        for (int c = 0; c < 3; c++) {
          T ur = dpr * k * nr * rv[c] * ir2 + h1r * (nv[c] * ir - nr * rv[c] * ir2 * ir);
          T ui = dpi * k * nr * rv[c] * ir2 + h1i * (nv[c] * ir - nr * rv[c] * ir2 * ir);
          acc[2 + 2 * c] += ur * dr - ui * di;
          acc[3 + 2 * c] += ur * di + ui * dr;
        }
      }
    }
  } else {
    const T q = tl.q[j];
    const T ir2 = ir * ir;
    if (want_pot) {
      T v = q;
      if (hd) v += tl.d[j] * (rx * tl.nx[j] + ry * tl.ny[j] + rz * tl.nz[j]) * ir2;
      acc[0] = fma(v, ir, acc[0]);
    }
    if (want_grad) {
      const T ir3 = ir * ir2;
      const T gq = -q * ir3;
      acc[1] = fma(gq, rx, acc[1]); acc[2] = fma(gq, ry, acc[2]); acc[3] = fma(gq, rz, acc[3]);
      if (hd) {
        const T nxs = tl.nx[j], nys = tl.ny[j], nzs = tl.nz[j];
        const T nr = rx * nxs + ry * nys + rz * nzs;
        const T ad = tl.d[j] * ir3;
        acc[1] += ad * (nxs - T(3) * nr * rx * ir2);
        acc[2] += ad * (nys - T(3) * nr * ry * ir2);
        acc[3] += ad * (nzs - T(3) * nr * rz * ir2);
      }
    }
  }
}

// the constant factor of accumulator c of p2p_pair (see there)
template <bool HELM>
__device__ __forceinline__ double p2p_scale(int c, double k) {
  const double f4pi = 0.25 / kPi;
  return HELM ? (c < 2 ? f4pi : -k * f4pi) : f4pi;
}

// POT / GRAD: the fields computed, fixed at compile time (dipoles at run time).
// 128-thread CTAs are held to 4 (Helmholtz) / 5 (Laplace) resident per SM:
// with the masked runs the compiler's own choice took 149 registers; the
// caps measured best (FP32 Helmholtz pot+grad evaluation of 2e5 points:
// 1.152 ms before the masking, 1.130 ms masked, 1.046 ms with 4 CTAs, 1.093
// with 5; Laplace 0.615 / 0.564 / 0.566 / 0.544 ms)
// DIP: dipole sources (p.dip set), fixed at compile time so that the
// monopole kernels carry no dipole code (a smaller loop body: fewer
// instruction-fetch stalls)
template <typename T, bool HELM, int NT, bool POT, bool GRAD, bool DIP>
__global__ void __launch_bounds__(NT, NT == 32 ? 20 : (HELM ? 4 : 5))
k_p2p(EvalParams<T> p) {
  constexpr bool F32 = sizeof(T) == 4;
  constexpr int NA = HELM ? 8 : 4;
  __shared__ P2PTile<T, HELM, NT> tl;
  __shared__ uint32_t s_st[27], s_pref[28];
  __shared__ double s_red[NA][NT];     // each lane's sums, for its target's group
  const int64_t b = blockIdx.x;
  const uint32_t tc = p.tcount[b];
  if (tc == 0) return;
  const int tid = threadIdx.x;
  if (tid < 32) {
    uint32_t bi, bj, bk;
    demorton((uint64_t)b, &bi, &bj, &bk);
    const int nside = 1 << p.level;
    uint32_t cnt = 0, st = 0;
    if (tid < 27) {
      int ii = (int)bi + tid / 9 - 1, jj = (int)bj + (tid / 3) % 3 - 1,
          kk = (int)bk + tid % 3 - 1;
      if (ii >= 0 && jj >= 0 && kk >= 0 && ii < nside && jj < nside && kk < nside) {
        uint64_t nb = morton((uint32_t)ii, (uint32_t)jj, (uint32_t)kk);
        cnt = p.box_n[nb];
        st = p.box_i[nb];
      }
    }
    uint32_t incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
      if (tid >= o) incl += v;
    }
    if (tid < 27) { s_st[tid] = st; s_pref[tid] = incl - cnt; }
    if (tid == 26) s_pref[27] = incl;
  }
  __syncthreads();
  const uint32_t total = s_pref[27];
  if (total == 0) return;   // no sources near: the whole CTA, before any other barrier
  const T rc2 = T(kCutoffRadius * kCutoffRadius);
  const T k = p.k;
  const T kinv = HELM ? T(1) / k : T(0);
  const bool hq = p.q != nullptr;
  constexpr bool hd = DIP, want_pot = POT, want_grad = GRAD;
  // FP32 form: source coordinates as float pairs (hi, lo) in the FP64 arrays' bytes
  float2* xp = (float2*)tl.x;
  float2* yp = (float2*)tl.y;
  float2* zp = (float2*)tl.z;
  // Each pass takes m = min(NT, targets left) targets and spreads them over
  // all NT lanes: NT / m lanes per target, one more for the first
  // NT mod m targets, the lanes of a target consecutive; lane gl of a
  // target's g lanes takes tile entries gl, gl + g, ... (every lane busy
  // whatever the box's target count)
  for (uint32_t t0 = 0; t0 < tc; t0 += NT) {
    const int m = (int)min((uint32_t)NT, tc - t0);
    const int glo = NT / m, extra = NT - glo * m, split = extra * (glo + 1);
    const int ti = tid < split ? tid / (glo + 1) : extra + (tid - split) / glo;
    const int g = tid < split ? glo + 1 : glo;
    const int gl = tid < split ? tid % (glo + 1) : (tid - split) % glo;
    const uint32_t jt = p.tstart[b] + t0 + ti;
    const double x = p.tx[jt], y = p.ty[jt], z = p.tz[jt];
    const float txh = (float)x, tyh = (float)y, tzh = (float)z;
    const float txl = (float)(x - (double)txh), tyl = (float)(y - (double)tyh),
                tzl = (float)(z - (double)tzh);
    double a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (uint32_t f0 = 0; f0 < total; f0 += NT) {
      const uint32_t f = f0 + tid;
      __syncthreads();
      if (f < total) {
        int l = 0;
        while (l < 26 && s_pref[l + 1] <= f) l++;
        const uint32_t s = s_st[l] + (f - s_pref[l]);
        const double sx = p.x[s], sy = p.y[s], sz = p.z[s];
        if constexpr (F32) {
          const float hx = (float)sx, hy = (float)sy, hz = (float)sz;
          xp[tid] = make_float2(hx, (float)(sx - (double)hx));
          yp[tid] = make_float2(hy, (float)(sy - (double)hy));
          zp[tid] = make_float2(hz, (float)(sz - (double)hz));
        } else {
          tl.x[tid] = sx; tl.y[tid] = sy; tl.z[tid] = sz;
        }
        if (HELM) {
          tl.q[2 * tid] = hq ? p.q[2 * s] : T(0);
          tl.q[2 * tid + 1] = hq ? p.q[2 * s + 1] : T(0);
          if (hd) { tl.d[2 * tid] = p.dip[2 * s]; tl.d[2 * tid + 1] = p.dip[2 * s + 1]; }
        } else {
          tl.q[tid] = hq ? p.q[s] : T(0);
          if (hd) tl.d[tid] = p.dip[s];
        }
        if (hd) { tl.nx[tid] = p.nx[s]; tl.ny[tid] = p.ny[s]; tl.nz[tid] = p.nz[s]; }
      }
      __syncthreads();
      const int nt = (int)min((uint32_t)NT, total - f0);
      if constexpr (F32) {
        // runs of kP2PRun pairs: a full run without bounds checks, the
        // tile's last run with them; the cutoff by masking (p2p_pair)
        auto pair_at = [&](int j, T* acc) {
          const float2 cx = xp[j], cy = yp[j], cz = zp[j];
          const T rx = (T)((txh - cx.x) + (txl - cx.y));
          const T ry = (T)((tyh - cy.x) + (tyl - cy.y));
          const T rz = (T)((tzh - cz.x) + (tzl - cz.y));
          const T r2 = rx * rx + ry * ry + rz * rz;
          p2p_pair<T, HELM, NT, POT, GRAD, true>(tl, j, rx, ry, rz, r2, k, kinv, hd, acc, rc2);
        };
        for (int j0 = gl; j0 < nt; j0 += kP2PRun * g) {
          T acc[NA];
          for (int c = 0; c < NA; c++) acc[c] = T(0);
          if (j0 + (kP2PRun - 1) * g < nt) {
#pragma unroll
            for (int u = 0; u < kP2PRun; u++) pair_at(j0 + u * g, acc);
          } else {
#pragma unroll
            for (int u = 0; u < kP2PRun; u++)
              if (j0 + u * g < nt) pair_at(j0 + u * g, acc);
          }
          for (int c = 0; c < NA; c++) a[c] += (double)acc[c];
        }
      } else {
        for (int j = gl; j < nt; j += g) {
          // separation formed in FP64, the rest in T
          const T rx = (T)(x - tl.x[j]), ry = (T)(y - tl.y[j]), rz = (T)(z - tl.z[j]);
          const T r2 = rx * rx + ry * ry + rz * rz;
          if (!(r2 > rc2)) continue;
          T acc[NA];
          for (int c = 0; c < NA; c++) acc[c] = T(0);
          p2p_pair<T, HELM, NT, POT, GRAD>(tl, j, rx, ry, rz, r2, k, kinv, hd, acc);
          for (int c = 0; c < NA; c++) a[c] += (double)acc[c];
        }
      }
    }
    // the sums of a target's lanes, in lane order, by its first lane (the
    // next pass writes s_red only after its first tile barrier)
    for (int c = 0; c < NA; c++) s_red[c][tid] = a[c];
    __syncthreads();
    if (gl != 0) continue;
    double v[8];
    for (int c = 0; c < NA; c++) {
      double sum = s_red[c][tid];
      for (int i = 1; i < g; i++) sum += s_red[c][tid + i];
      v[c] = sum * p2p_scale<HELM>(c, (double)p.k);
    }
    const uint32_t o = p.tperm[jt];
    if (HELM) {
      if (want_pot) {
        p.pot[2 * (size_t)o] = (T)((double)p.pot[2 * (size_t)o] + v[0]);
        p.pot[2 * (size_t)o + 1] = (T)((double)p.pot[2 * (size_t)o + 1] + v[1]);
      }
      if (want_grad)
        for (int c = 0; c < 6; c++)
          p.grad[6 * (size_t)o + c] = (T)((double)p.grad[6 * (size_t)o + c] + v[2 + c]);
    } else {
      if (want_pot) p.pot[o] = (T)((double)p.pot[o] + v[0]);
      if (want_grad)
        for (int c = 0; c < 3; c++)
          p.grad[3 * (size_t)o + c] = (T)((double)p.grad[3 * (size_t)o + c] + v[1 + c]);
    }
  }
}

template <typename T, bool HELM>
int launch_p2p(const EvalParams<T>& p, cudaStream_t s) {
  if (p.nbox <= 0 || p.ntgt <= 0) return 0;
  auto go = [&](auto pot, auto grad, auto dip) {
    constexpr bool P = decltype(pot)::value, G = decltype(grad)::value;
    constexpr bool D = decltype(dip)::value;
    if (p.ntgt <= 8 * p.nbox)   // a few targets per leaf on average
      k_p2p<T, HELM, 32, P, G, D><<<(unsigned)p.nbox, 32, 0, s>>>(p);
    else
      k_p2p<T, HELM, 128, P, G, D><<<(unsigned)p.nbox, 128, 0, s>>>(p);
  };
  auto fields = [&](auto dip) {
    if (p.pot && p.grad) go(std::true_type(), std::true_type(), dip);
    else if (p.pot) go(std::true_type(), std::false_type(), dip);
    else if (p.grad) go(std::false_type(), std::true_type(), dip);
  };
  if (p.dip) fields(std::true_type());
  else fields(std::false_type());
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

// dst[i] = (float)src[i]; dst[i] += src[i] (FP64 solvers' FP32 near field)
__global__ void k_narrow(const double* __restrict__ src, float* __restrict__ dst, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = (float)src[i];
}
__global__ void k_add_widened(double* __restrict__ dst, const float* __restrict__ src, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] += (double)src[i];
}
int launch_narrow(const double* src, float* dst, int64_t n, cudaStream_t s) {
  if (n <= 0) return 0;
  k_narrow<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}
int launch_add_widened(double* dst, const float* src, int64_t n, cudaStream_t s) {
  if (n <= 0) return 0;
  k_add_widened<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(dst, src, n);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

// largest |sin| and |cos| errors of sincos_near and of sincosf against the
// FP64 values at the same FP32 arguments x_i = i * xmax / n (one block;
// err[0] ours, err[1] sincosf)
__global__ void k_sincos_check(double xmax, int n, double* err) {
  __shared__ double m[2][256];
  double e0 = 0, e1 = 0;
  for (int i = threadIdx.x; i <= n; i += blockDim.x) {
    const float x = (float)(xmax * i / n);
    float s, c, s1, c1;
    sincos_near(x, &s, &c);
    sincosf(x, &s1, &c1);
    const double sd = sin((double)x), cd = cos((double)x);
    e0 = fmax(e0, fmax(fabs(s - sd), fabs(c - cd)));
    e1 = fmax(e1, fmax(fabs(s1 - sd), fabs(c1 - cd)));
  }
  m[0][threadIdx.x] = e0; m[1][threadIdx.x] = e1;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int t = 1; t < blockDim.x; t++) { e0 = fmax(e0, m[0][t]); e1 = fmax(e1, m[1][t]); }
    err[0] = e0; err[1] = e1;
  }
}

int sincos_near_errors(double xmax, int n, double* host_err) {
  double* d = nullptr;
  WBFMM_CUDA(cudaMalloc(&d, 2 * sizeof(double)));
  k_sincos_check<<<1, 256>>>(xmax, n, d);
  cudaError_t e = cudaMemcpy(host_err, d, 2 * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(d);
  WBFMM_CUDA(e);
  return 0;
}

// ------------------------------------------------------ instantiations
#define WBFMM_INST(T, H)                                                      \
  template int launch_p2m<T, H>(const P2MParams<T>&, cudaStream_t);          \
  template int launch_m2m<T, H>(const XlateParams<T>&, const OpTables<T>&,   \
                                cudaStream_t);                               \
  template int launch_m2l<T, H>(const XlateParams<T>&, const OpTables<T>&,   \
                                cudaStream_t);                               \
  template int launch_l2l<T, H>(const XlateParams<T>&, const OpTables<T>&,   \
                                cudaStream_t);                               \
  template int launch_l2p<T, H>(const EvalParams<T>&, cudaStream_t);         \
  template int launch_p2p<T, H>(const EvalParams<T>&, cudaStream_t);
WBFMM_INST(double, true)
WBFMM_INST(double, false)
WBFMM_INST(float, true)
WBFMM_INST(float, false)

}  // namespace wbfmm
