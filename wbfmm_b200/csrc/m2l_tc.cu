// Laplace M2L on the tensor cores (tcgen05, FP32 form).
//
// The rotate / coaxial / rotate-back shift of the reference's Laplace M2L
// (src/pass-laplace.c:35-360: wbfmm_laplace_rotate_H, the scaled S|R
// coaxial translation, rotate back) is, for one shift code, a fixed linear
// map of the C = (p+1)^2 real-packed coefficients of the source box to those
// of the target box.  With box width w, degree l of the source and n of the
// target, it factors as
//
//   L_n = w^-(n+1) sum_l That_op[n, l] (w^-l M_l),
//
// where That_op, the shift at unit box width (distance |d| in box widths),
// depends only on the order and the shift code.  So the M2L of a level is,
// per target child type, a dense matrix product summed over the type's 189
// offsets:  L(C x targets) += sum_o That_o (C x C) . M_shift_o (C x targets).
//
// That_o is built once per order on the GPU in FP64 (the engine's
// warp-cooperative shift applied to unit vectors), split into TF32 hi + lo
// parts and stored in the tensor core's shared-memory layout.  The product
// runs as tcgen05.mma kind::tf32 with the FP32 accumulator in tensor memory:
// 3xTF32 (A_hi B_hi + A_hi B_lo + A_lo B_hi, both parts rounded to TF32)
// keeps FP32 accuracy.  One CTA
// takes up to 128 target boxes of one child type; its 128 threads stage the
// shifted source vectors (split into hi / lo) while the tensor core works
// on the previous stage, the operator tiles arrive by bulk copy, and one
// thread issues the MMAs.  Every wait is bounded: a wait that runs out sets
// an error flag and the kernel drains and returns.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <map>
#include <mutex>

#include "../../include/wbfmm_b200.h"
#include "engine.h"
#include "kernels.h"
#include "m2l_lanes.h"
#include "m2l_tc.h"
#include "table_cache.h"
#include "translate.cuh"

namespace wbfmm {

namespace {

// ------------------------------------------------------ layout constants
constexpr int kTcRows = 128;                 // MMA M (rows of one tile)
constexpr int kTcN = 128;                    // MMA N (target boxes per CTA)
constexpr int kTcThreads = 128;
constexpr int kTcStageK = 2;                 // k-steps (8 K each) per stage
constexpr int kTcStages = 4;
constexpr int kTileBytes = kTcRows * 8 * 4;  // one 128 x 8 TF32 tile: 4 KB

// byte offset of element (row r, k) in a 128 x 8 K-major tile without
// swizzle: 8-row x 16-byte core matrices, K-adjacent ones 128 bytes apart
// (leading-dimension offset), row groups 256 bytes apart (stride offset)
__host__ __device__ inline int tile_off(int r, int k) {
  return (r >> 3) * 256 + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4;
}

// ---------------------------------------------------------------- PTX
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// shared-memory matrix descriptor (tcgen05): K-major, no swizzle
__device__ __forceinline__ uint64_t mat_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((128u >> 4) & 0x3FFF) << 16;    // leading-dimension byte offset
  d |= (uint64_t)((256u >> 4) & 0x3FFF) << 32;    // stride-dimension byte offset
  d |= (uint64_t)1 << 46;                         // descriptor version
  return d;
}

// instruction descriptor: D F32, A and B TF32, both K-major, M x N
__host__ __device__ constexpr uint32_t tf32_idesc(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               ::"r"(smem_u32(bar)));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes));
}

// waits for the phase of the given parity to complete, at most `limit`
// polls; 1 when it completed
__device__ __forceinline__ int mbar_wait(uint64_t* bar, uint32_t parity, int limit) {
  uint32_t done = 0;
  for (int it = 0; it < limit && !done; it++) {
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity));
  }
  return (int)done;
}

// global -> shared bulk copy (16-byte aligned, multiple of 16 bytes),
// completing on the barrier's transaction count
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// ------------------------------------------------- dense shift operators
// Column j of That_op: the engine's FP64 Laplace shift (shift_vec: phase,
// forward rotation, scaled S|R at distance |d|, phase, back rotation) of
// the unit real-packed vector e_j, at unit box width.  One warp per (op, j);
// the result is rounded to TF32 hi + lo parts into the operator's tiles.
__global__ void k_lap_tc_ops(OpTables<double> t, int P, int KS, int MT, float* __restrict__ ops,
                             const int* __restrict__ slot) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int C = (P + 1) * (P + 1), V = nhalf(P);
  const int op = blockIdx.y, j = blockIdx.x * (blockDim.x >> 5) + warp;
  if (slot[op] < 0 || j >= C) return;
  double* A = (double*)smraw + (size_t)warp * (6 * V + 2 * P + 4);
  double* B = A + 2 * V;
  double* O = B + 2 * V;
  double* tp = O + 2 * V;
  const int dx = op / 49 - 3, dy = (op / 7) % 7 - 3, dz = op % 7 - 3;
  const double r = sqrt((double)(dx * dx + dy * dy + dz * dz));
  for (int i = lane; i < 2 * V; i += 32) { A[i] = 0.0; O[i] = 0.0; }
  if (lane == 0) {
    tp[0] = 1.0;
    for (int i = 1; i <= 2 * P + 2; i++) tp[i] = tp[i - 1] * r;
    // e_j in the half-vector form: j = n^2 (m = 0), n^2 + 2m - 1 (re), n^2 + 2m (im)
    const int n = (int)sqrt((double)j + 0.5);
    const int q = j - n * n;
    const int m = (q + 1) / 2;
    A[2 * hidx(n, m) + ((q > 0 && (q & 1) == 0) ? 1 : 0)] = 1.0;
  }
  __syncwarp();
  // phase e^{i m ch}, rotate and phase e^{-i nu ph}, scaled S|R, phase
  // e^{i m ph}, rotate back and phase e^{-i nu ch} (translate.cuh)
  const double* H = t.H + (int64_t)t.op_ith[op] * t.hstride;
  const double* eph = t.ph + (size_t)op * (t.lmax + 1) * 2;
  const double* ech = t.ch + (size_t)op * (t.lmax + 1) * 2;
  phase_half(A, P, ech, lane, 32);
  __syncwarp();
  hsum_half<double, double, false>(B, A, P, H, eph, lane, 32);
  __syncwarp();
  coax_half<double, double>(A, B, P, P, t.lapSR, t.lt, tp, 0, lane, 32);
  __syncwarp();
  phase_half(A, P, eph, lane, 32);
  __syncwarp();
  hsum_half<double, double, false>(O, A, P, H, ech, lane, 32);
  __syncwarp();
  float* base = ops + (int64_t)slot[op] * KS * MT * 2 * (kTileBytes / 4);
  for (int row = lane; row < C; row += 32) {
    const int n = (int)sqrt((double)row + 0.5), q = row - n * n, m = (q + 1) / 2;
    const double v = O[2 * hidx(n, m) + ((q > 0 && (q & 1) == 0) ? 1 : 0)];
    // both parts rounded to TF32 (the tensor core would truncate the low
    // bits of an FP32 operand, a bias of up to 2^-21 relative)
    const float hi = __uint_as_float(to_tf32((float)v));
    const float lo = __uint_as_float(to_tf32((float)(v - (double)hi)));
    const int s = j >> 3, kk = j & 7, mt = row / kTcRows, rr = row % kTcRows;
    float* tile = base + ((int64_t)s * MT + mt) * 2 * (kTileBytes / 4);
    tile[tile_off(rr, kk) / 4] = hi;
    tile[kTileBytes / 4 + tile_off(rr, kk) / 4] = lo;
  }
}

// ------------------------------------------------------ source vectors
// lin[sg][pp][s][16]: for each 8-K chunk s of the box's scaled vector
// (w^-n M_k, k real-packed of degree n, zero for k >= C) its TF32 hi parts
// (8) then lo parts (8); zero on the halo
__global__ void k_to_lin_tc(const float* __restrict__ mps, int level, int P, int KS,
                            const LapTcScales sc, float* __restrict__ lin) {
  const int C = (P + 1) * (P + 1);
  const int nx = 1 << (level - 1), npx = nx + 2;
  const int64_t np = (int64_t)nx * nx * nx;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np * 8 * C) return;
  const int k = (int)(e % C);
  const int tau = (int)((e / C) & 7);
  const int64_t Pm = (e / C) >> 3;                // parent Morton index
  uint32_t px, py, pz;
  demorton((uint64_t)Pm, &px, &py, &pz);
  const int64_t pp = (px + 1) + npx * ((int64_t)(py + 1) + npx * (int64_t)(pz + 1));
  const int64_t b = (Pm << 3) | tau;
  const int n = (int)sqrtf((float)k + 0.5f);
  const float v = mps[layout_off(b, k, C)] * sc.in[n];
  const float hi = __uint_as_float(to_tf32(v));
  const float lo = __uint_as_float(to_tf32(v - hi));
  float* row = lin + ((int64_t)tau * (npx * (int64_t)npx * npx) + pp) * KS * 16 + (k >> 3) * 16;
  row[k & 7] = hi;
  row[8 + (k & 7)] = lo;
}

// ----------------------------------------------------------- the GEMM
struct TcSmem {
  // per stage: operator tiles (kTcStageK x MT x {hi, lo} x 4 KB) and the
  // shifted sources (kTcStageK x {hi, lo} x 4 KB); sized for MT = 2
  unsigned char a[kTcStages][kTcStageK * 2 * 2 * kTileBytes];
  unsigned char b[kTcStages][kTcStageK * 2 * kTileBytes];
  uint64_t full[kTcStages];     // operator bulk copies landed
  uint64_t mma[kTcStages];      // the MMAs reading the stage finished
  int ns[kTcStages];            // k-steps in the stage
  uint32_t tmem;
  int pp[kTcN];                 // padded parent index of each target (or -1)
  int plin[kTcN];               // parent linear index of each target
};

constexpr int kWaitLimit = 1 << 22;

__device__ __forceinline__ void cp16(void* dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 16 : 0)
               : "memory");
}

// Accumulators in tensor memory (512 columns): per M tile, the hi*hi
// products (columns mt*128) and, apart, the hi*lo + lo*hi corrections
// (columns 256 + mt*128): the tensor core adds into its FP32 accumulator
// without rounding to nearest, and the corrections (2^-11 of the main
// terms) lose fewer bits summed on their own.  The epilogue adds the two.
__global__ void __launch_bounds__(kTcThreads, 1)
k_m2l_tc(LapTcParams p) {
  extern __shared__ __align__(16) unsigned char tc_smem[];
  TcSmem& sm = *(TcSmem*)(((uintptr_t)tc_smem + 1023) & ~(uintptr_t)1023);
  const int tid = threadIdx.x;
  const int C = (p.P + 1) * (p.P + 1);
  const int KS = p.KS, MT = p.MT;
  const int tau = blockIdx.x & 7, split = blockIdx.z;
  const int nx = 1 << (p.level - 1), npx = nx + 2;
  const int64_t npp = (int64_t)npx * npx * npx;
  const int64_t np = (int64_t)nx * nx * nx;
  const int64_t nlist = p.act ? (int64_t)p.act_n[tau] : np;
  const int64_t base = (int64_t)(blockIdx.x >> 3) * kTcN;
  if (base >= nlist) return;                      // the whole CTA, before any barrier

  // targets of the tile
  {
    const int64_t i = base + tid;
    int pp = -1, pl = -1;
    if (i < nlist) {
      int64_t plin = p.act ? p.act[(int64_t)tau * np + i] : i;
      const int px = (int)(plin % nx), py = (int)((plin / nx) % nx),
                pz = (int)(plin / ((int64_t)nx * nx));
      pp = (px + 1) + npx * ((py + 1) + npx * (pz + 1));
      pl = (int)plin;
    }
    sm.pp[tid] = pp;
    sm.plin[tid] = pl;
  }
  if (tid == 0) {
    for (int s = 0; s < kTcStages; s++) {
      mbar_init(&sm.full[s], 1);
      mbar_init(&sm.mma[s], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  if (tid < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;"
                 ::"r"(smem_u32(&sm.tmem)));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = sm.tmem;
  const uint32_t idesc = tf32_idesc(kTcRows, kTcN);
  const int64_t op_floats = (int64_t)KS * MT * 2 * (kTileBytes / 4);
  const int64_t row_floats = (int64_t)KS * 16;
  int ok = 1;                  // all waits completed
  int gl = 0, gm = 0;          // stages loaded / stages whose MMAs were issued
  bool started = false;        // thread 0: the accumulators hold a product
  int copy_pending = 0, mma_pending = 0;   // thread 0: unwaited operator copy / commit

  // thread 0: the MMAs of stage gm (its operator tiles and sources landed)
  auto issue = [&]() {
    const int buf = gm % kTcStages;
    const uint32_t use = (uint32_t)(gm / kTcStages);
    if (tid == 0 && ok) {
      if (!mbar_wait(&sm.full[buf], use & 1, kWaitLimit)) {
        ok = 0;
      } else {
        copy_pending = 0;
        asm volatile("tcgen05.fence::after_thread_sync;");
        for (int s = 0; s < sm.ns[buf]; s++) {
          const uint32_t bb = smem_u32(sm.b[buf] + s * 2 * kTileBytes);
          for (int mt = 0; mt < MT; mt++) {
            const uint32_t aa = smem_u32(sm.a[buf] + (s * MT + mt) * 2 * kTileBytes);
            const uint32_t dm = tmem + (uint32_t)(mt * kTcN);
            const uint32_t dc = tmem + (uint32_t)(2 * kTcN + mt * kTcN);
            mma_tf32(dm, mat_desc(aa), mat_desc(bb), idesc, started ? 1u : 0u);
            mma_tf32(dc, mat_desc(aa), mat_desc(bb + kTileBytes), idesc, started ? 1u : 0u);
            mma_tf32(dc, mat_desc(aa + kTileBytes), mat_desc(bb), idesc, 1u);
          }
          started = true;
        }
        mma_commit(&sm.mma[buf]);
        mma_pending = 1;
      }
    }
    gm++;
  };

  for (int j = split; j < 189 && ok; j += p.nsplit) {
    const int code = p.offsets[tau * 189 + j];
    const int op = code & 511, sg = (code >> 9) & 7;
    const int ddx = ((code >> 12) & 3) - 1, ddy = ((code >> 14) & 3) - 1,
              ddz = ((code >> 16) & 3) - 1;
    const int64_t doff = ddx + npx * ((int64_t)ddy + npx * (int64_t)ddz);
    // the source box of each target: in the grid (and holding sources, with
    // a source mask); an offset with none in the tile is skipped
    int64_t src = -1;
    if (sm.pp[tid] >= 0) {
      const int64_t pp = sm.pp[tid];
      const int sx = (int)(pp % npx) + ddx, sy = (int)((pp / npx) % npx) + ddy,
                sz = (int)(pp / ((int64_t)npx * npx)) + ddz;
      bool in = sx >= 1 && sx <= nx && sy >= 1 && sy <= nx && sz >= 1 && sz <= nx;
      if (in && p.smask) in = p.smask[(int64_t)sg * npp + pp + doff] != 0;
      if (in) src = ((int64_t)sg * npp + pp + doff) * row_floats;
    }
    if (!__syncthreads_or(src >= 0)) continue;
    const float* A = p.ops + (int64_t)p.slot[op] * op_floats;
    for (int s0 = 0; s0 < KS && ok; s0 += kTcStageK) {
      const int ns = KS - s0 < kTcStageK ? KS - s0 : kTcStageK;
      const int buf = gl % kTcStages;
      const uint32_t use = (uint32_t)(gl / kTcStages);
      // the buffer's previous MMAs must be done before it is overwritten
      if (gl >= kTcStages && !mbar_wait(&sm.mma[buf], (use - 1) & 1, kWaitLimit)) ok = 0;
      ok = __syncthreads_and(ok);
      if (!ok) break;
      if (tid == 0) {
        const uint32_t abytes = (uint32_t)(ns * MT * 2 * kTileBytes);
        sm.ns[buf] = ns;
        mbar_expect_tx(&sm.full[buf], abytes);
        bulk_g2s(sm.a[buf], A + (int64_t)s0 * MT * 2 * (kTileBytes / 4), abytes, &sm.full[buf]);
        copy_pending = 1;
      }
      // this target's source chunks, hi and lo, straight into the tiles
      const float* q = p.lin + (src >= 0 ? src : 0) + (int64_t)s0 * 16;
      for (int s = 0; s < ns; s++) {
        unsigned char* bt = sm.b[buf] + s * 2 * kTileBytes;
        cp16(bt + tile_off(tid, 0), q + s * 16, src >= 0);
        cp16(bt + tile_off(tid, 4), q + s * 16 + 4, src >= 0);
        cp16(bt + kTileBytes + tile_off(tid, 0), q + s * 16 + 8, src >= 0);
        cp16(bt + kTileBytes + tile_off(tid, 4), q + s * 16 + 12, src >= 0);
      }
      asm volatile("cp.async.commit_group;");
      gl++;
      if (gl - gm == kTcStages) {
        // the ring is full: the oldest stage's copies are done once at most
        // kTcStages - 1 groups are pending
        asm volatile("cp.async.wait_group %0;" ::"n"(kTcStages - 1));
        asm volatile("fence.proxy.async.shared::cta;");
        __syncthreads();
        issue();
        ok = __syncthreads_and(ok);
      }
    }
  }
  // the stages still in the ring
  asm volatile("cp.async.wait_all;");
  asm volatile("fence.proxy.async.shared::cta;");
  __syncthreads();
  while (gm < gl && ok) {
    issue();
    ok = __syncthreads_and(ok);
  }
  // the last stage's MMAs (MMAs complete in order)
  if (ok && gl > 0) {
    const int last = (gl - 1) % kTcStages;
    if (!mbar_wait(&sm.mma[last], ((gl - 1) / kTcStages) & 1, kWaitLimit)) ok = 0;
  }
  ok = __syncthreads_and(ok);
  asm volatile("tcgen05.fence::after_thread_sync;");
  const bool started_all = __syncthreads_or(started ? 1 : 0);
  if (!ok) {
    if (tid == 0) {
      atomicExch(p.err, 1);
      // let what this CTA started finish (bounded) before its memory goes
      if (gl > 0) {
        const int last = (gl - 1) % kTcStages;
        const uint32_t u = (uint32_t)((gl - 1) / kTcStages) & 1;
        if (copy_pending) mbar_wait(&sm.full[last], u, kWaitLimit);
        if (mma_pending) mbar_wait(&sm.mma[last], u, kWaitLimit);
      }
    }
  } else if (!started_all) {
    // no offset of this split had sources: its partial sums are zero
    if (p.nsplit > 1)
      for (int row = 0; row < C; row++) {
        const int pl = sm.plin[tid];
        if (pl >= 0) p.partial[(((int64_t)split * 8 + tau) * C + row) * np + pl] = 0.f;
      }
  } else {
    // epilogue: thread = row of an M tile (TMEM lane), columns = targets
    const int warp = tid >> 5;
    for (int mt = 0; mt < MT; mt++) {
      const int row = mt * kTcRows + tid;
      const int n = (int)sqrtf((float)row + 0.5f);
      const float sc = row < C ? p.sc.out[n] : 0.f;
      for (int c0 = 0; c0 < kTcN; c0 += 8) {
        uint32_t r[8], q[8];
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(mt * kTcN + c0);
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                       "=r"(r[6]), "=r"(r[7])
                     : "r"(addr));
        asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=r"(q[0]), "=r"(q[1]), "=r"(q[2]), "=r"(q[3]), "=r"(q[4]), "=r"(q[5]),
                       "=r"(q[6]), "=r"(q[7])
                     : "r"(addr + (uint32_t)(2 * kTcN)));
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        if (row >= C) continue;
        for (int c = 0; c < 8; c++) {
          const int t = c0 + c;
          const int pl = sm.plin[t];
          if (pl < 0) continue;
          const float v = (__uint_as_float(r[c]) + __uint_as_float(q[c])) * sc;
          if (p.nsplit > 1) {
            p.partial[(((int64_t)split * 8 + tau) * C + row) * np + pl] = v;
          } else {
            const int px = pl % nx, py = (pl / nx) % nx, pz = pl / (nx * nx);
            const int64_t b = ((int64_t)morton(px, py, pz) << 3) | tau;
            p.cout[layout_off(b, row, C)] += v;
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (tid < 32)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem));
}

// sum of the split partial results (split order) into the level array
__global__ void k_tc_reduce(LapTcParams p) {
  const int C = (p.P + 1) * (p.P + 1);
  const int nx = 1 << (p.level - 1);
  const int64_t np = (int64_t)nx * nx * nx;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= np * 8 * C) return;
  const int64_t pl = e % np;
  const int row = (int)((e / np) % C);
  const int tau = (int)(e / (np * C));
  const int px = (int)(pl % nx), py = (int)((pl / nx) % nx), pz = (int)(pl / ((int64_t)nx * nx));
  const int64_t b = ((int64_t)morton(px, py, pz) << 3) | tau;
  if (p.tmask && !p.tmask[b]) return;
  float v = 0.f;
  for (int s = 0; s < p.nsplit; s++)
    v += p.partial[(((int64_t)s * 8 + tau) * C + row) * np + pl];
  p.cout[layout_off(b, row, C)] += v;
}

// --------------------------------------------------- operator store
// the dense operators of an order, per device, built once and kept for the
// life of the process
struct TcOps {
  float* ops = nullptr;
  int* slot = nullptr;
  int* offsets = nullptr;
  int KS = 0, MT = 0;
};
std::mutex g_tc_mu;
std::map<std::pair<int, int>, TcOps> g_tc_ops;   // (device, order)
std::map<int, TableCache*> g_tc_tables;          // FP64 geometry per device

}  // namespace

bool tc_lap_supported(int Ns, int Nr) {
  return Ns == Nr && Ns >= 4 && (Ns + 1) * (Ns + 1) <= 2 * kTcRows;
}

size_t tc_lin_bytes(int level, int P) {
  const int64_t npx = (1 << (level - 1)) + 2;
  const int KS = ((P + 1) * (P + 1) + 7) / 8;
  return sizeof(float) * 8 * (size_t)(npx * npx * npx) * KS * 16;
}

// the order's operators, built on first use (FP64 tables, unit width)
int tc_lap_ops(int P, cudaStream_t s, LapTcParams* p) {
  int dev = 0;
  WBFMM_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_tc_mu);
  auto key = std::make_pair(dev, P);
  auto it = g_tc_ops.find(key);
  if (it == g_tc_ops.end()) {
    TableCache*& tc = g_tc_tables[dev];
    if (!tc) tc = new TableCache();
    OpTables<double> t64;
    {
      const int rc = tc->geometry<double>(P + 1, s, &t64);
      if (rc) return rc;
    }
    const int C = (P + 1) * (P + 1);
    TcOps o;
    o.KS = (C + 7) / 8;
    o.MT = (C + kTcRows - 1) / kTcRows;
    int slot[kNumOps], offs[8 * 189], nslot = 0;
    for (int op = 0; op < kNumOps; op++) {
      const int dx = op / 49 - 3, dy = (op / 7) % 7 - 3, dz = op % 7 - 3;
      const bool near = dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && dz >= -1 && dz <= 1;
      slot[op] = op < 343 && !near ? nslot++ : -1;
    }
    build_offset_table(offs);
    const size_t bytes = (size_t)nslot * o.KS * o.MT * 2 * kTileBytes;
    if (cudaMalloc(&o.ops, bytes) != cudaSuccess || cudaMalloc(&o.slot, sizeof(slot)) != cudaSuccess ||
        cudaMalloc(&o.offsets, sizeof(offs)) != cudaSuccess) {
      cudaGetLastError();
      if (o.ops) cudaFree(o.ops);
      if (o.slot) cudaFree(o.slot);
      return set_error(WBFMM_B200_E_NOMEM, "tensor-core M2L operators: allocation failed");
    }
    WBFMM_CUDA(cudaMemsetAsync(o.ops, 0, bytes, s));
    WBFMM_CUDA(cudaMemcpyAsync(o.slot, slot, sizeof(slot), cudaMemcpyHostToDevice, s));
    WBFMM_CUDA(cudaMemcpyAsync(o.offsets, offs, sizeof(offs), cudaMemcpyHostToDevice, s));
    const int V = nhalf(P);
    const int wpb = 4;
    const size_t smem = sizeof(double) * (size_t)wpb * (6 * V + 2 * P + 4);
    if (smem > 48 * 1024) WBFMM_SMEM(smem, k_lap_tc_ops);
    k_lap_tc_ops<<<dim3((C + wpb - 1) / wpb, 343), wpb * 32, smem, s>>>(t64, P, o.KS, o.MT,
                                                                        o.ops, o.slot);
    WBFMM_CUDA(cudaGetLastError());
    // the builds of other streams must see the operators complete
    WBFMM_CUDA(cudaStreamSynchronize(s));
    it = g_tc_ops.emplace(key, o).first;
  }
  p->ops = it->second.ops;
  p->slot = it->second.slot;
  p->offsets = it->second.offsets;
  p->KS = it->second.KS;
  p->MT = it->second.MT;
  return 0;
}

int launch_m2l_tc(LapTcParams p, const float* mps, void* lin, cudaStream_t s) {
  const int C = (p.P + 1) * (p.P + 1);
  p.KP = ((C + 7) / 8) * 8;
  if (p.KS * 8 != p.KP || p.MT > 2) return set_error(WBFMM_B200_E_ORDER, "tensor-core M2L: bad order");
  const int nx = 1 << (p.level - 1), npx = nx + 2;
  const int64_t np = (int64_t)nx * nx * nx;
  WBFMM_CUDA(cudaMemsetAsync(lin, 0, tc_lin_bytes(p.level, p.P), s));
  const int64_t tot = np * 8 * C;
  k_to_lin_tc<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(mps, p.level, p.P, p.KS, p.sc,
                                                            (float*)lin);
  WBFMM_CUDA(cudaGetLastError());
  p.lin = (const float*)lin;
  (void)npx;
  const size_t smem = sizeof(TcSmem) + 1024;
  WBFMM_SMEM(smem, k_m2l_tc);
  dim3 grid((unsigned)(8 * ((np + kTcN - 1) / kTcN)), 1, (unsigned)p.nsplit);
  k_m2l_tc<<<grid, kTcThreads, smem, s>>>(p);
  WBFMM_CUDA(cudaGetLastError());
  if (p.nsplit > 1) {
    k_tc_reduce<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(p);
    WBFMM_CUDA(cudaGetLastError());
  }
  return 0;
}

}  // namespace wbfmm
