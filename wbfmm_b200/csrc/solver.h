#pragma once
// The solver: engine orchestration behind the C ABI of include/wbfmm_b200.h.
//
// A solver owns, on one CUDA stream: the sorted sources and their Morton
// keys, the per-level box ranges, the per-level coefficient arrays in the
// reference's Layout L, the operator tables and the sorted targets.  The
// FP64 instantiation is the plain form; the FP32 instantiation keeps the
// same structure with FP32 coefficients, FP64-generated tables converted to
// FP32, FP64 point separations and FP64 accumulation of the P2P sums.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/wbfmm_b200.h"
#include "engine.h"
#include "kernels.h"
#include "m2l_lanes.h"
#include "m2l_tc.h"
#include "table_cache.h"
#include "tables.h"

namespace wbfmm {

// The library's stream-ordered memory pool of the current device (created
// on first use; release threshold unlimited, no reuse across streams before
// a free has completed), or null when it cannot be created.  Solvers trim it
// to kLibPoolKeep unused bytes when they are destroyed.
cudaMemPool_t library_pool();

// whether an FP32 Helmholtz level of these orders can run the scaled M2L
// (helm_m2l_exp), which only the tile kernel implements
inline bool helm_m2l_scalable(int order_s, int order_r) {
  return order_s == order_r && tiles_supported<float, true>(order_s, order_r);
}
constexpr size_t kLibPoolKeep = (size_t)4 << 30;

// ------------------------------------------------------------ buffers
// Device buffer that only grows.  With a stream set, device memory comes
// from a stream-ordered pool (the library's, a server's, or the device's
// default; cudaMallocFromPoolAsync / cudaFreeAsync on that stream): no
// device-wide synchronisation on reallocation or release.
template <typename T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  bool managed = false;
  bool owned = true;        // false: memory supplied by the caller (adopt)
  cudaStream_t so = nullptr;
  cudaMemPool_t pool = nullptr;   // stream-ordered pool (default: device's)
  DBuf() = default;
  explicit DBuf(cudaStream_t s) : so(s) {}
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  ~DBuf() { release(); }
  void adopt(T* q, size_t count, bool is_managed) {
    release();
    p = q; n = count; managed = is_managed; owned = false;
  }
  void release() {
    if (p && owned) {
      if (so && !managed) cudaFreeAsync(p, so);
      else cudaFree(p);
    }
    owned = true;
    p = nullptr; n = 0;
  }
  int alloc(size_t count, bool use_managed = false) {
    if (p && n >= count && managed == use_managed) return 0;
    release();
    managed = use_managed;
    size_t bytes = sizeof(T) * (count ? count : 1);
    cudaError_t e = use_managed ? cudaMallocManaged(&p, bytes)
                    : (so && pool) ? cudaMallocFromPoolAsync(&p, bytes, pool, so)
                    : so        ? cudaMallocAsync(&p, bytes, so)
                                : cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
      p = nullptr;
      cudaGetLastError();
      return set_error(WBFMM_B200_E_NOMEM, "device allocation failed");
    }
    n = count;
    return 0;
  }
};

#define WBFMM_TRY(call)            \
  do {                             \
    int rc_ = (call);              \
    if (rc_ != 0) return rc_;      \
  } while (0)
#define WBFMM_TRY_VOID(call)       \
  do {                             \
    if ((call) != 0) return;       \
  } while (0)

template <typename T>
__global__ void k_convert(const double* __restrict__ a, T* __restrict__ b,
                          int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (T)a[i];
}
template <typename T>
__global__ void k_widen(const T* __restrict__ a, double* __restrict__ b,
                        int64_t n) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (double)a[i];
}
static __global__ void k_u64_to_u32(const uint64_t* __restrict__ a,
                             uint32_t* __restrict__ b, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (uint32_t)a[i];
}
// targets that are the sources: leaf box of each sorted source key
static __global__ void k_leaf_of_keys(const uint64_t* __restrict__ keys, int shift,
                                      uint64_t* __restrict__ tkeys,
                                      uint32_t* __restrict__ tbox, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t b = keys[i] >> shift;
  tkeys[i] = b;
  tbox[i] = (uint32_t)b;
}
// box at `level` has targets below it
static __global__ void k_target_mask(const uint32_t* __restrict__ leaf_count,
                              int depth, int level, uint8_t* __restrict__ mask) {
  int64_t nb = (int64_t)1 << (3 * level);
  int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  int sh = 3 * (depth - level);
  int64_t lo = b << sh, hi = (b + 1) << sh;
  uint8_t any = 0;
  for (int64_t c = lo; c < hi && !any; c++) any = leaf_count[c] != 0;
  mask[b] = any;
}

// parent[b] = any of child[8 b .. 8 b + 7] (a target mask one level up)
static __global__ void k_mask_up(const uint8_t* __restrict__ child, int64_t n,
                                 uint8_t* __restrict__ parent) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  uint8_t any = 0;
  for (int c = 0; c < 8; c++) any |= child[8 * b + c];
  parent[b] = any ? 1 : 0;
}

template <typename T>
static int convert_to(const double* src, T* dst, int64_t n, cudaStream_t s) {
  if (n <= 0) return 0;
  k_convert<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, dst, n);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wbfmm

// ------------------------------------------------------------- solver
struct wbfmm_b200_solver {
  virtual ~wbfmm_b200_solver() {}
  wbfmm_b200_config_t cfg;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int64_t launches = 0;
  double stage_ms[6] = {0, 0, 0, 0, 0, 0};
  virtual int set_sources(int, const double*, int, const double*, int, int) = 0;
  virtual int set_strengths(const double*, int, const double*, int, int) = 0;
  virtual int set_targets(int, const double*, int, int) = 0;
  virtual int build_operators() = 0;
  virtual int leaf_expansions() = 0;
  virtual int upward(int level) = 0;
  virtual int downward(int level) = 0;
  virtual int evaluate() = 0;
  virtual int run() = 0;
  virtual int run_queued() = 0;
  virtual int run_graph() = 0;
  virtual int wait() = 0;
  virtual int set_deferred_checks(int on) = 0;
  virtual int get_field(double*, double*, int) = 0;
  virtual int hessian(double* hess, int neighbours) = 0;
  virtual int target_bases() = 0;
  virtual int evaluate_bases(int neighbours) = 0;
  virtual int sources() const = 0;
  virtual int targets() const = 0;
  virtual int get_tree(uint32_t*, uint32_t*, uint32_t*, int) = 0;
  virtual int get_coefficients(int, double*, double*) = 0;
  virtual int coefficient_pointers(int, void**, void**) = 0;
  virtual void invalidate_operators() = 0;
  virtual int m2l(int level) = 0;
  virtual void set_m2l_kernel(int lanes) = 0;
  virtual void set_evaluation(int field, int neighbours) = 0;
  virtual void set_p2m_accumulate(int on) = 0;
  virtual int adopt_coefficients(int level, void* ms, void* mr) = 0;
  virtual int l2l(int level) = 0;
  virtual int coefficient_storage(int level, int64_t* groups, int64_t* bytes) = 0;
};

namespace wbfmm {

template <typename T>
struct Solver : public wbfmm_b200_solver {
  bool helm = false;
  int depth = 0, lmax = 0;
  // sources
  int nsrc = 0;
  const double* src_arg = nullptr;  // the set_sources array (for targets = sources)
  int src_arg_dev = 0;
  DBuf<double> pts_in, nrm_in;
  int xstr = 3, nstr = 3;
  DBuf<uint64_t> keys;
  DBuf<uint32_t> ip;
  DBuf<double> sx, sy, sz;
  DBuf<T> snx, sny, snz, sq, sdip;
  DBuf<double> stage;       // strength staging
  DBuf<double> nstage;      // normals in tree order before conversion
  bool have_q = false, have_dip = false, have_normals = false;
  RadixScratch rs;
  DBuf<uint32_t> box_i[kMaxDepth + 1], box_n[kMaxDepth + 1];
  // coefficients (Layout L; with sparse storage, per stored group)
  DBuf<T> mps[kMaxDepth + 1], mpr[kMaxDepth + 1];
  // sparse level storage (sparse.cu): per level the group -> slot map, the
  // slot -> group list and the count of stored groups, for the sources and
  // targets of geometry sparse_geo
  DBuf<uint32_t> gmap[kMaxDepth + 1], glist[kMaxDepth + 1], gflag, gcount, pmap;
  DBuf<unsigned char> gscratch;
  int64_t ngroups[kMaxDepth + 1] = {0};
  uint64_t sparse_geo = ~0ull;
  DBuf<T> dense_tmp;                // a sparse level expanded for get_coefficients
  // targets
  int ntgt = 0;
  DBuf<double> tpts_in, tx, ty, tz;
  DBuf<uint64_t> tkeys;
  DBuf<uint32_t> tperm, tbox, tstart, tcount;
  DBuf<uint8_t> tmask[kMaxDepth + 1];
  DBuf<int> act[kMaxDepth + 1], act_n[kMaxDepth + 1], act_scr;   // M2L target lists
  DBuf<uint8_t> smask;              // M2L skip_empty: source boxes of the level holding sources
  DBuf<T> lapsr;                    // Laplace lane M2L: scaled operators of the level
  DBuf<T> hcx;                      // Helmholtz tile M2L: coaxial rows of the level
  DBuf<int> flag;
  // outputs (original order)
  DBuf<T> pot, grad;
  DBuf<T> hess_d, hess_g;           // Hessian: derived expansions, gradients
  // near_fp32 (FP64 solvers): FP32 strengths, normals and near-field sums
  DBuf<float> n32_q, n32_dip, n32_nx, n32_ny, n32_nz, n32_pot, n32_grad;
  // precomputed target bases (potential): CSR near-field weights, bases
  DBuf<int64_t> tl_off;
  DBuf<uint32_t> tl_src;
  DBuf<T> tl_wq, tl_wd, tl_basis;
  uint64_t geo = 0;                 // bumped by set_sources / set_targets
  uint64_t tl_geo = ~0ull;          // geo of the bases held
  bool tl_dip = false;
  DBuf<double> out64;
  // tables
  bool ops_ready = false;
  ShiftGeometry geom;
  DBuf<double> H64;
  DBuf<T> H;
  int64_t hstride = 0;
  DBuf<int> op_ith, op_dist;
  DBuf<T> op_r, op_ph, op_ch;
  // Helmholtz coaxial tables of every level, one set (helm_coaxial_set)
  DBuf<double> coax_set64;
  DBuf<T> coax_set;
  int64_t sr_stride[kMaxDepth + 1] = {0};
  const T* sr_ptr[kMaxDepth + 1] = {nullptr};   // (S|R) table per level
  const T* ss_ptr[kMaxDepth + 1] = {nullptr};   // (R|R) table per level
  int helm_e[kMaxDepth + 1] = {0};   // FP32 Helmholtz M2L scale exponents (helm_m2l_exp)
  bool tc_used = false;             // the tensor-core M2L ran since the sources were set
  DBuf<float> tc_part;              // its split partial sums
  DBuf<double> lap64[3];
  DBuf<T> lap[3];
  int lt = 0;
  DBuf<T> partial;
  DBuf<unsigned char> lin;         // M2L lane kernel: transposed sources
  DBuf<T> lanes_part;              // and its split partial sums
  int m2l_mode = 1;                // 0 warp per target, 1 automatic, 2 lanes, 3 tiles
  int64_t lanes_ctas = 1200;       // lane kernel: split offsets below this many CTAs
  bool tree_only = false;          // structure only: no coefficient arrays
  int eval_field = 3;              // fields evaluate() computes
  bool eval_neighbours = true;     // evaluate() adds the near field (P2P)
  bool p2m_accumulate = false;     // leaf expansions add to the arrays
  OpTables<T> tables;
  cudaEvent_t ev[8];
  bool events = false;
  // served form: shared tables, no host waits inside a solve
  TableCache* cache = nullptr;
  bool async_checks = false;   // domain checks read back after the solve
  int* hflag = nullptr;        // pinned copy of flag[0..2]
  cudaMemPool_t lib_pool = nullptr;
  // graph replay of the passes (run_graph): valid while nothing they depend
  // on has changed since the capture
  uint64_t gen = 0;                 // bumped by every change of tree, targets, tables, options
  struct GraphSig {
    uint64_t gen; const void* q; const void* dip; bool hq, hd;
    bool operator==(const GraphSig& o) const {
      return gen == o.gen && q == o.q && dip == o.dip && hq == o.hq && hd == o.hd;
    }
  } gsig{};
  cudaGraphExec_t gexec = nullptr;
  int64_t glaunches = 0;            // kernels in the captured graph
  bool capturing = false;

  template <class F>
  void each_buf(F&& f) {
    f(pts_in); f(nrm_in); f(keys); f(ip); f(sx); f(sy); f(sz);
    f(snx); f(sny); f(snz); f(sq); f(sdip); f(stage); f(nstage);
    for (int l = 0; l <= kMaxDepth; l++) {
      f(box_i[l]); f(box_n[l]); f(mps[l]); f(mpr[l]); f(tmask[l]);
      f(act[l]); f(act_n[l]); f(gmap[l]); f(glist[l]);
    }
    f(gflag); f(gcount); f(pmap); f(gscratch); f(dense_tmp);
    f(coax_set64); f(coax_set);
    f(tpts_in); f(tx); f(ty); f(tz); f(tkeys); f(tperm); f(tbox);
    f(tstart); f(tcount); f(flag); f(pot); f(grad); f(out64); f(hess_d); f(hess_g);
    f(tl_off); f(tl_src); f(tl_wq); f(tl_wd); f(tl_basis);
    f(n32_q); f(n32_dip); f(n32_nx); f(n32_ny); f(n32_nz); f(n32_pot); f(n32_grad);
    f(H64); f(H); f(op_ith); f(op_dist); f(op_r); f(op_ph); f(op_ch);
    for (int i = 0; i < 3; i++) { f(lap64[i]); f(lap[i]); }
    f(partial); f(lin); f(lanes_part); f(act_scr); f(lapsr); f(hcx); f(smask); f(tc_part);
  }

  ~Solver() override {
    if (gexec) cudaGraphExecDestroy(gexec);
    const bool trim = lib_pool && flag.pool == lib_pool;
    each_buf([](auto& b) { b.release(); });
    if (stream) cudaStreamSynchronize(stream);
    // what this solver freed stays cached up to kLibPoolKeep bytes
    if (trim) cudaMemPoolTrimTo(lib_pool, kLibPoolKeep);
    radix_scratch_free(&rs);
    if (events)
      for (int i = 0; i < 8; i++) cudaEventDestroy(ev[i]);
    if (hflag) cudaFreeHost(hflag);
    if (own_stream && stream) cudaStreamDestroy(stream);
  }

  double width(int level) const { return cfg.D / (double)(1 << level); }
  int ncoefs(int p) const { return (p + 1) * (p + 1); }
  size_t level_len(int level, int p) const {
    return ((size_t)1 << (3 * level)) * ncoefs(p) * (helm ? 2 : 1);
  }
  // values of the coefficient array of a level at order p as stored
  size_t coef_len(int level, int p) const {
    if (!cfg.sparse) return level_len(level, p);
    return (size_t)ngroups[level] * 8 * ncoefs(p) * (helm ? 2 : 1);
  }

  // validate and take a configuration (buffers already held are kept)
  int configure(const wbfmm_b200_config_t* c) {
    gen++;
    cfg = *c;
    helm = cfg.problem == WBFMM_B200_HELMHOLTZ;
    if (cfg.problem != WBFMM_B200_HELMHOLTZ && cfg.problem != WBFMM_B200_LAPLACE)
      return set_error(WBFMM_B200_E_ARG, "problem must be Laplace (1) or Helmholtz (2)");
    depth = cfg.depth;
    if ((depth < 2 && !tree_only) || depth < 0 || depth > 10)
      return set_error(WBFMM_B200_E_ARG, "depth must be in [2, 10]");
    if (!(cfg.D > 0.0)) return set_error(WBFMM_B200_E_ARG, "tree width must be positive");
    lmax = 0;
    for (int l = 1; l <= depth && !tree_only; l++) {
      if (cfg.order_s[l] < 1 || cfg.order_r[l] < 1 ||
          cfg.order_s[l] > kMaxOrder || cfg.order_r[l] > kMaxOrder)
        return set_error(WBFMM_B200_E_ORDER, "expansion orders must be in [1, 62]");
      lmax = std::max(lmax, std::max(cfg.order_s[l], cfg.order_r[l]));
    }
    if (cfg.field == 0) cfg.field = WBFMM_B200_POTENTIAL;
    if (cfg.sparse) {
      // coefficients of the boxes that hold sources or targets (and their
      // siblings) only: the M2L skips the rest, as skip_empty does
      if (cfg.managed) return set_error(WBFMM_B200_E_ARG, "sparse level storage does not take managed arrays");
      cfg.skip_empty = 1;
    }
    return 0;
  }

  int init(const wbfmm_b200_config_t* c, void* s) {
    WBFMM_TRY(configure(c));
    if (s) {
      stream = (cudaStream_t)s;
    } else {
      WBFMM_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
      own_stream = true;
    }
    for (int i = 0; i < 8; i++) WBFMM_CUDA(cudaEventCreate(&ev[i]));
    events = true;
    // plain solvers allocate from the library's pool of this device, which
    // keeps freed memory (repeated solves reallocate without mapping)
    lib_pool = library_pool();
    each_buf([&](auto& b) { b.so = stream; b.pool = lib_pool; });
    WBFMM_TRY(flag.alloc(3));
    return 0;
  }

  // Served form: start a new solve on the same stream and buffers.
  int reset(const wbfmm_b200_config_t* c) {
    WBFMM_TRY(configure(c));
    ops_ready = false;
    nsrc = ntgt = 0;
    have_q = have_dip = have_normals = false;
    if (!hflag) WBFMM_CUDA(cudaMallocHost(&hflag, 3 * sizeof(int)));
    return 0;
  }

  // device bytes of the work buffers this solver owns
  size_t buffer_bytes() {
    size_t b = 0;
    each_buf([&](auto& x) { if (x.owned && x.p) b += x.n * sizeof(*x.p); });
    return b;
  }

  // Served form: every work buffer back to the stream-ordered pool.
  void release_buffers() {
    each_buf([](auto& b) { if (b.owned) b.release(); });
    WBFMM_TRY_VOID(flag.alloc(3));
  }

  // flag[0]: first source outside the cube (0x7fffffff: none);
  // flag[1]: nonzero when a target lies outside the cube;
  // flag[2]: nonzero when a bounded wait of the tensor-core M2L ran out
  static int domain_error(int bad_source, int bad_target) {
    if (bad_source != 0x7fffffff) {
      char msg[160];
      snprintf(msg, sizeof(msg), "source point %d does not lie strictly inside the tree cube", bad_source);
      return set_error(WBFMM_B200_E_DOMAIN, msg);
    }
    if (bad_target) return set_error(WBFMM_B200_E_DOMAIN, "target point outside the tree cube");
    return 0;
  }

  // -------------------------------------------------------------- tree
  int set_sources(int n, const double* xs, int xs_str, const double* normals,
                  int n_str, int on_device) override {
    if (n <= 0 || xs == nullptr || xs_str < 3)
      return set_error(WBFMM_B200_E_ARG, "bad source points");
    if (normals && n_str < 3) return set_error(WBFMM_B200_E_ARG, "bad normal stride");
    cudaEventRecord(ev[0], stream);
    gen++;
    geo++;
    src_arg = nullptr;              // set again only when these sources are in place
    nsrc = n;
    xstr = xs_str;
    const double* dpts = xs;
    if (!on_device) {
      WBFMM_TRY(pts_in.alloc((size_t)n * xs_str));
      WBFMM_CUDA(cudaMemcpyAsync(pts_in.p, xs, sizeof(double) * n * xs_str,
                                 cudaMemcpyHostToDevice, stream));
      dpts = pts_in.p;
    }
    // strict-interior domain check (src/boxes.c:148-153)
    launch_set_words((uint32_t*)flag.p, 0x7fffffffu, (uint32_t*)flag.p + 2, 0, stream);
    launch_domain_check(dpts, xs_str, n, cfg.x0, cfg.D, flag.p, stream, cfg.keys_fp32 != 0);
    if (!async_checks) {
      int bad = 0;
      WBFMM_CUDA(cudaMemcpyAsync(&bad, flag.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
      WBFMM_CUDA(cudaStreamSynchronize(stream));
      WBFMM_TRY(domain_error(bad, 0));
    }
    WBFMM_TRY(keys.alloc(n));
    WBFMM_TRY(ip.alloc(n));
    launch_point_keys(dpts, xs_str, n, cfg.x0, cfg.D, keys.p, ip.p, stream, cfg.keys_fp32 != 0);
    // full 60-bit keys (the reference's point order), or with leaf_order
    // only the bits that select the leaf box
    const int sort_lo = cfg.leaf_order ? 60 - 3 * depth : 0;
    WBFMM_TRY(radix_sort_pairs(keys.p, ip.p, n, 60 - sort_lo, &rs, stream, sort_lo));
    launches += 4 + 3 * ((60 - sort_lo + 7) / 8);
    WBFMM_TRY(sx.alloc(n)); WBFMM_TRY(sy.alloc(n)); WBFMM_TRY(sz.alloc(n));
    launch_gather_points(dpts, xs_str, ip.p, n, sx.p, sy.p, sz.p, stream);
    launches++;
    have_normals = normals != nullptr;
    if (normals) {
      const double* dn = normals;
      nstr = n_str;
      if (!on_device) {
        WBFMM_TRY(nrm_in.alloc((size_t)n * n_str));
        WBFMM_CUDA(cudaMemcpyAsync(nrm_in.p, normals, sizeof(double) * n * n_str,
                                   cudaMemcpyHostToDevice, stream));
        dn = nrm_in.p;
      }
      WBFMM_TRY(nstage.alloc((size_t)3 * n));
      double* tmp = nstage.p;
      launch_gather_points(dn, n_str, ip.p, n, tmp, tmp + n, tmp + 2 * n, stream);
      WBFMM_TRY(snx.alloc(n)); WBFMM_TRY(sny.alloc(n)); WBFMM_TRY(snz.alloc(n));
      WBFMM_TRY(convert_to<T>(tmp, snx.p, n, stream));
      WBFMM_TRY(convert_to<T>(tmp + n, sny.p, n, stream));
      WBFMM_TRY(convert_to<T>(tmp + 2 * n, snz.p, n, stream));
      launches += 4;
    }
    // levels: box {i, n} by repeated refinement (src/boxes.c:208-277)
    WBFMM_TRY(box_i[0].alloc(1)); WBFMM_TRY(box_n[0].alloc(1));
    launch_set_words(box_i[0].p, 0u, box_n[0].p, (uint32_t)n, stream);
    for (int l = 1; l <= depth; l++) {
      size_t nb = (size_t)1 << (3 * l);
      WBFMM_TRY(box_i[l].alloc(nb)); WBFMM_TRY(box_n[l].alloc(nb));
      launch_refine_children(keys.p, n, l, box_i[l - 1].p, box_i[l].p, box_n[l].p, stream);
      launch_refine_parents(l - 1, box_i[l - 1].p, box_n[l - 1].p, stream);
      launches += 2;
    }
    WBFMM_CUDA(cudaGetLastError());
    // coefficient arrays (arrays adopted from the caller are kept; sparse
    // storage allocates once the targets are known, prepare_sparse)
    for (int l = 1; l <= depth && !tree_only && !cfg.sparse; l++) {
      WBFMM_TRY(mps[l].alloc(level_len(l, cfg.order_s[l]), cfg.managed != 0));
      WBFMM_TRY(mpr[l].alloc(level_len(l, cfg.order_r[l]), cfg.managed != 0));
    }
    src_arg = xs;
    src_arg_dev = on_device;
    cudaEventRecord(ev[1], stream);
    return 0;
  }

  int set_strengths(const double* q, int qstr, const double* dip, int dstr,
                    int on_device) override {
    if (nsrc <= 0) return set_error(WBFMM_B200_E_STATE, "set_sources first");
    const int nc = helm ? 2 : 1;
    if (dip && !have_normals)
      return set_error(WBFMM_B200_E_ARG, "dipole strengths given but the sources have no normals");
    if ((q && qstr < nc) || (dip && dstr < nc))
      return set_error(WBFMM_B200_E_ARG, "strength stride too small");
    have_q = q != nullptr;
    have_dip = dip != nullptr;
    auto upload = [&](const double* a, int str, DBuf<T>& dst) -> int {
      const double* d = a;
      if (!on_device) {
        WBFMM_TRY(stage.alloc((size_t)nsrc * str));
        WBFMM_CUDA(cudaMemcpyAsync(stage.p, a, sizeof(double) * nsrc * str,
                                   cudaMemcpyHostToDevice, stream));
        d = stage.p;
      }
      WBFMM_TRY(dst.alloc((size_t)nsrc * nc));
      if (sizeof(T) == 8)
        launch_gather_real(d, str, ip.p, nsrc, nc, (double*)dst.p, stream);
      else
        launch_gather_real_f32(d, str, ip.p, nsrc, nc, (float*)dst.p, stream);
      launches++;
      WBFMM_CUDA(cudaGetLastError());
      return 0;
    };
    if (q) WBFMM_TRY(upload(q, qstr, sq));
    if (dip) WBFMM_TRY(upload(dip, dstr, sdip));
    return 0;
  }

  int set_targets(int n, const double* xt, int tstr, int on_device) override {
    gen++;
    geo++;
    if (n <= 0 || xt == nullptr || tstr < 3)
      return set_error(WBFMM_B200_E_ARG, "bad target points");
    ntgt = n;
    WBFMM_CUDA(cudaMemsetAsync(flag.p + 1, 0, sizeof(int), stream));
    WBFMM_TRY(tkeys.alloc(n)); WBFMM_TRY(tperm.alloc(n));
    WBFMM_TRY(tx.alloc(n)); WBFMM_TRY(ty.alloc(n)); WBFMM_TRY(tz.alloc(n));
    WBFMM_TRY(tbox.alloc(n));
    if (xt == src_arg && on_device == src_arg_dev && tstr == xstr && n == nsrc) {
      // the sources' array again: the source sort already groups the points
      // by leaf box (the order inside a leaf changes no target's field), and
      // the sources passed the domain check
      WBFMM_CUDA(cudaMemcpyAsync(tperm.p, ip.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, stream));
      WBFMM_CUDA(cudaMemcpyAsync(tx.p, sx.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
      WBFMM_CUDA(cudaMemcpyAsync(ty.p, sy.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
      WBFMM_CUDA(cudaMemcpyAsync(tz.p, sz.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
      k_leaf_of_keys<<<(n + 255) / 256, 256, 0, stream>>>(keys.p, 60 - 3 * depth, tkeys.p,
                                                         tbox.p, n);
      launches++;
    } else {
      const double* d = xt;
      if (!on_device) {
        WBFMM_TRY(tpts_in.alloc((size_t)n * tstr));
        WBFMM_CUDA(cudaMemcpyAsync(tpts_in.p, xt, sizeof(double) * n * tstr,
                                   cudaMemcpyHostToDevice, stream));
        d = tpts_in.p;
      }
      launch_target_keys(d, tstr, n, cfg.x0, cfg.D, depth, tkeys.p, tperm.p,
                         flag.p + 1, stream, cfg.keys_fp32 != 0);
      WBFMM_TRY(radix_sort_pairs(tkeys.p, tperm.p, n, 3 * depth, &rs, stream));
      launch_gather_points(d, tstr, tperm.p, n, tx.p, ty.p, tz.p, stream);
      k_u64_to_u32<<<(n + 255) / 256, 256, 0, stream>>>(tkeys.p, tbox.p, n);
      launches += 3 + 3 * ((3 * depth + 7) / 8);
    }
    size_t nb = (size_t)1 << (3 * depth);
    WBFMM_TRY(tstart.alloc(nb)); WBFMM_TRY(tcount.alloc(nb));
    launch_box_ranges(tkeys.p, n, depth, tstart.p, tcount.p, stream);
    launches++;
    if (cfg.skip_empty) {
      for (int l = 2; l <= depth; l++) {
        size_t nbl = (size_t)1 << (3 * l);
        WBFMM_TRY(tmask[l].alloc(nbl));
        k_target_mask<<<(unsigned)((nbl + 255) / 256), 256, 0, stream>>>(
            tcount.p, depth, l, tmask[l].p);
        // the M2L kernels' per-child-type lists of the boxes with targets
        WBFMM_TRY(act[l].alloc(nbl));
        WBFMM_TRY(act_n[l].alloc(8));
        WBFMM_TRY(act_scr.alloc(active_list_scratch(l)));
        WBFMM_TRY(build_active_lists(tmask[l].p, l, act[l].p, act_n[l].p, act_scr.p, stream));
        launches += 4;
      }
    }
    if (!async_checks) {
      int bad = 0;
      WBFMM_CUDA(cudaMemcpyAsync(&bad, flag.p + 1, sizeof(int), cudaMemcpyDeviceToHost, stream));
      WBFMM_CUDA(cudaStreamSynchronize(stream));
      WBFMM_TRY(domain_error(0x7fffffff, bad));
    }
    const int w = helm ? 2 : 1;
    if (cfg.field & WBFMM_B200_POTENTIAL) WBFMM_TRY(pot.alloc((size_t)n * w));
    if (cfg.field & WBFMM_B200_GRADIENT) WBFMM_TRY(grad.alloc((size_t)n * 3 * w));
    return 0;
  }

  // ------------------------------------------------------- operators
  int build_operators() override {
    if (ops_ready) return 0;
    cudaEventRecord(ev[2], stream);
    if (cache) {
      WBFMM_TRY(shared_operators());
    } else {
      WBFMM_TRY(own_operators());
    }
    ops_ready = true;
    cudaEventRecord(ev[3], stream);
    return 0;
  }

  // tables from the server's cache (served form): the order-only tables are
  // shared; the Helmholtz coaxial tables depend on k w (every request of a
  // served stream has its own k) and are built per solve, all levels in one
  // set, into this solver's buffers
  int shared_operators() {
    WBFMM_TRY(cache->geometry<T>(lmax + 1, stream, &tables));
    if (!helm) return 0;
    return helm_coaxial_set();
  }

  // Helmholtz coaxial tables of every level in one launch set: per level
  // l >= 2, (S|R) at the 15 list-4 distances k w_l sqrt(d2) (order of the
  // level; M2L), then (R|R) = (S|S) at k w_l sqrt(3)/2 (order of levels l-1
  // and l; M2M l -> l-1 and L2L l-1 -> l); FP64, and converted for FP32
  int helm_coaxial_set() {
    CoaxJob jobs[kMaxCoaxJobs];
    int nj = 0;
    int64_t off = 0, sr_off[kMaxDepth + 1] = {0}, ss_off[kMaxDepth + 1] = {0};
    for (int l = 2; l <= depth; l++) {
      const int Ll = std::max(cfg.order_s[l], cfg.order_r[l]);
      sr_stride[l] = 2 * ((int64_t)(Ll + 1) * (Ll + 2) * (Ll + 3) / 6 + 1);
      sr_off[l] = off;
      for (int i = 0; i < 15; i++) {
        jobs[nj++] = CoaxJob{cfg.k * width(l) * sqrt((double)kListDist2[i]), Ll, 2, off, 0};
        off += sr_stride[l];
      }
      const int Ls = std::max(std::max(cfg.order_s[l], cfg.order_r[l]),
                              std::max(cfg.order_s[l - 1], cfg.order_r[l - 1]));
      ss_off[l] = off;
      jobs[nj++] = CoaxJob{cfg.k * width(l) * 0.5 * sqrt(3.0), Ls, 1, off, 0};
      off += (int64_t)(Ls + 1) * (Ls + 2) * (Ls + 3) / 6 + 1;
    }
    WBFMM_TRY(coax_set64.alloc((size_t)off));
    WBFMM_TRY(generate_coaxial_set(jobs, nj, coax_set64.p, stream));
    const T* base = (const T*)coax_set64.p;
    if (sizeof(T) != 8) {
      WBFMM_TRY(coax_set.alloc((size_t)off));
      WBFMM_TRY(convert_to<T>(coax_set64.p, coax_set.p, off, stream));
      base = coax_set.p;
      launches++;
      // levels whose (S|R) coefficients leave the FP32 range: the scaled
      // form of their M2L (helm_m2l_exp), tables written scaled
      for (int l = 2; l <= depth; l++) {
        helm_e[l] = helm_m2l_scalable(cfg.order_s[l], cfg.order_r[l])
                        ? helm_m2l_exp(cfg.k, width(l), cfg.order_s[l]) : 0;
        if (!helm_e[l]) continue;
        const int Ll = std::max(cfg.order_s[l], cfg.order_r[l]);
        WBFMM_TRY(narrow_coax_scaled(coax_set64.p + sr_off[l], (float*)coax_set.p + sr_off[l],
                                     Ll, sr_stride[l], 15, helm_e[l], stream));
        launches++;
      }
    } else {
      for (int l = 2; l <= depth; l++) helm_e[l] = 0;
    }
    for (int l = 2; l <= depth; l++) {
      sr_ptr[l] = base + sr_off[l];
      ss_ptr[l] = base + ss_off[l];
    }
    launches += 2;
    return 0;
  }

  // tables owned by this solver (plain form)
  int own_operators() {
    build_shift_geometry(&geom);
    const int L = lmax + 1;
    std::vector<int> ith, dist;
    std::vector<double> r, ph, ch;
    shift_op_tables(geom, L, ith, dist, r, ph, ch);
    WBFMM_TRY(op_ith.alloc(kNumOps)); WBFMM_TRY(op_dist.alloc(kNumOps));
    WBFMM_CUDA(cudaMemcpyAsync(op_ith.p, ith.data(), sizeof(int) * kNumOps, cudaMemcpyHostToDevice, stream));
    WBFMM_CUDA(cudaMemcpyAsync(op_dist.p, dist.data(), sizeof(int) * kNumOps, cudaMemcpyHostToDevice, stream));
    {
      DBuf<double> tmp(stream);
      tmp.pool = flag.pool;
      size_t nph = ph.size();
      WBFMM_TRY(tmp.alloc(nph * 2 + kNumOps));
      WBFMM_CUDA(cudaMemcpyAsync(tmp.p, ph.data(), sizeof(double) * nph, cudaMemcpyHostToDevice, stream));
      WBFMM_CUDA(cudaMemcpyAsync(tmp.p + nph, ch.data(), sizeof(double) * nph, cudaMemcpyHostToDevice, stream));
      WBFMM_CUDA(cudaMemcpyAsync(tmp.p + 2 * nph, r.data(), sizeof(double) * kNumOps, cudaMemcpyHostToDevice, stream));
      WBFMM_TRY(op_ph.alloc(nph)); WBFMM_TRY(op_ch.alloc(nph)); WBFMM_TRY(op_r.alloc(kNumOps));
      WBFMM_TRY(convert_to<T>(tmp.p, op_ph.p, nph, stream));
      WBFMM_TRY(convert_to<T>(tmp.p + nph, op_ch.p, nph, stream));
      WBFMM_TRY(convert_to<T>(tmp.p + 2 * nph, op_r.p, kNumOps, stream));
    }
    // rotation tables (FP64 on the GPU)
    hstride = rot_count(L) + 8;
    int nth = (int)geom.thetas.size();
    WBFMM_TRY(H64.alloc((size_t)hstride * nth));
    WBFMM_TRY(generate_rotation_tables(geom.thetas, L, H64.p, hstride, stream));
    WBFMM_TRY(H.alloc((size_t)hstride * nth));
    WBFMM_TRY(convert_to<T>(H64.p, H.p, (int64_t)hstride * nth, stream));
    launches += 2;
    if (helm) {
      WBFMM_TRY(helm_coaxial_set());
    } else {
      lt = L;
      size_t n3 = (size_t)(lt + 1) * (lt + 1) * (lt + 1);
      for (int i = 0; i < 3; i++) {
        WBFMM_TRY(lap64[i].alloc(n3));
        WBFMM_TRY(lap[i].alloc(n3));
      }
      WBFMM_TRY(generate_laplace_tables(lt, lap64[0].p, lap64[1].p, lap64[2].p, stream));
      for (int i = 0; i < 3; i++)
        WBFMM_TRY(convert_to<T>(lap64[i].p, lap[i].p, (int64_t)n3, stream));
      launches += 4;
    }
    tables.H = H.p; tables.hstride = hstride;
    tables.op_ith = op_ith.p; tables.op_dist = op_dist.p; tables.op_r = op_r.p;
    tables.ph = op_ph.p; tables.ch = op_ch.p; tables.lmax = L;
    if (!helm) {
      tables.lapSS = lap[0].p; tables.lapRR = lap[1].p; tables.lapSR = lap[2].p;
      tables.lt = lt;
    }
    return 0;
  }

  // Sparse level storage: the group maps of every level from the boxes
  // holding sources (box counts) or targets (target masks), then the
  // compact coefficient arrays.  Once per geometry; one host wait (the
  // group counts size the arrays).
  int prepare_sparse() {
    if (!cfg.sparse || tree_only || sparse_geo == geo) return 0;
    if (nsrc <= 0 || ntgt <= 0)
      return set_error(WBFMM_B200_E_STATE, "sparse level storage: set the sources and the targets first");
    // target masks of levels 1 and 0 from level 2's (set_targets builds the
    // levels >= 2 with skip_empty, which sparse storage implies)
    if (!tmask[2].p) return set_error(WBFMM_B200_E_STATE, "sparse level storage: no target masks");
    for (int l = 1; l >= 0; l--) {
      const int64_t nbl = (int64_t)1 << (3 * l);
      WBFMM_TRY(tmask[l].alloc((size_t)nbl));
      k_mask_up<<<1, 64, 0, stream>>>(tmask[l + 1].p, nbl, tmask[l].p);
      launches++;
    }
    WBFMM_TRY(gcount.alloc(kMaxDepth + 1));
    const int64_t nmax = (int64_t)1 << (3 * (depth - 1));
    WBFMM_TRY(gflag.alloc((size_t)nmax));
    const size_t scr = sparse_scan_scratch(nmax);
    WBFMM_TRY(gscratch.alloc(scr));
    for (int l = 1; l <= depth; l++) {
      const int64_t n = (int64_t)1 << (3 * (l - 1));    // groups: boxes of level l - 1
      WBFMM_TRY(gmap[l].alloc((size_t)n));
      WBFMM_TRY(sparse_group_map(box_n[l - 1].p, tmask[l - 1].p, n, gflag.p, gmap[l].p,
                                 gcount.p + l, gscratch.p, scr, stream));
      launches += 3;
    }
    uint32_t cnt[kMaxDepth + 1] = {0};
    WBFMM_CUDA(cudaMemcpyAsync(cnt + 1, gcount.p + 1, sizeof(uint32_t) * depth,
                               cudaMemcpyDeviceToHost, stream));
    WBFMM_CUDA(cudaStreamSynchronize(stream));
    const int w = helm ? 2 : 1;
    for (int l = 1; l <= depth; l++) {
      const int64_t n = (int64_t)1 << (3 * (l - 1));
      ngroups[l] = cnt[l];
      if (ngroups[l] <= 0 || ngroups[l] > n)
        return set_error(WBFMM_B200_E_STATE, "sparse level storage: bad group count");
      WBFMM_TRY(glist[l].alloc((size_t)ngroups[l]));
      WBFMM_TRY(sparse_group_list(gmap[l].p, n, glist[l].p, stream));
      WBFMM_TRY(mps[l].alloc((size_t)ngroups[l] * 8 * ncoefs(cfg.order_s[l]) * w));
      WBFMM_TRY(mpr[l].alloc((size_t)ngroups[l] * 8 * ncoefs(cfg.order_r[l]) * w));
      launches++;
    }
    sparse_geo = geo;
    return 0;
  }

  // ------------------------------------------------------------- passes
  int leaf_expansions() override {
    if (nsrc <= 0) return set_error(WBFMM_B200_E_STATE, "set_sources first");
    WBFMM_TRY(prepare_sparse());
    P2MParams<T> p;
    p.nbox = (int64_t)1 << (3 * depth);
    p.level = depth; p.N = cfg.order_s[depth];
    p.x0 = cfg.x0[0]; p.y0 = cfg.x0[1]; p.z0 = cfg.x0[2]; p.wb = width(depth);
    p.k = (T)cfg.k;
    p.box_i = box_i[depth].p; p.box_n = box_n[depth].p;
    p.x = sx.p; p.y = sy.p; p.z = sz.p;
    p.q = have_q ? sq.p : nullptr;
    p.dip = have_dip ? sdip.p : nullptr;
    p.nx = snx.p; p.ny = sny.p; p.nz = snz.p;
    p.mps = mps[depth].p;
    p.accumulate = p2m_accumulate ? 1 : 0;
    if (cfg.sparse) {
      p.nbox = 8 * ngroups[depth];
      p.glist = glist[depth].p;
    }
    launches++;
    return helm ? launch_p2m<T, true>(p, stream) : launch_p2m<T, false>(p, stream);
  }

  XlateParams<T> xparams() const {
    XlateParams<T> x;
    memset(&x, 0, sizeof(x));
    x.k = (T)cfg.k;
    x.nsplit = 1;
    return x;
  }

  int upward(int level) override {
    if (level < 3 || level > depth) return set_error(WBFMM_B200_E_ARG, "upward pass level must be in [3, depth]");
    WBFMM_TRY(build_operators());
    WBFMM_TRY(prepare_sparse());
    XlateParams<T> x = xparams();
    x.level = level - 1;
    x.nbox = (int64_t)1 << (3 * (level - 1));
    x.Nin = cfg.order_s[level]; x.Nout = cfg.order_s[level - 1];
    x.cin = mps[level].p; x.cout = mps[level - 1].p;
    x.coax = helm ? ss_ptr[level] : nullptr;
    x.width = (T)width(level);
    if (cfg.sparse) {
      // one CTA per stored group of the children; the parents' other
      // siblings (no sources or targets) hold zeros
      WBFMM_CUDA(cudaMemsetAsync(x.cout, 0, sizeof(T) * coef_len(level - 1, x.Nout), stream));
      x.nbox = ngroups[level];
      x.glist = glist[level].p;
      x.gmap = gmap[level - 1].p;
    }
    launches++;
    return helm ? launch_m2m<T, true>(x, tables, stream)
                : launch_m2m<T, false>(x, tables, stream);
  }

  int downward(int level) override {
    WBFMM_TRY(m2l(level));
    if (level == depth) return 0;
    return l2l(level);
  }

  int m2l(int level) override {
    if (level < 2 || level > depth) return set_error(WBFMM_B200_E_ARG, "downward pass level must be in [2, depth]");
    WBFMM_TRY(build_operators());
    WBFMM_TRY(prepare_sparse());
    if (level == 2)
      WBFMM_CUDA(cudaMemsetAsync(mpr[2].p, 0, sizeof(T) * coef_len(2, cfg.order_r[2]), stream));
    XlateParams<T> x = xparams();
    x.level = level;
    x.nbox = (int64_t)1 << (3 * level);
    x.Nin = cfg.order_s[level]; x.Nout = cfg.order_r[level];
    x.cin = mps[level].p; x.cout = mpr[level].p;
    x.src_n = box_n[level].p;
    x.coax = helm ? sr_ptr[level] : nullptr;
    x.coax_stride = sr_stride[level];
    x.width = (T)width(level);
    x.tmask = cfg.skip_empty && tmask[level].p ? tmask[level].p : nullptr;
    x.lap_e = helm ? 0 : lap_scale_exp(width(level));
    const bool lanes_ok = helm ? lanes_supported<T, true>(x.Nin, x.Nout)
                               : lanes_supported<T, false>(x.Nin, x.Nout);
    const bool tiles_ok = helm ? tiles_supported<T, true>(x.Nin, x.Nout)
                               : tiles_supported<T, false>(x.Nin, x.Nout);
    // automatic: lanes at the orders where their unrolled code wins, tiles
    // above, the warp-per-target kernel for what neither covers (Helmholtz
    // p = 8 runs as fast or faster as tiles in both forms, up to 2x on small
    // levels, and FP64 Laplace p = 10 15-20% faster, dense or on target
    // lists; Helmholtz p = 7, FP32 Laplace p = 10 and FP64 Laplace p = 9 run
    // faster as lanes)
    const int lanes_max = helm ? 7 : sizeof(T) == 8 ? 9 : 10;
    bool use_tiles = false, use_lanes = false;
    const int he = helm ? helm_e[level] : 0;
    if (cfg.sparse) return m2l_sparse(level, x, he, tiles_ok, lanes_ok, lanes_max);
    // tensor cores: Laplace, FP32, equal orders up to (p+1)^2 = 256, mode 4
    if (!helm && sizeof(T) == 4 && m2l_mode == 4 && tc_lap_supported(x.Nin, x.Nout))
      return m2l_tc(level, x);
    if (he) {
      // the scaled Helmholtz M2L (FP32 tables out of range unscaled) runs
      // in the tile kernel only
      if (!tiles_ok)
        return set_error(WBFMM_B200_E_ORDER, "FP32 Helmholtz M2L out of range at this order; use the FP64 form");
      use_tiles = true;
    } else if (m2l_mode == 1) {
      use_lanes = lanes_ok && x.Nin <= lanes_max;
      use_tiles = !use_lanes && tiles_ok;
    } else if (m2l_mode == 2) {
      use_lanes = lanes_ok;
    } else if (m2l_mode == 3) {
      use_tiles = tiles_ok;
    }
    if (use_tiles) {
      // offset-major target tiles on the transposed singular expansions
      WBFMM_TRY(lin.alloc(lanes_lin_bytes(level, x.Nin, helm, sizeof(T))));
      WBFMM_TRY((helm ? lanes_to_lin<T, true>(x.cin, level, x.Nin, he, lin.p, stream)
                      : lanes_to_lin<T, false>(x.cin, level, x.Nin, x.lap_e, lin.p, stream)));
      LanesParams<T> lp;
      memset(&lp, 0, sizeof(lp));
      lp.level = level; lp.N = x.Nin;
      lp.lin_raw = lin.p; lp.cout = x.cout;
      lp.coax = x.coax; lp.coax_stride = x.coax_stride;
      lp.width = x.width; lp.tmask = x.tmask; lp.lap_e = x.lap_e;
      lp.helm_e = he;
      if (x.tmask && act[level].p) { lp.act = act[level].p; lp.act_n = act_n[level].p; }
      if (x.tmask) {
        WBFMM_TRY(smask.alloc(source_mask_bytes(level)));
        WBFMM_TRY(build_source_mask(x.src_n, level, smask.p, stream));
        lp.smask = smask.p;
        launches++;
      }
      if (!helm) {
        const int P1 = x.Nin + 1;
        WBFMM_TRY(lapsr.alloc((size_t)kNumOps * P1 * P1 * P1));
        WBFMM_TRY(build_lap_sr_ops<T>(tables, x.Nin, x.width, x.lap_e, lapsr.p, stream));
        lp.lapsr = lapsr.p;
        launches++;
      }
      bool dense = false;
      const int tc = helm ? tiles_per_cta<T, true>(x.Nin, &dense) : tiles_per_cta<T, false>(x.Nin);
      if (dense) {
        WBFMM_TRY(hcx.alloc(helm_coax_rows_count(x.Nin)));
        WBFMM_TRY(build_helm_coax_rows<T>(x.coax, x.coax_stride, x.Nin, hcx.p, stream));
        lp.hcx = hcx.p;
        launches++;
      }
      const int64_t np = (int64_t)1 << (3 * (level - 1));
      const int64_t ctas = ((np + tc - 1) / tc) * 8;
      int ns = 1;
      while (ctas * ns < 2 * 148 && ns < 32) ns *= 2;
      lp.nsplit = ns;
      if (ns > 1) {
        const int V = helm ? (x.Nin + 1) * (x.Nin + 1) : (x.Nin + 1) * (x.Nin + 2) / 2;
        WBFMM_TRY(lanes_part.alloc((size_t)ns * 8 * V * np * 2));
        lp.partial_raw = lanes_part.p;
      }
      launches += ns > 1 ? 3 : 2;
      return helm ? launch_m2l_tiles<T, true>(lp, tables, stream)
                  : launch_m2l_tiles<T, false>(lp, tables, stream);
    }
    if (use_lanes) {
      // lane-per-pair kernel on a transposed copy of the singular expansions
      // (box-major for target lists)
      const bool boxmajor = x.tmask && act[level].p;
      WBFMM_TRY(lin.alloc(lanes_lin_bytes(level, x.Nin, helm, sizeof(T))));
      WBFMM_TRY((helm ? lanes_to_lin<T, true>(x.cin, level, x.Nin, 0, lin.p, stream, boxmajor)
                      : lanes_to_lin<T, false>(x.cin, level, x.Nin, x.lap_e, lin.p, stream,
                                               boxmajor)));
      LanesParams<T> lp;
      memset(&lp, 0, sizeof(lp));
      lp.boxmajor = boxmajor;
      lp.level = level; lp.N = x.Nin;
      lp.lin_raw = lin.p; lp.cout = x.cout;
      lp.coax = x.coax; lp.coax_stride = x.coax_stride;
      lp.width = x.width; lp.tmask = x.tmask; lp.lap_e = x.lap_e;
      if (x.tmask && act[level].p) { lp.act = act[level].p; lp.act_n = act_n[level].p; }
      if (x.tmask) {
        WBFMM_TRY(smask.alloc(source_mask_bytes(level)));
        WBFMM_TRY(build_source_mask(x.src_n, level, smask.p, stream));
        lp.smask = smask.p;
        launches++;
      }
      if (!helm) {
        const int P1 = x.Nin + 1;
        WBFMM_TRY(lapsr.alloc((size_t)kNumOps * P1 * P1 * P1));
        WBFMM_TRY(build_lap_sr_ops<T>(tables, x.Nin, x.width, x.lap_e, lapsr.p, stream));
        lp.lapsr = lapsr.p;
        launches++;
      }
      const int64_t np = (int64_t)1 << (3 * (level - 1));
      const int64_t base = ((np + 127) / 128) * 8;
      int ns = 1;
      while (base * ns < lanes_ctas && ns < 32) ns *= 2;
      lp.nsplit = ns;
      if (ns > 1) {
        const int V = helm ? (x.Nin + 1) * (x.Nin + 1) : (x.Nin + 1) * (x.Nin + 2) / 2;
        WBFMM_TRY(lanes_part.alloc((size_t)ns * 8 * V * np * 2));
        lp.partial_raw = lanes_part.p;
      }
      launches += ns > 1 ? 3 : 2;
      return helm ? launch_m2l_lanes<T, true>(lp, tables, stream)
                  : launch_m2l_lanes<T, false>(lp, tables, stream);
    }
    // split the source lists of coarse levels over several CTAs
    int64_t want = 148 * 8;
    int nsplit = 1;
    while (x.nbox * nsplit < want && nsplit < 16) nsplit *= 2;
    x.nsplit = nsplit;
    if (nsplit > 1) {
      int outlen = helm ? (x.Nout + 1) * (x.Nout + 1) : (x.Nout + 1) * (x.Nout + 2) / 2;
      WBFMM_TRY(partial.alloc((size_t)nsplit * x.nbox * 2 * outlen));
      x.partial = partial.p;
    }
    launches += nsplit > 1 ? 2 : 1;
    return helm ? launch_m2l<T, true>(x, tables, stream)
                : launch_m2l<T, false>(x, tables, stream);
  }

  // The M2L of a level with sparse storage: the lane or tile kernel (the
  // automatic choice, or the one set with set_m2l_kernel 2 / 3) on compact
  // transposed sources, one column per stored source group and a zero
  // column, source parents found through the padded-grid slot map, targets
  // from the level's active lists written at their slots
  int m2l_sparse(int level, const XlateParams<T>& x, int he, bool tiles_ok, bool lanes_ok,
                 int lanes_max) {
    bool dense = false;
    const int tc = !tiles_ok ? 0
                   : helm ? tiles_per_cta<T, true>(x.Nin, &dense, true)
                          : tiles_per_cta<T, false>(x.Nin, nullptr, true);
    bool use_lanes = !he && lanes_ok && (m2l_mode == 2 || (m2l_mode != 3 && x.Nin <= lanes_max));
    if (!use_lanes && tc == 0) use_lanes = !he && lanes_ok;
    if (!use_lanes && tc == 0)
      return set_error(WBFMM_B200_E_ORDER, "sparse level storage: the M2L needs equal orders in [2, 60] at each level");
    const int64_t G = ngroups[level];
    const int se = helm ? he : x.lap_e;
    WBFMM_TRY(lin.alloc(lanes_lin_groups_bytes(G, x.Nin, helm, sizeof(T))));
    WBFMM_TRY((helm ? lanes_to_lin_groups<T, true>(x.cin, G, x.Nin, se, lin.p, stream, use_lanes)
                    : lanes_to_lin_groups<T, false>(x.cin, G, x.Nin, se, lin.p, stream, use_lanes)));
    WBFMM_TRY(pmap.alloc(source_mask_bytes(level) / 8));
    WBFMM_TRY(build_parent_slot_map(gmap[level].p, level, (uint32_t)G, pmap.p, stream));
    LanesParams<T> lp;
    memset(&lp, 0, sizeof(lp));
    lp.level = level; lp.N = x.Nin;
    lp.lin_raw = lin.p; lp.cout = x.cout;
    lp.coax = x.coax; lp.coax_stride = x.coax_stride;
    lp.width = x.width; lp.tmask = x.tmask; lp.lap_e = x.lap_e;
    lp.helm_e = he;
    lp.act = act[level].p; lp.act_n = act_n[level].p;
    lp.pmap = pmap.p; lp.gmap = gmap[level].p; lp.lin_stride = G + 1;
    lp.boxmajor = use_lanes ? 1 : 0;
    WBFMM_TRY(smask.alloc(source_mask_bytes(level)));
    WBFMM_TRY(build_source_mask(x.src_n, level, smask.p, stream));
    lp.smask = smask.p;
    if (!helm) {
      const int P1 = x.Nin + 1;
      WBFMM_TRY(lapsr.alloc((size_t)kNumOps * P1 * P1 * P1));
      WBFMM_TRY(build_lap_sr_ops<T>(tables, x.Nin, x.width, x.lap_e, lapsr.p, stream));
      lp.lapsr = lapsr.p;
      launches++;
    }
    if (!use_lanes && dense) {
      WBFMM_TRY(hcx.alloc(helm_coax_rows_count(x.Nin)));
      WBFMM_TRY(build_helm_coax_rows<T>(x.coax, x.coax_stride, x.Nin, hcx.p, stream));
      lp.hcx = hcx.p;
      launches++;
    }
    const int64_t np = (int64_t)1 << (3 * (level - 1));
    int ns = 1;
    if (use_lanes) {
      const int64_t base = ((np + 127) / 128) * 8;
      while (base * ns < lanes_ctas && ns < 32) ns *= 2;
    } else {
      const int64_t ctas = ((np + tc - 1) / tc) * 8;
      while (ctas * ns < 2 * 148 && ns < 32) ns *= 2;
    }
    lp.nsplit = ns;
    if (ns > 1) {
      const int V = helm ? (x.Nin + 1) * (x.Nin + 1) : (x.Nin + 1) * (x.Nin + 2) / 2;
      WBFMM_TRY(lanes_part.alloc((size_t)ns * 8 * V * np * 2));
      lp.partial_raw = lanes_part.p;
    }
    launches += 3 + (ns > 1 ? 2 : 1);
    if (use_lanes)
      return helm ? launch_m2l_lanes<T, true>(lp, tables, stream)
                  : launch_m2l_lanes<T, false>(lp, tables, stream);
    return helm ? launch_m2l_tiles<T, true>(lp, tables, stream)
                : launch_m2l_tiles<T, false>(lp, tables, stream);
  }

  // The Laplace M2L of a level on the tensor cores (m2l_tc.cu).
  int m2l_tc(int level, const XlateParams<T>& x) {
    LapTcParams lp;
    memset(&lp, 0, sizeof(lp));
    lp.level = level;
    lp.P = x.Nin;
    WBFMM_TRY(tc_lap_ops(lp.P, stream, &lp));
    // w^-n in, w^-(n+1) out, per degree (finite in FP32 within the range rule)
    const double w = width(level);
    for (int n = 0; n <= lp.P; n++) {
      lp.sc.in[n] = (float)pow(w, -(double)n);
      lp.sc.out[n] = (float)pow(w, -(double)(n + 1));
      if (!std::isfinite(lp.sc.out[n]) || !std::isfinite(lp.sc.in[n]))
        return set_error(WBFMM_B200_E_ORDER, "tensor-core M2L: level scaling out of the FP32 range");
    }
    lp.cout = (float*)x.cout;
    lp.tmask = x.tmask;
    if (x.tmask && act[level].p) { lp.act = act[level].p; lp.act_n = act_n[level].p; }
    if (x.tmask) {
      WBFMM_TRY(smask.alloc(source_mask_bytes(level)));
      WBFMM_TRY(build_source_mask(x.src_n, level, smask.p, stream));
      lp.smask = smask.p;
      launches++;
    }
    lp.err = flag.p + 2;
    const int64_t np = (int64_t)1 << (3 * (level - 1));
    const int64_t ctas = ((np + 127) / 128) * 8;
    // the tensor core's FP32 accumulation does not round to nearest: its
    // error grows with the number of products summed into one accumulator,
    // so each CTA takes at most 6 of the 189 offsets (and enough CTAs to
    // fill the GPU); the splits' partial sums are added in FP32.  Measured
    // on 300,000 points at depth 5 (orders 10-14), the potentials differ
    // from the tile kernel's by 1.8e-5 (relative L2) with all 189 offsets
    // in one accumulator, 2.2e-6 with 12 and 1.4e-6 with 6
    int ns = 32;
    while (ctas * ns < 148 && ns < 64) ns *= 2;
    lp.nsplit = ns;
    if (ns > 1) {
      WBFMM_TRY(tc_part.alloc((size_t)ns * 8 * (lp.P + 1) * (lp.P + 1) * np));
      lp.partial = tc_part.p;
    }
    WBFMM_TRY(lin.alloc(tc_lin_bytes(level, lp.P)));
    tc_used = true;
    launches += ns > 1 ? 3 : 2;
    return launch_m2l_tc(lp, (const float*)x.cin, lin.p, stream);
  }

  int l2l(int level) override {
    if (level < 2 || level >= depth) return set_error(WBFMM_B200_E_ARG, "L2L level must be in [2, depth-1]");
    WBFMM_TRY(build_operators());
    WBFMM_TRY(prepare_sparse());
    XlateParams<T> d = xparams();
    d.level = level + 1;
    d.nbox = (int64_t)1 << (3 * level);
    d.Nin = cfg.order_r[level]; d.Nout = cfg.order_r[level + 1];
    d.cin = mpr[level].p; d.cout = mpr[level + 1].p;
    d.coax = helm ? ss_ptr[level + 1] : nullptr;
    d.width = (T)width(level + 1);
    if (cfg.sparse) {
      // one CTA per stored group of the children (every box of a stored
      // group is written)
      d.nbox = ngroups[level + 1];
      d.glist = glist[level + 1].p;
      d.gmap = gmap[level].p;
    }
    launches++;
    return helm ? launch_l2l<T, true>(d, tables, stream)
                : launch_l2l<T, false>(d, tables, stream);
  }

  EvalParams<T> eparams() {
    EvalParams<T> e;
    memset(&e, 0, sizeof(e));
    e.ntgt = ntgt; e.level = depth; e.N = cfg.order_r[depth];
    e.x0 = cfg.x0[0]; e.y0 = cfg.x0[1]; e.z0 = cfg.x0[2]; e.wb = width(depth);
    e.k = (T)cfg.k;
    e.tx = tx.p; e.ty = ty.p; e.tz = tz.p;
    e.tperm = tperm.p; e.tbox = tbox.p; e.tstart = tstart.p; e.tcount = tcount.p;
    e.box_i = box_i[depth].p; e.box_n = box_n[depth].p;
    e.x = sx.p; e.y = sy.p; e.z = sz.p;
    e.q = have_q ? sq.p : nullptr; e.dip = have_dip ? sdip.p : nullptr;
    e.nx = snx.p; e.ny = sny.p; e.nz = snz.p;
    e.mpr = mpr[depth].p;
    e.pot = (cfg.field & eval_field & WBFMM_B200_POTENTIAL) ? pot.p : nullptr;
    e.grad = (cfg.field & eval_field & WBFMM_B200_GRADIENT) ? grad.p : nullptr;
    e.nbox = (int64_t)1 << (3 * depth);
    e.gmap = cfg.sparse ? gmap[depth].p : nullptr;
    return e;
  }

  int evaluate() override {
    if (ntgt <= 0) return set_error(WBFMM_B200_E_STATE, "set_targets first");
    WBFMM_TRY(prepare_sparse());
    EvalParams<T> e = eparams();
    launches += eval_neighbours ? 2 : 1;
    if (helm) WBFMM_TRY((launch_l2p<T, true>(e, stream)));
    else WBFMM_TRY((launch_l2p<T, false>(e, stream)));
    if (!eval_neighbours) return 0;
    if constexpr (sizeof(T) == 8)
      if (cfg.near_fp32) return p2p_fp32(e);
    return helm ? launch_p2p<T, true>(e, stream) : launch_p2p<T, false>(e, stream);
  }

  // FP64 solver, near_fp32: the near field in the FP32 form's P2P kernel on
  // FP32 copies of the strengths and normals (positions stay FP64), its
  // results added to the FP64 fields
  int p2p_fp32(const EvalParams<T>& e) {
    EvalParams<float> f;
    memset(&f, 0, sizeof(f));
    f.ntgt = e.ntgt; f.level = e.level; f.N = e.N;
    f.x0 = e.x0; f.y0 = e.y0; f.z0 = e.z0; f.wb = e.wb;
    f.k = (float)e.k;
    f.tx = e.tx; f.ty = e.ty; f.tz = e.tz;
    f.tperm = e.tperm; f.tbox = e.tbox; f.tstart = e.tstart; f.tcount = e.tcount;
    f.box_i = e.box_i; f.box_n = e.box_n;
    f.x = e.x; f.y = e.y; f.z = e.z;
    f.nbox = e.nbox;
    const int w = helm ? 2 : 1;
    const int64_t ns = nsrc, nt = ntgt;
    auto narrow = [&](const T* src, DBuf<float>& dst, int64_t n, const float** out) -> int {
      if (!src) { *out = nullptr; return 0; }
      WBFMM_TRY(dst.alloc((size_t)n));
      WBFMM_TRY(launch_narrow((const double*)src, dst.p, n, stream));
      *out = dst.p;
      return 0;
    };
    WBFMM_TRY(narrow(e.q, n32_q, ns * w, &f.q));
    WBFMM_TRY(narrow(e.dip, n32_dip, ns * w, &f.dip));
    if (e.dip) {
      WBFMM_TRY(narrow(e.nx, n32_nx, ns, &f.nx));
      WBFMM_TRY(narrow(e.ny, n32_ny, ns, &f.ny));
      WBFMM_TRY(narrow(e.nz, n32_nz, ns, &f.nz));
    }
    if (e.pot) {
      WBFMM_TRY(n32_pot.alloc((size_t)(nt * w)));
      WBFMM_CUDA(cudaMemsetAsync(n32_pot.p, 0, sizeof(float) * nt * w, stream));
      f.pot = n32_pot.p;
    }
    if (e.grad) {
      WBFMM_TRY(n32_grad.alloc((size_t)(nt * 3 * w)));
      WBFMM_CUDA(cudaMemsetAsync(n32_grad.p, 0, sizeof(float) * nt * 3 * w, stream));
      f.grad = n32_grad.p;
    }
    WBFMM_TRY((helm ? launch_p2p<float, true>(f, stream) : launch_p2p<float, false>(f, stream)));
    if (e.pot) WBFMM_TRY(launch_add_widened((double*)e.pot, n32_pot.p, nt * w, stream));
    if (e.grad) WBFMM_TRY(launch_add_widened((double*)e.grad, n32_grad.p, nt * 3 * w, stream));
    launches += 2 + (e.q ? 1 : 0) + (e.dip ? 4 : 0) + (e.pot ? 1 : 0) + (e.grad ? 1 : 0);
    return 0;
  }

  int run() override {
    WBFMM_TRY(run_queued());
    return wait();
  }

  // every pass queued on the stream; with deferred checks, the copy of the
  // domain-check flags too
  int run_queued() override {
    if (nsrc <= 0 || ntgt <= 0) return set_error(WBFMM_B200_E_STATE, "sources and targets must be set");
    WBFMM_TRY(build_operators());
    return passes();
  }

  // P2M, upward, downward, evaluation (and the flags' copy with deferred
  // checks); stage events unless the stream is being captured
  int passes() {
    auto mark = [&](int i) { if (!capturing) cudaEventRecord(ev[i], stream); };
    mark(4);
    WBFMM_TRY(leaf_expansions());
    mark(5);
    for (int l = depth; l >= 3; l--) WBFMM_TRY(upward(l));
    mark(6);
    for (int l = 2; l <= depth; l++) WBFMM_TRY(downward(l));
    mark(7);
    WBFMM_TRY(evaluate());
    mark(2);
    if (async_checks && hflag)
      WBFMM_CUDA(cudaMemcpyAsync(hflag, flag.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, stream));
    return 0;
  }

  // The passes as one CUDA graph launch.  The first call after anything
  // they depend on changed (sources, targets, tables, options, the strength
  // buffers) runs them as usual, which sizes every work buffer, then
  // captures the same launches; later calls launch the graph.  Stage times
  // stay those of the last call that ran the passes directly.
  int run_graph() override {
    if (nsrc <= 0 || ntgt <= 0) return set_error(WBFMM_B200_E_STATE, "sources and targets must be set");
    const GraphSig sig{gen, (const void*)sq.p, (const void*)sdip.p, have_q, have_dip};
    if (gexec && ops_ready && sig == gsig) {
      WBFMM_CUDA(cudaGraphLaunch(gexec, stream));
      launches += glaunches;
      return 0;
    }
    WBFMM_TRY(run_queued());
    if (gexec) { cudaGraphExecDestroy(gexec); gexec = nullptr; }
    const int64_t l0 = launches;
    cudaGraph_t g = nullptr;
    WBFMM_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    capturing = true;
    const int rc = passes();
    capturing = false;
    const cudaError_t e = cudaStreamEndCapture(stream, &g);
    glaunches = launches - l0;
    launches = l0;                      // captured, not launched
    if (rc || e != cudaSuccess) {
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
      return rc ? rc : set_cuda_error(e, __FILE__, __LINE__);
    }
    const cudaError_t ei = cudaGraphInstantiate(&gexec, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
      gexec = nullptr;
      cudaGetLastError();
      return set_cuda_error(ei, __FILE__, __LINE__);
    }
    gsig = sig;
    return 0;
  }

  // the host waits for the queued solve: stage times, deferred checks
  int wait() override {
    WBFMM_CUDA(cudaStreamSynchronize(stream));
    float t;
    if (cudaEventElapsedTime(&t, ev[0], ev[1]) == cudaSuccess) stage_ms[0] = t;
    stage_ms[1] = 0;
    if (cudaEventElapsedTime(&t, ev[4], ev[5]) == cudaSuccess) stage_ms[2] = t;
    if (cudaEventElapsedTime(&t, ev[5], ev[6]) == cudaSuccess) stage_ms[3] = t;
    if (cudaEventElapsedTime(&t, ev[6], ev[7]) == cudaSuccess) stage_ms[4] = t;
    if (cudaEventElapsedTime(&t, ev[7], ev[2]) == cudaSuccess) stage_ms[5] = t;
    cudaGetLastError();
    if (tc_used && !async_checks) {
      int err = 0;
      WBFMM_CUDA(cudaMemcpy(&err, flag.p + 2, sizeof(int), cudaMemcpyDeviceToHost));
      if (err) return set_error(WBFMM_B200_E_STATE, "tensor-core M2L: a wait ran out");
    }
    return check_flags();
  }

  // set_sources / set_targets queue their domain checks; run / wait report
  int set_deferred_checks(int on) override {
    if (on && !hflag) {
      WBFMM_CUDA(cudaMallocHost(&hflag, 3 * sizeof(int)));
      hflag[0] = 0x7fffffff; hflag[1] = 0; hflag[2] = 0;
    }
    async_checks = on != 0;
    return 0;
  }

  // Served form: every pass queued on the stream, no host wait.
  int run_async() {
    if (nsrc <= 0 || ntgt <= 0) return set_error(WBFMM_B200_E_STATE, "sources and targets must be set");
    WBFMM_TRY(build_operators());
    WBFMM_TRY(leaf_expansions());
    for (int l = depth; l >= 3; l--) WBFMM_TRY(upward(l));
    for (int l = 2; l <= depth; l++) WBFMM_TRY(downward(l));
    return evaluate();
  }

  // Served form: queue the copies of the fields (FP64, original target
  // order) into pinned host arrays (kind cudaMemcpyDeviceToHost) or device
  // arrays (cudaMemcpyDeviceToDevice), and of the domain-check flags.
  int fetch_async(double* hpot, double* hgrad, cudaMemcpyKind kind) {
    const int w = helm ? 2 : 1;
    const size_t np = hpot ? (size_t)ntgt * w : 0;
    const size_t ng = hgrad ? (size_t)ntgt * 3 * w : 0;
    if (np && !pot.p) return set_error(WBFMM_B200_E_STATE, "potential was not requested");
    if (ng && !grad.p) return set_error(WBFMM_B200_E_STATE, "gradient was not requested");
    const double* fp = (const double*)pot.p;
    const double* fg = (const double*)grad.p;
    if (sizeof(T) != 8) {
      WBFMM_TRY(out64.alloc(np + ng));
      if (np) k_widen<T><<<(unsigned)((np + 255) / 256), 256, 0, stream>>>(pot.p, out64.p, (int64_t)np);
      if (ng) k_widen<T><<<(unsigned)((ng + 255) / 256), 256, 0, stream>>>(grad.p, out64.p + np, (int64_t)ng);
      fp = out64.p;
      fg = out64.p + np;
      launches += (np ? 1 : 0) + (ng ? 1 : 0);
    }
    if (np) WBFMM_CUDA(cudaMemcpyAsync(hpot, fp, sizeof(double) * np, kind, stream));
    if (ng) WBFMM_CUDA(cudaMemcpyAsync(hgrad, fg, sizeof(double) * ng, kind, stream));
    if (async_checks && hflag)
      WBFMM_CUDA(cudaMemcpyAsync(hflag, flag.p, 3 * sizeof(int), cudaMemcpyDeviceToHost, stream));
    return 0;
  }

  // Served form, after the stream has drained: the deferred domain checks
  // and the tensor-core M2L's bounded waits.
  int check_flags() const {
    if (!(async_checks && hflag)) return 0;
    if (hflag[2]) return set_error(WBFMM_B200_E_STATE, "tensor-core M2L: a wait ran out");
    return domain_error(hflag[0], hflag[1]);
  }

  // ------------------------------------------------------------ outputs
  int fetch(DBuf<T>& src, size_t n, double* dst, int on_device) {
    const double* from = nullptr;
    if (sizeof(T) == 8) {
      from = (const double*)src.p;
    } else {
      WBFMM_TRY(out64.alloc(n));
      k_widen<T><<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(src.p, out64.p, (int64_t)n);
      from = out64.p;
    }
    WBFMM_CUDA(cudaMemcpyAsync(dst, from, sizeof(double) * n,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               stream));
    WBFMM_CUDA(cudaStreamSynchronize(stream));
    return 0;
  }

  // Laplace: second derivatives of the potential at the targets into the
  // device array hess[9 ntgt] (original order, d_a d_b at 3 a + b), from
  // the leaf regular expansions (after the downward pass) and, with
  // neighbours, the monopoles of the 27 neighbour boxes
  int hessian(double* hess, int neighbours) override {
    if (helm) return set_error(WBFMM_B200_E_ARG, "the Hessian is for Laplace solvers");
    if (cfg.sparse) return set_error(WBFMM_B200_E_ARG, "the Hessian needs dense level storage");
    if (nsrc <= 0 || ntgt <= 0) return set_error(WBFMM_B200_E_STATE, "sources and targets must be set");
    if (neighbours && have_dip)
      return set_error(WBFMM_B200_E_ARG, "the near-field Hessian takes monopole sources only");
    const int N = cfg.order_r[depth];
    const int64_t nb = (int64_t)1 << (3 * depth);
    if (N >= 1) {
      const size_t len = level_len(depth, N - 1);
      WBFMM_TRY(hess_d.alloc(3 * len));
      WBFMM_TRY(hess_g.alloc(9 * (size_t)ntgt));
      WBFMM_TRY(launch_laplace_deriv<T>(mpr[depth].p, N, nb, hess_d.p, hess_d.p + len,
                                        hess_d.p + 2 * len, stream));
      for (int a = 0; a < 3; a++) {
        EvalParams<T> e = eparams();
        e.N = N - 1;
        e.mpr = hess_d.p + a * len;
        e.pot = nullptr;
        e.grad = hess_g.p + (size_t)a * 3 * ntgt;
        WBFMM_TRY((launch_l2p<T, false>(e, stream)));
      }
      WBFMM_TRY(launch_hess_gather<T>(hess_g.p, ntgt, hess, stream));
      launches += 5;
    } else {
      WBFMM_TRY(launch_hess_gather<T>(nullptr, ntgt, hess, stream));
      launches++;
    }
    if (neighbours && have_q) {
      WBFMM_TRY(launch_p2p_hessian<T>(eparams(), hess, stream));
      launches++;
    }
    return 0;
  }

  // precomputed target bases for repeated potential evaluations at these
  // targets (target_bases.cu): held until the sources or targets change
  int target_bases() override {
    if (nsrc <= 0 || ntgt <= 0) return set_error(WBFMM_B200_E_STATE, "sources and targets must be set");
    if (cfg.sparse) return set_error(WBFMM_B200_E_ARG, "target bases need dense level storage");
    const EvalParams<T> e = eparams();
    int64_t np = 0;
    WBFMM_TRY(tl_off.alloc((size_t)ntgt + 1));
    WBFMM_TRY(tl_offsets<T>(e, tl_off.p, &np, stream));
    const int w = helm ? 2 : 1;
    tl_dip = have_normals;
    WBFMM_TRY(tl_src.alloc((size_t)np + 1));
    WBFMM_TRY(tl_wq.alloc(((size_t)np + 1) * w));
    if (tl_dip) WBFMM_TRY(tl_wd.alloc(((size_t)np + 1) * w));
    WBFMM_TRY(tl_basis.alloc((size_t)ncoefs(cfg.order_r[depth]) * ntgt * w));
    T* wd = tl_dip ? tl_wd.p : nullptr;
    WBFMM_TRY((helm ? tl_fill<T, true>(e, tl_off.p, tl_src.p, tl_wq.p, wd, tl_basis.p, stream)
                    : tl_fill<T, false>(e, tl_off.p, tl_src.p, tl_wq.p, wd, tl_basis.p, stream)));
    launches += 3;
    tl_geo = geo;
    return 0;
  }

  // the potential at the targets from the bases, the leaf regular
  // expansions (after the downward pass) and, with neighbours, the current
  // strengths
  int evaluate_bases(int neighbours) override {
    if (tl_geo != geo)
      return set_error(WBFMM_B200_E_STATE, "target bases must be computed for these sources and targets");
    if (!(cfg.field & WBFMM_B200_POTENTIAL))
      return set_error(WBFMM_B200_E_ARG, "the bases give the potential field");
    EvalParams<T> e = eparams();
    e.pot = pot.p;
    if (!neighbours) e.q = e.dip = nullptr;
    const T* wd = tl_dip ? tl_wd.p : nullptr;
    WBFMM_TRY((helm ? tl_apply<T, true>(e, tl_basis.p, tl_off.p, tl_src.p, tl_wq.p, wd, stream)
                    : tl_apply<T, false>(e, tl_basis.p, tl_off.p, tl_src.p, tl_wq.p, wd, stream)));
    launches += 2;
    return 0;
  }

  int get_field(double* po, double* go, int on_device) override {
    const int w = helm ? 2 : 1;
    if (po) {
      if (!pot.p) return set_error(WBFMM_B200_E_STATE, "potential was not requested");
      WBFMM_TRY(fetch(pot, (size_t)ntgt * w, po, on_device));
    }
    if (go) {
      if (!grad.p) return set_error(WBFMM_B200_E_STATE, "gradient was not requested");
      WBFMM_TRY(fetch(grad, (size_t)ntgt * 3 * w, go, on_device));
    }
    return 0;
  }

  int get_tree(uint32_t* ipo, uint32_t* bi, uint32_t* bn, int level) override {
    if (nsrc <= 0) return set_error(WBFMM_B200_E_STATE, "no tree");
    if (level < 0 || level > depth) return set_error(WBFMM_B200_E_ARG, "bad level");
    size_t nb = (size_t)1 << (3 * level);
    if (ipo) WBFMM_CUDA(cudaMemcpyAsync(ipo, ip.p, sizeof(uint32_t) * nsrc, cudaMemcpyDeviceToHost, stream));
    if (bi) WBFMM_CUDA(cudaMemcpyAsync(bi, box_i[level].p, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost, stream));
    if (bn) WBFMM_CUDA(cudaMemcpyAsync(bn, box_n[level].p, sizeof(uint32_t) * nb, cudaMemcpyDeviceToHost, stream));
    WBFMM_CUDA(cudaStreamSynchronize(stream));
    return 0;
  }

  int get_coefficients(int level, double* ms, double* mr) override {
    if (level < 1 || level > depth) return set_error(WBFMM_B200_E_ARG, "bad level");
    if (cfg.sparse) {
      // the dense Layout L arrays, zero outside the stored groups
      WBFMM_TRY(prepare_sparse());
      const int w = helm ? 2 : 1;
      auto one = [&](DBuf<T>& a, int p, double* out) -> int {
        const size_t dl = level_len(level, p);
        WBFMM_TRY(dense_tmp.alloc(dl));
        WBFMM_TRY(sparse_expand<T>(a.p, glist[level].p, ngroups[level],
                                   (int64_t)8 * ncoefs(p) * w, dense_tmp.p, (int64_t)dl, stream));
        launches++;
        return fetch(dense_tmp, dl, out, 0);
      };
      if (ms) WBFMM_TRY(one(mps[level], cfg.order_s[level], ms));
      if (mr) WBFMM_TRY(one(mpr[level], cfg.order_r[level], mr));
      return 0;
    }
    if (ms) WBFMM_TRY(fetch(mps[level], level_len(level, cfg.order_s[level]), ms, 0));
    if (mr) WBFMM_TRY(fetch(mpr[level], level_len(level, cfg.order_r[level]), mr, 0));
    return 0;
  }

  int sources() const override { return nsrc; }
  int targets() const override { return ntgt; }
  void invalidate_operators() override { ops_ready = false; gen++; }
  void set_m2l_kernel(int mode) override { m2l_mode = mode; gen++; }
  void set_p2m_accumulate(int on) override { p2m_accumulate = on != 0; gen++; }
  void set_evaluation(int field, int neighbours) override {
    gen++;
    eval_field = field;
    eval_neighbours = neighbours != 0;
  }
  int adopt_coefficients(int level, void* ms, void* mr) override {
    if (level < 1 || level > depth) return set_error(WBFMM_B200_E_ARG, "bad level");
    if (cfg.sparse) return set_error(WBFMM_B200_E_ARG, "adopted arrays need dense level storage");
    gen++;
    if (ms) mps[level].adopt((T*)ms, level_len(level, cfg.order_s[level]), cfg.managed != 0);
    if (mr) mpr[level].adopt((T*)mr, level_len(level, cfg.order_r[level]), cfg.managed != 0);
    return 0;
  }

  int coefficient_pointers(int level, void** ms, void** mr) override {
    if (level < 1 || level > depth) return set_error(WBFMM_B200_E_ARG, "bad level");
    if (cfg.sparse) return set_error(WBFMM_B200_E_ARG, "Layout L pointers need dense level storage");
    if (ms) *ms = mps[level].p;
    if (mr) *mr = mpr[level].p;
    return 0;
  }

  // stored groups of eight boxes of a level (dense: 8^(level-1)) and the
  // bytes of its two coefficient arrays; level 0: totals over levels 1..depth
  int coefficient_storage(int level, int64_t* groups, int64_t* bytes) override {
    if (level < 0 || level > depth) return set_error(WBFMM_B200_E_ARG, "bad level");
    if (tree_only) return set_error(WBFMM_B200_E_STATE, "no coefficient arrays");
    if (cfg.sparse) WBFMM_TRY(prepare_sparse());
    int64_t g = 0, by = 0;
    for (int l = level ? level : 1; l <= (level ? level : depth); l++) {
      g += cfg.sparse ? ngroups[l] : (int64_t)1 << (3 * (l - 1));
      by += (int64_t)sizeof(T) * (int64_t)(coef_len(l, cfg.order_s[l]) + coef_len(l, cfg.order_r[l]));
    }
    if (groups) *groups = g;
    if (bytes) *bytes = by;
    return 0;
  }
};

}  // namespace wbfmm
