// The C ABI declared in include/wbfmm_b200.h over the solver (solver.h).
#include "solver.h"

using namespace wbfmm;

namespace wbfmm {
cudaMemPool_t library_pool() {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
    cudaGetLastError();
    return nullptr;
  }
  std::lock_guard<std::mutex> g(mu);
  if (!pools[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pl = nullptr;
    if (cudaMemPoolCreate(&pl, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t thr = UINT64_MAX;
    int off = 0;
    cudaMemPoolSetAttribute(pl, cudaMemPoolAttrReleaseThreshold, &thr);
    cudaMemPoolSetAttribute(pl, cudaMemPoolReuseAllowInternalDependencies, &off);
    pools[dev] = pl;
  }
  return pools[dev];
}
}  // namespace wbfmm


// -------------------------------------------------------------- C ABI
extern "C" {

const char* wbfmm_b200_last_error(void) { return wbfmm::last_error(); }

int wbfmm_b200_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int wbfmm_b200_solver_create(wbfmm_b200_solver_t** s,
                             const wbfmm_b200_config_t* cfg, void* stream) {
  if (!s || !cfg) return set_error(WBFMM_B200_E_ARG, "null argument");
  *s = nullptr;
  if (wbfmm_b200_device_count() < 1)
    return set_error(WBFMM_B200_E_NOGPU, "no CUDA device is available");
  wbfmm_b200_solver* o = nullptr;
  int rc;
  if (cfg->precision == WBFMM_B200_FP32) {
    auto* x = new Solver<float>();
    rc = x->init(cfg, stream);
    o = x;
  } else if (cfg->precision == WBFMM_B200_FP64) {
    auto* x = new Solver<double>();
    rc = x->init(cfg, stream);
    o = x;
  } else {
    return set_error(WBFMM_B200_E_ARG, "precision must be FP64 (0) or FP32 (1)");
  }
  if (rc) { delete o; return rc; }
  *s = o;
  return 0;
}

int wbfmm_b200_solver_destroy(wbfmm_b200_solver_t* s) {
  delete s;
  return 0;
}

// log10 of the large-order magnitudes: |h_n(x)| ~ (2n-1)!!/x^(n+1) and
// j_n(x) ~ x^n/(2n+1)!! for n > x
static double log10_dfact(int n) {   // log10 n!! for odd n
  double s = 0;
  for (int i = n; i > 1; i -= 2) s += log10((double)i);
  return s;
}

int wbfmm_b200_fp32_range_ok(const wbfmm_b200_config_t* c) {
  if (!c) return 0;
  for (int l = 2; l <= c->depth; l++) {
    const int p = std::max(c->order_s[l], c->order_r[l]);
    const double w = c->D / (double)(1 << l);
    if (c->problem == WBFMM_B200_LAPLACE) {
      // scale-free coaxial tables hold (n+n')! / ... up to n + n' = 2p
      if (p > 16) return 0;
      // for strengths of order one, local coefficients of degree n scale
      // like (2w)^-(n+1) and multipole coefficients like (0.87 w)^n: keep
      // both within 1e+-30, leaving the rest of the range to the sums
      if (fabs((c->order_r[l] + 1) * log10(2.0 * w)) > 30.0) return 0;
      if (fabs(c->order_s[l] * log10(0.87 * w)) > 30.0) return 0;
      continue;
    }
    const double x = 2.0 * c->k * w;            // nearest list-4 distance
    const int N = 2 * p;
    // the level's (S|R) table holds degrees n + l up to 2p, about
    // (2N-1)!! / x^(N+1): beyond the FP32 range the M2L runs in its scaled
    // form (helm_m2l_exp; tile kernel, equal orders), exact in itself, but
    // admitted only for x >= 0.8: at smaller k w the real parts of the
    // fields come from the cancellation of much larger imaginary-part terms
    // (h_n(x) ~ -i y_n(x)), and the FP32 form was measured to lose accuracy
    // there (relative L2 against FP64 at order 14: below 1e-6 for x >= 0.8,
    // 2e-6 at x = 0.5, 9e-6 at x = 0.15; unchanged by the scaling)
    if (x < N && log10_dfact(2 * N - 1) - (N + 1) * log10(x) > 36.0 &&
        !(wbfmm::helm_m2l_scalable(c->order_s[l], c->order_r[l]) && x >= 0.8))
      return 0;
    // local coefficients, stored unscaled, reach about (2p-1)!! / x^(p+1)
    // per unit strength at the nearest list-4 distance
    if (x < p && log10_dfact(2 * p - 1) - (p + 1) * log10(x) > 34.0) return 0;
    if (l == c->depth) {
      const double xr = 0.5 * c->k * w;         // a typical leaf radius
      if (xr < p && p * log10(xr) - log10_dfact(2 * p + 1) < -36.0) return 0;
    }
  }
  return 1;
}

int64_t wbfmm_b200_footprint(const wbfmm_b200_config_t* c, int64_t ns,
                             int64_t nt) {
  if (!c) return -1;
  const int64_t w = c->problem == WBFMM_B200_HELMHOLTZ ? 2 : 1;
  const int64_t ts = c->precision == WBFMM_B200_FP32 ? 4 : 8;
  int64_t b = 0, mps_max = 0;
  for (int l = 1; l <= c->depth; l++) {
    int64_t nb = (int64_t)1 << (3 * l);
    int64_t ms = nb * w * ts * (int64_t)(c->order_s[l] + 1) * (c->order_s[l] + 1);
    b += ms + nb * w * ts * (int64_t)(c->order_r[l] + 1) * (c->order_r[l] + 1);
    b += nb * 8;  // box ranges
    if (ms > mps_max) mps_max = ms;
  }
  // points, sort keys and scratch, strengths, normals
  b += ns * (24 + 8 + 4 + 12 + 24 + 2 * w * ts + 3 * ts);
  // targets, their keys and boxes, fields and their FP64 copies
  b += nt * (24 + 24 + 8 + 4 + 4 + 4 * w * ts + 4 * w * 8);
  b += ((int64_t)1 << (3 * c->depth)) * 8;
  // skip_empty: target masks (1 byte) and M2L lists (4 bytes) of every
  // level, sum_l 8^l < 8^depth * 8/7
  if (c->skip_empty) b += ((int64_t)1 << (3 * c->depth)) * 6;
  // M2L working copies: the transposed, halo-padded sources and split sums
  b += 2 * mps_max;
  return b;
}

#define SOLVER_CALL(expr)                                            \
  do {                                                               \
    if (!s) return set_error(WBFMM_B200_E_ARG, "null solver");       \
    return (expr);                                                   \
  } while (0)

int wbfmm_b200_set_sources(wbfmm_b200_solver_t* s, int n, const double* xs,
                           int xstr, const double* normals, int nstr,
                           int on_device) {
  SOLVER_CALL(s->set_sources(n, xs, xstr, normals, nstr, on_device));
}
int wbfmm_b200_set_strengths(wbfmm_b200_solver_t* s, const double* q, int qstr,
                             const double* d, int dstr, int on_device) {
  SOLVER_CALL(s->set_strengths(q, qstr, d, dstr, on_device));
}
int wbfmm_b200_set_targets(wbfmm_b200_solver_t* s, int n, const double* xt,
                           int tstr, int on_device) {
  SOLVER_CALL(s->set_targets(n, xt, tstr, on_device));
}
int wbfmm_b200_build_operators(wbfmm_b200_solver_t* s) { SOLVER_CALL(s->build_operators()); }
int wbfmm_b200_leaf_expansions(wbfmm_b200_solver_t* s) { SOLVER_CALL(s->leaf_expansions()); }
int wbfmm_b200_upward_pass(wbfmm_b200_solver_t* s, int level) { SOLVER_CALL(s->upward(level)); }
int wbfmm_b200_downward_pass(wbfmm_b200_solver_t* s, int level) { SOLVER_CALL(s->downward(level)); }
int wbfmm_b200_m2l(wbfmm_b200_solver_t* s, int level) { SOLVER_CALL(s->m2l(level)); }
int wbfmm_b200_l2l(wbfmm_b200_solver_t* s, int level) { SOLVER_CALL(s->l2l(level)); }
int wbfmm_b200_evaluate(wbfmm_b200_solver_t* s) { SOLVER_CALL(s->evaluate()); }
int wbfmm_b200_run(wbfmm_b200_solver_t* s) { SOLVER_CALL(s->run()); }
int wbfmm_b200_run_async(wbfmm_b200_solver_t* s) { SOLVER_CALL(s->run_queued()); }
int wbfmm_b200_run_graph(wbfmm_b200_solver_t* s) { SOLVER_CALL(s->run_graph()); }
int wbfmm_b200_wait(wbfmm_b200_solver_t* s) { SOLVER_CALL(s->wait()); }
int wbfmm_b200_target_bases(wbfmm_b200_solver_t* s) { SOLVER_CALL(s->target_bases()); }
int wbfmm_b200_evaluate_bases(wbfmm_b200_solver_t* s, int neighbours) {
  SOLVER_CALL(s->evaluate_bases(neighbours));
}

int wbfmm_b200_laplace_hessian(wbfmm_b200_solver_t* s, double* hess, int neighbours,
                               int on_device) {
  if (!s || !hess) return set_error(WBFMM_B200_E_ARG, "bad Hessian arguments");
  const int nt = s->targets();
  if (nt <= 0) return set_error(WBFMM_B200_E_STATE, "set_targets first");
  cudaStream_t st = s->stream;
  double* hd = hess;
  int rc = 0;
  cudaError_t e = cudaSuccess;
  if (!on_device) e = cudaMallocAsync(&hd, sizeof(double) * 9 * (size_t)nt, st);
  if (e != cudaSuccess) return set_cuda_error(e, __FILE__, __LINE__);
  rc = s->hessian(hd, neighbours);
  if (!rc && !on_device) {
    e = cudaMemcpyAsync(hess, hd, sizeof(double) * 9 * (size_t)nt, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  }
  if (!on_device) cudaFreeAsync(hd, st);
  e = cudaStreamSynchronize(st);
  if (!rc && e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  return rc;
}

int wbfmm_b200_laplace_curl_gradient(wbfmm_b200_solver_t* s, const double* q3, int qstr,
                                     double* out, int on_device) {
  if (!s || !q3 || !out || qstr < 3) return set_error(WBFMM_B200_E_ARG, "bad curl arguments");
  if (s->cfg.problem != WBFMM_B200_LAPLACE)
    return set_error(WBFMM_B200_E_ARG, "the curl needs a Laplace solver");
  if (!(s->cfg.field & WBFMM_B200_GRADIENT))
    return set_error(WBFMM_B200_E_ARG, "the curl needs the gradient field");
  const int ns = s->sources(), nt = s->targets();
  if (ns <= 0 || nt <= 0) return set_error(WBFMM_B200_E_STATE, "sources and targets must be set");
  cudaStream_t st = s->stream;
  double *g = nullptr, *h = nullptr, *qd = nullptr, *od = nullptr;
  int rc = 0;
  cudaError_t e = cudaMallocAsync(&g, sizeof(double) * 9 * (size_t)nt, st);
  if (e == cudaSuccess) e = cudaMallocAsync(&h, sizeof(double) * 27 * (size_t)nt, st);
  const double* q = q3;
  if (e == cudaSuccess && !on_device) {
    e = cudaMallocAsync(&qd, sizeof(double) * (size_t)ns * qstr, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(qd, q3, sizeof(double) * (size_t)ns * qstr, cudaMemcpyHostToDevice, st);
    q = qd;
  }
  if (e == cudaSuccess && !on_device) e = cudaMallocAsync(&od, sizeof(double) * 12 * (size_t)nt, st);
  if (e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  for (int c = 0; c < 3 && !rc; c++) {
    rc = s->set_strengths(q + c, qstr, nullptr, 0, 1);
    if (!rc) rc = s->run();
    if (!rc) rc = s->get_field(nullptr, g + (size_t)c * 3 * nt, 1);
    if (!rc) rc = s->hessian(h + (size_t)c * 9 * nt, 1);
  }
  if (!rc) rc = launch_curl_gradient_combine(g, h, nt, on_device ? out : od, st);
  if (!rc && !on_device) {
    e = cudaMemcpyAsync(out, od, sizeof(double) * 12 * (size_t)nt, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  }
  if (g) cudaFreeAsync(g, st);
  if (h) cudaFreeAsync(h, st);
  if (qd) cudaFreeAsync(qd, st);
  if (od) cudaFreeAsync(od, st);
  e = cudaStreamSynchronize(st);
  if (!rc && e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  return rc;
}

int wbfmm_b200_laplace_curl(wbfmm_b200_solver_t* s, const double* q3, int qstr,
                            double* curl, int on_device) {
  if (!s || !q3 || !curl || qstr < 3) return set_error(WBFMM_B200_E_ARG, "bad curl arguments");
  if (s->cfg.problem != WBFMM_B200_LAPLACE)
    return set_error(WBFMM_B200_E_ARG, "the curl needs a Laplace solver");
  if (!(s->cfg.field & WBFMM_B200_GRADIENT))
    return set_error(WBFMM_B200_E_ARG, "the curl needs the gradient field");
  const int ns = s->sources(), nt = s->targets();
  if (ns <= 0 || nt <= 0) return set_error(WBFMM_B200_E_STATE, "sources and targets must be set");
  cudaStream_t st = s->stream;
  double *g = nullptr, *qd = nullptr, *cd = nullptr;
  int rc = 0;
  cudaError_t e = cudaMallocAsync(&g, sizeof(double) * 9 * (size_t)nt, st);
  // host strengths go to the device whole, so that component c (offset c,
  // stride qstr) is read inside the array
  const double* q = q3;
  if (e == cudaSuccess && !on_device) {
    e = cudaMallocAsync(&qd, sizeof(double) * (size_t)ns * qstr, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(qd, q3, sizeof(double) * (size_t)ns * qstr, cudaMemcpyHostToDevice, st);
    q = qd;
  }
  if (e == cudaSuccess && !on_device) e = cudaMallocAsync(&cd, sizeof(double) * 3 * (size_t)nt, st);
  if (e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  for (int c = 0; c < 3 && !rc; c++) {
    rc = s->set_strengths(q + c, qstr, nullptr, 0, 1);
    if (!rc) rc = s->run();
    if (!rc) rc = s->get_field(nullptr, g + (size_t)c * 3 * nt, 1);
  }
  if (!rc) rc = launch_curl_combine(g, nt, on_device ? curl : cd, st);
  if (!rc && !on_device) {
    e = cudaMemcpyAsync(curl, cd, sizeof(double) * 3 * (size_t)nt, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  }
  if (g) cudaFreeAsync(g, st);
  if (qd) cudaFreeAsync(qd, st);
  if (cd) cudaFreeAsync(cd, st);
  e = cudaStreamSynchronize(st);
  if (!rc && e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  return rc;
}

int wbfmm_b200_selftest_sincos(double xmax, int n, double* err2) {
  if (!err2 || n < 1 || !(xmax > 0)) return set_error(WBFMM_B200_E_ARG, "bad self-test arguments");
  if (wbfmm_b200_device_count() < 1) return set_error(WBFMM_B200_E_NOGPU, "no CUDA device is available");
  return sincos_near_errors(xmax, n, err2);
}
int wbfmm_b200_set_deferred_checks(wbfmm_b200_solver_t* s, int on) {
  SOLVER_CALL(s->set_deferred_checks(on));
}
int wbfmm_b200_synchronize(wbfmm_b200_solver_t* s) {
  if (!s) return set_error(WBFMM_B200_E_ARG, "null solver");
  WBFMM_CUDA(cudaStreamSynchronize(s->stream));
  return 0;
}
int wbfmm_b200_get_field(wbfmm_b200_solver_t* s, double* pot, double* grad,
                         int on_device) {
  SOLVER_CALL(s->get_field(pot, grad, on_device));
}
int wbfmm_b200_get_tree(wbfmm_b200_solver_t* s, uint32_t* ip, uint32_t* bi,
                        uint32_t* bn, int level) {
  SOLVER_CALL(s->get_tree(ip, bi, bn, level));
}
int wbfmm_b200_get_coefficients(wbfmm_b200_solver_t* s, int level, double* ms,
                                double* mr) {
  SOLVER_CALL(s->get_coefficients(level, ms, mr));
}
int wbfmm_b200_coefficient_pointers(wbfmm_b200_solver_t* s, int level,
                                    void** ms, void** mr) {
  SOLVER_CALL(s->coefficient_pointers(level, ms, mr));
}
int wbfmm_b200_coefficient_storage(wbfmm_b200_solver_t* s, int level, int64_t* groups,
                                   int64_t* bytes) {
  SOLVER_CALL(s->coefficient_storage(level, groups, bytes));
}
int wbfmm_b200_set_p2m_accumulate(wbfmm_b200_solver_t* s, int on) {
  if (!s) return set_error(WBFMM_B200_E_ARG, "null solver");
  s->set_p2m_accumulate(on);
  return 0;
}
int wbfmm_b200_set_evaluation(wbfmm_b200_solver_t* s, int field, int neighbours) {
  if (!s) return set_error(WBFMM_B200_E_ARG, "null solver");
  s->set_evaluation(field, neighbours);
  return 0;
}
int wbfmm_b200_adopt_coefficients(wbfmm_b200_solver_t* s, int level, void* ms,
                                  void* mr) {
  SOLVER_CALL(s->adopt_coefficients(level, ms, mr));
}
void* wbfmm_b200_managed_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocManaged(&p, bytes ? bytes : 1) != cudaSuccess) {
    cudaGetLastError();
    set_error(WBFMM_B200_E_NOMEM, "managed allocation failed");
    return nullptr;
  }
  memset(p, 0, bytes);
  return p;
}
void wbfmm_b200_managed_free(void* p) {
  if (p) cudaFree(p);
}
static int tree_structure(int n, const double* pts, int pstr, const double* x0, double D,
                          int depth, int keys_fp32, uint32_t* ip, uint32_t* box_i,
                          uint32_t* box_n) {
  if (depth < 0 || depth > 10) return set_error(WBFMM_B200_E_ARG, "depth must be in [0, 10]");
  if (wbfmm_b200_device_count() < 1)
    return set_error(WBFMM_B200_E_NOGPU, "no CUDA device is available");
  wbfmm_b200_config_t c;
  memset(&c, 0, sizeof(c));
  c.problem = WBFMM_B200_LAPLACE;
  c.depth = depth;
  c.x0[0] = x0[0]; c.x0[1] = x0[1]; c.x0[2] = x0[2];
  c.D = D;
  c.keys_fp32 = keys_fp32;
  Solver<double> sv;
  sv.tree_only = true;
  int rc = sv.init(&c, nullptr);
  if (!rc) rc = sv.set_sources(n, pts, pstr, nullptr, 3, 0);
  if (rc) return rc;
  size_t off = 0;
  for (int l = 0; l <= depth; l++) {
    rc = sv.get_tree(l == 0 ? ip : nullptr, box_i ? box_i + off : nullptr,
                     box_n ? box_n + off : nullptr, l);
    if (rc) return rc;
    off += (size_t)1 << (3 * l);
  }
  return 0;
}
int wbfmm_b200_tree_structure(int n, const double* pts, int pstr,
                              const double* x0, double D, int depth,
                              uint32_t* ip, uint32_t* box_i, uint32_t* box_n) {
  return tree_structure(n, pts, pstr, x0, D, depth, 0, ip, box_i, box_n);
}
int wbfmm_b200_tree_structure_f(int n, const float* pts, int pstr,
                                const float* x0, float D, int depth,
                                uint32_t* ip, uint32_t* box_i, uint32_t* box_n) {
  if (n < 0 || (n > 0 && (!pts || pstr < 3)) || !x0)
    return set_error(WBFMM_B200_E_ARG, "bad points");
  std::vector<double> p64((size_t)3 * (n > 0 ? n : 1));
  for (int i = 0; i < n; i++)
    for (int a = 0; a < 3; a++) p64[3 * (size_t)i + a] = pts[(size_t)i * pstr + a];
  const double o64[3] = {x0[0], x0[1], x0[2]};
  return tree_structure(n, p64.data(), 3, o64, (double)D, depth, 1, ip, box_i, box_n);
}
int wbfmm_b200_set_m2l_kernel(wbfmm_b200_solver_t* s, int mode) {
  if (!s) return set_error(WBFMM_B200_E_ARG, "null solver");
  s->set_m2l_kernel(mode);
  return 0;
}
int wbfmm_b200_invalidate_operators(wbfmm_b200_solver_t* s) {
  if (!s) return set_error(WBFMM_B200_E_ARG, "null solver");
  s->invalidate_operators();
  return 0;
}
int wbfmm_b200_stage_times(wbfmm_b200_solver_t* s, double* ms6) {
  if (!s || !ms6) return set_error(WBFMM_B200_E_ARG, "null argument");
  for (int i = 0; i < 6; i++) ms6[i] = s->stage_ms[i];
  return 0;
}
int64_t wbfmm_b200_kernel_launches(wbfmm_b200_solver_t* s) {
  return s ? s->launches : -1;
}

int wbfmm_b200_solve(const wbfmm_b200_config_t* cfg, int nsrc,
                     const double* xs, const double* q, const double* normals,
                     const double* dipoles, int ntgt, const double* xt,
                     double* pot, double* grad) {
  wbfmm_b200_solver_t* s = nullptr;
  int rc = wbfmm_b200_solver_create(&s, cfg, nullptr);
  if (rc) return rc;
  const int w = cfg->problem == WBFMM_B200_HELMHOLTZ ? 2 : 1;
  rc = s->set_sources(nsrc, xs, 3, normals, 3, 0);
  if (!rc) rc = s->set_strengths(q, w, dipoles, w, 0);
  if (!rc) rc = s->set_targets(ntgt, xt, 3, 0);
  if (!rc) rc = s->run();
  if (!rc) rc = s->get_field(pot, grad, 0);
  delete s;
  return rc;
}

}  // extern "C"
