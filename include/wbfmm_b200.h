/*
 * C ABI of the B200 FMM engine (libwbfmm_b200.so).
 *
 * Plain pointers and sizes only.  Every call returns 0 on success or a
 * negative status; wbfmm_b200_last_error() describes the last failure of the
 * calling thread.  All device work of a solver runs on the CUDA stream given
 * at creation (0 = the library's own stream).
 *
 * The solver replays the reference drivers' call sequence
 * (tools/wbfmm-tree-calc.c.in:270-414, tools/wbfmm-laplace-tree-calc.c.in:
 * 336-460) on the GPU:
 *   tree build          wbfmm_tree_add_points + wbfmm_tree_refine x depth
 *                       (src/boxes.c:118-277)
 *   operators           wbfmm_shift_operators_new / _coaxial_SR_init /
 *                       _coaxial_SS_init (src/shift.c:726-861),
 *                       wbfmm_laplace_coaxial_translate_init (src/laplace.c:727)
 *   P2M                 wbfmm_tree_leaf_expansions (src/boxes.c:341-490),
 *                       wbfmm_tree_laplace_leaf_expansions (src/laplace.c:854)
 *   upward pass         wbfmm_upward_pass, wbfmm_laplace_upward_pass
 *   downward pass       wbfmm_downward_pass_{ref,avx},
 *                       wbfmm_laplace_downward_pass_{ref,avx}
 *   evaluation          wbfmm_tree_box_local_field (src/local.c:264-310),
 *                       wbfmm_laplace_box_field (src/local-laplace.c:1293)
 * with coefficients in the reference's Layout L (groups of eight boxes).
 */
#ifndef WBFMM_B200_H
#define WBFMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WBFMM_B200_LAPLACE 1
#define WBFMM_B200_HELMHOLTZ 2

#define WBFMM_B200_FP64 0 /* plain form: FP64 everywhere */
#define WBFMM_B200_FP32 1 /* FP32 bulk, FP64 tables, FP64 P2P sums */

#define WBFMM_B200_POTENTIAL 1
#define WBFMM_B200_GRADIENT 2

#define WBFMM_B200_MAX_DEPTH 16

/* status codes */
#define WBFMM_B200_OK 0
#define WBFMM_B200_E_ARG (-1)       /* invalid argument */
#define WBFMM_B200_E_DOMAIN (-2)    /* point outside the tree cube */
#define WBFMM_B200_E_ORDER (-3)     /* expansion order unsupported */
#define WBFMM_B200_E_STATE (-4)     /* call out of sequence */
#define WBFMM_B200_E_NOMEM (-5)     /* device allocation failed */
#define WBFMM_B200_E_ADMISSION (-6) /* over the device-memory budget */
#define WBFMM_B200_E_NOGPU (-7)     /* no CUDA device */

typedef struct {
  int problem;        /* WBFMM_B200_LAPLACE or WBFMM_B200_HELMHOLTZ */
  int depth;          /* tree depth, >= 2 */
  int order_s[WBFMM_B200_MAX_DEPTH + 1]; /* singular order per level */
  int order_r[WBFMM_B200_MAX_DEPTH + 1]; /* regular order per level */
  double k;           /* wavenumber (Helmholtz) */
  double x0[3];       /* tree cube origin */
  double D;           /* tree cube width */
  int precision;      /* WBFMM_B200_FP64 or WBFMM_B200_FP32 */
  int field;          /* WBFMM_B200_POTENTIAL | WBFMM_B200_GRADIENT */
  int skip_empty;     /* 1: skip M2L work for boxes with no sources / no
                         targets below (exact for the fields; the regular
                         expansions of target-free boxes are then left 0) */
  int managed;        /* 1: coefficient arrays in CUDA managed memory so the
                         host can read them in place */
  int leaf_order;     /* 1: sort the sources by leaf box only (the top
                         3*depth Morton bits, stable): points inside a leaf
                         keep their input order instead of the reference's
                         full-key order (t->ip differs inside leaves; boxes
                         and fields do not); fewer radix passes */
  int keys_fp32;      /* 1: Morton keys, domain checks and target boxes in
                         FP32 arithmetic, as the reference's single-precision
                         build (its *_f API) computes them; points, origin
                         and width must then be FP32 values */
  int near_fp32;      /* FP64 solvers, 1: the near field (P2P) in the FP32
                         form's kernel (FP32 pair terms from FP64 positions,
                         one FP64 add per run of 8 terms), the expansions and
                         the L2P in FP64 */
  int sparse;         /* 1: sparse level storage: a level's coefficient arrays
                         hold only the groups of eight sibling boxes whose
                         parent holds sources or targets (implies skip_empty;
                         not with managed; arrays sized after the targets are
                         set, with one host wait).  The M2L runs the tile
                         kernel (equal orders in [2, 60] per level); the
                         Hessian, target bases, coefficient pointers and
                         adopted arrays need dense storage, and
                         wbfmm_b200_get_coefficients returns the dense
                         Layout L arrays (zeros outside the stored groups).
                         Not for served requests. */
} wbfmm_b200_config_t;

typedef struct wbfmm_b200_solver wbfmm_b200_solver_t;

/* library */
const char *wbfmm_b200_last_error(void);
int wbfmm_b200_device_count(void);

/* solver lifetime */
int wbfmm_b200_solver_create(wbfmm_b200_solver_t **s,
                             const wbfmm_b200_config_t *cfg, void *stream);
int wbfmm_b200_solver_destroy(wbfmm_b200_solver_t *s);
/* bytes of device memory the solver would hold for n sources and m targets
   (dense level storage; an upper bound for sparse storage) */
int64_t wbfmm_b200_footprint(const wbfmm_b200_config_t *cfg, int64_t nsrc,
                             int64_t ntgt);

/* Sources: xs[i*xstr + 0..2]; normals (may be NULL) likewise.  Pointers are
   host memory unless on_device != 0.  Builds the tree: Morton keys, stable
   sort, per-level box ranges. */
int wbfmm_b200_set_sources(wbfmm_b200_solver_t *s, int nsrc, const double *xs,
                           int xstr, const double *normals, int nstr,
                           int on_device);
/* Strengths: Laplace q[i*qstr], Helmholtz (q[i*qstr], q[i*qstr+1]);
   dipole strengths likewise (need normals).  Either may be NULL. */
int wbfmm_b200_set_strengths(wbfmm_b200_solver_t *s, const double *q,
                             int qstr, const double *dipoles, int dstr,
                             int on_device);
/* Targets: xt[i*tstr + 0..2] (closed cube).  Passing the array (same
   pointer, stride and count) given to the last wbfmm_b200_set_sources makes
   the sources the targets: their ordering is reused, so the array must not
   have changed in between. */
int wbfmm_b200_set_targets(wbfmm_b200_solver_t *s, int ntgt,
                           const double *xt, int tstr, int on_device);

/* stages */
int wbfmm_b200_build_operators(wbfmm_b200_solver_t *s);
int wbfmm_b200_leaf_expansions(wbfmm_b200_solver_t *s);
int wbfmm_b200_upward_pass(wbfmm_b200_solver_t *s, int level);
int wbfmm_b200_downward_pass(wbfmm_b200_solver_t *s, int level);
/* the two halves of a downward-pass level: M2L into level `level`, and L2L
   from `level` into `level+1` (level < depth) */
int wbfmm_b200_m2l(wbfmm_b200_solver_t *s, int level);
int wbfmm_b200_l2l(wbfmm_b200_solver_t *s, int level);
int wbfmm_b200_evaluate(wbfmm_b200_solver_t *s);
/* all stages after set_sources/set_strengths/set_targets */
int wbfmm_b200_run(wbfmm_b200_solver_t *s);
/* the same stages queued on the solver's stream, returning at once;
   wbfmm_b200_wait blocks until they are done (stage times, deferred checks) */
int wbfmm_b200_run_async(wbfmm_b200_solver_t *s);
int wbfmm_b200_wait(wbfmm_b200_solver_t *s);
/* Repeated solves on an unchanged tree (new strengths each time, as in an
   iterative solver): queue the passes (P2M to evaluation) as one CUDA graph
   launch.  The first call after the sources, targets, configuration,
   operators or options changed runs them as wbfmm_b200_run_async does and
   captures them; later calls launch the captured graph.  Returns at once;
   wbfmm_b200_wait blocks. */
int wbfmm_b200_run_graph(wbfmm_b200_solver_t *s);
/* on = 1: set_sources / set_targets queue their checks that the points lie
   inside the cube instead of waiting for them, and WBFMM_B200_E_DOMAIN is
   returned by the next wbfmm_b200_run / wbfmm_b200_wait; a solve that
   fails the check leaves its fields undefined.  Default 0. */
int wbfmm_b200_set_deferred_checks(wbfmm_b200_solver_t *s, int on);

/* Laplace curl of a vector potential (the reference's WBFMM_FIELD_CURL for
   three source components, src/local-laplace.c:632-750,
   src/direct-laplace.c:87-130): curl[3 j + i] = sum over sources of
   (grad 1/(4 pi r) x q)_i at target j, q = (q3[s qstr], q3[s qstr + 1],
   q3[s qstr + 2]).  The solver must be Laplace with the gradient field and
   have its sources and targets set; it runs the three components' solves on
   its tree (the strengths it holds afterwards are the z components).
   Blocks until the curl is written. */
int wbfmm_b200_laplace_curl(wbfmm_b200_solver_t *s, const double *q3, int qstr,
                            double *curl, int on_device);

/* Precomputed target bases (the reference's target-list strategy,
   src/targets.c:168-603, potential only): for the solver's current sources
   and targets, the basis of each target's leaf regular expansion and the
   near-field weights of the sources of its 27 neighbour boxes, stored on the
   device until the sources or targets change.  wbfmm_b200_evaluate_bases
   then writes the potential at the targets (read with
   wbfmm_b200_get_field) from the leaf regular expansions of the last
   downward pass and, with neighbours != 0, the current strengths: a product
   with stored bases and weights instead of the L2P and P2P's special
   functions, for repeated solves at fixed targets. */
int wbfmm_b200_target_bases(wbfmm_b200_solver_t *s);
int wbfmm_b200_evaluate_bases(wbfmm_b200_solver_t *s, int neighbours);

/* Second derivatives of the Laplace potential at the solver's targets,
   after a run (or the downward passes): hess[9 j + 3 a + b] = d_a d_b phi
   at target j (original order), from the leaf regular expansions (the
   coefficients of d/dx, d/dy, d/dz of each leaf expansion, evaluated with
   the gradient L2P) and, with neighbours != 0, the monopoles of the 27
   neighbour boxes (dipole sources: WBFMM_B200_E_ARG).  The second
   derivatives behind the reference's curl gradient
   (src/local-laplace.c:752-1010, :147-197).  Blocks until written. */
int wbfmm_b200_laplace_hessian(wbfmm_b200_solver_t *s, double *hess,
                               int neighbours, int on_device);

/* The curl of a vector potential and its gradient (the reference's
   WBFMM_FIELD_CURL | WBFMM_FIELD_GRADIENT for three source components,
   src/local-laplace.c:1229-1291): out[12 j + i] = curl_i, then
   out[12 j + 3 + 3 a + i] = d_a curl_i at target j; q3 as for
   wbfmm_b200_laplace_curl.  Blocks until written. */
int wbfmm_b200_laplace_curl_gradient(wbfmm_b200_solver_t *s, const double *q3,
                                     int qstr, double *out, int on_device);

/* Self-test of the FP32 near-field sine and cosine: the largest absolute
   error of the engine's own routine (err2[0]) and of CUDA's sincosf
   (err2[1]) against FP64 sin/cos at the FP32 arguments i * xmax / n,
   i = 0..n. */
int wbfmm_b200_selftest_sincos(double xmax, int n, double *err2);
int wbfmm_b200_synchronize(wbfmm_b200_solver_t *s);

/* Measured FP32 FMA throughput of the current GPU (TFLOP/s, 2 flops per
   FMA; best of three timed launches of a register-only FMA kernel over
   every SM): the peak that the roofline fractions of the engine's SIMT
   kernels are quoted against.  Allocates and synchronises. */
int wbfmm_b200_fp32_fma_peak(double *tflops);

/* Results in ORIGINAL target order.  pot: Laplace [n], Helmholtz [2n];
   grad: Laplace [3n], Helmholtz [6n] (d/dx re, im, d/dy re, im, d/dz re,
   im).  Host pointers unless on_device. */
int wbfmm_b200_get_field(wbfmm_b200_solver_t *s, double *pot, double *grad,
                         int on_device);

/* tree and coefficient inspection (host copies) */
int wbfmm_b200_get_tree(wbfmm_b200_solver_t *s, uint32_t *ip,
                        uint32_t *box_i, uint32_t *box_n, int level);
/* level coefficient arrays in Layout L as FP64 (FP32 forms are widened):
   Helmholtz 2*8^l*(p+1)^2 doubles, Laplace 8^l*(p+1)^2 */
int wbfmm_b200_get_coefficients(wbfmm_b200_solver_t *s, int level,
                                double *mps, double *mpr);
/* device pointers of the level arrays (precision of the solver) */
int wbfmm_b200_coefficient_pointers(wbfmm_b200_solver_t *s, int level,
                                    void **mps, void **mpr);
/* Storage of the coefficient arrays: for level in [1, depth], the groups of
   eight boxes stored (dense: 8^(level-1); sparse: those whose parent holds
   sources or targets) and the device bytes of the level's two arrays;
   level 0 gives the totals over every level.  Replaces reading the
   reference's per-level allocation (src/boxes.c:518-583), which is always
   dense. */
int wbfmm_b200_coefficient_storage(wbfmm_b200_solver_t *s, int level,
                                   int64_t *groups, int64_t *bytes);
/* per-stage device times of the last run (ms): tree, operators, P2M,
   upward, downward, evaluation */
int wbfmm_b200_stage_times(wbfmm_b200_solver_t *s, double *ms6);
/* number of kernels the solver launched since creation */
int64_t wbfmm_b200_kernel_launches(wbfmm_b200_solver_t *s);

/* Drop cached operator tables so the next stage regenerates them (tables
   otherwise persist for the solver's lifetime, keyed by its config). */
int wbfmm_b200_invalidate_operators(wbfmm_b200_solver_t *s);

/* Fields wbfmm_b200_evaluate computes (subset of the config's field) and
   whether it adds the near field of the 27 neighbour boxes (the reference's
   eval_neighbours, src/local.c:264-310). */
int wbfmm_b200_set_evaluation(wbfmm_b200_solver_t *s, int field,
                              int neighbours);

/* 1: wbfmm_b200_leaf_expansions adds to the existing leaf coefficients (the
   reference's zero_expansions = FALSE); 0 (default): overwrites them. */
int wbfmm_b200_set_p2m_accumulate(wbfmm_b200_solver_t *s, int on);

/* Use caller-supplied coefficient arrays for a level (Layout L, the
   solver's precision, device-accessible, e.g. from wbfmm_b200_managed_alloc)
   instead of allocating them; call before wbfmm_b200_set_sources. */
int wbfmm_b200_adopt_coefficients(wbfmm_b200_solver_t *s, int level,
                                  void *mps, void *mpr);
/* zeroed CUDA managed memory (host- and device-accessible) */
void *wbfmm_b200_managed_alloc(size_t bytes);
void wbfmm_b200_managed_free(void *p);

/* Tree structure only: the stable Morton permutation ip[n] (t->ip) and the
   box {i, n} arrays of levels 0..depth concatenated (sum 8^l entries each),
   exactly as wbfmm_tree_add_points followed by `depth` calls of
   wbfmm_tree_refine leave them (src/boxes.c:118-277).  Host buffers;
   pts[i*pstr + 0..2]. */
int wbfmm_b200_tree_structure(int n, const double *pts, int pstr,
                              const double *x0, double D, int depth,
                              uint32_t *ip, uint32_t *box_i, uint32_t *box_n);
/* The same for FP32 points (pts[i*pstr + 0..2], stride in floats), with the
   keys computed as the reference's single-precision build computes them
   (wbfmm_tree_add_points_f / wbfmm_tree_refine_f). */
int wbfmm_b200_tree_structure_f(int n, const float *pts, int pstr,
                                const float *x0, float D, int depth,
                                uint32_t *ip, uint32_t *box_i, uint32_t *box_n);

/* M2L kernel selection (all need equal singular and regular orders, else
   the warp kernel runs): 1 (default) = automatic: lane-per-pair kernel up to
   order 7 (Helmholtz) / 10 (Laplace FP32) / 9 (Laplace FP64), offset-major
   target tiles above, while their shared memory suffices;
   2 = lane-per-pair wherever instantiated
   (Helmholtz <= 8, Laplace <= 16); 3 = target tiles wherever they fit;
   0 = always the warp-per-target kernel; 4 = Laplace FP32 on the tensor
   cores (dense per-shift operators, tcgen05 kind::tf32 with 3xTF32
   splitting, FP32 accumulation in tensor memory) for equal orders with
   (p+1)^2 <= 256, the automatic choice elsewhere. */
int wbfmm_b200_set_m2l_kernel(wbfmm_b200_solver_t *s, int mode);

/* FP64 direct sum with self-exclusion (r <= 1e-6) and compensated
   accumulation: the GPU counterpart of wbfmm_total_field[_grad]
   (src/direct.c:35-294) and wbfmm_laplace_field[_grad]
   (src/direct-laplace.c:200-336).  xs[3ns], xt[3nt]; q / dipoles as in
   wbfmm_b200_set_strengths with unit stride; pot/grad may be NULL. */
int wbfmm_b200_direct(int problem, double k, int ns, const double *xs,
                      const double *q, const double *normals,
                      const double *dipoles, int nt, const double *xt,
                      double *pot, double *grad, int on_device);

/* Accuracy of a field against a reference, reduced on the GPU in FP64 with
   a fixed order: out4 = {||f - ref||_2, ||ref||_2, max |f - ref|,
   max |ref|} over n values (host or device arrays). */
int wbfmm_b200_error_norms(int64_t n, const double *f, const double *ref,
                           int on_device, double *out4);

/* Largest point count wbfmm_b200_morton_sort_noalloc accepts. */
#define WBFMM_B200_NOALLOC_MAX_POINTS (1 << 20)

/* Morton keys and the stable Morton permutation of device-resident points
   (the ordering wbfmm_b200_set_sources computes for the tree), with no
   device allocation.  This entry point has no counterpart in the reference.
   It is for callers that cannot allocate device memory where they need the
   sort: serving loops that must not take cudaMalloc's device-wide
   synchronisation, and processes whose device memory belongs to another
   allocator.  They pass their own buffers: pts[i*pstr + 0..2] (device),
   keys[n] and ip[n] (device, outputs: sorted keys and the permutation); x0
   (3 doubles) is host memory.  The sort's scratch is a fixed array of about
   12.6 MB in device memory that every GPU which loads the library holds
   until the process exits, so n may not exceed
   WBFMM_B200_NOALLOC_MAX_POINTS (larger n returns WBFMM_B200_E_ARG).  The
   first call on a device looks up that array's device address (make it
   before any stream capture); the address is kept for the process, so the
   device must not be reset while the library is in use.  All calls on a
   device share the array: calls that overlap on the GPU race with each
   other.  The call returns after its work on `stream` has finished (it
   reads back a domain-check flag; points not strictly inside the cube
   return WBFMM_B200_E_DOMAIN). */
int wbfmm_b200_morton_sort_noalloc(int n, const double *pts, int pstr,
                                   const double *x0, double D, uint64_t *keys,
                                   uint32_t *ip, void *stream);

/* One call: create, build, run, copy out, destroy.  Host buffers. */
int wbfmm_b200_solve(const wbfmm_b200_config_t *cfg, int nsrc,
                     const double *xs, const double *q, const double *normals,
                     const double *dipoles, int ntgt, const double *xt,
                     double *pot, double *grad);

/* 1 when the FP32 form keeps this configuration's tables and expansions
   inside the FP32 range (Helmholtz (S|R) coefficients at the nearest list-4
   distance and leaf Bessel terms within 1e+-36; Laplace order <= 16 with
   (2w)^-(p+1) and (0.87w)^p within 1e+-30 at every level of box width w,
   for strengths of order one); 0 when the solve needs the FP64 form. */
int wbfmm_b200_fp32_range_ok(const wbfmm_b200_config_t *cfg);

/* ------------------------------------------------------------------------
   Served form (no reference counterpart): continuous batching of
   independent solves on one GPU.  `nslots` solves run at once, each on its
   own stream, admitted first come first served (or largest first,
   wbfmm_b200_server_set_order) while the summed
   wbfmm_b200_footprint of the solves in flight stays within `hbm_budget`
   bytes less the slots' allowance for keeping work buffers between solves
   (per slot hbm_budget / (4 nslots), at most 4 GB; a slot whose buffers
   grow past it releases them).  The order-only operator tables (rotations,
   shift phases, Laplace coaxial tables) are shared across solves; Helmholtz
   coaxial tables (which depend on k) are built per solve.  Inputs and outputs are host
   arrays (or device arrays, with on_device) that the caller keeps alive
   until the request completes; fields come back in FP64 in the layouts of
   wbfmm_b200_get_field.  All calls are thread-safe.
   ------------------------------------------------------------------------ */
typedef struct wbfmm_b200_server wbfmm_b200_server_t;

typedef struct {
  wbfmm_b200_config_t cfg;  /* problem, tree, orders, k, precision, field */
  int nsrc;
  const double *xs;         /* [3 nsrc] */
  const double *q;          /* [w nsrc] or NULL (w = 2 Helmholtz, 1 Laplace) */
  const double *normals;    /* [3 nsrc] or NULL */
  const double *dipoles;    /* [w nsrc] or NULL */
  int ntgt;
  const double *xt;         /* [3 ntgt]; may be xs (targets = sources) */
  double *pot;              /* [w ntgt] or NULL */
  double *grad;             /* [3 w ntgt] or NULL */
  double arrival;           /* server-clock seconds before which the request
                               is not started (0: on submission) */
  int on_device;            /* 1: xs, q, normals, dipoles, xt, pot and grad
                               are device pointers (no host staging; the
                               fields are written there in place) */
} wbfmm_b200_request_t;

int wbfmm_b200_server_create(wbfmm_b200_server_t **srv, int nslots,
                             int64_t hbm_budget);
/* waits for every request, then releases the server */
int wbfmm_b200_server_destroy(wbfmm_b200_server_t *srv);
/* seconds since the server was created (the clock of `arrival`) */
double wbfmm_b200_server_clock(wbfmm_b200_server_t *srv);
/* queue a request; WBFMM_B200_E_ADMISSION when its footprint alone exceeds
   the budget */
int wbfmm_b200_server_submit(wbfmm_b200_server_t *srv,
                             const wbfmm_b200_request_t *req, int64_t *ticket);
/* Order in which free slots take the requests that have arrived: 0 (the
   default) first come first served; 1 the largest device-memory footprint
   first (for batches submitted together: the big solves start first and the
   small ones fill the end, which shortens the batch's span). */
int wbfmm_b200_server_set_order(wbfmm_b200_server_t *srv, int largest_first);
/* 1 when the request has completed, 0 when not yet */
int wbfmm_b200_server_poll(wbfmm_b200_server_t *srv, int64_t ticket);
/* blocks until the request has completed; returns its status */
int wbfmm_b200_server_wait(wbfmm_b200_server_t *srv, int64_t ticket);
/* server-clock times of a completed request: arrival, start (taken by a
   slot), queued (all its device work and copies issued on the slot's
   stream) and completion (fields in the caller's arrays) */
int wbfmm_b200_server_times(wbfmm_b200_server_t *srv, int64_t ticket,
                            double *t4);
/* drops a completed request's record */
int wbfmm_b200_server_forget(wbfmm_b200_server_t *srv, int64_t ticket);
/* blocks until the queue is empty and no solve is running */
int wbfmm_b200_server_drain(wbfmm_b200_server_t *srv);
/* completed requests, peak bytes in flight, peak solves in flight, lookups
   of the shared order-only tables served by an existing set and building a
   new one, the sets' device bytes, kernels launched by completed solves */
int wbfmm_b200_server_stats(wbfmm_b200_server_t *srv, int64_t *out7);

#ifdef __cplusplus
}
#endif

#endif /* WBFMM_B200_H */
