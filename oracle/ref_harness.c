/*
 * Harness around the UNMODIFIED wbfmm reference sources (built from
 * the reference's src/ directory by oracle/build_oracle.py into
 * oracle/_ref/libwbfmm_ref.so).  It replays the reference drivers' call
 * sequence on in-memory inputs, with no text I/O:
 *
 *   Helmholtz: tools/wbfmm-tree-calc.c.in:270-414
 *   Laplace:   tools/wbfmm-laplace-tree-calc.c.in:336-460
 *
 * and returns the field, the gradient (a second evaluation call, since the
 * reference computes one field type per call: src/local.c:264-310,
 * src/local-laplace.c:1293-1336), the tree (t->ip and per-level box i/n) and
 * the per-level coefficient arrays in the reference's own layout.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker and the timed CPU baseline.
 * The wbfmm_b200 product never links or calls it.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <glib.h>
#include <wbfmm.h>

static double now_s(void)
{
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

/* number of coefficients (doubles) of one level's coefficient array */
static size_t level_coeff_doubles(int problem, int l, int order)
{
  size_t nb = (size_t)1 << (3 * l);
  size_t nc = (size_t)(order + 1) * (order + 1);
  return nb * nc * (problem == WBFMM_PROBLEM_HELMHOLTZ ? 2 : 1);
}

/*
 * Run one FMM solve through the reference API.
 *
 * problem: 1 Laplace, 2 Helmholtz; nq = 1.
 * xs[3*nsrc]; q: Laplace real[nsrc], Helmholtz complex[2*nsrc] (may be
 * NULL when dipoles are given); normals[3*nsrc] and dipoles (same layout as
 * q) may be NULL.
 * order_s/order_r: per-level orders, index 0..depth (entries 1..depth used).
 * pot_out: Laplace [ntgt], Helmholtz [2*ntgt]; grad_out: Laplace [3*ntgt],
 * Helmholtz [6*ntgt]; either may be NULL to skip that evaluation.
 * ip_out[nsrc], boxes_out[2*sum_l 8^l] ({i,n} per box, levels 0..depth),
 * mps_out / mpr_out (levels 1..depth concatenated, reference layout) may be
 * NULL.
 * times_out[6]: tree, operators, P2M, upward, downward, evaluation (s).
 */
int ref_fmm_run(int problem, int depth, const int *order_s,
                const int *order_r, double k, int bw, int nthreads,
                const double *x0, double D, int nsrc, const double *xs,
                const double *q, const double *normals,
                const double *dipoles, int ntgt, const double *xt,
                double *pot_out, double *grad_out, unsigned *ip_out,
                unsigned *boxes_out, double *mps_out, double *mpr_out,
                double *times_out)
{
  wbfmm_tree_t *tree;
  wbfmm_shift_operators_t *shifts;
  double *work, t0, t1;
  int i, level, order_max = 0;
  size_t sizew;
  double xtree[3];
  int nq = 1;

  for (level = 1; level <= depth; level++) {
    if (order_s[level] > order_max) order_max = order_s[level];
    if (order_r[level] > order_max) order_max = order_r[level];
  }
  if (nthreads < 1) nthreads = 1;
  if (nthreads > WBFMM_THREAD_NUMBER_MAX) nthreads = WBFMM_THREAD_NUMBER_MAX;

  sizew = wbfmm_element_number_rotation(2 * order_max);
  if (problem == WBFMM_PROBLEM_HELMHOLTZ) {
    size_t s2 = 64 * nq * wbfmm_coefficient_index_nm(order_max + 1, 0);
    if (s2 > sizew) sizew = s2;
  } else {
    size_t s2 = (size_t)(order_max + 1) * (order_max + 1) * nq * 16;
    if (s2 > sizew) sizew = s2;
  }
  work = g_malloc0((size_t)(nthreads + 1) * sizew * sizeof(double));

  xtree[0] = x0[0]; xtree[1] = x0[1]; xtree[2] = x0[2];

  /* operators (timed separately, as in the drivers) */
  t0 = now_s();
  wbfmm_shift_angle_table_init();
  shifts = wbfmm_shift_operators_new(order_max, bw, work);
  if (problem == WBFMM_PROBLEM_HELMHOLTZ) {
    for (i = 1; i <= depth; i++)
      wbfmm_shift_operators_coaxial_SR_init(shifts, D, i, order_s[i], k, work);
    for (level = 2; level <= depth; level++)
      wbfmm_shift_operators_coaxial_SS_init(shifts, D, level,
                                            order_s[level - 1], k, work);
  } else {
    wbfmm_laplace_coaxial_translate_init(order_max + 2);
  }
  t1 = now_s();
  if (times_out) times_out[1] = t1 - t0;

  /* tree */
  t0 = now_s();
  tree = wbfmm_tree_new(xtree, D, 2 * nsrc);
  wbfmm_tree_source_size(tree) = nq;
  wbfmm_tree_add_points(tree, (gpointer)xs, 3 * sizeof(double),
                        (gpointer)normals, 3 * sizeof(double), nsrc, FALSE);
  for (i = 0; i < depth; i++) wbfmm_tree_refine(tree);
  wbfmm_tree_problem(tree) = problem;
  for (i = 1; i <= depth; i++) {
    if (problem == WBFMM_PROBLEM_HELMHOLTZ)
      wbfmm_tree_coefficient_init(tree, i, order_r[i], order_s[i]);
    else
      wbfmm_tree_laplace_coefficient_init(tree, i, order_r[i], order_s[i]);
  }
  /* the Helmholtz coefficient arrays come from posix_memalign and are not
     zeroed; M2L at level 2 accumulates into them (src/boxes.c:568) */
  for (i = 1; i <= depth; i++) {
    size_t n = level_coeff_doubles(problem, i, order_r[i]);
    memset(tree->mpr[i], 0, n * sizeof(double));
  }
  t1 = now_s();
  if (times_out) times_out[0] = t1 - t0;

  /* P2M */
  t0 = now_s();
  if (problem == WBFMM_PROBLEM_HELMHOLTZ)
    wbfmm_tree_leaf_expansions(tree, k, (double *)q, 2, (double *)dipoles, 2,
                               TRUE, work);
  else
    wbfmm_tree_laplace_leaf_expansions(tree, (double *)q, 1,
                                       (double *)dipoles, 1, TRUE, work);
  t1 = now_s();
  if (times_out) times_out[2] = t1 - t0;

  /* upward pass */
  t0 = now_s();
  for (level = depth; level >= 3; level--) {
    if (problem == WBFMM_PROBLEM_HELMHOLTZ)
      wbfmm_upward_pass(tree, shifts, level, work);
    else
      wbfmm_laplace_upward_pass(tree, shifts, level, work);
  }
  t1 = now_s();
  if (times_out) times_out[3] = t1 - t0;

  /* downward pass */
  t0 = now_s();
  for (level = 2; level <= depth; level++) {
    if (problem == WBFMM_PROBLEM_HELMHOLTZ)
      wbfmm_downward_pass(tree, shifts, level, work, nthreads);
    else
      wbfmm_laplace_downward_pass(tree, shifts, level, work, nthreads);
  }
  t1 = now_s();
  if (times_out) times_out[4] = t1 - t0;

  /* evaluation: one call per field type per target */
  t0 = now_s();
  if (problem == WBFMM_PROBLEM_HELMHOLTZ) {
    if (pot_out) {
      memset(pot_out, 0, 2 * (size_t)ntgt * sizeof(double));
      for (i = 0; i < ntgt; i++) {
        guint64 b = wbfmm_point_box(tree, depth, (double *)&xt[3 * i]);
        wbfmm_tree_box_local_field(tree, depth, b, k, (double *)&xt[3 * i],
                                   &pot_out[2 * i], 2, (double *)q, 2,
                                   (double *)dipoles, 2, TRUE,
                                   WBFMM_FIELD_POTENTIAL, work);
      }
    }
    if (grad_out) {
      memset(grad_out, 0, 6 * (size_t)ntgt * sizeof(double));
      for (i = 0; i < ntgt; i++) {
        guint64 b = wbfmm_point_box(tree, depth, (double *)&xt[3 * i]);
        wbfmm_tree_box_local_field(tree, depth, b, k, (double *)&xt[3 * i],
                                   &grad_out[6 * i], 6, (double *)q, 2,
                                   (double *)dipoles, 2, TRUE,
                                   WBFMM_FIELD_GRADIENT, work);
      }
    }
  } else {
    if (pot_out) {
      memset(pot_out, 0, (size_t)ntgt * sizeof(double));
      for (i = 0; i < ntgt; i++) {
        guint64 b = wbfmm_point_box(tree, depth, (double *)&xt[3 * i]);
        wbfmm_laplace_box_field(tree, depth, b, (double *)q, 1,
                                (double *)dipoles, 1, WBFMM_FIELD_POTENTIAL,
                                TRUE, (double *)&xt[3 * i], &pot_out[i], 1,
                                work);
      }
    }
    if (grad_out) {
      memset(grad_out, 0, 3 * (size_t)ntgt * sizeof(double));
      for (i = 0; i < ntgt; i++) {
        guint64 b = wbfmm_point_box(tree, depth, (double *)&xt[3 * i]);
        wbfmm_laplace_box_field(tree, depth, b, (double *)q, 1,
                                (double *)dipoles, 1, WBFMM_FIELD_GRADIENT,
                                TRUE, (double *)&xt[3 * i], &grad_out[3 * i],
                                1, work);
      }
    }
  }
  t1 = now_s();
  if (times_out) times_out[5] = t1 - t0;

  if (ip_out) memcpy(ip_out, tree->ip, (size_t)nsrc * sizeof(unsigned));
  if (boxes_out) {
    size_t off = 0;
    for (level = 0; level <= depth; level++) {
      size_t nb = (size_t)1 << (3 * level), b;
      for (b = 0; b < nb; b++) {
        boxes_out[2 * (off + b) + 0] = tree->boxes[level][b].i;
        boxes_out[2 * (off + b) + 1] = tree->boxes[level][b].n;
      }
      off += nb;
    }
  }
  if (mps_out || mpr_out) {
    size_t offs = 0, offr = 0;
    for (level = 1; level <= depth; level++) {
      size_t ns = level_coeff_doubles(problem, level, order_s[level]);
      size_t nr = level_coeff_doubles(problem, level, order_r[level]);
      if (mps_out) memcpy(&mps_out[offs], tree->mps[level], ns * sizeof(double));
      if (mpr_out) memcpy(&mpr_out[offr], tree->mpr[level], nr * sizeof(double));
      offs += ns; offr += nr;
    }
  }

  /* the reference has no free functions for trees or operators
     (objects leak by design); release what this harness can reach */
  for (level = 1; level <= depth; level++) {
    free(tree->mps[level]);
    free(tree->mpr[level]);
  }
  for (level = 0; level <= depth; level++) free(tree->boxes[level]);
  free(tree->ip);
  free(tree);
  free(work);
  return 0;
}

/* list-4 interaction list of box idx at level (src/indexing.c:330-377),
   unsorted: list[2*j] = box, list[2*j+1] = shift index; returns count */
int ref_interaction_list_4(unsigned level, unsigned long long idx,
                           unsigned long long *list)
{
  extern gint wbfmm_box_interaction_list_4(guint level, guint64 idx,
                                           guint64 *list, gboolean sort);
  return wbfmm_box_interaction_list_4(level, idx, (guint64 *)list, FALSE);
}

/* 27-neighbour list (src/indexing.c:250-286) */
int ref_box_neighbours(unsigned level, unsigned long long idx,
                       unsigned long long *nb)
{
  extern gint wbfmm_box_neighbours(guint level, guint64 idx,
                                   guint64 *neighbours);
  return wbfmm_box_neighbours(level, idx, (guint64 *)nb);
}

/* Morton key of a point (src/boxes.c:324-339) and target box
   (src/boxes.c:585-634) */
unsigned long long ref_point_index_3d(const double *x, const double *c,
                                      double D)
{
  return wbfmm_point_index_3d((double *)x, (double *)c, D);
}

unsigned long long ref_point_box(const double *x0, double D, unsigned level,
                                 const double *x)
{
  wbfmm_tree_t t;
  memset(&t, 0, sizeof(t));
  memcpy(t.x, x0, 3 * sizeof(double));
  t.D = D;
  t.size = sizeof(double);
  return wbfmm_point_box(&t, level, (double *)x);
}

/* rotation coefficients H (src/rotations.c:131-207), nerot doubles */
int ref_rotation_H(int N, double th, double *H)
{
  double *work = g_malloc0(wbfmm_element_number_rotation(2 * N + 2) *
                           2 * sizeof(double) + 4096);
  wbfmm_coefficients_H_rotation(H, N, th, work);
  free(work);
  return 0;
}

/* coaxial (S|R) coefficients (src/translations.c:340-409), complex */
int ref_coaxial_SR(int L, double kr, double *cfft)
{
  double *work = g_malloc0(2 * wbfmm_element_number_coaxial(2 * L + 2) *
                           sizeof(double) + 4096);
  wbfmm_coefficients_SR_coaxial(cfft, L, kr, work);
  free(work);
  return 0;
}

/* coaxial (R|R) coefficients (src/translations.c:272-338), real */
int ref_coaxial_RR(int L, double kr, double *cfft)
{
  double *work = g_malloc0(wbfmm_element_number_coaxial(2 * L + 2) *
                           sizeof(double) + 4096);
  wbfmm_coefficients_RR_coaxial(cfft, L, kr, work);
  free(work);
  return 0;
}

/* FP64 direct sums through the reference's own direct.c / direct-laplace.c
   (no self-exclusion: callers pass targets distinct from sources) */
int ref_direct_helmholtz(double k, int nsrc, const double *xs,
                         const double *q, const double *normals,
                         const double *dipoles, int ntgt, const double *xt,
                         int grad, double *f)
{
  int i;
  for (i = 0; i < ntgt; i++) {
    if (grad)
      wbfmm_total_field_grad(k, (double *)xs, 3, (double *)q, 2,
                             (double *)normals, 3, (double *)dipoles, 2, 1,
                             nsrc, (double *)&xt[3 * i], &f[6 * i], 6);
    else
      wbfmm_total_field(k, (double *)xs, 3, (double *)q, 2,
                        (double *)normals, 3, (double *)dipoles, 2, 1, nsrc,
                        (double *)&xt[3 * i], &f[2 * i], 2);
  }
  return 0;
}

int ref_direct_laplace(int nsrc, const double *xs, const double *q,
                       const double *normals, const double *dipoles,
                       int ntgt, const double *xt, int grad, double *f)
{
  int i;
  for (i = 0; i < ntgt; i++) {
    if (grad)
      wbfmm_laplace_field_grad((double *)xs, 3, (double *)q, 1, 1,
                               (double *)normals, 3, (double *)dipoles, 1,
                               nsrc, (double *)&xt[3 * i], &f[3 * i], 3);
    else
      wbfmm_laplace_field((double *)xs, 3, (double *)q, 1, 1,
                          (double *)normals, 3, (double *)dipoles, 1, nsrc,
                          (double *)&xt[3 * i], &f[i], 1);
  }
  return 0;
}
