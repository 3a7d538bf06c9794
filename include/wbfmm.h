/*
 * Drop-in replacement for the wbfmm C API (mjcarley/wbfmm, src/wbfmm.h),
 * backed by the B200 engine (include/wbfmm_b200.h).
 *
 * Type layouts, enumerations, macros and the signatures of the functions
 * below are those of the reference header so that existing callers compile
 * and link unchanged (double-precision API).  Differences in behaviour are
 * stated beside each function; the per-function reference lines are in
 * wbfmm_b200/csrc/wbfmm_api.c.
 *
 * As with the reference, callers include <glib.h> first; without GLib the
 * GLib scalar types are defined here.
 */
#ifndef WBFMM_H_INCLUDED
#define WBFMM_H_INCLUDED

#include <stdint.h>
#include <stdio.h>
#include <stddef.h>

#if !defined(__G_LIB_H__) && !defined(WBFMM_ORACLE_GLIB_SHIM_H)
typedef int gint;
typedef unsigned int guint;
typedef int gboolean;
typedef double gdouble;
typedef float gfloat;
typedef char gchar;
typedef size_t gsize;
typedef void *gpointer;
typedef const void *gconstpointer;
typedef uint32_t guint32;
typedef uint64_t guint64;
#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define WBFMM_INDEX_SCALE (1LU << 63)
#define WBFMM_INDEX_SHIFT (1U << 20)
#define WBFMM_LOCAL_CUTOFF_RADIUS 1e-6
#ifndef WBFMM_THREAD_NUMBER_MAX
#define WBFMM_THREAD_NUMBER_MAX 16
#endif

typedef struct {
  gboolean avx, avx2, fma, openmp;
  char *switches;
  gsize real_size;
} wbfmm_library_config_t;

typedef struct {
  guint32 i, n;         /* first point (sorted order) and point count */
  gpointer mps, mpr;    /* singular / regular coefficients, Layout L */
} wbfmm_box_t;

#define WBFMM_TREE_MAX_DEPTH 16

typedef enum {
  WBFMM_PROBLEM_LAPLACE = 1,
  WBFMM_PROBLEM_HELMHOLTZ = 2
} wbfmm_problem_t;

typedef enum {
  WBFMM_FIELD_POTENTIAL = 1 << 0,
  WBFMM_FIELD_GRADIENT = 1 << 1,
  WBFMM_FIELD_CURL = 1 << 2,
  WBFMM_FIELD_CURL_GRADIENT = 1 << 3
} wbfmm_field_t;

typedef struct {
  wbfmm_problem_t problem;
  wbfmm_box_t *boxes[WBFMM_TREE_MAX_DEPTH + 1];
  gboolean sorted;
  guint maxpoints, npoints, *ip, nq, depth,
      order_s[WBFMM_TREE_MAX_DEPTH + 1], order_r[WBFMM_TREE_MAX_DEPTH + 1];
  char x[24], *normals, *points;
  gpointer mps[WBFMM_TREE_MAX_DEPTH + 1], mpr[WBFMM_TREE_MAX_DEPTH + 1];
  gsize size, nstr, pstr;
  gdouble D;
} wbfmm_tree_t;

typedef enum {
  WBFMM_SOURCE_MONOPOLE = 1 << 0,
  WBFMM_SOURCE_DIPOLE = 1 << 1
} wbfmm_source_t;

typedef struct {
  wbfmm_tree_t *t;
  guint field, source, maxpoints, npoints, *ip, nc;
  guint32 *boxes;
  char *points;
  gsize size, pstr;
  gint *ibox, *isrc, *ics;
  gpointer cfft, csrc;
  gboolean complex;
} wbfmm_target_list_t;

#define wbfmm_target_list_field(_l) ((_l)->field)
#define wbfmm_target_point_box(_l, _i) ((_l)->boxes[(_i)])

typedef struct {
  gsize size;
  guint Lmax, nlevels, L[WBFMM_TREE_MAX_DEPTH + 1], nerot;
  gpointer SR[WBFMM_TREE_MAX_DEPTH + 1], SS[WBFMM_TREE_MAX_DEPTH + 1], rotations;
  gboolean bw;
} wbfmm_shift_operators_t;

#define wbfmm_tree_point_number(_t) ((_t)->npoints)
#define wbfmm_tree_point_number_max(_t) ((_t)->maxpoints)
#define wbfmm_tree_depth(_t) ((_t)->depth)
#define wbfmm_tree_boxes_level(_t, _l) ((_t)->boxes[(_l)])
#define wbfmm_tree_width(_t) ((_t)->D)
#define wbfmm_tree_origin(_t) ((gpointer)(&((_t)->x[0])))
#define wbfmm_tree_problem(_t) ((_t)->problem)
#define wbfmm_tree_source_size(_t) ((_t)->nq)

#define wbfmm_target_list_tree(_t) ((_t)->t)
#define wbfmm_target_list_point_number(_t) ((_t)->npoints)
#define wbfmm_target_list_point_number_max(_t) ((_t)->maxpoints)

#define wbfmm_element_number_coaxial(_N) \
  (((_N) + 1) * ((_N) + 2) * ((_N) + 3) / 6 + ((_N) + 1) * ((_N) + 2) / 2 + (_N) + 1)
#define wbfmm_element_number_rotation(_N)                            \
  ((((_N) + 1) * (4 * (_N) + 3) * ((_N) + 2) / 6 +                   \
    (((_N) + 1) + ((_N) + 1)) * (((_N) + 1) + 1) + (_N)))
#define wbfmm_T_rotation_matrix_size(_n) (((_n) + 1) * (2 * (_n) + 1) * (2 * (_n) + 3) / 3)

#define wbfmm_box_index_parent(_i) ((_i) / 8)
#define wbfmm_box_index_first_child(_i) ((_i) * 8)

#define wbfmm_coefficient_index_nm(_n, _m) ((_n) * ((_n) + 1) + (_m))
#define wbfmm_coefficient_number(_n) \
  wbfmm_coefficient_index_nm(((_n) + 1), (-((_n) + 1)))
#define wbfmm_conjugate_index_nm(_n, _m) (((_n) * ((_n) + 1) / 2) + (_m))

/* ------------------------------------------------ trees and indexing */
wbfmm_tree_t *wbfmm_tree_new(gdouble *x, gdouble D, guint maxpoints);
gint wbfmm_tree_add_points(wbfmm_tree_t *t, gpointer pts, gsize pstr,
                           gpointer normals, gsize nstr, guint npts,
                           gboolean sorted);
gint wbfmm_tree_sort_points(wbfmm_tree_t *t, gpointer pts, gsize psize,
                            guint npts);
gint wbfmm_tree_refine(wbfmm_tree_t *t);
gint wbfmm_tree_add_level(wbfmm_tree_t *tree);
gint wbfmm_tree_coefficient_init(wbfmm_tree_t *t, guint l, guint nr, guint ns);
gint wbfmm_tree_laplace_coefficient_init(wbfmm_tree_t *t, guint l, guint nr,
                                         guint ns);
gint wbfmm_tree_coefficient_clear(wbfmm_tree_t *t, guint l);
gint wbfmm_tree_coefficients_zero(wbfmm_tree_t *t, guint level);
guint64 wbfmm_point_box(wbfmm_tree_t *t, guint level, gdouble *x);
guint64 wbfmm_point_index_3d(gdouble *x, gdouble *c, gdouble D);
/* the tree's points in tree order, "i ip[i] x y z" per line (q, stride
   unused, as in the reference) */
gint wbfmm_tree_write_sources(wbfmm_tree_t *t,
                              gdouble *q, gint stride,
                              FILE *f);
guint64 wbfmm_point_locate_box(guint64 x, guint level);
gint wbfmm_point_from_index(guint64 i, guint32 *x, guint32 *y, guint32 *z);
guint64 wbfmm_box_index(guint32 i, guint32 j, guint32 k);
gint wbfmm_box_location(guint64 idx, guint32 *i, guint32 *j, guint32 *k);
guint64 wbfmm_box_parent(guint64 idx);
guint64 wbfmm_box_first_child(guint64 idx);
gint wbfmm_box_neighbours(guint level, guint64 idx, guint64 *neighbours);
gint wbfmm_box_interaction_list_4(guint level, guint64 idx, guint64 *list,
                                  gboolean sort);
gint wbfmm_box_interaction_grid_4(guint level, guint64 idx, guint64 list[]);
gint wbfmm_box_location_from_index(guint64 i, guint32 level, gdouble *x0,
                                   gdouble D, gdouble *x, gdouble *wb);
gint wbfmm_tree_box_centre(wbfmm_tree_t *t, guint level, guint64 b,
                           gdouble *xb, gdouble *wb);
gint wbfmm_points_origin_width(gdouble *x, gint str, gint n, gdouble *xmin,
                               gdouble *xmax, gdouble *D,
                               gboolean init_limits);
gint wbfmm_truncation_number(wbfmm_tree_t *t, gdouble k, guint level,
                             gdouble tol);

/* ------------------------------------------------------- operators */
/* Tables are generated on the GPU for each tree (FP64); these calls record
   the requested orders and are otherwise no-ops. */
gint wbfmm_shift_angle_table_init(void);
wbfmm_shift_operators_t *wbfmm_shift_operators_new(guint L, gboolean bw,
                                                   gdouble *work);
gint wbfmm_shift_operators_coaxial_SR_init(wbfmm_shift_operators_t *w,
                                           gdouble D, guint level, guint L,
                                           gdouble k, gdouble *work);
gint wbfmm_shift_operators_coaxial_SS_init(wbfmm_shift_operators_t *w,
                                           gdouble D, guint level, guint L,
                                           gdouble k, gdouble *work);
gint wbfmm_laplace_coaxial_translate_init(gint N);

/* ---------------------------------------------------------- passes */
gint wbfmm_tree_leaf_expansions(wbfmm_tree_t *t, gdouble k, gdouble *src,
                                gint sstr, gdouble *dipoles, gint dstr,
                                gboolean zero_expansions, gdouble *work);
gint wbfmm_tree_laplace_leaf_expansions(wbfmm_tree_t *t, gdouble *src,
                                        gint sstr, gdouble *dipoles,
                                        gint dstr, gboolean zero_expansions,
                                        gdouble *work);
gint wbfmm_upward_pass(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                       guint level, gdouble *work);
gint wbfmm_laplace_upward_pass(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                               guint level, gdouble *work);
gint wbfmm_downward_pass_ref(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                             guint level, gdouble *work, gint nthreads);
gint wbfmm_downward_pass_avx(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                             guint level, gdouble *work, gint nthreads);
gint wbfmm_laplace_downward_pass_ref(wbfmm_tree_t *t,
                                     wbfmm_shift_operators_t *op, guint level,
                                     gdouble *work, gint nthreads);
gint wbfmm_laplace_downward_pass_avx(wbfmm_tree_t *t,
                                     wbfmm_shift_operators_t *op, guint level,
                                     gdouble *work, gint nthreads);

/* ------------------------------------------------------ evaluation */
/* One target per call (slow on any accelerator: use target lists for many
   targets).  level must be the tree depth; b is recomputed from x. */
gint wbfmm_tree_box_local_field(wbfmm_tree_t *t, guint level, guint b,
                                gdouble k, gdouble *x, gdouble *f, gint fstr,
                                gdouble *src, gint sstr, gdouble *d,
                                gint dstr, gboolean eval_neighbours,
                                guint field, gdouble *work);
gint wbfmm_laplace_box_field(wbfmm_tree_t *t, guint level, guint b,
                             gdouble *src, gint sstr, gdouble *d, gint dstr,
                             guint field, gboolean eval_neighbours,
                             gdouble *x, gdouble *f, gint fstr,
                             gdouble *work);

/* target lists: all targets in one GPU evaluation; potential, gradient, and
   (an extension of the reference, whose gradient branches are unfinished)
   potential and gradient together */
wbfmm_target_list_t *wbfmm_target_list_new(wbfmm_tree_t *t, guint npts);
gint wbfmm_target_list_add_points(wbfmm_target_list_t *l, gpointer pts,
                                  gsize pstr, guint npts);
gint wbfmm_target_list_coefficients_init(wbfmm_target_list_t *l, guint field);
gint wbfmm_target_list_local_coefficients(wbfmm_target_list_t *l, gdouble k,
                                          gdouble *work);
gint wbfmm_laplace_target_list_local_coefficients(wbfmm_target_list_t *l,
                                                  guint source, gdouble *work);
gint wbfmm_target_list_local_field(wbfmm_target_list_t *l, gdouble *src,
                                   gint sstr, gdouble *nsrc, gint nstr,
                                   gdouble *f, gint fstr);

/* ---------------------------------------------------- direct sums */
/* FP64 on the GPU; source-target pairs closer than 1e-6 contribute 0 (the
   reference's direct sums divide by zero there) */
gint wbfmm_total_field(gdouble k, gdouble *xs, gint xstride, gdouble *src,
                       gint sstride, gdouble *normals, gint nstr,
                       gdouble *dipoles, gint dstr, gint nq, gint nsrc,
                       gdouble *xf, gdouble *field, gint fstr);
gint wbfmm_total_field_grad(gdouble k, gdouble *xs, gint xstride, gdouble *src,
                            gint sstride, gdouble *normals, gint nstr,
                            gdouble *dipoles, gint dstr, gint nq, gint nsrc,
                            gdouble *xf, gdouble *field, gint fstr);
gint wbfmm_laplace_field(gdouble *xs, gint xstride, gdouble *src,
                         gint sstride, gint nq, gdouble *normals, gint nstr,
                         gdouble *dipoles, gint dstr, gint nsrc, gdouble *xf,
                         gdouble *field, gint fstr);
gint wbfmm_laplace_field_grad(gdouble *xs, gint xstride, gdouble *src,
                              gint sstride, gint nq, gdouble *normals,
                              gint nstr, gdouble *dipoles, gint dstr,
                              gint nsrc, gdouble *xf, gdouble *field,
                              gint fstr);

/* ---------------------------------------------------------- config */
gint wbfmm_library_config(wbfmm_library_config_t *c);
gint wbfmm_library_config_print(wbfmm_library_config_t *c, FILE *f);

/* ------------------------------------------- single precision (*_f) */
/* The reference's single-precision API (src/wbfmm.h:993-1112, the same
   sources compiled with WBFMM_REAL = gfloat): trees of FP32 points and
   coefficients, evaluated by the engine's FP32 form. */
wbfmm_tree_t *wbfmm_tree_new_f(gfloat *x, gfloat D, guint maxpoints);
gint wbfmm_tree_add_points_f(wbfmm_tree_t *t, gpointer pts, gsize pstr,
                             gpointer normals, gsize nstr, guint npts,
                             gboolean sorted);
gint wbfmm_tree_sort_points_f(wbfmm_tree_t *t, gpointer pts, gsize psize,
                              guint npts);
gint wbfmm_tree_refine_f(wbfmm_tree_t *t);
gint wbfmm_tree_coefficient_init_f(wbfmm_tree_t *t, guint l, guint nr, guint ns);
gint wbfmm_tree_laplace_coefficient_init_f(wbfmm_tree_t *t, guint l, guint nr,
                                           guint ns);
gint wbfmm_tree_coefficient_clear_f(wbfmm_tree_t *t, guint l);
guint64 wbfmm_point_box_f(wbfmm_tree_t *t, guint level, gfloat *x);
guint64 wbfmm_point_index_3d_f(gfloat *x, gfloat *c, gfloat D);
gint wbfmm_box_location_from_index_f(guint64 i, guint32 level, gfloat *x0,
                                     gfloat D, gfloat *x, gfloat *wb);
gint wbfmm_tree_box_centre_f(wbfmm_tree_t *t, guint level, guint64 b,
                             gfloat *xb, gfloat *wb);
gint wbfmm_points_origin_width_f(gfloat *x, gint str, gint n, gfloat *xmin,
                                 gfloat *xmax, gfloat *D, gboolean init_limits);
gint wbfmm_tree_write_sources_f(wbfmm_tree_t *t, gfloat *q, gint stride,
                                FILE *f);
gint wbfmm_truncation_number_f(wbfmm_tree_t *t, gfloat k, guint level,
                               gfloat tol);
gint wbfmm_shift_angle_table_init_f(void);
wbfmm_shift_operators_t *wbfmm_shift_operators_new_f(guint L, gboolean bw,
                                                     gfloat *work);
gint wbfmm_shift_operators_coaxial_SR_init_f(wbfmm_shift_operators_t *w,
                                             gfloat D, guint level, guint L,
                                             gfloat k, gfloat *work);
gint wbfmm_shift_operators_coaxial_SS_init_f(wbfmm_shift_operators_t *w,
                                             gfloat D, guint level, guint L,
                                             gfloat k, gfloat *work);
gint wbfmm_laplace_coaxial_translate_init_f(gint N);
gint wbfmm_tree_leaf_expansions_f(wbfmm_tree_t *t, gfloat k, gfloat *src,
                                  gint sstr, gfloat *dipoles, gint dstr,
                                  gboolean zero_expansions, gfloat *work);
gint wbfmm_tree_laplace_leaf_expansions_f(wbfmm_tree_t *t, gfloat *src,
                                          gint sstr, gfloat *dipoles,
                                          gint dstr, gboolean zero_expansions,
                                          gfloat *work);
gint wbfmm_upward_pass_f(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                         guint level, gfloat *work);
gint wbfmm_laplace_upward_pass_f(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                                 guint level, gfloat *work);
gint wbfmm_downward_pass_ref_f(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                               guint level, gfloat *work, gint nthreads);
gint wbfmm_laplace_downward_pass_ref_f(wbfmm_tree_t *t,
                                       wbfmm_shift_operators_t *op,
                                       guint level, gfloat *work,
                                       gint nthreads);
gint wbfmm_tree_box_local_field_f(wbfmm_tree_t *t, guint level, guint b,
                                  gfloat k, gfloat *x, gfloat *f, gint fstr,
                                  gfloat *src, gint sstr, gfloat *d, gint dstr,
                                  gboolean eval_neighbours, guint field,
                                  gfloat *work);
gint wbfmm_laplace_box_field_f(wbfmm_tree_t *t, guint level, guint b,
                               gfloat *src, gint sstr, gfloat *d, gint dstr,
                               guint field, gboolean eval_neighbours,
                               gfloat *x, gfloat *f, gint fstr, gfloat *work);
wbfmm_target_list_t *wbfmm_target_list_new_f(wbfmm_tree_t *t, guint npts);
gint wbfmm_target_list_add_points_f(wbfmm_target_list_t *l, gpointer pts,
                                    gsize pstr, guint npts);
gint wbfmm_target_list_local_coefficients_f(wbfmm_target_list_t *l, gfloat k,
                                            gfloat *work);
gint wbfmm_laplace_target_list_local_coefficients_f(wbfmm_target_list_t *l,
                                                    guint source,
                                                    gfloat *work);
gint wbfmm_target_list_local_field_f(wbfmm_target_list_t *l, gfloat *src,
                                     gint sstr, gfloat *nsrc, gint nstr,
                                     gfloat *f, gint fstr);
gint wbfmm_total_field_f(gfloat k, gfloat *xs, gint xstride, gfloat *src,
                         gint sstride, gfloat *normals, gint nstr,
                         gfloat *dipoles, gint dstr, gint nq, gint nsrc,
                         gfloat *xf, gfloat *field, gint fstr);
gint wbfmm_total_field_grad_f(gfloat k, gfloat *xs, gint xstride, gfloat *src,
                              gint sstride, gfloat *normals, gint nstr,
                              gfloat *dipoles, gint dstr, gint nq, gint nsrc,
                              gfloat *xf, gfloat *field, gint fstr);
gint wbfmm_laplace_field_f(gfloat *xs, gint xstride, gfloat *src,
                           gint sstride, gint nq, gfloat *normals, gint nstr,
                           gfloat *dipoles, gint dstr, gint nsrc, gfloat *xf,
                           gfloat *field, gint fstr);
gint wbfmm_laplace_field_grad_f(gfloat *xs, gint xstride, gfloat *src,
                                gint sstride, gint nq, gfloat *normals,
                                gint nstr, gfloat *dipoles, gint dstr,
                                gint nsrc, gfloat *xf, gfloat *field,
                                gint fstr);

/* ------------------------------------- single-expansion primitives
   (src/wbfmm.h:247-263, :266-320, :347-361, :402-420, :525-643).  The
   array primitives run on the GPU (one CTA per call; the caller's host
   arrays are copied in and out before the call returns); the scalar
   helpers run on the host.  Coefficient c of component j: Helmholtz at
   cfft[2 (c cstr + j)] (complex), Laplace at cfft[c cstr + j]
   (real-packed); rotation and coaxial translation leave Co = sc Co + T(Ci);
   expansions and fields are added to what the caller holds.  The FP32
   twins compute in FP64 and round. */
gint wbfmm_cartesian_to_spherical(gdouble *x0, gdouble *x, gdouble *r,
                                  gdouble *th, gdouble *ph);
gint wbfmm_legendre_init(gdouble C, gdouble S, gdouble *P0, gdouble *P10,
                         gdouble *P11);
gint wbfmm_legendre_recursion_array(gdouble **Pnm1, gdouble **Pn, gint n,
                                    gdouble C, gdouble S);
gint wbfmm_bessel_j_init(gdouble x, gdouble *j0, gdouble *j1);
gint wbfmm_bessel_j_recursion(gdouble *jnm1, gdouble *jn, gdouble x, gint n);
gint wbfmm_bessel_h_init(gdouble x, gdouble *h0, gdouble *h1);
gint wbfmm_bessel_h_recursion(gdouble *hnm1, gdouble *hn, gdouble x, gint n);
gint wbfmm_coefficients_H_rotation(gdouble *H, gint N, gdouble th,
                                   gdouble *work);
gint wbfmm_coefficients_RR_coaxial(gdouble *cfftRR, gint L, gdouble kr,
                                   gdouble *work);
gint wbfmm_coefficients_SR_coaxial(gdouble *cfftSR, gint L, gdouble kr,
                                   gdouble *work);
gint wbfmm_rotate_H_ref(gdouble *Co, gint cstro, gdouble *Ci, gint cstri,
                        gint N, gint nq, gdouble *H, gdouble ph, gdouble ch,
                        gdouble sc);
gint wbfmm_rotate_H_avx(gdouble *Co, gint cstro, gdouble *Ci, gint cstri,
                        gint N, gint nq, gdouble *H, gdouble ph, gdouble ch,
                        gdouble sc);
gint wbfmm_coaxial_translate_ref(gdouble *Co, gint cstro, gint No,
                                 gdouble *Ci, gint cstri, gint Ni, gint nq,
                                 gdouble *cfft, gint L, gboolean complex,
                                 gdouble sc);
gint wbfmm_expansion_h_cfft(gdouble k, gint N, gdouble *x0, gdouble *xs,
                            gdouble *q, gint nq, gdouble *cfft, gint cstr,
                            gdouble *work);
gint wbfmm_expansion_j_evaluate(gdouble k, gdouble *x0, gdouble *cfft,
                                gint cstr, gint N, gint nq, gdouble *xf,
                                gdouble *field, gint fstr, gdouble *work);
gint wbfmm_expansion_h_evaluate(gdouble k, gdouble *x0, gdouble *cfft,
                                gint cstr, gint N, gint nq, gdouble *xf,
                                gdouble *field, gint fstr, gdouble *work);
gint wbfmm_laplace_expansion_cfft(gint N, gdouble *x0, gdouble *xs,
                                  gdouble *q, gint nq, gdouble *cfft,
                                  gint cstr, gdouble *work);
gint wbfmm_laplace_expansion_evaluate(gdouble *x0, gdouble *cfft, gint cstr,
                                      gint N, gint nq, gdouble *xf,
                                      gdouble *field, gdouble *work);
/* potential and gradient fields (curl fields: wbfmm_laplace_box_field) */
gint wbfmm_laplace_expansion_local_eval(gdouble *x0, gdouble *cfft,
                                        gint cstr, gint N, gint nq,
                                        guint field, gdouble *xf,
                                        gdouble *f, gint fstr, gdouble *work);
gint wbfmm_laplace_rotate_H_ref(gdouble *Co, gint cstro, gdouble *Ci,
                                gint cstri, gint N, gint nq, gdouble *H,
                                gdouble ph, gdouble ch, gdouble sc);
gint wbfmm_laplace_rotate_H_avx(gdouble *Co, gint cstro, gdouble *Ci,
                                gint cstri, gint N, gint nq, gdouble *H,
                                gdouble ph, gdouble ch, gdouble sc);
gint wbfmm_laplace_coaxial_translate_SS(gdouble *Co, gint cstro, gint No,
                                        gdouble *Ci, gint cstri, gint Ni,
                                        gint nq, gdouble t, gdouble sc);
gint wbfmm_laplace_coaxial_translate_RR(gdouble *Co, gint cstro, gint No,
                                        gdouble *Ci, gint cstri, gint Ni,
                                        gint nq, gdouble t, gdouble sc);
gint wbfmm_laplace_coaxial_translate_SR(gdouble *Co, gint cstro, gint No,
                                        gdouble *Ci, gint cstri, gint Ni,
                                        gint nq, gdouble t, gdouble sc);

gint wbfmm_cartesian_to_spherical_f(gfloat *x0, gfloat *x, gfloat *r,
                                    gfloat *th, gfloat *ph);
gint wbfmm_legendre_init_f(gfloat C, gfloat S, gfloat *P0, gfloat *P10,
                           gfloat *P11);
gint wbfmm_legendre_recursion_array_f(gfloat **Pnm1, gfloat **Pn, gint n,
                                      gfloat C, gfloat S);
gint wbfmm_bessel_j_init_f(gfloat x, gfloat *j0, gfloat *j1);
gint wbfmm_bessel_j_recursion_f(gfloat *jnm1, gfloat *jn, gfloat x, gint n);
gint wbfmm_bessel_h_init_f(gfloat x, gfloat *h0, gfloat *h1);
gint wbfmm_bessel_h_recursion_f(gfloat *hnm1, gfloat *hn, gfloat x, gint n);
gint wbfmm_coefficients_H_rotation_f(gfloat *H, gint N, gfloat th,
                                     gfloat *work);
gint wbfmm_coefficients_RR_coaxial_f(gfloat *cfftRR, gint L, gfloat kr,
                                     gfloat *work);
gint wbfmm_coefficients_SR_coaxial_f(gfloat *cfftSR, gint L, gfloat kr,
                                     gfloat *work);
gint wbfmm_rotate_H_ref_f(gfloat *Co, gint cstro, gfloat *Ci, gint cstri,
                          gint N, gint nq, gfloat *H, gfloat ph, gfloat ch,
                          gfloat sc);
gint wbfmm_coaxial_translate_ref_f(gfloat *Co, gint cstro, gint No,
                                   gfloat *Ci, gint cstri, gint Ni, gint nq,
                                   gfloat *cfft, gint L, gboolean complex,
                                   gfloat sc);
gint wbfmm_expansion_h_cfft_f(gfloat k, gint N, gfloat *x0, gfloat *xs,
                              gfloat *q, gint nq, gfloat *cfft, gint cstr,
                              gfloat *work);
gint wbfmm_expansion_j_evaluate_f(gfloat k, gfloat *x0, gfloat *cfft,
                                  gint cstr, gint N, gint nq, gfloat *xf,
                                  gfloat *field, gint fstr, gfloat *work);
gint wbfmm_expansion_h_evaluate_f(gfloat k, gfloat *x0, gfloat *cfft,
                                  gint cstr, gint N, gint nq, gfloat *xf,
                                  gfloat *field, gint fstr, gfloat *work);
gint wbfmm_laplace_expansion_cfft_f(gint N, gfloat *x0, gfloat *xs,
                                    gfloat *q, gint nq, gfloat *cfft,
                                    gint cstr, gfloat *work);
gint wbfmm_laplace_expansion_evaluate_f(gfloat *x0, gfloat *cfft, gint cstr,
                                        gint N, gint nq, gfloat *xf,
                                        gfloat *field, gfloat *work);
gint wbfmm_laplace_expansion_local_eval_f(gfloat *x0, gfloat *cfft,
                                          gint cstr, gint N, gint nq,
                                          guint field, gfloat *xf, gfloat *f,
                                          gint fstr, gfloat *work);
gint wbfmm_laplace_rotate_H_ref_f(gfloat *Co, gint cstro, gfloat *Ci,
                                  gint cstri, gint N, gint nq, gfloat *H,
                                  gfloat ph, gfloat ch, gfloat sc);
gint wbfmm_laplace_coaxial_translate_SS_f(gfloat *Co, gint cstro, gint No,
                                          gfloat *Ci, gint cstri, gint Ni,
                                          gint nq, gfloat t, gfloat sc);
gint wbfmm_laplace_coaxial_translate_RR_f(gfloat *Co, gint cstro, gint No,
                                          gfloat *Ci, gint cstri, gint Ni,
                                          gint nq, gfloat t, gfloat sc);
gint wbfmm_laplace_coaxial_translate_SR_f(gfloat *Co, gint cstro, gint No,
                                          gfloat *Ci, gint cstri, gint Ni,
                                          gint nq, gfloat t, gfloat sc);

/* dispatch as in the reference (src/wbfmm.h:1138-1194) */
#define wbfmm_downward_pass_f wbfmm_downward_pass_ref_f
#define wbfmm_laplace_downward_pass_f wbfmm_laplace_downward_pass_ref_f
#define wbfmm_rotate_H_f wbfmm_rotate_H_ref_f
#define wbfmm_laplace_rotate_H_f wbfmm_laplace_rotate_H_ref_f
#define wbfmm_coaxial_translate wbfmm_coaxial_translate_ref
#define wbfmm_coaxial_translate_f wbfmm_coaxial_translate_ref_f
#ifdef WBFMM_USE_AVX
#define wbfmm_downward_pass wbfmm_downward_pass_avx
#define wbfmm_laplace_downward_pass wbfmm_laplace_downward_pass_avx
#define wbfmm_rotate_H wbfmm_rotate_H_avx
#define wbfmm_laplace_rotate_H wbfmm_laplace_rotate_H_avx
#else
#define wbfmm_downward_pass wbfmm_downward_pass_ref
#define wbfmm_laplace_downward_pass wbfmm_laplace_downward_pass_ref
#define wbfmm_rotate_H wbfmm_rotate_H_ref
#define wbfmm_laplace_rotate_H wbfmm_laplace_rotate_H_ref
#endif

#ifdef __cplusplus
}
#endif

#endif /* WBFMM_H_INCLUDED */
