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

/* dispatch as in the reference (src/wbfmm.h:1138-1194) */
#define wbfmm_downward_pass_f wbfmm_downward_pass_ref_f
#define wbfmm_laplace_downward_pass_f wbfmm_laplace_downward_pass_ref_f
#ifdef WBFMM_USE_AVX
#define wbfmm_downward_pass wbfmm_downward_pass_avx
#define wbfmm_laplace_downward_pass wbfmm_laplace_downward_pass_avx
#else
#define wbfmm_downward_pass wbfmm_downward_pass_ref
#define wbfmm_laplace_downward_pass wbfmm_laplace_downward_pass_ref
#endif

#ifdef __cplusplus
}
#endif

#endif /* WBFMM_H_INCLUDED */
