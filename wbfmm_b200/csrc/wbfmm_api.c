/*
 * The wbfmm C API (include/wbfmm.h) on the B200 engine (include/wbfmm_b200.h).
 *
 * Host-side state keeps the reference's structures and their host-visible
 * contents: t->ip and every box {i, n} after each call (computed on the GPU),
 * coefficient arrays in Layout L that the host can dereference (CUDA managed
 * memory, written by the GPU passes), fields accumulated into the caller's
 * arrays.  All FMM arithmetic runs on the GPU; this file only orchestrates.
 * Errors that the reference reports with g_error abort here too, with the
 * engine's message.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "wbfmm.h"
#include "wbfmm_b200.h"

/* ------------------------------------------------------------ helpers */
static void die(const char *fn, const char *msg) {
  fprintf(stderr, "wbfmm: %s: %s\n", fn, msg);
  abort();
}

static void check(const char *fn, int rc) {
  if (rc != 0) die(fn, wbfmm_b200_last_error());
}

#define DT_MAX_NQ 16             /* source components of one tree */

/* the tree as callers see it, followed by the engine state behind it */
typedef struct {
  wbfmm_tree_t t;
  wbfmm_b200_solver_t *s;
  double k;
  int ready;                     /* solver holds the current points */
  const void *q, *dip;           /* strengths last uploaded */
  int qstr, dstr;
  const void *targets;           /* target set last uploaded */
  guint ntargets;
  gboolean managed[2][WBFMM_TREE_MAX_DEPTH + 1];
  int fp32;                      /* a tree of the single-precision API (*_f) */
  double *pts64, *nrm64;         /* FP64 copies of FP32 points and normals */
  /* Laplace sources of nq > 1 components: one engine solver per component
     (s for component 0, sc[c] for the others), each on its own coefficient
     arrays cms/cmr (engine layout), copied into the tree's interleaved
     arrays (src/laplace.c:795-852) after every pass */
  int nq;
  wbfmm_b200_solver_t *sc[DT_MAX_NQ];
  void *cms[DT_MAX_NQ][WBFMM_TREE_MAX_DEPTH + 1], *cmr[DT_MAX_NQ][WBFMM_TREE_MAX_DEPTH + 1];
} dtree_t;

#define DT(_t) ((dtree_t *)(_t))

static int ncomp(const dtree_t *d) { return d->nq > 1 ? d->nq : 1; }
static wbfmm_b200_solver_t *comp_solver(dtree_t *d, int c) { return c ? d->sc[c] : d->s; }

static void drop_solver(dtree_t *d) {
  int c;
  if (d->s) wbfmm_b200_solver_destroy(d->s);
  d->s = NULL;
  for (c = 1; c < DT_MAX_NQ; c++) {
    if (d->sc[c]) wbfmm_b200_solver_destroy(d->sc[c]);
    d->sc[c] = NULL;
  }
  d->ready = 0;
  d->q = d->dip = NULL;
  d->targets = NULL;
}

/* n records of 3 FP32 values at a byte stride, as 3 n doubles (exact) */
static double *widen3(const char *p, gsize stride, guint n) {
  double *o = malloc(sizeof(double) * 3 * (n ? n : 1));
  guint i;
  int a;
  if (!o) die("wbfmm", "out of memory");
  for (i = 0; i < n; i++)
    for (a = 0; a < 3; a++) o[3 * (size_t)i + a] = ((const float *)(p + (size_t)i * stride))[a];
  return o;
}

/* n strengths of w values at a stride of `str` FP32 values, as doubles */
static double *widen_strengths(const float *q, gint str, guint n, int w) {
  double *o;
  guint i;
  int c;
  if (!q) return NULL;
  o = malloc(sizeof(double) * w * (n ? n : 1));
  if (!o) die("wbfmm", "out of memory");
  for (i = 0; i < n; i++)
    for (c = 0; c < w; c++) o[(size_t)i * w + c] = q[(size_t)i * str + c];
  return o;
}

static uint64_t spread3(uint64_t v) {
  uint64_t r = 0;
  int b;
  for (b = 0; b < 21; b++) r |= ((v >> b) & 1ull) << (3 * b);
  return r;
}

static uint32_t gather3(uint64_t m) {
  uint32_t r = 0;
  int b;
  for (b = 0; b < 21; b++) r |= (uint32_t)((m >> (3 * b)) & 1ull) << b;
  return r;
}

/* ------------------------------------------------ trees and indexing */
/* src/boxes.c:58-91 */
wbfmm_tree_t *wbfmm_tree_new(gdouble *x, gdouble D, guint maxpoints) {
  dtree_t *d = calloc(1, sizeof(dtree_t));
  wbfmm_tree_t *t;
  double *xt;
  if (!d) die(__func__, "out of memory");
  t = &d->t;
  t->maxpoints = maxpoints;
  t->ip = malloc(sizeof(guint) * (maxpoints ? maxpoints : 1));
  t->boxes[0] = calloc(1, sizeof(wbfmm_box_t));
  t->size = sizeof(gdouble);
  xt = (double *)t->x;
  xt[0] = x[0]; xt[1] = x[1]; xt[2] = x[2];
  t->D = D;
  return t;
}

/* box {i, n} of levels 0..depth from the GPU tree build */
static void refresh_boxes(wbfmm_tree_t *t) {
  size_t total = 0, off = 0;
  guint l;
  uint32_t *bi, *bn;
  for (l = 0; l <= t->depth; l++) total += (size_t)1 << (3 * l);
  bi = malloc(sizeof(uint32_t) * total);
  bn = malloc(sizeof(uint32_t) * total);
  if (DT(t)->fp32)
    check("wbfmm_tree_refine_f",
          wbfmm_b200_tree_structure_f((int)t->npoints, (const float *)t->points,
                                      (int)(t->pstr / sizeof(float)),
                                      (const float *)t->x, (float)t->D, (int)t->depth,
                                      t->ip, bi, bn));
  else
    check("wbfmm_tree_refine",
          wbfmm_b200_tree_structure((int)t->npoints, (const double *)t->points,
                                    (int)(t->pstr / sizeof(double)),
                                    (const double *)t->x, t->D, (int)t->depth,
                                    t->ip, bi, bn));
  for (l = 0; l <= t->depth; l++) {
    size_t nb = (size_t)1 << (3 * l), b;
    for (b = 0; b < nb; b++) {
      t->boxes[l][b].i = bi[off + b];
      t->boxes[l][b].n = bn[off + b];
    }
    off += nb;
  }
  free(bi);
  free(bn);
}

/* src/boxes.c:118-166: domain check, stable Morton sort of t->ip */
gint wbfmm_tree_add_points(wbfmm_tree_t *t, gpointer pts, gsize pstr,
                           gpointer normals, gsize nstr, guint npts,
                           gboolean sorted) {
  if (npts > t->maxpoints) die(__func__, "too many points for tree");
  if (pstr % sizeof(double) || (normals && nstr % sizeof(double)))
    die(__func__, "point and normal strides must be multiples of sizeof(double)");
  t->npoints = npts;
  t->points = (char *)pts;
  t->pstr = pstr;
  t->normals = (char *)normals;
  t->nstr = nstr;
  t->sorted = sorted;
  drop_solver(DT(t));
  refresh_boxes(t);
  t->boxes[0][0].i = 0;
  t->boxes[0][0].n = npts;
  return 0;
}

/* src/boxes.c:190-206: sort the caller's point records by Morton key */
gint wbfmm_tree_sort_points(wbfmm_tree_t *t, gpointer pts, gsize psize,
                            guint npts) {
  uint32_t *ip = malloc(sizeof(uint32_t) * (npts ? npts : 1));
  char *tmp = malloc(psize * (npts ? npts : 1));
  guint i;
  if (psize % sizeof(double)) die(__func__, "record size must be a multiple of sizeof(double)");
  check(__func__, wbfmm_b200_tree_structure((int)npts, (const double *)pts,
                                            (int)(psize / sizeof(double)),
                                            (const double *)t->x, t->D, 0, ip,
                                            NULL, NULL));
  for (i = 0; i < npts; i++)
    memcpy(tmp + (size_t)i * psize, (char *)pts + (size_t)ip[i] * psize, psize);
  memcpy(pts, tmp, psize * npts);
  free(tmp);
  free(ip);
  return 0;
}

/* src/tree.c:57-72 */
gint wbfmm_tree_add_level(wbfmm_tree_t *t) {
  if (t->depth >= WBFMM_TREE_MAX_DEPTH) die(__func__, "tree already at maximum depth");
  t->depth++;
  if (!t->boxes[t->depth])
    t->boxes[t->depth] = calloc((size_t)1 << (3 * t->depth), sizeof(wbfmm_box_t));
  return 0;
}

/* src/boxes.c:208-277: one more level; {i, n} of every level as the
   reference leaves them after this many refinements */
gint wbfmm_tree_refine(wbfmm_tree_t *t) {
  wbfmm_tree_add_level(t);
  drop_solver(DT(t));
  refresh_boxes(t);
  return 0;
}

static void *managed_or_die(size_t bytes) {
  void *p = wbfmm_b200_managed_alloc(bytes);
  if (!p) die("wbfmm_tree_coefficient_init", wbfmm_b200_last_error());
  return p;
}

static void free_components(dtree_t *d, guint l) {
  int c;
  for (c = 0; c < DT_MAX_NQ; c++) {
    if (d->cms[c][l]) wbfmm_b200_managed_free(d->cms[c][l]);
    if (d->cmr[c][l]) wbfmm_b200_managed_free(d->cmr[c][l]);
    d->cms[c][l] = d->cmr[c][l] = NULL;
  }
}

/* box b's coefficients start at ((b & ~7) nc + (b & 7)) nq, coefficient c
   of component q at +8 nq c + q (w values each) */
static void coefficient_init(wbfmm_tree_t *t, guint l, guint nr, guint ns,
                             int w) {
  dtree_t *d = DT(t);
  size_t nb = (size_t)1 << (3 * l), b, nc;
  gint nq = wbfmm_tree_source_size(t), c;
  if (nq < 1) die("wbfmm_tree_coefficient_init", "tree has invalid number of components in source terms");
  if (nq > 1 && w != 1) die("wbfmm_tree_coefficient_init", "multi-component sources (nq > 1) are supported for Laplace trees");
  if (nq > DT_MAX_NQ) die("wbfmm_tree_coefficient_init", "too many source components (at most 16)");
  if (l > t->depth) die("wbfmm_tree_coefficient_init", "level deeper than the tree");
  drop_solver(d);
  d->nq = nq;
  t->order_s[l] = ns;
  t->order_r[l] = nr;
  if (d->managed[0][l]) wbfmm_b200_managed_free(t->mps[l]);
  if (d->managed[1][l]) wbfmm_b200_managed_free(t->mpr[l]);
  free_components(d, l);
  t->mps[l] = t->mpr[l] = NULL;
  d->managed[0][l] = d->managed[1][l] = FALSE;
  if (ns) {
    nc = (size_t)(ns + 1) * (ns + 1);
    t->mps[l] = managed_or_die(nb * nc * w * nq * t->size);
    d->managed[0][l] = TRUE;
    for (b = 0; b < nb; b++)
      t->boxes[l][b].mps = (char *)t->mps[l] + ((b & ~7) * nc + (b & 7)) * nq * w * t->size;
    if (nq > 1)
      for (c = 0; c < nq; c++) d->cms[c][l] = managed_or_die(nb * nc * t->size);
  }
  if (nr) {
    nc = (size_t)(nr + 1) * (nr + 1);
    t->mpr[l] = managed_or_die(nb * nc * w * nq * t->size);
    d->managed[1][l] = TRUE;
    for (b = 0; b < nb; b++)
      t->boxes[l][b].mpr = (char *)t->mpr[l] + ((b & ~7) * nc + (b & 7)) * nq * w * t->size;
    if (nq > 1)
      for (c = 0; c < nq; c++) d->cmr[c][l] = managed_or_die(nb * nc * t->size);
  }
}

/* nq > 1: the components' level-l arrays into the tree's interleaved one */
static void interleave(wbfmm_tree_t *t, guint l, int singular) {
  dtree_t *d = DT(t);
  const int nq = d->nq;
  const guint p = singular ? t->order_s[l] : t->order_r[l];
  const size_t nb = (size_t)1 << (3 * l), nc = (size_t)(p + 1) * (p + 1), es = t->size;
  char *dst = (char *)(singular ? t->mps[l] : t->mpr[l]);
  size_t g, i, j;
  int q;
  if (nq <= 1 || !dst) return;
  for (q = 0; q < nq; q++) {
    const char *src = (const char *)(singular ? d->cms[q][l] : d->cmr[q][l]);
    for (g = 0; g < nb / 8 + (nb < 8); g++)
      for (i = 0; i < nc; i++)
        for (j = 0; j < 8 && g * 8 + j < nb; j++)
          memcpy(dst + ((g * 8 * nc + i * 8 + j) * nq + q) * es,
                 src + ((g * nc + i) * 8 + j) * es, es);
  }
}

/* src/boxes.c:518-583 (Helmholtz, complex Layout L) */
gint wbfmm_tree_coefficient_init(wbfmm_tree_t *t, guint l, guint nr, guint ns) {
  if (t->problem != WBFMM_PROBLEM_HELMHOLTZ) die(__func__, "tree problem is not Helmholtz");
  coefficient_init(t, l, nr, ns, 2);
  return 0;
}

/* src/laplace.c:795-852 (Laplace, real-packed Layout L) */
gint wbfmm_tree_laplace_coefficient_init(wbfmm_tree_t *t, guint l, guint nr,
                                         guint ns) {
  if (t->problem != WBFMM_PROBLEM_LAPLACE) die(__func__, "tree problem is not Laplace");
  coefficient_init(t, l, nr, ns, 1);
  return 0;
}

/* bytes of a level's coefficient array of order p */
/* bytes of one component's level array of order p */
static size_t level_bytes(wbfmm_tree_t *t, guint l, guint p) {
  return ((size_t)1 << (3 * l)) * (size_t)(p + 1) * (p + 1) *
         (t->problem == WBFMM_PROBLEM_HELMHOLTZ ? 2 : 1) * t->size;
}

/* zero the singular (or regular) expansions of level l, every component */
static void zero_level(wbfmm_tree_t *t, guint l, int singular) {
  dtree_t *d = DT(t);
  const guint p = singular ? t->order_s[l] : t->order_r[l];
  void *a = singular ? t->mps[l] : t->mpr[l];
  int c;
  if (!a) return;
  memset(a, 0, level_bytes(t, l, p) * ncomp(d));
  if (d->nq > 1)
    for (c = 0; c < d->nq; c++) memset(singular ? d->cms[c][l] : d->cmr[c][l], 0, level_bytes(t, l, p));
}

/* src/boxes.c:636-673 */
gint wbfmm_tree_coefficient_clear(wbfmm_tree_t *t, guint l) {
  zero_level(t, l, 1);
  zero_level(t, l, 0);
  return 0;
}

/* src/tree.c:137-153 */
gint wbfmm_tree_coefficients_zero(wbfmm_tree_t *t, guint level) {
  zero_level(t, level, 0);
  return 0;
}

/* src/boxes.c:585-634 */
guint64 wbfmm_point_box(wbfmm_tree_t *t, guint level, gdouble *x) {
  const double *x0 = (const double *)t->x;
  double wb = t->D / (double)(1u << level);
  if (x[0] < x0[0] || x[0] > x0[0] + t->D || x[1] < x0[1] ||
      x[1] > x0[1] + t->D || x[2] < x0[2] || x[2] > x0[2] + t->D)
    die(__func__, "point not in octree");
  return wbfmm_box_index((guint32)floor((x[0] - x0[0]) / wb),
                         (guint32)floor((x[1] - x0[1]) / wb),
                         (guint32)floor((x[2] - x0[2]) / wb));
}

/* src/boxes.c:324-339 */
guint64 wbfmm_point_index_3d(gdouble *x, gdouble *c, gdouble D) {
  return wbfmm_box_index((guint32)((x[0] - c[0]) / D * WBFMM_INDEX_SHIFT),
                         (guint32)((x[1] - c[1]) / D * WBFMM_INDEX_SHIFT),
                         (guint32)((x[2] - c[2]) / D * WBFMM_INDEX_SHIFT));
}

/* src/indexing.c:170-246 */
guint64 wbfmm_point_locate_box(guint64 x, guint level) {
  return x >> 3 * (20 - level);
}
gint wbfmm_point_from_index(guint64 i, guint32 *x, guint32 *y, guint32 *z) {
  return wbfmm_box_location(i, x, y, z);
}
guint64 wbfmm_box_index(guint32 i, guint32 j, guint32 k) {
  return spread3(i) | (spread3(j) << 1) | (spread3(k) << 2);
}
gint wbfmm_box_location(guint64 idx, guint32 *i, guint32 *j, guint32 *k) {
  if (i) *i = gather3(idx);
  if (j) *j = gather3(idx >> 1);
  if (k) *k = gather3(idx >> 2);
  return 0;
}
guint64 wbfmm_box_parent(guint64 idx) { return idx >> 3; }
guint64 wbfmm_box_first_child(guint64 idx) { return idx << 3; }

/* src/indexing.c:250-286 */
gint wbfmm_box_neighbours(guint level, guint64 idx, guint64 *nb) {
  guint32 i, j, k, a, b, c, n1 = (1u << level) - 1;
  guint32 i0, i1, j0, j1, k0, k1;
  gint n = 0;
  wbfmm_box_location(idx, &i, &j, &k);
  i0 = i > 0 ? i - 1 : 0; j0 = j > 0 ? j - 1 : 0; k0 = k > 0 ? k - 1 : 0;
  i1 = i < n1 ? i + 1 : n1; j1 = j < n1 ? j + 1 : n1; k1 = k < n1 ? k + 1 : n1;
  for (a = i0; a <= i1; a++)
    for (b = j0; b <= j1; b++)
      for (c = k0; c <= k1; c++) nb[n++] = wbfmm_box_index(a, b, c);
  return n;
}

static void list4_range(guint level, guint32 i, gint *lo, gint *hi) {
  gint n = 1 << level;
  *lo = (gint)(i - i % 2);
  *hi = *lo + 3 < n - 1 ? *lo + 3 : n - 1;
  if (*lo > 0) *lo -= 2;
}

/* exact order of azimuths atan2(y, x) in (-pi, pi] of integer vectors */
static int azimuth_cmp(int ax, int ay, int bx, int by) {
  int ha, hb, pa, pb, cross;
  if (ax == 0 && ay == 0) ax = 1;
  if (bx == 0 && by == 0) bx = 1;
  ha = ay < 0 ? 0 : 1;
  hb = by < 0 ? 0 : 1;
  if (ha != hb) return ha - hb;
  pa = ay == 0 && ax < 0;        /* azimuth pi, the largest */
  pb = by == 0 && bx < 0;
  if (pa || pb) return pa - pb;
  cross = ax * by - ay * bx;
  return cross > 0 ? -1 : (cross < 0 ? 1 : 0);
}

/* list-4 shift code (dx+3)*49 + (dy+3)*7 + dz+3 -> offset */
static void shift_offset(guint64 code, int *dx, int *dy, int *dz) {
  *dx = (int)(code / 49) - 3;
  *dy = (int)(code / 7 % 7) - 3;
  *dz = (int)(code % 7) - 3;
}

/* Entries with the same shift direction (hence the same rotations) become
   contiguous, directions ordered as the reference's rotation tables are:
   polar angle increasing (cos theta decreasing), then azimuth increasing;
   equal directions by increasing distance.  Comparisons are exact. */
static int cmp_shift(const void *a, const void *b) {
  const guint64 *x = a, *y = b;
  int ax, ay, az, bx, by, bz, c;
  long r2a, r2b, ca, cb;
  shift_offset(x[1], &ax, &ay, &az);
  shift_offset(y[1], &bx, &by, &bz);
  r2a = (long)ax * ax + ay * ay + az * az;
  r2b = (long)bx * bx + by * by + bz * bz;
  /* cos^2 theta with sign, compared as az|az|/r2a against bz|bz|/r2b */
  ca = (long)az * (az < 0 ? -az : az) * r2b;
  cb = (long)bz * (bz < 0 ? -bz : bz) * r2a;
  if (ca != cb) return ca > cb ? -1 : 1;
  c = azimuth_cmp(ax, ay, bx, by);
  if (c) return c;
  return r2a < r2b ? -1 : (r2a > r2b ? 1 : 0);
}

/* src/indexing.c:330-377 */
gint wbfmm_box_interaction_list_4(guint level, guint64 idx, guint64 *list,
                                  gboolean sort) {
  guint32 i, j, k;
  gint a0, a1, b0, b1, c0, c1, a, b, c, n = 0;
  wbfmm_box_location(idx, &i, &j, &k);
  list4_range(level, i, &a0, &a1);
  list4_range(level, j, &b0, &b1);
  list4_range(level, k, &c0, &c1);
  for (a = a0; a <= a1; a++)
    for (b = b0; b <= b1; b++)
      for (c = c0; c <= c1; c++) {
        gint dx = a - (gint)i, dy = b - (gint)j, dz = c - (gint)k;
        if (abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1) continue;
        list[2 * n] = wbfmm_box_index(a, b, c);
        list[2 * n + 1] = (guint64)((dx + 3) * 49 + (dy + 3) * 7 + dz + 3);
        n++;
      }
  if (sort) qsort(list, n, 2 * sizeof(guint64), cmp_shift);
  return n;
}

/* src/indexing.c:394-427 */
gint wbfmm_box_interaction_grid_4(guint level, guint64 idx, guint64 grid[]) {
  guint64 list[2 * 189];
  gint n = wbfmm_box_interaction_list_4(level, idx, list, FALSE), m;
  memset(grid, 0, 343 * sizeof(guint64));
  for (m = 0; m < n; m++) grid[list[2 * m + 1]] = list[2 * m] + 1;
  return 0;
}

/* src/util.c:290-330 */
gint wbfmm_box_location_from_index(guint64 idx, guint32 level, gdouble *x0,
                                   gdouble D, gdouble *x, gdouble *wb) {
  guint32 i, j, k;
  if (!(idx < ((guint64)1 << (3 * level)))) die(__func__, "box is not at this level");
  *wb = D / (double)(1u << level);
  wbfmm_box_location(idx, &i, &j, &k);
  x[0] = x0[0] + (*wb) * i;
  x[1] = x0[1] + (*wb) * j;
  x[2] = x0[2] + (*wb) * k;
  return 0;
}

gint wbfmm_tree_box_centre(wbfmm_tree_t *t, guint level, guint64 b,
                           gdouble *xb, gdouble *wb) {
  wbfmm_box_location_from_index(b, level, (gdouble *)t->x, t->D, xb, wb);
  xb[0] += 0.5 * (*wb); xb[1] += 0.5 * (*wb); xb[2] += 0.5 * (*wb);
  return 0;
}

/* src/util.c:375-405 */
gint wbfmm_points_origin_width(gdouble *x, gint str, gint n, gdouble *xmin,
                               gdouble *xmax, gdouble *D,
                               gboolean init_limits) {
  gint i, a;
  if (init_limits)
    for (a = 0; a < 3; a++) { xmin[a] = 3.4028234663852886e38; xmax[a] = -3.4028234663852886e38; }
  for (i = 0; i < n; i++)
    for (a = 0; a < 3; a++) {
      if (x[str * i + a] < xmin[a]) xmin[a] = x[str * i + a];
      if (x[str * i + a] > xmax[a]) xmax[a] = x[str * i + a];
    }
  *D = xmax[0] - xmin[0];
  if (xmax[1] - xmin[1] > *D) *D = xmax[1] - xmin[1];
  if (xmax[2] - xmin[2] > *D) *D = xmax[2] - xmin[2];
  return 0;
}

/* src/util.c:425-450: the points in tree order (q and stride unused) */
gint wbfmm_tree_write_sources(wbfmm_tree_t *t, gdouble *q, gint stride, FILE *f)
{
  guint i;
  (void)q; (void)stride;
  for (i = 0; i < t->npoints; i++) {
    const guint idx = t->ip[i];
    const gdouble *x = (const gdouble *)(t->points + (gsize)idx * t->pstr);
    fprintf(f, "%u %u %g %g %g\n", i, idx, x[0], x[1], x[2]);
  }
  return 0;
}

/* Gumerov & Duraiswami (2009) truncation rule, as src/util.c:474-503 */
gint wbfmm_truncation_number(wbfmm_tree_t *t, gdouble k, guint level,
                             gdouble tol) {
  const double del = 2.0;
  double ka = t->D / (double)(1u << level) * 0.5 * sqrt(3.0) * k;
  double plo = 1.0 - log(tol * (1.0 - 1.0 / del) * sqrt(1.0 - 1.0 / del)) / log(del);
  double phi = cbrt(3.0 * log(1.0 / tol));
  phi = ka + 0.5 * phi * phi * cbrt(ka);
  return (gint)ceil(sqrt(sqrt(plo * plo * plo * plo + phi * phi * phi * phi)));
}

/* ------------------------------------------------------- operators */
gint wbfmm_shift_angle_table_init(void) { return 0; }

wbfmm_shift_operators_t *wbfmm_shift_operators_new(guint L, gboolean bw,
                                                   gdouble *work) {
  wbfmm_shift_operators_t *op = calloc(1, sizeof(wbfmm_shift_operators_t));
  (void)work;
  op->size = sizeof(gdouble);
  op->Lmax = L;
  op->bw = bw;
  op->nerot = wbfmm_element_number_rotation(L);
  return op;
}

gint wbfmm_shift_operators_coaxial_SR_init(wbfmm_shift_operators_t *w,
                                           gdouble D, guint level, guint L,
                                           gdouble k, gdouble *work) {
  (void)D; (void)k; (void)work;
  w->L[level] = L;
  if (level + 1 > w->nlevels) w->nlevels = level + 1;
  return 0;
}

gint wbfmm_shift_operators_coaxial_SS_init(wbfmm_shift_operators_t *w,
                                           gdouble D, guint level, guint L,
                                           gdouble k, gdouble *work) {
  (void)w; (void)D; (void)level; (void)L; (void)k; (void)work;
  return 0;
}

gint wbfmm_laplace_coaxial_translate_init(gint N) {
  (void)N;
  return 0;
}

/* ---------------------------------------------------------- engine */
static wbfmm_b200_solver_t *solver_for(wbfmm_tree_t *t, double k,
                                       const char *fn) {
  dtree_t *d = DT(t);
  wbfmm_b200_config_t c;
  guint l;
  int q;
  if (d->s && d->ready && (t->problem == WBFMM_PROBLEM_LAPLACE || d->k == k))
    return d->s;
  drop_solver(d);
  memset(&c, 0, sizeof(c));
  c.problem = t->problem == WBFMM_PROBLEM_HELMHOLTZ ? WBFMM_B200_HELMHOLTZ
                                                    : WBFMM_B200_LAPLACE;
  c.depth = (int)t->depth;
  for (l = 1; l <= t->depth; l++) {
    if (!t->mps[l] || !t->mpr[l])
      die(fn, "coefficients must be initialised at every level 1..depth");
    c.order_s[l] = (int)t->order_s[l];
    c.order_r[l] = (int)t->order_r[l];
  }
  c.k = k;
  if (d->fp32) {
    const float *xf = (const float *)t->x;
    c.x0[0] = xf[0]; c.x0[1] = xf[1]; c.x0[2] = xf[2];
  } else {
    memcpy(c.x0, t->x, sizeof(c.x0));
  }
  c.D = t->D;
  /* the single-precision API runs the FP32 form, with the tree's keys and
     boxes computed as the reference's single-precision build does */
  c.precision = d->fp32 ? WBFMM_B200_FP32 : WBFMM_B200_FP64;
  c.keys_fp32 = d->fp32;
  c.field = WBFMM_B200_POTENTIAL | WBFMM_B200_GRADIENT;
  c.managed = 1;
  if (d->fp32) {
    free(d->pts64);
    free(d->nrm64);
    d->pts64 = widen3(t->points, t->pstr, t->npoints);
    d->nrm64 = t->normals ? widen3(t->normals, t->nstr, t->npoints) : NULL;
  }
  for (q = 0; q < ncomp(d); q++) {
    wbfmm_b200_solver_t **sp = q ? &d->sc[q] : &d->s;
    check(fn, wbfmm_b200_solver_create(sp, &c, NULL));
    for (l = 1; l <= t->depth; l++)
      check(fn, wbfmm_b200_adopt_coefficients(*sp, (int)l, d->nq > 1 ? d->cms[q][l] : t->mps[l],
                                              d->nq > 1 ? d->cmr[q][l] : t->mpr[l]));
    if (d->fp32)
      check(fn, wbfmm_b200_set_sources(*sp, (int)t->npoints, d->pts64, 3, d->nrm64, 3, 0));
    else
      check(fn, wbfmm_b200_set_sources(*sp, (int)t->npoints, (const double *)t->points,
                                       (int)(t->pstr / sizeof(double)),
                                       (const double *)t->normals,
                                       (int)(t->nstr / sizeof(double)), 0));
  }
  d->k = k;
  d->ready = 1;
  return d->s;
}

/* strengths q[i*qstr], dip[i*dstr] (doubles, or floats for an FP32 tree);
   component c of a multi-component tree at q[i*qstr + c], dip[i*dstr + c] */
static void strengths_for(dtree_t *d, const void *q, int qstr,
                          const void *dip, int dstr, const char *fn) {
  int c;
  if (d->q == q && d->qstr == qstr && d->dip == dip && d->dstr == dstr && (q || dip))
    return;
  if (dip && !d->t.normals) die(fn, "no normals in tree but dipole strengths specified");
  for (c = 0; c < ncomp(d); c++) {
    wbfmm_b200_solver_t *s = comp_solver(d, c);
    if (d->fp32) {
      const int w = d->t.problem == WBFMM_PROBLEM_HELMHOLTZ ? 2 : 1;
      double *q64 = widen_strengths(q ? (const float *)q + c : NULL, qstr, d->t.npoints, w);
      double *d64 = widen_strengths(dip ? (const float *)dip + c : NULL, dstr, d->t.npoints, w);
      check(fn, wbfmm_b200_set_strengths(s, q64, w, d64, w, 0));
      free(q64);
      free(d64);
    } else {
      check(fn, wbfmm_b200_set_strengths(s, q ? (const double *)q + c : NULL, qstr,
                                         dip ? (const double *)dip + c : NULL, dstr, 0));
    }
  }
  d->q = q; d->qstr = qstr; d->dip = dip; d->dstr = dstr;
}

/* ---------------------------------------------------------- passes */
static gint leaf(wbfmm_tree_t *t, double k, const void *src, gint sstr,
                 const void *dipoles, gint dstr, gboolean zero, const char *fn) {
  dtree_t *d = DT(t);
  int c;
  solver_for(t, k, fn);
  if (!src && !dipoles) {
    if (zero) zero_level(t, t->depth, 1);
    return 0;
  }
  d->q = d->dip = NULL;       /* strengths may have changed in place */
  strengths_for(d, src, sstr, dipoles, dstr, fn);
  for (c = 0; c < ncomp(d); c++) {
    wbfmm_b200_solver_t *s = comp_solver(d, c);
    check(fn, wbfmm_b200_set_p2m_accumulate(s, zero ? 0 : 1));
    check(fn, wbfmm_b200_leaf_expansions(s));
    check(fn, wbfmm_b200_synchronize(s));
  }
  interleave(t, t->depth, 1);
  return 0;
}

/* src/boxes.c:341-490 */
gint wbfmm_tree_leaf_expansions(wbfmm_tree_t *t, gdouble k, gdouble *src,
                                gint sstr, gdouble *dipoles, gint dstr,
                                gboolean zero_expansions, gdouble *work) {
  (void)work;
  if (t->problem != WBFMM_PROBLEM_HELMHOLTZ) die(__func__, "tree problem is not Helmholtz");
  return leaf(t, k, src, sstr, dipoles, dstr, zero_expansions, __func__);
}

/* src/laplace.c:854-989 */
gint wbfmm_tree_laplace_leaf_expansions(wbfmm_tree_t *t, gdouble *src,
                                        gint sstr, gdouble *dipoles,
                                        gint dstr, gboolean zero_expansions,
                                        gdouble *work) {
  (void)work;
  if (t->problem != WBFMM_PROBLEM_LAPLACE) die(__func__, "tree problem is not Laplace");
  return leaf(t, 0.0, src, sstr, dipoles, dstr, zero_expansions, __func__);
}

static gint upward(wbfmm_tree_t *t, guint level, const char *fn) {
  dtree_t *d = DT(t);
  int c;
  if (!d->s || !d->ready) die(fn, "leaf expansions must be computed first");
  for (c = 0; c < ncomp(d); c++) {
    check(fn, wbfmm_b200_upward_pass(comp_solver(d, c), (int)level));
    check(fn, wbfmm_b200_synchronize(comp_solver(d, c)));
  }
  if (level >= 1) interleave(t, level - 1, 1);
  return 0;
}

static gint downward(wbfmm_tree_t *t, guint level, const char *fn) {
  dtree_t *d = DT(t);
  int c;
  if (!d->s || !d->ready) die(fn, "leaf expansions must be computed first");
  for (c = 0; c < ncomp(d); c++) {
    check(fn, wbfmm_b200_downward_pass(comp_solver(d, c), (int)level));
    check(fn, wbfmm_b200_synchronize(comp_solver(d, c)));
  }
  interleave(t, level, 0);
  if (level < t->depth) interleave(t, level + 1, 0);   /* its L2L part */
  return 0;
}

/* src/pass.c:581-632 */
gint wbfmm_upward_pass(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                       guint level, gdouble *work) {
  (void)op; (void)work;
  return upward(t, level, __func__);
}
/* src/pass-laplace.c:433-486 */
gint wbfmm_laplace_upward_pass(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                               guint level, gdouble *work) {
  (void)op; (void)work;
  return upward(t, level, __func__);
}
/* src/pass.c:448-579; nthreads has no meaning on the GPU */
gint wbfmm_downward_pass_ref(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                             guint level, gdouble *work, gint nthreads) {
  (void)op; (void)work; (void)nthreads;
  return downward(t, level, __func__);
}
gint wbfmm_downward_pass_avx(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                             guint level, gdouble *work, gint nthreads) {
  (void)op; (void)work; (void)nthreads;
  return downward(t, level, __func__);
}
/* src/pass-laplace.c:362-431 */
gint wbfmm_laplace_downward_pass_ref(wbfmm_tree_t *t,
                                     wbfmm_shift_operators_t *op, guint level,
                                     gdouble *work, gint nthreads) {
  (void)op; (void)work; (void)nthreads;
  return downward(t, level, __func__);
}
gint wbfmm_laplace_downward_pass_avx(wbfmm_tree_t *t,
                                     wbfmm_shift_operators_t *op, guint level,
                                     gdouble *work, gint nthreads) {
  (void)op; (void)work; (void)nthreads;
  return downward(t, level, __func__);
}

/* ------------------------------------------------------ evaluation */
/* evaluate `n` targets with `field` and add into f[i*fstr + ...]:
   potential (w values) and/or gradient (3w values, after the potential when
   both are asked for) */
static void evaluate_targets(dtree_t *d, const void *key, guint n,
                             const double *x, int xstr, guint field,
                             gboolean neighbours, void *fv, gint fstr,
                             const char *fn) {
  int w = d->t.problem == WBFMM_PROBLEM_HELMHOLTZ ? 2 : 1;
  int want = (field & WBFMM_FIELD_POTENTIAL ? WBFMM_B200_POTENTIAL : 0) |
             (field & WBFMM_FIELD_GRADIENT ? WBFMM_B200_GRADIENT : 0);
  double *pot = NULL, *grad = NULL;
  guint i;
  int c, off;
  if (d->targets != key || d->ntargets != n || !key) {
    if (!x) die(fn, "targets are not in place");
    check(fn, wbfmm_b200_set_targets(d->s, (int)n, x, xstr, 0));
    d->targets = key;
    d->ntargets = n;
  }
  check(fn, wbfmm_b200_set_evaluation(d->s, want, neighbours));
  check(fn, wbfmm_b200_evaluate(d->s));
  if (want & WBFMM_B200_POTENTIAL) pot = malloc(sizeof(double) * n * w);
  if (want & WBFMM_B200_GRADIENT) grad = malloc(sizeof(double) * n * 3 * w);
  check(fn, wbfmm_b200_get_field(d->s, pot, grad, 0));
  /* fields added into the caller's doubles, or floats for an FP32 tree */
#define WBFMM_ADD_FIELDS(_T)                                                  \
  do {                                                                        \
    _T *f = (_T *)fv;                                                         \
    for (i = 0; i < n; i++) {                                                 \
      off = 0;                                                                \
      if (pot) {                                                              \
        for (c = 0; c < w; c++) f[(size_t)i * fstr + c] += (_T)pot[(size_t)i * w + c]; \
        off = w;                                                              \
      }                                                                       \
      if (grad)                                                               \
        for (c = 0; c < 3 * w; c++)                                           \
          f[(size_t)i * fstr + off + c] += (_T)grad[(size_t)i * 3 * w + c];   \
    }                                                                         \
  } while (0)
  if (d->fp32)
    WBFMM_ADD_FIELDS(float);
  else
    WBFMM_ADD_FIELDS(double);
#undef WBFMM_ADD_FIELDS
  free(pot);
  free(grad);
}

/* Laplace field at one point x for a multi-component tree, or a curl
   field (src/local-laplace.c:1293-1336): added into fv (doubles, or floats
   for an FP32 tree).  Potential: component c at fv[c fstr]; gradient:
   fv[c fstr + 0..2] (fstr >= 3 when nq > 1); curl (nq >= 3, the first
   three components): fv[0..2]; curl and gradient: fv[0..11], the curl then
   d/dx, d/dy, d/dz of its components (fstr ignored, as the reference) */
static void laplace_field_point(dtree_t *d, const double *x, guint field,
                                gboolean nb, void *fv, gint fstr, const char *fn) {
  const int nq = ncomp(d);
  double out[DT_MAX_NQ * 3], g[3][3], h[3][9];
  int c, j, n = 0, stride = 1;
  memset(out, 0, sizeof(out));
  if (field & WBFMM_FIELD_CURL) {
    const int cg = (field & WBFMM_FIELD_GRADIENT) != 0;
    if (nq < 3) die(fn, "not enough source components for curl calculation");
    for (c = 0; c < 3; c++) {
      wbfmm_b200_solver_t *s = comp_solver(d, c);
      check(fn, wbfmm_b200_set_targets(s, 1, x, 3, 0));
      check(fn, wbfmm_b200_set_evaluation(s, WBFMM_B200_GRADIENT, nb));
      check(fn, wbfmm_b200_evaluate(s));
      check(fn, wbfmm_b200_get_field(s, NULL, g[c], 0));
      if (cg) check(fn, wbfmm_b200_laplace_hessian(s, h[c], nb, 0));
    }
    out[0] = g[2][1] - g[1][2];
    out[1] = g[0][2] - g[2][0];
    out[2] = g[1][0] - g[0][1];
    n = 3;
    if (cg) {
      for (j = 0; j < 3; j++) {
        out[3 + 3 * j + 0] = h[2][3 * j + 1] - h[1][3 * j + 2];
        out[3 + 3 * j + 1] = h[0][3 * j + 2] - h[2][3 * j + 0];
        out[3 + 3 * j + 2] = h[1][3 * j + 0] - h[0][3 * j + 1];
      }
      n = 12;
    }
  } else {
    const int grad = (field & WBFMM_FIELD_GRADIENT) != 0;
    if (grad && nq > 1 && fstr < 3) die(fn, "field data stride must be greater than two");
    for (c = 0; c < nq; c++) {
      wbfmm_b200_solver_t *s = comp_solver(d, c);
      check(fn, wbfmm_b200_set_targets(s, 1, x, 3, 0));
      check(fn, wbfmm_b200_set_evaluation(s, grad ? WBFMM_B200_GRADIENT : WBFMM_B200_POTENTIAL, nb));
      check(fn, wbfmm_b200_evaluate(s));
      check(fn, wbfmm_b200_get_field(s, grad ? NULL : out + 3 * c, grad ? out + 3 * c : NULL, 0));
    }
    /* out[3 c + j] -> f[c fstr + j] */
    stride = fstr;
    n = -(grad ? 3 : 1);
  }
  d->targets = NULL;   /* the solvers' targets are this point now */
#define WBFMM_ADD_POINT(_T)                                                   \
  do {                                                                        \
    _T *f = (_T *)fv;                                                         \
    if (n > 0)                                                                \
      for (j = 0; j < n; j++) f[j] += (_T)out[j];                             \
    else                                                                      \
      for (c = 0; c < nq; c++)                                                \
        for (j = 0; j < -n; j++) f[(size_t)c * stride + j] += (_T)out[3 * c + j]; \
  } while (0)
  if (d->fp32)
    WBFMM_ADD_POINT(float);
  else
    WBFMM_ADD_POINT(double);
#undef WBFMM_ADD_POINT
}

/* src/local.c:264-310 */
gint wbfmm_tree_box_local_field(wbfmm_tree_t *t, guint level, guint b,
                                gdouble k, gdouble *x, gdouble *f, gint fstr,
                                gdouble *src, gint sstr, gdouble *d,
                                gint dstr, gboolean eval_neighbours,
                                guint field, gdouble *work) {
  dtree_t *dt = DT(t);
  (void)b; (void)work;
  if (t->problem != WBFMM_PROBLEM_HELMHOLTZ) die(__func__, "tree problem is not Helmholtz");
  if (level != t->depth) die(__func__, "evaluation is supported at the leaf level");
  if (field == WBFMM_FIELD_POTENTIAL && fstr < 2) die(__func__, "field stride too small");
  if (field == WBFMM_FIELD_GRADIENT && fstr < 6) die(__func__, "field stride too small for gradient");
  if (field != WBFMM_FIELD_POTENTIAL && field != WBFMM_FIELD_GRADIENT)
    die(__func__, "unrecognized field identifier");
  solver_for(t, k, __func__);
  if (eval_neighbours && (src || d)) strengths_for(dt, src, sstr, d, dstr, __func__);
  evaluate_targets(dt, NULL, 1, x, 3, field, eval_neighbours && (src || d), f,
                   fstr, __func__);
  return 0;
}

/* src/local-laplace.c:1293-1336: POTENTIAL|GRADIENT gives the gradient */
gint wbfmm_laplace_box_field(wbfmm_tree_t *t, guint level, guint b,
                             gdouble *src, gint sstr, gdouble *d, gint dstr,
                             guint field, gboolean eval_neighbours,
                             gdouble *x, gdouble *f, gint fstr,
                             gdouble *work) {
  dtree_t *dt = DT(t);
  (void)b; (void)work;
  if (t->problem != WBFMM_PROBLEM_LAPLACE) die(__func__, "tree problem is not Laplace");
  if (level != t->depth) die(__func__, "evaluation is supported at the leaf level");
  if (field < 1 || field > 7) die(__func__, "unrecognized field type");
  solver_for(t, 0.0, __func__);
  if (eval_neighbours && (src || d)) strengths_for(dt, src, sstr, d, dstr, __func__);
  if ((field & WBFMM_FIELD_CURL) || dt->nq > 1) {
    laplace_field_point(dt, x, field, eval_neighbours && (src || d), f, fstr, __func__);
    return 0;
  }
  if (field & WBFMM_FIELD_GRADIENT) field = WBFMM_FIELD_GRADIENT;
  evaluate_targets(dt, NULL, 1, x, 3, field, eval_neighbours && (src || d), f,
                   0, __func__);
  return 0;
}

/* ---------------------------------------------------- target lists */
/* src/targets.c:32-166 */
wbfmm_target_list_t *wbfmm_target_list_new(wbfmm_tree_t *t, guint npts) {
  wbfmm_target_list_t *l = calloc(1, sizeof(wbfmm_target_list_t));
  l->t = t;
  l->maxpoints = npts;
  l->size = sizeof(gdouble);
  l->complex = t->problem == WBFMM_PROBLEM_HELMHOLTZ;
  l->boxes = calloc(npts ? npts : 1, sizeof(guint32));
  return l;
}

gint wbfmm_target_list_add_points(wbfmm_target_list_t *l, gpointer pts,
                                  gsize pstr, guint npts) {
  guint i;
  if (npts > l->maxpoints) die(__func__, "too many points for target list");
  if (pstr % sizeof(double)) die(__func__, "point stride must be a multiple of sizeof(double)");
  l->points = (char *)pts;
  l->pstr = pstr;
  l->npoints = npts;
  for (i = 0; i < npts; i++)
    l->boxes[i] = (guint32)wbfmm_point_box(l->t, l->t->depth,
                                           (gdouble *)(l->points + (size_t)i * pstr));
  return 0;
}

gint wbfmm_target_list_coefficients_init(wbfmm_target_list_t *l, guint field) {
  l->field = field;
  return 0;
}

static gint list_prepare(wbfmm_target_list_t *l, double k, const char *fn) {
  dtree_t *d = DT(l->t);
  solver_for(l->t, k, fn);
  if (d->fp32) {
    double *x64 = widen3(l->points, l->pstr, l->npoints);
    check(fn, wbfmm_b200_set_targets(d->s, (int)l->npoints, x64, 3, 0));
    free(x64);
  } else {
    check(fn, wbfmm_b200_set_targets(d->s, (int)l->npoints, (const double *)l->points,
                                     (int)(l->pstr / sizeof(double)), 0));
  }
  d->targets = l;
  d->ntargets = l->npoints;
  /* the potential (the reference's only target-list field) from
     precomputed bases, as its local_coefficients prepares them */
  if (l->field == WBFMM_FIELD_POTENTIAL && d->nq <= 1)
    check(fn, wbfmm_b200_target_bases(d->s));
  return 0;
}

gint wbfmm_target_list_local_coefficients(wbfmm_target_list_t *l, gdouble k,
                                          gdouble *work) {
  (void)work;
  return list_prepare(l, k, __func__);
}

gint wbfmm_laplace_target_list_local_coefficients(wbfmm_target_list_t *l,
                                                  guint source, gdouble *work) {
  (void)work;
  l->source = source;
  return list_prepare(l, 0.0, __func__);
}

/* src/targets.c:424-603 */
static gint list_field(wbfmm_target_list_t *l, const void *src, gint sstr,
                       const void *nsrc, gint nstr, void *f, gint fstr, const char *fn) {
  dtree_t *d = DT(l->t);
  if (!l->field) die(fn, "field not set (wbfmm_target_list_coefficients_init)");
  if (l->field & (WBFMM_FIELD_CURL | WBFMM_FIELD_CURL_GRADIENT))
    die(fn, "curl fields are not supported with target lists");
  if (d->nq > 1) die(fn, "multi-component sources are not supported with target lists");
  if (!d->s || !d->ready) list_prepare(l, d->k, fn);
  if (src || nsrc) strengths_for(d, src, sstr, nsrc, nstr, fn);
  if (d->targets != l || d->ntargets != l->npoints) list_prepare(l, d->k, fn);
  if (l->field == WBFMM_FIELD_POTENTIAL) {
    const int w = l->t->problem == WBFMM_PROBLEM_HELMHOLTZ ? 2 : 1;
    double *pot = malloc(sizeof(double) * w * (l->npoints ? l->npoints : 1));
    guint i;
    int c;
    check(fn, wbfmm_b200_evaluate_bases(d->s, (src || nsrc) ? 1 : 0));
    check(fn, wbfmm_b200_get_field(d->s, pot, NULL, 0));
    for (i = 0; i < l->npoints; i++)
      for (c = 0; c < w; c++) {
        if (d->fp32) ((float *)f)[(size_t)i * fstr + c] += (float)pot[(size_t)i * w + c];
        else ((double *)f)[(size_t)i * fstr + c] += pot[(size_t)i * w + c];
      }
    free(pot);
    return 0;
  }
  /* the targets are in place (list_prepare), so no points are passed */
  evaluate_targets(d, l, l->npoints, NULL, 3, l->field, (src || nsrc), f, fstr, fn);
  return 0;
}

gint wbfmm_target_list_local_field(wbfmm_target_list_t *l, gdouble *src,
                                   gint sstr, gdouble *nsrc, gint nstr,
                                   gdouble *f, gint fstr) {
  return list_field(l, src, sstr, nsrc, nstr, f, fstr, __func__);
}

/* ------------------------------------------ single precision (*_f) */
/* The reference's single-precision API: the same sources compiled with
   WBFMM_REAL = gfloat (its libsub, src/Makefile.am), trees holding FP32
   points, origin and coefficients.  Here an FP32 tree runs the engine's
   FP32 form; its Morton keys, domain checks and target boxes are computed
   in FP32 arithmetic as the reference's build computes them, so t->ip and
   every box {i, n} are those of the reference's *_f calls.  Operator
   tables are generated in FP64 on the GPU and rounded, near-field sums
   are accumulated in FP64. */

/* src/boxes.c:58-91 */
wbfmm_tree_t *wbfmm_tree_new_f(gfloat *x, gfloat D, guint maxpoints) {
  dtree_t *d = calloc(1, sizeof(dtree_t));
  wbfmm_tree_t *t;
  float *xt;
  if (!d) die(__func__, "out of memory");
  d->fp32 = 1;
  t = &d->t;
  t->maxpoints = maxpoints;
  t->ip = malloc(sizeof(guint) * (maxpoints ? maxpoints : 1));
  t->boxes[0] = calloc(1, sizeof(wbfmm_box_t));
  t->size = sizeof(gfloat);
  xt = (float *)t->x;
  xt[0] = x[0]; xt[1] = x[1]; xt[2] = x[2];
  t->D = D;
  return t;
}

static void need_fp32(wbfmm_tree_t *t, const char *fn) {
  if (t->size != sizeof(gfloat))
    die(fn, "mixed precision not implemented (tree is not single precision)");
}

/* src/boxes.c:118-166 */
gint wbfmm_tree_add_points_f(wbfmm_tree_t *t, gpointer pts, gsize pstr,
                             gpointer normals, gsize nstr, guint npts,
                             gboolean sorted) {
  need_fp32(t, __func__);
  if (npts > t->maxpoints) die(__func__, "too many points for tree");
  if (pstr % sizeof(float) || (normals && nstr % sizeof(float)))
    die(__func__, "point and normal strides must be multiples of sizeof(float)");
  t->npoints = npts;
  t->points = (char *)pts;
  t->pstr = pstr;
  t->normals = (char *)normals;
  t->nstr = nstr;
  t->sorted = sorted;
  drop_solver(DT(t));
  refresh_boxes(t);
  t->boxes[0][0].i = 0;
  t->boxes[0][0].n = npts;
  return 0;
}

/* src/boxes.c:190-206 */
gint wbfmm_tree_sort_points_f(wbfmm_tree_t *t, gpointer pts, gsize psize, guint npts) {
  uint32_t *ip = malloc(sizeof(uint32_t) * (npts ? npts : 1));
  char *tmp = malloc(psize * (npts ? npts : 1));
  guint i;
  need_fp32(t, __func__);
  if (psize % sizeof(float)) die(__func__, "record size must be a multiple of sizeof(float)");
  check(__func__, wbfmm_b200_tree_structure_f((int)npts, (const float *)pts,
                                              (int)(psize / sizeof(float)),
                                              (const float *)t->x, (float)t->D, 0, ip,
                                              NULL, NULL));
  for (i = 0; i < npts; i++)
    memcpy(tmp + (size_t)i * psize, (char *)pts + (size_t)ip[i] * psize, psize);
  memcpy(pts, tmp, psize * npts);
  free(tmp);
  free(ip);
  return 0;
}

/* src/boxes.c:208-277 */
gint wbfmm_tree_refine_f(wbfmm_tree_t *t) {
  need_fp32(t, __func__);
  return wbfmm_tree_refine(t);
}

gint wbfmm_tree_coefficient_init_f(wbfmm_tree_t *t, guint l, guint nr, guint ns) {
  need_fp32(t, __func__);
  return wbfmm_tree_coefficient_init(t, l, nr, ns);
}
gint wbfmm_tree_laplace_coefficient_init_f(wbfmm_tree_t *t, guint l, guint nr, guint ns) {
  need_fp32(t, __func__);
  return wbfmm_tree_laplace_coefficient_init(t, l, nr, ns);
}
gint wbfmm_tree_coefficient_clear_f(wbfmm_tree_t *t, guint l) {
  return wbfmm_tree_coefficient_clear(t, l);
}

/* src/boxes.c:585-634 in FP32 arithmetic */
guint64 wbfmm_point_box_f(wbfmm_tree_t *t, guint level, gfloat *x) {
  const float *x0 = (const float *)t->x;
  const float D = (float)t->D, wb = D / (float)(1u << level);
  if (x[0] < x0[0] || x[0] > x0[0] + D || x[1] < x0[1] || x[1] > x0[1] + D ||
      x[2] < x0[2] || x[2] > x0[2] + D)
    die(__func__, "point not in octree");
  return wbfmm_box_index((guint32)floorf((x[0] - x0[0]) / wb),
                         (guint32)floorf((x[1] - x0[1]) / wb),
                         (guint32)floorf((x[2] - x0[2]) / wb));
}

/* src/boxes.c:324-339 in FP32 arithmetic */
guint64 wbfmm_point_index_3d_f(gfloat *x, gfloat *c, gfloat D) {
  return wbfmm_box_index((guint32)((x[0] - c[0]) / D * (float)WBFMM_INDEX_SHIFT),
                         (guint32)((x[1] - c[1]) / D * (float)WBFMM_INDEX_SHIFT),
                         (guint32)((x[2] - c[2]) / D * (float)WBFMM_INDEX_SHIFT));
}

/* src/util.c:290-330 */
gint wbfmm_box_location_from_index_f(guint64 idx, guint32 level, gfloat *x0,
                                     gfloat D, gfloat *x, gfloat *wb) {
  guint32 i, j, k;
  if (!(idx < ((guint64)1 << (3 * level)))) die(__func__, "box is not at this level");
  *wb = D / (float)(1u << level);
  wbfmm_box_location(idx, &i, &j, &k);
  x[0] = x0[0] + (*wb) * i;
  x[1] = x0[1] + (*wb) * j;
  x[2] = x0[2] + (*wb) * k;
  return 0;
}
gint wbfmm_tree_box_centre_f(wbfmm_tree_t *t, guint level, guint64 b, gfloat *xb,
                             gfloat *wb) {
  wbfmm_box_location_from_index_f(b, level, (gfloat *)t->x, (gfloat)t->D, xb, wb);
  xb[0] += 0.5f * (*wb); xb[1] += 0.5f * (*wb); xb[2] += 0.5f * (*wb);
  return 0;
}

/* src/util.c:375-405 */
gint wbfmm_points_origin_width_f(gfloat *x, gint str, gint n, gfloat *xmin,
                                 gfloat *xmax, gfloat *D, gboolean init_limits) {
  gint i, a;
  if (init_limits)
    for (a = 0; a < 3; a++) { xmin[a] = 3.4028234663852886e38f; xmax[a] = -3.4028234663852886e38f; }
  for (i = 0; i < n; i++)
    for (a = 0; a < 3; a++) {
      if (x[str * i + a] < xmin[a]) xmin[a] = x[str * i + a];
      if (x[str * i + a] > xmax[a]) xmax[a] = x[str * i + a];
    }
  *D = xmax[0] - xmin[0];
  if (xmax[1] - xmin[1] > *D) *D = xmax[1] - xmin[1];
  if (xmax[2] - xmin[2] > *D) *D = xmax[2] - xmin[2];
  return 0;
}

/* src/util.c:425-450 */
gint wbfmm_tree_write_sources_f(wbfmm_tree_t *t, gfloat *q, gint stride, FILE *f) {
  guint i;
  (void)q; (void)stride;
  for (i = 0; i < t->npoints; i++) {
    const guint idx = t->ip[i];
    const gfloat *x = (const gfloat *)(t->points + (gsize)idx * t->pstr);
    fprintf(f, "%u %u %g %g %g\n", i, idx, x[0], x[1], x[2]);
  }
  return 0;
}

gint wbfmm_truncation_number_f(wbfmm_tree_t *t, gfloat k, guint level, gfloat tol) {
  return wbfmm_truncation_number(t, k, level, tol);
}

/* operators: recorded orders, as the double-precision calls */
gint wbfmm_shift_angle_table_init_f(void) { return 0; }
wbfmm_shift_operators_t *wbfmm_shift_operators_new_f(guint L, gboolean bw, gfloat *work) {
  wbfmm_shift_operators_t *op = wbfmm_shift_operators_new(L, bw, NULL);
  (void)work;
  op->size = sizeof(gfloat);
  return op;
}
gint wbfmm_shift_operators_coaxial_SR_init_f(wbfmm_shift_operators_t *w, gfloat D,
                                             guint level, guint L, gfloat k, gfloat *work) {
  (void)work;
  return wbfmm_shift_operators_coaxial_SR_init(w, D, level, L, k, NULL);
}
gint wbfmm_shift_operators_coaxial_SS_init_f(wbfmm_shift_operators_t *w, gfloat D,
                                             guint level, guint L, gfloat k, gfloat *work) {
  (void)work;
  return wbfmm_shift_operators_coaxial_SS_init(w, D, level, L, k, NULL);
}
gint wbfmm_laplace_coaxial_translate_init_f(gint N) { return wbfmm_laplace_coaxial_translate_init(N); }

/* passes */
gint wbfmm_tree_leaf_expansions_f(wbfmm_tree_t *t, gfloat k, gfloat *src, gint sstr,
                                  gfloat *dipoles, gint dstr, gboolean zero_expansions,
                                  gfloat *work) {
  (void)work;
  need_fp32(t, __func__);
  if (t->problem != WBFMM_PROBLEM_HELMHOLTZ) die(__func__, "tree problem is not Helmholtz");
  return leaf(t, k, src, sstr, dipoles, dstr, zero_expansions, __func__);
}
gint wbfmm_tree_laplace_leaf_expansions_f(wbfmm_tree_t *t, gfloat *src, gint sstr,
                                          gfloat *dipoles, gint dstr,
                                          gboolean zero_expansions, gfloat *work) {
  (void)work;
  need_fp32(t, __func__);
  if (t->problem != WBFMM_PROBLEM_LAPLACE) die(__func__, "tree problem is not Laplace");
  return leaf(t, 0.0, src, sstr, dipoles, dstr, zero_expansions, __func__);
}
gint wbfmm_upward_pass_f(wbfmm_tree_t *t, wbfmm_shift_operators_t *op, guint level,
                         gfloat *work) {
  (void)op; (void)work;
  return upward(t, level, __func__);
}
gint wbfmm_laplace_upward_pass_f(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                                 guint level, gfloat *work) {
  (void)op; (void)work;
  return upward(t, level, __func__);
}
gint wbfmm_downward_pass_ref_f(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                               guint level, gfloat *work, gint nthreads) {
  (void)op; (void)work; (void)nthreads;
  return downward(t, level, __func__);
}
gint wbfmm_laplace_downward_pass_ref_f(wbfmm_tree_t *t, wbfmm_shift_operators_t *op,
                                       guint level, gfloat *work, gint nthreads) {
  (void)op; (void)work; (void)nthreads;
  return downward(t, level, __func__);
}

/* evaluation (src/local.c:264-310, src/local-laplace.c:1293-1336) */
gint wbfmm_tree_box_local_field_f(wbfmm_tree_t *t, guint level, guint b, gfloat k,
                                  gfloat *x, gfloat *f, gint fstr, gfloat *src,
                                  gint sstr, gfloat *d, gint dstr,
                                  gboolean eval_neighbours, guint field, gfloat *work) {
  dtree_t *dt = DT(t);
  double x64[3] = {x[0], x[1], x[2]};
  (void)b; (void)work;
  need_fp32(t, __func__);
  if (t->problem != WBFMM_PROBLEM_HELMHOLTZ) die(__func__, "tree problem is not Helmholtz");
  if (level != t->depth) die(__func__, "evaluation is supported at the leaf level");
  if (field == WBFMM_FIELD_POTENTIAL && fstr < 2) die(__func__, "field stride too small");
  if (field == WBFMM_FIELD_GRADIENT && fstr < 6) die(__func__, "field stride too small for gradient");
  if (field != WBFMM_FIELD_POTENTIAL && field != WBFMM_FIELD_GRADIENT)
    die(__func__, "unrecognized field identifier");
  solver_for(t, k, __func__);
  if (eval_neighbours && (src || d)) strengths_for(dt, src, sstr, d, dstr, __func__);
  evaluate_targets(dt, NULL, 1, x64, 3, field, eval_neighbours && (src || d), f, fstr,
                   __func__);
  return 0;
}
gint wbfmm_laplace_box_field_f(wbfmm_tree_t *t, guint level, guint b, gfloat *src,
                               gint sstr, gfloat *d, gint dstr, guint field,
                               gboolean eval_neighbours, gfloat *x, gfloat *f, gint fstr,
                               gfloat *work) {
  dtree_t *dt = DT(t);
  double x64[3] = {x[0], x[1], x[2]};
  (void)b; (void)work;
  need_fp32(t, __func__);
  if (t->problem != WBFMM_PROBLEM_LAPLACE) die(__func__, "tree problem is not Laplace");
  if (level != t->depth) die(__func__, "evaluation is supported at the leaf level");
  if (field < 1 || field > 7) die(__func__, "unrecognized field type");
  solver_for(t, 0.0, __func__);
  if (eval_neighbours && (src || d)) strengths_for(dt, src, sstr, d, dstr, __func__);
  if ((field & WBFMM_FIELD_CURL) || dt->nq > 1) {
    laplace_field_point(dt, x64, field, eval_neighbours && (src || d), f, fstr, __func__);
    return 0;
  }
  if (field & WBFMM_FIELD_GRADIENT) field = WBFMM_FIELD_GRADIENT;
  evaluate_targets(dt, NULL, 1, x64, 3, field, eval_neighbours && (src || d), f, 0,
                   __func__);
  return 0;
}

/* target lists (src/targets.c) */
wbfmm_target_list_t *wbfmm_target_list_new_f(wbfmm_tree_t *t, guint npts) {
  wbfmm_target_list_t *l = wbfmm_target_list_new(t, npts);
  l->size = sizeof(gfloat);
  return l;
}
gint wbfmm_target_list_add_points_f(wbfmm_target_list_t *l, gpointer pts, gsize pstr,
                                    guint npts) {
  guint i;
  if (npts > l->maxpoints) die(__func__, "too many points for target list");
  if (pstr % sizeof(float)) die(__func__, "point stride must be a multiple of sizeof(float)");
  l->points = (char *)pts;
  l->pstr = pstr;
  l->npoints = npts;
  for (i = 0; i < npts; i++)
    l->boxes[i] = (guint32)wbfmm_point_box_f(l->t, l->t->depth,
                                             (gfloat *)(l->points + (size_t)i * pstr));
  return 0;
}
gint wbfmm_target_list_local_coefficients_f(wbfmm_target_list_t *l, gfloat k, gfloat *work) {
  (void)work;
  return list_prepare(l, k, __func__);
}
gint wbfmm_laplace_target_list_local_coefficients_f(wbfmm_target_list_t *l, guint source,
                                                    gfloat *work) {
  (void)work;
  l->source = source;
  return list_prepare(l, 0.0, __func__);
}
gint wbfmm_target_list_local_field_f(wbfmm_target_list_t *l, gfloat *src, gint sstr,
                                     gfloat *nsrc, gint nstr, gfloat *f, gint fstr) {
  return list_field(l, src, sstr, nsrc, nstr, f, fstr, __func__);
}

/* ---------------------------------------------------- direct sums */
/* The reference's direct sums, one target point xf per call, evaluated on
   the GPU by wbfmm_b200_direct one source component at a time.  Semantics
   kept from src/direct.c and src/direct-laplace.c:
   * no sources, normals or dipoles: nothing is added;
   * normals without dipole strengths stop the program;
   * component j of nq is written at field[j*fstr + c];
   * Helmholtz monopoles plus dipoles: the terms are summed without the
     1/(4 pi) and the first 2*nq entries of field are then divided by 4 pi,
     including what the caller had stored there (src/direct.c:133-134);
   * Laplace monopoles plus dipoles: the dipole term has no 1/(4 pi)
     (src/direct-laplace.c:261-263).
   Where the reference stops instead (dipole-only Helmholtz potential,
   gradients of dipole fields) this library returns the field of the
   kernels the FMM uses. */
static const double kFourPi = 12.566370614359172953850573533118; /* 4 pi */

static gint direct(int problem, double k, gdouble *xs, gint xstride,
                   gdouble *src, gint sstride, gdouble *normals, gint nstr,
                   gdouble *dipoles, gint dstr, gint nq, gint nsrc,
                   gdouble *xf, gdouble *field, gint fstr, int grad,
                   const char *fn) {
  const int helm = problem == WBFMM_B200_HELMHOLTZ;
  const int w = helm ? 2 : 1, nout = grad ? 3 * w : w;
  const int mixed = src != NULL && normals != NULL;
  /* Helmholtz mixed potential: unnormalised sums, then the division */
  const int helm_mixed = helm && mixed && !grad;
  int i, c, j;
  double *x, *q, *n, *d;
  if (src == NULL && normals == NULL && dipoles == NULL) return 0;
  if (normals != NULL && dipoles == NULL)
    die(fn, "normals specified but no dipole strengths (dipoles == NULL)");
  if (nq < 1) die(fn, "nq must be positive");
  if (nq > 1 && fstr < (grad ? 3 * w : w))
    die(fn, "field stride too small for multi-component sources");
  x = malloc(sizeof(double) * 3 * nsrc);
  q = src ? malloc(sizeof(double) * w * nsrc) : NULL;
  n = normals ? malloc(sizeof(double) * 3 * nsrc) : NULL;
  d = dipoles ? malloc(sizeof(double) * w * nsrc) : NULL;
  for (i = 0; i < nsrc; i++) {
    for (c = 0; c < 3; c++) x[3 * i + c] = xs[(size_t)i * xstride + c];
    for (c = 0; c < 3 && n; c++) n[3 * i + c] = normals[(size_t)i * nstr + c];
  }
  for (j = 0; j < nq; j++) {
    double out[6] = {0, 0, 0, 0, 0, 0};
    /* the Laplace mixed sum's dipole term carries no 1/(4 pi) */
    const double dscale = (!helm && mixed) ? kFourPi : 1.0;
    for (i = 0; i < nsrc; i++)
      for (c = 0; c < w; c++) {
        if (q) q[w * i + c] = src[(size_t)i * sstride + w * j + c];
        if (d) d[w * i + c] = dscale * dipoles[(size_t)i * dstr + w * j + c];
      }
    check(fn, wbfmm_b200_direct(problem, k, nsrc, x, q, n, d, 1, xf,
                                grad ? NULL : out, grad ? out : NULL, 0));
    for (c = 0; c < nout; c++)
      field[(size_t)j * fstr + c] += helm_mixed ? kFourPi * out[c] : out[c];
  }
  if (helm_mixed)
    for (c = 0; c < 2 * nq; c++) field[c] /= kFourPi;
  free(x); free(q); free(n); free(d);
  return 0;
}

/* src/direct.c:35-160 */
gint wbfmm_total_field(gdouble k, gdouble *xs, gint xstride, gdouble *src,
                       gint sstride, gdouble *normals, gint nstr,
                       gdouble *dipoles, gint dstr, gint nq, gint nsrc,
                       gdouble *xf, gdouble *field, gint fstr) {
  return direct(WBFMM_B200_HELMHOLTZ, k, xs, xstride, src, sstride, normals,
                nstr, dipoles, dstr, nq, nsrc, xf, field, fstr, 0, __func__);
}
/* src/direct.c:162-294 */
gint wbfmm_total_field_grad(gdouble k, gdouble *xs, gint xstride, gdouble *src,
                            gint sstride, gdouble *normals, gint nstr,
                            gdouble *dipoles, gint dstr, gint nq, gint nsrc,
                            gdouble *xf, gdouble *field, gint fstr) {
  return direct(WBFMM_B200_HELMHOLTZ, k, xs, xstride, src, sstride, normals,
                nstr, dipoles, dstr, nq, nsrc, xf, field, fstr, 1, __func__);
}
/* src/direct-laplace.c:200-263 */
gint wbfmm_laplace_field(gdouble *xs, gint xstride, gdouble *src,
                         gint sstride, gint nq, gdouble *normals, gint nstr,
                         gdouble *dipoles, gint dstr, gint nsrc, gdouble *xf,
                         gdouble *field, gint fstr) {
  return direct(WBFMM_B200_LAPLACE, 0.0, xs, xstride, src, sstride, normals,
                nstr, dipoles, dstr, nq, nsrc, xf, field, fstr, 0, __func__);
}
/* src/direct-laplace.c:265-336 */
gint wbfmm_laplace_field_grad(gdouble *xs, gint xstride, gdouble *src,
                              gint sstride, gint nq, gdouble *normals,
                              gint nstr, gdouble *dipoles, gint dstr,
                              gint nsrc, gdouble *xf, gdouble *field,
                              gint fstr) {
  return direct(WBFMM_B200_LAPLACE, 0.0, xs, xstride, src, sstride, normals,
                nstr, dipoles, dstr, nq, nsrc, xf, field, fstr, 1, __func__);
}

/* The single-precision direct sums: the same semantics on FP32 arrays
   (widened exactly, summed on the GPU in FP64, rounded once into the
   caller's FP32 field). */
static double *widen_n(const float *a, size_t n) {
  double *o;
  size_t i;
  if (!a) return NULL;
  o = malloc(sizeof(double) * (n ? n : 1));
  if (!o) die("wbfmm", "out of memory");
  for (i = 0; i < n; i++) o[i] = a[i];
  return o;
}

static gint direct_f(int problem, float k, gfloat *xs, gint xstride, gfloat *src,
                     gint sstride, gfloat *normals, gint nstr, gfloat *dipoles,
                     gint dstr, gint nq, gint nsrc, gfloat *xf, gfloat *field,
                     gint fstr, int grad, const char *fn) {
  const int w = problem == WBFMM_B200_HELMHOLTZ ? 2 : 1;
  const size_t n = (size_t)(nsrc > 0 ? nsrc : 0);
  size_t nf = (size_t)(nq > 0 ? nq - 1 : 0) * (size_t)(fstr > 0 ? fstr : 0) + (grad ? 3 * w : w), i;
  /* the records' extent: (n - 1) strides plus the values of the last one */
#define WBFMM_EXTENT(_str, _cnt) (n ? (n - 1) * (size_t)(_str) + (size_t)(_cnt) : 0)
  double *x64 = widen_n(xs, WBFMM_EXTENT(xstride, 3));
  double *q64 = widen_n(src, WBFMM_EXTENT(sstride, w * nq));
  double *n64 = widen_n(normals, WBFMM_EXTENT(nstr, 3));
  double *d64 = widen_n(dipoles, WBFMM_EXTENT(dstr, w * nq));
#undef WBFMM_EXTENT
  double xf64[3] = {xf[0], xf[1], xf[2]};
  double *f64;
  if (nf < (size_t)(2 * nq)) nf = (size_t)(2 * nq);
  f64 = widen_n(field, nf);
  direct(problem, k, x64, xstride, q64, sstride, n64, nstr, d64, dstr, nq, nsrc, xf64,
         f64, fstr, grad, fn);
  for (i = 0; i < nf; i++) field[i] = (float)f64[i];
  free(x64); free(q64); free(n64); free(d64); free(f64);
  return 0;
}

gint wbfmm_total_field_f(gfloat k, gfloat *xs, gint xstride, gfloat *src, gint sstride,
                         gfloat *normals, gint nstr, gfloat *dipoles, gint dstr, gint nq,
                         gint nsrc, gfloat *xf, gfloat *field, gint fstr) {
  return direct_f(WBFMM_B200_HELMHOLTZ, k, xs, xstride, src, sstride, normals, nstr,
                  dipoles, dstr, nq, nsrc, xf, field, fstr, 0, __func__);
}
gint wbfmm_total_field_grad_f(gfloat k, gfloat *xs, gint xstride, gfloat *src,
                              gint sstride, gfloat *normals, gint nstr, gfloat *dipoles,
                              gint dstr, gint nq, gint nsrc, gfloat *xf, gfloat *field,
                              gint fstr) {
  return direct_f(WBFMM_B200_HELMHOLTZ, k, xs, xstride, src, sstride, normals, nstr,
                  dipoles, dstr, nq, nsrc, xf, field, fstr, 1, __func__);
}
gint wbfmm_laplace_field_f(gfloat *xs, gint xstride, gfloat *src, gint sstride, gint nq,
                           gfloat *normals, gint nstr, gfloat *dipoles, gint dstr,
                           gint nsrc, gfloat *xf, gfloat *field, gint fstr) {
  return direct_f(WBFMM_B200_LAPLACE, 0.0f, xs, xstride, src, sstride, normals, nstr,
                  dipoles, dstr, nq, nsrc, xf, field, fstr, 0, __func__);
}
gint wbfmm_laplace_field_grad_f(gfloat *xs, gint xstride, gfloat *src, gint sstride,
                                gint nq, gfloat *normals, gint nstr, gfloat *dipoles,
                                gint dstr, gint nsrc, gfloat *xf, gfloat *field,
                                gint fstr) {
  return direct_f(WBFMM_B200_LAPLACE, 0.0f, xs, xstride, src, sstride, normals, nstr,
                  dipoles, dstr, nq, nsrc, xf, field, fstr, 1, __func__);
}

/* ---------------------------------------------------------- config */
/* src/config.c:30-85 */
gint wbfmm_library_config(wbfmm_library_config_t *c) {
  c->avx = c->avx2 = c->fma = c->openmp = FALSE;
  c->switches = "nvcc -gencode arch=compute_100a,code=sm_100a -O3 (B200 engine)";
  c->real_size = sizeof(gdouble);
  return 0;
}

gint wbfmm_library_config_print(wbfmm_library_config_t *c, FILE *f) {
  fprintf(f,
          "AVX extensions: no\nFMA extensions: no\nOpenMP:         no\n"
          "precision:      double\ncompiler flags: %s\n"
          "device:         %d CUDA device(s)\n",
          c->switches, wbfmm_b200_device_count());
  return 0;
}
