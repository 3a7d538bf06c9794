/*
 * A wbfmm client program written only against the wbfmm.h API, in the call
 * order of the reference's own drivers:
 *
 *   Helmholtz: tools/wbfmm-tree-calc.c.in:262-414
 *   Laplace:   tools/wbfmm-laplace-tree-calc.c.in:336-460
 *
 * The same source compiles against the B200 drop-in header (include/wbfmm.h,
 * linked with libwbfmm_b200.so) and against the reference's own header and
 * sources (the test oracle's build), so a test can run one client over both
 * libraries and compare what the client sees: the fields, t->ip, every box's
 * {i, n}, and the coefficient arrays behind t->mps / t->mpr.
 *
 * Usage: driver <input> <output>
 *
 * Input (native endianness): int32 header[10] = {problem, depth, nsrc, ntgt,
 * has_q, has_normals, has_dipoles, mode, field, bw}; float64 k, x0[3], D;
 * int32 order_s[depth + 1], order_r[depth + 1]; float64 xs[3 nsrc],
 * q[w nsrc] (if has_q), normals[3 nsrc] (if has_normals), dipoles[w nsrc]
 * (if has_dipoles), xt[3 ntgt].  w = 2 (Helmholtz) or 1 (Laplace).
 * mode 0 evaluates target by target (wbfmm_tree_box_local_field /
 * wbfmm_laplace_box_field), mode 1 through a target list.
 *
 * Output: float64 f[ntgt * nf] (nf = w for the potential, 3w for the
 * gradient), uint32 ip[nsrc], uint32 {i, n} of every box of levels
 * 0..depth, then float64 mps[l] and mpr[l] for l = 1..depth.
 *
 * Exit status 0, or 2 when a box's coefficient pointers are not where the
 * Layout L formula puts them.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#if defined(__has_include)
#if __has_include(<glib.h>)
#include <glib.h>
#endif
#endif
#include <wbfmm.h>

static void *slurp(FILE *f, size_t bytes) {
  void *p = malloc(bytes ? bytes : 1);
  if (bytes && fread(p, 1, bytes, f) != bytes) {
    fprintf(stderr, "driver: short input\n");
    exit(1);
  }
  return p;
}

int main(int argc, char **argv) {
  FILE *in, *out;
  gint hdr[10], problem, depth, nsrc, ntgt, mode, w, nf, i, l, bw;
  guint field, source = 0;
  gdouble k, x0[3], D, *xs, *q = NULL, *nrm = NULL, *dip = NULL, *xt, *f;
  gdouble *work;
  gint *order_s, *order_r, order_max = 0, sizew;
  wbfmm_tree_t *tree;
  wbfmm_shift_operators_t *shifts;
  wbfmm_target_list_t *targets = NULL;
  gint bad = 0;

  if (argc != 3) {
    fprintf(stderr, "usage: %s input output\n", argv[0]);
    return 1;
  }
  in = fopen(argv[1], "rb");
  if (!in) return 1;
  memcpy(hdr, slurp(in, sizeof(hdr)), sizeof(hdr));
  problem = hdr[0]; depth = hdr[1]; nsrc = hdr[2]; ntgt = hdr[3];
  mode = hdr[7]; field = (guint)hdr[8]; bw = hdr[9];
  w = problem == WBFMM_PROBLEM_HELMHOLTZ ? 2 : 1;
  k = *(gdouble *)slurp(in, sizeof(gdouble));
  memcpy(x0, slurp(in, 3 * sizeof(gdouble)), sizeof(x0));
  D = *(gdouble *)slurp(in, sizeof(gdouble));
  order_s = slurp(in, sizeof(gint) * (depth + 1));
  order_r = slurp(in, sizeof(gint) * (depth + 1));
  xs = slurp(in, sizeof(gdouble) * 3 * nsrc);
  if (hdr[4]) q = slurp(in, sizeof(gdouble) * w * nsrc);
  if (hdr[5]) nrm = slurp(in, sizeof(gdouble) * 3 * nsrc);
  if (hdr[6]) dip = slurp(in, sizeof(gdouble) * w * nsrc);
  xt = slurp(in, sizeof(gdouble) * 3 * ntgt);
  fclose(in);

  nf = field & WBFMM_FIELD_GRADIENT ? 3 * w : w;
  f = calloc((size_t)ntgt * nf, sizeof(gdouble));
  for (l = 1; l <= depth; l++) {
    if (order_s[l] > order_max) order_max = order_s[l];
    if (order_r[l] > order_max) order_max = order_r[l];
  }
  sizew = wbfmm_element_number_rotation(2 * order_max);
  if (problem == WBFMM_PROBLEM_HELMHOLTZ) {
    if (64 * wbfmm_coefficient_index_nm(order_max + 1, 0) > sizew)
      sizew = 64 * wbfmm_coefficient_index_nm(order_max + 1, 0);
  } else {
    if ((order_max + 1) * (order_max + 1) * 16 > sizew)
      sizew = (order_max + 1) * (order_max + 1) * 16;
    sizew *= 2;
  }
  /* one spare block beyond the drivers' nthreads * sizew, as the oracle's
     harness allocates */
  work = calloc((size_t)2 * sizew, sizeof(gdouble));

  tree = wbfmm_tree_new(x0, D, 2 * nsrc);
  wbfmm_tree_source_size(tree) = 1;
  wbfmm_shift_angle_table_init();
  shifts = wbfmm_shift_operators_new(order_max, bw, work);
  if (problem == WBFMM_PROBLEM_HELMHOLTZ) {
    for (l = 1; l <= depth; l++)
      wbfmm_shift_operators_coaxial_SR_init(shifts, D, l, order_s[l], k, work);
    for (l = 2; l <= depth; l++)
      wbfmm_shift_operators_coaxial_SS_init(shifts, D, l, order_s[l - 1], k, work);
  } else {
    wbfmm_laplace_coaxial_translate_init(order_max + 2);
  }

  wbfmm_tree_add_points(tree, xs, 3 * sizeof(gdouble), nrm,
                        3 * sizeof(gdouble), nsrc, FALSE);
  for (l = 0; l < depth; l++) wbfmm_tree_refine(tree);

  wbfmm_tree_problem(tree) = problem;
  for (l = 1; l <= depth; l++) {
    if (problem == WBFMM_PROBLEM_HELMHOLTZ)
      wbfmm_tree_coefficient_init(tree, l, order_r[l], order_s[l]);
    else
      wbfmm_tree_laplace_coefficient_init(tree, l, order_r[l], order_s[l]);
    wbfmm_tree_coefficient_clear(tree, l);
  }

  if (mode == 1) {
    targets = wbfmm_target_list_new(tree, ntgt);
    if (problem == WBFMM_PROBLEM_HELMHOLTZ) {
      wbfmm_target_list_coefficients_init(targets, field);
      wbfmm_target_list_add_points(targets, xt, 3 * sizeof(gdouble), ntgt);
      wbfmm_target_list_local_coefficients(targets, k, work);
    } else {
      if (q) source |= WBFMM_SOURCE_MONOPOLE;
      if (nrm) source |= WBFMM_SOURCE_DIPOLE;
      wbfmm_target_list_add_points(targets, xt, 3 * sizeof(gdouble), ntgt);
      wbfmm_target_list_coefficients_init(targets, field);
      wbfmm_laplace_target_list_local_coefficients(targets, source, work);
    }
  }

  if (problem == WBFMM_PROBLEM_HELMHOLTZ)
    wbfmm_tree_leaf_expansions(tree, k, q, w, dip, w, TRUE, work);
  else
    wbfmm_tree_laplace_leaf_expansions(tree, q, w, dip, w, TRUE, work);
  for (l = depth; l >= 3; l--) {
    if (problem == WBFMM_PROBLEM_HELMHOLTZ)
      wbfmm_upward_pass(tree, shifts, l, work);
    else
      wbfmm_laplace_upward_pass(tree, shifts, l, work);
  }
  for (l = 2; l <= depth; l++) {
    if (problem == WBFMM_PROBLEM_HELMHOLTZ)
      wbfmm_downward_pass(tree, shifts, l, work, 1);
    else
      wbfmm_laplace_downward_pass(tree, shifts, l, work, 1);
  }

  if (mode == 1) {
    wbfmm_target_list_local_field(targets, q, w, dip, w, f, nf);
  } else {
    for (i = 0; i < ntgt; i++) {
      guint64 b = wbfmm_point_box(tree, tree->depth, &xt[3 * i]);
      if (problem == WBFMM_PROBLEM_HELMHOLTZ)
        wbfmm_tree_box_local_field(tree, tree->depth, b, k, &xt[3 * i],
                                   &f[(size_t)nf * i], nf, q, w, dip, w, TRUE,
                                   field, work);
      else
        wbfmm_laplace_box_field(tree, tree->depth, b, q, 1, dip, 1, field,
                                TRUE, &xt[3 * i], &f[(size_t)nf * i], nf, work);
    }
  }

  out = fopen(argv[2], "wb");
  if (!out) return 1;
  fwrite(f, sizeof(gdouble), (size_t)ntgt * nf, out);
  fwrite(tree->ip, sizeof(guint), nsrc, out);
  for (l = 0; l <= depth; l++) {
    wbfmm_box_t *boxes = wbfmm_tree_boxes_level(tree, l);
    guint64 b, nb = (guint64)1 << (3 * l);
    for (b = 0; b < nb; b++) {
      guint32 in2[2] = {boxes[b].i, boxes[b].n};
      fwrite(in2, sizeof(guint32), 2, out);
    }
  }
  for (l = 1; l <= depth; l++) {
    wbfmm_box_t *boxes = wbfmm_tree_boxes_level(tree, l);
    guint64 b, nb = (guint64)1 << (3 * l);
    size_t ns = (size_t)(order_s[l] + 1) * (order_s[l] + 1);
    size_t nr = (size_t)(order_r[l] + 1) * (order_r[l] + 1);
    for (b = 0; b < nb; b++) {
      /* Layout L: [group of 8 boxes][coefficient][box in group] */
      size_t os = ((b & ~(guint64)7) * ns + (b & 7)) * w;
      size_t orr = ((b & ~(guint64)7) * nr + (b & 7)) * w;
      if ((gdouble *)boxes[b].mps != (gdouble *)tree->mps[l] + os ||
          (gdouble *)boxes[b].mpr != (gdouble *)tree->mpr[l] + orr)
        bad = 1;
    }
    fwrite(tree->mps[l], sizeof(gdouble), nb * ns * w, out);
    fwrite(tree->mpr[l], sizeof(gdouble), nb * nr * w, out);
  }
  fclose(out);
  if (bad) fprintf(stderr, "driver: box coefficient pointers off Layout L\n");
  return bad ? 2 : 0;
}
