/*
 * CPU restatement of the wbfmm reference's tree, indexing and direct-sum
 * semantics (mjcarley/wbfmm).  TEST INFRASTRUCTURE ONLY: the tests use it as
 * the checker of the GPU product (bit-exact tree/indexing, FP64 direct-sum
 * accuracy oracle); the product never links or calls it.
 *
 * Pinning: every function here is checked against the unmodified reference
 * (oracle/_ref/libwbfmm_ref.so) by tests/test_oracle.py and against the
 * committed fixtures in tests/golden/.
 *
 * Each function names the reference code it restates (paths inside the
 * reference project).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------- indexing */

/* spread the low 21 bits of v so that bit b lands at bit 3b */
static uint64_t spread3(uint64_t v)
{
  uint64_t r = 0;
  int b;
  for (b = 0; b < 21; b++) r |= ((v >> b) & 1ull) << (3 * b);
  return r;
}

static uint32_t gather3(uint64_t m)
{
  uint32_t r = 0;
  int b;
  for (b = 0; b < 21; b++) r |= (uint32_t)((m >> (3 * b)) & 1ull) << b;
  return r;
}

/* Morton interleave, x in bit 0, y in bit 1, z in bit 2
   (src/boxes.c:279-322, src/indexing.c:113-163) */
uint64_t oracle_morton_encode(uint32_t i, uint32_t j, uint32_t k)
{
  return spread3(i) | (spread3(j) << 1) | (spread3(k) << 2);
}

void oracle_morton_decode(uint64_t m, uint32_t *i, uint32_t *j, uint32_t *k)
{
  *i = gather3(m);
  *j = gather3(m >> 1);
  *k = gather3(m >> 2);
}

/* point key: 20-bit truncation of (x-c)/D per axis (src/boxes.c:324-339);
   the division happens before the scaling, as in the reference */
uint64_t oracle_point_index_3d(const double *x, const double *c, double D)
{
  uint32_t xi = (uint32_t)((x[0] - c[0]) / D * (double)(1u << 20));
  uint32_t yi = (uint32_t)((x[1] - c[1]) / D * (double)(1u << 20));
  uint32_t zi = (uint32_t)((x[2] - c[2]) / D * (double)(1u << 20));
  return oracle_morton_encode(xi, yi, zi);
}

/* target box at a level: floor((x-x0)/wb) with wb = D/2^level
   (src/boxes.c:585-634); returns ~0 when x is outside the closed cube */
uint64_t oracle_point_box(const double *x0, double D, unsigned level,
                          const double *x)
{
  double wb;
  uint32_t i, j, k;
  if (x[0] < x0[0] || x[0] > x0[0] + D || x[1] < x0[1] ||
      x[1] > x0[1] + D || x[2] < x0[2] || x[2] > x0[2] + D)
    return ~0ull;
  wb = D / (double)(1u << level);
  i = (uint32_t)floor((x[0] - x0[0]) / wb);
  j = (uint32_t)floor((x[1] - x0[1]) / wb);
  k = (uint32_t)floor((x[2] - x0[2]) / wb);
  return oracle_morton_encode(i, j, k);
}

/* ------------------------------------------------------------------- tree */

static const uint64_t *g_sort_keys;

/* stable LSD radix sort of indices by 64-bit key (16-bit digits) */
static void stable_sort_by_key(uint32_t *idx, const uint64_t *key, size_t n)
{
  uint32_t *tmp = malloc(n * sizeof(uint32_t));
  size_t cnt[65536];
  int pass;
  size_t i;
  for (pass = 0; pass < 4; pass++) {
    int sh = 16 * pass;
    size_t s = 0;
    memset(cnt, 0, sizeof(cnt));
    for (i = 0; i < n; i++) cnt[(key[idx[i]] >> sh) & 0xffff]++;
    for (i = 0; i < 65536; i++) {
      size_t c = cnt[i];
      cnt[i] = s;
      s += c;
    }
    for (i = 0; i < n; i++) tmp[cnt[(key[idx[i]] >> sh) & 0xffff]++] = idx[i];
    memcpy(idx, tmp, n * sizeof(uint32_t));
  }
  free(tmp);
  (void)g_sort_keys;
}

/*
 * Tree build: domain check, stable Morton sort of the point permutation
 * (src/boxes.c:118-166) and `depth` refinements (src/boxes.c:208-277),
 * reproducing the reference's box {i, n} values exactly, including its
 * side effects: a refined parent's .i ends at its end offset, and children
 * that are never visited keep .i = 0.
 *
 * pts: npts points with stride pstr doubles.  ip_out[npts];
 * boxes_out[2*sum_{l=0..depth} 8^l] as {i, n} pairs, levels concatenated.
 * Returns 0, or -1 (index of the failing point in *bad) when a point is not
 * strictly inside the cube.
 */
int oracle_tree_build(const double *x0, double D, int depth, int npts,
                      const double *pts, int pstr, uint32_t *ip_out,
                      uint32_t *boxes_out, int *bad)
{
  uint64_t *key = malloc((size_t)(npts ? npts : 1) * sizeof(uint64_t));
  size_t off_p, off_c;
  int i, level;
  for (i = 0; i < npts; i++) {
    const double *x = &pts[(size_t)i * pstr];
    if (x[0] <= x0[0] || x[0] >= x0[0] + D || x[1] <= x0[1] ||
        x[1] >= x0[1] + D || x[2] <= x0[2] || x[2] >= x0[2] + D) {
      if (bad) *bad = i;
      free(key);
      return -1;
    }
    key[i] = oracle_point_index_3d(x, x0, D);
    ip_out[i] = (uint32_t)i;
  }
  stable_sort_by_key(ip_out, key, (size_t)npts);

  boxes_out[0] = 0;
  boxes_out[1] = (uint32_t)npts;
  off_p = 0;
  for (level = 0; level < depth; level++) {
    size_t np = (size_t)1 << (3 * level), nc = np * 8, b;
    uint32_t *par, *chi;
    off_c = off_p + np;
    par = &boxes_out[2 * off_p];
    chi = &boxes_out[2 * off_c];
    memset(chi, 0, 2 * nc * sizeof(uint32_t));
    for (b = 0; b < np; b++) {
      uint64_t child = 8 * b;
      uint32_t j = par[2 * b + 0], n = par[2 * b + 1];
      chi[2 * child + 0] = par[2 * b + 0];
      chi[2 * child + 1] = 0;
      while (n != 0) {
        uint64_t box = key[ip_out[j]] >> (3 * (20 - (level + 1)));
        if (box == child) {
          n--;
          par[2 * b + 0]++;
          chi[2 * child + 1]++;
          j++;
        } else {
          child++;
          chi[2 * child + 1] = 0;
          chi[2 * child + 0] = par[2 * b + 0];
        }
      }
    }
    off_p = off_c;
  }
  free(key);
  return 0;
}

/* clipped 3x3x3 neighbourhood, in the reference's loop order
   (src/indexing.c:250-286) */
int oracle_box_neighbours(unsigned level, uint64_t idx, uint64_t *nb)
{
  uint32_t i, j, k, i0, i1, j0, j1, k0, k1, a, b, c, nbox = 1u << level;
  int n = 0;
  oracle_morton_decode(idx, &i, &j, &k);
  i0 = i > 0 ? i - 1 : 0; j0 = j > 0 ? j - 1 : 0; k0 = k > 0 ? k - 1 : 0;
  i1 = i + 1 < nbox ? i + 1 : nbox - 1;
  j1 = j + 1 < nbox ? j + 1 : nbox - 1;
  k1 = k + 1 < nbox ? k + 1 : nbox - 1;
  for (a = i0; a <= i1; a++)
    for (b = j0; b <= j1; b++)
      for (c = k0; c <= k1; c++) nb[n++] = oracle_morton_encode(a, b, c);
  return n;
}

/* list 4: children of the parent's neighbours that are not neighbours of
   the box, with shift index (dx+3)*49+(dy+3)*7+dz+3 (src/indexing.c:330-377);
   unsorted, in the reference's enumeration order */
int oracle_interaction_list_4(unsigned level, uint64_t idx, uint64_t *list)
{
  uint32_t i, j, k, a, b, c, nbox = 1u << level;
  int i0, i1, j0, j1, k0, k1, n = 0;
  oracle_morton_decode(idx, &i, &j, &k);
  i0 = (int)(i - i % 2); j0 = (int)(j - j % 2); k0 = (int)(k - k % 2);
  i1 = i0 + 3 < (int)nbox - 1 ? i0 + 3 : (int)nbox - 1;
  j1 = j0 + 3 < (int)nbox - 1 ? j0 + 3 : (int)nbox - 1;
  k1 = k0 + 3 < (int)nbox - 1 ? k0 + 3 : (int)nbox - 1;
  if (i0 > 0) i0 -= 2;
  if (j0 > 0) j0 -= 2;
  if (k0 > 0) k0 -= 2;
  for (a = (uint32_t)i0; (int)a <= i1; a++)
    for (b = (uint32_t)j0; (int)b <= j1; b++)
      for (c = (uint32_t)k0; (int)c <= k1; c++) {
        int dx = (int)a - (int)i, dy = (int)b - (int)j, dz = (int)c - (int)k;
        if (abs(dx) <= 1 && abs(dy) <= 1 && abs(dz) <= 1) continue;
        list[2 * n + 0] = oracle_morton_encode(a, b, c);
        list[2 * n + 1] = (uint64_t)((dx + 3) * 49 + (dy + 3) * 7 + dz + 3);
        n++;
      }
  return n;
}

/* ------------------------------------------------------------ direct sums */

/*
 * FP64 direct sums with explicit self-exclusion (pairs with r <= 1e-6, the
 * reference's near-field cutoff WBFMM_LOCAL_CUTOFF_RADIUS, src/wbfmm.h:36,
 * are skipped).  Kernels:
 *   Laplace   G = 1/(4 pi r)                     (src/direct-laplace.c:200-336)
 *   Helmholtz G = h0(kr)/(4 pi) = e^{ikr}/(4 pi i k r)   (src/direct.c:35-294)
 * Dipoles: strength d along the source normal n, field d n.grad_s G
 * (src/local.c:117-148 for Helmholtz, src/local-laplace.c:482-506 for
 * Laplace).  Outputs: Laplace pot[nt], grad[3nt]; Helmholtz pot[2nt],
 * grad[6nt] (re,im interleaved per component).  Sums are accumulated with
 * Neumaier compensation so the oracle is accurate beyond FP64 rounding of a
 * naive loop.  q / normals / dipoles may be NULL.
 */
typedef struct {
  int problem, ns, t0, t1, want_pot, want_grad;
  double k;
  const double *xs, *q, *nrm, *dip, *xt;
  double *pot, *grad;
} direct_job_t;

typedef struct { double s, c; } ksum_t;

static inline void kadd(ksum_t *a, double v)
{
  double t = a->s + v;
  if (fabs(a->s) >= fabs(v)) a->c += (a->s - t) + v;
  else a->c += (v - t) + a->s;
  a->s = t;
}

static void *direct_worker(void *p)
{
  direct_job_t *J = p;
  const double rc2 = 1e-6 * 1e-6, f4pi = 0.25 / M_PI;
  int t, s, c;
  for (t = J->t0; t < J->t1; t++) {
    const double *x = &J->xt[3 * (size_t)t];
    ksum_t acc[8];
    memset(acc, 0, sizeof(acc));
    for (s = 0; s < J->ns; s++) {
      const double *y = &J->xs[3 * (size_t)s];
      double rx = x[0] - y[0], ry = x[1] - y[1], rz = x[2] - y[2];
      double r2 = rx * rx + ry * ry + rz * rz, r;
      if (r2 <= rc2) continue;
      r = sqrt(r2);
      if (J->problem == 1) {
        double q = J->q ? J->q[s] : 0.0, g = f4pi / r;
        double dn = 0.0;
        if (J->dip) {
          const double *n = &J->nrm[3 * (size_t)s];
          dn = J->dip[s] * (rx * n[0] + ry * n[1] + rz * n[2]) / r2;
        }
        if (J->want_pot) kadd(&acc[0], (q + dn) * g);
        if (J->want_grad) {
          /* grad_x of q/(4 pi r): -q r_vec/(4 pi r^3) */
          double gq = -q * g / r2;
          double gd[3] = {0.0, 0.0, 0.0};
          if (J->dip) {
            /* grad_x of d (n.r)/(4 pi r^3) = d (n - 3 (n.r) r/r^2)/(4 pi r^3) */
            const double *n = &J->nrm[3 * (size_t)s];
            double nr = rx * n[0] + ry * n[1] + rz * n[2];
            double a = J->dip[s] * g / r2;
            gd[0] = a * (n[0] - 3.0 * nr * rx / r2);
            gd[1] = a * (n[1] - 3.0 * nr * ry / r2);
            gd[2] = a * (n[2] - 3.0 * nr * rz / r2);
          }
          kadd(&acc[1], gq * rx + gd[0]);
          kadd(&acc[2], gq * ry + gd[1]);
          kadd(&acc[3], gq * rz + gd[2]);
        }
      } else {
        double kr = J->k * r, sn = sin(kr), cs = cos(kr);
        /* h0 = (sin x - i cos x)/x ; h1 = h0/x + (-cos x/x - i ... ) */
        double h0r = sn / kr, h0i = -cs / kr;
        double h1r = h0r / kr + h0i, h1i = h0i / kr - h0r;
        double qr = J->q ? J->q[2 * (size_t)s] : 0.0;
        double qi = J->q ? J->q[2 * (size_t)s + 1] : 0.0;
        if (J->want_pot) {
          double fr = (h0r * qr - h0i * qi) * f4pi;
          double fi = (h0i * qr + h0r * qi) * f4pi;
          if (J->dip) {
            const double *n = &J->nrm[3 * (size_t)s];
            double nr = (rx * n[0] + ry * n[1] + rz * n[2]) / r;
            double dr = J->dip[2 * (size_t)s] * nr;
            double di = J->dip[2 * (size_t)s + 1] * nr;
            fr -= J->k * (h1r * dr - h1i * di) * f4pi;
            fi -= J->k * (h1r * di + h1i * dr) * f4pi;
          }
          kadd(&acc[0], fr);
          kadd(&acc[1], fi);
        }
        if (J->want_grad) {
          /* grad_x h0(k r) = -k h1(k r) r_vec/r */
          double ar = -J->k * (h1r * qr - h1i * qi) * f4pi / r;
          double ai = -J->k * (h1r * qi + h1i * qr) * f4pi / r;
          double comp[3] = {rx, ry, rz};
          if (J->dip) {
            /* d * grad_x [ -k h1(kr) (n.r)/r ]:
               = -k d [ h1'(kr) k (n.r) r_vec/r^2 + h1(kr) (n/r - (n.r) r_vec/r^3) ]
               with h1'(x) = h0(x) - 2 h1(x)/x */
            const double *n = &J->nrm[3 * (size_t)s];
            double nr = rx * n[0] + ry * n[1] + rz * n[2];
            double dpr = h0r - 2.0 * h1r / kr, dpi = h0i - 2.0 * h1i / kr;
            double dr = J->dip[2 * (size_t)s], di = J->dip[2 * (size_t)s + 1];
            for (c = 0; c < 3; c++) {
              double ur = dpr * J->k * nr * comp[c] / r2 +
                          h1r * (n[c] / r - nr * comp[c] / (r2 * r));
              double ui = dpi * J->k * nr * comp[c] / r2 +
                          h1i * (n[c] / r - nr * comp[c] / (r2 * r));
              double vr = -J->k * (ur * dr - ui * di) * f4pi;
              double vi = -J->k * (ur * di + ui * dr) * f4pi;
              kadd(&acc[2 + 2 * c], vr);
              kadd(&acc[3 + 2 * c], vi);
            }
          }
          for (c = 0; c < 3; c++) {
            kadd(&acc[2 + 2 * c], ar * comp[c]);
            kadd(&acc[3 + 2 * c], ai * comp[c]);
          }
        }
      }
    }
    if (J->problem == 1) {
      if (J->want_pot) J->pot[t] = acc[0].s + acc[0].c;
      if (J->want_grad)
        for (c = 0; c < 3; c++) J->grad[3 * (size_t)t + c] = acc[1 + c].s + acc[1 + c].c;
    } else {
      if (J->want_pot) {
        J->pot[2 * (size_t)t] = acc[0].s + acc[0].c;
        J->pot[2 * (size_t)t + 1] = acc[1].s + acc[1].c;
      }
      if (J->want_grad)
        for (c = 0; c < 6; c++) J->grad[6 * (size_t)t + c] = acc[2 + c].s + acc[2 + c].c;
    }
  }
  return NULL;
}

int oracle_direct(int problem, double k, int ns, const double *xs,
                  const double *q, const double *normals,
                  const double *dipoles, int nt, const double *xt,
                  double *pot, double *grad, int nthreads)
{
  pthread_t th[256];
  direct_job_t jobs[256];
  int i, chunk;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  chunk = (nt + nthreads - 1) / nthreads;
  for (i = 0; i < nthreads; i++) {
    direct_job_t *J = &jobs[i];
    J->problem = problem; J->k = k; J->ns = ns; J->xs = xs; J->q = q;
    J->nrm = normals; J->dip = dipoles; J->xt = xt; J->pot = pot;
    J->grad = grad; J->want_pot = pot != NULL; J->want_grad = grad != NULL;
    J->t0 = i * chunk;
    J->t1 = (i + 1) * chunk < nt ? (i + 1) * chunk : nt;
    if (J->t0 > J->t1) J->t0 = J->t1;
    pthread_create(&th[i], NULL, direct_worker, J);
  }
  for (i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
  return 0;
}
