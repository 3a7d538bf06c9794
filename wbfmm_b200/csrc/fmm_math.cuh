// Special functions, expansion and translation primitives of the octree FMM,
// written once as __host__ __device__ code and used by every kernel.
//
// Conventions follow the wbfmm reference (mjcarley/wbfmm) exactly, because
// the drop-in keeps its coefficient layout and must reproduce its numbers:
//  * normalised associated Legendre functions with the Gumerov-Duraiswami
//    normalisation, P(n,m) includes 1/sqrt(4 pi), no Condon-Shortley phase
//    (src/util.c:58-113);
//  * Helmholtz coefficients are complex, index n(n+1)+m, m in [-n,n]
//    (src/wbfmm.h:242);
//  * Laplace coefficients are real-packed: n^2 for m = 0, n^2+2m-1 / n^2+2m
//    for (re, im) of m > 0, negative m implied by conjugate symmetry
//    (src/wbfmm-private.h:76);
//  * rotation coefficients H_n^{nu,m}(theta) stored at
//    n(4n-1)(n+1)/6 + (nu+n)(n+1) + m, m >= 0, with H^{nu,-m} = H^{-nu,m}
//    (src/wbfmm-private.h:73-74);
//  * coaxial coefficients (E|F)_{l,n}^m stored at l(l+1)(l+2)/6+n(n+1)/2+m for
//    l >= n >= m >= 0, sign (-1)^{n+l} when the first index is the smaller
//    (src/wbfmm-private.h:149-157).
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define HD __host__ __device__ __forceinline__
#else
#define HD inline
#endif

namespace wbfmm {

constexpr double kPi = 3.14159265358979323846;
constexpr double kCutoffRadius = 1e-6;   // src/wbfmm.h:36

// ------------------------------------------------------------- indexing
HD int cidx(int n, int m) { return n * (n + 1) + m; }
HD int lidx(int n, int m) { return n * n + 2 * m - 1; }       // m >= 1 (re)
HD int ncoef(int p) { return (p + 1) * (p + 1); }
HD int rot_idx(int nu, int m, int n) {
  return n * (4 * n - 1) * (n + 1) / 6 + (nu + n) * (n + 1) + m;
}
HD int rot_count(int N) { return rot_idx(N + 1, 0, N + 1); }  // entries n<=N
HD int coax_idx(int l, int m, int n) {
  return l * (l + 1) * (l + 2) / 6 + n * (n + 1) / 2 + m;
}
HD int coax_count(int L) {    // wbfmm_element_number_coaxial (src/wbfmm.h:231)
  return (L + 1) * (L + 2) * (L + 3) / 6 + (L + 1) * (L + 2) / 2 + L + 1;
}

// Layout L: coefficient c of box b in a level array, nq = 1, in units of
// one coefficient (complex for Helmholtz, real for Laplace); boxes are packed
// in groups of eight (src/boxes.c:545-583, src/laplace.c:819-849).
HD int64_t layout_off(int64_t b, int c, int nc) {
  return ((b >> 3) * (int64_t)nc + c) * 8 + (b & 7);
}

// Sparse level storage keeps only the groups of eight boxes whose parent
// holds sources or targets, each group still in Layout L, at consecutive
// slots in Morton order; gmap[group] is the group's slot, kNoGroup for a
// group not stored.  The compact index of box b is 8 slot + (b & 7) (-1
// when its group is not stored; dense storage, gmap null: b), and
// layout_off of the compact index addresses its coefficients.
constexpr uint32_t kNoGroup = 0xffffffffu;
HD int64_t compact_box(const uint32_t* gmap, int64_t b) {
  if (!gmap) return b;
  const uint32_t g = gmap[b >> 3];
  return g == kNoGroup ? -1 : (((int64_t)g << 3) | (b & 7));
}

// Morton interleave, x in bit 0 (src/boxes.c:279-322)
HD uint64_t spread3(uint64_t v) {
  v &= 0x1fffffull;
  v = (v | (v << 32)) & 0x1f00000000ffffull;
  v = (v | (v << 16)) & 0x1f0000ff0000ffull;
  v = (v | (v << 8)) & 0x100f00f00f00f00full;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
  v = (v | (v << 2)) & 0x1249249249249249ull;
  return v;
}
HD uint32_t compact3(uint64_t v) {
  v &= 0x1249249249249249ull;
  v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ull;
  v = (v ^ (v >> 4)) & 0x100f00f00f00f00full;
  v = (v ^ (v >> 8)) & 0x1f0000ff0000ffull;
  v = (v ^ (v >> 16)) & 0x1f00000000ffffull;
  v = (v ^ (v >> 32)) & 0x1fffffull;
  return (uint32_t)v;
}
HD uint64_t morton(uint32_t i, uint32_t j, uint32_t k) {
  return spread3(i) | (spread3(j) << 1) | (spread3(k) << 2);
}
HD void demorton(uint64_t m, uint32_t* i, uint32_t* j, uint32_t* k) {
  *i = compact3(m); *j = compact3(m >> 1); *k = compact3(m >> 2);
}

// ------------------------------------------------------ recursion weights
// a_n^m and b_n^m of the Gumerov-Duraiswami recursions
// (src/translations.c:182-204)
template <typename T>
HD T rec_a(int n, int m) {
  m = m < 0 ? -m : m;
  if (n < m) return T(0);
  return sqrt((T)((n + 1 + m) * (n + 1 - m)) / (T)(2 * n + 1) / (T)(2 * n + 3));
}
template <typename T>
HD T rec_b(int n, int m) {
  int am = m < 0 ? -m : m;
  if (n < am) return T(0);
  T v = sqrt((T)((n - m - 1) * (n - m)) / (T)(2 * n - 1) / (T)(2 * n + 1));
  return m >= 0 ? v : -v;
}

// the recursion constants rec_a / rec_b as computed on the fly; L2P kernels
// pass table-backed equivalents
template <typename T>
struct RecDirect {
  HD T a(int n, int m) const { return rec_a<T>(n, m); }
  HD T b(int n, int m) const { return rec_b<T>(n, m); }
};

// the constants of the Laplace solid-harmonic derivatives at (n, m >= 0):
// f = (2n+1)/(2n-1); m = 0: a0 = sqrt(f n n), a1 = sqrt(f n (n-1));
// m > 0: am = sqrt(f (n+m)(n+m-1)), a0 = sqrt(f (n-m)(n+m)),
// ap = sqrt(f (n-m)(n-m-1))
template <typename T>
struct LapRecDirect {
  HD void c(int n, int m, T* am, T* a0, T* ap) const {
    const T f = (T)(2 * n + 1) / (T)(2 * n - 1);
    if (m == 0) {
      *am = T(0);
      *a0 = sqrt(f * (T)n * (T)n);
      *ap = sqrt(f * (T)n * (T)(n - 1));
    } else {
      *am = sqrt(f * (T)(n + m) * (T)(n + m - 1));
      *a0 = sqrt(f * (T)(n - m) * (T)(n + m));
      *ap = sqrt(f * (T)(n - m) * (T)(n - m - 1));
    }
  }
};

// ------------------------------------------------------------- geometry
// r, theta, phi of x relative to x0 (src/util.c:30-49)
template <typename T>
HD void cart2sph(const T* x0, const T* x, T* r, T* th, T* ph) {
  T dx = x[0] - x0[0], dy = x[1] - x0[1], dz = x[2] - x0[2];
  T rr = dx * dx + dy * dy + dz * dz;
  if (rr == T(0)) { *r = *th = *ph = T(0); return; }
  rr = sqrt(rr);
  *r = rr;
  *ph = atan2(dy, dx);
  *th = acos(dz / rr);
}

// Normalised Legendre functions: init degree 0 and 1 (src/util.c:97-116)
template <typename T>
HD void legendre_init(T C, T S, T* P0, T* P10, T* P11) {
  const T s4pi = (T)sqrt(4.0 * kPi);
  *P0 = T(1) / s4pi;
  *P10 = C * (T)sqrt(3.0) / s4pi;
  *P11 = S * (T)sqrt(1.5) / s4pi;
}
// The constants of one step of the normalised Legendre recursion from
// degree n: d(n) = sqrt((2n+3)/(2n+2)) (new diagonal), c(n) = sqrt(2n+1),
// a(n, m) = sqrt((n^2 - m^2)/(2n-1)), b(n, m) = 1/sqrt(((n+1)^2 - m^2)/(2n+3)).
// LegDirect computes them; kernels pass shared-memory tables (LegTab).
template <typename T>
struct LegDirect {
  HD T d(int n) const { return sqrt((T)(2 * n + 3) / (T)(2 * n + 2)); }
  HD T c(int n) const { return sqrt((T)(2 * n + 1)); }
  HD T a(int n, int m) const { return sqrt((T)(n * n - m * m) / (T)(2 * n - 1)); }
  HD T b(int n, int m) const {
    return T(1) / sqrt((T)((n + 1) * (n + 1) - m * m) / (T)(2 * n + 3));
  }
};
// the same from tables of degrees n <= nmax (rows of nmax + 1 orders)
template <typename T>
struct LegTab {
  const T* t;    // [4][nmax + 1][nmax + 1]: a, b, then c and d in row 0 of planes 2, 3
  int W;         // nmax + 1
  HD T d(int n) const { return t[3 * W * W + n]; }
  HD T c(int n) const { return t[2 * W * W + n]; }
  HD T a(int n, int m) const { return t[n * W + m]; }
  HD T b(int n, int m) const { return t[W * W + n * W + m]; }
};
// fill a LegTab's storage (4 (nmax+1)^2 values) with threads tid, tid+nt, ...
template <typename T>
HD void leg_table_fill(T* t, int nmax, int tid, int nt) {
  const int W = nmax + 1;
  const LegDirect<T> L;
  for (int i = tid; i < W * W; i += nt) {
    const int n = i / W, m = i - n * W;
    t[i] = m <= n && n >= 1 ? L.a(n, m) : T(0);
    t[W * W + i] = m <= n ? L.b(n, m) : T(0);
    if (i < W) { t[2 * W * W + i] = L.c(i); t[3 * W * W + i] = L.d(i); }
  }
}

// Advance: pnm1 holds degree n-1 on entry, pn degree n; on exit pnm1 holds
// degree n+1 (caller swaps roles).  Entry n+1 of pn is zeroed, as in the
// reference (src/util.c:58-86).
template <typename T, class R, class Leg = LegDirect<T>>
HD void legendre_step(R pnm1, R pn, int n, T C, T S, const Leg& L = Leg()) {
  pnm1[n + 1] = L.d(n) * S * pn[n];
  pn[n + 1] = T(0);
  const T sq = L.c(n);
#pragma unroll
  for (int m = 0; m <= n; m++) {
    const T v = C * sq * pn[m] - L.a(n, m) * pnm1[m];
    pnm1[m] = v * L.b(n, m);
  }
}

// One step of the recursion from degree n into a third row: out receives
// degree n + 1 from pnm1 (degree n - 1) and pn (degree n), which are left
// as they are; the arithmetic of legendre_step.  Entries of out above n + 1
// must be zero already (rows start zeroed and only ever take higher degrees).
template <typename T, class R, class Leg>
HD void legendre_next(R out, R pnm1, R pn, int n, T C, T S, const Leg& L) {
  out[n + 1] = L.d(n) * S * pn[n];
  const T sq = L.c(n);
  for (int m = 0; m <= n; m++) {
    const T v = C * sq * pn[m] - L.a(n, m) * pnm1[m];
    out[m] = v * L.b(n, m);
  }
}

// A row of per-point scratch values with entry i at p[i * s]: the kernels
// give each thread strided slices of shared memory (s = the CTA's thread
// count, so that a warp's 32 threads touch 32 consecutive words), host code
// a plain array (s = 1).
template <typename T>
struct Row {
  T* p;
  int s;
  HD T& operator[](int i) const { return p[i * s]; }
};
// k rows of len entries each: row k at p + k len s
template <typename T>
struct Scratch {
  T* p;
  int len, s;
  HD Row<T> row(int k) const { return Row<T>{p + k * len * s, s}; }
};

// Spherical Bessel j_n by series, used when x <= n (src/util.c:118-141):
// the prefactor x^n / (2n+1)!! times the sum of the series
template <typename T>
HD T bessel_j_series_sum(int n, T x) {
  const T tol = sizeof(T) == 4 ? T(1e-7) : T(1e-15);
  T x2q = T(1), x2 = x * x;
  T jn = x2q;
  for (int q = 0; (q < 64) && (fabs(x2q) > tol); q++) {
    x2q *= -x2 / (T)((2 * q + 2) * (2 * n + 2 * (q + 1) + 1));
    jn += x2q;
  }
  return jn;
}
template <typename T>
HD T bessel_j_series(int n, T x) {
  T sc = T(1) / (T)(2 * n + 1);
  for (int q = 0; q < n; q++) sc *= x / (T)(2 * q + 1);
  return bessel_j_series_sum<T>(n, x) * sc;
}
template <typename T>
HD void bessel_j_init(T x, T* j0, T* j1) {
  if (x > T(0)) {
    *j0 = sin(x) / x;
    *j1 = *j0 / x - cos(x) / x;
    return;
  }
  *j0 = T(1); *j1 = T(0);
}
// (j_{n-1}, j_n) -> (j_n, j_{n+1}) (src/util.c:155-175)
template <typename T>
HD void bessel_j_step(T* jnm1, T* jn, T x, int n) {
  if (x > (T)(n + 1)) {
    T jnp1 = (*jn) * (T)(2 * n + 1) / x - (*jnm1);
    *jnm1 = *jn; *jn = jnp1;
    return;
  }
  *jnm1 = *jn;
  *jn = bessel_j_series<T>(n + 1, x);
}
// j_{n-1}, j_n at x for n = 1, 2, ...: the steps of bessel_j_step, with the
// series prefactor x^n / (2n-1)!! carried from degree to degree (one
// division a step instead of n)
template <typename T>
struct BesselJSeq {
  T x, jm, j, a;
  int n;
  HD explicit BesselJSeq(T x_) : x(x_), n(1) {
    bessel_j_init(x, &jm, &j);
    a = x;
  }
  HD void step() {
    a *= x / (T)(2 * n + 1);               // x^(n+1) / (2n+1)!!
    T jn1;
    if (x > (T)(n + 1)) jn1 = j * (T)(2 * n + 1) / x - jm;
    else jn1 = bessel_j_series_sum<T>(n + 1, x) * (a / (T)(2 * n + 3));
    jm = j; j = jn1; n++;
  }
};

// h_n = j_n + i y_n, upward recursion (src/util.c:177-202)
template <typename T>
HD void bessel_h_init(T x, T* h0, T* h1) {
  T s = sin(x), c = cos(x);
  h0[0] = s / x; h0[1] = -c / x;
  h1[0] = h0[0] / x + h0[1];
  h1[1] = h0[1] / x - h0[0];
}
template <typename T>
HD void bessel_h_step(T* hnm1, T* hn, T x, int n) {
  T t = hn[0] * (T)(2 * n + 1) / x - hnm1[0];
  hnm1[0] = hn[0]; hn[0] = t;
  t = hn[1] * (T)(2 * n + 1) / x - hnm1[1];
  hnm1[1] = hn[1]; hn[1] = t;
}

// Coordinate frame for a shift from x to y, z axis along y-x
// (src/util.c:227-266), and the Euler angles between frames
// (src/rotations.c:99-129).
HD void shift_frame(const double* x, const double* y, double* ix, double* iy,
                    double* iz, double* r) {
  iz[0] = y[0] - x[0]; iz[1] = y[1] - x[1]; iz[2] = y[2] - x[2];
  *r = sqrt(iz[0] * iz[0] + iz[1] * iz[1] + iz[2] * iz[2]);
  iz[0] /= *r; iz[1] /= *r; iz[2] /= *r;
  if (iz[0] != 0.0) {
    ix[0] = iz[1]; ix[1] = -iz[0]; ix[2] = 0.0;
  } else if (iz[1] != 0.0) {
    ix[0] = 1.0; ix[1] = iz[2]; ix[2] = -iz[1];
  } else {
    ix[0] = 1.0; ix[1] = 0.0; ix[2] = 0.0;
  }
  double l = sqrt(ix[0] * ix[0] + ix[1] * ix[1] + ix[2] * ix[2]);
  ix[0] /= l; ix[1] /= l; ix[2] /= l;
  iy[0] = iz[1] * ix[2] - iz[2] * ix[1];
  iy[1] = iz[2] * ix[0] - iz[0] * ix[2];
  iy[2] = iz[0] * ix[1] - iz[1] * ix[0];
}
// angles of the rotation taking the unit frame to (jx, jy, jz)
HD void frame_angles(const double* jx, const double* jy, const double* jz,
                     double* th, double* ph, double* ch) {
  *th = acos(jz[2]);
  *ch = atan2(jz[1], jz[0]);
  *ph = atan2(jy[2], jx[2]);
}
// angles and distance of a shift from point a to point b
HD void shift_angles(const double* a, const double* b, double* th, double* ph,
                     double* ch, double* r) {
  double ix[3], iy[3], iz[3];
  shift_frame(a, b, ix, iy, iz, r);
  frame_angles(ix, iy, iz, th, ph, ch);
}

}  // namespace wbfmm
