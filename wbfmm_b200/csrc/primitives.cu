// The reference's single-expansion primitives (src/wbfmm.h:247-263,
// :266-320, :347-361, :402-420, :525-643, :1138-1194): expansion
// coefficients of a point source, evaluation of a regular or singular
// expansion at a point, H rotation and coaxial translation tables, and the
// rotation and coaxial translation of one expansion.  The array primitives
// run on the GPU through the engine's own device code (expand.cuh,
// translate.cuh, tables.cu): the caller's host arrays are copied to a
// library scratch area, one CTA computes, and the result is copied back
// before the call returns.  The scalar helpers (Legendre, Bessel, spherical
// coordinates) are the same __host__ __device__ routines run on the host.
//
// Semantics kept from the reference: coefficient c of component j of a
// Helmholtz array at Ci[2 (c cstr + j)] (complex), of a Laplace array at
// Ci[c cstr + j] (real-packed, src/wbfmm-private.h:76); fields at
// field[j fstr] (Helmholtz, complex) or field[j] (Laplace); rotation and
// coaxial translation leave Co = sc Co + T(Ci); expansion coefficients and
// fields are added to what the caller holds.  The Laplace R|R translation
// keeps the reference's summation ranges and its repeated scaling of Co by
// sc (src/laplace.c:571-627).  Where the reference reads or writes outside
// the expansions it is given, these stay inside them: the Helmholtz coaxial
// translation sums input degrees <= Ni (the reference reads degrees up to
// No - 1 for outputs above Ni + 1, src/translations.c:455-462), and the
// Laplace R|R writes output degrees <= No (the reference writes m = 0
// outputs up to degree Ni, src/laplace.c:600-610).
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "engine.h"
#include "expand.cuh"
#include "wbfmm_b200.h"
#include "fmm_math.cuh"
#include "tables.h"
#include "translate.cuh"
#include "wbfmm.h"

namespace wbfmm {
namespace {

constexpr int kPrimThreads = 128;

#define PRIM_TRY(call)             \
  do {                             \
    const int rc_ = (call);        \
    if (rc_) return rc_;           \
  } while (0)

// ---------------------------------------------------------------- kernels
// Co = sc Co + rotation of Ci (Helmholtz, complex, cidx layout)
__global__ void k_prim_rotate_h(double* Co, int cstro, const double* Ci, int cstri, int N,
                                int nq, const double* H, double ph, double ch, double sc,
                                double* v, double* o, double* eph, double* ech) {
  const int tid = threadIdx.x, nt = blockDim.x, nc = (N + 1) * (N + 1);
  for (int j = tid; j <= N; j += nt) {
    eph[2 * j] = cos(j * ph); eph[2 * j + 1] = sin(j * ph);
    ech[2 * j] = cos(j * ch); ech[2 * j + 1] = sin(j * ch);
  }
  for (int q = 0; q < nq; q++) {
    __syncthreads();
    for (int c = tid; c < nc; c += nt) {
      v[2 * c] = Ci[2 * ((int64_t)c * cstri + q)];
      v[2 * c + 1] = Ci[2 * ((int64_t)c * cstri + q) + 1];
    }
    __syncthreads();
    phase_full(v, N, ech, tid, nt);
    __syncthreads();
    hsum_full<double, double, false>(o, v, N, H, eph, tid, nt);
    __syncthreads();
    for (int c = tid; c < nc; c += nt) {
      double* y = Co + 2 * ((int64_t)c * cstro + q);
      y[0] = sc * y[0] + o[2 * c];
      y[1] = sc * y[1] + o[2 * c + 1];
    }
  }
}

// Co = sc Co + coaxial translation of Ci (Helmholtz; complex table S|R or
// real R|R, coax_idx layout)
__global__ void k_prim_coax_h(double* Co, int cstro, int No, const double* Ci, int cstri,
                              int Ni, int nq, const double* tab, int cplx, double sc,
                              double* v, double* o) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int nci = (Ni + 1) * (Ni + 1), nco = (No + 1) * (No + 1);
  for (int q = 0; q < nq; q++) {
    __syncthreads();
    for (int c = tid; c < nci; c += nt) {
      v[2 * c] = Ci[2 * ((int64_t)c * cstri + q)];
      v[2 * c + 1] = Ci[2 * ((int64_t)c * cstri + q) + 1];
    }
    __syncthreads();
    if (cplx) coax_full<double, double, true>(o, v, No, Ni, tab, tid, nt);
    else coax_full<double, double, false>(o, v, No, Ni, tab, tid, nt);
    __syncthreads();
    for (int c = tid; c < nco; c += nt) {
      double* y = Co + 2 * ((int64_t)c * cstro + q);
      y[0] = sc * y[0] + o[2 * c];
      y[1] = sc * y[1] + o[2 * c + 1];
    }
  }
}

// Laplace: Co = sc Co + rotation of Ci (real-packed; half vectors inside)
__global__ void k_prim_rotate_l(double* Co, int cstro, const double* Ci, int cstri, int N,
                                int nq, const double* H, double ph, double ch, double sc,
                                double* v, double* o, double* eph, double* ech) {
  const int tid = threadIdx.x, nt = blockDim.x, nh = nhalf(N);
  for (int j = tid; j <= N; j += nt) {
    eph[2 * j] = cos(j * ph); eph[2 * j + 1] = sin(j * ph);
    ech[2 * j] = cos(j * ch); ech[2 * j + 1] = sin(j * ch);
  }
  for (int q = 0; q < nq; q++) {
    __syncthreads();
    for (int c = tid; c < nh; c += nt) {
      const int n = half_degree(c), m = c - n * (n + 1) / 2;
      if (m == 0) {
        v[2 * c] = Ci[(int64_t)n * n * cstri + q];
        v[2 * c + 1] = 0.0;
      } else {
        const int id = lidx(n, m);
        v[2 * c] = Ci[(int64_t)id * cstri + q];
        v[2 * c + 1] = Ci[(int64_t)(id + 1) * cstri + q];
      }
    }
    __syncthreads();
    phase_half(v, N, ech, tid, nt);
    __syncthreads();
    hsum_half<double, double, false>(o, v, N, H, eph, tid, nt);
    __syncthreads();
    for (int c = tid; c < nh; c += nt) {
      const int n = half_degree(c), m = c - n * (n + 1) / 2;
      if (m == 0) {
        double* y = Co + (int64_t)n * n * cstro + q;
        *y = sc * (*y) + o[2 * c];
      } else {
        const int id = lidx(n, m);
        double* y0 = Co + (int64_t)id * cstro + q;
        double* y1 = Co + (int64_t)(id + 1) * cstro + q;
        *y0 = sc * (*y0) + o[2 * c];
        *y1 = sc * (*y1) + o[2 * c + 1];
      }
    }
  }
}

// Laplace coaxial translations with the reference's ranges
// (src/laplace.c:496-696): kind 0 S|R, 1 S|S, 2 R|R; dense tables
// [n][nd][m] of dimension Lt + 1; one thread per output (n, m, slot)
__global__ void k_prim_coax_l(double* Co, int cstro, int No, const double* Ci, int cstri,
                              int Ni, int nq, double t, double sc, int kind,
                              const double* tab, int Lt) {
  const int Dm = Lt + 1;
  const int nout = nhalf(No);
  for (int i = threadIdx.x; i < nout * nq; i += blockDim.x) {
    const int c = i / nq, q = i - c * nq;
    const int n = half_degree(c), m = c - n * (n + 1) / 2;
    // input range and the number of times Co is scaled by sc
    int lo = m, hi = Ni, nscale = 1;
    if (kind == 1) hi = n < Ni ? n : Ni;
    if (kind == 2) {
      if (n > Ni) continue;             // untouched by the reference
      lo = n;
      hi = m == 0 ? Ni : No;
      nscale = (m == 0 ? Ni : No) - n + 1;
    }
    double sr = 0.0, si = 0.0;
    for (int nd = lo; nd <= hi; nd++) {
      double w = tab[((int64_t)n * Dm + nd) * Dm + m];
      if (kind == 0) {
        // tn[j] = sign(t) t^j
        w /= (t < 0 ? -1.0 : 1.0) * pow(t, (double)(n + nd + 1));
      } else if (kind == 1) {
        w *= pow(-t, (double)(n - nd));
      } else {
        w *= pow(t, (double)(nd - n));
      }
      if (m == 0) {
        sr += w * Ci[(int64_t)nd * nd * cstri + q];
      } else {
        const int id = lidx(nd, m);
        sr += w * Ci[(int64_t)id * cstri + q];
        si += w * Ci[(int64_t)(id + 1) * cstri + q];
      }
    }
    double s = 1.0;
    for (int k = 0; k < nscale; k++) s *= sc;
    if (m == 0) {
      double* y = Co + (int64_t)n * n * cstro + q;
      *y = s * (*y) + sr;
    } else {
      const int id = lidx(n, m);
      double* y0 = Co + (int64_t)id * cstro + q;
      double* y1 = Co + (int64_t)(id + 1) * cstro + q;
      *y0 = s * (*y0) + sr;
      *y1 = s * (*y1) + si;
    }
  }
}

// expansion coefficients of one point source, thread q per component:
// Helmholtz (complex strengths q[2 j]) or Laplace (q[j])
__global__ void k_prim_p2m(int helm, double k, int N, const double* x0, const double* xs,
                           const double* q, int nq, double* cfft, int cstr) {
  const int j = threadIdx.x;
  if (j >= nq) return;
  double loc[2 * kPtMax];
  const Scratch<double> sc{loc, N + kRowPad, 1};
  if (helm) {
    auto emit = [&](int idx, double re, double im) {
      cfft[2 * ((int64_t)idx * cstr + j)] += re;
      cfft[2 * ((int64_t)idx * cstr + j) + 1] += im;
    };
    p2m_helmholtz<double>(N, k, x0, xs, q[2 * j], q[2 * j + 1], emit, LegDirect<double>(), sc);
  } else {
    auto emit = [&](int idx, double v) { cfft[(int64_t)idx * cstr + j] += v; };
    p2m_laplace<double>(N, x0, xs, q[j], emit, LegDirect<double>(), sc);
  }
}

// evaluation of one expansion at xf, thread q per component.  kind 0:
// Helmholtz regular (j_n), 1: Helmholtz singular (h_n), 2: Laplace
// singular (r^-(n+1)), 3: Laplace regular potential, 4: Laplace regular
// gradient (field[3 j + a] with fstr 3... as the reference: field[fstr j])
__global__ void k_prim_eval(int kind, double k, const double* x0, const double* cfft, int cstr,
                            int N, int nq, const double* xf, double* field, int fstr) {
  const int j = threadIdx.x;
  if (j >= nq) return;
  double loc[3 * kPtMax];
  const Scratch<double> sc{loc, N + kRowPad, 1};
  if (kind == 0) {
    auto coef = [&](int idx, double* re, double* im) {
      *re = cfft[2 * ((int64_t)idx * cstr + j)];
      *im = cfft[2 * ((int64_t)idx * cstr + j) + 1];
    };
    double fr = 0.0, fi = 0.0;
    l2p_helmholtz<double>(N, k, x0, xf, coef, &fr, &fi, LegDirect<double>(), sc);
    field[(int64_t)j * fstr] += fr;
    field[(int64_t)j * fstr + 1] += fi;
    return;
  }
  if (kind == 3 || kind == 4) {
    auto coef = [&](int idx) { return cfft[(int64_t)idx * cstr + j]; };
    if (kind == 3) {
      field[j] += l2p_laplace<double>(N, x0, xf, coef, LegDirect<double>(), sc);
    } else {
      double g[3] = {0.0, 0.0, 0.0};
      l2p_laplace_grad<double>(N, x0, xf, coef, g, nullptr, LapRecDirect<double>(),
                               LegDirect<double>(), sc);
      for (int a = 0; a < 3; a++) field[(int64_t)fstr * j + a] += g[a];
    }
    return;
  }
  // singular expansions: the degree-n radial factor h_n(kr) (Helmholtz) or
  // r^-(n+1) (Laplace) times P_n^|m| e^{i m ph}
  if (N == 0) return;
  double r, th, ph;
  cart2sph(x0, xf, &r, &th, &ph);
  const double C = cos(th), S = sin(th), c1 = cos(ph), s1 = sin(ph);
  zero_rows(sc, 2);
  Row<double> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  if (kind == 1) {
    double hm[2], h[2];
    const double kr = k * r;
    bessel_h_init(kr, hm, h);
    double fr = 0.0, fi = 0.0;
    auto term = [&](int n, int m, int sgn, const double* hn, double P, double cm, double sm) {
      const int idx = cidx(n, sgn * m);
      const double ar = cfft[2 * ((int64_t)idx * cstr + j)], ai = cfft[2 * ((int64_t)idx * cstr + j) + 1];
      const double tr = ar * hn[0] - ai * hn[1], ti = ai * hn[0] + ar * hn[1];
      fr += (cm * tr - sgn * sm * ti) * P;
      fi += (cm * ti + sgn * sm * tr) * P;
    };
    term(0, 0, 1, hm, pm[0], 1.0, 0.0);
    if (N > 1) {
      term(1, 0, 1, h, pn[0], 1.0, 0.0);
      term(1, 1, 1, h, pn[1], c1, s1);
      term(1, 1, -1, h, pn[1], c1, s1);
      for (int n = 2; n <= N; n++) {
        legendre_step(pm, pn, n - 1, C, S);
        Row<double> tt = pm; pm = pn; pn = tt;
        bessel_h_step(hm, h, kr, n - 1);
        term(n, 0, 1, h, pn[0], 1.0, 0.0);
        double cm = 1.0, sm = 0.0;
        for (int m = 1; m <= n; m++) {
          rot_next(cm, sm, c1, s1, &cm, &sm);
          term(n, m, 1, h, pn[m], cm, sm);
          term(n, m, -1, h, pn[m], cm, sm);
        }
      }
    }
    field[(int64_t)j * fstr] += fr;
    field[(int64_t)j * fstr + 1] += fi;
    return;
  }
  // Laplace singular: L[n^2] r^-(n+1) P_n^0 + 2 sum r^-(n+1) P_n^m (L[id] cos - L[id+1] sin)
  double f = 0.0, rn = 1.0 / r;
  f += cfft[0 * cstr + j] * rn * pm[0];
  rn /= r;
  f += cfft[(int64_t)1 * cstr + j] * rn * pn[0];
  f += 2.0 * pn[1] * rn * (cfft[(int64_t)lidx(1, 1) * cstr + j] * c1 -
                           cfft[(int64_t)(lidx(1, 1) + 1) * cstr + j] * s1);
  for (int n = 2; n <= N; n++) {
    rn /= r;
    legendre_step(pm, pn, n - 1, C, S);
    Row<double> tt = pm; pm = pn; pn = tt;
    f += cfft[(int64_t)n * n * cstr + j] * rn * pn[0];
    double cm = 1.0, sm = 0.0;
    for (int m = 1; m <= n; m++) {
      rot_next(cm, sm, c1, s1, &cm, &sm);
      const int id = lidx(n, m);
      f += 2.0 * pn[m] * rn * (cfft[(int64_t)id * cstr + j] * cm - cfft[(int64_t)(id + 1) * cstr + j] * sm);
    }
  }
  field[j] += f;
}

// ------------------------------------------------------------- host side
struct PrimCtx {
  std::mutex mu;
  cudaStream_t s = nullptr;
  double* buf = nullptr;
  size_t cap = 0;
  double* lap = nullptr;     // dense Laplace SS, RR, SR tables of dimension lap_lt + 1
  int lap_lt = -1;
};
PrimCtx g_prim;

int prim_stream() {
  if (!g_prim.s) WBFMM_CUDA(cudaStreamCreateWithFlags(&g_prim.s, cudaStreamNonBlocking));
  return 0;
}

// device scratch of n doubles (grows; the stream is idle between calls)
int prim_scratch(size_t n, double** p) {
  if (n > g_prim.cap) {
    if (g_prim.buf) WBFMM_CUDA(cudaFree(g_prim.buf));
    g_prim.buf = nullptr;
    g_prim.cap = 0;
    WBFMM_CUDA(cudaMalloc(&g_prim.buf, sizeof(double) * n));
    g_prim.cap = n;
  }
  *p = g_prim.buf;
  return 0;
}

int h2d(double* d, const double* h, size_t n) {
  if (n && h) WBFMM_CUDA(cudaMemcpyAsync(d, h, sizeof(double) * n, cudaMemcpyHostToDevice, g_prim.s));
  return 0;
}
int d2h(double* h, const double* d, size_t n) {
  if (n && h) WBFMM_CUDA(cudaMemcpyAsync(h, d, sizeof(double) * n, cudaMemcpyDeviceToHost, g_prim.s));
  return 0;
}
int finish() {
  WBFMM_CUDA(cudaGetLastError());
  WBFMM_CUDA(cudaStreamSynchronize(g_prim.s));
  return 0;
}

// doubles spanned by coefficients 0..nc-1 of nq components at stride cstr
// (w doubles per value)
size_t extent(int nc, int cstr, int nq, int w) {
  if (nc <= 0 || nq <= 0) return 0;
  return (size_t)w * ((size_t)(nc - 1) * cstr + nq);
}

void die(const char* fn, const char* msg) {
  fprintf(stderr, "wbfmm: %s: %s\n", fn, msg);
  abort();
}
void check(const char* fn, int rc) {
  if (rc) die(fn, wbfmm_b200_last_error());
}

int laplace_tables(int Lt) {
  if (Lt <= g_prim.lap_lt) return 0;
  if (g_prim.lap) WBFMM_CUDA(cudaFree(g_prim.lap));
  g_prim.lap = nullptr;
  g_prim.lap_lt = -1;
  const size_t n = (size_t)(Lt + 1) * (Lt + 1) * (Lt + 1);
  WBFMM_CUDA(cudaMalloc(&g_prim.lap, sizeof(double) * 3 * n));
  PRIM_TRY(generate_laplace_tables(Lt, g_prim.lap, g_prim.lap + n, g_prim.lap + 2 * n, g_prim.s));
  g_prim.lap_lt = Lt;
  return 0;
}

// rotation (helm) of one expansion set
int rotate(int helm, double* Co, int cstro, const double* Ci, int cstri, int N, int nq,
           const double* H, double ph, double ch, double sc) {
  const int nc = (N + 1) * (N + 1);
  const size_t eo = extent(nc, cstro, nq, helm ? 2 : 1), ei = extent(nc, cstri, nq, helm ? 2 : 1);
  const size_t nh = rot_count(N), nv = 2 * (size_t)nc;
  double* d;
  PRIM_TRY(prim_stream());
  PRIM_TRY(prim_scratch(eo + ei + nh + 2 * nv + 4 * (N + 1), &d));
  double *dCo = d, *dCi = dCo + eo, *dH = dCi + ei, *v = dH + nh, *o = v + nv, *e = o + nv;
  PRIM_TRY(h2d(dCo, Co, eo));
  PRIM_TRY(h2d(dCi, Ci, ei));
  PRIM_TRY(h2d(dH, H, nh));
  if (helm)
    k_prim_rotate_h<<<1, kPrimThreads, 0, g_prim.s>>>(dCo, cstro, dCi, cstri, N, nq, dH, ph, ch,
                                                      sc, v, o, e, e + 2 * (N + 1));
  else
    k_prim_rotate_l<<<1, kPrimThreads, 0, g_prim.s>>>(dCo, cstro, dCi, cstri, N, nq, dH, ph, ch,
                                                      sc, v, o, e, e + 2 * (N + 1));
  PRIM_TRY(d2h(Co, dCo, eo));
  return finish();
}

int coax_h(double* Co, int cstro, int No, const double* Ci, int cstri, int Ni, int nq,
           const double* cfft, int L, int cplx, double sc) {
  const int nco = (No + 1) * (No + 1), nci = (Ni + 1) * (Ni + 1);
  const size_t eo = extent(nco, cstro, nq, 2), ei = extent(nci, cstri, nq, 2);
  const size_t nt = (size_t)coax_count(L) * (cplx ? 2 : 1);
  const size_t nv = 2 * (size_t)(nco > nci ? nco : nci);
  double* d;
  PRIM_TRY(prim_stream());
  PRIM_TRY(prim_scratch(eo + ei + nt + 2 * nv, &d));
  double *dCo = d, *dCi = dCo + eo, *dT = dCi + ei, *v = dT + nt, *o = v + nv;
  PRIM_TRY(h2d(dCo, Co, eo));
  PRIM_TRY(h2d(dCi, Ci, ei));
  PRIM_TRY(h2d(dT, cfft, nt));
  k_prim_coax_h<<<1, kPrimThreads, 0, g_prim.s>>>(dCo, cstro, No, dCi, cstri, Ni, nq, dT, cplx,
                                                  sc, v, o);
  PRIM_TRY(d2h(Co, dCo, eo));
  return finish();
}

int coax_l(double* Co, int cstro, int No, const double* Ci, int cstri, int Ni, int nq,
           double t, double sc, int kind) {
  const int nco = (No + 1) * (No + 1);
  // R|R reads input degrees up to No for m > 0 (src/laplace.c:612-624)
  const int nin = kind == 2 ? (No > Ni ? No : Ni) : Ni;
  const int nci = (nin + 1) * (nin + 1);
  const size_t eo = extent(nco, cstro, nq, 1), ei = extent(nci, cstri, nq, 1);
  double* d;
  PRIM_TRY(prim_stream());
  const int Lt = (No > nin ? No : nin) + 1;
  PRIM_TRY(laplace_tables(Lt));
  PRIM_TRY(prim_scratch(eo + ei, &d));
  double *dCo = d, *dCi = dCo + eo;
  PRIM_TRY(h2d(dCo, Co, eo));
  PRIM_TRY(h2d(dCi, Ci, ei));
  const size_t n3 = (size_t)(g_prim.lap_lt + 1) * (g_prim.lap_lt + 1) * (g_prim.lap_lt + 1);
  // generate_laplace_tables order: SS, RR, SR
  const double* tab = g_prim.lap + (kind == 1 ? 0 : kind == 2 ? n3 : 2 * n3);
  k_prim_coax_l<<<1, kPrimThreads, 0, g_prim.s>>>(dCo, cstro, No, dCi, cstri, Ni, nq, t, sc,
                                                  kind, tab, g_prim.lap_lt);
  PRIM_TRY(d2h(Co, dCo, eo));
  return finish();
}

int p2m(int helm, double k, int N, const double* x0, const double* xs, const double* q,
        int nq, double* cfft, int cstr) {
  if (nq > kPrimThreads) return set_error(WBFMM_B200_E_ARG, "at most 128 source components");
  const int nc = (N + 1) * (N + 1);
  const size_t ec = extent(nc, cstr, nq, helm ? 2 : 1), eq = (size_t)nq * (helm ? 2 : 1);
  double* d;
  PRIM_TRY(prim_stream());
  PRIM_TRY(prim_scratch(ec + eq + 6, &d));
  double *dc = d, *dq = dc + ec, *dx = dq + eq;
  PRIM_TRY(h2d(dc, cfft, ec));
  PRIM_TRY(h2d(dq, q, eq));
  PRIM_TRY(h2d(dx, x0, 3));
  PRIM_TRY(h2d(dx + 3, xs, 3));
  k_prim_p2m<<<1, kPrimThreads, 0, g_prim.s>>>(helm, k, N, dx, dx + 3, dq, nq, dc, cstr);
  PRIM_TRY(d2h(cfft, dc, ec));
  return finish();
}

// evaluation: nf doubles of field (the caller's span)
int eval(int kind, double k, const double* x0, const double* cfft, int cstr, int N, int nq,
         const double* xf, double* field, size_t nf, int fstr) {
  if (nq > kPrimThreads) return set_error(WBFMM_B200_E_ARG, "at most 128 source components");
  const int helm = kind <= 1;
  // Helmholtz j_n evaluation reads degree 1 even for N = 0, as the reference
  const int Nr = N < 1 ? 1 : N;
  const size_t ec = extent((Nr + 1) * (Nr + 1), cstr, nq, helm ? 2 : 1);
  double* d;
  PRIM_TRY(prim_stream());
  PRIM_TRY(prim_scratch(ec + nf + 6, &d));
  double *dc = d, *df = dc + ec, *dx = df + nf;
  PRIM_TRY(h2d(dc, cfft, ec));
  PRIM_TRY(h2d(df, field, nf));
  PRIM_TRY(h2d(dx, x0, 3));
  PRIM_TRY(h2d(dx + 3, xf, 3));
  k_prim_eval<<<1, kPrimThreads, 0, g_prim.s>>>(kind, k, dx, dc, cstr, N, nq, dx + 3, df, fstr);
  PRIM_TRY(d2h(field, df, nf));
  return finish();
}

int tables_h(int kind, double* out, int N, double arg) {
  double* d;
  PRIM_TRY(prim_stream());
  if (kind == 0) {   // H rotation
    const size_t n = rot_count(N) + 16;
    PRIM_TRY(prim_scratch(n, &d));
    WBFMM_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * n, g_prim.s));
    PRIM_TRY(generate_rotation_tables(std::vector<double>{arg}, N, d, (int64_t)n, g_prim.s));
    PRIM_TRY(d2h(out, d, rot_count(N)));
  } else {           // coaxial: 1 R|R (real), 2 S|R (complex)
    const size_t n = (size_t)coax_count(N) * kind;
    PRIM_TRY(prim_scratch(n + 16, &d));
    WBFMM_CUDA(cudaMemsetAsync(d, 0, sizeof(double) * (n + 16), g_prim.s));
    PRIM_TRY(generate_coaxial_tables(std::vector<double>{arg}, N, kind, d, (int64_t)n, g_prim.s));
    PRIM_TRY(d2h(out, d, n));
  }
  return finish();
}

// ------------------------------------------------------------ FP32 twins
// float arrays of n values as doubles, and back (exact both ways for the
// values the call does not change)
std::vector<double> wide(const float* p, size_t n) {
  std::vector<double> o(n);
  for (size_t i = 0; i < n; i++) o[i] = p ? (double)p[i] : 0.0;
  return o;
}
void narrow(float* p, const std::vector<double>& v) {
  for (size_t i = 0; i < v.size(); i++) p[i] = (float)v[i];
}

std::lock_guard<std::mutex> lock_prim() { return std::lock_guard<std::mutex>(g_prim.mu); }

}  // namespace
}  // namespace wbfmm

using namespace wbfmm;

extern "C" {

// ------------------------------------------------------- scalar helpers
/* src/util.c:30-56 */
gint wbfmm_cartesian_to_spherical(gdouble* x0, gdouble* x, gdouble* r, gdouble* th, gdouble* ph) {
  cart2sph<double>(x0, x, r, th, ph);
  return 0;
}
gint wbfmm_cartesian_to_spherical_f(gfloat* x0, gfloat* x, gfloat* r, gfloat* th, gfloat* ph) {
  cart2sph<float>(x0, x, r, th, ph);
  return 0;
}
/* src/util.c:97-116 */
gint wbfmm_legendre_init(gdouble C, gdouble S, gdouble* P0, gdouble* P10, gdouble* P11) {
  legendre_init<double>(C, S, P0, P10, P11);
  return 0;
}
gint wbfmm_legendre_init_f(gfloat C, gfloat S, gfloat* P0, gfloat* P10, gfloat* P11) {
  legendre_init<float>(C, S, P0, P10, P11);
  return 0;
}
/* src/util.c:58-86: *Pnm1 (degree n-1) and *Pn (degree n) become degrees
   n and n+1 (the arrays swap roles) */
gint wbfmm_legendre_recursion_array(gdouble** Pnm1, gdouble** Pn, gint n, gdouble C, gdouble S) {
  legendre_step<double>(*Pnm1, *Pn, n, C, S);
  gdouble* t = *Pnm1; *Pnm1 = *Pn; *Pn = t;
  return 0;
}
gint wbfmm_legendre_recursion_array_f(gfloat** Pnm1, gfloat** Pn, gint n, gfloat C, gfloat S) {
  legendre_step<float>(*Pnm1, *Pn, n, C, S);
  gfloat* t = *Pnm1; *Pnm1 = *Pn; *Pn = t;
  return 0;
}
/* src/util.c:143-175 */
gint wbfmm_bessel_j_init(gdouble x, gdouble* j0, gdouble* j1) {
  bessel_j_init<double>(x, j0, j1);
  return 0;
}
gint wbfmm_bessel_j_init_f(gfloat x, gfloat* j0, gfloat* j1) {
  bessel_j_init<float>(x, j0, j1);
  return 0;
}
gint wbfmm_bessel_j_recursion(gdouble* jnm1, gdouble* jn, gdouble x, gint n) {
  bessel_j_step<double>(jnm1, jn, x, n);
  return 0;
}
gint wbfmm_bessel_j_recursion_f(gfloat* jnm1, gfloat* jn, gfloat x, gint n) {
  bessel_j_step<float>(jnm1, jn, x, n);
  return 0;
}
/* src/util.c:177-202 */
gint wbfmm_bessel_h_init(gdouble x, gdouble* h0, gdouble* h1) {
  bessel_h_init<double>(x, h0, h1);
  return 0;
}
gint wbfmm_bessel_h_init_f(gfloat x, gfloat* h0, gfloat* h1) {
  bessel_h_init<float>(x, h0, h1);
  return 0;
}
gint wbfmm_bessel_h_recursion(gdouble* hnm1, gdouble* hn, gdouble x, gint n) {
  bessel_h_step<double>(hnm1, hn, x, n);
  return 0;
}
gint wbfmm_bessel_h_recursion_f(gfloat* hnm1, gfloat* hn, gfloat x, gint n) {
  bessel_h_step<float>(hnm1, hn, x, n);
  return 0;
}

// ------------------------------------------------------------ tables
/* src/rotations.c:131-207 */
gint wbfmm_coefficients_H_rotation(gdouble* H, gint N, gdouble th, gdouble* work) {
  (void)work;
  auto l = lock_prim();
  check(__func__, tables_h(0, H, N, th));
  return 0;
}
/* src/translations.c:182-409 */
gint wbfmm_coefficients_RR_coaxial(gdouble* cfft, gint L, gdouble kr, gdouble* work) {
  (void)work;
  auto l = lock_prim();
  check(__func__, tables_h(1, cfft, L, kr));
  return 0;
}
gint wbfmm_coefficients_SR_coaxial(gdouble* cfft, gint L, gdouble kr, gdouble* work) {
  (void)work;
  auto l = lock_prim();
  check(__func__, tables_h(2, cfft, L, kr));
  return 0;
}
gint wbfmm_coefficients_H_rotation_f(gfloat* H, gint N, gfloat th, gfloat* work) {
  std::vector<double> h((size_t)rot_count(N));
  (void)work;
  wbfmm_coefficients_H_rotation(h.data(), N, th, nullptr);
  narrow(H, h);
  return 0;
}
gint wbfmm_coefficients_RR_coaxial_f(gfloat* cfft, gint L, gfloat kr, gfloat* work) {
  std::vector<double> c((size_t)coax_count(L));
  (void)work;
  wbfmm_coefficients_RR_coaxial(c.data(), L, kr, nullptr);
  narrow(cfft, c);
  return 0;
}
gint wbfmm_coefficients_SR_coaxial_f(gfloat* cfft, gint L, gfloat kr, gfloat* work) {
  std::vector<double> c(2 * (size_t)coax_count(L));
  (void)work;
  wbfmm_coefficients_SR_coaxial(c.data(), L, kr, nullptr);
  narrow(cfft, c);
  return 0;
}

// ------------------------------------------- rotation and translation
/* src/rotations.c:419-593 */
gint wbfmm_rotate_H_ref(gdouble* Co, gint cstro, gdouble* Ci, gint cstri, gint N, gint nq,
                        gdouble* H, gdouble ph, gdouble ch, gdouble sc) {
  if (cstro < nq || cstri < nq) die(__func__, "coefficient stride less than number of source components");
  auto l = lock_prim();
  check(__func__, rotate(1, Co, cstro, Ci, cstri, N, nq, H, ph, ch, sc));
  return 0;
}
gint wbfmm_rotate_H_avx(gdouble* Co, gint cstro, gdouble* Ci, gint cstri, gint N, gint nq,
                        gdouble* H, gdouble ph, gdouble ch, gdouble sc) {
  return wbfmm_rotate_H_ref(Co, cstro, Ci, cstri, N, nq, H, ph, ch, sc);
}
/* src/rotations-laplace.c:35-216 */
gint wbfmm_laplace_rotate_H_ref(gdouble* Co, gint cstro, gdouble* Ci, gint cstri, gint N,
                                gint nq, gdouble* H, gdouble ph, gdouble ch, gdouble sc) {
  if (cstro < nq || cstri < nq) die(__func__, "coefficient stride less than number of source components");
  auto l = lock_prim();
  check(__func__, rotate(0, Co, cstro, Ci, cstri, N, nq, H, ph, ch, sc));
  return 0;
}
gint wbfmm_laplace_rotate_H_avx(gdouble* Co, gint cstro, gdouble* Ci, gint cstri, gint N,
                                gint nq, gdouble* H, gdouble ph, gdouble ch, gdouble sc) {
  return wbfmm_laplace_rotate_H_ref(Co, cstro, Ci, cstri, N, nq, H, ph, ch, sc);
}
/* src/translations.c:411-604 */
gint wbfmm_coaxial_translate_ref(gdouble* Co, gint cstro, gint No, gdouble* Ci, gint cstri,
                                 gint Ni, gint nq, gdouble* cfft, gint L, gboolean complex,
                                 gdouble sc) {
  if (L < No || L < Ni) die(__func__, "coaxial table order below the expansion orders");
  if (cstro < nq || cstri < nq) die(__func__, "coefficient stride less than number of source components");
  auto l = lock_prim();
  check(__func__, coax_h(Co, cstro, No, Ci, cstri, Ni, nq, cfft, L, complex ? 1 : 0, sc));
  return 0;
}
/* src/laplace.c:496-696 */
gint wbfmm_laplace_coaxial_translate_SS(gdouble* Co, gint cstro, gint No, gdouble* Ci,
                                        gint cstri, gint Ni, gint nq, gdouble t, gdouble sc) {
  auto l = lock_prim();
  check(__func__, coax_l(Co, cstro, No, Ci, cstri, Ni, nq, t, sc, 1));
  return 0;
}
gint wbfmm_laplace_coaxial_translate_RR(gdouble* Co, gint cstro, gint No, gdouble* Ci,
                                        gint cstri, gint Ni, gint nq, gdouble t, gdouble sc) {
  auto l = lock_prim();
  check(__func__, coax_l(Co, cstro, No, Ci, cstri, Ni, nq, t, sc, 2));
  return 0;
}
gint wbfmm_laplace_coaxial_translate_SR(gdouble* Co, gint cstro, gint No, gdouble* Ci,
                                        gint cstri, gint Ni, gint nq, gdouble t, gdouble sc) {
  auto l = lock_prim();
  check(__func__, coax_l(Co, cstro, No, Ci, cstri, Ni, nq, t, sc, 0));
  return 0;
}

// --------------------------------------------------- expansions
/* src/expansions.c:48-123 */
gint wbfmm_expansion_h_cfft(gdouble k, gint N, gdouble* x0, gdouble* xs, gdouble* q, gint nq,
                            gdouble* cfft, gint cstr, gdouble* work) {
  (void)work;
  if (cstr < nq) die(__func__, "coefficient stride less than number of source elements");
  auto l = lock_prim();
  check(__func__, p2m(1, k, N, x0, xs, q, nq, cfft, cstr));
  return 0;
}
/* src/laplace.c:35-129 */
gint wbfmm_laplace_expansion_cfft(gint N, gdouble* x0, gdouble* xs, gdouble* q, gint nq,
                                  gdouble* cfft, gint cstr, gdouble* work) {
  (void)work;
  if (cstr < nq) die(__func__, "coefficient stride less than number of source elements");
  auto l = lock_prim();
  check(__func__, p2m(0, 0.0, N, x0, xs, q, nq, cfft, cstr));
  return 0;
}
/* src/expansions.c:230-344 */
gint wbfmm_expansion_j_evaluate(gdouble k, gdouble* x0, gdouble* cfft, gint cstr, gint N, gint nq,
                                gdouble* xf, gdouble* field, gint fstr, gdouble* work) {
  (void)work;
  if (cstr < nq) die(__func__, "coefficient stride less than number of source elements");
  if (fstr < 2 && nq > 1) die(__func__, "field stride must be greater than 1 for multi-component sources");
  auto l = lock_prim();
  check(__func__, eval(0, k, x0, cfft, cstr, N, nq, xf, field,
                       (size_t)(nq - 1) * fstr + 2, fstr));
  return 0;
}
/* src/expansions.c:147-228 */
gint wbfmm_expansion_h_evaluate(gdouble k, gdouble* x0, gdouble* cfft, gint cstr, gint N, gint nq,
                                gdouble* xf, gdouble* field, gint fstr, gdouble* work) {
  (void)work;
  if (cstr < nq) die(__func__, "coefficient stride less than number of source elements");
  if (fstr < 2 && nq > 1) die(__func__, "field stride must be greater than 1 for multi-component sources");
  auto l = lock_prim();
  check(__func__, eval(1, k, x0, cfft, cstr, N, nq, xf, field,
                       (size_t)(nq - 1) * fstr + 2, fstr));
  return 0;
}
/* src/laplace.c:425-494: field[j] for component j */
gint wbfmm_laplace_expansion_evaluate(gdouble* x0, gdouble* cfft, gint cstr, gint N, gint nq,
                                      gdouble* xf, gdouble* field, gdouble* work) {
  (void)work;
  auto l = lock_prim();
  check(__func__, eval(2, 0.0, x0, cfft, cstr, N, nq, xf, field, (size_t)nq, 1));
  return 0;
}
/* src/local-laplace.c:1338-1373: the potential (field[j]) and the
   gradient (field[fstr j + a]); the curl modes from a single expansion are
   not provided (use wbfmm_laplace_box_field, or wbfmm_b200_laplace_curl*) */
gint wbfmm_laplace_expansion_local_eval(gdouble* x0, gdouble* cfft, gint cstr, gint N, gint nq,
                                        guint field, gdouble* xf, gdouble* f, gint fstr,
                                        gdouble* work) {
  (void)work;
  auto l = lock_prim();
  if (field == WBFMM_FIELD_POTENTIAL) {
    check(__func__, eval(3, 0.0, x0, cfft, cstr, N, nq, xf, f, (size_t)nq, 1));
  } else if (field == WBFMM_FIELD_GRADIENT || field == (WBFMM_FIELD_GRADIENT | WBFMM_FIELD_POTENTIAL)) {
    if (fstr < 3 && nq != 1) die(__func__, "field data stride must be greater than two");
    check(__func__, eval(4, 0.0, x0, cfft, cstr, N, nq, xf, f,
                         (size_t)(nq - 1) * fstr + 3, fstr));
  } else {
    die(__func__, "only the potential and gradient fields are evaluated from a single expansion");
  }
  return 0;
}

// ---------------------------------------------------- FP32 twins
gint wbfmm_rotate_H_ref_f(gfloat* Co, gint cstro, gfloat* Ci, gint cstri, gint N, gint nq,
                          gfloat* H, gfloat ph, gfloat ch, gfloat sc) {
  const int nc = (N + 1) * (N + 1);
  auto co = wide(Co, extent(nc, cstro, nq, 2)), ci = wide(Ci, extent(nc, cstri, nq, 2));
  auto h = wide(H, rot_count(N));
  wbfmm_rotate_H_ref(co.data(), cstro, ci.data(), cstri, N, nq, h.data(), ph, ch, sc);
  narrow(Co, co);
  return 0;
}
gint wbfmm_laplace_rotate_H_ref_f(gfloat* Co, gint cstro, gfloat* Ci, gint cstri, gint N,
                                  gint nq, gfloat* H, gfloat ph, gfloat ch, gfloat sc) {
  const int nc = (N + 1) * (N + 1);
  auto co = wide(Co, extent(nc, cstro, nq, 1)), ci = wide(Ci, extent(nc, cstri, nq, 1));
  auto h = wide(H, rot_count(N));
  wbfmm_laplace_rotate_H_ref(co.data(), cstro, ci.data(), cstri, N, nq, h.data(), ph, ch, sc);
  narrow(Co, co);
  return 0;
}
gint wbfmm_coaxial_translate_ref_f(gfloat* Co, gint cstro, gint No, gfloat* Ci, gint cstri,
                                   gint Ni, gint nq, gfloat* cfft, gint L, gboolean complex,
                                   gfloat sc) {
  auto co = wide(Co, extent((No + 1) * (No + 1), cstro, nq, 2));
  auto ci = wide(Ci, extent((Ni + 1) * (Ni + 1), cstri, nq, 2));
  auto c = wide(cfft, (size_t)coax_count(L) * (complex ? 2 : 1));
  wbfmm_coaxial_translate_ref(co.data(), cstro, No, ci.data(), cstri, Ni, nq, c.data(), L,
                              complex, sc);
  narrow(Co, co);
  return 0;
}
static gint lap_coax_f(int kind, gfloat* Co, gint cstro, gint No, gfloat* Ci, gint cstri,
                       gint Ni, gint nq, gfloat t, gfloat sc) {
  const int nin = kind == 2 ? (No > Ni ? No : Ni) : Ni;
  auto co = wide(Co, extent((No + 1) * (No + 1), cstro, nq, 1));
  auto ci = wide(Ci, extent((nin + 1) * (nin + 1), cstri, nq, 1));
  if (kind == 0) wbfmm_laplace_coaxial_translate_SR(co.data(), cstro, No, ci.data(), cstri, Ni, nq, t, sc);
  else if (kind == 1) wbfmm_laplace_coaxial_translate_SS(co.data(), cstro, No, ci.data(), cstri, Ni, nq, t, sc);
  else wbfmm_laplace_coaxial_translate_RR(co.data(), cstro, No, ci.data(), cstri, Ni, nq, t, sc);
  narrow(Co, co);
  return 0;
}
gint wbfmm_laplace_coaxial_translate_SR_f(gfloat* Co, gint cstro, gint No, gfloat* Ci,
                                          gint cstri, gint Ni, gint nq, gfloat t, gfloat sc) {
  return lap_coax_f(0, Co, cstro, No, Ci, cstri, Ni, nq, t, sc);
}
gint wbfmm_laplace_coaxial_translate_SS_f(gfloat* Co, gint cstro, gint No, gfloat* Ci,
                                          gint cstri, gint Ni, gint nq, gfloat t, gfloat sc) {
  return lap_coax_f(1, Co, cstro, No, Ci, cstri, Ni, nq, t, sc);
}
gint wbfmm_laplace_coaxial_translate_RR_f(gfloat* Co, gint cstro, gint No, gfloat* Ci,
                                          gint cstri, gint Ni, gint nq, gfloat t, gfloat sc) {
  return lap_coax_f(2, Co, cstro, No, Ci, cstri, Ni, nq, t, sc);
}
gint wbfmm_expansion_h_cfft_f(gfloat k, gint N, gfloat* x0, gfloat* xs, gfloat* q, gint nq,
                              gfloat* cfft, gint cstr, gfloat* work) {
  (void)work;
  double a[3] = {x0[0], x0[1], x0[2]}, b[3] = {xs[0], xs[1], xs[2]};
  auto c = wide(cfft, extent((N + 1) * (N + 1), cstr, nq, 2));
  auto qq = wide(q, 2 * (size_t)nq);
  wbfmm_expansion_h_cfft(k, N, a, b, qq.data(), nq, c.data(), cstr, nullptr);
  narrow(cfft, c);
  return 0;
}
gint wbfmm_laplace_expansion_cfft_f(gint N, gfloat* x0, gfloat* xs, gfloat* q, gint nq,
                                    gfloat* cfft, gint cstr, gfloat* work) {
  (void)work;
  double a[3] = {x0[0], x0[1], x0[2]}, b[3] = {xs[0], xs[1], xs[2]};
  auto c = wide(cfft, extent((N + 1) * (N + 1), cstr, nq, 1));
  auto qq = wide(q, (size_t)nq);
  wbfmm_laplace_expansion_cfft(N, a, b, qq.data(), nq, c.data(), cstr, nullptr);
  narrow(cfft, c);
  return 0;
}
static gint h_eval_f(int regular, gfloat k, gfloat* x0, gfloat* cfft, gint cstr, gint N, gint nq,
                     gfloat* xf, gfloat* field, gint fstr) {
  double a[3] = {x0[0], x0[1], x0[2]}, b[3] = {xf[0], xf[1], xf[2]};
  const int Nr = N < 1 ? 1 : N;
  auto c = wide(cfft, extent((Nr + 1) * (Nr + 1), cstr, nq, 2));
  auto f = wide(field, (size_t)(nq - 1) * fstr + 2);
  if (regular) wbfmm_expansion_j_evaluate(k, a, c.data(), cstr, N, nq, b, f.data(), fstr, nullptr);
  else wbfmm_expansion_h_evaluate(k, a, c.data(), cstr, N, nq, b, f.data(), fstr, nullptr);
  narrow(field, f);
  return 0;
}
gint wbfmm_expansion_j_evaluate_f(gfloat k, gfloat* x0, gfloat* cfft, gint cstr, gint N, gint nq,
                                  gfloat* xf, gfloat* field, gint fstr, gfloat* work) {
  (void)work;
  return h_eval_f(1, k, x0, cfft, cstr, N, nq, xf, field, fstr);
}
gint wbfmm_expansion_h_evaluate_f(gfloat k, gfloat* x0, gfloat* cfft, gint cstr, gint N, gint nq,
                                  gfloat* xf, gfloat* field, gint fstr, gfloat* work) {
  (void)work;
  return h_eval_f(0, k, x0, cfft, cstr, N, nq, xf, field, fstr);
}
gint wbfmm_laplace_expansion_evaluate_f(gfloat* x0, gfloat* cfft, gint cstr, gint N, gint nq,
                                        gfloat* xf, gfloat* field, gfloat* work) {
  double a[3] = {x0[0], x0[1], x0[2]}, b[3] = {xf[0], xf[1], xf[2]};
  (void)work;
  auto c = wide(cfft, extent((N + 1) * (N + 1), cstr, nq, 1));
  auto f = wide(field, (size_t)nq);
  wbfmm_laplace_expansion_evaluate(a, c.data(), cstr, N, nq, b, f.data(), nullptr);
  narrow(field, f);
  return 0;
}
gint wbfmm_laplace_expansion_local_eval_f(gfloat* x0, gfloat* cfft, gint cstr, gint N, gint nq,
                                          guint field, gfloat* xf, gfloat* f, gint fstr,
                                          gfloat* work) {
  double a[3] = {x0[0], x0[1], x0[2]}, b[3] = {xf[0], xf[1], xf[2]};
  const int grad = field != WBFMM_FIELD_POTENTIAL;
  (void)work;
  auto c = wide(cfft, extent((N + 1) * (N + 1), cstr, nq, 1));
  auto ff = wide(f, grad ? (size_t)(nq - 1) * fstr + 3 : (size_t)nq);
  wbfmm_laplace_expansion_local_eval(a, c.data(), cstr, N, nq, field, b, ff.data(), fstr, nullptr);
  narrow(f, ff);
  return 0;
}

}  // extern "C"
