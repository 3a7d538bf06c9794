// Translation-operator tables, generated on the GPU in FP64:
//  * rotation coefficients H_n^{nu,m}(theta), Gumerov-Duraiswami recursion
//    (5.55) seeded by Legendre functions up to degree 2N
//    (src/rotations.c:131-207);
//  * Helmholtz coaxial (S|R) and (R|R) = (S|S) coefficients, G&D
//    recursions (4.79), (4.84) seeded by h_l / j_l up to 2L
//    (src/translations.c:205-409);
//  * Laplace coaxial coefficients from log-gamma closed forms
//    (src/laplace.c:536-792).
// Plus the host-side shift geometry: for every list-4 offset and every
// child octant, the rotation angles and distance of the shift
// (src/shift.c:587-724 tabulates the same angles; src/util.c:227-266 and
// src/rotations.c:99-129 define them).
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <vector>

#include "../../include/wbfmm_b200.h"
#include "tables.h"

namespace wbfmm {

cudaMemPool_t library_pool();   // solver.cu

// Scratch of a table build, from the library's pool: its freed blocks stay
// cached there, so the builds of a serving loop (one per Helmholtz request)
// map no new device memory.  The device's default pool would return them
// at the next synchronisation and map them again for the next build.
static cudaError_t table_scratch(double** p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pl = library_pool();
  return pl ? cudaMallocFromPoolAsync((void**)p, bytes, pl, s)
            : cudaMallocAsync((void**)p, bytes, s);
}

// ------------------------------------------------------- host geometry
static int find_or_add(std::vector<double>& v, double x) {
  for (size_t i = 0; i < v.size(); i++)
    if (fabs(v[i] - x) < 1e-13) return (int)i;
  v.push_back(x);
  return (int)v.size() - 1;
}

void build_shift_geometry(ShiftGeometry* g) {
  g->thetas.clear();
  // list-4 offsets d = source - target, shift from source centre to target
  // centre (tools/wbfmm-tests.c.in:2082-2146 checks the reference's table
  // against exactly this construction)
  for (int i = -3; i <= 3; i++)
    for (int j = -3; j <= 3; j++)
      for (int k = -3; k <= 3; k++) {
        int idx = (i + 3) * 49 + (j + 3) * 7 + k + 3;
        ShiftAngles& a = g->offset[idx];
        if (i == 0 && j == 0 && k == 0) { a = ShiftAngles(); continue; }
        double xs[3] = {(double)i, (double)j, (double)k}, xt[3] = {0, 0, 0};
        shift_angles(xs, xt, &a.th, &a.ph, &a.ch, &a.r);
        a.ith = find_or_add(g->thetas, a.th);
        a.idist = i * i + j * j + k * k;
      }
  // child octants: child centre = parent centre + (w_child/2)(2b-1) per axis;
  // distances in units of the child width
  for (int c = 0; c < 8; c++) {
    double s[3] = {(c & 1) ? 0.5 : -0.5, (c & 2) ? 0.5 : -0.5,
                   (c & 4) ? 0.5 : -0.5};
    double o[3] = {0, 0, 0};
    ShiftAngles& up = g->child_to_parent[c];
    shift_angles(s, o, &up.th, &up.ph, &up.ch, &up.r);
    up.ith = find_or_add(g->thetas, up.th);
    ShiftAngles& dn = g->parent_to_child[c];
    shift_angles(o, s, &dn.th, &dn.ph, &dn.ch, &dn.r);
    dn.ith = find_or_add(g->thetas, dn.th);
  }
}

// ------------------------------------------------------ rotation tables
// One block per theta.  scratch holds rot_count(2N+1) doubles per block.
// small per-launch argument lists travel by value in the kernel parameters
struct Vals64 {
  double v[64];
};

__global__ void k_rotation_tables(const Vals64 thetas, int N,
                                  double* __restrict__ H, int64_t hstride,
                                  double* __restrict__ scratch,
                                  int64_t sstride) {
  const int it = blockIdx.x;
  double* h = scratch + (int64_t)it * sstride;
  const double th = thetas.v[it], C = cos(th), S = sin(th);
  const int NN = 2 * N;
  extern __shared__ double sm[];
  double* Pa = sm;                 // NN + 3 entries each
  double* Pb = sm + (NN + 3);

  for (int i = threadIdx.x; i < rot_count(NN) + 8; i += blockDim.x) h[i] = 0.0;
  __syncthreads();
  // m = 0 plane: H_n^{nu,0} = P_n^nu(cos th) sqrt(4 pi/(2n+1)), both signs
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2 * (NN + 3); i++) sm[i] = 0.0;
    double* pnm1 = Pa;
    double* pn = Pb;
    legendre_init(C, S, &pnm1[0], &pn[0], &pn[1]);
    const double s4 = sqrt(4.0 * kPi);
    h[rot_idx(0, 0, 0)] = pnm1[0] / sqrt(1.0) * s4;
    for (int nu = 0; nu <= 1; nu++) {
      h[rot_idx(nu, 0, 1)] = h[rot_idx(-nu, 0, 1)] = pn[nu] / sqrt(3.0) * s4;
    }
    for (int n = 2; n <= NN; n++) {
      legendre_step(pnm1, pn, n - 1, C, S);
      double* t = pnm1; pnm1 = pn; pn = t;    // pn now holds degree n
      for (int nu = 0; nu <= n; nu++)
        h[rot_idx(nu, 0, n)] = h[rot_idx(-nu, 0, n)] =
            pn[nu] / sqrt((double)(2 * n + 1)) * s4;
    }
  }
  __syncthreads();
  // recursion (5.55), advancing (nu, n) planes in the direction of m
  for (int m = 0; m <= N; m++) {
    const int nlo = m + 2, nhi = NN - m;
    if (nhi >= nlo) {
      // flatten (n, nu) with nu in [-n+1, n-1]: (2n-1) entries per n
      int total = 0;
      for (int n = nlo; n <= nhi; n++) total += 2 * n - 1;
      for (int e = threadIdx.x; e < total; e += blockDim.x) {
        int n = nlo, r = e;
        while (r >= 2 * n - 1) { r -= 2 * n - 1; n++; }
        int nu = r - (n - 1);
        double b = rec_b<double>(n, m);
        double b1 = rec_b<double>(n, -nu - 1);
        double b2 = rec_b<double>(n, nu - 1);
        double a3 = rec_a<double>(n - 1, nu);
        h[rot_idx(nu, m + 1, n - 1)] =
            (0.5 * (b1 * (1.0 - C) * h[rot_idx(nu + 1, m, n)] -
                    b2 * (1.0 + C) * h[rot_idx(nu - 1, m, n)]) -
             a3 * S * h[rot_idx(nu, m, n)]) / b;
      }
    }
    __syncthreads();
  }
  const int cnt = rot_count(N);
  for (int i = threadIdx.x; i < cnt; i += blockDim.x)
    H[(int64_t)it * hstride + i] = h[i];
}

int generate_rotation_tables(const std::vector<double>& thetas, int N,
                             double* dH, int64_t hstride, cudaStream_t s) {
  int nt = (int)thetas.size();
  if (nt > 64) return set_error(WBFMM_B200_E_ARG, "too many rotation angles");
  Vals64 th;
  memset(&th, 0, sizeof(th));
  for (int i = 0; i < nt; i++) th.v[i] = thetas[i];
  double* scratch = nullptr;
  int64_t sstride = rot_count(2 * N + 1) + 16;
  WBFMM_CUDA(table_scratch(&scratch, sizeof(double) * sstride * nt, s));
  size_t smem = sizeof(double) * 2 * (2 * N + 3);
  k_rotation_tables<<<nt, 256, smem, s>>>(th, N, dH, hstride, scratch, sstride);
  WBFMM_CUDA(cudaGetLastError());
  WBFMM_CUDA(cudaFreeAsync(scratch, s));
  return 0;
}

// --------------------------------------------- Helmholtz coaxial tables
// One block per table; a launch builds any set of tables, each with its
// own kr, order L and kind: nc = 2 (complex S|R) or 1 (real R|R).  kr may
// be negative (reverses the sense of the translation).  A table keeps the
// entries l <= L (coax_idx(L,L,L) < coax_count(L)); scratch holds the
// recursion's work range l <= 2L+1.
__global__ void k_coaxial_tables(const CoaxJobs jobs, double* __restrict__ scratch) {
  const int it = blockIdx.x;
  const int L = jobs.j[it].L, nc = jobs.j[it].nc;
  double* cf = scratch + jobs.j[it].scr_off;
  double kr = jobs.j[it].kr;
  int sw = 1;
  if (kr < 0) { kr = -kr; sw = -1; }
  const int LL = 2 * L + 2;
  for (int64_t i = threadIdx.x; i < (int64_t)coax_idx(LL, LL, LL) + 1; i += blockDim.x)
    cf[i * nc] = 0.0, cf[i * nc + nc - 1] = 0.0;
  __syncthreads();
  if (threadIdx.x == 0) {
    // seeds (E|F)_{l,0}^0 = (+-1)^l sqrt(2l+1) f_l(kr), G&D (4.83)
    int sgnl = 1;
    if (nc == 2) {
      double hm[2], h[2];
      bessel_h_init(kr, hm, h);
      cf[2 * coax_idx(0, 0, 0) + 0] = hm[0];
      cf[2 * coax_idx(0, 0, 0) + 1] = hm[1];
      sgnl *= sw;
      cf[2 * coax_idx(1, 0, 0) + 0] = sgnl * sqrt(3.0) * h[0];
      cf[2 * coax_idx(1, 0, 0) + 1] = sgnl * sqrt(3.0) * h[1];
      for (int l = 2; l <= 2 * L; l++) {
        bessel_h_step(hm, h, kr, l - 1);
        sgnl *= sw;
        cf[2 * coax_idx(l, 0, 0) + 0] = sgnl * sqrt((double)(2 * l + 1)) * h[0];
        cf[2 * coax_idx(l, 0, 0) + 1] = sgnl * sqrt((double)(2 * l + 1)) * h[1];
      }
    } else {
      double jm, j;
      bessel_j_init(kr, &jm, &j);
      cf[coax_idx(0, 0, 0)] = jm;
      sgnl *= sw;
      cf[coax_idx(1, 0, 0)] = sgnl * sqrt(3.0) * j;
      for (int l = 2; l <= 2 * L; l++) {
        bessel_j_step(&jm, &j, kr, l - 1);
        sgnl *= sw;
        cf[coax_idx(l, 0, 0)] = sgnl * sqrt((double)(2 * l + 1)) * j;
      }
    }
  }
  __syncthreads();
  // G&D (4.79): fill (E|F)_{l,n+1}^0
  for (int n = 0; n <= L; n++) {
    const int m = 0;
    for (int l = n + 1 + threadIdx.x; l <= 2 * L - n; l += blockDim.x) {
      int i1 = coax_idx(l, m, n - 1), i2 = coax_idx(l, m, n + 1);
      int i3 = coax_idx(l + 1, m, n), i4 = coax_idx(l - 1, m, n);
      double a1 = rec_a<double>(n - 1, m), a2 = rec_a<double>(n, m);
      double a3 = rec_a<double>(l, m), a4 = rec_a<double>(l - 1, m);
      for (int c = 0; c < nc; c++)
        cf[nc * i2 + c] = (a1 * (n >= 1 ? cf[nc * i1 + c] : 0.0) -
                           a3 * cf[nc * i3 + c] + a4 * cf[nc * i4 + c]) / a2;
    }
    __syncthreads();
  }
  // G&D (4.84): fill (E|F)_{l,m+1}^{m+1}
  for (int m = 0; m <= L; m++) {
    for (int l = m + 1 + threadIdx.x; l <= 2 * L - m; l += blockDim.x) {
      double a1 = rec_b<double>(m + 1, -m - 1), a2 = rec_b<double>(l, -m - 1);
      double a3 = rec_b<double>(l + 1, m);
      int i1 = coax_idx(l, m + 1, m + 1), i2 = coax_idx(l - 1, m, m);
      int i3 = coax_idx(l + 1, m, m);
      for (int c = 0; c < nc; c++)
        cf[nc * i1 + c] = (a2 * cf[nc * i2 + c] - a3 * cf[nc * i3 + c]) / a1;
    }
    __syncthreads();
  }
}

// G&D (4.79) for each order m >= 1 (independent of the other orders once
// the (4.84) diagonal is in place), one block per (m, table); then the
// order-m entries l <= L are copied out to the table's place in `out`.
// Block m = 0 only copies; blocks with m above the table's order leave.
__global__ void k_coaxial_orders(const CoaxJobs jobs, double* __restrict__ out,
                                 double* __restrict__ scratch) {
  const int m = blockIdx.x, it = blockIdx.y;
  const int L = jobs.j[it].L, nc = jobs.j[it].nc;
  if (m > L) return;
  double* cf = scratch + jobs.j[it].scr_off;
  double* o = out + jobs.j[it].out_off;
  if (m >= 1) {
    for (int n = m; n <= L; n++) {
      for (int l = n + 1 + threadIdx.x; l <= 2 * L - n; l += blockDim.x) {
        int i1 = coax_idx(l, m, n - 1), i2 = coax_idx(l, m, n + 1);
        int i3 = coax_idx(l + 1, m, n), i4 = coax_idx(l - 1, m, n);
        double a1 = rec_a<double>(n - 1, m), a2 = rec_a<double>(n, m);
        double a3 = rec_a<double>(l, m), a4 = rec_a<double>(l - 1, m);
        // a1 is zero when n-1 < m; the (l,m,n-1) slot is then not a
        // coefficient and is skipped
        for (int c = 0; c < nc; c++)
          cf[nc * i2 + c] = ((a1 != 0.0 ? a1 * cf[nc * i1 + c] : 0.0) -
                             a3 * cf[nc * i3 + c] + a4 * cf[nc * i4 + c]) / a2;
      }
      __syncthreads();
    }
  }
  // entries (l, m, n), m <= n <= l <= L
  for (int l = m; l <= L; l++)
    for (int n = m + threadIdx.x; n <= l; n += blockDim.x) {
      const int64_t i = coax_idx(l, m, n);
      for (int c = 0; c < nc; c++) o[nc * i + c] = cf[nc * i + c];
    }
}

int generate_coaxial_set(const CoaxJob* jobs, int njobs, double* dout, cudaStream_t s) {
  if (njobs <= 0) return 0;
  if (njobs > kMaxCoaxJobs) return set_error(WBFMM_B200_E_ARG, "too many coaxial tables in one set");
  CoaxJobs js;
  memset(&js, 0, sizeof(js));
  int Lmax = 0;
  int64_t scr = 0;
  for (int i = 0; i < njobs; i++) {
    js.j[i] = jobs[i];
    const int LL = 2 * jobs[i].L + 2;
    js.j[i].scr_off = scr;
    scr += ((int64_t)coax_idx(LL, LL, LL) + 2) * jobs[i].nc;
    Lmax = jobs[i].L > Lmax ? jobs[i].L : Lmax;
  }
  double* scratch = nullptr;
  WBFMM_CUDA(table_scratch(&scratch, sizeof(double) * scr, s));
  k_coaxial_tables<<<njobs, 128, 0, s>>>(js, scratch);
  WBFMM_CUDA(cudaGetLastError());
  k_coaxial_orders<<<dim3(Lmax + 1, njobs), 64, 0, s>>>(js, dout, scratch);
  WBFMM_CUDA(cudaGetLastError());
  WBFMM_CUDA(cudaFreeAsync(scratch, s));
  return 0;
}

int generate_coaxial_tables(const std::vector<double>& krs, int L, int nc,
                            double* dout, int64_t ostride, cudaStream_t s) {
  const int nt = (int)krs.size();
  if (nt > kMaxCoaxJobs) return set_error(WBFMM_B200_E_ARG, "too many coaxial distances");
  std::vector<CoaxJob> jobs(nt);
  for (int i = 0; i < nt; i++) {
    jobs[i].kr = krs[i];
    jobs[i].L = L;
    jobs[i].nc = nc;
    jobs[i].out_off = (int64_t)i * ostride;
    jobs[i].scr_off = 0;
  }
  return generate_coaxial_set(jobs.data(), nt, dout, s);
}

// FP32 copies of `ntables` complex (S|R) tables of order L (stride
// `stride` doubles) with entry (l, m, n) scaled by 2^(-e (l + n)): the
// scaled form of the Helmholtz FP32 M2L (helm_m2l_exp).  Thread per entry.
__global__ void k_narrow_coax_scaled(const double* __restrict__ src, float* __restrict__ dst,
                                     int L, int64_t stride, int ntables, int e) {
  const int64_t ne = coax_idx(L, L, L) + 1;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ne * ntables) return;
  const int t = (int)(i / ne);
  const int64_t c = i % ne;
  // (l, m, n) of entry c = coax_idx(l, m, n) = l(l+1)(l+2)/6 + n(n+1)/2 + m,
  // m <= n <= l: l is the largest with coax_idx(l, 0, 0) <= c, then n the
  // largest with n(n+1)/2 <= c - coax_idx(l, 0, 0)
  int l = 0;
  while (l < L && coax_idx(l + 1, 0, 0) <= c) l++;
  const int64_t r = c - coax_idx(l, 0, 0);
  int n = 0;
  while (n < l && (int64_t)(n + 1) * (n + 2) / 2 <= r) n++;
  const double f = ldexp(1.0, -e * (l + n));
  const double* a = src + (int64_t)t * stride + 2 * c;
  float* b = dst + (int64_t)t * stride + 2 * c;
  b[0] = (float)(a[0] * f);
  b[1] = (float)(a[1] * f);
}

int narrow_coax_scaled(const double* src, float* dst, int L, int64_t stride, int ntables,
                       int e, cudaStream_t s) {
  const int64_t tot = ((int64_t)coax_idx(L, L, L) + 1) * ntables;
  k_narrow_coax_scaled<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(src, dst, L, stride,
                                                                      ntables, e);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

// ----------------------------------------------- Laplace coaxial tables
// dense [n][nd][m] arrays for n, nd, m <= Lt (m <= min(n, nd));
// SS(n,nd,m) n >= nd, RR(n,nd,m) nd >= n, SR(n,nd,m) with (-1)^{n+m}
__global__ void k_laplace_tables(int Lt, double* __restrict__ SS,
                                 double* __restrict__ RR,
                                 double* __restrict__ SR) {
  const int D = Lt + 1;
  int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (int64_t)D * D * D) return;
  int m = (int)(e % D), nd = (int)((e / D) % D), n = (int)(e / ((int64_t)D * D));
  double ss = 0.0, rr = 0.0, sr = 0.0;
  if (m <= n && m <= nd) {
    double ln = log((2.0 * nd + 1) / (2.0 * n + 1));
    if (n >= nd) {
      double c = lgamma((double)(n - m + 1)) + lgamma((double)(n + m + 1)) -
                 lgamma((double)(nd - m + 1)) - lgamma((double)(nd + m + 1)) -
                 2.0 * lgamma((double)(n - nd + 1));
      ss = exp(0.5 * (c + ln));
    }
    if (nd >= n) {
      double c = lgamma((double)(nd - m + 1)) + lgamma((double)(nd + m + 1)) -
                 lgamma((double)(n - m + 1)) - lgamma((double)(n + m + 1)) -
                 2.0 * lgamma((double)(nd - n + 1));
      rr = exp(0.5 * (c + ln));
    }
    double c = 2.0 * lgamma((double)(n + nd + 1)) -
               lgamma((double)(n - m + 1)) - lgamma((double)(n + m + 1)) -
               lgamma((double)(nd - m + 1)) - lgamma((double)(nd + m + 1));
    sr = exp(0.5 * (c + ln)) * (((n + m) & 1) ? -1.0 : 1.0);
  }
  SS[e] = ss; RR[e] = rr; SR[e] = sr;
}

int generate_laplace_tables(int Lt, double* SS, double* RR, double* SR,
                            cudaStream_t s) {
  int64_t n = (int64_t)(Lt + 1) * (Lt + 1) * (Lt + 1);
  k_laplace_tables<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(Lt, SS, RR, SR);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

}  // namespace wbfmm
