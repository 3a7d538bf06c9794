// Precomputed target bases for repeated potential evaluations at fixed
// targets: the reference's target-list strategy (src/targets.c:168-422 and
// :424-603, potential only, as there).  For every target (in leaf-box
// order) the basis of the regular expansion of its leaf box (the value that
// multiplies each coefficient in the L2P: j_n(kr) P_n^|m| e^{i m ph} for
// Helmholtz, the real-packed r^n P_n^m (1, 2 cos, -2 sin) for Laplace) is
// stored coefficient-major, and the near-field weights of the sources of
// its 27 neighbour boxes (G(r) for a monopole, the normal derivative for a
// dipole, zero for pairs within the 1e-6 cutoff) in a CSR array over the
// sorted sources.  A repeated evaluation is then a product of the bases
// with the current local expansions plus a sparse product of the weights
// with the current strengths: bandwidth instead of special functions.
#include <cub/cub.cuh>

#include "engine.h"
#include "expand.cuh"
#include "fmm_math.cuh"
#include "kernels.h"

namespace wbfmm {

namespace {

// source range [s0, s0 + n) of neighbour a (0..26) of leaf box b, or n = 0
template <typename T>
__device__ __forceinline__ void neighbour(const EvalParams<T>& p, uint64_t b, int a,
                                         uint32_t* s0, uint32_t* n) {
  uint32_t bi, bj, bk;
  demorton(b, &bi, &bj, &bk);
  const int64_t n1 = ((int64_t)1 << p.level) - 1;
  const int64_t i = (int64_t)bi + a / 9 - 1, j = (int64_t)bj + (a / 3) % 3 - 1,
                k = (int64_t)bk + a % 3 - 1;
  if (i < 0 || j < 0 || k < 0 || i > n1 || j > n1 || k > n1) {
    *s0 = 0; *n = 0;
    return;
  }
  const uint64_t nb = morton((uint32_t)i, (uint32_t)j, (uint32_t)k);
  *s0 = p.box_i[nb];
  *n = p.box_n[nb];
}

template <typename T>
__global__ void k_tl_count(EvalParams<T> p, int64_t* cnt) {
  const int jt = blockIdx.x * blockDim.x + threadIdx.x;
  if (jt >= p.ntgt) return;
  int64_t c = 0;
  for (int a = 0; a < 27; a++) {
    uint32_t s0, n;
    neighbour(p, p.tbox[jt], a, &s0, &n);
    c += n;
  }
  cnt[jt] = c;
}

// warp per target: source indices and weights at off[jt] ...
template <typename T, bool HELM>
__global__ void k_tl_fill(EvalParams<T> p, const int64_t* __restrict__ off,
                          uint32_t* __restrict__ src, T* __restrict__ wq,
                          T* __restrict__ wd) {
  const int lane = threadIdx.x & 31;
  const int jt = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (jt >= p.ntgt) return;
  const double x = p.tx[jt], y = p.ty[jt], z = p.tz[jt];
  const double f4pi = 0.25 / kPi, k = (double)p.k;
  int64_t pos = off[jt];
  for (int a = 0; a < 27; a++) {
    uint32_t s0, n;
    neighbour(p, p.tbox[jt], a, &s0, &n);
    for (uint32_t u = lane; u < n; u += 32) {
      const uint32_t s = s0 + u;
      const int64_t o = pos + u;
      src[o] = s;
      const double rx = x - p.x[s], ry = y - p.y[s], rz = z - p.z[s];
      const double r2 = rx * rx + ry * ry + rz * rz;
      const bool ok = r2 > kCutoffRadius * kCutoffRadius;
      const double ir = ok ? 1.0 / sqrt(r2) : 0.0;
      double nr = 0.0;
      if (wd) nr = ((double)p.nx[s] * rx + (double)p.ny[s] * ry + (double)p.nz[s] * rz) * ir;
      if (HELM) {
        double h0r = 0.0, h0i = 0.0, h1r = 0.0, h1i = 0.0;
        if (ok) {
          double sn, cs;
          sincos(k * r2 * ir, &sn, &cs);
          const double ikr = ir / k;
          h0r = sn * ikr; h0i = -cs * ikr;
          h1r = h0r * ikr + h0i; h1i = h0i * ikr - h0r;
        }
        wq[2 * o] = (T)(f4pi * h0r);
        wq[2 * o + 1] = (T)(f4pi * h0i);
        if (wd) {
          wd[2 * o] = (T)(-k * f4pi * h1r * nr);
          wd[2 * o + 1] = (T)(-k * f4pi * h1i * nr);
        }
      } else {
        wq[o] = (T)(f4pi * ir);
        if (wd) wd[o] = (T)(f4pi * nr * ir * ir);
      }
    }
    pos += n;
  }
}

// thread per target: the basis of its leaf's regular expansion, entry
// (c, jt) at B[(c * nt + jt) * w]
template <typename T, bool HELM>
__global__ void k_tl_basis(EvalParams<T> p, T* __restrict__ B) {
  const int jt = blockIdx.x * blockDim.x + threadIdx.x;
  if (jt >= p.ntgt) return;
  const int N = p.N;
  const int64_t nt = p.ntgt;
  double cd[3];
  {
    // the box centre as the L2P forms it
    uint32_t i, j, k;
    demorton((uint64_t)p.tbox[jt], &i, &j, &k);
    cd[0] = p.x0 + p.wb * i; cd[1] = p.y0 + p.wb * j; cd[2] = p.z0 + p.wb * k;
    cd[0] += 0.5 * p.wb; cd[1] += 0.5 * p.wb; cd[2] += 0.5 * p.wb;
  }
  const double xc[3] = {0.0, 0.0, 0.0};
  const double xf[3] = {p.tx[jt] - cd[0], p.ty[jt] - cd[1], p.tz[jt] - cd[2]};
  double loc[2 * kPtMax];
  const Scratch<double> sc{loc, N + kRowPad, 1};
  double r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  const double C = cos(th), S = sin(th), c1 = cos(ph), s1 = sin(ph);
  zero_rows(sc, 2);
  Row<double> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  auto put = [&](int c, double re, double im) {
    if (HELM) {
      B[2 * ((int64_t)c * nt + jt)] = (T)re;
      B[2 * ((int64_t)c * nt + jt) + 1] = (T)im;
    } else {
      B[(int64_t)c * nt + jt] = (T)re;
    }
  };
  if (HELM) {
    BesselJSeq<double> bj((double)p.k * r);
    // degree n: j_n P_n^|m| e^{+-i m ph}
    auto degree = [&](int n, double jn, Row<double> P) {
      put(cidx(n, 0), jn * P[0], 0.0);
      double cm = 1.0, sm = 0.0;
      for (int m = 1; m <= n; m++) {
        rot_next(cm, sm, c1, s1, &cm, &sm);
        const double a = jn * P[m];
        put(cidx(n, m), a * cm, a * sm);
        put(cidx(n, -m), a * cm, -a * sm);
      }
    };
    degree(0, bj.jm, pm);
    degree(1, bj.j, pn);
    for (int n = 2; n <= N; n++) {
      legendre_step(pm, pn, n - 1, C, S);
      Row<double> t = pm; pm = pn; pn = t;
      bj.step();
      degree(n, bj.j, pn);
    }
  } else {
    double rn = 1.0;
    auto degree = [&](int n, double rr, Row<double> P) {
      put(n * n, rr * P[0], 0.0);
      double cm = 1.0, sm = 0.0;
      for (int m = 1; m <= n; m++) {
        rot_next(cm, sm, c1, s1, &cm, &sm);
        const int id = lidx(n, m);
        put(id, 2.0 * P[m] * rr * cm, 0.0);
        put(id + 1, -2.0 * P[m] * rr * sm, 0.0);
      }
    };
    degree(0, rn, pm);
    if (N >= 1) {
      rn *= r;
      degree(1, rn, pn);
    }
    for (int n = 2; n <= N; n++) {
      rn *= r;
      legendre_step(pm, pn, n - 1, C, S);
      Row<double> t = pm; pm = pn; pn = t;
      degree(n, rn, pn);
    }
  }
}

// thread per target: pot[o] = basis . local coefficients of its leaf
template <typename T, bool HELM>
__global__ void k_tl_far(EvalParams<T> p, const T* __restrict__ B) {
  const int jt = blockIdx.x * blockDim.x + threadIdx.x;
  if (jt >= p.ntgt) return;
  const int nc = ncoef(p.N);
  const int64_t nt = p.ntgt, b = p.tbox[jt];
  const uint32_t o = p.tperm[jt];
  double sr = 0.0, si = 0.0;
  for (int c = 0; c < nc; c++) {
    const int64_t lo = layout_off(b, c, nc);
    if (HELM) {
      const double br = B[2 * ((int64_t)c * nt + jt)], bi = B[2 * ((int64_t)c * nt + jt) + 1];
      const double ar = p.mpr[2 * lo], ai = p.mpr[2 * lo + 1];
      sr += br * ar - bi * ai;
      si += br * ai + bi * ar;
    } else {
      sr += (double)B[(int64_t)c * nt + jt] * (double)p.mpr[lo];
    }
  }
  if (HELM) {
    p.pot[2 * (size_t)o] = (T)sr;
    p.pot[2 * (size_t)o + 1] = (T)si;
  } else {
    p.pot[o] = (T)sr;
  }
}

// warp per target: pot[o] += weights . strengths of its near sources
template <typename T, bool HELM>
__global__ void k_tl_near(EvalParams<T> p, const int64_t* __restrict__ off,
                          const uint32_t* __restrict__ src, const T* __restrict__ wq,
                          const T* __restrict__ wd) {
  const int lane = threadIdx.x & 31;
  const int jt = (int)(((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  if (jt >= p.ntgt) return;
  double sr = 0.0, si = 0.0;
  const bool hq = p.q != nullptr, hd = wd != nullptr && p.dip != nullptr;
  for (int64_t o = off[jt] + lane; o < off[jt + 1]; o += 32) {
    const uint32_t s = src[o];
    if (HELM) {
      if (hq) {
        const double wr = wq[2 * o], wi = wq[2 * o + 1];
        const double qr = p.q[2 * s], qi = p.q[2 * s + 1];
        sr += wr * qr - wi * qi;
        si += wr * qi + wi * qr;
      }
      if (hd) {
        const double wr = wd[2 * o], wi = wd[2 * o + 1];
        const double dr = p.dip[2 * s], di = p.dip[2 * s + 1];
        sr += wr * dr - wi * di;
        si += wr * di + wi * dr;
      }
    } else {
      if (hq) sr += (double)wq[o] * (double)p.q[s];
      if (hd) sr += (double)wd[o] * (double)p.dip[s];
    }
  }
  for (int m = 16; m > 0; m >>= 1) {
    sr += __shfl_xor_sync(0xffffffffu, sr, m);
    si += __shfl_xor_sync(0xffffffffu, si, m);
  }
  if (lane) return;
  const uint32_t o = p.tperm[jt];
  if (HELM) {
    p.pot[2 * (size_t)o] = (T)((double)p.pot[2 * (size_t)o] + sr);
    p.pot[2 * (size_t)o + 1] = (T)((double)p.pot[2 * (size_t)o + 1] + si);
  } else {
    p.pot[o] = (T)((double)p.pot[o] + sr);
  }
}

}  // namespace

// pair counts and their offsets off[0..nt] (off[0] = 0); *npairs = off[nt]
template <typename T>
int tl_offsets(const EvalParams<T>& p, int64_t* off, int64_t* npairs, cudaStream_t s) {
  const int64_t nt = p.ntgt;
  WBFMM_CUDA(cudaMemsetAsync(off, 0, sizeof(int64_t), s));
  k_tl_count<T><<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(p, off + 1);
  WBFMM_CUDA(cudaGetLastError());
  size_t tmp = 0;
  void* scr = nullptr;
  WBFMM_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp, off + 1, off + 1, (int)nt, s));
  WBFMM_CUDA(cudaMallocAsync(&scr, tmp + 16, s));
  cudaError_t e = cub::DeviceScan::InclusiveSum(scr, tmp, off + 1, off + 1, (int)nt, s);
  cudaFreeAsync(scr, s);
  WBFMM_CUDA(e);
  WBFMM_CUDA(cudaMemcpyAsync(npairs, off + nt, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  WBFMM_CUDA(cudaStreamSynchronize(s));
  return 0;
}

template <typename T, bool HELM>
int tl_fill(const EvalParams<T>& p, const int64_t* off, uint32_t* src, T* wq, T* wd, T* basis,
            cudaStream_t s) {
  const int64_t nt = p.ntgt;
  k_tl_fill<T, HELM><<<(unsigned)((32 * nt + 255) / 256), 256, 0, s>>>(p, off, src, wq, wd);
  WBFMM_CUDA(cudaGetLastError());
  k_tl_basis<T, HELM><<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(p, basis);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

template <typename T, bool HELM>
int tl_apply(const EvalParams<T>& p, const T* basis, const int64_t* off, const uint32_t* src,
             const T* wq, const T* wd, cudaStream_t s) {
  const int64_t nt = p.ntgt;
  if (nt <= 0) return 0;
  k_tl_far<T, HELM><<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(p, basis);
  WBFMM_CUDA(cudaGetLastError());
  k_tl_near<T, HELM><<<(unsigned)((32 * nt + 255) / 256), 256, 0, s>>>(p, off, src, wq, wd);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

#define WBFMM_TL_INST(T, H)                                                                  \
  template int tl_fill<T, H>(const EvalParams<T>&, const int64_t*, uint32_t*, T*, T*, T*,    \
                             cudaStream_t);                                                  \
  template int tl_apply<T, H>(const EvalParams<T>&, const T*, const int64_t*, const uint32_t*, \
                              const T*, const T*, cudaStream_t);
WBFMM_TL_INST(double, true)
WBFMM_TL_INST(double, false)
WBFMM_TL_INST(float, true)
WBFMM_TL_INST(float, false)
template int tl_offsets<double>(const EvalParams<double>&, int64_t*, int64_t*, cudaStream_t);
template int tl_offsets<float>(const EvalParams<float>&, int64_t*, int64_t*, cudaStream_t);

}  // namespace wbfmm
