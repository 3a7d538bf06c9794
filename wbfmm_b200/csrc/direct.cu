// FP64 direct summation on the GPU: the GPU counterpart of the reference's
// wbfmm_total_field[_grad] (src/direct.c:35-294) and
// wbfmm_laplace_field[_grad] (src/direct-laplace.c:200-336), with explicit
// self-exclusion at r <= 1e-6 (WBFMM_LOCAL_CUTOFF_RADIUS, src/wbfmm.h:36)
// and compensated (two-sum) accumulation.  It is the accuracy reference the
// FMM forms are measured against.
#include <cuda_runtime.h>

#include <algorithm>

#include "../../include/wbfmm_b200.h"
#include "engine.h"

namespace wbfmm {

struct KS {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v) {
    double t = s + v;
    if (fabs(s) >= fabs(v)) c += (s - t) + v; else c += (v - t) + s;
    s = t;
  }
  __device__ __forceinline__ double get() const { return s + c; }
};

constexpr int kDirTile = 128;

template <bool HELM>
__global__ void k_direct(double k, int ns, const double* __restrict__ xs,
                         const double* __restrict__ q,
                         const double* __restrict__ nrm,
                         const double* __restrict__ dip, int nt,
                         const double* __restrict__ xt,
                         double* __restrict__ pot, double* __restrict__ grad) {
  __shared__ double sx[kDirTile], sy[kDirTile], sz[kDirTile];
  __shared__ double sq[2 * kDirTile], sd[2 * kDirTile], sn[3 * kDirTile];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = t < nt;
  double x = 0, y = 0, z = 0;
  if (act) { x = xt[3 * t]; y = xt[3 * t + 1]; z = xt[3 * t + 2]; }
  KS a[8];
  const double f4 = 0.25 / kPi, rc2 = kCutoffRadius * kCutoffRadius;
  const int w = HELM ? 2 : 1;
  for (int base = 0; base < ns; base += kDirTile) {
    const int m = min(kDirTile, ns - base);
    __syncthreads();
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
      int s = base + i;
      sx[i] = xs[3 * s]; sy[i] = xs[3 * s + 1]; sz[i] = xs[3 * s + 2];
      for (int c = 0; c < w; c++) {
        sq[w * i + c] = q ? q[w * s + c] : 0.0;
        sd[w * i + c] = dip ? dip[w * s + c] : 0.0;
      }
      if (nrm) { sn[3 * i] = nrm[3 * s]; sn[3 * i + 1] = nrm[3 * s + 1]; sn[3 * i + 2] = nrm[3 * s + 2]; }
    }
    __syncthreads();
    if (!act) continue;
    for (int i = 0; i < m; i++) {
      const double rx = x - sx[i], ry = y - sy[i], rz = z - sz[i];
      const double r2 = rx * rx + ry * ry + rz * rz;
      if (!(r2 > rc2)) continue;
      const double r = sqrt(r2);
      if (HELM) {
        const double kr = k * r;
        double sn_, cs;
        sincos(kr, &sn_, &cs);
        const double h0r = sn_ / kr, h0i = -cs / kr;
        const double h1r = h0r / kr + h0i, h1i = h0i / kr - h0r;
        const double qr = sq[2 * i], qi = sq[2 * i + 1];
        if (pot) {
          double fr = (h0r * qr - h0i * qi) * f4, fi = (h0i * qr + h0r * qi) * f4;
          if (dip) {
            double nr = (rx * sn[3 * i] + ry * sn[3 * i + 1] + rz * sn[3 * i + 2]) / r;
            double dr = sd[2 * i] * nr, di = sd[2 * i + 1] * nr;
            fr -= k * (h1r * dr - h1i * di) * f4;
            fi -= k * (h1r * di + h1i * dr) * f4;
          }
          a[0].add(fr); a[1].add(fi);
        }
        if (grad) {
          const double ar = -k * (h1r * qr - h1i * qi) * f4 / r;
          const double ai = -k * (h1r * qi + h1i * qr) * f4 / r;
          double gr[3] = {ar * rx, ar * ry, ar * rz}, gi[3] = {ai * rx, ai * ry, ai * rz};
          if (dip) {
            const double rv[3] = {rx, ry, rz};
            const double nv[3] = {sn[3 * i], sn[3 * i + 1], sn[3 * i + 2]};
            const double nr = rx * nv[0] + ry * nv[1] + rz * nv[2];
            const double dpr = h0r - 2.0 * h1r / kr, dpi = h0i - 2.0 * h1i / kr;
            const double dr = sd[2 * i], di = sd[2 * i + 1];
            for (int c = 0; c < 3; c++) {
              double ur = dpr * k * nr * rv[c] / r2 + h1r * (nv[c] / r - nr * rv[c] / (r2 * r));
              double ui = dpi * k * nr * rv[c] / r2 + h1i * (nv[c] / r - nr * rv[c] / (r2 * r));
              gr[c] += -k * (ur * dr - ui * di) * f4;
              gi[c] += -k * (ur * di + ui * dr) * f4;
            }
          }
          for (int c = 0; c < 3; c++) { a[2 + 2 * c].add(gr[c]); a[3 + 2 * c].add(gi[c]); }
        }
      } else {
        const double g = f4 / r;
        const double qv = sq[i];
        if (pot) {
          double v = qv;
          if (dip) v += sd[i] * (rx * sn[3 * i] + ry * sn[3 * i + 1] + rz * sn[3 * i + 2]) / r2;
          a[0].add(v * g);
        }
        if (grad) {
          const double gq = -qv * g / r2;
          double gv[3] = {gq * rx, gq * ry, gq * rz};
          if (dip) {
            const double nv[3] = {sn[3 * i], sn[3 * i + 1], sn[3 * i + 2]};
            const double nr = rx * nv[0] + ry * nv[1] + rz * nv[2];
            const double ad = sd[i] * g / r2;
            const double rv[3] = {rx, ry, rz};
            for (int c = 0; c < 3; c++) gv[c] += ad * (nv[c] - 3.0 * nr * rv[c] / r2);
          }
          for (int c = 0; c < 3; c++) a[1 + c].add(gv[c]);
        }
      }
    }
  }
  if (!act) return;
  if (HELM) {
    if (pot) { pot[2 * t] = a[0].get(); pot[2 * t + 1] = a[1].get(); }
    if (grad) for (int c = 0; c < 6; c++) grad[6 * t + c] = a[2 + c].get();
  } else {
    if (pot) pot[t] = a[0].get();
    if (grad) for (int c = 0; c < 3; c++) grad[3 * t + c] = a[1 + c].get();
  }
}

}  // namespace wbfmm

using namespace wbfmm;

extern "C" int wbfmm_b200_direct(int problem, double k, int ns,
                                 const double* xs, const double* q,
                                 const double* normals, const double* dipoles,
                                 int nt, const double* xt, double* pot,
                                 double* grad, int on_device) {
  if (ns <= 0 || nt <= 0 || !xs || !xt)
    return set_error(WBFMM_B200_E_ARG, "bad direct-sum arguments");
  if (dipoles && !normals)
    return set_error(WBFMM_B200_E_ARG, "dipoles need normals");
  const bool helm = problem == WBFMM_B200_HELMHOLTZ;
  const int w = helm ? 2 : 1;
  cudaStream_t s;
  WBFMM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  double *dxs = nullptr, *dq = nullptr, *dn = nullptr, *dd = nullptr,
         *dxt = nullptr, *dp = nullptr, *dg = nullptr;
  int rc = 0;
  auto up = [&](const double* h, size_t n, double** d) -> int {
    if (!h) { *d = nullptr; return 0; }
    if (on_device) { *d = (double*)h; return 0; }
    WBFMM_CUDA(cudaMalloc(d, sizeof(double) * n));
    WBFMM_CUDA(cudaMemcpyAsync(*d, h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    return 0;
  };
  auto out = [&](double* h, size_t n, double** d) -> int {
    if (!h) { *d = nullptr; return 0; }
    if (on_device) { *d = h; return 0; }
    WBFMM_CUDA(cudaMalloc(d, sizeof(double) * n));
    return 0;
  };
  if (!rc) rc = up(xs, (size_t)3 * ns, &dxs);
  if (!rc) rc = up(q, (size_t)w * ns, &dq);
  if (!rc) rc = up(normals, (size_t)3 * ns, &dn);
  if (!rc) rc = up(dipoles, (size_t)w * ns, &dd);
  if (!rc) rc = up(xt, (size_t)3 * nt, &dxt);
  if (!rc) rc = out(pot, (size_t)w * nt, &dp);
  if (!rc) rc = out(grad, (size_t)3 * w * nt, &dg);
  if (!rc) {
    unsigned grid = (unsigned)((nt + kDirTile - 1) / kDirTile);
    if (helm)
      k_direct<true><<<grid, kDirTile, 0, s>>>(k, ns, dxs, dq, dn, dd, nt, dxt, dp, dg);
    else
      k_direct<false><<<grid, kDirTile, 0, s>>>(k, ns, dxs, dq, dn, dd, nt, dxt, dp, dg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  }
  if (!rc && !on_device) {
    if (pot) cudaMemcpyAsync(pot, dp, sizeof(double) * w * nt, cudaMemcpyDeviceToHost, s);
    if (grad) cudaMemcpyAsync(grad, dg, sizeof(double) * 3 * w * nt, cudaMemcpyDeviceToHost, s);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (!rc && e != cudaSuccess) rc = set_cuda_error(e, __FILE__, __LINE__);
  if (!on_device) {
    cudaFree(dxs); cudaFree(dq); cudaFree(dn); cudaFree(dd); cudaFree(dxt);
    cudaFree(dp); cudaFree(dg);
  }
  cudaStreamDestroy(s);
  return rc;
}

// ------------------------------------------------------------ Laplace curl
// curl of the vector potential A_k = sum q_k / (4 pi r) from the target
// gradients g_k of its three components: curl_i = e_ijk d_j A_k
namespace {
__global__ void k_curl_combine(const double* __restrict__ g, int nt, double* __restrict__ curl) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nt) return;
  const double* gx = g + 3 * (size_t)j;                 // grad A_x
  const double* gy = g + 3 * ((size_t)nt + j);          // grad A_y
  const double* gz = g + 3 * (2 * (size_t)nt + j);      // grad A_z
  curl[3 * (size_t)j] = gz[1] - gy[2];
  curl[3 * (size_t)j + 1] = gx[2] - gz[0];
  curl[3 * (size_t)j + 2] = gy[0] - gx[1];
}
}  // namespace

namespace wbfmm {
int launch_curl_combine(const double* g, int nt, double* curl, cudaStream_t s) {
  if (nt <= 0) return 0;
  k_curl_combine<<<(nt + 255) / 256, 256, 0, s>>>(g, nt, curl);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}
}  // namespace wbfmm

// ------------------------------------------------------------ error norms
// The accuracy reduction of a field f against a reference r (FP64): per
// block sums of (f - r)^2 and r^2 and maxima of |f - r| and |r| in a fixed
// order, then one block combines the partials in block order, so the
// result does not depend on scheduling.
namespace {
constexpr int kErrThreads = 256;
constexpr int kErrBlocks = 592;   // 4 per SM

__device__ void err_block_reduce(double v[4], double (*sm)[kErrThreads]) {
  const int t = threadIdx.x;
  for (int k = 0; k < 4; k++) sm[k][t] = v[k];
  __syncthreads();
  for (int s = kErrThreads / 2; s > 0; s >>= 1) {
    if (t < s) {
      sm[0][t] += sm[0][t + s];
      sm[1][t] += sm[1][t + s];
      sm[2][t] = fmax(sm[2][t], sm[2][t + s]);
      sm[3][t] = fmax(sm[3][t], sm[3][t + s]);
    }
    __syncthreads();
  }
  for (int k = 0; k < 4; k++) v[k] = sm[k][0];
}

__global__ void k_err_partial(const double* __restrict__ f, const double* __restrict__ r,
                              int64_t n, double* __restrict__ part) {
  __shared__ double sm[4][kErrThreads];
  double v[4] = {0, 0, 0, 0};
  for (int64_t i = (int64_t)blockIdx.x * kErrThreads + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * kErrThreads) {
    const double d = f[i] - r[i];
    v[0] = fma(d, d, v[0]);
    v[1] = fma(r[i], r[i], v[1]);
    v[2] = fmax(v[2], fabs(d));
    v[3] = fmax(v[3], fabs(r[i]));
  }
  err_block_reduce(v, sm);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; k++) part[4 * blockIdx.x + k] = v[k];
}

__global__ void k_err_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  __shared__ double sm[4][kErrThreads];
  double v[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < nb; b += kErrThreads) {
    v[0] += part[4 * b];
    v[1] += part[4 * b + 1];
    v[2] = fmax(v[2], part[4 * b + 2]);
    v[3] = fmax(v[3], part[4 * b + 3]);
  }
  err_block_reduce(v, sm);
  if (threadIdx.x == 0) {
    out[0] = sqrt(v[0]); out[1] = sqrt(v[1]); out[2] = v[2]; out[3] = v[3];
  }
}
}  // namespace

extern "C" int wbfmm_b200_error_norms(int64_t n, const double* f, const double* ref,
                                      int on_device, double* out4) {
  if (n < 0 || (n > 0 && (!f || !ref)) || !out4)
    return wbfmm::set_error(WBFMM_B200_E_ARG, "bad error-norm arguments");
  if (wbfmm_b200_device_count() < 1)
    return wbfmm::set_error(WBFMM_B200_E_NOGPU, "no CUDA device is available");
  cudaStream_t s;
  WBFMM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  const double *df = f, *dr = ref;
  double *buf = nullptr, *part = nullptr;
  const int nb = (int)std::min<int64_t>(kErrBlocks, std::max<int64_t>(1, (n + kErrThreads - 1) / kErrThreads));
  int rc = 0;
  cudaError_t e = cudaMallocAsync(&part, sizeof(double) * (4 * nb + 4), s);
  if (e == cudaSuccess && !on_device && n > 0) {
    e = cudaMallocAsync(&buf, sizeof(double) * 2 * n, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf, f, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(buf + n, ref, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    df = buf; dr = buf + n;
  }
  if (e == cudaSuccess) {
    k_err_partial<<<nb, kErrThreads, 0, s>>>(df, dr, n, part);
    k_err_final<<<1, kErrThreads, 0, s>>>(part, nb, part + 4 * nb);
    e = cudaMemcpyAsync(out4, part + 4 * nb, 4 * sizeof(double), cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) rc = wbfmm::set_cuda_error(e, __FILE__, __LINE__);
  if (buf) cudaFreeAsync(buf, s);
  if (part) cudaFreeAsync(part, s);
  cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  return rc;
}
