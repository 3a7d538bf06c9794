// Second derivatives of the Laplace field (the Hessian of the potential) at
// the targets, and from them the gradient of the curl of a vector potential
// (the reference's WBFMM_FIELD_CURL | WBFMM_FIELD_GRADIENT,
// src/local-laplace.c:752-1010 and :1229-1291).
//
// Far field: the derivative of a regular (local) expansion of degree N is a
// regular expansion of degree N - 1.  k_laplace_deriv forms, per leaf box,
// the coefficients of d/dx, d/dy and d/dz of the box's local expansion: the
// identities are those of the L2P gradient (l2p_laplace_grad: each
// coefficient (n, m) feeds the degree n - 1 harmonics of orders m - 1, m and
// m + 1), regrouped by the harmonic they multiply.  The gradient L2P of the
// derived expansions then gives the nine second derivatives.  Near field:
// second derivatives of 1/(4 pi r) summed over the sources of the 27
// neighbour boxes, as the reference's box_curl_gradient_evaluate
// (src/local-laplace.c:147-197) does for each source.
#include "engine.h"
#include "fmm_math.cuh"
#include "kernels.h"

namespace wbfmm {

namespace {

// add A r^n P_n^m cos(m ph) + B r^n P_n^m sin(m ph) to the real-packed
// expansion D (evaluated as D[n^2] r^n P_n^0 + 2 sum_m r^n P_n^m
// (D[id] cos - D[id+1] sin), src/local-laplace.c:333-398)
template <typename T>
__device__ __forceinline__ void add_term(T* D, int64_t b, int nco, int n, int m,
                                         T A, T B) {
  if (m > n) return;
  if (m == 0) {
    D[layout_off(b, n * n, nco)] += A;
    return;
  }
  const int id = lidx(n, m);
  D[layout_off(b, id, nco)] += A / T(2);
  D[layout_off(b, id + 1, nco)] -= B / T(2);
}

// one thread per box: Dx, Dy, Dz (degree N - 1, zeroed first) from L
// (degree N); Layout L, real-packed
template <typename T>
__global__ void k_laplace_deriv(const T* __restrict__ L, int N, int64_t nbox,
                                T* Dx, T* Dy, T* Dz) {
  const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbox) return;
  const int nci = ncoef(N), nco = ncoef(N - 1);
  for (int c = 0; c < nco; c++) {
    const int64_t o = layout_off(b, c, nco);
    Dx[o] = Dy[o] = Dz[o] = T(0);
  }
  const LapRecDirect<T> rec;
  for (int n = 1; n <= N; n++) {
    const int np = n - 1;
    {  // m = 0
      T am, a0, a1;
      rec.c(n, 0, &am, &a0, &a1);
      const T cr = L[layout_off(b, n * n, nci)];
      add_term(Dx, b, nco, np, 1, -cr * a1, T(0));
      add_term(Dy, b, nco, np, 1, T(0), -cr * a1);
      add_term(Dz, b, nco, np, 0, cr * a0, T(0));
    }
    for (int m = 1; m <= n; m++) {
      T am, a0, ap;
      rec.c(n, m, &am, &a0, &ap);
      const int id = lidx(n, m);
      const T cr = L[layout_off(b, id, nci)];
      const T ci = -L[layout_off(b, id + 1, nci)];
      add_term(Dx, b, nco, np, m + 1, -cr * ap, -ci * ap);
      add_term(Dx, b, nco, np, m - 1, cr * am, ci * am);
      add_term(Dy, b, nco, np, m + 1, ci * ap, -cr * ap);
      add_term(Dy, b, nco, np, m - 1, ci * am, -cr * am);
      add_term(Dz, b, nco, np, m, T(2) * cr * a0, T(2) * ci * a0);
    }
  }
}

// hess[9 t + 3 a + b] = g[a][3 t + b]  (original target order)
template <typename T>
__global__ void k_hess_gather(const T* __restrict__ g, int nt, double* hess) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 9 * (int64_t)nt) return;
  const int64_t t = i / 9;
  const int r = (int)(i - 9 * t), a = r / 3, c = r - 3 * a;
  hess[i] = g ? (double)g[(int64_t)a * 3 * nt + 3 * t + c] : 0.0;
}

// near field: one thread per target (leaf-box order); adds into hess
template <typename T>
__global__ void k_p2p_hessian(EvalParams<T> p, double* hess) {
  const int jt = blockIdx.x * blockDim.x + threadIdx.x;
  if (jt >= p.ntgt) return;
  const uint64_t b = p.tbox[jt];
  uint32_t bi, bj, bk;
  demorton(b, &bi, &bj, &bk);
  const int64_t n1 = ((int64_t)1 << p.level) - 1;
  const double x = p.tx[jt], y = p.ty[jt], z = p.tz[jt];
  const double c4 = 1.0 / (4.0 * kPi);
  double h[6] = {0, 0, 0, 0, 0, 0};   // xx yy zz xy yz zx
  for (int di = -1; di <= 1; di++)
    for (int dj = -1; dj <= 1; dj++)
      for (int dk = -1; dk <= 1; dk++) {
        const int64_t i = (int64_t)bi + di, j = (int64_t)bj + dj, k = (int64_t)bk + dk;
        if (i < 0 || j < 0 || k < 0 || i > n1 || j > n1 || k > n1) continue;
        const uint64_t nb = morton((uint32_t)i, (uint32_t)j, (uint32_t)k);
        const uint32_t s0 = p.box_i[nb], s1 = s0 + p.box_n[nb];
        for (uint32_t s = s0; s < s1; s++) {
          const double dx = x - p.x[s], dy = y - p.y[s], dz = z - p.z[s];
          const double r2 = dx * dx + dy * dy + dz * dz;
          if (!(r2 > kCutoffRadius * kCutoffRadius)) continue;
          const double r = sqrt(r2), r3 = r2 * r, r5 = r3 * r2;
          const double q = (double)p.q[s] * c4;
          const double a = 3.0 * q / r5, d = q / r3;
          h[0] += a * dx * dx - d;
          h[1] += a * dy * dy - d;
          h[2] += a * dz * dz - d;
          h[3] += a * dx * dy;
          h[4] += a * dy * dz;
          h[5] += a * dz * dx;
        }
      }
  double* o = hess + 9 * (size_t)p.tperm[jt];
  o[0] += h[0]; o[1] += h[3]; o[2] += h[5];
  o[3] += h[3]; o[4] += h[1]; o[5] += h[4];
  o[6] += h[5]; o[7] += h[4]; o[8] += h[2];
}

// out[12 t ...] = curl (3), then d/dx, d/dy, d/dz of the curl's three
// components, from the gradients g[c][3 t + j] and Hessians h[c][9 t + 3 j
// + l] of the vector potential's components c
__global__ void k_curl_gradient_combine(const double* __restrict__ g,
                                        const double* __restrict__ h, int nt,
                                        double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  // d_j A_c
  auto G = [&](int c, int j) { return g[(size_t)c * 3 * nt + 3 * (size_t)t + j]; };
  // d_j d_l A_c
  auto H = [&](int c, int j, int l) { return h[(size_t)c * 9 * nt + 9 * (size_t)t + 3 * j + l]; };
  double* o = out + 12 * (size_t)t;
  o[0] = G(2, 1) - G(1, 2);
  o[1] = G(0, 2) - G(2, 0);
  o[2] = G(1, 0) - G(0, 1);
  for (int j = 0; j < 3; j++) {
    o[3 + 3 * j + 0] = H(2, j, 1) - H(1, j, 2);
    o[3 + 3 * j + 1] = H(0, j, 2) - H(2, j, 0);
    o[3 + 3 * j + 2] = H(1, j, 0) - H(0, j, 1);
  }
}

}  // namespace

template <typename T>
int launch_laplace_deriv(const T* L, int N, int64_t nbox, T* Dx, T* Dy, T* Dz,
                         cudaStream_t s) {
  if (nbox <= 0 || N < 1) return 0;
  k_laplace_deriv<T><<<(unsigned)((nbox + 127) / 128), 128, 0, s>>>(L, N, nbox, Dx, Dy, Dz);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

template <typename T>
int launch_hess_gather(const T* g, int nt, double* hess, cudaStream_t s) {
  if (nt <= 0) return 0;
  const int64_t n = 9 * (int64_t)nt;
  k_hess_gather<T><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(g, nt, hess);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

template <typename T>
int launch_p2p_hessian(const EvalParams<T>& p, double* hess, cudaStream_t s) {
  if (p.ntgt <= 0 || !p.q) return 0;
  k_p2p_hessian<T><<<(p.ntgt + 127) / 128, 128, 0, s>>>(p, hess);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

int launch_curl_gradient_combine(const double* g, const double* h, int nt, double* out,
                                 cudaStream_t s) {
  if (nt <= 0) return 0;
  k_curl_gradient_combine<<<(nt + 127) / 128, 128, 0, s>>>(g, h, nt, out);
  WBFMM_CUDA(cudaGetLastError());
  return 0;
}

#define WBFMM_HESS_INST(T)                                                         \
  template int launch_laplace_deriv<T>(const T*, int, int64_t, T*, T*, T*, cudaStream_t); \
  template int launch_hess_gather<T>(const T*, int, double*, cudaStream_t);        \
  template int launch_p2p_hessian<T>(const EvalParams<T>&, double*, cudaStream_t);
WBFMM_HESS_INST(double)
WBFMM_HESS_INST(float)

}  // namespace wbfmm
