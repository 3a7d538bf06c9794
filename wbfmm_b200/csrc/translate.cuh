// Warp-cooperative translation primitives on shared-memory coefficient
// vectors: the point-and-shoot sequence of Gumerov & Duraiswami
// (rotate -> coaxial translate -> rotate back) that the reference applies
// in every M2M, M2L and L2L (src/rotations.c:419-593,
// src/rotations-laplace.c:35-216, src/translations.c:411-604,
// src/laplace.c:496-696).
//
// Vectors are interleaved complex.  Helmholtz ("full") vectors hold every
// (n, m), |m| <= n, at cidx(n,m).  Laplace ("half") vectors hold m >= 0 at
// hidx(n,m) = n(n+1)/2 + m; negative m is the conjugate.
//
// Rotation, as applied by wbfmm_rotate_H with angles (a, b):
//   out[n,nu] = e^{-i nu a} sum_m H_n^{nu,m} e^{i m b} in[n,m],
// with H_n^{nu,-m} = H_n^{-nu,m}.  A shift uses (a, b) = (ph, ch) forward
// and (ch, ph) back.  Each routine strides lane, lane+nl, ... over outputs.
#pragma once

#include "fmm_math.cuh"

namespace wbfmm {

HD int hidx(int n, int m) { return n * (n + 1) / 2 + m; }

// x * 2^e, exact (no overflow of an intermediate power)
HD float scale2(float x, int e) { return ldexpf(x, e); }
HD double scale2(double x, int e) { return ldexp(x, e); }
HD int nhalf(int p) { return (p + 1) * (p + 2) / 2; }

// degree of flattened full index c = n(n+1)+m
HD int full_degree(int c) {
  int n = (int)sqrt((double)c);
  while ((n + 1) * (n + 1) <= c) n++;
  while (n * n > c) n--;
  return n;
}
HD int half_degree(int c) {
  int n = (int)((sqrt(8.0 * c + 1.0) - 1.0) * 0.5);
  while ((n + 1) * (n + 2) / 2 <= c) n++;
  while (n * (n + 1) / 2 > c) n--;
  return n;
}

// ------------------------------------------------------------ phases
// v[n,m] *= e^{i m b}; e[j] = (cos jb, sin jb), j >= 0
template <typename T>
HD void phase_full(T* v, int N, const T* e, int lane, int nl) {
  for (int c = lane; c < (N + 1) * (N + 1); c += nl) {
    int n = full_degree(c), m = c - n * (n + 1);
    int am = m < 0 ? -m : m;
    T er = e[2 * am], ei = m < 0 ? -e[2 * am + 1] : e[2 * am + 1];
    T xr = v[2 * c], xi = v[2 * c + 1];
    v[2 * c] = xr * er - xi * ei;
    v[2 * c + 1] = xr * ei + xi * er;
  }
}
template <typename T>
HD void phase_half(T* v, int N, const T* e, int lane, int nl) {
  for (int c = lane; c < nhalf(N); c += nl) {
    int n = half_degree(c), m = c - n * (n + 1) / 2;
    T er = e[2 * m], ei = e[2 * m + 1];
    T xr = v[2 * c], xi = v[2 * c + 1];
    v[2 * c] = xr * er - xi * ei;
    v[2 * c + 1] = xr * ei + xi * er;
  }
}

// -------------------------------------------------------- H rotation
// out[n,nu] (+)= e^{-i nu a} sum_m H_n^{nu,m} in[n,m]   (in already phased)
template <typename T, typename TH, bool ACC>
HD void hsum_full(T* out, const T* in, int N, const TH* H, const T* ea,
                  int lane, int nl) {
  for (int c = lane; c < (N + 1) * (N + 1); c += nl) {
    int n = full_degree(c), nu = c - n * (n + 1);
    const T* row = in + 2 * n * (n + 1);     // in[n, m] at row[2m]
    T sr = T(0), si = T(0);
    // m = 0 .. n : H(nu, m, n); m = -1 .. -n : H(-nu, |m|, n)
    int bp = rot_idx(nu, 0, n), bm = rot_idx(-nu, 0, n);
    T h = (T)H[bp];
    sr += h * row[0]; si += h * row[1];
    for (int m = 1; m <= n; m++) {
      T hp = (T)H[bp + m], hm = (T)H[bm + m];
      sr += hp * row[2 * m] + hm * row[-2 * m];
      si += hp * row[2 * m + 1] + hm * row[-2 * m + 1];
    }
    int an = nu < 0 ? -nu : nu;
    T er = ea[2 * an], ei = nu < 0 ? ea[2 * an + 1] : -ea[2 * an + 1];
    T orr = sr * er - si * ei, oi = sr * ei + si * er;
    if (ACC) { out[2 * c] += orr; out[2 * c + 1] += oi; }
    else { out[2 * c] = orr; out[2 * c + 1] = oi; }
  }
}

// Laplace half vectors, wbfmm_laplace_rotate_H (src/rotations-laplace.c:35-110)
template <typename T, typename TH, bool ACC>
HD void hsum_half(T* out, const T* in, int N, const TH* H, const T* ea,
                  int lane, int nl) {
  for (int c = lane; c < nhalf(N); c += nl) {
    int n = half_degree(c), nu = c - n * (n + 1) / 2;
    const T* row = in + 2 * hidx(n, 0);
    int bp = rot_idx(nu, 0, n), bm = rot_idx(-nu, 0, n);
    T tr = (T)H[bp] * row[0], ti = T(0);
    for (int m = 1; m <= n; m++) {
      T hp = (T)H[bp + m], hm = (T)H[bm + m];
      tr += (hp + hm) * row[2 * m];
      ti += (hp - hm) * row[2 * m + 1];
    }
    T er = ea[2 * nu], ei = ea[2 * nu + 1];   // e^{-i nu a} = (er, -ei)
    T orr = er * tr + ei * ti, oi = er * ti - ei * tr;
    if (nu == 0) oi = T(0);
    if (ACC) { out[2 * c] += orr; out[2 * c + 1] += oi; }
    else { out[2 * c] = orr; out[2 * c + 1] = oi; }
  }
}

// ------------------------------------------------- coaxial (Helmholtz)
// out[n,m] = sum_{l=|m|}^{Ni} s (E|F)_{max,min}^{|m|} in[l,m], n <= No,
// s = (-1)^{n+l} when l < n (src/translations.c:411-604).  CPLX: complex
// table (S|R), else real (R|R).
template <typename T, typename TT, bool CPLX>
HD void coax_full(T* out, const T* in, int No, int Ni, const TT* tab,
                  int lane, int nl) {
  for (int c = lane; c < (No + 1) * (No + 1); c += nl) {
    int n = full_degree(c), m = c - n * (n + 1);
    int am = m < 0 ? -m : m;
    T sr = T(0), si = T(0);
    for (int l = am; l <= Ni; l++) {
      int ic = l >= n ? coax_idx(l, am, n) : coax_idx(n, am, l);
      T s = (l >= n || ((n + l) & 1) == 0) ? T(1) : T(-1);
      T xr = in[2 * cidx(l, m)], xi = in[2 * cidx(l, m) + 1];
      if (CPLX) {
        T tr = s * (T)tab[2 * ic], ti = s * (T)tab[2 * ic + 1];
        sr += tr * xr - ti * xi;
        si += ti * xr + tr * xi;
      } else {
        T tr = s * (T)tab[ic];
        sr += tr * xr;
        si += tr * xi;
      }
    }
    out[2 * c] = sr; out[2 * c + 1] = si;
  }
}

// --------------------------------------------------- coaxial (Laplace)
// Dense [n][nd][m] tables of dimension Lt+1.  tp[j] = t^j (j <= 2Lt+1).
// kind 0: S|R  out[n] = sum_{nd=m}^{Ni} SR(n,nd,m)/t^{n+nd+1} in[nd]
// kind 1: S|S  out[n] = sum_{nd=m}^{min(n,Ni)} SS(n,nd,m)(-t)^{n-nd} in[nd]
// kind 2: R|R  out[n] = sum_{nd=max(n,m)}^{Ni} RR(n,nd,m) t^{nd-n} in[nd]
// (src/laplace.c:496-696, src/shift-laplace.c:340-360, :675-700)
template <typename T, typename TT>
HD void coax_half(T* out, const T* in, int No, int Ni, const TT* tab, int Lt,
                  const T* tp, int kind, int lane, int nl) {
  const int Dm = Lt + 1;
  for (int c = lane; c < nhalf(No); c += nl) {
    int n = half_degree(c), m = c - n * (n + 1) / 2;
    T sr = T(0), si = T(0);
    int lo = m, hi = Ni;
    if (kind == 1 && hi > n) hi = n;
    if (kind == 2 && lo < n) lo = n;
    for (int nd = lo; nd <= hi; nd++) {
      T w = (T)tab[((int64_t)n * Dm + nd) * Dm + m];
      if (kind == 0) w /= tp[n + nd + 1];
      else if (kind == 1) w *= (((n - nd) & 1) ? -tp[n - nd] : tp[n - nd]);
      else w *= tp[nd - n];
      const T* x = in + 2 * hidx(nd, m);
      sr += w * x[0];
      si += w * x[1];
    }
    if (m == 0) si = T(0);
    out[2 * c] = sr; out[2 * c + 1] = si;
  }
}

}  // namespace wbfmm
