// Per-point expansion primitives: P2M (leaf expansion of one source) and
// L2P (field and gradient of a regular expansion at one target).  Written
// once as __host__ __device__ code; the kernels in kernels.cu call them one
// point per lane/thread.
//
// P2M routines generate their coefficient contributions in a fixed order
// that depends only on the expansion order, through an `emit(index, re, im)`
// callback; the warp kernels reduce each emission across lanes, so the
// lanes of a warp must (and do) follow the same sequence.
#pragma once

#include "fmm_math.cuh"

namespace wbfmm {

constexpr int kPtMax = 66;   // per-point scratch: degree <= 64

// --------------------------------------------------- Helmholtz monopole
// C_n^m += q j_n(kr) P_n^{|m|}(cos th) e^{-i m ph}
// (src/expansions.c:30-123; an order-1 expansion keeps only n = 0 there)
template <typename T, class Emit, class Leg = LegDirect<T>>
HD void p2m_helmholtz(int N, T k, const T* xc, const T* xs, T qr, T qi,
                      Emit&& emit, const Leg& leg = Leg()) {
  if (N == 0) return;
  T Pa[kPtMax], Pb[kPtMax], Cm[kPtMax], Sm[kPtMax];
  T r, th, ph;
  cart2sph(xc, xs, &r, &th, &ph);
  T C = cos(th), S = sin(th), kr = k * r;
  T jm, j;
  bessel_j_init(kr, &jm, &j);
  T* pm = Pa; T* pn = Pb;
  for (int i = 0; i < N + 3 && i < kPtMax; i++) Pa[i] = Pb[i] = T(0);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  Cm[0] = T(1); Sm[0] = T(0); Cm[1] = cos(ph); Sm[1] = sin(ph);
  auto term = [&](int n, int m, int sgn, T jn, const T* P) {
    T a = jn * P[m];
    emit(cidx(n, sgn * m), a * (qr * Cm[m] + sgn * qi * Sm[m]),
         a * (qi * Cm[m] - sgn * qr * Sm[m]));
  };
  term(0, 0, 1, jm, pm);
  if (N == 1) return;
  term(1, 0, 1, j, pn);
  term(1, 1, 1, j, pn);
  term(1, 1, -1, j, pn);
  for (int n = 2; n <= N; n++) {
    legendre_step(pm, pn, n - 1, C, S, leg);
    T* t = pm; pm = pn; pn = t;
    bessel_j_step(&jm, &j, kr, n - 1);
    Cm[n] = Cm[n - 1] * Cm[1] - Sm[n - 1] * Sm[1];
    Sm[n] = Sm[n - 1] * Cm[1] + Cm[n - 1] * Sm[1];
    term(n, 0, 1, j, pn);
    for (int m = 1; m <= n; m++) {
      term(n, m, 1, j, pn);
      term(n, m, -1, j, pn);
    }
  }
}

// ---------------------------------------------------- Helmholtz dipole
// Dipole of complex strength d along the unit normal nrm, through the
// derivative relations G&D (3.2)-(3.7); regular terms of degree n >= N are
// not propagated, as in the reference (src/expansions.c:346-631).
template <typename T, class Emit, class Leg = LegDirect<T>>
HD void p2m_helmholtz_dipole(int N, T k, const T* xc, const T* xs,
                             const T* nrm, T dr, T di, Emit&& emit,
                             const Leg& leg = Leg()) {
  T Pa[kPtMax], Pb[kPtMax], Cm[kPtMax], Sm[kPtMax];
  T fm[2], fp[2], fz[2];
  fm[0] = T(0.5) * k * (dr * nrm[0] + di * nrm[1]);
  fm[1] = T(0.5) * k * (di * nrm[0] - dr * nrm[1]);
  fp[0] = T(0.5) * k * (dr * nrm[0] - di * nrm[1]);
  fp[1] = T(0.5) * k * (di * nrm[0] + dr * nrm[1]);
  fz[0] = k * dr * nrm[2];
  fz[1] = k * di * nrm[2];
  T r, th, ph;
  cart2sph(xc, xs, &r, &th, &ph);
  T C = cos(th), S = sin(th), kr = k * r;
  T jm, j;
  bessel_j_init(kr, &jm, &j);
  T* pm = Pa; T* pn = Pb;
  for (int i = 0; i < N + 3 && i < kPtMax; i++) Pa[i] = Pb[i] = T(0);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  Cm[0] = T(1); Sm[0] = T(0); Cm[1] = cos(ph); Sm[1] = sin(ph);
  // contribution w * R * f e^{-i sgn m ph} to coefficient (nn, mm)
  auto put = [&](int nn, int mm, T w, T R, const T* f, int m, int sgn) {
    if (nn < 0 || mm > nn || mm < -nn || w == T(0)) return;
    T er = f[0] * Cm[m] + sgn * f[1] * Sm[m];
    T ei = f[1] * Cm[m] - sgn * f[0] * Sm[m];
    emit(cidx(nn, mm), w * R * er, w * R * ei);
  };
  auto inc = [&](int n, int m, int sgn, T jn, const T* P) {
    if (n >= N) return;
    T R = jn * P[m];
    int sm = sgn * m;
    put(n - 1, sm + 1, -rec_b<T>(n, sm), R, fm, m, sgn);
    put(n - 1, sm - 1, -rec_b<T>(n, -sm), R, fp, m, sgn);
    put(n - 1, sm, rec_a<T>(n - 1, sm), R, fz, m, sgn);
    put(n + 1, sm + 1, rec_b<T>(n + 1, -sm - 1), R, fm, m, sgn);
    put(n + 1, sm - 1, rec_b<T>(n + 1, sm - 1), R, fp, m, sgn);
    put(n + 1, sm, -rec_a<T>(n, sm), R, fz, m, sgn);
  };
  inc(0, 0, 1, jm, pm);
  inc(1, 0, 1, j, pn);
  inc(1, 1, 1, j, pn);
  inc(1, 1, -1, j, pn);
  for (int n = 2; n <= N; n++) {
    legendre_step(pm, pn, n - 1, C, S, leg);
    T* t = pm; pm = pn; pn = t;
    bessel_j_step(&jm, &j, kr, n - 1);
    Cm[n] = Cm[n - 1] * Cm[1] - Sm[n - 1] * Sm[1];
    Sm[n] = Sm[n - 1] * Cm[1] + Cm[n - 1] * Sm[1];
    inc(n, 0, 1, j, pn);
    for (int m = 1; m <= n; m++) {
      inc(n, m, 1, j, pn);
      inc(n, m, -1, j, pn);
    }
  }
}

// ----------------------------------------------------- Laplace monopole
// M_n^m += q r^n P_n^m(cos th) e^{-i m ph} / (2n+1), real-packed
// (src/laplace.c:35-129); emit(index, value) per real slot
template <typename T, class Emit, class Leg = LegDirect<T>>
HD void p2m_laplace(int N, const T* xc, const T* xs, T q, Emit&& emit,
                    const Leg& leg = Leg()) {
  if (N == 0) return;
  T Pa[kPtMax], Pb[kPtMax], Cm[kPtMax], Sm[kPtMax];
  T r, th, ph;
  cart2sph(xc, xs, &r, &th, &ph);
  T C = cos(th), S = sin(th);
  T* pm = Pa; T* pn = Pb;
  for (int i = 0; i < N + 3 && i < kPtMax; i++) Pa[i] = Pb[i] = T(0);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  Cm[0] = T(1); Cm[1] = cos(ph); Sm[0] = T(0); Sm[1] = sin(ph);
  T rn = T(1);
  emit(0, q * rn * pm[0] / T(1));
  rn = r;
  emit(1, q * rn * pn[0] / T(3));
  emit(lidx(1, 1), q * rn * pn[1] * Cm[1] / T(3));
  emit(lidx(1, 1) + 1, -(q * rn * pn[1] * Sm[1] / T(3)));
  for (int n = 2; n <= N; n++) {
    rn *= r;
    legendre_step(pm, pn, n - 1, C, S, leg);
    T* t = pm; pm = pn; pn = t;
    Cm[n] = Cm[n - 1] * Cm[1] - Sm[n - 1] * Sm[1];
    Sm[n] = Sm[n - 1] * Cm[1] + Cm[n - 1] * Sm[1];
    T inv = T(1) / (T)(2 * n + 1);
    emit(n * n, q * rn * pn[0] * inv);
    for (int m = 1; m <= n; m++) {
      int id = lidx(n, m);
      emit(id, q * rn * pn[m] * Cm[m] * inv);
      emit(id + 1, -(q * rn * pn[m] * Sm[m] * inv));
    }
  }
}

// ------------------------------------------------------- Laplace dipole
// Dipole of strength d along the unit normal (src/laplace.c:181-423)
template <typename T, class Emit, class Leg = LegDirect<T>>
HD void p2m_laplace_dipole(int N, const T* xc, const T* xs, const T* nrm,
                           T d, Emit&& emit, const Leg& leg = Leg()) {
  if (N == 0) return;
  T Pa[kPtMax], Pb[kPtMax], Cm[kPtMax], Sm[kPtMax];
  T fx = nrm[0] * d, fy = nrm[1] * d, fz = nrm[2] * d;
  T r, th, ph;
  cart2sph(xc, xs, &r, &th, &ph);
  T C = cos(th), S = sin(th);
  T* pm = Pa; T* pn = Pb;
  for (int i = 0; i < N + 3 && i < kPtMax; i++) Pa[i] = Pb[i] = T(0);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  Cm[0] = T(1); Cm[1] = cos(ph); Sm[0] = T(0); Sm[1] = sin(ph);
  auto weights = [](int n, int m, T* a0, T* a1, T* a2) {
    T f = (T)(2 * n + 1) / (T)(2 * n + 3);
    *a0 = sqrt(f * (T)(n + m + 1) * (T)(n + m + 2));
    *a1 = -sqrt(f * (T)(n - m + 1) * (T)(n - m + 2));
    *a2 = sqrt(((T)(n + 1) * (T)(n + 1) - (T)(m * m)) * (T)(2 * n + 1) /
               (T)(2 * n + 3));
  };
  auto inc_m0 = [&](int n, T rn, const T* P) {
    T R = rn * P[0] / (T)(2 * n + 1), a0, a1, a2;
    weights(n, 0, &a0, &a1, &a2);
    int ip = lidx(n + 1, 1), i0 = (n + 1) * (n + 1);
    emit(ip, fx * T(0.5) * a0 * R * Cm[0] - fy * T(0.5) * a0 * R * Sm[0]);
    emit(ip + 1, -(fx * T(0.5) * a0 * R * Sm[0]) - fy * T(0.5) * a0 * R * Cm[0]);
    emit(i0, fz * a2 * R);
  };
  auto inc_m1 = [&](int n, T rn, const T* P) {
    const int m = 1;
    T R = rn * P[m] / (T)(2 * n + 1), a0, a1, a2;
    weights(n, m, &a0, &a1, &a2);
    int ip = lidx(n + 1, m + 1), i0 = (n + 1) * (n + 1), id = lidx(n + 1, m);
    emit(ip, fx * T(0.5) * a0 * R * Cm[m] - fy * T(0.5) * a0 * R * Sm[m]);
    emit(ip + 1, -(fx * T(0.5) * a0 * R * Sm[m]) - fy * T(0.5) * a0 * R * Cm[m]);
    emit(i0, fx * a1 * R * Cm[m] + fy * a1 * R * Sm[m]);
    emit(id, fz * a2 * R * Cm[m]);
    emit(id + 1, -(fz * a2 * R * Sm[m]));
  };
  auto inc = [&](int n, int m, T rn, const T* P) {
    T R = rn * P[m] / (T)(2 * n + 1), a0, a1, a2;
    weights(n, m, &a0, &a1, &a2);
    int ip = lidx(n + 1, m + 1), im = lidx(n + 1, m - 1), id = lidx(n + 1, m);
    emit(ip, fx * T(0.5) * a0 * R * Cm[m] - fy * T(0.5) * a0 * R * Sm[m]);
    emit(ip + 1, -(fx * T(0.5) * a0 * R * Sm[m]) - fy * T(0.5) * a0 * R * Cm[m]);
    emit(im, fx * T(0.5) * a1 * R * Cm[m] + fy * T(0.5) * a1 * R * Sm[m]);
    emit(im + 1, -(fx * T(0.5) * a1 * R * Sm[m]) + fy * T(0.5) * a1 * R * Cm[m]);
    emit(id, fz * a2 * R * Cm[m]);
    emit(id + 1, -(fz * a2 * R * Sm[m]));
  };
  T rn = T(1);
  inc_m0(0, rn, pm);
  if (N == 1) return;
  rn *= r;
  Cm[2] = Cm[1] * Cm[1] - Sm[1] * Sm[1];
  Sm[2] = Sm[1] * Cm[1] + Cm[1] * Sm[1];
  inc_m0(1, rn, pn);
  inc_m1(1, rn, pn);
  if (N == 2) return;
  for (int n = 2; n < N; n++) {
    rn *= r;
    legendre_step(pm, pn, n - 1, C, S, leg);
    T* t = pm; pm = pn; pn = t;
    Cm[n + 1] = Cm[n] * Cm[1] - Sm[n] * Sm[1];
    Sm[n + 1] = Sm[n] * Cm[1] + Cm[n] * Sm[1];
    inc_m0(n, rn, pn);
    inc_m1(n, rn, pn);
    for (int m = 2; m <= n; m++) inc(n, m, rn, pn);
  }
}

// ---------------------------------------------------- Helmholtz L2P
// f += sum C_n^m j_n(kr) P_n^{|m|} e^{i m ph}   (src/expansions.c:230-344)
// coef(idx) returns coefficient idx as (re, im)
template <typename T, class Coef, class Leg = LegDirect<T>>
HD void l2p_helmholtz(int N, T k, const T* xc, const T* xf, Coef&& coef,
                      T* fr, T* fi, const Leg& leg = Leg()) {
  T Pa[kPtMax], Pb[kPtMax], Cm[kPtMax], Sm[kPtMax];
  T r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  T C = cos(th), S = sin(th), kr = k * r;
  T jm, j;
  bessel_j_init(kr, &jm, &j);
  T* pm = Pa; T* pn = Pb;
  for (int i = 0; i < N + 3 && i < kPtMax; i++) Pa[i] = Pb[i] = T(0);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  Cm[0] = T(1); Sm[0] = T(0); Cm[1] = cos(ph); Sm[1] = sin(ph);
  T sr = T(0), si = T(0);
  auto inc0 = [&](int n, T jn, const T* P) {
    T a, b;
    coef(cidx(n, 0), &a, &b);
    T w = Cm[0] * jn * P[0];
    sr += a * w; si += b * w;
  };
  auto inc = [&](int n, int m, T jn, const T* P) {
    T ar, ai, br, bi;
    coef(cidx(n, m), &ar, &ai);
    coef(cidx(n, -m), &br, &bi);
    T wc = jn * P[m] * Cm[m], ws = jn * P[m] * Sm[m];
    sr += wc * (ar + br) - ws * (ai - bi);
    si += wc * (ai + bi) + ws * (ar - br);
  };
  inc0(0, jm, pm);
  inc0(1, j, pn);
  inc(1, 1, j, pn);
  for (int n = 2; n <= N; n++) {
    legendre_step(pm, pn, n - 1, C, S, leg);
    T* t = pm; pm = pn; pn = t;
    bessel_j_step(&jm, &j, kr, n - 1);
    Cm[n] = Cm[n - 1] * Cm[1] - Sm[n - 1] * Sm[1];
    Sm[n] = Sm[n - 1] * Cm[1] + Cm[n - 1] * Sm[1];
    inc0(n, j, pn);
    for (int m = 1; m <= n; m++) inc(n, m, j, pn);
  }
  *fr += sr; *fi += si;
}

// gradient of the regular expansion, G&D (2004) (3.7)
// (src/gradient.c:193-399); g[0..5] += (dx re, dx im, dy re, dy im, dz re, dz im)
// pot (optional): the potential of l2p_helmholtz added in the same sweep
template <typename T, class Coef, class Rec = RecDirect<T>, class Leg = LegDirect<T>>
HD void l2p_helmholtz_grad(int N, T k, const T* xc, const T* xf, Coef&& coef,
                           T* g, T* pot = nullptr, const Rec& rec = Rec(),
                           const Leg& leg = Leg()) {
  T Pm1[kPtMax], Pa[kPtMax], Pb[kPtMax], Cm[kPtMax + 1], Sm[kPtMax + 1];
  T r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  T C = cos(th), S = sin(th), Cph = cos(ph), Sph = sin(ph), kr = k * r;
  T jn, jnp1, jnm1;
  for (int i = 0; i < N + 4 && i < kPtMax; i++) Pm1[i] = Pa[i] = Pb[i] = T(0);
  bessel_j_init(kr, &jn, &jnp1);
  T* pn = Pa; T* pnp1 = Pb;
  legendre_init(C, S, &pn[0], &pnp1[0], &pnp1[1]);
  Cm[0] = T(1); Sm[0] = T(0); Cm[1] = Cph; Sm[1] = Sph;
  jnm1 = T(0);
  T acc[6] = {T(0), T(0), T(0), T(0), T(0), T(0)};
  T pr = T(0), pi = T(0);
  auto inc = [&](int n, int m, int sgn, T cm1, T sm1, T cmm, T smm, T cp1,
                 T sp1) {
    T tm = k * jnm1, tp = k * jnp1;
    int mm1 = sgn * m - 1; mm1 = mm1 < 0 ? -mm1 : mm1;
    int mp1 = sgn * m + 1; mp1 = mp1 < 0 ? -mp1 : mp1;
    T c[6];
    T b1 = rec.b(n + 1, -sgn * m - 1) / T(2);
    T b2 = rec.b(n, sgn * m) / T(2);
    T u = b1 * tp * pnp1[mp1] - b2 * tm * Pm1[mp1];
    c[0] = c[4] = cp1 * u;
    c[1] = c[5] = sp1 * u;
    b1 = rec.b(n + 1, sgn * m - 1) / T(2);
    b2 = rec.b(n, -sgn * m) / T(2);
    u = b1 * tp * pnp1[mm1] - b2 * tm * Pm1[mm1];
    c[3] = cm1 * u;
    c[2] = -sm1 * u;
    c[0] += c[3]; c[1] -= c[2];
    c[2] += c[5]; c[3] -= c[4];
    T a1 = rec.a(n - 1, m), a2 = rec.a(n, m);
    u = a1 * tm * Pm1[m] - a2 * tp * pnp1[m];
    c[4] = cmm * u;
    c[5] = smm * u;
    T ar, ai;
    coef(cidx(n, sgn * m), &ar, &ai);
    acc[0] += c[0] * ar - c[1] * ai; acc[1] += c[0] * ai + c[1] * ar;
    acc[2] += c[2] * ar - c[3] * ai; acc[3] += c[2] * ai + c[3] * ar;
    acc[4] += c[4] * ar - c[5] * ai; acc[5] += c[4] * ai + c[5] * ar;
    if (pot) {   // j_n P_n^|m| e^(i sgn m ph) C_n^(sgn m)
      const T w = jn * pn[m];
      pr += w * (cmm * ar - smm * ai);
      pi += w * (cmm * ai + smm * ar);
    }
  };
  inc(0, 0, 1, Cm[1], -Sm[1], Cm[0], Sm[0], Cm[1], Sm[1]);
  jnm1 = jn;
  bessel_j_step(&jn, &jnp1, kr, 1);
  // n = 1
  Pm1[0] = pn[0]; Pm1[1] = pn[1];
  legendre_step(pn, pnp1, 1, C, S, leg);
  { T* t = pn; pn = pnp1; pnp1 = t; }
  Cm[2] = Cm[1] * Cph - Sm[1] * Sph;
  Sm[2] = Sm[1] * Cph + Cm[1] * Sph;
  inc(1, 0, 1, Cm[1], -Sm[1], Cm[0], Sm[0], Cm[1], Sm[1]);
  inc(1, 1, 1, Cm[0], Sm[0], Cm[1], Sm[1], Cm[2], Sm[2]);
  inc(1, 1, -1, Cm[2], -Sm[2], Cm[1], -Sm[1], Cm[0], -Sm[0]);
  for (int n = 2; n <= N; n++) {
    for (int i = 0; i <= n; i++) Pm1[i] = pn[i];
    legendre_step(pn, pnp1, n, C, S, leg);
    { T* t = pn; pn = pnp1; pnp1 = t; }
    jnm1 = jn;
    bessel_j_step(&jn, &jnp1, kr, n);
    Cm[n + 1] = Cm[n] * Cph - Sm[n] * Sph;
    Sm[n + 1] = Sm[n] * Cph + Cm[n] * Sph;
    inc(n, 0, 1, Cm[1], -Sm[1], Cm[0], Sm[0], Cm[1], Sm[1]);
    for (int m = 1; m <= n; m++) {
      inc(n, m, 1, Cm[m - 1], Sm[m - 1], Cm[m], Sm[m], Cm[m + 1], Sm[m + 1]);
      inc(n, m, -1, Cm[m + 1], -Sm[m + 1], Cm[m], -Sm[m], Cm[m - 1], -Sm[m - 1]);
    }
  }
  for (int i = 0; i < 6; i++) g[i] += acc[i];
  if (pot) { pot[0] += pr; pot[1] += pi; }
}

// ------------------------------------------------------- Laplace L2P
// f += L_n^0 r^n P_n^0 + 2 sum_{m>0} r^n P_n^m Re(L_n^m e^{i m ph})
// (src/local-laplace.c:333-398); coef(idx) returns real slot idx
template <typename T, class Coef, class Leg = LegDirect<T>>
HD T l2p_laplace(int N, const T* xc, const T* xf, Coef&& coef,
                 const Leg& leg = Leg()) {
  T Pa[kPtMax], Pb[kPtMax], Cm[kPtMax], Sm[kPtMax];
  T r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  T C = cos(th), S = sin(th);
  T* pm = Pa; T* pn = Pb;
  for (int i = 0; i < N + 3 && i < kPtMax; i++) Pa[i] = Pb[i] = T(0);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  Cm[0] = T(1); Cm[1] = cos(ph); Sm[0] = T(0); Sm[1] = sin(ph);
  T f = T(0), rn = T(1);
  f += coef(0) * rn * pm[0];
  rn *= r;
  f += coef(1) * rn * pn[0];
  f += T(2) * pn[1] * rn * (coef(lidx(1, 1)) * Cm[1] - coef(lidx(1, 1) + 1) * Sm[1]);
  for (int n = 2; n <= N; n++) {
    rn *= r;
    legendre_step(pm, pn, n - 1, C, S, leg);
    T* t = pm; pm = pn; pn = t;
    Cm[n] = Cm[n - 1] * Cm[1] - Sm[n - 1] * Sm[1];
    Sm[n] = Sm[n - 1] * Cm[1] + Cm[n - 1] * Sm[1];
    f += coef(n * n) * rn * pn[0];
    for (int m = 1; m <= n; m++) {
      int id = lidx(n, m);
      f += T(2) * pn[m] * rn * (coef(id) * Cm[m] - coef(id + 1) * Sm[m]);
    }
  }
  return f;
}

// gradient of the Laplace regular expansion via the derivatives of the
// solid harmonics (src/local-laplace.c:525-630, src/wbfmm-derivatives.h);
// pot (optional): the potential of l2p_laplace added in the same sweep
template <typename T, class Coef, class LRec = LapRecDirect<T>, class Leg = LegDirect<T>>
HD void l2p_laplace_grad(int N, const T* xc, const T* xf, Coef&& coef, T* g,
                         T* pot = nullptr, const LRec& rec = LRec(),
                         const Leg& leg = Leg()) {
  if (N == 0) return;
  T Pa[kPtMax], Pb[kPtMax], Cm[kPtMax + 1], Sm[kPtMax + 1];
  T r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  T C = cos(th), S = sin(th);
  T* pm = Pa; T* pn = Pb;
  for (int i = 0; i < N + 3 && i < kPtMax; i++) Pa[i] = Pb[i] = T(0);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  Cm[0] = T(1); Sm[0] = T(0); Cm[1] = cos(ph); Sm[1] = sin(ph);
  T gx = T(0), gy = T(0), gz = T(0), f = T(0);
  // degree n >= 2: P holds degree n-1 (gradient), Pn degree n (potential)
  auto d_m0 = [&](int n, T rnm1, const T* P, const T* Pn) {
    T am, a0, a1;
    rec.c(n, 0, &am, &a0, &a1);
    T R0 = rnm1 * P[0] * a0, R1 = rnm1 * P[1] * a1;
    T cr = coef(n * n);
    gx += cr * (-R1 * Cm[1]);
    gy += cr * (-R1 * Sm[1]);
    gz += cr * R0;
    if (pot) f += cr * rnm1 * r * Pn[0];
  };
  auto d_m = [&](int n, int m, T rnm1, const T* P, const T* Pn) {
    T am, a0, ap;
    rec.c(n, m, &am, &a0, &ap);
    T Rm = rnm1 * P[m - 1] * am, R0 = rnm1 * P[m] * a0 * T(2);
    T Rp = rnm1 * P[m + 1] * ap;
    T xr = -Rp * Cm[m + 1] + Rm * Cm[m - 1], xi = -Rp * Sm[m + 1] + Rm * Sm[m - 1];
    T yr = -Rp * Sm[m + 1] - Rm * Sm[m - 1], yi = Rp * Cm[m + 1] + Rm * Cm[m - 1];
    T zr = R0 * Cm[m], zi = R0 * Sm[m];
    int id = lidx(n, m);
    T cr = coef(id), ci = -coef(id + 1);
    gx += cr * xr + ci * xi;
    gy += cr * yr + ci * yi;
    gz += cr * zr + ci * zi;
    if (pot) f += T(2) * Pn[m] * rnm1 * r * (cr * Cm[m] + ci * Sm[m]);
  };
  T rnm1 = T(1);
  Cm[2] = Cm[1] * Cm[1] - Sm[1] * Sm[1];
  Sm[2] = Sm[1] * Cm[1] + Cm[1] * Sm[1];
  {  // n = 1, m = 0: only the z derivative is non-zero
    T R0 = rnm1 * pm[0] * sqrt(T(3));
    gz += coef(1) * R0;
    if (pot) f += coef(0) * pm[0] + coef(1) * r * pn[0];
  }
  d_m(1, 1, rnm1, pm, pn);
  for (int n = 2; n <= N; n++) {
    rnm1 *= r;
    legendre_step(pm, pn, n - 1, C, S, leg);
    T* t = pm; pm = pn; pn = t;       // pm now degree n-1, pn degree n
    Cm[n + 1] = Cm[n] * Cm[1] - Sm[n] * Sm[1];
    Sm[n + 1] = Sm[n] * Cm[1] + Cm[n] * Sm[1];
    d_m0(n, rnm1, pm, pn);
    for (int m = 1; m <= n; m++) d_m(n, m, rnm1, pm, pn);
  }
  g[0] += gx; g[1] += gy; g[2] += gz;
  if (pot) *pot += f;
}

}  // namespace wbfmm
