// Per-point expansion primitives: P2M (leaf expansion of one source) and
// L2P (field and gradient of a regular expansion at one target).  Written
// once as __host__ __device__ code; the kernels in kernels.cu call them one
// point per lane/thread.
//
// Per-point state: the Legendre rows of the recursion live in caller
// scratch (Scratch: per-thread slices of shared memory in the kernels, so
// that they stay out of local memory), rows of kRowPad + N entries, the
// number of rows given by p2m_rows / l2p_rows; cos(m ph), sin(m ph) are
// advanced in registers along m (the recurrence the reference applies to
// its arrays, so the same values); the spherical Bessel functions come
// from BesselJSeq.
//
// The P2M and Laplace L2P loops are marked for unrolling: with a
// compile-time order (the kernels' fixed-order instantiations, scratch rows
// in a per-thread array) every index becomes a constant and the rows stay
// in registers.  The Helmholtz L2P is not: unrolled at order 14 it needed
// 170-255 registers and ran slower.
//
// P2M routines generate their coefficient contributions in a fixed order
// that depends only on the expansion order, through an `emit(index, re, im)`
// callback; the warp kernels reduce each emission across lanes, so the
// lanes of a warp must (and do) follow the same sequence.  Two coefficients
// computed together (Helmholtz orders +m and -m, Laplace's cos and sin
// parts) go through the emitter's pair(...) where it has one (a warp
// reduction of several values at once), else one by one (emit_two).
#pragma once

#include "fmm_math.cuh"

namespace wbfmm {

constexpr int kPtMax = 66;   // degree <= 64
constexpr int kRowPad = 4;   // row length: N + kRowPad entries

// scratch rows of the P2M and L2P routines (gradient: L2P with grad)
HD int p2m_rows() { return 2; }
HD int l2p_rows(bool helm, bool grad) { return helm && grad ? 3 : 2; }

// zero rows 0..k-1 (entries 0..len-1)
template <typename T>
HD void zero_rows(const Scratch<T>& sc, int k) {
#pragma unroll
  for (int r = 0; r < k; r++) {
    Row<T> w = sc.row(r);
#pragma unroll
    for (int i = 0; i < sc.len; i++) w[i] = T(0);
  }
}

// two emissions: e.pair(...) when the emitter has it, else e(...) twice
template <class E, typename T>
HD auto emit_two(E& e, int i1, T r1, T m1, int i2, T r2, T m2, int)
    -> decltype(e.pair(i1, r1, m1, i2, r2, m2), void()) {
  e.pair(i1, r1, m1, i2, r2, m2);
}
template <class E, typename T>
HD void emit_two(E& e, int i1, T r1, T m1, int i2, T r2, T m2, long) {
  e(i1, r1, m1);
  e(i2, r2, m2);
}
template <class E, typename T>
HD auto emit_two(E& e, int i1, T v1, int i2, T v2, int)
    -> decltype(e.pair(i1, v1, i2, v2), void()) {
  e.pair(i1, v1, i2, v2);
}
template <class E, typename T>
HD void emit_two(E& e, int i1, T v1, int i2, T v2, long) {
  e(i1, v1);
  e(i2, v2);
}

// (cos, sin) of (m+1) ph from those of m ph and ph
template <typename T>
HD void rot_next(T c, T s, T c1, T s1, T* cn, T* sn) {
  *cn = c * c1 - s * s1;
  *sn = s * c1 + c * s1;
}

// --------------------------------------------------- Helmholtz monopole
// C_n^m += q j_n(kr) P_n^{|m|}(cos th) e^{-i m ph}
// (src/expansions.c:30-123; an order-1 expansion keeps only n = 0 there)
template <typename T, class Emit, class Leg = LegDirect<T>>
HD void p2m_helmholtz(int N, T k, const T* xc, const T* xs, T qr, T qi,
                      Emit&& emit, const Leg& leg, const Scratch<T>& sc) {
  if (N == 0) return;
  T r, th, ph;
  cart2sph(xc, xs, &r, &th, &ph);
  T C = cos(th), S = sin(th), kr = k * r;
  BesselJSeq<T> bj(kr);
  zero_rows(sc, 2);
  Row<T> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  const T c1 = cos(ph), s1 = sin(ph);
  auto term = [&](int n, int m, int sgn, T jn, T P, T cm, T smm) {
    T a = jn * P;
    emit(cidx(n, sgn * m), a * (qr * cm + sgn * qi * smm),
         a * (qi * cm - sgn * qr * smm));
  };
  // orders +m and -m together
  auto pair = [&](int n, int m, T jn, T P, T cm, T smm) {
    const T a = jn * P;
    emit_two(emit, cidx(n, m), a * (qr * cm + qi * smm), a * (qi * cm - qr * smm),
             cidx(n, -m), a * (qr * cm - qi * smm), a * (qi * cm + qr * smm), 0);
  };
  term(0, 0, 1, bj.jm, pm[0], T(1), T(0));
  if (N == 1) return;
  term(1, 0, 1, bj.j, pn[0], T(1), T(0));
  pair(1, 1, bj.j, pn[1], c1, s1);
#pragma unroll
  for (int n = 2; n <= N; n++) {
    legendre_step(pm, pn, n - 1, C, S, leg);
    Row<T> t = pm; pm = pn; pn = t;
    bj.step();
    term(n, 0, 1, bj.j, pn[0], T(1), T(0));
    T cm = T(1), smm = T(0);
#pragma unroll
    for (int m = 1; m <= n; m++) {
      rot_next(cm, smm, c1, s1, &cm, &smm);
      pair(n, m, bj.j, pn[m], cm, smm);
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
                             const Leg& leg, const Scratch<T>& sc) {
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
  BesselJSeq<T> bj(kr);
  zero_rows(sc, 2);
  Row<T> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  const T c1 = cos(ph), s1 = sin(ph);
  // contribution w * R * f e^{-i sgn m ph} to coefficient (nn, mm)
  auto put = [&](int nn, int mm, T w, T R, const T* f, T cm, T smm, int sgn) {
    if (nn < 0 || mm > nn || mm < -nn || w == T(0)) return;
    T er = f[0] * cm + sgn * f[1] * smm;
    T ei = f[1] * cm - sgn * f[0] * smm;
    emit(cidx(nn, mm), w * R * er, w * R * ei);
  };
  auto inc = [&](int n, int m, int sgn, T jn, T P, T cm, T smm) {
    if (n >= N) return;
    T R = jn * P;
    int sm = sgn * m;
    put(n - 1, sm + 1, -rec_b<T>(n, sm), R, fm, cm, smm, sgn);
    put(n - 1, sm - 1, -rec_b<T>(n, -sm), R, fp, cm, smm, sgn);
    put(n - 1, sm, rec_a<T>(n - 1, sm), R, fz, cm, smm, sgn);
    put(n + 1, sm + 1, rec_b<T>(n + 1, -sm - 1), R, fm, cm, smm, sgn);
    put(n + 1, sm - 1, rec_b<T>(n + 1, sm - 1), R, fp, cm, smm, sgn);
    put(n + 1, sm, -rec_a<T>(n, sm), R, fz, cm, smm, sgn);
  };
  inc(0, 0, 1, bj.jm, pm[0], T(1), T(0));
  inc(1, 0, 1, bj.j, pn[0], T(1), T(0));
  inc(1, 1, 1, bj.j, pn[1], c1, s1);
  inc(1, 1, -1, bj.j, pn[1], c1, s1);
#pragma unroll
  for (int n = 2; n <= N; n++) {
    legendre_step(pm, pn, n - 1, C, S, leg);
    Row<T> t = pm; pm = pn; pn = t;
    bj.step();
    inc(n, 0, 1, bj.j, pn[0], T(1), T(0));
    T cm = T(1), smm = T(0);
#pragma unroll
    for (int m = 1; m <= n; m++) {
      rot_next(cm, smm, c1, s1, &cm, &smm);
      const T P = pn[m];
      inc(n, m, 1, bj.j, P, cm, smm);
      inc(n, m, -1, bj.j, P, cm, smm);
    }
  }
}

// ----------------------------------------------------- Laplace monopole
// M_n^m += q r^n P_n^m(cos th) e^{-i m ph} / (2n+1), real-packed
// (src/laplace.c:35-129); emit(index, value) per real slot
template <typename T, class Emit, class Leg = LegDirect<T>>
HD void p2m_laplace(int N, const T* xc, const T* xs, T q, Emit&& emit,
                    const Leg& leg, const Scratch<T>& sc) {
  if (N == 0) return;
  T r, th, ph;
  cart2sph(xc, xs, &r, &th, &ph);
  T C = cos(th), S = sin(th);
  zero_rows(sc, 2);
  Row<T> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  const T c1 = cos(ph), s1 = sin(ph);
  T rn = T(1);
  emit(0, q * rn * pm[0] / T(1));
  rn = r;
  emit(1, q * rn * pn[0] / T(3));
  emit_two(emit, lidx(1, 1), q * rn * pn[1] * c1 / T(3), lidx(1, 1) + 1,
           -(q * rn * pn[1] * s1 / T(3)), 0);
#pragma unroll
  for (int n = 2; n <= N; n++) {
    rn *= r;
    legendre_step(pm, pn, n - 1, C, S, leg);
    Row<T> t = pm; pm = pn; pn = t;
    T inv = T(1) / (T)(2 * n + 1);
    emit(n * n, q * rn * pn[0] * inv);
    T cm = T(1), smm = T(0);
#pragma unroll
    for (int m = 1; m <= n; m++) {
      rot_next(cm, smm, c1, s1, &cm, &smm);
      const int id = lidx(n, m);
      const T P = pn[m];
      emit_two(emit, id, q * rn * P * cm * inv, id + 1, -(q * rn * P * smm * inv), 0);
    }
  }
}

// ------------------------------------------------------- Laplace dipole
// Dipole of strength d along the unit normal (src/laplace.c:181-423)
template <typename T, class Emit, class Leg = LegDirect<T>>
HD void p2m_laplace_dipole(int N, const T* xc, const T* xs, const T* nrm,
                           T d, Emit&& emit, const Leg& leg,
                           const Scratch<T>& sc) {
  if (N == 0) return;
  T fx = nrm[0] * d, fy = nrm[1] * d, fz = nrm[2] * d;
  T r, th, ph;
  cart2sph(xc, xs, &r, &th, &ph);
  T C = cos(th), S = sin(th);
  zero_rows(sc, 2);
  Row<T> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  const T c1 = cos(ph), s1 = sin(ph);
  auto weights = [](int n, int m, T* a0, T* a1, T* a2) {
    T f = (T)(2 * n + 1) / (T)(2 * n + 3);
    *a0 = sqrt(f * (T)(n + m + 1) * (T)(n + m + 2));
    *a1 = -sqrt(f * (T)(n - m + 1) * (T)(n - m + 2));
    *a2 = sqrt(((T)(n + 1) * (T)(n + 1) - (T)(m * m)) * (T)(2 * n + 1) /
               (T)(2 * n + 3));
  };
  auto inc_m0 = [&](int n, T rn, T P0) {
    T R = rn * P0 / (T)(2 * n + 1), a0, a1, a2;
    weights(n, 0, &a0, &a1, &a2);
    int ip = lidx(n + 1, 1), i0 = (n + 1) * (n + 1);
    const T cm = T(1), smm = T(0);
    emit(ip, fx * T(0.5) * a0 * R * cm - fy * T(0.5) * a0 * R * smm);
    emit(ip + 1, -(fx * T(0.5) * a0 * R * smm) - fy * T(0.5) * a0 * R * cm);
    emit(i0, fz * a2 * R);
  };
  auto inc_m1 = [&](int n, T rn, T P1) {
    const int m = 1;
    T R = rn * P1 / (T)(2 * n + 1), a0, a1, a2;
    weights(n, m, &a0, &a1, &a2);
    int ip = lidx(n + 1, m + 1), i0 = (n + 1) * (n + 1), id = lidx(n + 1, m);
    emit(ip, fx * T(0.5) * a0 * R * c1 - fy * T(0.5) * a0 * R * s1);
    emit(ip + 1, -(fx * T(0.5) * a0 * R * s1) - fy * T(0.5) * a0 * R * c1);
    emit(i0, fx * a1 * R * c1 + fy * a1 * R * s1);
    emit(id, fz * a2 * R * c1);
    emit(id + 1, -(fz * a2 * R * s1));
  };
  auto inc = [&](int n, int m, T rn, T P, T cm, T smm) {
    T R = rn * P / (T)(2 * n + 1), a0, a1, a2;
    weights(n, m, &a0, &a1, &a2);
    int ip = lidx(n + 1, m + 1), im = lidx(n + 1, m - 1), id = lidx(n + 1, m);
    emit(ip, fx * T(0.5) * a0 * R * cm - fy * T(0.5) * a0 * R * smm);
    emit(ip + 1, -(fx * T(0.5) * a0 * R * smm) - fy * T(0.5) * a0 * R * cm);
    emit(im, fx * T(0.5) * a1 * R * cm + fy * T(0.5) * a1 * R * smm);
    emit(im + 1, -(fx * T(0.5) * a1 * R * smm) + fy * T(0.5) * a1 * R * cm);
    emit(id, fz * a2 * R * cm);
    emit(id + 1, -(fz * a2 * R * smm));
  };
  T rn = T(1);
  inc_m0(0, rn, pm[0]);
  if (N == 1) return;
  rn *= r;
  inc_m0(1, rn, pn[0]);
  inc_m1(1, rn, pn[1]);
  if (N == 2) return;
#pragma unroll
  for (int n = 2; n < N; n++) {
    rn *= r;
    legendre_step(pm, pn, n - 1, C, S, leg);
    Row<T> t = pm; pm = pn; pn = t;
    inc_m0(n, rn, pn[0]);
    inc_m1(n, rn, pn[1]);
    T cm = c1, smm = s1;
#pragma unroll
    for (int m = 2; m <= n; m++) {
      rot_next(cm, smm, c1, s1, &cm, &smm);
      inc(n, m, rn, pn[m], cm, smm);
    }
  }
}

// ---------------------------------------------------- Helmholtz L2P
// f += sum C_n^m j_n(kr) P_n^{|m|} e^{i m ph}   (src/expansions.c:230-344)
// coef(idx) returns coefficient idx as (re, im)
template <typename T, class Coef, class Leg = LegDirect<T>>
HD void l2p_helmholtz(int N, T k, const T* xc, const T* xf, Coef&& coef,
                      T* fr, T* fi, const Leg& leg, const Scratch<T>& sc) {
  T r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  T C = cos(th), S = sin(th), kr = k * r;
  BesselJSeq<T> bj(kr);
  zero_rows(sc, 2);
  Row<T> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  const T c1 = cos(ph), s1 = sin(ph);
  T sr = T(0), si = T(0);
  auto inc0 = [&](int n, T jn, T P0) {
    T a, b;
    coef(cidx(n, 0), &a, &b);
    T w = T(1) * jn * P0;
    sr += a * w; si += b * w;
  };
  auto inc = [&](int n, int m, T jn, T P, T cm, T smm) {
    T ar, ai, br, bi;
    coef(cidx(n, m), &ar, &ai);
    coef(cidx(n, -m), &br, &bi);
    T wc = jn * P * cm, ws = jn * P * smm;
    sr += wc * (ar + br) - ws * (ai - bi);
    si += wc * (ai + bi) + ws * (ar - br);
  };
  inc0(0, bj.jm, pm[0]);
  inc0(1, bj.j, pn[0]);
  inc(1, 1, bj.j, pn[1], c1, s1);
  for (int n = 2; n <= N; n++) {
    legendre_step(pm, pn, n - 1, C, S, leg);
    Row<T> t = pm; pm = pn; pn = t;
    bj.step();
    inc0(n, bj.j, pn[0]);
    T cm = T(1), smm = T(0);
    for (int m = 1; m <= n; m++) {
      rot_next(cm, smm, c1, s1, &cm, &smm);
      inc(n, m, bj.j, pn[m], cm, smm);
    }
  }
  *fr += sr; *fi += si;
}

// gradient of the regular expansion, G&D (2004) (3.7)
// (src/gradient.c:193-399); g[0..5] += (dx re, dx im, dy re, dy im, dz re, dz im)
// pot (optional): the potential of l2p_helmholtz added in the same sweep.
// Three scratch rows hold degrees n - 1, n, n + 1 and rotate as n grows.
template <typename T, class Coef, class Rec = RecDirect<T>, class Leg = LegDirect<T>>
HD void l2p_helmholtz_grad(int N, T k, const T* xc, const T* xf, Coef&& coef,
                           T* g, T* pot, const Rec& rec, const Leg& leg,
                           const Scratch<T>& sc) {
  T r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  T C = cos(th), S = sin(th), Cph = cos(ph), Sph = sin(ph), kr = k * r;
  zero_rows(sc, 3);
  Row<T> pm1 = sc.row(2), pn = sc.row(0), pnp1 = sc.row(1);
  legendre_init(C, S, &pn[0], &pnp1[0], &pnp1[1]);
  BesselJSeq<T> bj(kr);
  T jnm1 = T(0), jn = bj.jm, jnp1 = bj.j;
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
    T u = b1 * tp * pnp1[mp1] - b2 * tm * pm1[mp1];
    c[0] = c[4] = cp1 * u;
    c[1] = c[5] = sp1 * u;
    b1 = rec.b(n + 1, sgn * m - 1) / T(2);
    b2 = rec.b(n, -sgn * m) / T(2);
    u = b1 * tp * pnp1[mm1] - b2 * tm * pm1[mm1];
    c[3] = cm1 * u;
    c[2] = -sm1 * u;
    c[0] += c[3]; c[1] -= c[2];
    c[2] += c[5]; c[3] -= c[4];
    T a1 = rec.a(n - 1, m), a2 = rec.a(n, m);
    u = a1 * tm * pm1[m] - a2 * tp * pnp1[m];
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
  // advance the rows and Bessel values from degree n - 1 to degree n
  auto advance = [&](int n) {
    Row<T> out = pm1;
    legendre_next(out, pn, pnp1, n, C, S, leg);
    pm1 = pn; pn = pnp1; pnp1 = out;
    jnm1 = bj.jm;
    bj.step();
    jn = bj.jm; jnp1 = bj.j;
  };
  inc(0, 0, 1, Cph, -Sph, T(1), T(0), Cph, Sph);
  advance(1);
  {  // n = 1
    T c2, s2;
    rot_next(Cph, Sph, Cph, Sph, &c2, &s2);
    inc(1, 0, 1, Cph, -Sph, T(1), T(0), Cph, Sph);
    inc(1, 1, 1, T(1), T(0), Cph, Sph, c2, s2);
    inc(1, 1, -1, c2, -s2, Cph, -Sph, T(1), -T(0));
  }
  for (int n = 2; n <= N; n++) {
    advance(n);
    inc(n, 0, 1, Cph, -Sph, T(1), T(0), Cph, Sph);
    // (cos, sin) of (m - 1) ph, m ph, (m + 1) ph
    T ca = T(1), sa = T(0), cb = Cph, sb = Sph, cc, scc;
    for (int m = 1; m <= n; m++) {
      rot_next(cb, sb, Cph, Sph, &cc, &scc);
      inc(n, m, 1, ca, sa, cb, sb, cc, scc);
      inc(n, m, -1, cc, -scc, cb, -sb, ca, -sa);
      ca = cb; sa = sb; cb = cc; sb = scc;
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
                 const Leg& leg, const Scratch<T>& sc) {
  T r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  T C = cos(th), S = sin(th);
  zero_rows(sc, 2);
  Row<T> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  const T c1 = cos(ph), s1 = sin(ph);
  T f = T(0), rn = T(1);
  f += coef(0) * rn * pm[0];
  rn *= r;
  f += coef(1) * rn * pn[0];
  f += T(2) * pn[1] * rn * (coef(lidx(1, 1)) * c1 - coef(lidx(1, 1) + 1) * s1);
#pragma unroll
  for (int n = 2; n <= N; n++) {
    rn *= r;
    legendre_step(pm, pn, n - 1, C, S, leg);
    Row<T> t = pm; pm = pn; pn = t;
    f += coef(n * n) * rn * pn[0];
    T cm = T(1), smm = T(0);
#pragma unroll
    for (int m = 1; m <= n; m++) {
      rot_next(cm, smm, c1, s1, &cm, &smm);
      int id = lidx(n, m);
      f += T(2) * pn[m] * rn * (coef(id) * cm - coef(id + 1) * smm);
    }
  }
  return f;
}

// gradient of the Laplace regular expansion via the derivatives of the
// solid harmonics (src/local-laplace.c:525-630, src/wbfmm-derivatives.h);
// pot (optional): the potential of l2p_laplace added in the same sweep
template <typename T, class Coef, class LRec = LapRecDirect<T>, class Leg = LegDirect<T>>
HD void l2p_laplace_grad(int N, const T* xc, const T* xf, Coef&& coef, T* g,
                         T* pot, const LRec& rec, const Leg& leg,
                         const Scratch<T>& sc) {
  if (N == 0) {   // a constant: no gradient
    if (pot) *pot += coef(0) * (T(1) / (T)sqrt(4.0 * kPi));
    return;
  }
  T r, th, ph;
  cart2sph(xc, xf, &r, &th, &ph);
  T C = cos(th), S = sin(th);
  zero_rows(sc, 2);
  Row<T> pm = sc.row(0), pn = sc.row(1);
  legendre_init(C, S, &pm[0], &pn[0], &pn[1]);
  const T c1 = cos(ph), s1 = sin(ph);
  T gx = T(0), gy = T(0), gz = T(0), f = T(0);
  // degree n >= 2: P holds degree n-1 (gradient), Pn degree n (potential)
  auto d_m0 = [&](int n, T rnm1, Row<T> P, Row<T> Pn) {
    T am, a0, a1;
    rec.c(n, 0, &am, &a0, &a1);
    T R0 = rnm1 * P[0] * a0, R1 = rnm1 * P[1] * a1;
    T cr = coef(n * n);
    gx += cr * (-R1 * c1);
    gy += cr * (-R1 * s1);
    gz += cr * R0;
    if (pot) f += cr * rnm1 * r * Pn[0];
  };
  // (ca, sa), (cb, sb), (cc, scc): (cos, sin) of (m - 1) ph, m ph, (m + 1) ph
  auto d_m = [&](int n, int m, T rnm1, Row<T> P, Row<T> Pn, T ca, T sa, T cb,
                 T sb, T cc, T scc) {
    T am, a0, ap;
    rec.c(n, m, &am, &a0, &ap);
    T Rm = rnm1 * P[m - 1] * am, R0 = rnm1 * P[m] * a0 * T(2);
    T Rp = rnm1 * P[m + 1] * ap;
    T xr = -Rp * cc + Rm * ca, xi = -Rp * scc + Rm * sa;
    T yr = -Rp * scc - Rm * sa, yi = Rp * cc + Rm * ca;
    T zr = R0 * cb, zi = R0 * sb;
    int id = lidx(n, m);
    T cr = coef(id), ci = -coef(id + 1);
    gx += cr * xr + ci * xi;
    gy += cr * yr + ci * yi;
    gz += cr * zr + ci * zi;
    if (pot) f += T(2) * Pn[m] * rnm1 * r * (cr * cb + ci * sb);
  };
  T rnm1 = T(1);
  T c2, s2;
  rot_next(c1, s1, c1, s1, &c2, &s2);
  {  // n = 1, m = 0: only the z derivative is non-zero
    T R0 = rnm1 * pm[0] * sqrt(T(3));
    gz += coef(1) * R0;
    if (pot) f += coef(0) * pm[0] + coef(1) * r * pn[0];
  }
  d_m(1, 1, rnm1, pm, pn, T(1), T(0), c1, s1, c2, s2);
#pragma unroll
  for (int n = 2; n <= N; n++) {
    rnm1 *= r;
    legendre_step(pm, pn, n - 1, C, S, leg);
    Row<T> t = pm; pm = pn; pn = t;       // pm now degree n-1, pn degree n
    d_m0(n, rnm1, pm, pn);
    T ca = T(1), sa = T(0), cb = c1, sb = s1, cc, scc;
#pragma unroll
    for (int m = 1; m <= n; m++) {
      rot_next(cb, sb, c1, s1, &cc, &scc);
      d_m(n, m, rnm1, pm, pn, ca, sa, cb, sb, cc, scc);
      ca = cb; sa = sb; cb = cc; sb = scc;
    }
  }
  g[0] += gx; g[1] += gy; g[2] += gz;
  if (pot) *pot += f;
}

}  // namespace wbfmm
