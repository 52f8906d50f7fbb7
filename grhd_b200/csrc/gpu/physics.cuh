// physics.cuh -- pointwise GRHD physics for the sm_100a kernels.
//
// Every routine restates one reference routine (file:line in RuelasF/GRHD) with the
// reference's evaluation order; built with --fmad=false the FP64 instantiation rounds
// exactly as the reference's operation sequence does.  The arithmetic type R is double
// for the parity path and float for the reconstruction/Riemann/source part of the mixed
// policy; con2prim is always double.
//
// Processor-dependent Fortran semantics, fixed the same way in the CPU oracle:
//   MAX/MIN with NaN arguments keep the first non-NaN value (m=a; if (b>m || m!=m) m=b).
#pragma once

#include <cfloat>
#include <cstdint>

namespace grhd {

constexpr int NEQ = 5;
constexpr int EQ_DE = 0, EQ_PR = 1, EQ_VX = 2, EQ_VY = 3, EQ_VZ = 4;
constexpr int REC_GODUNOV = 1, REC_TVD = 2, REC_WENO3 = 3, REC_MP5 = 4, REC_WENO5 = 5;
constexpr int RS_HLLE = 1, RS_HLLC = 2;
constexpr int LIM_MINMOD = 1, LIM_SUPERBEE = 2, LIM_MC = 3;

// recon branch codes (one per face: the reference's conditions do not depend on the variable)
constexpr int BR_GODUNOV = 0, BR_TVD = 1, BR_TVD_MC = 2, BR_WENO3 = 3, BR_MP5 = 4, BR_WENO5 = 5;

struct Phys {
  int rec, lim, rs, sensor;
  int nonmink;  // metric_type /= 'Minkowski' (reconstruction.f90:356 etc.)
  int srhd;     // Minkowski + Cartesian: SRHD wavespeeds and no sources (fluxes.f90:45, equations.f90:521)
  double adb, g1, rho_floor, p_floor, v_max;
};

// per-face metric (k-invariant): lapse, normal shift, symmetric gamma_ij, sqrt(gamma), gamma^dd
template <class R>
struct FaceMetric {
  R alpha, beta_n, g11, g12, g13, g22, g23, g33, sqg, gup;
  __device__ __forceinline__ R G(int a, int b) const {  // 1-based symmetric access
    const int m = a < b ? a * 4 + b : b * 4 + a;
    switch (m) {
      case 5: return g11; case 6: return g12; case 7: return g13;
      case 10: return g22; case 11: return g23; default: return g33;
    }
  }
};

template <class R> __device__ __forceinline__ R rmax(R a, R b) { return (b > a || a != a) ? b : a; }
// n / d for a denominator that is positive (+inf included) or NaN.  The correctly rounded
// FP64 division runs about three times slower for a zero numerator, and exactly smooth or
// static regions (a floored atmosphere) produce zero numerators in bulk: a zero never
// reaches the divider (it divides 1 instead) and is returned as it is -- the quotient, to
// the bit.  FP32 (the mixed policy's approximate division) divides.
template <class R> __device__ __forceinline__ R div_pos(R n, R d) {
  if (sizeof(R) == sizeof(float)) return n / d;
  const bool z = n == R(0);
  const R q = (z ? R(1) : n) / d;
  return (z && d == d) ? n : q;
}
template <class R> __device__ __forceinline__ R rmin(R a, R b) { return (b < a || a != a) ? b : a; }
template <class R> __device__ __forceinline__ R sgn1(R x) { return copysign(R(1), x); }
template <class R> __device__ __forceinline__ bool fin(R x) { return isfinite(x); }
template <class R> __device__ __forceinline__ R tiny_of();
template <> __device__ __forceinline__ double tiny_of<double>() { return DBL_MIN; }
template <> __device__ __forceinline__ float tiny_of<float>() { return FLT_MIN; }
template <class R> __device__ __forceinline__ R eps_of();
template <> __device__ __forceinline__ double eps_of<double>() { return DBL_EPSILON; }
template <> __device__ __forceinline__ float eps_of<float>() { return FLT_EPSILON; }
// Relative tolerance of the reference (FP64) kept as is for double; for the FP32 arithmetic
// of the mixed policy never tighter than 64 ulp, so round-off alone does not fail a test
// that the FP64 path passes (the HLLC consistency checks, the wavespeed radicand).
template <class R> __device__ __forceinline__ R ftol(double ref);
template <> __device__ __forceinline__ double ftol<double>(double ref) { return ref; }
template <> __device__ __forceinline__ float ftol<float>(double ref) {
  return (float)(ref > 64.0 * FLT_EPSILON ? ref : 64.0 * FLT_EPSILON);
}

// exp for the WENO3 adaptive epsilon (reconstruction.f90:169).  CUDA's exp and the host C
// library's (which the reference calls) round differently in the last bit, and a one-ulp
// difference flips downstream branches (MP5's "< 1e-10" test, the HLLC tolerances), so the
// kernels and the CPU oracle evaluate exp with one published method and the same
// operation order: Cody-Waite reduction x = k ln2 + r, k = rint(x/ln2), ln2 split into a
// 32-bit head and a tail; e^r by its Taylor series through r^13/13! on |r| <= ln2/2
// (truncation below 5e-18 relative) in Horner form; exact scaling by 2^k.  Accurate to
// about one ulp.
__device__ __forceinline__ double exp_cw(double x) {
  if (x != x) return x;
  if (x > 709.78) return HUGE_VAL;
  if (x < -745.2) return 0.0;
  const double log2e = 0x1.71547652b82fep+0;
  const double ln2_hi = 0x1.62e42feep-1;        // ln 2 to 32 significant bits
  const double ln2_lo = 0x1.a39ef35793c76p-33;  // ln 2 - ln2_hi
  const double k = rint(x * log2e);
  const double r = (x - k * ln2_hi) - k * ln2_lo;
  double p = 1.0 / 6227020800.0;
  p = 1.0 / 479001600.0 + r * p;
  p = 1.0 / 39916800.0 + r * p;
  p = 1.0 / 3628800.0 + r * p;
  p = 1.0 / 362880.0 + r * p;
  p = 1.0 / 40320.0 + r * p;
  p = 1.0 / 5040.0 + r * p;
  p = 1.0 / 720.0 + r * p;
  p = 1.0 / 120.0 + r * p;
  p = 1.0 / 24.0 + r * p;
  p = 1.0 / 6.0 + r * p;
  p = 0.5 + r * p;
  p = 1.0 + r * p;
  return ldexp(1.0 + r * p, (int)k);
}
__device__ __forceinline__ float exp_cw(float x) { return expf(x); }  // mixed policy: FP32

// ------------------------------------------------------------------------------------
// reconstruction.f90:28-278
// ------------------------------------------------------------------------------------
template <class R> __device__ __forceinline__ R minmod_2(R a, R b) {
  return R(0.5) * (sgn1(a) + sgn1(b)) * rmin(fabs(a), fabs(b));
}
template <class R> __device__ __forceinline__ R minmod_3(R a, R b, R c) {
  return sgn1(a) * rmax(R(0), rmin(rmin(fabs(a), sgn1(a) * b), sgn1(a) * c));
}
template <class R> __device__ __forceinline__ R minmod_4(R a, R b, R c, R d) {
  return R(0.125) * (sgn1(a) + sgn1(b)) * fabs(sgn1(a) + sgn1(c)) * fabs(sgn1(a) + sgn1(d)) *
         rmin(rmin(rmin(fabs(a), fabs(b)), fabs(c)), fabs(d));
}
// reconstruction.f90:141-181, q(-1:1)
template <class R> __device__ __forceinline__ R weno3(R qm, R q0, R qp) {
  const R eps_min = R(1.0e-14);
  const R d0 = R(2.0 / 3.0), d1 = R(1.0 / 3.0);
  R p0 = R(0.5) * q0 + R(0.5) * qp;
  R p1 = R(-0.5) * qm + R(1.5) * q0;
  R t0 = q0 - qp, t1 = qm - q0;
  R b0 = t0 * t0, b1 = t1 * t1;
  R sensor = div_pos(fabs(b0 - b1), rmax(b0, b1) + eps_min);
  R eh = eps_min + (qm * qm + q0 * q0 + qp * qp) * exp_cw(R(-10) * sensor);
  R e0 = eh + b0, e1 = eh + b1;
  R a0 = d0 / (e0 * e0), a1 = d1 / (e1 * e1);
  R w0 = a0 / (a0 + a1), w1 = a1 / (a0 + a1);
  return w0 * p0 + w1 * p1;
}
// reconstruction.f90:187-215, q(-2:2)
template <class R> __device__ __forceinline__ R weno5(R q_2, R q_1, R q0, R q1, R q2) {
  const R eps = R(1.0e-14);
  const R d0 = R(0.3), d1 = R(0.6), d2 = R(0.1);
  const R c1312 = R(13.0 / 12.0);
  R a, b;
  a = q0 - R(2) * q1 + q2; b = R(3) * q0 - R(4) * q1 + q2;
  R b0 = c1312 * (a * a) + R(0.25) * (b * b);
  a = q_1 - R(2) * q0 + q1; b = q_1 - q1;
  R b1 = c1312 * (a * a) + R(0.25) * (b * b);
  a = q_2 - R(2) * q_1 + q0; b = q_2 - R(4) * q_1 + R(3) * q0;
  R b2 = c1312 * (a * a) + R(0.25) * (b * b);
  R tau5 = fabs(b0 - b2);
  R w0, w1, w2;
  if (sizeof(R) == sizeof(double) && tau5 == R(0) && b1 == b1) {
    // an exactly smooth stencil (a uniform atmosphere, say): every tau5 / (eps + b_k) is +0
    // (tau5 == 0 means b0 and b2 are not NaN; each eps + b_k >= eps > 0 or +inf), so the
    // alphas are d_k and the weights the constants d_k / (d0 + d1 + d2), folded at compile
    // time with the same correctly rounded arithmetic.  The FP64 divisions skipped here run
    // about three times slower than usual for zero numerators.
    const R a0 = d0 * (R(1) + R(0)), a1 = d1 * (R(1) + R(0)), a2 = d2 * (R(1) + R(0));
    const R s = a0 + a1 + a2;
    w0 = a0 / s; w1 = a1 / s; w2 = a2 / s;
  } else {
    const R a0 = d0 * (R(1) + (tau5 / (eps + b0)));
    const R a1 = d1 * (R(1) + (tau5 / (eps + b1)));
    const R a2 = d2 * (R(1) + (tau5 / (eps + b2)));
    const R s = a0 + a1 + a2;
    if (sizeof(R) == sizeof(float)) {  // mixed policy: one reciprocal for the three weights
      const R inv_s = R(1) / s;
      w0 = a0 * inv_s; w1 = a1 * inv_s; w2 = a2 * inv_s;
    } else {
      w0 = a0 / s; w1 = a1 / s; w2 = a2 / s;
    }
  }
  R p0 = R(1.0 / 3.0) * q0 + R(5.0 / 6.0) * q1 - R(1.0 / 6.0) * q2;
  R p1 = -(R(1.0 / 6.0) * q_1) + R(5.0 / 6.0) * q0 + R(1.0 / 3.0) * q1;
  R p2 = R(1.0 / 3.0) * q_2 - R(7.0 / 6.0) * q_1 + R(11.0 / 6.0) * q0;
  return w0 * p0 + w1 * p1 + w2 * p2;
}
// reconstruction.f90:222-254, q(-2:2)
template <class R> __device__ __forceinline__ R mp5(R q_2, R q_1, R q0, R q1, R q2) {
  const R alpha = R(4), eps = R(1.0e-10);
  R val_L = div_pos(R(2) * q_2 - R(13) * q_1 + R(47) * q0 + R(27) * q1 - R(3) * q2, R(60));
  R val_mp = q0 + minmod_2(q1 - q0, alpha * (q0 - q_1));
  if ((val_L - q0) * (val_L - val_mp) < eps) return val_L;
  R d_jm1 = q_2 - R(2) * q_1 + q0;
  R d_j = q_1 - R(2) * q0 + q1;
  R d_jp1 = q0 - R(2) * q1 + q2;
  R dm4_jph = minmod_4(R(4) * d_j - d_jp1, R(4) * d_jp1 - d_j, d_j, d_jp1);
  R dm4_jmh = minmod_4(R(4) * d_j - d_jm1, R(4) * d_jm1 - d_j, d_j, d_jm1);
  R val_ul = q0 + alpha * (q0 - q_1);
  R val_av = R(0.5) * (q0 + q1);
  R val_md = val_av - R(0.5) * dm4_jph;
  R val_lc = q0 + R(0.5) * (q0 - q_1) + div_pos(R(4) * dm4_jmh, R(3));
  R vmin = rmax(rmin(rmin(q0, q1), val_md), rmin(rmin(q0, val_ul), val_lc));
  R vmax = rmin(rmax(rmax(q0, q1), val_md), rmax(rmax(q0, val_ul), val_lc));
  return val_L + minmod_2(vmin - val_L, vmax - val_L);
}
// reconstruction.f90:259-278
template <class R> __device__ __forceinline__ R tvd_slope(R a, R b, int lim) {
  if (lim == LIM_SUPERBEE) {
    if (a * b <= R(0)) return R(0);
    return sgn1(a) * rmax(rmin(R(2) * fabs(a), fabs(b)), rmin(fabs(a), R(2) * fabs(b)));
  }
  if (lim == LIM_MC) return minmod_3(R(2) * b, R(0.5) * (a + b), R(2) * a);
  return minmod_2(a, b);
}

// Cells [lo, hi] of the 6-point window (i-2 .. i+3 for face i) that a scheme reads.
__host__ __device__ __forceinline__ void stencil_range(int rec, int sensor, int &lo, int &hi) {
  if (rec == REC_GODUNOV) { lo = 2; hi = 3; }
  else if (rec == REC_TVD || rec == REC_WENO3) { lo = sensor ? 0 : 1; hi = 4; }
  else { lo = 0; hi = 5; }
}

// ------------------------------------------------------------------------------------
// equations.f90:434-502, fluxes.f90:76-156, 669-803
// ------------------------------------------------------------------------------------
// velocity cap shared by calc_fluxes, prim_to_cons_face and the wavespeed routines
template <class R>
__device__ __forceinline__ R cap_velocity(const FaceMetric<R> &m, R (&v)[3], R v_max) {
  R vsq = R(0);
#pragma unroll
  for (int a = 1; a <= 3; ++a)
#pragma unroll
    for (int b = 1; b <= 3; ++b) vsq = vsq + m.G(a, b) * v[a - 1] * v[b - 1];
  if (vsq >= v_max) {
    v[0] = v[0] * sqrt(v_max / vsq);
    v[1] = v[1] * sqrt(v_max / vsq);
    v[2] = v[2] * sqrt(v_max / vsq);
    vsq = v_max;
  }
  return vsq;
}
template <class R>
__device__ __forceinline__ void lower(const FaceMetric<R> &m, const R (&v)[3], R (&vc)[3]) {
#pragma unroll
  for (int a = 1; a <= 3; ++a) {
    R s = R(0);
#pragma unroll
    for (int b = 1; b <= 3; ++b) s = s + m.G(a, b) * v[b - 1];
    vc[a - 1] = s;
  }
}

// calc_fluxes (F) and prim_to_cons_face (U) together: they share v_sq, h, W, v_cov
template <class R>
__device__ __forceinline__ void flux_and_cons(const Phys &P, const R (&q)[NEQ], int dir,
                                              const FaceMetric<R> &m, R (&f)[NEQ], R (&u)[NEQ]) {
  R v[3] = {q[EQ_VX], q[EQ_VY], q[EQ_VZ]}, vc[3];
  const R vsq = cap_velocity(m, v, R(P.v_max));
  lower(m, v, vc);
  const R v_norm = dir == 1 ? v[0] : (dir == 2 ? v[1] : v[2]);
  const R h = R(1) + R(P.g1) * q[EQ_PR] / q[EQ_DE];
  const R W = R(1) / sqrt(R(1) - vsq);
  const R v_eff = m.alpha * v_norm - m.beta_n;
  const R rhW2 = q[EQ_DE] * h * (W * W);
  f[EQ_DE] = q[EQ_DE] * W * v_eff;
  f[EQ_PR] = rhW2 * v_eff + q[EQ_PR] * m.beta_n - f[EQ_DE];
  f[EQ_VX] = rhW2 * vc[0] * v_eff + (dir == 1 ? m.alpha * q[EQ_PR] : R(0));
  f[EQ_VY] = rhW2 * vc[1] * v_eff + (dir == 2 ? m.alpha * q[EQ_PR] : R(0));
  f[EQ_VZ] = rhW2 * vc[2] * v_eff + (dir == 3 ? m.alpha * q[EQ_PR] : R(0));
  u[EQ_DE] = q[EQ_DE] * W;
  u[EQ_PR] = rhW2 - q[EQ_PR] - q[EQ_DE] * W;
  u[EQ_VX] = rhW2 * vc[0];
  u[EQ_VY] = rhW2 * vc[1];
  u[EQ_VZ] = rhW2 * vc[2];
#pragma unroll
  for (int n = 0; n < NEQ; ++n) { f[n] = f[n] * m.sqg; u[n] = u[n] * m.sqg; }
}

// calc_wavespeeds_srhd / calc_wavespeeds_grhd; gamma^dd of the face comes precomputed
// with the reference's Cramer formula (fluxes.f90:760-774)
template <class R>
__device__ __forceinline__ void wavespeeds(const Phys &P, const R (&q)[NEQ], int dir,
                                           const FaceMetric<R> &m, R &wmin, R &wmax) {
  R v[3] = {q[EQ_VX], q[EQ_VY], q[EQ_VZ]};
  const R vsq = cap_velocity(m, v, R(P.v_max));
  const R enth = R(1) + R(P.g1) * q[EQ_PR] / q[EQ_DE];
  const R cs2 = R(P.adb) * q[EQ_PR] / (q[EQ_DE] * enth);
  const R cs = sqrt(cs2);
  const R vn = dir == 1 ? v[0] : (dir == 2 ? v[1] : v[2]);
  R e1, e2, e3;
  if (P.srhd) {
    const R t1 = R(1) / (R(1) - vsq * cs2);
    const R t2 = cs * sqrt((R(1) - vsq) * (R(1) / t1 - (vn * vn) * (R(1) - cs2)));
    e1 = vn;
    e2 = t1 * (vn * (R(1) - cs2) + t2);
    e3 = t1 * (vn * (R(1) - cs2) - t2);
  } else {
    const R t1 = m.alpha / (R(1) - vsq * cs2);
    const R t2 = cs * sqrt(rmax(R(0), (R(1) - vsq) * (m.gup * (R(1) - vsq * cs2) - (vn * vn) * (R(1) - cs2))));
    e1 = m.alpha * vn - m.beta_n;
    e2 = t1 * (vn * (R(1) - cs2) + t2) - m.beta_n;
    e3 = t1 * (vn * (R(1) - cs2) - t2) - m.beta_n;
  }
  wmax = rmax(rmax(rmax(R(0), e1), e2), e3);
  wmin = rmin(rmin(rmin(R(0), e1), e2), e3);
}

// calc_hlle_fluxes, fluxes.f90:125-156
template <class R>
__device__ __forceinline__ void hlle(const Phys &P, const R (&qL)[NEQ], const R (&qR)[NEQ], int dir,
                                     const FaceMetric<R> &m, R (&flux)[NEQ]) {
  R fL[NEQ], fR[NEQ], uL[NEQ], uR[NEQ], lLmin, lLmax, lRmin, lRmax;
  flux_and_cons(P, qL, dir, m, fL, uL);
  flux_and_cons(P, qR, dir, m, fR, uR);
  wavespeeds(P, qL, dir, m, lLmin, lLmax);
  wavespeeds(P, qR, dir, m, lRmin, lRmax);
  const R ap = rmax(rmax(R(0), lLmax), lRmax);
  const R am = rmin(rmin(R(0), lLmin), lRmin);
  if (fabs(ap - am) < R(1.0e-14)) {
#pragma unroll
    for (int n = 0; n < NEQ; ++n) flux[n] = R(0);
  } else if (sizeof(R) == sizeof(float)) {  // mixed policy: one reciprocal for the five components
    const R inv = R(1) / (ap - am);
#pragma unroll
    for (int n = 0; n < NEQ; ++n) flux[n] = (ap * fL[n] - am * fR[n] + ap * am * (uR[n] - uL[n])) * inv;
  } else {
#pragma unroll
    for (int n = 0; n < NEQ; ++n)  // ap - am > 0 here (or NaN)
      flux[n] = div_pos(ap * fL[n] - am * fR[n] + ap * am * (uR[n] - uL[n]), ap - am);
  }
}

// Orthonormal face frame of build_face_orthonormal_frame (fluxes.f90:402-473), precomputed
// per face: cof[a][i] = coframe(a+1,i+1), gup = gamma^dd, ok flag.
template <class R>
struct FaceFrame {
  R cof[3][3];
  R gup;
  int ok;
};

// fluxes.f90:509-568 calc_srhd_local_state
template <class R>
__device__ __forceinline__ bool srhd_local(const Phys &P, const R (&ql)[NEQ], R (&u)[NEQ], R (&f)[NEQ],
                                           R &wmin, R &wmax) {
#pragma unroll
  for (int n = 0; n < NEQ; ++n) { u[n] = R(0); f[n] = R(0); }
  wmin = R(0); wmax = R(0);
  const R rho = ql[EQ_DE], pr = ql[EQ_PR], v0 = ql[EQ_VX], v1 = ql[EQ_VY], v2 = ql[EQ_VZ];
  if (!fin(rho) || !fin(pr) || !fin(v0) || !fin(v1) || !fin(v2) || rho <= R(0) || pr < R(0)) return false;
  const R vsq = v0 * v0 + v1 * v1 + v2 * v2;
  if (!fin(vsq) || vsq < R(0)) return false;
  if (vsq >= R(P.v_max)) return false;
  const R h = R(1) + R(P.g1) * pr / rho;
  if (!fin(h) || h <= R(0)) return false;
  const R cs2 = R(P.adb) * pr / (rho * h);
  if (!fin(cs2) || cs2 < R(0) || cs2 >= R(1)) return false;
  const R W = R(1) / sqrt(R(1) - vsq);
  const R D = rho * W;
  const R rhW2 = rho * h * (W * W);
  const R m0 = rhW2 * v0, m1 = rhW2 * v1, m2 = rhW2 * v2;
  u[EQ_DE] = D; u[EQ_PR] = rhW2 - pr - D; u[EQ_VX] = m0; u[EQ_VY] = m1; u[EQ_VZ] = m2;
  f[EQ_DE] = D * v0;
  f[EQ_PR] = m0 - D * v0;
  f[EQ_VX] = m0 * v0 + pr;
  f[EQ_VY] = m1 * v0;
  f[EQ_VZ] = m2 * v0;
  const R den = R(1) - vsq * cs2;
  const R rad = (R(1) - vsq) * (R(1) - vsq * cs2 - (v0 * v0) * (R(1) - cs2));
  if (den <= R(1.0e-14) || rad < -ftol<R>(1.0e-12)) return false;
  const R ac = sqrt(cs2) * sqrt(rmax(R(0), rad));
  wmin = (v0 * (R(1) - cs2) - ac) / den;
  wmax = (v0 * (R(1) - cs2) + ac) / den;
#pragma unroll
  for (int n = 0; n < NEQ; ++n) if (!fin(u[n]) || !fin(f[n])) return false;
  if (!fin(wmin) || !fin(wmax)) return false;
  return true;
}

// fluxes.f90:571-591
template <class R>
__device__ __forceinline__ bool admissible(const R (&u)[NEQ]) {
#pragma unroll
  for (int n = 0; n < NEQ; ++n) if (!fin(u[n])) return false;
  if (u[EQ_DE] <= R(0)) return false;
  const R E = u[EQ_PR] + u[EQ_DE];
  const R msq = u[EQ_VX] * u[EQ_VX] + u[EQ_VY] * u[EQ_VY] + u[EQ_VZ] * u[EQ_VZ];
  const R scale = rmax(rmax(tiny_of<R>(), E * E), u[EQ_DE] * u[EQ_DE] + msq);
  if (E <= R(0)) return false;
  if (E * E - u[EQ_DE] * u[EQ_DE] - msq <= R(1.0e-13) * scale) return false;
  return true;
}

// fluxes.f90:596-624
template <class R>
__device__ __forceinline__ bool local_to_coord(const R (&ul)[NEQ], const R (&fl)[NEQ], R w, R alpha,
                                               R sqg, const FaceFrame<R> &fr, R (&flux)[NEQ]) {
  R mf[NEQ];
#pragma unroll
  for (int n = 0; n < NEQ; ++n) { flux[n] = R(0); mf[n] = fl[n] - w * ul[n]; }
  const R factor = sqg * alpha * sqrt(fr.gup);
  if (!fin(factor)) return false;
#pragma unroll
  for (int n = 0; n < NEQ; ++n) if (!fin(mf[n])) return false;
  flux[EQ_DE] = factor * mf[EQ_DE];
  flux[EQ_PR] = factor * mf[EQ_PR];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    R s = R(0);
#pragma unroll
    for (int a = 0; a < 3; ++a) s = s + factor * fr.cof[a][i] * mf[EQ_VX + a];
    flux[EQ_VX + i] = s;
  }
#pragma unroll
  for (int n = 0; n < NEQ; ++n) if (!fin(flux[n])) return false;
  return true;
}

// calc_hllc_fluxes, fluxes.f90:174-397, without its HLLE exits: returns true when the
// reference would fall back to calc_hlle_fluxes (the caller then runs HLLE, so a kernel
// holds one copy of the HLLE code).
template <class R>
__device__ bool hllc_try(const Phys &P, const R (&qL)[NEQ], const R (&qR)[NEQ], int dir,
                         const FaceMetric<R> &m, const FaceFrame<R> &fr, R (&flux)[NEQ]) {
  const R alpha = m.alpha, sqg = m.sqg;
  R qLh[NEQ], qRh[NEQ], uL[NEQ], uR[NEQ], fL[NEQ], fR[NEQ];
  R lLmin, lLmax, lRmin, lRmax;
  R ls, denom, face_speed, lam_l, lam_r;
  if (!(alpha > R(0)) || !(sqg > R(0)) || !fin(alpha) || !fin(sqg) || !fr.ok) goto fallback;
  // primitives_to_local_frame (fluxes.f90:490-504)
#pragma unroll
  for (int n = 0; n < 2; ++n) { qLh[n] = qL[n]; qRh[n] = qR[n]; }
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    R sl = R(0), sr = R(0);
#pragma unroll
    for (int i = 0; i < 3; ++i) { sl = sl + fr.cof[a][i] * qL[EQ_VX + i]; sr = sr + fr.cof[a][i] * qR[EQ_VX + i]; }
    qLh[EQ_VX + a] = sl; qRh[EQ_VX + a] = sr;
  }
  if (!srhd_local(P, qLh, uL, fL, lLmin, lLmax)) goto fallback;
  if (!srhd_local(P, qRh, uR, fR, lRmin, lRmax)) goto fallback;
  lam_l = rmin(lLmin, lRmin);
  lam_r = rmax(lLmax, lRmax);
  face_speed = m.beta_n / (alpha * sqrt(fr.gup));
  if (!fin(face_speed) || lam_r - lam_l <= R(1.0e-13)) goto fallback;
  if (face_speed <= lam_l) {
    if (!local_to_coord(uL, fL, face_speed, alpha, sqg, fr, flux)) goto fallback;
    return false;
  } else if (face_speed >= lam_r) {
    if (!local_to_coord(uR, fR, face_speed, alpha, sqg, fr, flux)) goto fallback;
    return false;
  }
  {
    R uh[NEQ], fh[NEQ];
    denom = lam_r - lam_l;
#pragma unroll
    for (int n = 0; n < NEQ; ++n) {
      uh[n] = (lam_r * uR[n] - lam_l * uL[n] + fL[n] - fR[n]) / denom;
      fh[n] = (lam_r * fL[n] - lam_l * fR[n] + lam_r * lam_l * (uR[n] - uL[n])) / denom;
    }
#pragma unroll
    for (int n = 0; n < NEQ; ++n) if (!fin(uh[n]) || !fin(fh[n])) goto fallback;
    const R E_hll = uh[EQ_PR] + uh[EQ_DE];
    const R FE_hll = fh[EQ_PR] + fh[EQ_DE];
    const R A = FE_hll, B = -(E_hll + fh[EQ_VX]), Cq = uh[EQ_VX];
    R disc = B * B - R(4) * A * Cq;
    const R disc_scale = rmax(rmax(tiny_of<R>(), B * B), fabs(R(4) * A * Cq));
    if (!fin(disc) || disc < -ftol<R>(1.0e-12) * disc_scale) goto fallback;
    disc = rmax(R(0), disc);
    const R coef_scale = rmax(rmax(tiny_of<R>(), fabs(B)), fabs(Cq));
    // Under the mixed policy (R = float) the zero tests scale with FP32 round-off (ftol):
    // on a face without normal motion A and Cq vanish in exact arithmetic, FP32 leaves them
    // at ~1e-8 of their scale, and with the FP64 threshold the quadratic's root
    // (-B - sqrt(disc)) / (2A) then cancels to noise, falls outside [lam_l, lam_r] and the
    // face drops to HLLE.  FP32 also takes both roots without cancellation, q = -(B +
    // sgn(B) sqrt(disc)) / 2 and the roots q / A, Cq / q (the standard stable form),
    // choosing the reference's first root (-B - sqrt(disc)) / (2A) and its alternative as
    // below.  Measured: a 33 x 9 x-y Sod tube, 13 steps, 927 FP32 fallbacks -> 0 (5730 -> 0
    // with 5 % pressure noise), relative L1 against FP64 2.3e-5 -> 1.0e-7 (2e-3 -> 1.1e-7);
    // the 3D torus 256x128x128 after 500 steps 9.8e-6 -> 4.2e-7.  FP64 keeps the
    // reference's constants and formulas.
    constexpr bool f32 = sizeof(R) == sizeof(float);
    const bool quad = fabs(A) > ftol<R>(1.0e-13) * coef_scale;
    R alt32 = R(0);
    if (!quad) {
      if (fabs(B) <= ftol<R>(1.0e-14) * rmax(tiny_of<R>(), fabs(Cq))) goto fallback;
      ls = -Cq / B;
    } else if (f32) {
      const R q = R(-0.5) * (B + copysign(sqrt(disc), B));
      if (q == R(0)) goto fallback;
      const R ra = q / A, rb = Cq / q;
      ls = B >= R(0) ? ra : rb;
      alt32 = B >= R(0) ? rb : ra;
    } else {
      denom = -B - sqrt(disc);
      if (fabs(denom) > R(1.0e-14) * rmax(rmax(tiny_of<R>(), fabs(B)), sqrt(disc))) {
        ls = denom / (R(2) * A);
      } else {
        denom = -B + sqrt(disc);
        if (fabs(denom) <= R(1.0e-14) * rmax(rmax(tiny_of<R>(), fabs(B)), sqrt(disc))) goto fallback;
        ls = (R(2) * Cq) / denom;
      }
    }
    const R root_tol = ftol<R>(1.0e-10) * rmax(rmax(R(1), fabs(lam_l)), fabs(lam_r));
    bool valid = fin(ls) && ls >= lam_l - root_tol && ls <= lam_r + root_tol && fabs(ls) <= R(1) + root_tol;
    if (!valid && quad) {
      const R alt = f32 ? alt32 : (-B + sqrt(disc)) / (R(2) * A);
      if (fin(alt) && alt >= lam_l - root_tol && alt <= lam_r + root_tol && fabs(alt) <= R(1) + root_tol) {
        ls = alt;
        valid = true;
      }
    }
    if (!valid) goto fallback;
    ls = rmin(lam_r, rmax(lam_l, ls));
    const R A_l = lam_l * (uL[EQ_PR] + uL[EQ_DE]) - uL[EQ_VX];
    const R B_l = uL[EQ_VX] * (lam_l - qLh[EQ_VX]) - qLh[EQ_PR];
    const R A_r = lam_r * (uR[EQ_PR] + uR[EQ_DE]) - uR[EQ_VX];
    const R B_r = uR[EQ_VX] * (lam_r - qRh[EQ_VX]) - qRh[EQ_PR];
    denom = R(1) - lam_l * ls;
    if (fabs(denom) <= R(1.0e-13)) goto fallback;
    const R psl = (A_l * ls - B_l) / denom;
    denom = R(1) - lam_r * ls;
    if (fabs(denom) <= R(1.0e-13)) goto fallback;
    const R psr = (A_r * ls - B_r) / denom;
    const R state_scale = rmax(rmax(rmax(rmax(tiny_of<R>(), fabs(uL[EQ_PR] + uL[EQ_DE])), fabs(uR[EQ_PR] + uR[EQ_DE])),
                                    fabs(uL[EQ_VX])), fabs(uR[EQ_VX]));
    const R ptol = ftol<R>(1.0e-8) * rmax(rmax(rmax(rmax(tiny_of<R>(), fabs(qLh[EQ_PR])), fabs(qRh[EQ_PR])), fabs(psl)), fabs(psr)) +
                   R(1.0e2) * eps_of<R>() * state_scale;
    if (!fin(psl) || !fin(psr) || fabs(psl - psr) > ptol) goto fallback;
    const R ps = R(0.5) * (psl + psr);
    if (!fin(ps) || fabs(lam_l - ls) <= R(1.0e-13) || fabs(lam_r - ls) <= R(1.0e-13)) goto fallback;
    R usL[NEQ], usR[NEQ], fsL[NEQ], fsR[NEQ];
#pragma unroll
    for (int n = 0; n < NEQ; ++n) {
      const R pv = (n == EQ_PR) ? ls : ((n == EQ_VX) ? R(1) : R(0));
      usL[n] = (lam_l * uL[n] - fL[n] + ps * pv) / (lam_l - ls);
      usR[n] = (lam_r * uR[n] - fR[n] + ps * pv) / (lam_r - ls);
    }
#pragma unroll
    for (int n = 0; n < NEQ; ++n) {
      fsL[n] = fL[n] + lam_l * (usL[n] - uL[n]);
      fsR[n] = fR[n] + lam_r * (usR[n] - uR[n]);
    }
    if (!admissible(usL) || !admissible(usR)) goto fallback;
#pragma unroll
    for (int n = 0; n < NEQ; ++n) if (!fin(fsL[n]) || !fin(fsR[n])) goto fallback;
    bool ok;
    if (face_speed <= ls) ok = local_to_coord(usL, fsL, face_speed, alpha, sqg, fr, flux);
    else ok = local_to_coord(usR, fsR, face_speed, alpha, sqg, fr, flux);
    if (!ok) goto fallback;
    return false;
  }
fallback:
  return true;
}

// calc_hllc_fluxes with its HLLE exits; returns true when it fell back
template <class R>
__device__ __forceinline__ bool hllc(const Phys &P, const R (&qL)[NEQ], const R (&qR)[NEQ], int dir,
                                     const FaceMetric<R> &m, const FaceFrame<R> &fr, R (&flux)[NEQ]) {
  const bool fb = hllc_try(P, qL, qR, dir, m, fr, flux);
  if (fb) hlle(P, qL, qR, dir, m, flux);
  return fb;
}

// ------------------------------------------------------------------------------------
// equations.f90:94-424 con2prim (always FP64)
// ------------------------------------------------------------------------------------
// symmetric gamma_ij and gamma^ij, sqrt(gamma) of a cell, held in registers.  con2prim
// reads a metric through the accessors g11() .. sqg(), so it also takes views that fetch
// each field where it is used (a cell kernel's shared-memory slice of the table).
struct CellMetric {
  double g11_, g12_, g13_, g22_, g23_, g33_;
  double i11_, i12_, i13_, i22_, i23_, i33_;
  double sqg_;
  __device__ __forceinline__ double g11() const { return g11_; }
  __device__ __forceinline__ double g12() const { return g12_; }
  __device__ __forceinline__ double g13() const { return g13_; }
  __device__ __forceinline__ double g22() const { return g22_; }
  __device__ __forceinline__ double g23() const { return g23_; }
  __device__ __forceinline__ double g33() const { return g33_; }
  __device__ __forceinline__ double i11() const { return i11_; }
  __device__ __forceinline__ double i12() const { return i12_; }
  __device__ __forceinline__ double i13() const { return i13_; }
  __device__ __forceinline__ double i22() const { return i22_; }
  __device__ __forceinline__ double i23() const { return i23_; }
  __device__ __forceinline__ double i33() const { return i33_; }
  __device__ __forceinline__ double sqg() const { return sqg_; }
};

enum C2PFlags : unsigned {
  C2P_FLOOR_PRE = 1u, C2P_CAUSAL = 2u, C2P_BRENT = 4u, C2P_ROOT_FAIL = 8u, C2P_BAD_V = 16u, C2P_SANITISE = 32u
};

template <class M>
__device__ __forceinline__ double qsq(const M &m, double S1, double S2, double S3) {
  // sum over (ii, jj) in the reference's loop order (equations.f90:273-277, :236-242)
  double s = 0.0;
  s = s + m.i11() * S1 * S1; s = s + m.i12() * S1 * S2; s = s + m.i13() * S1 * S3;
  s = s + m.i12() * S2 * S1; s = s + m.i22() * S2 * S2; s = s + m.i23() * S2 * S3;
  s = s + m.i13() * S3 * S1; s = s + m.i23() * S3 * S2; s = s + m.i33() * S3 * S3;
  return s;
}
// equations.f90:212-246
__device__ __forceinline__ void residual(double g1, double W, double D, double tau, double Q2,
                                         double &res, double &dres) {
  const double den = g1 * (W * W) - 1.0;
  const double V = (g1 * (W * W) * (tau + D) - D * W) / den;
  const double dV = (g1 * W * (D * W - 2.0 * (tau + D)) + D) / (den * den);
  const double W3 = W * W * W;
  res = (V * V) * (1.0 - 1.0 / (W * W)) - Q2;
  dres = 2.0 * V * (dV * (W3 - W) + V) / W3;
}
// Mixed policy only: reciprocal of a positive normal x in FP64, by Newton-Raphson
// refinement (r <- r + r (1 - x r), each step doubling the correct bits) of the hardware
// approximation rcp.approx.ftz.f64.  Two steps: on 2.7e8 random x with exponents in
// [-60, 60] the result equals the correctly rounded 1.0 / x bit for bit (one step: 1e-12
// relative).  Zero, subnormal or infinite x give NaN or 0; callers pass positive normals.
__device__ __forceinline__ double rcp_mixed(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}
// The residual of equations.f90:212-246 for the mixed policy's root finder: the same
// expressions with one reciprocal of den and one of W shared by its four quotients.
__device__ __forceinline__ void residual_mixed(double g1, double W, double D, double tau, double Q2,
                                               double &res, double &dres) {
  const double W2 = W * W;
  const double den = g1 * W2 - 1.0;  // > 0: g1 > 1, W >= 1
  const double iden = rcp_mixed(den);
  const double V = (g1 * W2 * (tau + D) - D * W) * iden;
  const double dV = (g1 * W * (D * W - 2.0 * (tau + D)) + D) * (iden * iden);
  const double iW = rcp_mixed(W);
  const double iW2 = iW * iW;
  res = (V * V) * (1.0 - iW2) - Q2;
  dres = 2.0 * V * (dV * (W2 * W - W) + V) * (iW2 * iW);
}
// the reference's starting point for Newton (the bracket midpoint): no seed
struct NoSeed {
  static constexpr bool seeded = false;
  __device__ __forceinline__ double operator()() const { return 0.0; }
};

// equations.f90:343-424 (per-call locals reproduce the reference: its SAVE'd d, e are
// written in the first iteration before being read)
__device__ inline double root_brent(double g1, double rho_floor, double D, double tau, double Q2) {
  const double EPS = 3.0e-8, x_acc = 1.0e-8, x1 = 1.0;
  const double Wg = (sqrt(Q2) + D) / rmax(D, rho_floor);
  const double x2 = rmax(1.0e4, Wg * 2.0);
  double a, b, c, d = 0.0, e = 0.0, fa, fb, fc, o, q, r, y1, tol1, xm, df;
  residual(g1, x1, D, tau, Q2, fa, df);
  residual(g1, x2, D, tau, Q2, fb, df);
  if (sgn1(fa) * sgn1(fb) > 0.0) return -1.0;
  a = x1; b = x2; c = b; fc = fb;
  for (int it = 0; it < 100; ++it) {
    if (sgn1(fb) * sgn1(fc) > 0.0) { c = a; fc = fa; d = b - a; e = d; }
    if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
    tol1 = 2.0 * EPS * fabs(b) + 0.5 * x_acc;
    xm = 0.5 * (c - b);
    if (fabs(xm) <= tol1 || fabs(fb) < 1.0e-14) return b;
    if (fabs(e) >= tol1 && fabs(fa) > fabs(fb)) {
      y1 = fb / fa;
      if (fabs(a - c) < 1.0e-14) { o = 2.0 * xm * y1; q = 1.0 - y1; }
      else {
        q = fa / fc; r = fb / fc;
        o = y1 * (2.0 * xm * q * (q - r) - (b - a) * (r - 1.0));
        q = (q - 1.0) * (r - 1.0) * (y1 - 1.0);
      }
      if (o > 0.0) q = -q;
      o = fabs(o);
      if (2.0 * o < rmin(3.0 * xm * q - fabs(tol1 * q), fabs(e * q))) { e = d; d = o / q; }
      else { d = xm; e = d; }
    } else { d = xm; e = d; }
    a = b; fa = fb;
    if (fabs(d) > tol1) b = b + d; else b = b + copysign(tol1, xm);
    residual(g1, b, D, tau, Q2, fb, df);
  }
  return -1.0;
}
// equations.f90:249-340
__device__ inline double root_safe_newton(double g1, double rho_floor, double D, double tau, double Q2, unsigned &flags) {
  const double x_acc = 1.0e-10, x1 = 1.0;
  double f_low, f_high, df, f, root, dx, dx_old, tmp;
  residual(g1, x1, D, tau, Q2, f_low, df);
  // The reference evaluates the upper end before this test; nothing of it reaches the
  // return, so a cell at rest in the atmosphere (f(1) = -Q2 ~ 0) skips it.
  if (fabs(f_low) < 1.0e-14) return x1;
  const double Wg = (sqrt(Q2) + D) / rmax(D, rho_floor);
  const double x2 = rmax(1.0e3, Wg * 2.0);
  double x_low = x1, x_high = x2;
  residual(g1, x2, D, tau, Q2, f_high, df);
  if (fabs(f_high) < 1.0e-14) return x_high;
  if (sgn1(f_low) * sgn1(f_high) > 0.0) return -1.0;
  if (f_low < 0.0) { x_low = x1; x_high = x2; } else { x_high = x1; x_low = x2; }
  root = 0.5 * (x1 + x2);
  dx_old = fabs(x2 - x1);
  dx = dx_old;
  residual(g1, root, D, tau, Q2, f, df);
  for (int it = 0; it < 100; ++it) {
    if (((root - x_high) * df - f) * ((root - x_low) * df - f) > 0.0 || fabs(2.0 * f) > fabs(dx_old * df)) {
      dx_old = dx;
      dx = 0.5 * (x_high - x_low);
      root = x_low + dx;
      if (fabs(x_low - root) < 1.0e-14) return root;
    } else {
      dx_old = dx;
      dx = f / df;
      tmp = root;
      root = root - dx;
      if (fabs(tmp - root) < 1.0e-14) return root;
    }
    if (fabs(dx) < x_acc) return root;
    residual(g1, root, D, tau, Q2, f, df);
    if (f < 0.0) x_low = root; else x_high = root;
  }
  flags |= C2P_BRENT;
  return root_brent(g1, rho_floor, D, tau, Q2);
}

// Mixed-policy root finder: the residual and bracket [1, max(1e3, 2 W_guess)] of
// root_safe_newton (the residual with shared reciprocals), but Newton starts from the seed
// (the Lorentz factor of the cell's current primitives, a few 1e-3 off the root after one
// stage, evaluated only for a cell that reaches the root finder) instead of the bracket
// midpoint, so it converges in a few iterations instead of ~10 bisections plus Newton.
// f(1) = -Q2 <= 0 analytically (V is finite at W = 1 since g1 > 1), so the lower end needs
// no evaluation.  Not converged after 20 iterations, or no sign change at the upper end:
// the reference iteration decides (same result class as the FP64 path).
template <class Seed>
__device__ inline double root_seeded_newton(double g1, double rho_floor, double D, double tau, double Q2,
                                            const Seed &seed, unsigned &flags) {
  const double x_acc = 1.0e-10;
  if (Q2 < 1.0e-14) return 1.0;  // root_safe_newton: |f(1)| = Q2 < 1e-14 returns W = 1
  const double W_seed = seed();
  const double Wg = (sqrt(Q2) + D) * rcp_mixed(rmax(D, rho_floor));
  const double x2 = rmax(1.0e3, Wg * 2.0);
  double lo = 1.0, hi = x2;
  double root = (W_seed > 1.0 && W_seed < x2) ? W_seed : 0.5 * (1.0 + x2);
  double f, df;
  bool hi_checked = false;
  for (int it = 0; it < 20; ++it) {
    residual_mixed(g1, root, D, tau, Q2, f, df);
    if (!(f == f) || !(df == df)) break;
    if (f < 0.0) lo = root; else { hi = root; hi_checked = true; }
    double next = root - f / df;
    if (fabs(next - root) < x_acc) return next;  // converged Newton step
    if (!(next > lo && next < hi)) {             // outside the bracket: bisect
      if (!hi_checked) {                         // confirm the upper end brackets the root first
        double fh, dfh;
        residual_mixed(g1, x2, D, tau, Q2, fh, dfh);
        if (!(fh > 0.0)) break;
        hi_checked = true;
      }
      next = 0.5 * (lo + hi);
      if (fabs(next - root) < x_acc) return next;
    }
    root = next;
  }
  return root_safe_newton(g1, rho_floor, D, tau, Q2, flags);
}

// cons_to_prim, equations.f90:94-205: cons modified in place (intent(inout)); returns flags.
// A seed (Seed::seeded) selects the mixed policy's root finder and its primitive recovery
// with shared reciprocals; the FP64 path passes NoSeed and follows the reference exactly.
template <class M, class Seed = NoSeed>
__device__ inline unsigned cons_to_prim(const Phys &P, const M &m, double (&cs)[NEQ], double (&pr)[NEQ],
                                        const Seed &seed = Seed()) {
  unsigned flags = 0;
  const double lDf = P.rho_floor * m.sqg();
  const double lTf = P.p_floor * (P.g1 - 1.0) * m.sqg();
  bool floor_state = false;
  if (cs[EQ_DE] <= lDf) {
    flags |= C2P_FLOOR_PRE;
    floor_state = true;
  } else {
    const double S1 = cs[EQ_VX], S2 = cs[EQ_VY], S3 = cs[EQ_VZ];
    const double S_sq = S1 * (m.i11() * S1 + m.i12() * S2 + m.i13() * S3) + S2 * (m.i12() * S1 + m.i22() * S2 + m.i23() * S3) +
                        S3 * (m.i13() * S1 + m.i23() * S2 + m.i33() * S3);
    const double E = cs[EQ_PR] + cs[EQ_DE];
    const double S_sq_max = rmax(0.0, E * E - cs[EQ_DE] * cs[EQ_DE]) * P.v_max;
    if (S_sq > S_sq_max && S_sq > 1.0e-20) {
      flags |= C2P_CAUSAL;
      const double sf = sqrt(S_sq_max / S_sq);
      cs[EQ_VX] = cs[EQ_VX] * sf;
      cs[EQ_VY] = cs[EQ_VY] * sf;
      cs[EQ_VZ] = cs[EQ_VZ] * sf;
    }
    const double D = cs[EQ_DE], tau = cs[EQ_PR];
    const double Q2 = qsq(m, cs[EQ_VX], cs[EQ_VY], cs[EQ_VZ]);
    double W;
    if (Seed::seeded) W = root_seeded_newton(P.g1, P.rho_floor, D, tau, Q2, seed, flags);
    else W = root_safe_newton(P.g1, P.rho_floor, D, tau, Q2, flags);
    if (W < 1.0) {
      flags |= C2P_ROOT_FAIL;
      floor_state = true;
    } else {
      const double den = P.g1 * (W * W) - 1.0;
      const double V = Seed::seeded ? (P.g1 * (W * W) * (tau + D) - D * W) * rcp_mixed(den)
                                    : (P.g1 * (W * W) * (tau + D) - D * W) / den;
      if (V <= 0.0 || isnan(V)) {
        flags |= C2P_BAD_V;
        floor_state = true;
      } else {
        const double s1 = cs[EQ_VX], s2 = cs[EQ_VY], s3 = cs[EQ_VZ];
        if (Seed::seeded) {  // mixed policy: one reciprocal of V and one of sqrt(gamma)
          const double isq = rcp_mixed(m.sqg()), iV = rcp_mixed(V);
          pr[EQ_DE] = D * rcp_mixed(W) * isq;
          pr[EQ_PR] = (V - tau - D) * isq;
          pr[EQ_VX] = (m.i11() * s1 + m.i12() * s2 + m.i13() * s3) * iV;
          pr[EQ_VY] = (m.i12() * s1 + m.i22() * s2 + m.i23() * s3) * iV;
          pr[EQ_VZ] = (m.i13() * s1 + m.i23() * s2 + m.i33() * s3) * iV;
        } else {
          pr[EQ_DE] = D / (W * m.sqg());
          pr[EQ_PR] = (V - tau - D) / m.sqg();
          pr[EQ_VX] = div_pos(m.i11() * s1 + m.i12() * s2 + m.i13() * s3, V);  // V > 0 here
          pr[EQ_VY] = div_pos(m.i12() * s1 + m.i22() * s2 + m.i23() * s3, V);
          pr[EQ_VZ] = div_pos(m.i13() * s1 + m.i23() * s2 + m.i33() * s3, V);
        }
        const double a = pr[EQ_VX], b = pr[EQ_VY], c = pr[EQ_VZ];
        double vsf = 0.0;
        vsf = vsf + m.g11() * a * a; vsf = vsf + m.g12() * a * b; vsf = vsf + m.g13() * a * c;
        vsf = vsf + m.g12() * b * a; vsf = vsf + m.g22() * b * b; vsf = vsf + m.g23() * b * c;
        vsf = vsf + m.g13() * c * a; vsf = vsf + m.g23() * c * b; vsf = vsf + m.g33() * c * c;
        if (pr[EQ_DE] < P.rho_floor || pr[EQ_PR] < P.p_floor || isnan(pr[EQ_DE]) || isnan(pr[EQ_PR]) ||
            isnan(a) || isnan(b) || isnan(c) || isnan(vsf) || vsf >= P.v_max) {
          flags |= C2P_SANITISE;
          floor_state = true;
        }
      }
    }
  }
  if (floor_state) {
    pr[EQ_DE] = P.rho_floor; pr[EQ_PR] = P.p_floor; pr[EQ_VX] = 0.0; pr[EQ_VY] = 0.0; pr[EQ_VZ] = 0.0;
    cs[EQ_DE] = lDf; cs[EQ_PR] = lTf; cs[EQ_VX] = 0.0; cs[EQ_VY] = 0.0; cs[EQ_VZ] = 0.0;
  }
  return flags;
}

// prim_to_cons, equations.f90:30-88 (FP64)
__device__ __forceinline__ void prim_to_cons(const Phys &P, const CellMetric &m, const double (&q)[NEQ], double (&u)[NEQ]) {
  FaceMetric<double> fm;
  fm.g11 = m.g11(); fm.g12 = m.g12(); fm.g13 = m.g13(); fm.g22 = m.g22(); fm.g23 = m.g23(); fm.g33 = m.g33();
  double v[3] = {q[EQ_VX], q[EQ_VY], q[EQ_VZ]}, vc[3];
  const double vsq = cap_velocity(fm, v, P.v_max);
  lower(fm, v, vc);
  const double h = 1.0 + P.g1 * q[EQ_PR] / q[EQ_DE];
  const double W = 1.0 / sqrt(1.0 - vsq);
  const double rhW2 = q[EQ_DE] * h * (W * W);
  u[EQ_DE] = q[EQ_DE] * W;
  u[EQ_PR] = rhW2 - q[EQ_PR] - q[EQ_DE] * W;
  u[EQ_VX] = rhW2 * vc[0];
  u[EQ_VY] = rhW2 * vc[1];
  u[EQ_VZ] = rhW2 * vc[2];
#pragma unroll
  for (int n = 0; n < NEQ; ++n) u[n] = u[n] * m.sqg();
}

}  // namespace grhd
