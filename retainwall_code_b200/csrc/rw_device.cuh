// Device-side algebra, SPH kernel functions and constitutive models of the step.
//
// The semantics follow the reference's float build exactly where it matters for
// parity: expressions in which the reference's double literals (2.0, 3.0, 0.5, ...)
// promote scalar operands to double are evaluated in double here too, and scalar
// transcendentals use the float overloads the reference's device code resolves to
// (src/functions.h, src/constitutive_model.h).  For T = double everything is double.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "rw_params.h"

namespace rw {

template <class T> struct alignas(4 * sizeof(T)) V4 { T x, y, z, w; };
template <class T> struct alignas(2 * sizeof(T)) V2 { T x, y; };
template <class T> struct V3 { T x, y, z; };
template <class T> struct S6 { T xx, yy, zz, xy, xz, yz; };
template <class T> struct F9 { T xx, xy, xz, yx, yy, yz, zx, zy, zz; };
struct I3 { int x, y, z; };

#define RWD __device__ __forceinline__
#define RWHD __host__ __device__ __forceinline__

template <class T> RWD V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> RWD V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> RWD V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> RWD V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> RWD V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> RWD V3<T> mulI(I3 c, T s) { return {(T)c.x * s, (T)c.y * s, (T)c.z * s}; }
template <class T> RWD V4<T> operator+(V4<T> a, V4<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class T> RWD V4<T> operator*(V4<T> a, T s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class T> RWD V4<T> add3(V4<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w}; }
template <class T> RWD V4<T> sub3(V4<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w}; }
template <class T> RWD V3<T> xyz(V4<T> a) { return {a.x, a.y, a.z}; }
template <class T> RWD V4<T> v4(V3<T> a, T w) { return {a.x, a.y, a.z, w}; }
template <class T> RWD T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> RWD V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

RWD float f_sqrt(float x) { return sqrtf(x); }
RWD double f_sqrt(double x) { return sqrt(x); }
RWD float f_rsqrt(float x) { return rsqrtf(x); }
RWD double f_rsqrt(double x) { return rsqrt(x); }
RWD float f_fma(float a, float b, float c) { return fmaf(a, b, c); }
RWD double f_fma(double a, double b, double c) { return fma(a, b, c); }
// Quotient through the hardware reciprocal (float) or the correctly rounded divide (double).
RWD float f_fastdiv(float a, float b) { return __fdividef(a, b); }
RWD double f_fastdiv(double a, double b) { return a / b; }
RWD float f_pow(float a, float b) { return powf(a, b); }
RWD double f_pow(double a, double b) { return pow(a, b); }
RWD float f_exp(float a) { return expf(a); }
RWD double f_exp(double a) { return exp(a); }
RWD float f_sin(float a) { return sinf(a); }
RWD double f_sin(double a) { return sin(a); }
RWD float f_cos(float a) { return cosf(a); }
RWD double f_cos(double a) { return cos(a); }
RWD float f_abs(float a) { return fabsf(a); }
RWD double f_abs(double a) { return fabs(a); }
RWD float f_max(float a, float b) { return fmaxf(a, b); }
RWD double f_max(double a, double b) { return fmax(a, b); }
RWD float f_min(float a, float b) { return fminf(a, b); }
RWD double f_min(double a, double b) { return fmin(a, b); }

// EulerianNorm (src/functions.h:105).
template <class T> RWD T enorm(V3<T> v) { return f_sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

// |dr| for the pair tests: round-to-nearest float squares and sums (no fused
// multiply-add) and an IEEE square root, so every device and the CPU restatement
// obtain the same r and therefore the same q < 2 neighbour sets.  (The reference
// calls norm3df, which is within a couple of ulp of this.)
RWD float pair_r2(float x, float y, float z) {
  return __fadd_rn(__fadd_rn(__fmul_rn(x, x), __fmul_rn(y, y)), __fmul_rn(z, z));
}
RWD double pair_r2(double x, double y, double z) {
  return __dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z));
}
RWD float pair_r(float r2) { return __fsqrt_rn(r2); }
RWD double pair_r(double r2) { return __dsqrt_rn(r2); }

// Arithmetic policy of the pair loop.  Every product is an explicit round-to-nearest
// multiply, so the compiler cannot fuse it differently in different kernels:
// Strict = false fuses multiply-adds (fma) at fixed places; Strict = true rounds every
// product and sum separately, i.e. exactly the written evaluation order of the
// reference's expressions (and of the CPU restatement).
template <bool Strict> struct Fp {
  static RWD float mul(float a, float b) { return __fmul_rn(a, b); }
  static RWD double mul(double a, double b) { return __dmul_rn(a, b); }
  static RWD float mad(float a, float b, float c) { return Strict ? __fadd_rn(__fmul_rn(a, b), c) : __fmaf_rn(a, b, c); }
  static RWD double mad(double a, double b, double c) { return Strict ? __dadd_rn(__dmul_rn(a, b), c) : __fma_rn(a, b, c); }
  // c - a*b
  static RWD float msub(float a, float b, float c) { return Strict ? __fsub_rn(c, __fmul_rn(a, b)) : __fmaf_rn(-a, b, c); }
  static RWD double msub(double a, double b, double c) { return Strict ? __dsub_rn(c, __dmul_rn(a, b)) : __fma_rn(-a, b, c); }
  // a.x*b.x + a.y*b.y + a.z*b.z, left to right
  template <class T> static RWD T dot3(T ax, T ay, T az, T bx, T by, T bz) { return mad(az, bz, mad(ay, by, mul(ax, bx))); }
};

// Wendland C2 (src/functions.h:142-143): GetKernel is a double expression in the
// float build (its 2.0 / 0.5 literals), GetGradKernel stays in scalar.
template <class T> RWD T kernel_w(T par, T q) {
  double t = 2.0 - (double)q;
  return (T)((double)par * t * t * t * t * ((double)q + 0.5));
}
template <class T> RWD T kernel_f(T par, T q) {
  T t = T(2.0f) - q;
  return par * t * t * t;
}

template <class T> RWD S6<T> operator+(S6<T> a, S6<T> b) {
  return {a.xx + b.xx, a.yy + b.yy, a.zz + b.zz, a.xy + b.xy, a.xz + b.xz, a.yz + b.yz};
}
template <class T> RWD S6<T> operator-(S6<T> a, S6<T> b) {
  return {a.xx - b.xx, a.yy - b.yy, a.zz - b.zz, a.xy - b.xy, a.xz - b.xz, a.yz - b.yz};
}
template <class T> RWD S6<T> operator*(S6<T> a, T s) {
  return {a.xx * s, a.yy * s, a.zz * s, a.xy * s, a.xz * s, a.yz * s};
}
template <class T> RWD S6<T> operator/(S6<T> a, T s) {
  return {a.xx / s, a.yy / s, a.zz / s, a.xy / s, a.xz / s, a.yz / s};
}
template <class T> RWD S6<T> zero6() { return {T(0), T(0), T(0), T(0), T(0), T(0)}; }
template <class T> RWD S6<T> ident6() { return {T(1), T(1), T(1), T(0), T(0), T(0)}; }
template <class T> RWD T trace(S6<T> v) { return v.xx + v.yy + v.zz; }
// trace(v1, v2) / J2 of src/functions.h:101-108: the 2.0 literals make the
// off-diagonal part, and the sum from there on, double in the float build.
template <class T> RWD T trace2(S6<T> a, S6<T> b) {
  T s = a.xx * b.xx + a.yy * b.yy + a.zz * b.zz;
  double d = (double)s + 2.0 * (double)a.xy * (double)b.xy;
  d = d + 2.0 * (double)a.xz * (double)b.xz;
  d = d + 2.0 * (double)a.yz * (double)b.yz;
  return (T)d;
}
template <class T> RWD V3<T> dotSV(S6<T> a, V3<T> b) {
  return {a.xx * b.x + a.xy * b.y + a.xz * b.z, a.xy * b.x + a.yy * b.y + a.yz * b.z,
          a.xz * b.x + a.yz * b.y + a.zz * b.z};
}
template <class T> RWD S6<T> subdiag(S6<T> a, V3<T> v) { return {a.xx - v.x, a.yy - v.y, a.zz - v.z, a.xy, a.xz, a.yz}; }

template <class T> RWD F9<T> operator-(F9<T> a, F9<T> b) {
  return {a.xx - b.xx, a.xy - b.xy, a.xz - b.xz, a.yx - b.yx, a.yy - b.yy,
          a.yz - b.yz, a.zx - b.zx, a.zy - b.zy, a.zz - b.zz};
}
template <class T> RWD F9<T> operator+(F9<T> a, F9<T> b) {
  return {a.xx + b.xx, a.xy + b.xy, a.xz + b.xz, a.yx + b.yx, a.yy + b.yy,
          a.yz + b.yz, a.zx + b.zx, a.zy + b.zy, a.zz + b.zz};
}
template <class T> RWD F9<T> operator*(F9<T> a, T s) {
  return {a.xx * s, a.xy * s, a.xz * s, a.yx * s, a.yy * s, a.yz * s, a.zx * s, a.zy * s, a.zz * s};
}
template <class T> RWD F9<T> identF() { return {T(1), T(0), T(0), T(0), T(1), T(0), T(0), T(0), T(1)}; }
template <class T> RWD F9<T> skew2full(V3<T> v) { return {T(0), -v.z, v.y, v.z, T(0), -v.x, -v.y, v.x, T(0)}; }
template <class T> RWD F9<T> sym2full(S6<T> v) { return {v.xx, v.xy, v.xz, v.xy, v.yy, v.yz, v.xz, v.yz, v.zz}; }
template <class T> RWD S6<T> full2sym(F9<T> v) {
  return {v.xx, v.yy, v.zz, T(0.5f) * (v.xy + v.yx), T(0.5f) * (v.xz + v.zx), T(0.5f) * (v.yz + v.zy)};
}
template <class T> RWD V3<T> skewpart(F9<T> v) {
  return {T(0.5f) * (v.yx - v.xy), T(0.5f) * (v.zx - v.xz), T(0.5f) * (v.zy - v.yz)};
}
template <class T> RWD F9<T> lin(F9<T> a, F9<T> b) {
  return {a.xx * b.xx + a.xy * b.yx + a.xz * b.zx, a.xx * b.xy + a.xy * b.yy + a.xz * b.zy,
          a.xx * b.xz + a.xy * b.yz + a.xz * b.zz, a.yx * b.xx + a.yy * b.yx + a.yz * b.zx,
          a.yx * b.xy + a.yy * b.yy + a.yz * b.zy, a.yx * b.xz + a.yy * b.yz + a.yz * b.zz,
          a.zx * b.xx + a.zy * b.yx + a.zz * b.zx, a.zx * b.xy + a.zy * b.yy + a.zz * b.zy,
          a.zx * b.xz + a.zy * b.yz + a.zz * b.zz};
}
template <class T> RWD V3<T> dotFV(F9<T> a, V3<T> b) {
  return {a.xx * b.x + a.xy * b.y + a.xz * b.z, a.yx * b.x + a.yy * b.y + a.yz * b.z,
          a.zx * b.x + a.zy * b.y + a.zz * b.z};
}
// GetRodriguesMatrix (src/functions.h:125-131).
template <class T> RWD F9<T> rodrigues(V3<T> angle) {
  T na = enorm(angle);
  V3<T> axis = angle / na;
  F9<T> K = skew2full(axis);
  T omc = (T)(1.0 - (double)f_cos(na));
  return identF<T>() + K * f_sin(na) + lin(K, K) * omc;
}

// ---------------------------------------------------------------------------------
// Constitutive models (src/constitutive_model.h).
// ---------------------------------------------------------------------------------
template <class T> RWD S6<T> jaumann(V3<T> om, F9<T> sf) {
  F9<T> spin = skew2full(om);
  return full2sym(lin(spin, sf) - lin(sf, spin));
}

// cuMatModDP, src/constitutive_model.h:38-84.
template <class T> RWD void mat_dp(T dt, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp, bool& yld) {
  S6<T> jau = jaumann(om, sym2full(sigma));
  T bulk = mp[0], shear = mp[1];
  T lame = (T)((double)bulk - 2.0 / 3.0 * (double)shear);
  S6<T> rate = jau + D * (T)(2.0 * (double)shear) + ident6<T>() * (lame * trace(D));
  S6<T> pre = sigma + rate * dt;
  T sph = (T)((double)trace(pre) / 3.0);
  S6<T> dev = pre - ident6<T>() * (T)((double)trace(pre) / 3.0);
  T k_psi = mp[3], k_c = mp[4], k_phi = mp[2];
  T tenlt = (k_phi == T(0)) ? T(0) : k_c / k_phi;
  if (sph - tenlt >= T(0)) sph = tenlt;
  T tau = f_sqrt((T)(0.5 * (double)trace2(dev, dev)));
  T shr = tau - (-sph * k_phi + k_c);
  if (shr > T(0)) {
    T dl = shr / (shear + bulk * k_phi * k_psi);
    sph -= bulk * k_psi * dl;
    T ratio = (T)(tau < 1e-10 ? 1.0 : (double)((k_c - k_phi * sph) / tau));
    dev = dev * ratio;
    yld = true;
  }
  sigma = dev + ident6<T>() * sph;
}

// cuMatModMuIDP, src/constitutive_model.h:90-130.
template <class T> RWD void mat_muidp(T dt, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp) {
  S6<T> jau = jaumann(om, sym2full(sigma));
  T bulk = mp[0], shear = mp[1];
  T lame = (T)((double)bulk - 2.0 / 3.0 * (double)shear);
  S6<T> rate = jau + D * (T)(2.0 * (double)shear) + ident6<T>() * (lame * trace(D));
  S6<T> pre = sigma + rate * dt;
  T sph = (T)((double)trace(pre) / 3.0);
  S6<T> dev = pre - ident6<T>() * (T)((double)trace(pre) / 3.0);
  S6<T> Ddev = D - ident6<T>() * (T)((double)trace(D) / 3.0);
  T gamma = (T)sqrt(2.0 * (double)trace2(Ddev, Ddev));
  if (sph > T(0)) sph = T(0);
  T mu_s = mp[2], dmu = mp[3] - mp[2], I0 = mp[4], rho_g = mp[5], dg = mp[6], lam = mp[7];
  T pressure = -sph;
  T mu = mu_s + dmu * gamma * dg / (I0 * f_sqrt(pressure / rho_g) + dg * f_sqrt(gamma * gamma + lam * lam));
  T tau = (T)sqrt(0.5 * (double)trace2(dev, dev));
  if (tau + sph * mu > T(0)) {
    T ratio = (T)(tau < 1e-10 ? 1.0 : (0.0 - (double)(mu * sph)) / (double)tau);
    dev = dev * ratio;
  }
  sigma = dev + ident6<T>() * sph;
}

// Material constants of the hypoplastic update (HypoC, rw_params.h): C1..C4 and a of
// src/constitutive_model.h:149-153 and :226-230, and the ratios fa, fb, fc and t1 of the
// cone projection (:276-279).  They depend on the material only, so the step evaluates
// them once per material on the device (Params::hypo) with these same expressions.
template <class T> RWD HypoC<T> hypo_coef(T Ei, T Vi, T phi_c, T p_ref) {
  HypoC<T> c;
  c.C1 = (T)(-(double)Ei / (3.0 * (double)p_ref * (double)(T(1) + Vi)));
  c.a = (T)(3.0 / (sqrt(2.0) * (double)f_sin(phi_c)));
  c.C2 = (T)((double)c.C1 * ((3.0 * (double)Vi + (double)c.a * sqrt(1.0 + (double)(Vi * Vi))) / (double)(T(1) - Vi) -
                             (double)(c.a * c.a) / 3.0));
  c.C3 = c.a * c.a * c.C1;
  c.C4 = c.a * c.C1;
  c.fa = c.C2 / c.C1;
  c.fb = c.C3 / c.C1;
  c.fc = c.C4 / c.C1;
  c.t1 = 1.0 + (double)c.fa + (double)c.fb / 3.0;
  return c;
}
template <class T> RWD HypoC<T> hypo_coef(const T* mp, const HypoC<T>* pre) {
  return pre ? *pre : hypo_coef(mp[0], mp[1], mp[2], mp[4]);
}

// cuMatModHypo (basic), src/constitutive_model.h:136-202.
template <class T> RWD void mat_hypo_basic(T dt, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp, bool dnorm = false,
                                           const HypoC<T>* pre = nullptr) {
  T coh = mp[3];
  HypoC<T> c = hypo_coef(mp, pre);
  F9<T> sf = sym2full(sigma);
  if (coh > T(0)) sf = sf - identF<T>() * coh;
  S6<T> jau = jaumann(om, sf);
  S6<T> str = full2sym(sf);
  T I1 = trace(str);
  if ((double)I1 > -4.0) {
    sigma = {T(-1), T(-1), T(-2), T(0), T(0), T(0)};
    return;
  }
  S6<T> dev = str - ident6<T>() * (T)((double)I1 / 3.0);
  T tr_str = trace(str), tr_D = trace(D), tr_sD = trace2(str, D);
  T nD = rate_norm(D, dnorm);
  S6<T> rate = jau + D * (c.C1 * tr_str) + str * (c.C2 * tr_D) + str * (c.C3 * tr_sD / tr_str) + (str + dev) * (c.C4 * nD);
  str = sigma + rate * dt;
  T sph = (T)((double)trace(str) / 3.0);
  if ((double)sph > 0.0) {
    sigma = {(T)(-1.0 + (double)coh), (T)(-1.0 + (double)coh), (T)(-2.0 + (double)coh), T(0), T(0), T(0)};
    return;
  }
  dev = str - ident6<T>() * sph;
  T k_phi = (T)(3.0 / (sqrt(2.0) * (double)c.a));
  T tau = f_sqrt((T)(0.5 * (double)trace2(dev, dev)));
  if (tau - (-sph * k_phi) > T(0)) {
    T ratio = (T)(tau < 1e-10 ? 1.0 : (double)((-k_phi * sph) / tau));
    dev = dev * ratio;
  }
  sigma = dev + ident6<T>() * (sph + coh);
}

// cuMatModHypo (critical state, HypoCS), src/constitutive_model.h:209-299, in three
// pieces so that the learned closure can replace the objective stress rate alone:
// hypo_cs_pre (state quantities, :211-264), hypo_cs_rate (:269, Jaumann term first, in
// the reference's order) and hypo_cs_post (tension cut-off and cone projection, :270-298).
template <class T> struct HypoPre {
  S6<T> str, dev, jau;
  T tr_str, tr_D, tr_sD, nD, p, e, e_crt, fd, coh;
  HypoC<T> c;
};

// false: the zero-stress reset branch (I1 > -4) was taken and sigma is final.
template <class T> RWD bool hypo_cs_pre(T density, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp, T& M_crt, bool dnorm,
                                        HypoPre<T>& h, const HypoC<T>* pre = nullptr) {
  T coh = mp[3], p_ref = mp[4], void_co = mp[5], lambda = mp[6];
  T xi = mp[7], alpha = mp[8], void_min = mp[9], void_max = mp[10], void_0 = mp[11], rho0 = mp[12];
  h.c = hypo_coef(mp, pre);
  h.coh = coh;
  F9<T> sf = sym2full(sigma);
  if (coh > T(0)) sf = sf - identF<T>() * coh;
  h.jau = jaumann(om, sf);
  h.str = full2sym(sf);
  T I1 = trace(h.str);
  if ((double)I1 > -4.0) {
    sigma = {T(-1), T(-1), T(-2), T(0), T(0), T(0)};
    return false;
  }
  h.dev = h.str - ident6<T>() * (T)((double)I1 / 3.0);
  h.tr_str = trace(h.str);
  h.tr_D = trace(D);
  h.tr_sD = trace2(h.str, D);
  h.nD = rate_norm(D, dnorm);
  h.p = (T)(-(double)I1 / 3.0);
  T e = (T)((1.0 + (double)void_0) * (double)rho0 / (double)density - 1.0);
  e = f_max(e, void_min);
  h.e = f_min(e, void_max);
  h.e_crt = void_co * f_exp(-lambda * f_pow(h.p / p_ref, xi));
  h.fd = f_pow((h.e - void_min) / (h.e_crt - void_min), alpha);
  M_crt = h.e - h.e_crt;
  return true;
}

// Jaumann term plus the objective rate, as the reference sums them.
template <class T> RWD S6<T> hypo_cs_rate(const HypoPre<T>& h, S6<T> D) {
  return h.jau + D * (h.c.C1 * h.tr_str) + h.str * (h.c.C2 * h.tr_D) + h.str * (h.c.C3 * h.tr_sD / h.tr_str) +
         (h.str + h.dev) * (h.fd * h.c.C4 * h.nD);
}
// The objective rate alone (what the learned closure predicts).
template <class T> RWD S6<T> hypo_cs_objective(const HypoPre<T>& h, S6<T> D) {
  return D * (h.c.C1 * h.tr_str) + h.str * (h.c.C2 * h.tr_D) + h.str * (h.c.C3 * h.tr_sD / h.tr_str) +
         (h.str + h.dev) * (h.fd * h.c.C4 * h.nD);
}

template <class T> RWD void hypo_cs_post(T dt, const HypoPre<T>& h, S6<T> rate, S6<T>& sigma) {
  const T coh = h.coh, fd = h.fd;
  const HypoC<T>& c = h.c;
  S6<T> str = sigma + rate * dt;
  T sph = (T)((double)trace(str) / 3.0);
  if ((double)sph > 0.0) {
    sigma = {(T)(-1.0 + (double)coh), (T)(-1.0 + (double)coh), (T)(-2.0 + (double)coh), T(0), T(0), T(0)};
    return;
  }
  S6<T> dev = str - ident6<T>() * sph;
  const T fa = c.fa, fb = c.fb, fc = c.fc;
  const double t1 = c.t1;
  T A = (T)((double)(fd * fd * fc * fc) / 3.0 - t1 * t1);
  T B = (T)(2.0 * (double)fd * (double)fd * (double)fc * (double)fc * (t1 * t1 + 2.0 * (double)fa + 3.0) -
            4.0 * (double)fb * ((double)(T(1) + fa) + (double)fb / 3.0));
  T C = (T)(4.0 / 3.0 * (double)fd * (double)fd * (double)fc * (double)fc * (double)fb * (double)fb -
            4.0 * (double)fb * (double)fb);
  T k2 = (T)((-(double)B - sqrt((double)(B * B) - 4.0 * (double)A * (double)C)) / (2.0 * (double)A));
  T k_phi = (T)(3.0 / (double)f_sqrt(k2));
  T tau = f_sqrt((T)(0.5 * (double)trace2(dev, dev)));
  if (tau - (-sph * k_phi) > T(0)) {
    T ratio = (T)(tau < 1e-10 ? 1.0 : (double)((-k_phi * sph) / tau));
    dev = dev * ratio;
  }
  sigma = dev + ident6<T>() * (sph + coh);
}

template <class T> RWD void mat_hypo_cs(T dt, T density, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp, T& M_crt,
                                        bool dnorm = false, const HypoC<T>* pre = nullptr) {
  HypoPre<T> h;
  if (!hypo_cs_pre(density, om, D, sigma, mp, M_crt, dnorm, h, pre)) return;
  hypo_cs_post(dt, h, hypo_cs_rate(h, D), sigma);
}

// Strain-rate norm sqrt(D:D).  The precision form evaluates it in double (the
// survey's "hypoplastic substep norm"); otherwise the reference's scalar sqrt.
template <class T> RWD T rate_norm(S6<T> D, bool dnorm) {
  if (!dnorm) return f_sqrt(trace2(D, D));
  const double d = (double)D.xx * D.xx + (double)D.yy * D.yy + (double)D.zz * D.zz +
                   2.0 * ((double)D.xy * D.xy + (double)D.xz * D.xz + (double)D.yz * D.yz);
  return (T)sqrt(d);
}

// Model dispatch of cuPredictorMaterial / cuCorrectorMaterial
// (src/predictor_corrector.cu:72-75, :169-172).
template <class T> RWD void constitutive(int model, const T* mp, T dt, T rho, V3<T> om, S6<T> D, S6<T>& sig,
                                         bool& yld, T& M_crt, bool dnorm = false, const HypoC<T>* pre = nullptr) {
  if (model == RW_MODEL_DP) mat_dp(dt, om, D, sig, mp, yld);
  else if (model == RW_MODEL_MUIDP) mat_muidp(dt, om, D, sig, mp);
  else if (model == RW_MODEL_HYPO_BASIC) mat_hypo_basic(dt, om, D, sig, mp, dnorm, pre);
  else if (model == RW_MODEL_HYPO_CS) mat_hypo_cs(dt, rho, om, D, sig, mp, M_crt, dnorm, pre);
}

// Compensated (Kahan) accumulation s += x with running compensation c.  Explicit
// round-to-nearest operations so the compensation is not optimised away.
RWD void kahan_add(float& s, float& c, float x) {
  const float y = __fsub_rn(x, c);
  const float t = __fadd_rn(s, y);
  c = __fsub_rn(__fsub_rn(t, s), y);
  s = t;
}
RWD void kahan_add(double& s, double& c, double x) {
  const double y = __dsub_rn(x, c);
  const double t = __dadd_rn(s, y);
  c = __dsub_rn(__dsub_rn(t, s), y);
  s = t;
}

}  // namespace rw
