// ORACLE - test infrastructure, not product code.  Only tests/, __graft_entry__.smoke()
// and bench.py's CPU baseline load this library (oracle/librw_oracle.so).
//
// A plain C++/OpenMP restatement of the reference's SPH geomechanics step
// (Xshuaizhang/Retainwall_code), written for a CPU and kept line-for-line close to the
// reference's arithmetic, including where the reference's float build promotes to
// double through double literals.  Every function names the reference lines it follows.
// Data layout is the reference's array-of-structures layout.  Deliberate, documented
// departures from the reference:
//   * r = |dr| is sqrtf of the float sum of squares (the reference calls CUDA's norm3df);
//   * the contact-force redistribution reads the other particles' contact state as it
//     was when the interaction stage started (the reference reads it while other
//     threads rewrite it, src/particle_interaction.cu:147-166 vs :160-161,:233-235);
//   * the gather-permute reads every permuted array from a full copy (the reference's
//     shared cache leaves stale values for tail particles after a deletion,
//     src/loquat_grid.cu:193-251 with sizes from src/loquat.cu:254-287).
// Compile with -ffp-contract=off so the written evaluation order is the one executed.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

#include "../include/retainwall.h"

namespace orc {

// Dynamic-schedule parallel loop over [0, n) on std::thread workers (no OpenMP runtime
// dependency).  fn(i) must only write data owned by index i.
static int g_threads = 0;
template <class F> void parallel_for(int n, int chunk, F fn) {
  int nt = g_threads > 0 ? g_threads : (int)std::max(1u, std::thread::hardware_concurrency());
  if (nt <= 1 || n <= chunk) {
    for (int i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int> next{0};
  auto work = [&]() {
    for (;;) {
      int b = next.fetch_add(chunk);
      if (b >= n) break;
      int e = std::min(n, b + chunk);
      for (int i = b; i < e; ++i) fn(i);
    }
  };
  std::vector<std::thread> th;
  th.reserve(nt - 1);
  for (int k = 1; k < nt; ++k) th.emplace_back(work);
  work();
  for (auto& t : th) t.join();
}

// ---------------------------------------------------------------------------------
// Small algebra with the reference's semantics (src/functions.h:33-143).
// ---------------------------------------------------------------------------------
template <class T> struct V3 { T x, y, z; };
template <class T> struct V4 { T x, y, z, w; };
template <class T> struct S6 { T xx, yy, zz, xy, xz, yz; };
template <class T> struct F9 { T xx, xy, xz, yx, yy, yz, zx, zy, zz; };
struct I4 { int x, y, z, w; };
struct I3 { int x, y, z; };

template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return {a.x * s, a.y * s, a.z * s}; }
template <class T> inline V3<T> operator*(V3<T> a, V3<T> b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class T> inline V3<T> operator/(V3<T> a, T s) { return {a.x / s, a.y / s, a.z / s}; }
template <class T> inline V3<T> mulI(I3 c, T s) { return {(T)c.x * s, (T)c.y * s, (T)c.z * s}; }
template <class T> inline V4<T> operator+(V4<T> a, V4<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
template <class T> inline V4<T> operator*(V4<T> a, T s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
template <class T> inline V4<T> add3(V4<T> a, V3<T> b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w}; }
template <class T> inline V4<T> sub3(V4<T> a, V3<T> b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w}; }
template <class T> inline V3<T> xyz(V4<T> a) { return {a.x, a.y, a.z}; }
template <class T> inline V4<T> v4(V3<T> a, T w) { return {a.x, a.y, a.z, w}; }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T> inline T enorm(V3<T> v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

template <class T> inline S6<T> operator+(S6<T> a, S6<T> b) {
  return {a.xx + b.xx, a.yy + b.yy, a.zz + b.zz, a.xy + b.xy, a.xz + b.xz, a.yz + b.yz};
}
template <class T> inline S6<T> operator-(S6<T> a, S6<T> b) {
  return {a.xx - b.xx, a.yy - b.yy, a.zz - b.zz, a.xy - b.xy, a.xz - b.xz, a.yz - b.yz};
}
template <class T> inline S6<T> operator*(S6<T> a, T s) {
  return {a.xx * s, a.yy * s, a.zz * s, a.xy * s, a.xz * s, a.yz * s};
}
template <class T> inline S6<T> operator/(S6<T> a, T s) {
  return {a.xx / s, a.yy / s, a.zz / s, a.xy / s, a.xz / s, a.yz / s};
}
template <class T> inline S6<T> subdiag(S6<T> a, V3<T> v) { return {a.xx - v.x, a.yy - v.y, a.zz - v.z, a.xy, a.xz, a.yz}; }
template <class T> inline S6<T> ident() { return {T(1), T(1), T(1), T(0), T(0), T(0)}; }
template <class T> inline T trace(S6<T> v) { return v.xx + v.yy + v.zz; }
// trace(v1, v2) of src/functions.h:108: the 2.0 literals make the off-diagonal part
// (and the sum from there on) double in the float build.
template <class T> inline T trace2(S6<T> a, S6<T> b) {
  T s = a.xx * b.xx + a.yy * b.yy + a.zz * b.zz;
  double d = (double)s + 2.0 * (double)a.xy * (double)b.xy;
  d = d + 2.0 * (double)a.xz * (double)b.xz;
  d = d + 2.0 * (double)a.yz * (double)b.yz;
  return (T)d;
}
template <class T> inline T J2(S6<T> v) { return trace2(v, v); }
template <class T> inline V3<T> dotSV(S6<T> a, V3<T> b) {
  return {a.xx * b.x + a.xy * b.y + a.xz * b.z, a.xy * b.x + a.yy * b.y + a.yz * b.z,
          a.xz * b.x + a.yz * b.y + a.zz * b.z};
}
template <class T> inline V3<T> dotFV(F9<T> a, V3<T> b) {
  return {a.xx * b.x + a.xy * b.y + a.xz * b.z, a.yx * b.x + a.yy * b.y + a.yz * b.z,
          a.zx * b.x + a.zy * b.y + a.zz * b.z};
}
template <class T> inline F9<T> operator+(F9<T> a, F9<T> b) {
  return {a.xx + b.xx, a.xy + b.xy, a.xz + b.xz, a.yx + b.yx, a.yy + b.yy,
          a.yz + b.yz, a.zx + b.zx, a.zy + b.zy, a.zz + b.zz};
}
template <class T> inline F9<T> operator-(F9<T> a, F9<T> b) {
  return {a.xx - b.xx, a.xy - b.xy, a.xz - b.xz, a.yx - b.yx, a.yy - b.yy,
          a.yz - b.yz, a.zx - b.zx, a.zy - b.zy, a.zz - b.zz};
}
template <class T> inline F9<T> operator*(F9<T> a, T s) {
  return {a.xx * s, a.xy * s, a.xz * s, a.yx * s, a.yy * s, a.yz * s, a.zx * s, a.zy * s, a.zz * s};
}
template <class T> inline F9<T> identF() { return {T(1), T(0), T(0), T(0), T(1), T(0), T(0), T(0), T(1)}; }
template <class T> inline F9<T> tprod(V3<T> a, V3<T> b) {
  return {a.x * b.x, a.x * b.y, a.x * b.z, a.y * b.x, a.y * b.y, a.y * b.z, a.z * b.x, a.z * b.y, a.z * b.z};
}
template <class T> inline F9<T> skew2full(V3<T> v) { return {T(0), -v.z, v.y, v.z, T(0), -v.x, -v.y, v.x, T(0)}; }
template <class T> inline F9<T> sym2full(S6<T> v) { return {v.xx, v.xy, v.xz, v.xy, v.yy, v.yz, v.xz, v.yz, v.zz}; }
template <class T> inline S6<T> full2sym(F9<T> v) {
  return {v.xx, v.yy, v.zz, T(0.5f) * (v.xy + v.yx), T(0.5f) * (v.xz + v.zx), T(0.5f) * (v.yz + v.zy)};
}
template <class T> inline V3<T> skewpart(F9<T> v) {
  return {T(0.5f) * (v.yx - v.xy), T(0.5f) * (v.zx - v.xz), T(0.5f) * (v.zy - v.yz)};
}
template <class T> inline F9<T> lin(F9<T> a, F9<T> b) {
  return {a.xx * b.xx + a.xy * b.yx + a.xz * b.zx, a.xx * b.xy + a.xy * b.yy + a.xz * b.zy,
          a.xx * b.xz + a.xy * b.yz + a.xz * b.zz, a.yx * b.xx + a.yy * b.yx + a.yz * b.zx,
          a.yx * b.xy + a.yy * b.yy + a.yz * b.zy, a.yx * b.xz + a.yy * b.yz + a.yz * b.zz,
          a.zx * b.xx + a.zy * b.yx + a.zz * b.zx, a.zx * b.xy + a.zy * b.yy + a.zz * b.zy,
          a.zx * b.xz + a.zy * b.yz + a.zz * b.zz};
}
// GetRodriguesMatrix (src/functions.h:125-131).
template <class T> inline F9<T> rodrigues(V3<T> angle) {
  T na = enorm(angle);
  V3<T> axis = angle / na;
  F9<T> K = skew2full(axis);
  T one_minus_cos = (T)(1.0 - (double)std::cos(na));
  return identF<T>() + K * (T)std::sin(na) + lin(K, K) * one_minus_cos;
}

// Float-precision helpers: the reference's float build calls the float overloads.
template <class T> inline T m_sqrtf(T x) { return std::sqrt(x); }
template <class T> inline T m_pow(T a, T b) { return std::pow(a, b); }
template <class T> inline T m_exp(T a) { return std::exp(a); }
template <class T> inline T m_sin(T a) { return std::sin(a); }

// Wendland C2 (src/functions.h:142-143).  GetKernel's 2.0 / 0.5 literals make the
// whole product double in the float build; GetGradKernel stays in scalar.
template <class T> inline T kernel_w(T par, T q) {
  double t = 2.0 - (double)q;
  return (T)((double)par * t * t * t * t * ((double)q + 0.5));
}
template <class T> inline T kernel_f(T par, T q) {
  T t = T(2.0f) - q;
  return par * t * t * t;
}
// |dr|: sqrtf of the float sum of squares (the reference uses CUDA's norm3df).
template <class T> inline T dist(V3<T> d) { return std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z); }

// ---------------------------------------------------------------------------------
// Constitutive models (src/constitutive_model.h).
// ---------------------------------------------------------------------------------
template <class T> inline S6<T> jaumann(V3<T> om, F9<T> sf) {
  F9<T> spin = skew2full(om);
  return full2sym(lin(spin, sf) - lin(sf, spin));
}

// cuMatModDP, src/constitutive_model.h:38-84.
template <class T> void mat_dp(T dt, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp, bool& yld) {
  S6<T> jau = jaumann(om, sym2full(sigma));
  T bulk = mp[0], shear = mp[1];
  T lame = (T)((double)bulk - 2.0 / 3.0 * (double)shear);
  S6<T> rate = jau + D * (T)(2.0 * (double)shear) + ident<T>() * (lame * trace(D));
  S6<T> pre = sigma + rate * dt;
  T sph = (T)((double)trace(pre) / 3.0);
  S6<T> dev = pre - ident<T>() * (T)((double)trace(pre) / 3.0);
  T k_psi = mp[3], k_c = mp[4], k_phi = mp[2];
  T tenlt = (k_phi == T(0)) ? T(0) : k_c / k_phi;
  T tenyld = sph - tenlt;
  if (tenyld >= T(0)) sph = tenlt;
  T tau = m_sqrtf((T)(0.5 * (double)trace2(dev, dev)));
  T shr = tau - (-sph * k_phi + k_c);
  if (shr > T(0)) {
    T dl = shr / (shear + bulk * k_phi * k_psi);
    sph -= bulk * k_psi * dl;
    T ratio = (T)(tau < 1e-10 ? 1.0 : (double)((k_c - k_phi * sph) / tau));
    dev = dev * ratio;
    yld = true;
  }
  sigma = dev + ident<T>() * sph;
}

// cuMatModMuIDP, src/constitutive_model.h:90-130.
template <class T> void mat_muidp(T dt, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp) {
  S6<T> jau = jaumann(om, sym2full(sigma));
  T bulk = mp[0], shear = mp[1];
  T lame = (T)((double)bulk - 2.0 / 3.0 * (double)shear);
  S6<T> rate = jau + D * (T)(2.0 * (double)shear) + ident<T>() * (lame * trace(D));
  S6<T> pre = sigma + rate * dt;
  T sph = (T)((double)trace(pre) / 3.0);
  S6<T> dev = pre - ident<T>() * (T)((double)trace(pre) / 3.0);
  S6<T> Ddev = D - ident<T>() * (T)((double)trace(D) / 3.0);
  T gamma = (T)std::sqrt(2.0 * (double)J2(Ddev));
  if (sph > T(0)) sph = T(0);
  T mu_s = mp[2], dmu = mp[3] - mp[2], I0 = mp[4], rho_g = mp[5], dg = mp[6], lam = mp[7];
  T pressure = -sph;
  T mu = mu_s + dmu * gamma * dg / (I0 * std::sqrt(pressure / rho_g) + dg * std::sqrt(gamma * gamma + lam * lam));
  T tau = (T)std::sqrt(0.5 * (double)trace2(dev, dev));
  T shr = tau + sph * mu;
  if (shr > T(0)) {
    T ratio = (T)(tau < 1e-10 ? 1.0 : (0.0 - (double)(mu * sph)) / (double)tau);
    dev = dev * ratio;
  }
  sigma = dev + ident<T>() * sph;
}

// Shared head of both hypoplastic models: C1..C4 (src/constitutive_model.h:149-153,226-230).
template <class T> struct HypoC { T C1, a, C2, C3, C4; };
template <class T> inline HypoC<T> hypo_coef(T Ei, T Vi, T phi_c, T p_ref) {
  HypoC<T> c;
  c.C1 = (T)(-(double)Ei / (3.0 * (double)p_ref * (double)(T(1) + Vi)));
  c.a = (T)(3.0 / (std::sqrt(2.0) * (double)m_sin(phi_c)));
  c.C2 = (T)((double)c.C1 * ((3.0 * (double)Vi + (double)c.a * std::sqrt(1.0 + (double)(Vi * Vi))) / (double)(T(1) - Vi) -
                             (double)(c.a * c.a) / 3.0));
  c.C3 = c.a * c.a * c.C1;
  c.C4 = c.a * c.C1;
  return c;
}

// cuMatModHypo (basic), src/constitutive_model.h:136-202.
template <class T> void mat_hypo_basic(T dt, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp) {
  T Ei = mp[0], Vi = mp[1], phi_c = mp[2], coh = mp[3], p_ref = mp[4];
  HypoC<T> c = hypo_coef(Ei, Vi, phi_c, p_ref);
  F9<T> sf = sym2full(sigma);
  if (coh > T(0)) sf = sf - identF<T>() * coh;
  S6<T> jau = jaumann(om, sf);
  S6<T> str = full2sym(sf);
  T I1 = trace(str);
  if ((double)I1 > -4.0) {
    sigma = {T(-1), T(-1), T(-2), T(0), T(0), T(0)};
    return;
  }
  S6<T> dev = str - ident<T>() * (T)((double)I1 / 3.0);
  T tr_str = trace(str), tr_D = trace(D), tr_sD = trace2(str, D);
  T nD = m_sqrtf(trace2(D, D));
  S6<T> rate = jau + D * (c.C1 * tr_str) + str * (c.C2 * tr_D) + str * (c.C3 * tr_sD / tr_str) + (str + dev) * (c.C4 * nD);
  str = sigma + rate * dt;
  T sph = (T)((double)trace(str) / 3.0);
  if ((double)sph > 0.0) {
    sigma = {(T)(-1.0 + (double)coh), (T)(-1.0 + (double)coh), (T)(-2.0 + (double)coh), T(0), T(0), T(0)};
    return;
  }
  dev = str - ident<T>() * sph;
  T k_phi = (T)(3.0 / (std::sqrt(2.0) * (double)c.a));
  T tau = m_sqrtf((T)(0.5 * (double)trace2(dev, dev)));
  T shr = tau - (-sph * k_phi);
  if (shr > T(0)) {
    T ratio = (T)(tau < 1e-10 ? 1.0 : (double)((-k_phi * sph) / tau));
    dev = dev * ratio;
  }
  sigma = dev + ident<T>() * (sph + coh);
}

// cuMatModHypo (critical state, HypoCS), src/constitutive_model.h:209-299.
template <class T> void mat_hypo_cs(T dt, T density, V3<T> om, S6<T> D, S6<T>& sigma, const T* mp, T& M_crt) {
  T Ei = mp[0], Vi = mp[1], phi_c = mp[2], coh = mp[3], p_ref = mp[4], void_co = mp[5], lambda = mp[6];
  T xi = mp[7], alpha = mp[8], void_min = mp[9], void_max = mp[10], void_0 = mp[11], rho0 = mp[12];
  HypoC<T> c = hypo_coef(Ei, Vi, phi_c, p_ref);
  F9<T> sf = sym2full(sigma);
  if (coh > T(0)) sf = sf - identF<T>() * coh;
  S6<T> jau = jaumann(om, sf);
  S6<T> str = full2sym(sf);
  T I1 = trace(str);
  if ((double)I1 > -4.0) {
    sigma = {T(-1), T(-1), T(-2), T(0), T(0), T(0)};
    return;
  }
  S6<T> dev = str - ident<T>() * (T)((double)I1 / 3.0);
  T tr_str = trace(str), tr_D = trace(D), tr_sD = trace2(str, D);
  T nD = m_sqrtf(trace2(D, D));
  T p = (T)(-(double)I1 / 3.0);
  T e = (T)((1.0 + (double)void_0) * (double)rho0 / (double)density - 1.0);
  e = std::max(e, void_min);
  e = std::min(e, void_max);
  T e_crt = void_co * m_exp(-lambda * m_pow(p / p_ref, xi));
  T fd = m_pow((e - void_min) / (e_crt - void_min), alpha);
  M_crt = e - e_crt;
  S6<T> rate = jau + D * (c.C1 * tr_str) + str * (c.C2 * tr_D) + str * (c.C3 * tr_sD / tr_str) +
               (str + dev) * (fd * c.C4 * nD);
  str = sigma + rate * dt;
  T sph = (T)((double)trace(str) / 3.0);
  if ((double)sph > 0.0) {
    sigma = {(T)(-1.0 + (double)coh), (T)(-1.0 + (double)coh), (T)(-2.0 + (double)coh), T(0), T(0), T(0)};
    return;
  }
  dev = str - ident<T>() * sph;
  T fa = c.C2 / c.C1, fb = c.C3 / c.C1, fc = c.C4 / c.C1;
  double t1 = 1.0 + (double)fa + (double)fb / 3.0;
  T A = (T)((double)(fd * fd * fc * fc) / 3.0 - t1 * t1);
  T B = (T)(2.0 * (double)fd * (double)fd * (double)fc * (double)fc * (t1 * t1 + 2.0 * (double)fa + 3.0) -
            4.0 * (double)fb * ((double)(T(1) + fa) + (double)fb / 3.0));
  T C = (T)(4.0 / 3.0 * (double)fd * (double)fd * (double)fc * (double)fc * (double)fb * (double)fb -
            4.0 * (double)fb * (double)fb);
  T k2 = (T)((-(double)B - std::sqrt((double)(B * B) - 4.0 * (double)A * (double)C)) / (2.0 * (double)A));
  T k_phi = (T)(3.0 / (double)std::sqrt(k2));
  T tau = m_sqrtf((T)(0.5 * (double)trace2(dev, dev)));
  T shr = tau - (-sph * k_phi);
  if (shr > T(0)) {
    T ratio = (T)(tau < 1e-10 ? 1.0 : (double)((-k_phi * sph) / tau));
    dev = dev * ratio;
  }
  sigma = dev + ident<T>() * (sph + coh);
}

enum { M_RIGID = 0, M_DP = 1, M_MUIDP = 2, M_HYPO_BASIC = 3, M_HYPO_CS = 4 };

// ---------------------------------------------------------------------------------
// Parameters (src/types.h:100-165) and InitializeParameters (src/loquat.cu:130-190).
// ---------------------------------------------------------------------------------
template <class T> struct Motion {  // RigidMotion, src/types.h:66-75
  bool is_trans = false, is_rotat = false;
  V3<T> trans_vel{}, trans_acc{}, pos_rp{}, rotat_vel{}, rotat_acc{};
  int pattern = 0;
};
template <class T> struct Table {  // MotionTable, src/types.h:77-97
  bool is_translation = false, is_rotation = false;
  int n_trans = 0, n_rot = 0, pattern = 0;
  V3<T> trans_vel[RW_TABLE_MAX]{}, trans_acc[RW_TABLE_MAX]{}, rotat_acc[RW_TABLE_MAX]{};
  T trans_time[RW_TABLE_MAX]{}, rotat_time[RW_TABLE_MAX]{};
  V3<T> pos_rp{}, rotat_vel{};
};

template <class T> struct Par {
  int dim, periodbound, n_motion, np, npb, npm, np_delete_m, n_model;
  V4<T> planeleft, planeright;
  Motion<T> mv[RW_MOTION_MAX];
  V3<T> domain_size, domain_min, gravity;
  I3 cell_num;
  int ncell, ncell_material, ncell_delete_m;
  T h, i_h, dr, hdr, vol_def, bound_thickness, rho0_m, damping;
  T model_par[RW_MODEL_MAX][RW_MATERIAL_SIZE];
  T knorm, kgrad;
  int stress_shepard_filter, dynamic_time_step, integration_method, viscosity_type;
  T alpha_m, cs_m, eta, cfl, art_coef, kernel_zero, kernel_dr;
  T time_max, time, dt, output_frequency;
  int output_number, output_format;
  T wall_fric;
};

template <class T> struct Sim {
  Par<T> P;
  Table<T> tab[RW_MOTION_MAX];
  std::vector<I4> codes, cellpos;
  std::vector<V4<T>> pospres, pospres_ori, velrhop, idm, normal, accad, spin, cvar, pospres_ini, velrhop_ini;
  std::vector<S6<T>> str, stn, str_ini, stn_ini, acestn, tcache;
  std::vector<F9<T>> cmag;
  std::vector<int> part_cel, part_idx, cell_beg, cell_end;
  double time = 0.0;
  int step = 0;
  bool compat_contact = true;

  int key_of(I3 c) const { return c.x * P.cell_num.y * P.cell_num.z + c.y * P.cell_num.z + c.z; }
  bool in_grid(I3 c) const {
    return c.x >= 0 && c.y >= 0 && c.z >= 0 && c.x < P.cell_num.x && c.y < P.cell_num.y && c.z < P.cell_num.z;
  }
  T two_h() const { return (T)(2.0 * (double)P.h); }
  bool period_image(I3 celli, V3<T> pos_i, bool abs_len, I3& cpb, V3<T>& ppb) const;
  void period_wrap(I4& cp, V4<T>& ps) const;

  void init(const rw_case* cs);
  void neighbor_search(int section);
  void rigid_body_update();
  void begin_step();
  void adami();
  void find_corner();
  void shepard(bool for_saving);
  void interaction();
  void predictor();
  void corrector();
  void end_step() {
    time += (double)P.dt;
    step++;
  }
  void whole_step() {
    begin_step();
    neighbor_search(0);
    if (P.n_motion > 0) rigid_body_update();
    adami();
    find_corner();
    if (P.stress_shepard_filter != 0 && step % P.stress_shepard_filter == 0 && step != 0) shepard(false);
    interaction();
    predictor();
    neighbor_search(1);
    adami();
    find_corner();
    interaction();
    corrector();
    end_step();
  }
};

template <class T> void Sim<T>::init(const rw_case* cs) {
  const rw_case_params& q = cs->params;
  Par<T>& p = P;
  std::memset(&p, 0, sizeof(p));
  p.dim = q.dim;
  p.periodbound = q.periodbound;
  p.n_motion = q.n_motion;
  p.np = q.np;
  p.npb = q.npb;
  p.npm = q.npm;
  p.n_model = q.n_model;
  p.planeleft = {(T)q.planeleft[0], (T)q.planeleft[1], (T)q.planeleft[2], (T)q.planeleft[3]};
  p.planeright = {(T)q.planeright[0], (T)q.planeright[1], (T)q.planeright[2], (T)q.planeright[3]};
  p.domain_size = {(T)q.domain_size[0], (T)q.domain_size[1], (T)q.domain_size[2]};
  p.domain_min = {(T)q.domain_min[0], (T)q.domain_min[1], (T)q.domain_min[2]};
  p.dr = (T)q.dr;
  p.hdr = (T)q.hdr;
  p.gravity = {(T)q.gravity[0], (T)q.gravity[1], (T)q.gravity[2]};
  p.rho0_m = (T)q.rho0_m;
  p.damping = (T)q.damping;
  for (int i = 0; i < RW_MODEL_MAX; ++i)
    for (int j = 0; j < RW_MATERIAL_SIZE; ++j) p.model_par[i][j] = (T)q.model_par[i][j];
  p.stress_shepard_filter = q.stress_shepard_filter;
  p.dynamic_time_step = q.dynamic_time_step;
  p.integration_method = q.integration_method;
  p.viscosity_type = q.viscosity_type;
  p.alpha_m = (T)q.artificial_viscosity_alpha_m;
  p.cs_m = (T)q.cs_m;
  p.cfl = (T)q.cfl;
  p.art_coef = (T)q.artificial_pressure_coefficient_material;
  p.time_max = (T)q.time_max;
  p.time = (T)q.time;
  p.dt = (T)q.dt;
  p.output_frequency = (T)q.output_frequency;
  p.output_number = q.output_number;
  p.output_format = q.output_format;
  p.wall_fric = (T)q.wall_friction;
  // InitializeParameters (3D branch), src/loquat.cu:130-190.
  p.h = p.dr * p.hdr;
  p.i_h = T(1.0f) / p.h;
  p.eta = T(0.01f) * p.h * p.h;
  p.bound_thickness = (T)(std::ceil(2.0 * (double)p.hdr) * (double)p.dr);
  double h_d = (double)p.h;
  p.vol_def = (T)std::pow((double)p.dr, 3.0);
  p.cell_num.x = (int)(T(0.5f) * p.i_h * p.domain_size.x) + 1;
  p.cell_num.y = (int)(T(0.5f) * p.i_h * p.domain_size.y) + 1;
  p.knorm = (T)(42.0 / (256.0 * 3.14159265358979323846 * std::pow(h_d, 3.0)));
  p.kgrad = (T)(-5.0 * 42 / (256.0 * 3.14159265358979323846 * std::pow(h_d, 5.0)));
  p.cell_num.z = (int)(T(0.5f) * p.i_h * p.domain_size.z) + 1;
  int one = p.cell_num.x * p.cell_num.y * p.cell_num.z;
  p.ncell_material = one;
  p.ncell_delete_m = 2 * one;
  p.ncell = p.ncell_delete_m + 1;
  p.np_delete_m = 0;
  T qq = p.dr * p.i_h;
  p.kernel_zero = p.knorm * T(2.0f) * T(2.0f) * T(2.0f) * T(2.0f) * T(0.5f);
  p.kernel_dr = p.knorm * (T(2.0f) - qq) * (T(2.0f) - qq) * (T(2.0f) - qq) * (T(2.0f) - qq) * (qq + T(0.5f));
  time = q.time;
  // Motion tables (LoadParticles, src/loquat_io.cu:266-303).
  for (int i = 0; i < p.n_motion && i < RW_MOTION_MAX; ++i) {
    const rw_motion& m = q.motion[i];
    Table<T>& t = tab[i];
    t.is_translation = m.is_translation != 0;
    t.is_rotation = m.is_rotation != 0;
    t.n_trans = m.n_trans;
    t.n_rot = m.n_rot;
    t.pattern = m.pattern;
    for (int j = 0; j < RW_TABLE_MAX; ++j) {
      t.trans_time[j] = (T)m.trans_time[j];
      t.trans_vel[j] = {(T)m.trans_vel[j][0], (T)m.trans_vel[j][1], (T)m.trans_vel[j][2]};
      t.trans_acc[j] = {(T)m.trans_acc[j][0], (T)m.trans_acc[j][1], (T)m.trans_acc[j][2]};
      t.rotat_time[j] = (T)m.rotat_time[j];
      t.rotat_acc[j] = {(T)m.rotat_acc[j][0], (T)m.rotat_acc[j][1], (T)m.rotat_acc[j][2]};
    }
    t.pos_rp = {(T)m.pos_rp[0], (T)m.pos_rp[1], (T)m.pos_rp[2]};
    t.rotat_vel = {(T)m.rotat_vel[0], (T)m.rotat_vel[1], (T)m.rotat_vel[2]};
    Motion<T>& mv = p.mv[i];
    mv.is_trans = t.is_translation;
    mv.is_rotat = t.is_rotation;
    mv.trans_vel = t.is_translation ? t.trans_vel[0] : V3<T>{T(0), T(0), T(0)};
    if (mv.is_rotat) {
      mv.pattern = t.pattern;
      mv.pos_rp = t.pos_rp;
      mv.rotat_vel = t.rotat_vel;
    }
  }
  const int np = p.np, npb = p.npb;
  codes.resize(np);
  cellpos.assign(np, I4{0, 0, 0, 0});
  pospres.resize(np);
  velrhop.resize(np);
  idm.resize(np);
  str.resize(np);
  stn.resize(np);
  normal.resize(npb);
  for (int i = 0; i < np; ++i) {
    const int32_t* c = cs->codes + 4 * i;
    codes[i] = {c[0], c[1], c[2], c[3]};
    const double* a = cs->pospres + 4 * i;
    pospres[i] = {(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
    a = cs->velrhop + 4 * i;
    velrhop[i] = {(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
    a = cs->idmassidx + 4 * i;
    idm[i] = {(T)a[0], (T)a[1], (T)i, (T)a[3]};
    a = cs->stress + 6 * i;
    str[i] = {(T)a[0], (T)a[1], (T)a[2], (T)a[3], (T)a[4], (T)a[5]};
    a = cs->strain + 6 * i;
    stn[i] = {(T)a[0], (T)a[1], (T)a[2], (T)a[3], (T)a[4], (T)a[5]};
  }
  for (int i = 0; i < npb; ++i) {
    const double* a = cs->normal + 4 * i;
    normal[i] = {(T)a[0], (T)a[1], (T)a[2], (T)a[3]};
  }
  pospres_ori = pospres;  // CopyDataFromHostToDevice copies the positions twice (src/loquat.cu:226)
  V4<T> z4{T(0), T(0), T(0), T(0)};
  S6<T> z6{T(0), T(0), T(0), T(0), T(0), T(0)};
  accad.assign(np, z4);
  spin.assign(np, z4);
  cvar.assign(np, z4);
  pospres_ini.assign(np, z4);
  velrhop_ini.assign(np, z4);
  str_ini.assign(np, z6);
  stn_ini.assign(np, z6);
  acestn.assign(np, z6);
  tcache.assign(np, z6);
  cmag.assign(np, F9<T>{});
  part_cel.assign(np, 0);
  part_idx.assign(np, 0);
  cell_beg.assign(p.ncell, -1);
  cell_end.assign(p.ncell, -1);
  // PositionFromAbsolute2Relative, src/loquat_grid.cu:253-271.
  const T half_ih = (T)(0.5 * (double)p.i_h);
  const T th = two_h();
  for (int i = 0; i < np; ++i) {
    V3<T> a = xyz(pospres[i]) * half_ih;
    I3 c{(int)a.x, (int)a.y, (int)a.z};
    cellpos[i] = {c.x, c.y, c.z, 0};
    // x - c 2h with one rounding: the reference's kernel is compiled with contraction,
    // which fuses the product into the subtraction (src/loquat_grid.cu:259)
    pospres[i].x = std::fma(-(T)c.x, th, pospres[i].x);
    pospres[i].y = std::fma(-(T)c.y, th, pospres[i].y);
    pospres[i].z = std::fma(-(T)c.z, th, pospres[i].z);
  }
  neighbor_search(0);
}

// NeighborSearch (src/loquat_grid.cu:147-191) + SortArraysPrimary/All (src/loquat.cu:254-287).
template <class T> void Sim<T>::neighbor_search(int section) {
  Par<T>& p = P;
  const int np = p.np;
  for (int i = 0; i < np; ++i) {  // cuGetParticleCellIndex, src/loquat_grid.cu:71-95
    if (cellpos[i].w == p.ncell_delete_m) {
      part_cel[i] = p.ncell_delete_m;
      part_idx[i] = i;
      continue;
    }
    I4 c = cellpos[i];
    int k = c.x * p.cell_num.y * p.cell_num.z + c.y * p.cell_num.z + c.z;
    if (idm[i].x < T(100.0f)) part_cel[i] = k;
    else if (idm[i].x >= T(100.0f)) part_cel[i] = k + p.ncell_material;
    cellpos[i].w = part_cel[i];
    part_idx[i] = i;
  }
  // SortParticleByCellIndex: a stable sort of (key, index) (src/loquat_grid.cu:98-113).
  std::vector<int> order(np);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return part_cel[a] < part_cel[b]; });
  std::vector<int> sk(np);
  for (int i = 0; i < np; ++i) sk[i] = part_cel[order[i]];
  part_cel = sk;
  part_idx = order;
  // cuFindBegEndInCell (src/loquat_grid.cu:116-144).
  std::fill(cell_beg.begin(), cell_beg.end(), -1);
  std::fill(cell_end.begin(), cell_end.end(), -1);
  for (int i = 0; i < np; ++i) {
    int c = part_cel[i];
    if (c < 0 || c >= p.ncell) continue;  // the reference writes out of bounds here
    if (i == 0 || c != part_cel[i - 1]) {
      cell_beg[c] = i;
      if (i > 0) cell_end[part_cel[i - 1]] = i;
    }
    if (i == np - 1) cell_end[c] = i + 1;
  }
  // Deleted-particle accounting (src/loquat_grid.cu:164-190).
  int beg = cell_beg[p.ncell_delete_m];
  if (beg != -1) {
    int end = cell_end[p.ncell_delete_m];
    int now = end - beg - p.np_delete_m;
    if (now != 0) {
      p.npm -= now;
      p.np_delete_m += now;
    }
  }
  // Gather-permute (src/loquat_grid.cu:193-251), array sets of src/loquat.cu:254-287.
  auto perm = [&](auto& v, int n) {
    auto src = v;
    for (int i = 0; i < n; ++i) v[i] = src[order[i]];
  };
  const int nbm = p.npb + p.npm;
  perm(codes, np);
  perm(cellpos, np);
  perm(pospres, np);
  perm(pospres_ori, np);
  perm(velrhop, np);
  perm(idm, np);
  if (section == 0) {
    perm(normal, p.npb);
    perm(str, nbm);
    perm(stn, nbm);
  } else {
    perm(pospres_ini, np);
    perm(velrhop_ini, np);
    if (p.npm != 0) {
      perm(str, nbm);
      perm(stn, nbm);
      perm(str_ini, nbm);
      perm(stn_ini, nbm);
    }
  }
  if (!compat_contact) {  // contact state follows the particle
    perm(cvar, np);
    perm(cmag, np);
  }
}

// StepCalculation (src/loquat.cu:366-374).
template <class T> void Sim<T>::begin_step() {
  T dt_m = P.h / P.cs_m;
  P.dt = P.cfl * dt_m;
  P.time = (T)time;
}

// RigidBodyUpdate (src/adami_boundary.cu:175-203).
template <class T> void Sim<T>::rigid_body_update() {
  for (int i = 0; i < P.n_motion; ++i) {
    Table<T>& t = tab[i];
    if (t.is_rotation) {
      for (int j = 0; j < t.n_rot; ++j) {
        if (P.time < t.rotat_time[j]) {
          t.rotat_vel = t.rotat_vel + t.rotat_acc[j] * P.dt;
          V3<T> vel = t.trans_vel[j] + t.trans_acc[j] * (T)(0.5 * (double)P.dt);
          t.pos_rp = t.pos_rp + vel * P.dt;
          P.mv[i].rotat_acc = t.rotat_acc[j];
          P.mv[i].rotat_vel = t.rotat_vel;
          P.mv[i].pos_rp = t.pos_rp;
          break;
        }
      }
    }
    if (t.is_translation) {
      for (int j = 0; j < t.n_trans; ++j) {
        if (P.time < t.trans_time[j]) {
          t.trans_vel[j] = t.trans_vel[j] + t.trans_acc[j] * P.dt;
          P.mv[i].trans_acc = t.trans_acc[j];
          P.mv[i].trans_vel = t.trans_vel[j];
          break;
        }
      }
    }
  }
}

#define ORC_FOR_NEIGHBOUR_CELLS(celli)                                              \
  for (int cz = -1; cz <= 1; cz++)                                                  \
    for (int cy = -1; cy <= 1; cy++)                                                \
      for (int cx = -1; cx <= 1; cx++)                                              \
        if (I3 off{cx, cy, cz}, cj{celli.x + cx, celli.y + cy, celli.z + cz}; !in_grid(cj)) { \
        } else

// Periodic planes.  Dist2Plane / AbsDist2Plane (src/functions.h:134-139).
template <class T> inline T plane_eval(V3<T> a, const V4<T>& pl) { return a.x * pl.x + a.y * pl.y + a.z * pl.z + pl.w; }
template <class T> inline T plane_norm(const V4<T>& pl) { return std::sqrt(pl.x * pl.x + pl.y * pl.y + pl.z * pl.z); }

// Periodic image of a particle within 2h of a periodic plane: its absolute position
// moved by one period along that plane's normal, as a cell and an in-cell position
// (the *LoopPeriod helpers: src/adami_boundary.cu:73-88, src/field_smoothing.cu:58-72,
// src/particle_interaction.cu:243-257).  The period is |D_left + D_right| in the Adami
// and Shepard loops (abs_len) and the signed sum in the interaction.
template <class T> bool Sim<T>::period_image(I3 celli, V3<T> pos_i, bool abs_len, I3& cpb, V3<T>& ppb) const {
  const T th = T(2.0f) * P.h;
  const V3<T> pabs = pos_i + mulI(celli, th);
  const bool left = std::fabs(plane_eval(pabs, P.planeleft)) / plane_norm(P.planeleft) < th;
  const bool right = std::fabs(plane_eval(pabs, P.planeright)) / plane_norm(P.planeright) < th;
  if (!left && !right) return false;
  T len = P.planeleft.w + P.planeright.w;
  if (abs_len) len = std::fabs(len);
  const V4<T>& pl = left ? P.planeleft : P.planeright;
  const V3<T> pb{pabs.x + pl.x * len, pabs.y + pl.y * len, pabs.z + pl.z * len};
  const T s = T(0.5f) * P.i_h;
  cpb = I3{int(pb.x * s), int(pb.y * s), int(pb.z * s)};
  ppb = pb - mulI(cpb, th);
  return true;
}

// A particle that left through a periodic plane re-enters through the other one
// (cuCheckOutDomainPeriod, src/predictor_corrector.cu:26-40).
template <class T> void Sim<T>::period_wrap(I4& cp, V4<T>& ps) const {
  const T th = T(2.0f) * P.h;
  const V3<T> pabs = xyz(ps) + mulI(I3{cp.x, cp.y, cp.z}, th);
  const bool left = plane_eval(pabs, P.planeleft) / plane_norm(P.planeleft) < T(0.0);
  const bool right = plane_eval(pabs, P.planeright) / plane_norm(P.planeright) < T(0.0);
  if (!left && !right) return;
  const T len = std::fabs(P.planeleft.w + P.planeright.w);
  const V4<T>& pl = left ? P.planeleft : P.planeright;
  const V3<T> pb{pabs.x + pl.x * len, pabs.y + pl.y * len, pabs.z + pl.z * len};
  const T s = T(0.5f) * P.i_h;
  const I3 c{int(pb.x * s), int(pb.y * s), int(pb.z * s)};
  const V3<T> pr = pb - mulI(c, th);
  cp = I4{c.x, c.y, c.z, cp.w};
  ps = V4<T>{pr.x, pr.y, pr.z, ps.w};
}

// cuAdamiBoundaryMaterial (src/adami_boundary.cu:26-158).
template <class T> void Sim<T>::adami() {
  Par<T>& p = P;
  if (p.npb == 0 || p.npm == 0) return;
  const T th = two_h();
  parallel_for(p.npb, 64, [&](int i) {
    V3<T> pos_i = xyz(pospres[i]);
    S6<T> rs{T(0), T(0), T(0), T(0), T(0), T(0)};
    V4<T> rps{T(0), T(0), T(0), T(0)}, rvr{T(0), T(0), T(0), T(0)};
    I3 celli{cellpos[i].x, cellpos[i].y, cellpos[i].z};
    V3<T> n_i{T(0), T(0), T(0)};
    bool contact = codes[i].x >= 10;
    auto scan = [&](I3 cc, V3<T> pp) {
     ORC_FOR_NEIGHBOUR_CELLS(cc) {
      int k = key_of(cj);
      for (int pass = 0; pass < 2; ++pass) {
        bool bound = pass == 0;
        int kk = bound ? k : k + p.ncell_material;
        for (int j = cell_beg[kk]; j < cell_end[kk]; ++j) {
          V3<T> dr = pp - xyz(pospres[j]);
          dr = dr - mulI(off, th);
          T r = dist(dr);
          T q = r * p.i_h;
          if (q < T(2.0f)) {
            T ker = kernel_w(p.knorm, q);
            T dwdr = kernel_f(p.kgrad, q);
            V3<T> gker = dr * dwdr;
            if (bound && contact) n_i = n_i - gker * p.vol_def;
            if (!bound) {
              T vol_j = idm[j].y / velrhop[j].w;
              rs = rs + str[j] * (ker * vol_j);
              rps = rps + v4(dr * (ker * idm[j].y), ker * vol_j);
              rvr = rvr + velrhop[j] * (ker * vol_j);
            }
          }
        }
      }
     }
    };
    scan(celli, pos_i);
    I3 cpb;
    V3<T> ppb;
    if (p.periodbound && period_image(celli, pos_i, true, cpb, ppb)) scan(cpb, ppb);
    if (enorm(n_i) > T(0)) {
      cmag[i].yx = n_i.x / enorm(n_i);
      cmag[i].yy = n_i.y / enorm(n_i);
      cmag[i].yz = n_i.z / enorm(n_i);
    }
    if (rps.w > T(0.0f)) {
      T kersum = rps.w;
      V3<T> dr_ref = xyz(rps);
      T fcoef = normal[i].w;
      V3<T> nrm = xyz(normal[i]);
      V3<T> vel_ref = xyz(rvr) / kersum;
      V3<T> vel_ref_n = nrm * dot(nrm, vel_ref);
      V3<T> vel_ref_t = vel_ref - vel_ref_n;
      V3<T> vel_rb{T(0.0f), T(0.0f), T(0.0f)};
      if (codes[i].y == 1) {
        const Motion<T>& mv = p.mv[codes[i].w];
        vel_rb = mv.trans_vel;
        if (mv.is_rotat) {
          V3<T> pabs = pos_i + mulI(celli, T(2.0f) * p.h);
          vel_rb = vel_rb + cross(mv.rotat_vel, pabs - mv.pos_rp);
        }
      }
      V3<T> vel_rb_n = nrm * dot(nrm, vel_rb);
      V3<T> vel_rb_t = vel_rb - vel_rb_n;
      V3<T> vel_ext_n = vel_rb_n * T(2.0f) - vel_ref_n;
      V3<T> vel_ext_t = fcoef == T(-1.0f) ? vel_rb_t * T(2.0f) - vel_ref_t : vel_ref_t;
      V3<T> vel_ext = vel_ext_n + vel_ext_t;
      velrhop[i] = v4(vel_ext, rvr.w / kersum);
      if (contact) {
        velrhop[i] = v4(vel_rb, rvr.w / kersum);
        cmag[i].zx = vel_ext.x;
        cmag[i].zy = vel_ext.y;
        cmag[i].zz = vel_ext.z;
      }
      S6<T> str_ref = rs / kersum;
      str[i] = subdiag(str_ref, (p.gravity * dr_ref) / kersum);
    } else {
      str[i] = S6<T>{T(0), T(0), T(0), T(0), T(0), T(0)};
    }
  });
}

// cuFindCornerParticleMaterial (src/adami_boundary.cu:209-292).
template <class T> void Sim<T>::find_corner() {
  Par<T>& p = P;
  if (p.npb == 0 || p.npm == 0) return;
  const T th = two_h();
  parallel_for(p.npm, 256, [&](int t) {
    int i = p.npb + t;
    V3<T> pos_i = xyz(pospres[i]);
    cvar[i].x = T(0.0f);
    cvar[i].y = T(999);
    T d_ij = T(999);
    I3 celli{cellpos[i].x, cellpos[i].y, cellpos[i].z};
    ORC_FOR_NEIGHBOUR_CELLS(celli) {
      int k = key_of(cj);
      for (int j = cell_beg[k]; j < cell_end[k]; ++j) {
        V3<T> dr = pos_i - xyz(pospres[j]) - mulI(off, th);
        T r = dist(dr);
        T q = r * p.i_h;
        if ((double)q < 2.0) {
          T dwdr = kernel_f(p.kgrad, q);
          V3<T> gker = dr * dwdr;
          if (codes[j].x >= 10) {
            if (r < d_ij && r > T(0)) {
              V3<T> n_ad{cmag[j].yx, cmag[j].yy, cmag[j].yz};
              V3<T> n_mat = dr / r;
              d_ij = r;
              cvar[i].y = std::fabs(dot(dr, n_ad));
              cvar[i].w = (T)codes[j].x;
              cmag[i].zx = velrhop[j].x;
              cmag[i].zy = velrhop[j].y;
              cmag[i].zz = velrhop[j].z;
              T cos_c = T(0.866f);
              T cos_n = std::fabs(dot(n_mat, n_ad));
              if (cos_n < cos_c) {
                cmag[i].yx = n_mat.x;
                cmag[i].yy = n_mat.y;
                cmag[i].yz = n_mat.z;
              } else {
                cmag[i].yx = n_ad.x;
                cmag[i].yy = n_ad.y;
                cmag[i].yz = n_ad.z;
              }
            }
            cvar[i].x += std::fabs((cmag[i].yx * gker.x + cmag[i].yy * gker.y + cmag[i].yz * gker.z) * p.vol_def);
          }
        }
      }
    }
  });
}

// cuStressRegularizationShepard (src/field_smoothing.cu:26-111).
template <class T> void Sim<T>::shepard(bool for_saving) {
  Par<T>& p = P;
  if (p.npm == 0) return;
  const T th = two_h();
  if (for_saving) tcache = str;
  parallel_for(p.npm, 256, [&](int t) {
    int i = t + p.npb;
    V3<T> pos_i = xyz(pospres[i]);
    I3 celli{cellpos[i].x, cellpos[i].y, cellpos[i].z};
    S6<T> sh{T(0), T(0), T(0), T(0), T(0), T(0)};
    T sumker = T(0.0f);
    auto scan = [&](I3 cc, V3<T> pp) {
      ORC_FOR_NEIGHBOUR_CELLS(cc) {
        int k = key_of(cj) + p.ncell_material;
        for (int j = cell_beg[k]; j < cell_end[k]; ++j) {
          V3<T> dr = pp - xyz(pospres[j]) - mulI(off, th);
          T r = dist(dr);
          T q = r * p.i_h;
          if (q < T(2.0f)) {
            T ker = kernel_w(p.knorm, q);
            T vol = idm[j].y / velrhop[j].w;
            sumker += ker * vol;
            sh = sh + str[j] * (ker * vol);
          }
        }
      }
    };
    scan(celli, pos_i);
    I3 cpb;
    V3<T> ppb;
    if (p.periodbound && period_image(celli, pos_i, true, cpb, ppb)) scan(cpb, ppb);
    if (sumker != T(0.f)) sh = sh / sumker;
    tcache[i] = sh;
  });
  if (!for_saving)
    for (int t = 0; t < p.npm; ++t) str[p.npb + t] = tcache[p.npb + t];
}

// cuParticleInteractionMaterial and its loops (src/particle_interaction.cu:26-297).
template <class T> void Sim<T>::interaction() {
  Par<T>& p = P;
  if (p.npm == 0) return;
  const T th = two_h();
  const std::vector<V4<T>> cvar0 = cvar;  // contact state as of the start of the stage
  const std::vector<F9<T>> cmag0 = cmag;
  parallel_for(p.npm, 256, [&](int t) {
    int i = p.npb + t;
    I3 celli{cellpos[i].x, cellpos[i].y, cellpos[i].z};
    V3<T> pos_i = xyz(pospres[i]);
    V4<T> vr_i = velrhop[i];
    S6<T> sor_i = str[i] / (vr_i.w * vr_i.w);
    T accden = T(0.f);
    V3<T> acc_s{T(0), T(0), T(0)}, acc_av{T(0), T(0), T(0)}, acc_as{T(0), T(0), T(0)}, acc_st{T(0), T(0), T(0)};
    F9<T> gv{};
    int shift_i = (int)cvar0[i].z;
    T rho_i = vr_i.w;
    V3<T> vel_i = xyz(vr_i);
    auto scan = [&](I3 cc, V3<T> pp) {
     ORC_FOR_NEIGHBOUR_CELLS(cc) {
      int k = key_of(cj);
      for (int pass = 0; pass < 2; ++pass) {
        bool bound = pass == 0;
        int kk = bound ? k : k + p.ncell_material;
        for (int j = cell_beg[kk]; j < cell_end[kk]; ++j) {
          V3<T> dr = pp - xyz(pospres[j]) - mulI(off, th);
          T r = dist(dr);
          T q = r * p.i_h;
          if (!(q < T(2.0f))) continue;
          T ker = kernel_w(p.knorm, q);
          T dwdr = kernel_f(p.kgrad, q);
          V3<T> gker = dr * dwdr;
          T rho_j = velrhop[j].w;
          V3<T> vel_j = xyz(velrhop[j]);
          T mass_j = bound ? p.vol_def * rho_j : idm[j].y;
          V3<T> dvel = vel_i - vel_j;
          S6<T> sor_j = str[j] / (rho_j * rho_j);
          if (codes[j].x >= 10 && shift_i == 1) dvel = V3<T>{T(0), T(0), T(0)};
          T vol_j = mass_j / rho_j;
          gv = gv - tprod(dvel, gker) * vol_j;
          if (codes[j].x < 10) {
            accden += rho_i * dot(dvel, gker) * vol_j;
            S6<T> sterm = sor_i + sor_j;
            acc_s = acc_s + dotSV(sterm, gker) * mass_j;
            if (p.viscosity_type == 1) {
              T artv = T(0.0f);
              T visc = dot(dvel, dr);
              if (visc < T(0.0f)) {
                T phi = p.h * visc / (r * r + p.eta);
                artv = p.alpha_m * p.cs_m * phi / (T(0.5f) * (rho_i + rho_j));
              }
              acc_av = acc_av + gker * (mass_j * artv);
            }
            if (p.art_coef != T(0.f)) {
              T artp = trace(sor_i);
              if (artp > T(0.0f)) artp *= p.art_coef;
              else artp = T(0.0f);
              T rj = trace(sor_j);
              if (rj > T(0.0f)) rj *= p.art_coef;
              else rj = T(0.0f);
              artp += rj;
              if (artp > T(0.0f)) {
                artp *= m_pow(ker / p.kernel_dr, p.kernel_zero / p.kernel_dr);
                acc_as = acc_as - gker * (mass_j * artp);
              }
            }
          }
        }
      }
     }
    };
    scan(celli, pos_i);
    {
      I3 cpb;
      V3<T> ppb;
      if (p.periodbound && period_image(celli, pos_i, false, cpb, ppb)) scan(cpb, ppb);
    }
    V3<T> acc_damp = vel_i * p.damping;
    V4<T> acc1 = v4(acc_s + acc_av + acc_as - acc_damp + p.gravity, accden);
    V4<T> vr_new = vr_i + acc1 * p.dt;
    // cuParticleInteractionMaterialLoopContact (src/particle_interaction.cu:174-241).
    V4<T> cv = cvar0[i];
    F9<T> cm = cmag0[i];
    V3<T> pos_abs_i = pos_i + mulI(celli, T(2.0f) * p.h);
    V3<T> nb{cm.yx, cm.yy, cm.yz};
    V3<T> vb{cm.zx, cm.zy, cm.zz};
    V3<T> fric{T(0.0f), T(0.0f), T(0.0f)};
    T mass_rate = T(2.0f) / (T(2.0f) + T(0.0f));
    V3<T> dv{(vb.x - vr_new.x) * mass_rate, (vb.y - vr_new.y) * mass_rate, (vb.z - vr_new.z) * mass_rate};
    int count = 0;
    if (cv.y <= p.h * T(2) && dot(dv, nb) > T(0)) {
      T fc = p.wall_fric;
      V3<T> dvn{nb.x * dot(dv, nb), nb.y * dot(dv, nb), nb.z * dot(dv, nb)};
      V3<T> fn = dvn * idm[i].y / p.dt;
      V3<T> dvt = dv - dvn;
      V3<T> ft = dvt * idm[i].y / p.dt;
      T afn = enorm(fn), aft = enorm(ft);
      if (aft > (fc * afn)) {
        ft = ft * (fc * afn / aft);
        cv.z = T(1);
      } else {
        cv.z = T(0);
      }
      fric = ft + fn;
      if (cv.y > p.dr * T(1.0f)) {
        ORC_FOR_NEIGHBOUR_CELLS(celli) {
          int kk = key_of(cj) + p.ncell_material;
          for (int j = cell_beg[kk]; j < cell_end[kk]; ++j) {
            if (cvar0[j].y <= p.dr * T(1.0001f)) {
              V3<T> pos_abs_j{pospres[j].x + (T)cellpos[j].x * (T(2.0f) * p.h),
                              pospres[j].y + (T)cellpos[j].y * (T(2.0f) * p.h),
                              pospres[j].z + (T)cellpos[j].z * (T(2.0f) * p.h)};
              V3<T> dc = pos_abs_i - pos_abs_j;
              T rcol = std::fabs(dc.x * cm.yz + dc.y * cm.yy + dc.z * cm.yx);
              bool same_line = rcol <= p.dr / T(2);
              T cvx_j = (j == i) ? cv.x : cvar0[j].x;
              if (same_line && cvx_j != T(0)) {
                if (cv.x > cvx_j) cv.x = cvx_j;
                cvx_j = (j == i) ? cv.x : cvar0[j].x;
                fric.x = cmag0[j].xx * cv.x / cvx_j;
                fric.y = cmag0[j].xy * cv.x / cvx_j;
                fric.z = cmag0[j].xz * cv.x / cvx_j;
                count++;
              }
            }
          }
        }
        if (count == 0) {
          fric.x *= T(0);
          fric.y *= T(0);
          fric.z *= T(0);
        }
      }
      cm.xx = fric.x;
      cm.xy = fric.y;
      cm.xz = fric.z;
      acc_st = fric * (T(1) / idm[i].y);
    }
    cvar[i] = cv;
    cmag[i] = cm;
    accad[i] = v4(acc_s + acc_av + acc_as + acc_st - acc_damp + p.gravity, accden);
    acestn[i] = full2sym(gv);
    spin[i] = v4(skewpart(gv), T(0.f));
  });
}

template <class T> void constitutive(const Par<T>& p, int model, int mat, T dt, T rho, V3<T> om, S6<T> D, S6<T>& sig,
                                     bool& yld, T& M_crt) {
  const T* mp = p.model_par[mat];
  if (model == M_DP) mat_dp(dt, om, D, sig, mp, yld);
  else if (model == M_MUIDP) mat_muidp(dt, om, D, sig, mp);
  else if (model == M_HYPO_BASIC) mat_hypo_basic(dt, om, D, sig, mp);
  else if (model == M_HYPO_CS) mat_hypo_cs(dt, rho, om, D, sig, mp, M_crt);
}

// Predictor (src/predictor_corrector.cu:52-103).
template <class T> void Sim<T>::predictor() {
  Par<T>& p = P;
  pospres_ini = pospres;
  velrhop_ini = velrhop;
  if (p.npm == 0) return;
  for (int i = 0; i < p.npb + p.npm; ++i) {
    str_ini[i] = str[i];
    stn_ini[i] = stn[i];
  }
  const T hdt = T(0.5f) * p.dt;
  parallel_for(p.npm, 1024, [&](int t) {
    int i = p.npb + t;
    if (codes[i].y != 1) return;
    velrhop[i] = velrhop[i] + accad[i] * hdt;
    pospres[i] = add3(pospres[i], xyz(velrhop[i]) * hdt);
    const T* mp = p.model_par[codes[i].w];
    velrhop[i].w = std::max(velrhop[i].w, mp[RW_MATERIAL_SIZE - 2]);
    velrhop[i].w = std::min(velrhop[i].w, mp[RW_MATERIAL_SIZE - 1]);
    S6<T> dstn = acestn[i] * hdt;
    stn[i] = stn[i] + dstn;
    S6<T> sigma = str[i];
    bool yld = false;
    T M_crt = T(0);
    constitutive(p, codes[i].z, codes[i].w, hdt, velrhop[i].w, xyz(spin[i]), acestn[i], sigma, yld, M_crt);
    str[i] = sigma;
    if (!yld) idm[i].x = T(100);
  });
}

// Corrector (src/predictor_corrector.cu:109-213).
template <class T> void Sim<T>::corrector() {
  Par<T>& p = P;
  const T th = two_h();
  if (p.n_motion > 0) {
    parallel_for(p.npb, 1024, [&](int i) {  // cuCorrectorBound
      if (codes[i].y != 1) return;
      const Motion<T>& mv = p.mv[codes[i].w];
      V3<T> vel = mv.trans_vel;
      if (mv.is_rotat && mv.pattern != 1) {
        V3<T> pos_i = xyz(pospres[i]);
        I3 celli{cellpos[i].x, cellpos[i].y, cellpos[i].z};
        V3<T> pabs = pos_i + mulI(celli, th);
        vel = vel + cross(mv.rotat_vel, pabs - mv.pos_rp);
        F9<T> R = rodrigues(mv.rotat_vel * p.dt);
        V3<T> n = dotFV(R, xyz(normal[i]));
        normal[i] = v4(n, normal[i].w);
      }
      pospres[i] = add3(pospres_ini[i], vel * p.dt);
      I3 dc{int(pospres[i].x >= th) - int(pospres[i].x < T(0)), int(pospres[i].y >= th) - int(pospres[i].y < T(0)),
            int(pospres[i].z >= th) - int(pospres[i].z < T(0))};
      pospres[i] = sub3(pospres[i], mulI(dc, th));
      cellpos[i] = {cellpos[i].x + dc.x, cellpos[i].y + dc.y, cellpos[i].z + dc.z, cellpos[i].w};
    });
  }
  if (p.npm == 0) return;
  const T hdt = T(0.5f) * p.dt;
  parallel_for(p.npm, 1024, [&](int t) {  // cuCorrectorMaterial
    int i = p.npb + t;
    if (codes[i].y != 1) return;
    velrhop[i] = velrhop_ini[i] + accad[i] * p.dt;
    pospres[i] = add3(pospres_ini[i], xyz(velrhop[i] + velrhop_ini[i]) * hdt);
    const T* mp = p.model_par[codes[i].w];
    velrhop[i].w = std::max(velrhop[i].w, mp[RW_MATERIAL_SIZE - 2]);
    velrhop[i].w = std::min(velrhop[i].w, mp[RW_MATERIAL_SIZE - 1]);
    I3 dc{int(pospres[i].x >= th) - int(pospres[i].x < T(0)), int(pospres[i].y >= th) - int(pospres[i].y < T(0)),
          int(pospres[i].z >= th) - int(pospres[i].z < T(0))};
    pospres[i] = sub3(pospres[i], mulI(dc, th));
    cellpos[i] = {cellpos[i].x + dc.x, cellpos[i].y + dc.y, cellpos[i].z + dc.z, cellpos[i].w};
    if (p.periodbound) period_wrap(cellpos[i], pospres[i]);
    S6<T> sigma = str_ini[i];
    S6<T> dstn = acestn[i] * p.dt;
    stn[i] = stn_ini[i] + dstn;
    bool yld = false;
    T M_crt = T(0);
    constitutive(p, codes[i].z, codes[i].w, p.dt, velrhop[i].w, xyz(spin[i]), acestn[i], sigma, yld, M_crt);
    str[i] = sigma;
    if (!yld) idm[i].x = T(100);
    idm[i].w = M_crt;
    I3 c{cellpos[i].x, cellpos[i].y, cellpos[i].z};
    if (!in_grid(c)) {
      cellpos[i].w = p.ncell_delete_m;
      idm[i].x = T(999.0);
    }
    if (p.time <= p.dt) pospres_ori[i] = V4<T>{T(0), T(0), T(0), T(0)};
    pospres_ori[i] = add3(pospres_ori[i], xyz(velrhop[i]) * p.dt);
    accad[i] = pospres_ori[i];
  });
}

// ---------------------------------------------------------------------------------
// Array export/import in the reference's layouts.
// ---------------------------------------------------------------------------------
template <class T> size_t row_bytes(int which) {
  switch (which) {
    case RW_ARR_CODES: case RW_ARR_CELLPOS: return 16;
    case RW_ARR_STR: case RW_ARR_STN: case RW_ARR_ACESTN: case RW_ARR_STR_INI: case RW_ARR_STN_INI: return 6 * sizeof(T);
    case RW_ARR_CONTACT_MAG: return 9 * sizeof(T);
    case RW_ARR_PART_IDX: case RW_ARR_CELL_BEG: case RW_ARR_CELL_END: return 4;
    default: return 4 * sizeof(T);
  }
}

template <class T> int get_set(Sim<T>& s, int which, void* buf, size_t bytes, bool set) {
  const int np = s.P.np;
  auto io = [&](auto& v, size_t n) -> int {
    using E = typename std::decay_t<decltype(v)>::value_type;
    if (bytes != n * sizeof(E)) return RW_EINVAL;
    if (set) std::memcpy(v.data(), buf, bytes);
    else std::memcpy(buf, v.data(), bytes);
    return RW_OK;
  };
  switch (which) {
    case RW_ARR_CODES: return io(s.codes, np);
    case RW_ARR_CELLPOS: return io(s.cellpos, np);
    case RW_ARR_POSPRES: return io(s.pospres, np);
    case RW_ARR_POSPRES_ORI: return io(s.pospres_ori, np);
    case RW_ARR_VELRHOP: return io(s.velrhop, np);
    case RW_ARR_IDMASSIDX: return io(s.idm, np);
    case RW_ARR_STR: return io(s.str, np);
    case RW_ARR_STN: return io(s.stn, np);
    case RW_ARR_NORMAL: return io(s.normal, (size_t)s.P.npb);
    case RW_ARR_CONTACT_MAG: return io(s.cmag, np);
    case RW_ARR_CONTACT_VAR: return io(s.cvar, np);
    case RW_ARR_ACCAD: return io(s.accad, np);
    case RW_ARR_SPIN: return io(s.spin, np);
    case RW_ARR_ACESTN: return io(s.acestn, np);
    case RW_ARR_POSPRES_INI: return io(s.pospres_ini, np);
    case RW_ARR_VELRHOP_INI: return io(s.velrhop_ini, np);
    case RW_ARR_STR_INI: return io(s.str_ini, np);
    case RW_ARR_STN_INI: return io(s.stn_ini, np);
    case RW_ARR_PART_IDX: return io(s.part_idx, np);
    case RW_ARR_CELL_BEG: return io(s.cell_beg, (size_t)s.P.ncell);
    case RW_ARR_CELL_END: return io(s.cell_end, (size_t)s.P.ncell);
    case RW_ARR_POS_ABS: {
      if (set) return RW_EINVAL;
      std::vector<V4<T>> a(np);
      for (int i = 0; i < np; ++i) {
        I3 c{s.cellpos[i].x, s.cellpos[i].y, s.cellpos[i].z};
        a[i] = add3(s.pospres[i], mulI(c, s.two_h()));
      }
      return io(a, np);
    }
    default: return RW_EINVAL;
  }
}

// Wall force.  mode 0/1: FP64 sums in N (see include/retainwall.h).  mode 2: the
// reference's own strip loop (src/utilities.cu:590-639): scalar accumulator,
// 0.001 * contact_mag.xx in kN, i over [npb, np) in order.
template <class T> void wall_force(Sim<T>& s, int mode, int wall_id, const double* strip, double out[3]) {
  const Par<T>& p = s.P;
  out[0] = out[1] = out[2] = 0.0;
  if (mode == 2) {
    T acc = T(0.0f);
    for (int i = p.npb; i < p.np; ++i) {
      T px = s.pospres[i].x + (T)s.cellpos[i].x * (T(2.0f) * p.h);
      T pz = s.pospres[i].z + (T)s.cellpos[i].z * (T(2.0f) * p.h);
      bool all = ((double)px <= (double)(T(0.04f) + p.bound_thickness + p.dr * T(3))) &&
                 ((double)pz >= (double)(p.bound_thickness + T(0.04f))) &&
                 ((double)pz <= (double)(p.bound_thickness + T(0.04f) + T(1.0f)));
      if (all) acc = (T)((double)acc + 0.001 * (double)s.cmag[i].xx);
    }
    out[0] = (double)acc;
    return;
  }
  double xmax, zmin, zmax;
  if (strip) {
    xmax = strip[0]; zmin = strip[1]; zmax = strip[2];
  } else {
    xmax = (double)(T(0.04f) + p.bound_thickness + p.dr * T(3));
    zmin = (double)(p.bound_thickness + T(0.04f));
    zmax = (double)(p.bound_thickness + T(0.04f) + T(1.0f));
  }
  for (int i = p.npb; i < p.npb + p.npm; ++i) {
    bool take;
    if (mode == 0) {
      take = (int)s.cvar[i].w == wall_id && s.cvar[i].y <= p.h * T(2);
    } else {
      double px = (double)(s.pospres[i].x + (T)s.cellpos[i].x * (T(2.0f) * p.h));
      double pz = (double)(s.pospres[i].z + (T)s.cellpos[i].z * (T(2.0f) * p.h));
      take = px <= xmax && pz >= zmin && pz <= zmax;
    }
    if (take) {
      out[0] += (double)s.cmag[i].xx;
      out[1] += (double)s.cmag[i].xy;
      out[2] += (double)s.cmag[i].xz;
    }
  }
}

struct Handle {
  int prec;
  void* sim;
};

}  // namespace orc

using namespace orc;

#define ORC_DISPATCH(h, call)                                  \
  do {                                                         \
    if ((h)->prec == 4) { auto& s = *(Sim<float>*)(h)->sim; call; } \
    else { auto& s = *(Sim<double>*)(h)->sim; call; }           \
  } while (0)

extern "C" {

void* orc_create(const rw_case* c, int precision, int nthreads) {
  g_threads = nthreads;
  Handle* h = new Handle{precision == 8 ? 8 : 4, nullptr};
  if (h->prec == 4) {
    auto* s = new Sim<float>();
    s->init(c);
    h->sim = s;
  } else {
    auto* s = new Sim<double>();
    s->init(c);
    h->sim = s;
  }
  return h;
}

void orc_destroy(void* hv) {
  Handle* h = (Handle*)hv;
  if (!h) return;
  if (h->prec == 4) delete (Sim<float>*)h->sim;
  else delete (Sim<double>*)h->sim;
  delete h;
}

int orc_stage(void* hv, int stage) {
  Handle* h = (Handle*)hv;
  ORC_DISPATCH(h, {
    switch (stage) {
      case 0: s.begin_step(); break;
      case 1: s.neighbor_search(0); break;
      case 2: s.neighbor_search(1); break;
      case 3: if (s.P.n_motion > 0) s.rigid_body_update(); break;
      case 4: s.adami(); break;
      case 5: s.find_corner(); break;
      case 6: s.shepard(false); break;
      case 7: s.interaction(); break;
      case 8: s.predictor(); break;
      case 9: s.corrector(); break;
      case 10: s.end_step(); break;
      default: return RW_EINVAL;
    }
  });
  return RW_OK;
}

int orc_step(void* hv, int n) {
  Handle* h = (Handle*)hv;
  ORC_DISPATCH(h, { for (int k = 0; k < n; ++k) s.whole_step(); });
  return RW_OK;
}

int orc_get_array(void* hv, int which, void* dst, size_t bytes) {
  Handle* h = (Handle*)hv;
  int r = RW_OK;
  ORC_DISPATCH(h, { r = get_set(s, which, dst, bytes, false); });
  return r;
}

int orc_set_array(void* hv, int which, const void* src, size_t bytes) {
  Handle* h = (Handle*)hv;
  int r = RW_OK;
  ORC_DISPATCH(h, { r = get_set(s, which, const_cast<void*>(src), bytes, true); });
  return r;
}

int orc_set_counters(void* hv, double time, int step, int npm, int np_delete_m) {
  Handle* h = (Handle*)hv;
  ORC_DISPATCH(h, {
    s.time = time;
    s.step = step;
    s.P.npm = npm;
    s.P.np_delete_m = np_delete_m;
  });
  return RW_OK;
}

int orc_set_option(void* hv, int opt, double v) {
  Handle* h = (Handle*)hv;
  ORC_DISPATCH(h, {
    if (opt == RW_OPT_WALL_FRICTION) s.P.wall_fric = (decltype(s.P.wall_fric))v;
    else if (opt == RW_OPT_COMPAT_CONTACT) s.compat_contact = v != 0.0;
    else return RW_EINVAL;
  });
  return RW_OK;
}

int orc_get_info(void* hv, rw_info* out) {
  Handle* h = (Handle*)hv;
  std::memset(out, 0, sizeof(*out));
  ORC_DISPATCH(h, {
    out->np = s.P.np;
    out->npb = s.P.npb;
    out->npm = s.P.npm;
    out->np_delete_m = s.P.np_delete_m;
    out->ncell = s.P.ncell;
    out->step = s.step;
    out->scalar_bytes = h->prec;
    out->cell_num[0] = s.P.cell_num.x;
    out->cell_num[1] = s.P.cell_num.y;
    out->cell_num[2] = s.P.cell_num.z;
    out->n_motion = s.P.n_motion;
    out->time = s.time;
    out->dt = (double)s.P.dt;
    out->h = (double)s.P.h;
    out->dr = (double)s.P.dr;
  });
  return RW_OK;
}

int orc_wall_force(void* hv, int mode, int wall_id, const double* strip, double* out3) {
  Handle* h = (Handle*)hv;
  ORC_DISPATCH(h, { wall_force(s, mode, wall_id, strip, out3); });
  return RW_OK;
}

// Stand-alone constitutive calls for known-answer tests against the reference's header.
int orc_hypo_cs(int precision, double dt, double density, const double* omega4, const double* rate6, double* sigma6,
                const double* par15, double* m_crt) {
  auto run = [&](auto zero) {
    using T = decltype(zero);
    T mp[RW_MATERIAL_SIZE];
    for (int j = 0; j < RW_MATERIAL_SIZE; ++j) mp[j] = (T)par15[j];
    S6<T> sg{(T)sigma6[0], (T)sigma6[1], (T)sigma6[2], (T)sigma6[3], (T)sigma6[4], (T)sigma6[5]};
    S6<T> D{(T)rate6[0], (T)rate6[1], (T)rate6[2], (T)rate6[3], (T)rate6[4], (T)rate6[5]};
    V3<T> om{(T)omega4[0], (T)omega4[1], (T)omega4[2]};
    T m = T(0);
    mat_hypo_cs((T)dt, (T)density, om, D, sg, mp, m);
    sigma6[0] = sg.xx; sigma6[1] = sg.yy; sigma6[2] = sg.zz; sigma6[3] = sg.xy; sigma6[4] = sg.xz; sigma6[5] = sg.yz;
    *m_crt = (double)m;
  };
  if (precision == 8) run(0.0);
  else run(0.0f);
  return RW_OK;
}

int orc_hypo_basic(int precision, double dt, const double* omega4, const double* rate6, double* sigma6,
                   const double* par15) {
  auto run = [&](auto zero) {
    using T = decltype(zero);
    T mp[RW_MATERIAL_SIZE];
    for (int j = 0; j < RW_MATERIAL_SIZE; ++j) mp[j] = (T)par15[j];
    S6<T> sg{(T)sigma6[0], (T)sigma6[1], (T)sigma6[2], (T)sigma6[3], (T)sigma6[4], (T)sigma6[5]};
    S6<T> D{(T)rate6[0], (T)rate6[1], (T)rate6[2], (T)rate6[3], (T)rate6[4], (T)rate6[5]};
    V3<T> om{(T)omega4[0], (T)omega4[1], (T)omega4[2]};
    mat_hypo_basic((T)dt, om, D, sg, mp);
    sigma6[0] = sg.xx; sigma6[1] = sg.yy; sigma6[2] = sg.zz; sigma6[3] = sg.xy; sigma6[4] = sg.xz; sigma6[5] = sg.yz;
  };
  if (precision == 8) run(0.0);
  else run(0.0f);
  return RW_OK;
}

// *yield (DP only) receives the reference's yield flag.
int orc_dp(int precision, int mui, double dt, const double* omega4, const double* rate6, double* sigma6,
           const double* par15, int* yield) {
  auto run = [&](auto zero) {
    using T = decltype(zero);
    T mp[RW_MATERIAL_SIZE];
    for (int j = 0; j < RW_MATERIAL_SIZE; ++j) mp[j] = (T)par15[j];
    S6<T> sg{(T)sigma6[0], (T)sigma6[1], (T)sigma6[2], (T)sigma6[3], (T)sigma6[4], (T)sigma6[5]};
    S6<T> D{(T)rate6[0], (T)rate6[1], (T)rate6[2], (T)rate6[3], (T)rate6[4], (T)rate6[5]};
    V3<T> om{(T)omega4[0], (T)omega4[1], (T)omega4[2]};
    bool yld = false;
    if (mui) mat_muidp((T)dt, om, D, sg, mp);
    else mat_dp((T)dt, om, D, sg, mp, yld);
    sigma6[0] = sg.xx; sigma6[1] = sg.yy; sigma6[2] = sg.zz; sigma6[3] = sg.xy; sigma6[4] = sg.xz; sigma6[5] = sg.yz;
    if (yield) *yield = yld ? 1 : 0;
  };
  if (precision == 8) run(0.0);
  else run(0.0f);
  return RW_OK;
}

double orc_kernel_w(int precision, double par, double q) {
  return precision == 8 ? kernel_w<double>(par, q) : (double)kernel_w<float>((float)par, (float)q);
}
double orc_kernel_f(int precision, double par, double q) {
  return precision == 8 ? kernel_f<double>(par, q) : (double)kernel_f<float>((float)par, (float)q);
}

}  // extern "C"
