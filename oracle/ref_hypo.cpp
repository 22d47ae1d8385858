// Test infrastructure, not product code.
//
// Host build of the reference's own per-particle functions: src/functions.h
// (Wendland kernel, tensor algebra) and src/constitutive_model.h (HypoCS,
// HypoBasic, DP, MuI-DP), compiled with g++ from where they lie (see
// oracle/build_ref.sh) into oracle/_ref/libref_hypo_{f32,f64}.so. It pins the
// oracle's restatement of those functions bit for bit; it is never linked into
// the product.
//
// The headers are written for nvcc; on the host the CUDA qualifiers expand to nothing
// (cuda_runtime.h host_defines).  Under nvcc, unqualified pow/exp/sin/sqrt of float
// arguments resolve to the float overloads; a plain g++ build would pick the double C
// functions.  The using-declarations below restore nvcc's overload resolution.
#include <algorithm>
#include <cmath>
using std::max;
using std::min;
using std::cos;
using std::exp;
using std::pow;
using std::sin;
using std::sqrt;

#include "functions.h"
#include "constitutive_model.h"

extern "C" {

// sigma6: xx yy zz xy xz yz (in/out); omega4: spin (x y z w); rate6: strain rate
// par15: model parameters; returns M_crt through *m_crt.
void ref_hypo_cs(scalar dt, scalar density, const scalar* omega4, const scalar* rate6, scalar* sigma6,
                 scalar* par15, scalar* m_crt) {
  scalar4 om = {omega4[0], omega4[1], omega4[2], omega4[3]};
  tensor2d d = {rate6[0], rate6[1], rate6[2], rate6[3], rate6[4], rate6[5]};
  tensor2d s = {sigma6[0], sigma6[1], sigma6[2], sigma6[3], sigma6[4], sigma6[5]};
  scalar m = 0;
  cuMatModHypo(dt, density, om, d, s, par15, m);
  sigma6[0] = s.xx; sigma6[1] = s.yy; sigma6[2] = s.zz; sigma6[3] = s.xy; sigma6[4] = s.xz; sigma6[5] = s.yz;
  *m_crt = m;
}

void ref_hypo_basic(scalar dt, const scalar* omega4, const scalar* rate6, scalar* sigma6, scalar* par15) {
  scalar4 om = {omega4[0], omega4[1], omega4[2], omega4[3]};
  tensor2d d = {rate6[0], rate6[1], rate6[2], rate6[3], rate6[4], rate6[5]};
  tensor2d s = {sigma6[0], sigma6[1], sigma6[2], sigma6[3], sigma6[4], sigma6[5]};
  cuMatModHypo(dt, om, d, s, par15);
  sigma6[0] = s.xx; sigma6[1] = s.yy; sigma6[2] = s.zz; sigma6[3] = s.xy; sigma6[4] = s.xz; sigma6[5] = s.yz;
}

void ref_dp(scalar dt, const scalar* omega4, const scalar* rate6, scalar* sigma6, scalar* par15, int* yield) {
  scalar4 om = {omega4[0], omega4[1], omega4[2], omega4[3]};
  tensor2d d = {rate6[0], rate6[1], rate6[2], rate6[3], rate6[4], rate6[5]};
  tensor2d s = {sigma6[0], sigma6[1], sigma6[2], sigma6[3], sigma6[4], sigma6[5]};
  bool yld = false;
  cuMatModDP(dt, om, d, s, par15, yld);
  sigma6[0] = s.xx; sigma6[1] = s.yy; sigma6[2] = s.zz; sigma6[3] = s.xy; sigma6[4] = s.xz; sigma6[5] = s.yz;
  *yield = yld ? 1 : 0;
}

void ref_mui_dp(scalar dt, const scalar* omega4, const scalar* rate6, scalar* sigma6, scalar* par15) {
  scalar4 om = {omega4[0], omega4[1], omega4[2], omega4[3]};
  tensor2d d = {rate6[0], rate6[1], rate6[2], rate6[3], rate6[4], rate6[5]};
  tensor2d s = {sigma6[0], sigma6[1], sigma6[2], sigma6[3], sigma6[4], sigma6[5]};
  cuMatModMuIDP(dt, om, d, s, par15);
  sigma6[0] = s.xx; sigma6[1] = s.yy; sigma6[2] = s.zz; sigma6[3] = s.xy; sigma6[4] = s.xz; sigma6[5] = s.yz;
}

scalar ref_kernel_w(scalar par, scalar q) { return GetKernel(par, q); }
scalar ref_kernel_f(scalar par, scalar q) { return GetGradKernel(par, q); }
int ref_scalar_bytes() { return (int)sizeof(scalar); }
}
