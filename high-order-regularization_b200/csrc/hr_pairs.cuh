// hr_pairs.cuh — per-pair regularized kernels (device functions).
//
// The formulas are the reference's:
//   reg_coeff         get_reg_coeff_7ord + evaluate_In_024   2S/utilities.cpp:163-175, 327-337
//   sl_7ord           Stokes_SL_7ord                         2S/utilities.cpp:179-207
//   sl_7ord_onsurf    Stokes_SL_7ord_onSurf                  2S/utilities.cpp:211-254
//   dl_7ord           Stokes_DL_7ord                         2S/utilities.cpp:258-288
//   dl_7ord_onsurf    Stokes_DL_7ord_onSurf                  2S/utilities.cpp:292-323
//   lapl_dl_7ord      Lapl_DL_7ord                           E2G/utilities.cpp:190-211
// evaluated from r^2 and one reciprocal square root per pair: every 1/r^k
// of the reference becomes a product of rinv = rsqrt(r^2), r/delta becomes
// r * (1/delta), and the switch r/delta > 8 becomes r^2 > 64 delta^2. Each
// step changes a result by a few ulp at most; the branch values agree to
// ~1e-28 relative at r = 8 delta, so the switch point does not matter.
// erf, erfc, exp and rsqrt are CUDA's own functions.
#pragma once
#include <cuda_runtime.h>

namespace hr {

// sqrt(pi) as the reference computes it: sqrt of the double nearest pi (0x1.c5bf891b4ef6ap+0)
__device__ __forceinline__ double d_rootpi() { return 1.7724538509055159; }

struct Coef {
  double c1, c2, c3;
};

// Per-target constants of the regularized kernels.
// Beyond r = sqrt(51) delta (r/delta = 7.14) the on-surface smoothing factors
// G1, G2, G3 equal the singular kernel's to a relative 2^-54 (their erfc and
// polynomial-times-Gaussian terms are smaller; 7.11 is the largest of the three
// thresholds), so the FP64 sums take the plain kernel there; below 28.5 delta^2
// (r/delta = 5.34) the same holds to 2^-25 for the FP32 sums.
constexpr double kPlainOnSurf64 = 51.0;
constexpr float kPlainOnSurf32 = 28.5f;

struct Reg {
  double d, inv_d, d64, r0sq;  // delta, 1/delta, 64 delta^2, (1e-14)^2
  double inv_d2, inv_d3, inv_d5;
  double dplain;               // kPlainOnSurf64 delta^2
};

__device__ __forceinline__ Reg make_reg(double d) {
  Reg g;
  g.d = d;
  g.inv_d = 1.0 / d;
  g.d64 = 64.0 * d * d;
  g.r0sq = 1e-28;
  g.inv_d2 = g.inv_d * g.inv_d;
  g.inv_d3 = g.inv_d2 * g.inv_d;
  g.inv_d5 = g.inv_d3 * g.inv_d2;
  g.dplain = kPlainOnSurf64 * d * d;
  return g;
}

__device__ __forceinline__ Coef reg_coeff(double lam) {
  const double rp = d_rootpi();
  double lam2 = lam * lam;
  double e2 = exp(lam2);
  double em2 = exp(-lam2);
  double al = fabs(lam);
  double t = al * erfc(al);
  double I0 = em2 / rp - t;
  double I2 = 2.0 / 3.0 * ((0.5 - lam2) * em2 / rp + lam2 * t);
  double I4 = 8.0 / 15.0 * ((0.75 - 0.5 * lam2 + lam2 * lam2) * em2 / rp - lam2 * lam2 * t);
  Coef c;
  c.c3 = e2 * (2.0 * I0 - 4.0 * I2 + I4) / 8.0;
  c.c2 = e2 * (I0 - I2) + (4.0 * lam2 + 7.0) * c.c3;
  c.c1 = 2.0 * e2 * I0 + 2.0 * (lam2 + 1.0) * c.c2 - (4.0 * lam2 * lam2 + 6.0 * lam2 + 6.0) * c.c3;
  return c;
}

// Regularized Stokeslet factors (s1 ~ 1/r, s2 ~ 1/r^3), off-surface target.
// Returns true when the smoothed (erf) branch was taken.
__device__ __forceinline__ bool sl_7ord(double r2, double rinv, const Reg& g, const Coef& c,
                                        double& s1, double& s2) {
  const double rp = d_rootpi();
  if (r2 < g.r0sq) {
    s1 = 32.0 / 5.0 / rp / g.d;
    s2 = 256.0 / 15.0 / rp / (g.d * g.d * g.d);
    return false;
  }
  double rinv3 = rinv * rinv * rinv;
  if (r2 > g.d64) {
    s1 = rinv;
    s2 = rinv3;
    return false;
  }
  double rd = r2 * rinv * g.inv_d;
  double rd2 = rd * rd;
  double rd4 = rd2 * rd2;
  double rd6 = rd4 * rd2;
  double errfn = erf(rd);
  double r_expfn = rd * exp(-rd2);
  double poly1 = c.c1 - 2.0 * (c.c2 + c.c3) * rd2 + 4.0 * c.c3 * rd4;
  double poly2 = -2.0 / rp + 2.0 * (c.c1 + 2.0 * (c.c2 + c.c3)) * rd2 -
                 4.0 * (c.c2 + 5.0 * c.c3) * rd4 + 8.0 * c.c3 * rd6;
  s1 = (errfn + poly1 * r_expfn) * rinv;
  s2 = (errfn + poly2 * r_expfn) * rinv3;
  return true;
}

// Regularized Stokeslet factors, on-surface target (lambda = 0).
__device__ __forceinline__ bool sl_7ord_onsurf(double r2, double rinv, const Reg& g, double& s1,
                                               double& s2) {
  const double rp = d_rootpi();
  if (r2 < g.r0sq) {
    s1 = 32.0 / 5.0 / rp / g.d;
    s2 = 256.0 / 15.0 / rp / (g.d * g.d * g.d);
    return false;
  }
  double rinv3 = rinv * rinv * rinv;
  if (r2 > g.d64) {
    s1 = rinv;
    s2 = rinv3;
    return false;
  }
  double rd = r2 * rinv * g.inv_d;
  double rd2 = rd * rd;
  double rd4 = rd2 * rd2;
  double rd6 = rd4 * rd2;
  double errfn = erf(rd);
  double r_expfn = 2.0 / rp * rd * exp(-rd2);
  double poly1 = 11.0 / 5.0 - 26.0 / 15.0 * rd2 + 4.0 / 15.0 * rd4;
  double poly2 = -1.0 + (118.0 * rd2 - 68.0 * rd4 + 8.0 * rd6) * (1.0 / 15.0);
  s1 = (errfn + poly1 * r_expfn) * rinv;
  s2 = (errfn + poly2 * r_expfn) * rinv3;
  return true;
}

// Regularized stresslet factors (s2 ~ 1/r^3, s3 ~ 1/r^5), off-surface target.
__device__ __forceinline__ bool dl_7ord(double r2, double rinv, const Reg& g, const Coef& c,
                                        double& s2, double& s3) {
  const double rp = d_rootpi();
  if (r2 < g.r0sq) {
    s2 = 256.0 / 15.0 / rp / (g.d * g.d * g.d);
    s3 = 0.0;
    return false;
  }
  double rinv2 = rinv * rinv;
  double rinv3 = rinv2 * rinv;
  if (r2 > g.d64) {
    s2 = rinv3;
    s3 = rinv3 * rinv2;
    return false;
  }
  double rd = r2 * rinv * g.inv_d;
  double rd2 = rd * rd;
  double rd4 = rd2 * rd2;
  double rd6 = rd4 * rd2;
  double errfn = erf(rd);
  double r_expfn = rd * exp(-rd2);
  double poly2 = -2.0 / rp + 2.0 * (c.c1 + 2.0 * (c.c2 + c.c3)) * rd2 -
                 4.0 * (c.c2 + 5.0 * c.c3) * rd4 + 8.0 * c.c3 * rd6;
  double poly3 = -2.0 / rp * (1.0 + 2.0 / 3.0 * rd2) +
                 4.0 / 3.0 *
                     ((c.c1 + 4.0 * c.c2 + 12.0 * c.c3) * rd4 - 2.0 * (c.c2 + 9.0 * c.c3) * rd6 +
                      4.0 * c.c3 * rd6 * rd2);
  s2 = (errfn + poly2 * r_expfn) * rinv3;
  s3 = (errfn + poly3 * r_expfn) * (rinv3 * rinv2);
  return true;
}

// Regularized stresslet factor s3 ~ 1/r^5, on-surface target.
__device__ __forceinline__ bool dl_7ord_onsurf(double r2, double rinv, const Reg& g, double& s3) {
  const double rp = d_rootpi();
  if (r2 < g.r0sq) {
    s3 = 128.0 / 45.0 / rp / (g.d * g.d * g.d * g.d * g.d);
    return false;
  }
  double rinv2 = rinv * rinv;
  double rinv5 = rinv2 * rinv2 * rinv;
  if (r2 > g.d64) {
    s3 = rinv5;
    return false;
  }
  double rd = r2 * rinv * g.inv_d;
  double rd2 = rd * rd;
  double rd4 = rd2 * rd2;
  double rd6 = rd4 * rd2;
  double errfn = erf(rd);
  double r_expfn = 2.0 / rp * rd * exp(-rd2);
  double poly3 = -1.0 - 2.0 / 3.0 * rd2 + 52.0 / 45.0 * rd4 - 8.0 / 45.0 * rd6;
  s3 = (errfn + poly3 * r_expfn) * rinv5;
  return true;
}

// Regularized 1/r^3 kernel of the pressure (Laplace double layer type).
__device__ __forceinline__ bool lapl_dl_7ord(double r2, double rinv, const Reg& g, const Coef& c,
                                             double& s2) {
  const double rp = d_rootpi();
  if (r2 < g.r0sq) {
    s2 = 256.0 / 15.0 / rp / (g.d * g.d * g.d);
    return false;
  }
  double rinv3 = rinv * rinv * rinv;
  if (r2 > g.d64) {
    s2 = rinv3;
    return false;
  }
  double rd = r2 * rinv * g.inv_d;
  double rd2 = rd * rd;
  double rd4 = rd2 * rd2;
  double errfn = erf(rd);
  double r_expfn = rd * exp(-rd2);
  double poly2 = -2.0 / rp + 2.0 * (c.c1 + 2.0 * (c.c2 + c.c3)) * rd2 -
                 4.0 * (c.c2 + 5.0 * c.c3) * rd4 + 8.0 * c.c3 * rd4 * rd2;
  s2 = (errfn + poly2 * r_expfn) * rinv3;
  return true;
}

// sl_7ord and lapl_dl_7ord of one pair together: s1, s2 as sl_7ord, s2p as
// lapl_dl_7ord (its own association of the last polynomial term), sharing
// the powers of r/delta, erf and exp.
__device__ __forceinline__ bool sl_lapl_7ord(double r2, double rinv, const Reg& g, const Coef& c, double& s1,
                                             double& s2, double& s2p) {
  const double rp = d_rootpi();
  if (r2 < g.r0sq) {
    s1 = 32.0 / 5.0 / rp / g.d;
    s2 = 256.0 / 15.0 / rp / (g.d * g.d * g.d);
    s2p = s2;
    return false;
  }
  double rinv3 = rinv * rinv * rinv;
  if (r2 > g.d64) {
    s1 = rinv;
    s2 = rinv3;
    s2p = rinv3;
    return false;
  }
  double rd = r2 * rinv * g.inv_d;
  double rd2 = rd * rd;
  double rd4 = rd2 * rd2;
  double rd6 = rd4 * rd2;
  double errfn = erf(rd);
  double r_expfn = rd * exp(-rd2);
  double poly1 = c.c1 - 2.0 * (c.c2 + c.c3) * rd2 + 4.0 * c.c3 * rd4;
  double poly2 = -2.0 / rp + 2.0 * (c.c1 + 2.0 * (c.c2 + c.c3)) * rd2 -
                 4.0 * (c.c2 + 5.0 * c.c3) * rd4 + 8.0 * c.c3 * rd6;
  double poly2p = -2.0 / rp + 2.0 * (c.c1 + 2.0 * (c.c2 + c.c3)) * rd2 -
                  4.0 * (c.c2 + 5.0 * c.c3) * rd4 + 8.0 * c.c3 * rd4 * rd2;
  s1 = (errfn + poly1 * r_expfn) * rinv;
  s2 = (errfn + poly2 * r_expfn) * rinv3;
  s2p = (errfn + poly2p * r_expfn) * rinv3;
  return true;
}

}  // namespace hr

// ------------------------------------------------------------------ FP32 forms
// The same kernels in FP32 for the mixed-precision path, used only for pairs
// with r > 3 delta. There, for every target distance |b| <= 8 delta (the
// coefficients c1..c3 of reg_coeff) the brackets erf + poly * (r/delta)
// exp(-r^2/delta^2) of s1, s2 and s3 satisfy
// (|erf| + |poly * ...|) / |bracket| < 1.005, so no term cancels and FP32
// keeps ~1e-7 relative accuracy per pair; at 2.5 delta that factor is 1.8, at
// 2 delta 11, and as r -> 0 the s2 / s3 brackets cancel to O((r/delta)^3),
// which is why closer pairs stay in FP64. erff and expf are CUDA's own
// functions.
namespace hr {

struct RegF {
  float inv_d, d64;             // 1/delta, 64 delta^2
  float inv_d2, inv_d3, inv_d5;  // 1/delta^k for the tabulated on-surface factors
};

struct CoefF {
  float c1, c2, c3;
};

constexpr float kRootPiF = 1.77245385f;

__device__ __forceinline__ void sl_7ord_f(float r2, float rinv, const RegF& g, const CoefF& c, float& s1,
                                          float& s2) {
  const float rinv3 = rinv * rinv * rinv;
  if (r2 > g.d64) {
    s1 = rinv;
    s2 = rinv3;
    return;
  }
  const float rd = r2 * rinv * g.inv_d, rd2 = rd * rd, rd4 = rd2 * rd2, rd6 = rd4 * rd2;
  const float errfn = erff(rd), r_expfn = rd * expf(-rd2);
  const float poly1 = c.c1 - 2.0f * (c.c2 + c.c3) * rd2 + 4.0f * c.c3 * rd4;
  const float poly2 = -2.0f / kRootPiF + 2.0f * (c.c1 + 2.0f * (c.c2 + c.c3)) * rd2 -
                      4.0f * (c.c2 + 5.0f * c.c3) * rd4 + 8.0f * c.c3 * rd6;
  s1 = (errfn + poly1 * r_expfn) * rinv;
  s2 = (errfn + poly2 * r_expfn) * rinv3;
}

__device__ __forceinline__ void sl_7ord_onsurf_f(float r2, float rinv, const RegF& g, float& s1, float& s2) {
  const float rinv3 = rinv * rinv * rinv;
  if (r2 > g.d64) {
    s1 = rinv;
    s2 = rinv3;
    return;
  }
  const float rd = r2 * rinv * g.inv_d, rd2 = rd * rd, rd4 = rd2 * rd2, rd6 = rd4 * rd2;
  const float errfn = erff(rd), r_expfn = 2.0f / kRootPiF * rd * expf(-rd2);
  const float poly1 = 11.0f / 5.0f - 26.0f / 15.0f * rd2 + 4.0f / 15.0f * rd4;
  const float poly2 = -1.0f + (118.0f * rd2 - 68.0f * rd4 + 8.0f * rd6) * (1.0f / 15.0f);
  s1 = (errfn + poly1 * r_expfn) * rinv;
  s2 = (errfn + poly2 * r_expfn) * rinv3;
}

__device__ __forceinline__ void dl_7ord_f(float r2, float rinv, const RegF& g, const CoefF& c, float& s2,
                                          float& s3) {
  const float rinv2 = rinv * rinv, rinv3 = rinv2 * rinv;
  if (r2 > g.d64) {
    s2 = rinv3;
    s3 = rinv3 * rinv2;
    return;
  }
  const float rd = r2 * rinv * g.inv_d, rd2 = rd * rd, rd4 = rd2 * rd2, rd6 = rd4 * rd2;
  const float errfn = erff(rd), r_expfn = rd * expf(-rd2);
  const float poly2 = -2.0f / kRootPiF + 2.0f * (c.c1 + 2.0f * (c.c2 + c.c3)) * rd2 -
                      4.0f * (c.c2 + 5.0f * c.c3) * rd4 + 8.0f * c.c3 * rd6;
  const float poly3 = -2.0f / kRootPiF * (1.0f + 2.0f / 3.0f * rd2) +
                      4.0f / 3.0f *
                          ((c.c1 + 4.0f * c.c2 + 12.0f * c.c3) * rd4 - 2.0f * (c.c2 + 9.0f * c.c3) * rd6 +
                           4.0f * c.c3 * rd6 * rd2);
  s2 = (errfn + poly2 * r_expfn) * rinv3;
  s3 = (errfn + poly3 * r_expfn) * (rinv3 * rinv2);
}

__device__ __forceinline__ void dl_7ord_onsurf_f(float r2, float rinv, const RegF& g, float& s3) {
  const float rinv2 = rinv * rinv, rinv5 = rinv2 * rinv2 * rinv;
  if (r2 > g.d64) {
    s3 = rinv5;
    return;
  }
  const float rd = r2 * rinv * g.inv_d, rd2 = rd * rd, rd4 = rd2 * rd2, rd6 = rd4 * rd2;
  const float errfn = erff(rd), r_expfn = 2.0f / kRootPiF * rd * expf(-rd2);
  const float poly3 = -1.0f - 2.0f / 3.0f * rd2 + 52.0f / 45.0f * rd4 - 8.0f / 45.0f * rd6;
  s3 = (errfn + poly3 * r_expfn) * rinv5;
}

// sl_7ord_f and lapl_dl_7ord_f of one pair together (as sl_lapl_7ord).
__device__ __forceinline__ void sl_lapl_7ord_f(float r2, float rinv, const RegF& g, const CoefF& c, float& s1,
                                               float& s2, float& s2p) {
  const float rinv3 = rinv * rinv * rinv;
  if (r2 > g.d64) {
    s1 = rinv;
    s2 = rinv3;
    s2p = rinv3;
    return;
  }
  const float rd = r2 * rinv * g.inv_d, rd2 = rd * rd, rd4 = rd2 * rd2, rd6 = rd4 * rd2;
  const float errfn = erff(rd), r_expfn = rd * expf(-rd2);
  const float poly1 = c.c1 - 2.0f * (c.c2 + c.c3) * rd2 + 4.0f * c.c3 * rd4;
  const float poly2 = -2.0f / kRootPiF + 2.0f * (c.c1 + 2.0f * (c.c2 + c.c3)) * rd2 -
                      4.0f * (c.c2 + 5.0f * c.c3) * rd4 + 8.0f * c.c3 * rd6;
  const float poly2p = -2.0f / kRootPiF + 2.0f * (c.c1 + 2.0f * (c.c2 + c.c3)) * rd2 -
                       4.0f * (c.c2 + 5.0f * c.c3) * rd4 + 8.0f * c.c3 * rd4 * rd2;
  s1 = (errfn + poly1 * r_expfn) * rinv;
  s2 = (errfn + poly2 * r_expfn) * rinv3;
  s2p = (errfn + poly2p * r_expfn) * rinv3;
}

__device__ __forceinline__ void lapl_dl_7ord_f(float r2, float rinv, const RegF& g, const CoefF& c, float& s2) {
  const float rinv3 = rinv * rinv * rinv;
  if (r2 > g.d64) {
    s2 = rinv3;
    return;
  }
  const float rd = r2 * rinv * g.inv_d, rd2 = rd * rd, rd4 = rd2 * rd2;
  const float errfn = erff(rd), r_expfn = rd * expf(-rd2);
  const float poly2 = -2.0f / kRootPiF + 2.0f * (c.c1 + 2.0f * (c.c2 + c.c3)) * rd2 -
                      4.0f * (c.c2 + 5.0f * c.c3) * rd4 + 8.0f * c.c3 * rd4 * rd2;
  s2 = (errfn + poly2 * r_expfn) * rinv3;
}

}  // namespace hr
