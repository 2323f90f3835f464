// hr_pairs.cuh — per-pair regularized kernels (device functions).
//
// FP64 versions follow the reference formulas term by term:
//   reg_coeff         get_reg_coeff_7ord + evaluate_In_024   2S/utilities.cpp:163-175, 327-337
//   sl_7ord           Stokes_SL_7ord                         2S/utilities.cpp:179-207
//   sl_7ord_onsurf    Stokes_SL_7ord_onSurf                  2S/utilities.cpp:211-254
//   dl_7ord           Stokes_DL_7ord                         2S/utilities.cpp:258-288
//   dl_7ord_onsurf    Stokes_DL_7ord_onSurf                  2S/utilities.cpp:292-323
//   lapl_dl_7ord      Lapl_DL_7ord                           E2G/utilities.cpp:190-211
// erf, erfc, exp and sqrt are CUDA's own functions; nothing here re-derives them.
// Branches: r < 1e-14 uses the limit values, r/delta > 8 the singular kernel.
#pragma once
#include <cuda_runtime.h>

namespace hr {

// sqrt(pi) as the reference computes it: sqrt of the double nearest pi (0x1.c5bf891b4ef6ap+0)
__device__ __forceinline__ double d_rootpi() { return 1.7724538509055159; }

struct Coef {
  double c1, c2, c3;
};

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

// Regularized Stokeslet factors (s1, s2) for an off-surface target.
__device__ __forceinline__ void sl_7ord(double r, double d, const Coef& c, double& s1, double& s2) {
  const double rp = d_rootpi();
  if (r < 1e-14) {
    s1 = 32.0 / 5.0 / rp / d;
    s2 = 256.0 / 15.0 / rp / (d * d * d);
  } else if (r / d > 8.0) {
    double r2 = r * r;
    s1 = 1.0 / r;
    s2 = 1.0 / (r2 * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double rd6 = rd4 * rd2;
    double errfn = erf(rd);
    double r_expfn = rd * exp(-rd2);
    double poly1 = c.c1 - 2.0 * (c.c2 + c.c3) * rd2 + 4.0 * c.c3 * rd4;
    double poly2 = -2.0 / rp + 2.0 * (c.c1 + 2.0 * (c.c2 + c.c3)) * rd2 -
                   4.0 * (c.c2 + 5.0 * c.c3) * rd4 + 8.0 * c.c3 * rd6;
    double r2 = r * r;
    s1 = (errfn + poly1 * r_expfn) / r;
    s2 = (errfn + poly2 * r_expfn) / (r2 * r);
  }
}

// Regularized Stokeslet factors for an on-surface target (lambda = 0).
__device__ __forceinline__ void sl_7ord_onsurf(double r, double d, double& s1, double& s2) {
  const double rp = d_rootpi();
  if (r < 1e-14) {
    s1 = 32.0 / 5.0 / rp / d;
    s2 = 256.0 / 15.0 / rp / (d * d * d);
  } else if (r / d > 8.0) {
    double r2 = r * r;
    s1 = 1.0 / r;
    s2 = 1.0 / (r2 * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double rd6 = rd4 * rd2;
    double errfn = erf(rd);
    double r_expfn = 2.0 / rp * rd * exp(-rd2);
    double poly1 = 11.0 / 5.0 - 26.0 / 15.0 * rd2 + 4.0 / 15.0 * rd4;
    double poly2 = -1.0 + (118.0 * rd2 - 68.0 * rd4 + 8.0 * rd6) / 15.0;
    double r2 = r * r;
    s1 = (errfn + poly1 * r_expfn) / r;
    s2 = (errfn + poly2 * r_expfn) / (r2 * r);
  }
}

// Regularized stresslet factors (s2, s3) for an off-surface target.
__device__ __forceinline__ void dl_7ord(double r, double d, const Coef& c, double& s2, double& s3) {
  const double rp = d_rootpi();
  if (r < 1e-14) {
    s2 = 256.0 / 15.0 / rp / (d * d * d);
    s3 = 0.0;
  } else if (r / d > 8.0) {
    double r2 = r * r;
    s2 = 1.0 / (r2 * r);
    s3 = 1.0 / (r2 * r2 * r);
  } else {
    double rd = r / d;
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
    double r2 = r * r;
    s2 = (errfn + poly2 * r_expfn) / (r2 * r);
    s3 = (errfn + poly3 * r_expfn) / (r2 * r2 * r);
  }
}

// Regularized stresslet factor s3 for an on-surface target.
__device__ __forceinline__ double dl_7ord_onsurf(double r, double d) {
  const double rp = d_rootpi();
  if (r < 1e-14) {
    return 128.0 / 45.0 / rp / (d * d * d * d * d);
  } else if (r / d > 8.0) {
    double r2 = r * r;
    return 1.0 / (r2 * r2 * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double rd6 = rd4 * rd2;
    double errfn = erf(rd);
    double r_expfn = 2.0 / rp * rd * exp(-rd2);
    double poly3 = -1.0 - 2.0 / 3.0 * rd2 + 52.0 / 45.0 * rd4 - 8.0 / 45.0 * rd6;
    double r2 = r * r;
    return (errfn + poly3 * r_expfn) / (r2 * r2 * r);
  }
}

// Regularized 1/r^3 kernel of the pressure (Laplace double layer type).
__device__ __forceinline__ double lapl_dl_7ord(double r, double d, const Coef& c) {
  const double rp = d_rootpi();
  if (r < 1e-14) {
    return 256.0 / 15.0 / rp / (d * d * d);
  } else if (r / d > 8.0) {
    return 1.0 / (r * r * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double errfn = erf(rd);
    double r_expfn = rd * exp(-rd2);
    double poly2 = -2.0 / rp + 2.0 * (c.c1 + 2.0 * (c.c2 + c.c3)) * rd2 -
                   4.0 * (c.c2 + 5.0 * c.c3) * rd4 + 8.0 * c.c3 * rd4 * rd2;
    return (errfn + poly2 * r_expfn) / (r * r * r);
  }
}

}  // namespace hr
