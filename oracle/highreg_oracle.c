/*
 * highreg_oracle.c — plain-C restatement of the reference's hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the oracle: tests/, the smoke test
 * and the CPU-baseline leg of bench.py call it to produce the expected answer.
 * The product (high-order-regularization_b200/) never links, loads or calls it.
 *
 * Every function restates one reference routine, cited as file:line within the
 * reference project (2S = highreg_stokes_2surf, E2G =
 * highreg_stokes_extend_to_grid). The operation order of each expression
 * follows the cited line so that, compiled without FMA contraction, results
 * are bit-identical to the reference built the same way; the pinning tests
 * check exactly that against oracle/_ref.
 */
#include "highreg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const double PI_ = 3.14159265358979323846;

static double rootPI(void) { return sqrt(PI_); }
static double denom_EightPI(void) { return 1.0 / (8.0 * PI_); }
static double denom_FourPI(void) { return 1.0 / (4.0 * PI_); }

/* ------------------------------------------------------------------ kernels */

/* evaluate_In_024 + get_reg_coeff_7ord: 2S/utilities.cpp:163-175, 327-337 */
void or_reg_coeff(double lam, double c[3]) {
  double lam2 = lam * lam;
  double e2 = exp(lam2);
  double em2 = exp(-lam2);
  double t = fabs(lam) * erfc(fabs(lam));
  double I0 = em2 / rootPI() - t;
  double I2 = 2.0 / 3.0 * ((0.5 - lam2) * em2 / rootPI() + lam2 * t);
  double I4 = 8.0 / 15.0 * ((0.75 - 0.5 * lam2 + lam2 * lam2) * em2 / rootPI() - lam2 * lam2 * t);
  double c3 = e2 * (2.0 * I0 - 4.0 * I2 + I4) / 8.0;
  double c2 = e2 * (I0 - I2) + (4.0 * lam2 + 7.0) * c3;
  double c1 = 2.0 * e2 * I0 + 2.0 * (lam2 + 1.0) * c2 - (4.0 * lam2 * lam2 + 6.0 * lam2 + 6.0) * c3;
  c[0] = c1;
  c[1] = c2;
  c[2] = c3;
}

/* Stokes_SL_7ord: 2S/utilities.cpp:179-207 */
void or_sl_7ord(double r, double d, const double c[3], double s[2]) {
  double c1 = c[0], c2 = c[1], c3 = c[2];
  if (r < 1e-14) {
    s[0] = 32.0 / 5.0 / rootPI() / d;
    s[1] = 256.0 / 15.0 / rootPI() / (d * d * d);
  } else if (r / d > 8.0) {
    double r2 = r * r;
    s[0] = 1.0 / r;
    s[1] = 1.0 / (r2 * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double rd6 = rd4 * rd2;
    double errfn = erf(rd);
    double r_expfn = rd * exp(-rd2);
    double poly1 = c1 - 2.0 * (c2 + c3) * rd2 + 4.0 * c3 * rd4;
    double poly2 = -2.0 / rootPI() + 2.0 * (c1 + 2.0 * (c2 + c3)) * rd2 -
                   4.0 * (c2 + 5.0 * c3) * rd4 + 8.0 * c3 * rd6;
    double r2 = r * r;
    s[0] = (errfn + poly1 * r_expfn) / r;
    s[1] = (errfn + poly2 * r_expfn) / (r2 * r);
  }
}

/* Stokes_SL_7ord_onSurf: 2S/utilities.cpp:211-254 */
void or_sl_7ord_onsurf(double r, double d, double s[2]) {
  if (r < 1e-14) {
    s[0] = 32.0 / 5.0 / rootPI() / d;
    s[1] = 256.0 / 15.0 / rootPI() / (d * d * d);
  } else if (r / d > 8.0) {
    double r2 = r * r;
    s[0] = 1.0 / r;
    s[1] = 1.0 / (r2 * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double rd6 = rd4 * rd2;
    double errfn = erf(rd);
    double r_expfn = 2.0 / rootPI() * rd * exp(-rd2);
    double poly1 = 11.0 / 5.0 - 26.0 / 15.0 * rd2 + 4.0 / 15.0 * rd4;
    double poly2 = -1.0 + (118.0 * rd2 - 68.0 * rd4 + 8.0 * rd6) / 15.0;
    double r2 = r * r;
    s[0] = (errfn + poly1 * r_expfn) / r;
    s[1] = (errfn + poly2 * r_expfn) / (r2 * r);
  }
}

/* Stokes_DL_7ord: 2S/utilities.cpp:258-288 */
void or_dl_7ord(double r, double d, const double c[3], double s[2]) {
  double c1 = c[0], c2 = c[1], c3 = c[2];
  if (r < 1e-14) {
    s[0] = 256.0 / 15.0 / rootPI() / (d * d * d);
    s[1] = 0.0;
  } else if (r / d > 8.0) {
    double r2 = r * r;
    s[0] = 1.0 / (r2 * r);
    s[1] = 1.0 / (r2 * r2 * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double rd6 = rd4 * rd2;
    double errfn = erf(rd);
    double r_expfn = rd * exp(-rd2);
    double poly2 = -2.0 / rootPI() + 2.0 * (c1 + 2.0 * (c2 + c3)) * rd2 -
                   4.0 * (c2 + 5.0 * c3) * rd4 + 8.0 * c3 * rd6;
    double poly3 = -2.0 / rootPI() * (1.0 + 2.0 / 3.0 * rd2) +
                   4.0 / 3.0 * ((c1 + 4.0 * c2 + 12.0 * c3) * rd4 - 2.0 * (c2 + 9.0 * c3) * rd6 +
                                4.0 * c3 * rd6 * rd2);
    double r2 = r * r;
    s[0] = (errfn + poly2 * r_expfn) / (r2 * r);
    s[1] = (errfn + poly3 * r_expfn) / (r2 * r2 * r);
  }
}

/* Stokes_DL_7ord_onSurf: 2S/utilities.cpp:292-323 */
double or_dl_7ord_onsurf(double r, double d) {
  if (r < 1e-14) {
    return 128.0 / 45.0 / rootPI() / (d * d * d * d * d);
  } else if (r / d > 8.0) {
    double r2 = r * r;
    return 1.0 / (r2 * r2 * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double rd6 = rd4 * rd2;
    double errfn = erf(rd);
    double r_expfn = 2.0 / rootPI() * rd * exp(-rd2);
    double poly3 = -1.0 - 2.0 / 3.0 * rd2 + 52.0 / 45.0 * rd4 - 8.0 / 45.0 * rd6;
    double r2 = r * r;
    return (errfn + poly3 * r_expfn) / (r2 * r2 * r);
  }
}

/* Lapl_DL_7ord: E2G/utilities.cpp:190-211 */
double or_lapl_dl_7ord(double r, double d, const double c[3]) {
  double c1 = c[0], c2 = c[1], c3 = c[2];
  if (r < 1e-14) {
    return 256.0 / 15.0 / rootPI() / (d * d * d);
  } else if (r / d > 8.0) {
    return 1.0 / (r * r * r);
  } else {
    double rd = r / d;
    double rd2 = rd * rd;
    double rd4 = rd2 * rd2;
    double errfn = erf(rd);
    double r_expfn = rd * exp(-rd2);
    double poly2 = -2.0 / rootPI() + 2.0 * (c1 + 2.0 * (c2 + c3)) * rd2 -
                   4.0 * (c2 + 5.0 * c3) * rd4 + 8.0 * c3 * rd4 * rd2;
    return (errfn + poly2 * r_expfn) / (r * r * r);
  }
}

/* ------------------------------------------------------------ direct sums */

/* stokes_SL_7ord: 2S/stokeslets.cpp:94-135 (also E2G/stokes.cpp:53-97) */
static void sl_7ord_one(double DEL, int nq, const double* xq, const double* nrm, const double* aq,
                        const double* f, double f0_dot_n0, double x, double y, double z, double b,
                        double SL[3]) {
  double c[3];
  or_reg_coeff(b / DEL, c);
  SL[0] = SL[1] = SL[2] = 0.0;
  for (int j = 0; j < nq; j++) {
    double dx = x - xq[3 * j], dy = y - xq[3 * j + 1], dz = z - xq[3 * j + 2];
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    double area = aq[j];
    double f_x = f[3 * j] - f0_dot_n0 * nrm[3 * j];
    double f_y = f[3 * j + 1] - f0_dot_n0 * nrm[3 * j + 1];
    double f_z = f[3 * j + 2] - f0_dot_n0 * nrm[3 * j + 2];
    double f_dot_dx = f_x * dx + f_y * dy + f_z * dz;
    double H[2];
    or_sl_7ord(r, DEL, c, H);
    double H1 = H[0] * area;
    double H2 = H[1] * (area * f_dot_dx);
    SL[0] += f_x * H1 + dx * H2;
    SL[1] += f_y * H1 + dy * H2;
    SL[2] += f_z * H1 + dz * H2;
  }
  SL[0] *= denom_EightPI();
  SL[1] *= denom_EightPI();
  SL[2] *= denom_EightPI();
}

/* eval_Stokes_SL_offSurf: 2S/stokeslets.cpp:12-86 */
void or_sl_offsurf_direct(double DEL, int nq, const double* xq, const double* nrm, const double* aq,
                          const double* f, int nt, const double* xt, const double* b,
                          const double* f0, const double* n0, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double pt[3] = {xt[3 * i], xt[3 * i + 1], xt[3 * i + 2]};
    double SL[3];
    if (fabs(b[i] / DEL) > 8.0) {
      SL[0] = SL[1] = SL[2] = 0.0;
      for (int j = 0; j < nq; j++) {
        double dx[3];
        for (int k = 0; k < 3; k++) dx[k] = pt[k] - xq[3 * j + k];
        double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        double r = sqrt(r2);
        const double* ft = &f[3 * j];
        double f_dot_dx = ft[0] * dx[0] + ft[1] * dx[1] + ft[2] * dx[2];
        double area = aq[j];
        double H1 = area / r;
        double H2 = f_dot_dx * area / (r2 * r);
        for (int k = 0; k < 3; k++) SL[k] += ft[k] * H1 + dx[k] * H2;
      }
      for (int k = 0; k < 3; k++) SL[k] *= denom_EightPI();
    } else {
      double f0_dot_n0 = f0[3 * i] * n0[3 * i] + f0[3 * i + 1] * n0[3 * i + 1] +
                         f0[3 * i + 2] * n0[3 * i + 2];
      sl_7ord_one(DEL, nq, xq, nrm, aq, f, f0_dot_n0, pt[0], pt[1], pt[2], b[i], SL);
    }
    out[3 * i] = SL[0];
    out[3 * i + 1] = SL[1];
    out[3 * i + 2] = SL[2];
  }
}

/* eval_Stokes_SL_onSurf + stokes_SL_7ord_onSurf: 2S/stokeslets.cpp:141-225 */
void or_sl_onsurf_direct(double DEL, int nq, const double* xq, const double* nrm, const double* aq,
                         const double* f, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nq; i++) {
    double x = xq[3 * i], y = xq[3 * i + 1], z = xq[3 * i + 2];
    double f0_dot_n0 = f[3 * i] * nrm[3 * i] + f[3 * i + 1] * nrm[3 * i + 1] +
                       f[3 * i + 2] * nrm[3 * i + 2];
    double SL[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < nq; j++) {
      double dx = x - xq[3 * j], dy = y - xq[3 * j + 1], dz = z - xq[3 * j + 2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      double area = aq[j];
      double f_x = f[3 * j] - f0_dot_n0 * nrm[3 * j];
      double f_y = f[3 * j + 1] - f0_dot_n0 * nrm[3 * j + 1];
      double f_z = f[3 * j + 2] - f0_dot_n0 * nrm[3 * j + 2];
      double f_dot_dx = f_x * dx + f_y * dy + f_z * dz;
      double H[2];
      or_sl_7ord_onsurf(r, DEL, H);
      double H1 = H[0] * area;
      double H2 = H[1] * (area * f_dot_dx);
      SL[0] += f_x * H1 + dx * H2;
      SL[1] += f_y * H1 + dy * H2;
      SL[2] += f_z * H1 + dz * H2;
    }
    out[3 * i] = SL[0] * denom_EightPI();
    out[3 * i + 1] = SL[1] * denom_EightPI();
    out[3 * i + 2] = SL[2] * denom_EightPI();
  }
}

/* eval_Stokes_DL_offSurf + stokes_DL_7ord: 2S/stresslets.cpp:13-179 */
void or_dl_offsurf_direct(double DEL, int nq, const double* xq, const double* nrm, const double* aq,
                          const double* g, int nt, const double* xt, const double* b,
                          const double* x0, const double* n0, const double* g0, double* out) {
  const double m6 = -6.0 * denom_EightPI();
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double pt[3] = {xt[3 * i], xt[3 * i + 1], xt[3 * i + 2]};
    double bb = b[i];
    double DL[3] = {0.0, 0.0, 0.0};
    if (fabs(bb) / DEL > 8.0) {
      for (int j = 0; j < nq; j++) {
        double dx[3];
        for (int k = 0; k < 3; k++) dx[k] = pt[k] - xq[3 * j + k];
        double r2 = dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2];
        double r = sqrt(r2);
        const double* gt = &g[3 * j];
        const double* nj = &nrm[3 * j];
        double g_dot_dx = gt[0] * dx[0] + gt[1] * dx[1] + gt[2] * dx[2];
        double n_dot_dx = nj[0] * dx[0] + nj[1] * dx[1] + nj[2] * dx[2];
        double kernel = g_dot_dx * n_dot_dx / (r2 * r2 * r) * aq[j];
        for (int k = 0; k < 3; k++) DL[k] += dx[k] * kernel;
      }
      for (int k = 0; k < 3; k++) DL[k] *= m6;
    } else {
      const double* X0 = &x0[3 * i];
      const double* N0 = &n0[3 * i];
      const double* G0 = &g0[3 * i];
      double c[3];
      or_reg_coeff(bb / DEL, c);
      for (int j = 0; j < nq; j++) {
        double dx = pt[0] - xq[3 * j], dy = pt[1] - xq[3 * j + 1], dz = pt[2] - xq[3 * j + 2];
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        double area = aq[j];
        double H[2];
        or_dl_7ord(r, DEL, c, H);
        double H2 = H[0] * area;
        double H3 = H[1] * area;
        double x_hat0 = xq[3 * j] - X0[0];
        double x_hat1 = xq[3 * j + 1] - X0[1];
        double x_hat2 = xq[3 * j + 2] - X0[2];
        double sig_sq = (x_hat0 * x_hat0 + x_hat1 * x_hat1 + x_hat2 * x_hat2) -
                        2.0 * bb * (x_hat0 * N0[0] + x_hat1 * N0[1] + x_hat2 * N0[2]);
        double g_dl0 = g[3 * j] - G0[0];
        double g_dl1 = g[3 * j + 1] - G0[1];
        double g_dl2 = g[3 * j + 2] - G0[2];
        double g_dot_n0 = g_dl0 * N0[0] + g_dl1 * N0[1] + g_dl2 * N0[2];
        double g_dot_x_hat = g_dl0 * x_hat0 + g_dl1 * x_hat1 + g_dl2 * x_hat2;
        const double* Nj = &nrm[3 * j];
        double n0_dot_n = N0[0] * Nj[0] + N0[1] * Nj[1] + N0[2] * Nj[2];
        double x_hat_dot_n = x_hat0 * Nj[0] + x_hat1 * Nj[1] + x_hat2 * Nj[2];
        double c_m1a = g_dot_n0 * n0_dot_n;
        double c_m1b = g_dot_x_hat * n0_dot_n + g_dot_n0 * x_hat_dot_n;
        double c_m2a = g_dot_x_hat * x_hat_dot_n;
        double c_m2b = bb * (g_dot_x_hat * n0_dot_n + g_dot_n0 * x_hat_dot_n);
        double t1_x = dx * c_m1a - N0[0] * c_m1b;
        double t1_y = dy * c_m1a - N0[1] * c_m1b;
        double t1_z = dz * c_m1a - N0[2] * c_m1b;
        DL[0] += t1_x * H2;
        DL[1] += t1_y * H2;
        DL[2] += t1_z * H2;
        DL[0] += (-sig_sq * t1_x + dx * c_m2a + x_hat0 * c_m2b) * H3;
        DL[1] += (-sig_sq * t1_y + dy * c_m2a + x_hat1 * c_m2b) * H3;
        DL[2] += (-sig_sq * t1_z + dz * c_m2a + x_hat2 * c_m2b) * H3;
      }
      for (int k = 0; k < 3; k++) DL[k] *= m6;
      if ((bb < 0.0) || (fabs(bb) < 1.0e-14)) {
        DL[0] += G0[0];
        DL[1] += G0[1];
        DL[2] += G0[2];
      }
    }
    out[3 * i] = DL[0];
    out[3 * i + 1] = DL[1];
    out[3 * i + 2] = DL[2];
  }
}

/* eval_Stokes_DL_onSurf + stokes_DL_7ord_onSurf: 2S/stresslets.cpp:186-279 */
void or_dl_onsurf_direct(double DEL, int nq, const double* xq, const double* nrm, const double* aq,
                         const double* g, double* out) {
  const double m6 = -6.0 * denom_EightPI();
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nq; i++) {
    double x = xq[3 * i], y = xq[3 * i + 1], z = xq[3 * i + 2];
    const double* G0 = &g[3 * i];
    double DL[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < nq; j++) {
      double dx = x - xq[3 * j], dy = y - xq[3 * j + 1], dz = z - xq[3 * j + 2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      double area = aq[j];
      double H3 = or_dl_7ord_onsurf(r, DEL);
      double g_dl0 = g[3 * j] - G0[0];
      double g_dl1 = g[3 * j + 1] - G0[1];
      double g_dl2 = g[3 * j + 2] - G0[2];
      const double* Nj = &nrm[3 * j];
      double dx_dot_n = dx * Nj[0] + dy * Nj[1] + dz * Nj[2];
      double dx_dot_g = dx * g_dl0 + dy * g_dl1 + dz * g_dl2;
      H3 *= dx_dot_n * dx_dot_g * area;
      DL[0] += dx * H3;
      DL[1] += dy * H3;
      DL[2] += dz * H3;
    }
    for (int k = 0; k < 3; k++) DL[k] *= m6;
    out[3 * i] = DL[0] + 0.5 * G0[0];
    out[3 * i + 1] = DL[1] + 0.5 * G0[1];
    out[3 * i + 2] = DL[2] + 0.5 * G0[2];
  }
}

/* ------------------------------------------------------ extend-to-grid sums */

/* stokes_SL_away: E2G/stokes.cpp:13-45 */
void or_e2g_sl_away(int nq, const double* xq, const double* aq, const double* f, int nt,
                    const double* xt, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double x = xt[3 * i], y = xt[3 * i + 1], z = xt[3 * i + 2];
    double SL[3] = {0.0, 0.0, 0.0};
    for (int j = 0; j < nq; j++) {
      double dx = x - xq[3 * j], dy = y - xq[3 * j + 1], dz = z - xq[3 * j + 2];
      double r2 = dx * dx + dy * dy + dz * dz;
      double area = aq[j];
      double f_dot_dx = f[3 * j] * dx + f[3 * j + 1] * dy + f[3 * j + 2] * dz;
      double H1 = 1.0 / sqrt(r2) * area;
      double H2 = H1 / r2 * f_dot_dx;
      SL[0] += f[3 * j] * H1 + dx * H2;
      SL[1] += f[3 * j + 1] * H1 + dy * H2;
      SL[2] += f[3 * j + 2] * H1 + dz * H2;
    }
    out[3 * i] = SL[0] * denom_EightPI();
    out[3 * i + 1] = SL[1] * denom_EightPI();
    out[3 * i + 2] = SL[2] * denom_EightPI();
  }
}

/* stokes_pressure_away: E2G/stokes.cpp:102-126 */
double or_e2g_p_away_one(int nq, const double* xq, const double* aq, const double* f, double x,
                         double y, double z) {
  double p = 0.0;
  for (int j = 0; j < nq; j++) {
    double dx = x - xq[3 * j], dy = y - xq[3 * j + 1], dz = z - xq[3 * j + 2];
    double r2 = dx * dx + dy * dy + dz * dz;
    double H2 = 1.0 / (r2 * sqrt(r2));
    H2 *= f[3 * j] * dx + f[3 * j + 1] * dy + f[3 * j + 2] * dz;
    p += H2 * aq[j];
  }
  return p * denom_FourPI();
}

void or_e2g_p_away(int nq, const double* xq, const double* aq, const double* f, int nt,
                   const double* xt, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++)
    out[i] = or_e2g_p_away_one(nq, xq, aq, f, xt[3 * i], xt[3 * i + 1], xt[3 * i + 2]);
}

/* E2G band Stokeslet: stokes_SL_7ord at each target, f0_dot_n0 from the exact
 * density at the nearest point (E2G/main.cpp:1337-1345, E2G/stokes.cpp:53-97) */
void or_e2g_sl_7ord(double DEL, int nq, const double* xq, const double* nrm, const double* aq,
                    const double* f, int nt, const double* xt, const double* b,
                    const double* f0, const double* n0, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double f0_dot_n0 = f0[3 * i] * n0[3 * i] + f0[3 * i + 1] * n0[3 * i + 1] +
                       f0[3 * i + 2] * n0[3 * i + 2];
    sl_7ord_one(DEL, nq, xq, nrm, aq, f, f0_dot_n0, xt[3 * i], xt[3 * i + 1], xt[3 * i + 2], b[i],
                &out[3 * i]);
  }
}

/* stokes_pressure_7ord: E2G/stokes.cpp:134-203 */
void or_e2g_p_7ord(double DEL, int nq, const double* xq, const double* nrm, const double* aq,
                   const double* f, int nt, const double* xt, const double* b, const double* f0,
                   const double* n0, double* out) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int i = 0; i < nt; i++) {
    double x = xt[3 * i], y = xt[3 * i + 1], z = xt[3 * i + 2];
    const double* F0 = &f0[3 * i];
    const double* N0 = &n0[3 * i];
    double c[3];
    or_reg_coeff(b[i] / DEL, c);
    double f0_dot_n0 = F0[0] * N0[0] + F0[1] * N0[1] + F0[2] * N0[2];
    double n0xf0[3] = {N0[1] * F0[2] - N0[2] * F0[1], N0[2] * F0[0] - N0[0] * F0[2],
                       N0[0] * F0[1] - N0[1] * F0[0]};
    double p = 0.0;
    for (int j = 0; j < nq; j++) {
      double dx[3] = {x - xq[3 * j], y - xq[3 * j + 1], z - xq[3 * j + 2]};
      double r = sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
      double area = aq[j];
      double H2 = or_lapl_dl_7ord(r, DEL, c);
      const double* n = &nrm[3 * j];
      const double* ff = &f[3 * j];
      double f_dot_n = ff[0] * n[0] + ff[1] * n[1] + ff[2] * n[2];
      double ncf[3] = {n[1] * ff[2] - n[2] * ff[1], n[2] * ff[0] - n[0] * ff[2],
                       n[0] * ff[1] - n[1] * ff[0]};
      ncf[0] -= n0xf0[0];
      ncf[1] -= n0xf0[1];
      ncf[2] -= n0xf0[2];
      double n_dot_dx = n[0] * dx[0] + n[1] * dx[1] + n[2] * dx[2];
      double ncdx[3] = {n[1] * dx[2] - n[2] * dx[1], n[2] * dx[0] - n[0] * dx[2],
                        n[0] * dx[1] - n[1] * dx[0]};
      double normal = -(f_dot_n - f0_dot_n0) * n_dot_dx;
      double tangential = -(ncf[0] * ncdx[0] + ncf[1] * ncdx[1] + ncf[2] * ncdx[2]);
      p += (normal + tangential) * H2 * area;
    }
    p *= -denom_FourPI();
    if (b[i] < -1.e-12) p -= f0_dot_n0;
    out[i] = p;
  }
}

/* ---------------------------------------------------------------- treecode */

typedef struct {
  long m0, m1; /* members[0..1], inclusive, in tree order */
  double xi[2], yi[2], zi[2];
  double xc, yc, zc, MAC;
  int child[8];
  int nchild;
} or_node;

typedef struct {
  int P, N0;
  double sq_theta;
  or_node* nodes;
  int nnodes, cap;
  /* particles in tree order */
  double *x, *y, *z, *nx, *ny, *nz, *area, *lam0, *lam1, *lam2;
  double* tcheb; /* per node: 3*(P+1) */
  double* mom;   /* per node: 12 * (P+1)^3 */
} or_tree;

static int tree_push(or_tree* T, const or_node* n) {
  if (T->nnodes == T->cap) {
    T->cap = T->cap ? 2 * T->cap : 64;
    T->nodes = (or_node*)realloc(T->nodes, sizeof(or_node) * T->cap);
  }
  T->nodes[T->nnodes] = *n;
  return T->nnodes++;
}

/* build_tree_init: 2S/KITC.cpp:30-69 */
static void tree_init(or_tree* T, const double ctr[3], long n) {
  or_node r;
  memset(&r, 0, sizeof(r));
  r.m0 = 0;
  r.m1 = n - 1;
  double eps = 1.e-8;
  r.xi[0] = -1.0 - eps + ctr[0];
  r.xi[1] = 1.0 + eps + ctr[0];
  r.yi[0] = -1.0 - eps + ctr[1];
  r.yi[1] = 1.0 + eps + ctr[1];
  r.zi[0] = -1.0 - eps + ctr[2];
  r.zi[1] = 1.0 + eps + ctr[2];
  r.xc = 0.5 * (r.xi[0] + r.xi[1]);
  r.yc = 0.5 * (r.yi[0] + r.yi[1]);
  r.zc = 0.5 * (r.zi[0] + r.zi[1]);
  r.MAC = (3 * 10 * 10 / 4) / T->sq_theta;
  tree_push(T, &r);
}

/* split_tree_node: 2S/KITC.cpp:116-322. The reference's swap loop with its
 * address table yields a stable partition of the node's range by octant
 * (octant 0..7 in the order of its if-chain), which is what is done here. */
static void tree_split(or_tree* T, int pi) {
  or_node par = T->nodes[pi];
  double x0 = par.xi[0], x1 = par.xi[1], y0 = par.yi[0], y1 = par.yi[1], z0 = par.zi[0],
         z1 = par.zi[1];
  double mx = (x0 + x1) / 2.0, my = (y0 + y1) / 2.0, mz = (z0 + z1) / 2.0;
  double xc0 = (x0 + mx) / 2.0, xc1 = (x1 + mx) / 2.0;
  double yc0 = (y0 + my) / 2.0, yc1 = (y1 + my) / 2.0;
  double zc0 = (z0 + mz) / 2.0, zc1 = (z1 + mz) / 2.0;
  long n = par.m1 - par.m0 + 1;
  int* oct = (int*)malloc(sizeof(int) * n);
  long cnt[8] = {0};
  for (long i = 0; i < n; i++) {
    long p = par.m0 + i;
    int bx = T->x[p] > mx, by = T->y[p] > my, bz = T->z[p] > mz;
    oct[i] = bx + 2 * by + 4 * bz;
    cnt[oct[i]]++;
  }
  /* stable partition of all particle arrays */
  double* arrs[10] = {T->x, T->y, T->z, T->nx, T->ny, T->nz, T->area, T->lam0, T->lam1, T->lam2};
  double* tmp = (double*)malloc(sizeof(double) * n);
  long start[8];
  long s = 0;
  for (int o = 0; o < 8; o++) {
    start[o] = s;
    s += cnt[o];
  }
  for (int a = 0; a < 10; a++) {
    long pos[8];
    memcpy(pos, start, sizeof(pos));
    for (long i = 0; i < n; i++) tmp[pos[oct[i]]++] = arrs[a][par.m0 + i];
    memcpy(arrs[a] + par.m0, tmp, sizeof(double) * n);
  }
  free(tmp);
  free(oct);
  T->nodes[pi].nchild = 0;
  for (int o = 0; o < 8; o++) {
    if (cnt[o] == 0) continue;
    int bx = o & 1, by = (o >> 1) & 1, bz = (o >> 2) & 1;
    or_node c;
    memset(&c, 0, sizeof(c));
    c.xi[0] = bx ? mx : x0;
    c.xi[1] = bx ? x1 : mx;
    c.yi[0] = by ? my : y0;
    c.yi[1] = by ? y1 : my;
    c.zi[0] = bz ? mz : z0;
    c.zi[1] = bz ? z1 : mz;
    c.xc = bx ? xc1 : xc0;
    c.yc = by ? yc1 : yc0;
    c.zc = bz ? zc1 : zc0;
    double ex = bx ? (x1 - xc1) : (mx - xc0);
    double ey = by ? (y1 - yc1) : (my - yc0);
    double ez = bz ? (z1 - zc1) : (mz - zc0);
    c.MAC = (ex * ex + ey * ey + ez * ez) / T->sq_theta;
    c.m0 = par.m0 + start[o];
    c.m1 = c.m0 + cnt[o] - 1;
    int ci = tree_push(T, &c);
    T->nodes[pi].child[T->nodes[pi].nchild++] = ci;
  }
}

/* build_tree_3D_Recursive: 2S/KITC.cpp:325-348 */
static void tree_build_rec(or_tree* T, int pi) {
  long n = T->nodes[pi].m1 - T->nodes[pi].m0 + 1;
  if (n >= (long)T->N0) {
    tree_split(T, pi);
    int nc = T->nodes[pi].nchild;
    int ch[8];
    memcpy(ch, T->nodes[pi].child, sizeof(ch));
    for (int i = 0; i < nc; i++) tree_build_rec(T, ch[i]);
  }
}

/* Cluster_Chev_Points: 2S/KITC.cpp:780-804 */
static void tree_cheb(or_tree* T) {
  int P = T->P;
  double h = 3.14159265358979323846 / P;
  double* t = (double*)malloc(sizeof(double) * (P + 1));
  for (int i = 0; i < P + 1; i++) t[i] = cos(i * h);
  T->tcheb = (double*)malloc(sizeof(double) * 3 * (P + 1) * T->nnodes);
  for (int n = 0; n < T->nnodes; n++) {
    const or_node* c = &T->nodes[n];
    double* tc = &T->tcheb[(size_t)n * 3 * (P + 1)];
    for (int i = 0; i < P + 1; i++) {
      tc[i] = c->xi[0] + (t[i] + 1) / 2 * (c->xi[1] - c->xi[0]);
      tc[P + 1 + i] = c->yi[0] + (t[i] + 1) / 2 * (c->yi[1] - c->yi[0]);
      tc[2 * (P + 1) + i] = c->zi[0] + (t[i] + 1) / 2 * (c->zi[1] - c->zi[0]);
    }
  }
  free(t);
}

/* Panel_Moments_SL / Panel_Moments_DL: 2S/KITC.cpp:351-668 */
static void tree_moments(or_tree* T, int ni, int dl) {
  int P = T->P, P1 = P + 1, Pf = P1 * P1 * P1;
  const or_node* c = &T->nodes[ni];
  const double* t1 = &T->tcheb[(size_t)ni * 3 * P1];
  const double* t2 = t1 + P1;
  const double* t3 = t2 + P1;
  double* w = (double*)malloc(sizeof(double) * P1);
  for (int j = 0; j < P1; j++) {
    double dj = (j == 0 || j == P) ? 0.5 : 1.0;
    w[j] = ((j % 2 == 0) ? 1 : -1) * dj;
  }
  long n = c->m1 - c->m0 + 1;
  double* a1 = (double*)calloc((size_t)P1 * n, sizeof(double));
  double* a2 = (double*)calloc((size_t)P1 * n, sizeof(double));
  double* a3 = (double*)calloc((size_t)P1 * n, sizeof(double));
  double* D = (double*)calloc(n, sizeof(double));
  for (long q = 0; q < n; q++) {
    long p = c->m0 + q;
    double x = T->x[p], y = T->y[p], z = T->z[p];
    int f1 = -1, f2 = -1, f3 = -1;
    double S1 = 0.0, S2 = 0.0, S3 = 0.0;
    for (int j = 0; j < P1; j++) {
      if (fabs(x - t1[j]) < 1.e-07) f1 = j;
      else {
        double tt = w[j] / (x - t1[j]);
        a1[(size_t)j * n + q] = tt;
        S1 += tt;
      }
      if (fabs(y - t2[j]) < 1.e-07) f2 = j;
      else {
        double tt = w[j] / (y - t2[j]);
        a2[(size_t)j * n + q] = tt;
        S2 += tt;
      }
      if (fabs(z - t3[j]) < 1.e-07) f3 = j;
      else {
        double tt = w[j] / (z - t3[j]);
        a3[(size_t)j * n + q] = tt;
        S3 += tt;
      }
    }
    if (f1 > -1) {
      S1 = 1.0;
      for (int j = 0; j < P1; j++) a1[(size_t)j * n + q] = 0.0;
      a1[(size_t)f1 * n + q] = 1.0;
    }
    if (f2 > -1) {
      S2 = 1.0;
      for (int j = 0; j < P1; j++) a2[(size_t)j * n + q] = 0.0;
      a2[(size_t)f2 * n + q] = 1.0;
    }
    if (f3 > -1) {
      S3 = 1.0;
      for (int j = 0; j < P1; j++) a3[(size_t)j * n + q] = 0.0;
      a3[(size_t)f3 * n + q] = 1.0;
    }
    D[q] = 1.0 / (S1 * S2 * S3);
  }
  double* M = &T->mom[(size_t)ni * 12 * Pf];
  int kk = -1;
  for (int i = 0; i < P1; i++)
    for (int j = 0; j < P1; j++)
      for (int k = 0; k < P1; k++) {
        kk++;
        double sum[12] = {0};
        for (long q = 0; q < n; q++) {
          long p = c->m0 + q;
          double nx = T->nx[p], ny = T->ny[p], nz = T->nz[p];
          double s = a1[(size_t)i * n + q] * a2[(size_t)j * n + q] * a3[(size_t)k * n + q] * D[q];
          s *= T->area[p];
          if (!dl) {
            sum[0] += s * T->lam0[p];
            sum[1] += s * T->lam1[p];
            sum[2] += s * T->lam2[p];
            sum[3] += s * nx;
            sum[4] += s * ny;
            sum[5] += s * nz;
          } else {
            sum[0] += s * T->lam0[p] * nx;
            sum[1] += s * T->lam0[p] * ny;
            sum[2] += s * T->lam0[p] * nz;
            sum[3] += s * T->lam1[p] * nx;
            sum[4] += s * T->lam1[p] * ny;
            sum[5] += s * T->lam1[p] * nz;
            sum[6] += s * T->lam2[p] * nx;
            sum[7] += s * T->lam2[p] * ny;
            sum[8] += s * T->lam2[p] * nz;
            sum[9] += s * nx;
            sum[10] += s * ny;
            sum[11] += s * nz;
          }
        }
        for (int cc = 0; cc < (dl ? 12 : 6); cc++) M[(size_t)cc * Pf + kk] = sum[cc];
      }
  free(a1);
  free(a2);
  free(a3);
  free(D);
  free(w);
}

/* Call_Treecode_SL: 2S/KITC.cpp:671-721 */
static void far_sl(const or_tree* T, int ni, double x, double y, double z, double f0n0,
                   double u[3]) {
  int P1 = T->P + 1, Pf = P1 * P1 * P1;
  const double* t1 = &T->tcheb[(size_t)ni * 3 * P1];
  const double* t2 = t1 + P1;
  const double* t3 = t2 + P1;
  const double* M = &T->mom[(size_t)ni * 12 * Pf];
  u[0] = u[1] = u[2] = 0.0;
  int kk = -1;
  for (int i = 0; i < P1; i++) {
    double dx0 = x - t1[i];
    double ti = dx0 * dx0;
    for (int j = 0; j < P1; j++) {
      double dx1 = y - t2[j];
      double tj = dx1 * dx1;
      for (int k = 0; k < P1; k++) {
        double dx2 = z - t3[k];
        double tk = dx2 * dx2;
        kk++;
        double m0 = M[kk] - f0n0 * M[3 * Pf + kk];
        double m1 = M[Pf + kk] - f0n0 * M[4 * Pf + kk];
        double m2 = M[2 * Pf + kk] - f0n0 * M[5 * Pf + kk];
        double r2 = ti + tj + tk;
        double r = sqrt(r2);
        double temp = (m0 * dx0 + m1 * dx1 + m2 * dx2) / (r2 * r);
        u[0] += m0 / r + temp * dx0;
        u[1] += m1 / r + temp * dx1;
        u[2] += m2 / r + temp * dx2;
      }
    }
  }
}

/* Call_Treecode_DL: 2S/KITC.cpp:724-777 */
static void far_dl(const or_tree* T, int ni, double x, double y, double z, const double g0[3],
                   double u[3]) {
  int P1 = T->P + 1, Pf = P1 * P1 * P1;
  const double* t1 = &T->tcheb[(size_t)ni * 3 * P1];
  const double* t2 = t1 + P1;
  const double* t3 = t2 + P1;
  const double* M = &T->mom[(size_t)ni * 12 * Pf];
  u[0] = u[1] = u[2] = 0.0;
  int kk = -1;
  for (int i = 0; i < P1; i++) {
    double dx0 = x - t1[i];
    double ti = dx0 * dx0;
    for (int j = 0; j < P1; j++) {
      double dx1 = y - t2[j];
      double tj = dx1 * dx1;
      for (int k = 0; k < P1; k++) {
        double dx2 = z - t3[k];
        double tk = dx2 * dx2;
        kk++;
        double tmp[3];
        for (int l = 0; l < 3; l++) {
          double a = M[(size_t)(3 * l) * Pf + kk] - g0[l] * M[9 * (size_t)Pf + kk];
          double b = M[(size_t)(3 * l + 1) * Pf + kk] - g0[l] * M[10 * (size_t)Pf + kk];
          double c = M[(size_t)(3 * l + 2) * Pf + kk] - g0[l] * M[11 * (size_t)Pf + kk];
          tmp[l] = a * dx0 + b * dx1 + c * dx2;
        }
        double r2 = ti + tj + tk;
        double r = sqrt(r2);
        double kernel = (tmp[0] * dx0 + tmp[1] * dx1 + tmp[2] * dx2) / (r2 * r2 * r);
        u[0] += dx0 * kernel;
        u[1] += dx1 * kernel;
        u[2] += dx2 * kernel;
      }
    }
  }
}

typedef struct {
  int kind;
  double DEL;
  double x, y, z, b, f0n0;
  const double *x0, *n0, *g0;
  long n_direct, n_proxy, n_far, n_leaf;
} or_tgt;

/* Call_Ds_SL_onSurf / Call_Ds_SL / Call_Ds_DL_onSurf / Call_Ds_DL:
 * 2S/KITC.cpp:807-1062 */
static void leaf_direct(const or_tree* T, const or_tgt* t, long l1, long l2, double u[3]) {
  u[0] = u[1] = u[2] = 0.0;
  double DEL = t->DEL;
  if (t->kind == 0) {
    for (long j = l1; j <= l2; j++) {
      double dx = t->x - T->x[j], dy = t->y - T->y[j], dz = t->z - T->z[j];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      double area = T->area[j];
      double f_x = T->lam0[j] - t->f0n0 * T->nx[j];
      double f_y = T->lam1[j] - t->f0n0 * T->ny[j];
      double f_z = T->lam2[j] - t->f0n0 * T->nz[j];
      double f_dot_dx = f_x * dx + f_y * dy + f_z * dz;
      double H[2];
      or_sl_7ord_onsurf(r, DEL, H);
      double H1 = H[0] * area;
      double H2 = H[1] * (area * f_dot_dx);
      u[0] += f_x * H1 + dx * H2;
      u[1] += f_y * H1 + dy * H2;
      u[2] += f_z * H1 + dz * H2;
    }
  } else if (t->kind == 1) {
    if (fabs(t->b) / DEL > 8.0) {
      for (long j = l1; j <= l2; j++) {
        double dx = t->x - T->x[j], dy = t->y - T->y[j], dz = t->z - T->z[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2);
        double area = T->area[j];
        double f_x = T->lam0[j], f_y = T->lam1[j], f_z = T->lam2[j];
        double f_dot_dx = f_x * dx + f_y * dy + f_z * dz;
        double H1 = area / r;
        double H2 = f_dot_dx * area / (r2 * r);
        u[0] += f_x * H1 + dx * H2;
        u[1] += f_y * H1 + dy * H2;
        u[2] += f_z * H1 + dz * H2;
      }
    } else {
      double c[3];
      or_reg_coeff(t->b / DEL, c);
      for (long j = l1; j <= l2; j++) {
        double dx = t->x - T->x[j], dy = t->y - T->y[j], dz = t->z - T->z[j];
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        double area = T->area[j];
        double f_x = T->lam0[j] - t->f0n0 * T->nx[j];
        double f_y = T->lam1[j] - t->f0n0 * T->ny[j];
        double f_z = T->lam2[j] - t->f0n0 * T->nz[j];
        double f_dot_dx = f_x * dx + f_y * dy + f_z * dz;
        double H[2];
        or_sl_7ord(r, DEL, c, H);
        double H1 = H[0] * area;
        double H2 = H[1] * (f_dot_dx * area);
        u[0] += f_x * H1 + dx * H2;
        u[1] += f_y * H1 + dy * H2;
        u[2] += f_z * H1 + dz * H2;
      }
    }
  } else if (t->kind == 2) {
    const double* g0 = t->g0;
    for (long j = l1; j <= l2; j++) {
      double dx = t->x - T->x[j], dy = t->y - T->y[j], dz = t->z - T->z[j];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      double g_x = T->lam0[j] - g0[0];
      double g_y = T->lam1[j] - g0[1];
      double g_z = T->lam2[j] - g0[2];
      double g_dot_dx = g_x * dx + g_y * dy + g_z * dz;
      double n_dot_dx = T->nx[j] * dx + T->ny[j] * dy + T->nz[j] * dz;
      double area = T->area[j];
      double H3 = or_dl_7ord_onsurf(r, DEL);
      double kernel = n_dot_dx * g_dot_dx * H3 * area;
      u[0] += dx * kernel;
      u[1] += dy * kernel;
      u[2] += dz * kernel;
    }
  } else {
    double b = t->b;
    if (fabs(b) / DEL > 8.0) {
      for (long j = l1; j <= l2; j++) {
        double dx = t->x - T->x[j], dy = t->y - T->y[j], dz = t->z - T->z[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2);
        double g_dot_dx = T->lam0[j] * dx + T->lam1[j] * dy + T->lam2[j] * dz;
        double n_dot_dx = T->nx[j] * dx + T->ny[j] * dy + T->nz[j] * dz;
        double area = T->area[j];
        double kernel = g_dot_dx * n_dot_dx / (r2 * r2 * r) * area;
        u[0] += dx * kernel;
        u[1] += dy * kernel;
        u[2] += dz * kernel;
      }
    } else {
      const double *x0 = t->x0, *n0 = t->n0, *g0 = t->g0;
      double c[3];
      or_reg_coeff(b / DEL, c);
      for (long j = l1; j <= l2; j++) {
        double dx = t->x - T->x[j], dy = t->y - T->y[j], dz = t->z - T->z[j];
        double r = sqrt(dx * dx + dy * dy + dz * dz);
        double x_hat0 = T->x[j] - x0[0];
        double x_hat1 = T->y[j] - x0[1];
        double x_hat2 = T->z[j] - x0[2];
        double n_x = T->nx[j], n_y = T->ny[j], n_z = T->nz[j];
        double g_x = T->lam0[j] - g0[0];
        double g_y = T->lam1[j] - g0[1];
        double g_z = T->lam2[j] - g0[2];
        double sig_sq = (x_hat0 * x_hat0 + x_hat1 * x_hat1 + x_hat2 * x_hat2) -
                        2.0 * b * (x_hat0 * n0[0] + x_hat1 * n0[1] + x_hat2 * n0[2]);
        double g_dot_n0 = g_x * n0[0] + g_y * n0[1] + g_z * n0[2];
        double g_dot_x_hat = g_x * x_hat0 + g_y * x_hat1 + g_z * x_hat2;
        double n0_dot_n = n0[0] * n_x + n0[1] * n_y + n0[2] * n_z;
        double x_hat_dot_n = x_hat0 * n_x + x_hat1 * n_y + x_hat2 * n_z;
        double c_m1a = g_dot_n0 * n0_dot_n;
        double c_m1b = g_dot_x_hat * n0_dot_n + g_dot_n0 * x_hat_dot_n;
        double c_m2a = g_dot_x_hat * x_hat_dot_n;
        double c_m2b = b * c_m1b;
        double H[2];
        or_dl_7ord(r, DEL, c, H);
        double area = T->area[j];
        double H2 = H[0] * area;
        double H3 = H[1] * area;
        double m1, m2;
        m1 = dx * c_m1a - n0[0] * c_m1b;
        m2 = -sig_sq * m1 + dx * c_m2a + x_hat0 * c_m2b;
        u[0] += m1 * H2 + m2 * H3;
        m1 = dy * c_m1a - n0[1] * c_m1b;
        m2 = -sig_sq * m1 + dy * c_m2a + x_hat1 * c_m2b;
        u[1] += m1 * H2 + m2 * H3;
        m1 = dz * c_m1a - n0[2] * c_m1b;
        m2 = -sig_sq * m1 + dz * c_m2a + x_hat2 * c_m2b;
        u[2] += m1 * H2 + m2 * H3;
      }
    }
  }
}

/* eval_{SL,DL}_Sum_cluster(_onSurf): 2S/KITC.cpp:1066-1386 */
static void traverse(const or_tree* T, or_tgt* t, int ni, double Sum[3]) {
  const or_node* c = &T->nodes[ni];
  double tpx = t->x - c->xc, tpy = t->y - c->yc, tpz = t->z - c->zc;
  double R_sq = tpx * tpx + tpy * tpy + tpz * tpz;
  Sum[0] = Sum[1] = Sum[2] = 0.0;
  if (c->MAC < R_sq) {
    double r[3];
    if (t->kind < 2) far_sl(T, ni, t->x, t->y, t->z, t->f0n0, r);
    else far_dl(T, ni, t->x, t->y, t->z, t->g0, r);
    Sum[0] += r[0];
    Sum[1] += r[1];
    Sum[2] += r[2];
    int P1 = T->P + 1;
    t->n_proxy += (long)P1 * P1 * P1;
    t->n_far++;
  } else if ((c->m1 - c->m0) < (long)T->N0) {
    double r[3];
    leaf_direct(T, t, c->m0, c->m1, r);
    Sum[0] += r[0];
    Sum[1] += r[1];
    Sum[2] += r[2];
    t->n_direct += c->m1 - c->m0 + 1;
    t->n_leaf++;
  } else {
    for (int i = 0; i < c->nchild; i++) {
      double r[3];
      traverse(T, t, c->child[i], r);
      Sum[0] += r[0];
      Sum[1] += r[1];
      Sum[2] += r[2];
    }
  }
}

/* eval_Stokes_{SL,DL}_{on,off}Surf_tree: 2S/KITC.cpp:1389-1830 */
int or_kitc_eval(int kind, int P, int N0, double theta, const double ctr[3], double DEL, int nq,
                 const double* xq, const double* nrm, const double* aq, const double* dens, int nt,
                 const double* xt, const double* b, const double* x0, const double* n0,
                 const double* dens0, double* out, long* stats) {
  or_tree T;
  memset(&T, 0, sizeof(T));
  T.P = P;
  T.N0 = N0;
  T.sq_theta = theta * theta;
  double** arrs[10] = {&T.x, &T.y, &T.z, &T.nx, &T.ny, &T.nz, &T.area, &T.lam0, &T.lam1, &T.lam2};
  for (int a = 0; a < 10; a++) *arrs[a] = (double*)malloc(sizeof(double) * (nq > 0 ? nq : 1));
  for (int i = 0; i < nq; i++) {
    T.x[i] = xq[3 * i];
    T.y[i] = xq[3 * i + 1];
    T.z[i] = xq[3 * i + 2];
    T.nx[i] = nrm[3 * i];
    T.ny[i] = nrm[3 * i + 1];
    T.nz[i] = nrm[3 * i + 2];
    T.area[i] = aq[i];
    T.lam0[i] = dens[3 * i];
    T.lam1[i] = dens[3 * i + 1];
    T.lam2[i] = dens[3 * i + 2];
  }
  tree_init(&T, ctr, nq);
  tree_build_rec(&T, 0);
  tree_cheb(&T);
  int P1 = P + 1, Pf = P1 * P1 * P1;
  T.mom = (double*)calloc((size_t)12 * Pf * T.nnodes, sizeof(double));
  int dl = kind >= 2;
  for (int i = 1; i < T.nnodes; i++) tree_moments(&T, i, dl); /* root skipped */
  const double EightPI = 1.0 / (8.0 * PI_);
  const double EightPI6 = -6.0 / (8.0 * PI_);
  long sd = 0, sp = 0, sf = 0, sl = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : sd, sp, sf, sl)
  for (int i = 0; i < nt; i++) {
    or_tgt t;
    memset(&t, 0, sizeof(t));
    t.kind = kind;
    t.DEL = DEL;
    t.x = xt[3 * i];
    t.y = xt[3 * i + 1];
    t.z = xt[3 * i + 2];
    double g0loc[3] = {0, 0, 0};
    if (kind == 0) {
      t.f0n0 = dens[3 * i] * nrm[3 * i] + dens[3 * i + 1] * nrm[3 * i + 1] +
               dens[3 * i + 2] * nrm[3 * i + 2];
    } else if (kind == 1) {
      t.b = b[i];
      t.f0n0 = dens0[3 * i] * n0[3 * i] + dens0[3 * i + 1] * n0[3 * i + 1] +
               dens0[3 * i + 2] * n0[3 * i + 2];
    } else if (kind == 2) {
      g0loc[0] = dens[3 * i];
      g0loc[1] = dens[3 * i + 1];
      g0loc[2] = dens[3 * i + 2];
      t.g0 = g0loc;
    } else {
      t.b = b[i];
      t.x0 = &x0[3 * i];
      t.n0 = &n0[3 * i];
      t.g0 = &dens0[3 * i];
    }
    double u[3];
    traverse(&T, &t, 0, u);
    if (kind < 2) {
      for (int k = 0; k < 3; k++) out[3 * i + k] = u[k] * EightPI;
    } else if (kind == 2) {
      for (int k = 0; k < 3; k++) out[3 * i + k] = u[k] * EightPI6 + 0.5 * g0loc[k];
    } else {
      double xi = 0.0;
      if (fabs(t.b) < 1.0e-12) xi = 0.5;
      else if (t.b < 0.0) xi = 1.0;
      for (int k = 0; k < 3; k++) out[3 * i + k] = u[k] * EightPI6 + xi * t.g0[k];
    }
    sd += t.n_direct;
    sp += t.n_proxy;
    sf += t.n_far;
    sl += t.n_leaf;
  }
  if (stats) {
    stats[0] = sd;
    stats[1] = sp;
    stats[2] = sf;
    stats[3] = sl;
  }
  for (int a = 0; a < 10; a++) free(*arrs[a]);
  free(T.nodes);
  free(T.tcheb);
  free(T.mom);
  return T.nnodes;
}

/* ------------------------------------------------- density interpolation */

/* sixPoint_coeff: 2S/main.cpp:750-757 */
static void six_coeff(double p, double c[6]) {
  c[0] = -p * (p * p - 1.0) * (p - 2.0) * (p - 3.0) / 120.0;
  c[1] = p * (p - 1.0) * (p * p - 4.0) * (p - 3.0) / 24.0;
  c[2] = -(p * p - 1.0) * (p * p - 4.0) * (p - 3.0) / 12.0;
  c[3] = p * (p + 1.0) * (p * p - 4.0) * (p - 3.0) / 12.0;
  c[4] = -p * (p * p - 1.0) * (p + 2.0) * (p - 3.0) / 24.0;
  c[5] = p * (p * p - 1.0) * (p * p - 4.0) / 120.0;
}

/* interpolate_DL_density + sixPoint_stencil + sixPointInterpolate:
 * 2S/main.cpp:682-778, 916-1046 (search over all quadrature points, last
 * match wins; unset slots read point 0 as the reference does) */
void or_interp_dl_density(double h, const double ctr[3], int nq, const double* xq,
                          const double* g, int nt, const int* nrst, const double* x0,
                          const int* i123, double* g0_out) {
#pragma omp parallel for schedule(dynamic, 8)
  for (int i = 0; i < nt; i++) {
    g0_out[3 * i] = g0_out[3 * i + 1] = g0_out[3 * i + 2] = 0.0;
    if (nrst[i] == 0) continue;
    const double* X0 = &x0[3 * i];
    int ind1 = i123[3 * i], ind2 = i123[3 * i + 1], ind3 = i123[3 * i + 2];
    double xLow = floor((X0[ind1] - ctr[ind1]) / h) * h + ctr[ind1];
    double yLow = floor((X0[ind2] - ctr[ind2]) / h) * h + ctr[ind2];
    double xHigh = xLow + h;
    double yHigh = yLow + h;
    double z0 = X0[ind3] - ctr[ind3];
    double tol = 1.e-14;
    int st[6][6];
    memset(st, 0, sizeof(st));
    double cx[6] = {xLow - 2.0 * h, xLow - h, xLow, xHigh, xHigh + h, xHigh + 2.0 * h};
    double cy[6] = {yLow - 2.0 * h, yLow - h, yLow, yHigh, yHigh + h, yHigh + 2.0 * h};
    for (int j = 0; j < nq; j++) {
      double z = xq[3 * j + ind3] - ctr[ind3];
      if (((z0 > 0) && (z > 0)) || ((z0 < 0) && (z < 0))) {
        double X = xq[3 * j + ind1];
        double Y = xq[3 * j + ind2];
        int col = -1;
        for (int a = 0; a < 6; a++)
          if (fabs(cx[a] - X) < tol) {
            col = a;
            break;
          }
        if (col < 0) continue;
        for (int bb = 0; bb < 6; bb++)
          if (fabs(cy[bb] - Y) < tol) {
            st[col][bb] = j;
            break;
          }
      }
    }
    double p = (X0[ind1] - xLow) / h;
    double q = (X0[ind2] - yLow) / h;
    double a[6], bq[6];
    six_coeff(p, a);
    six_coeff(q, bq);
    for (int comp = 0; comp < 3; comp++) {
      double ft[6];
      for (int jj = 0; jj < 6; jj++) {
        ft[jj] = 0.0;
        for (int ii = 0; ii < 6; ii++) ft[jj] += a[ii] * g[3 * st[ii][jj] + comp];
      }
      double v = 0.0;
      for (int jj = 0; jj < 6; jj++) v += bq[jj] * ft[jj];
      g0_out[3 * i + comp] = v;
    }
  }
}

/* --------------------------------------------------------- two-surface IE */

static void eval_dl(const or_scene2s* sc, int s, int t, const double* g, const double* g0t,
                    double* out) {
  int nq = sc->nq[s];
  if (s == t) {
    if (sc->tree)
      or_kitc_eval(2, sc->P, sc->N0, sc->theta, sc->ctr[s], sc->DEL, nq, sc->xq[s], sc->nrm[s],
                   sc->area[s], g, nq, sc->xq[s], NULL, NULL, NULL, NULL, out, NULL);
    else
      or_dl_onsurf_direct(sc->DEL, nq, sc->xq[s], sc->nrm[s], sc->area[s], g, out);
  } else {
    int nt = sc->nq[t];
    if (sc->tree)
      or_kitc_eval(3, sc->P, sc->N0, sc->theta, sc->ctr[s], sc->DEL, nq, sc->xq[s], sc->nrm[s],
                   sc->area[s], g, nt, sc->xq[t], sc->b[t], sc->x0[t], sc->n0[t], g0t, out, NULL);
    else
      or_dl_offsurf_direct(sc->DEL, nq, sc->xq[s], sc->nrm[s], sc->area[s], g, nt, sc->xq[t],
                           sc->b[t], sc->x0[t], sc->n0[t], g0t, out);
  }
}

static void eval_sl(const or_scene2s* sc, int s, int t, const double* f, double* out) {
  int nq = sc->nq[s];
  if (s == t) {
    if (sc->tree)
      or_kitc_eval(0, sc->P, sc->N0, sc->theta, sc->ctr[s], sc->DEL, nq, sc->xq[s], sc->nrm[s],
                   sc->area[s], f, nq, sc->xq[s], NULL, NULL, NULL, NULL, out, NULL);
    else
      or_sl_onsurf_direct(sc->DEL, nq, sc->xq[s], sc->nrm[s], sc->area[s], f, out);
  } else {
    int nt = sc->nq[t];
    if (sc->tree)
      or_kitc_eval(1, sc->P, sc->N0, sc->theta, sc->ctr[s], sc->DEL, nq, sc->xq[s], sc->nrm[s],
                   sc->area[s], f, nt, sc->xq[t], sc->b[t], NULL, sc->n0[t], sc->f0[t], out,
                   NULL);
    else
      or_sl_offsurf_direct(sc->DEL, nq, sc->xq[s], sc->nrm[s], sc->area[s], f, nt, sc->xq[t],
                           sc->b[t], sc->f0[t], sc->n0[t], out);
  }
}

/* solve_IE_1step: 2S/main.cpp:541-677 */
void or_matvec_2s(const or_scene2s* sc, const double* u_in, double* u_out) {
  int n1 = sc->nq[0], n2 = sc->nq[1];
  const double* g1 = u_in;
  const double* g2 = u_in + 3 * n1;
  double* g0_t2 = (double*)calloc(3 * (size_t)n2, sizeof(double));
  double* g0_t1 = (double*)calloc(3 * (size_t)n1, sizeof(double));
  or_interp_dl_density(sc->h, sc->ctr[0], n1, sc->xq[0], g1, n2, sc->nrst[1], sc->x0[1],
                       sc->i123[1], g0_t2);
  or_interp_dl_density(sc->h, sc->ctr[1], n2, sc->xq[1], g2, n1, sc->nrst[0], sc->x0[0],
                       sc->i123[0], g0_t1);
  double* on1 = (double*)malloc(sizeof(double) * 3 * n1);
  double* comp1 = (double*)malloc(sizeof(double) * 3 * n2);
  double* comp2 = (double*)malloc(sizeof(double) * 3 * n1);
  double* on2 = (double*)malloc(sizeof(double) * 3 * n2);
  eval_dl(sc, 0, 0, g1, NULL, on1);
  eval_dl(sc, 0, 1, g1, g0_t2, comp1);
  eval_dl(sc, 1, 0, g2, g0_t1, comp2);
  eval_dl(sc, 1, 1, g2, NULL, on2);
  double factor = 2.0 / 3.0;
  for (int i = 0; i < 3 * n1; i++) u_out[i] = u_in[i] - on1[i] * factor;
  for (int i = 0; i < 3 * n2; i++) u_out[3 * n1 + i] = u_in[3 * n1 + i] - comp1[i] * factor;
  for (int i = 0; i < 3 * n1; i++) u_out[i] -= comp2[i] * factor;
  for (int i = 0; i < 3 * n2; i++) u_out[3 * n1 + i] -= on2[i] * factor;
  free(g0_t1);
  free(g0_t2);
  free(on1);
  free(comp1);
  free(comp2);
  free(on2);
}

/* eval_SL + right-hand side: 2S/main.cpp:186-207, 421-537 */
void or_rhs_2s(const or_scene2s* sc, const double* f1, const double* f2, double* bvec) {
  int n1 = sc->nq[0], n2 = sc->nq[1];
  double* on1 = (double*)malloc(sizeof(double) * 3 * n1);
  double* comp1 = (double*)malloc(sizeof(double) * 3 * n2);
  double* comp2 = (double*)malloc(sizeof(double) * 3 * n1);
  double* on2 = (double*)malloc(sizeof(double) * 3 * n2);
  eval_sl(sc, 0, 0, f1, on1);
  eval_sl(sc, 0, 1, f1, comp1);
  eval_sl(sc, 1, 0, f2, comp2);
  eval_sl(sc, 1, 1, f2, on2);
  double factor = 2.0 / 3.0;
  for (int i = 0; i < 3 * n1; i++) {
    double SL = on1[i];
    SL += comp2[i];
    bvec[i] = -SL * factor;
  }
  for (int i = 0; i < 3 * n2; i++) {
    double SL = comp1[i];
    SL += on2[i];
    bvec[3 * n1 + i] = -SL * factor;
  }
  free(on1);
  free(comp1);
  free(comp2);
  free(on2);
}

/* GMRES: 2S/main.cpp:236-416 (MGS Arnoldi, Givens rotations, relative
 * residual), with r0 = b - A x0 at every (re)start. */
int or_gmres_2s(const or_scene2s* sc, const double* bvec, double* x, int im, int iter_max,
                double tol, double* resid_hist) {
  int n = 3 * (sc->nq[0] + sc->nq[1]);
  double* V = (double*)malloc(sizeof(double) * (size_t)n * (im + 1));
  double* H = (double*)calloc((size_t)(im + 1) * im, sizeof(double));
  double* gg = (double*)calloc(im + 1, sizeof(double));
  double* y = (double*)calloc(im + 1, sizeof(double));
  double* cs = (double*)calloc(im, sizeof(double));
  double* sn = (double*)calloc(im, sizeof(double));
  double* Ax = (double*)malloc(sizeof(double) * n);
  double b_norm = 0.0;
  for (int i = 0; i < n; i++) b_norm += bvec[i] * bvec[i];
  b_norm = sqrt(b_norm);
  int iter = 0;
  double error = 1.0;
#define Hm(i, j) H[(size_t)(i) * im + (j)]
  while (iter <= iter_max) {
    int nonzero = 0;
    for (int i = 0; i < n; i++)
      if (x[i] != 0.0) {
        nonzero = 1;
        break;
      }
    if (nonzero) or_matvec_2s(sc, x, Ax);
    else memset(Ax, 0, sizeof(double) * n);
    double r_norm = 0.0;
    for (int i = 0; i < n; i++) {
      V[i] = bvec[i] - Ax[i];
      r_norm += V[i] * V[i];
    }
    r_norm = sqrt(r_norm);
    error = r_norm;
    if (b_norm > 1.e-8) error /= b_norm;
    if (error <= tol || iter >= iter_max) break;
    double temp = 1.0 / r_norm;
    for (int i = 0; i < n; i++) V[i] *= temp;
    gg[0] = r_norm;
    int j = -1;
    while ((j < im - 1) && (error > tol) && (iter < iter_max)) {
      j++;
      iter++;
      double* vj1 = &V[(size_t)(j + 1) * n];
      or_matvec_2s(sc, &V[(size_t)j * n], vj1);
      for (int i = 0; i <= j; i++) {
        double t = 0.0;
        const double* vi = &V[(size_t)i * n];
        for (int k = 0; k < n; k++) t += vi[k] * vj1[k];
        Hm(i, j) = t;
        for (int k = 0; k < n; k++) vj1[k] -= t * vi[k];
      }
      double v_norm = 0.0;
      for (int i = 0; i < n; i++) v_norm += vj1[i] * vj1[i];
      v_norm = sqrt(v_norm);
      Hm(j + 1, j) = v_norm;
      if (v_norm != 0.0) {
        v_norm = 1.0 / v_norm;
        for (int k = 0; k < n; k++) vj1[k] *= v_norm;
      }
      for (int i = 0; i <= j - 1; i++) {
        double t = Hm(i, j);
        Hm(i, j) = cs[i] * t + sn[i] * Hm(i + 1, j);
        Hm(i + 1, j) = -sn[i] * t + cs[i] * Hm(i + 1, j);
      }
      double hh = sqrt(Hm(j, j) * Hm(j, j) + Hm(j + 1, j) * Hm(j + 1, j));
      if (hh == 0.0) hh = 1.e-16;
      cs[j] = Hm(j, j) / hh;
      sn[j] = Hm(j + 1, j) / hh;
      Hm(j, j) = cs[j] * Hm(j, j) + sn[j] * Hm(j + 1, j);
      for (int i = 0; i <= j; i++) Hm(j + 1, i) = 0.0;
      gg[j + 1] = -sn[j] * gg[j];
      gg[j] = cs[j] * gg[j];
      error = fabs(gg[j + 1]);
      if (b_norm > 1.e-8) error /= b_norm;
      if (resid_hist) resid_hist[iter - 1] = error;
    }
    /* x += V y with y from the triangular solve (2S/main.cpp:402-414) */
    for (int i = 0; i <= j; i++) y[i] = gg[i];
    y[j] = y[j] / Hm(j, j);
    for (int k = j - 1; k >= 0; k--) {
      double t = y[k];
      for (int i = k + 1; i <= j; i++) t -= Hm(k, i) * y[i];
      y[k] = t / Hm(k, k);
    }
    for (int i = 0; i <= j; i++) {
      const double* vi = &V[(size_t)i * n];
      for (int k = 0; k < n; k++) x[k] += y[i] * vi[k];
    }
    if (error <= tol || iter >= iter_max) break;
  }
#undef Hm
  free(V);
  free(H);
  free(gg);
  free(y);
  free(cs);
  free(sn);
  free(Ax);
  return iter;
}

/* ----------------------------------------------------- Poisson / DST path */

#define G3(a, i, j, k) (a)[(((size_t)(i) * (N + 1) + (j)) * (N + 1) + (k))]

/* extend_into_cube: E2G/main.cpp:1494-1527 */
void or_extend_into_cube(int N, double L, double h, const double* g, double* G) {
  for (int i = 0; i <= N; i++) {
    double x = i * h / L;
    for (int j = 0; j <= N; j++) {
      double y = j * h / L;
      for (int k = 0; k <= N; k++) {
        double z = k * h / L;
        double F, E1, E2, E3, C;
        F = x * G3(g, N, j, k) + (1.0 - x) * G3(g, 0, j, k);
        F += y * G3(g, i, N, k) + (1.0 - y) * G3(g, i, 0, k);
        F += z * G3(g, i, j, N) + (1.0 - z) * G3(g, i, j, 0);
        E1 = (1.0 - y) * (1.0 - z) * G3(g, i, 0, 0) + (1.0 - y) * z * G3(g, i, 0, N) +
             y * (1.0 - z) * G3(g, i, N, 0) + y * z * G3(g, i, N, N);
        E2 = (1.0 - x) * (1.0 - z) * G3(g, 0, j, 0) + (1.0 - x) * z * G3(g, 0, j, N) +
             x * (1.0 - z) * G3(g, N, j, 0) + x * z * G3(g, N, j, N);
        E3 = (1.0 - x) * (1.0 - y) * G3(g, 0, 0, k) + (1.0 - x) * y * G3(g, 0, N, k) +
             x * (1.0 - y) * G3(g, N, 0, k) + x * y * G3(g, N, N, k);
        C = (1.0 - x) * (1.0 - y) * (1.0 - z) * G3(g, 0, 0, 0) +
            (1.0 - x) * (1.0 - y) * z * G3(g, 0, 0, N) +
            (1.0 - x) * y * (1.0 - z) * G3(g, 0, N, 0) + (1.0 - x) * y * z * G3(g, 0, N, N) +
            x * (1.0 - y) * (1.0 - z) * G3(g, N, 0, 0) + x * (1.0 - y) * z * G3(g, N, 0, N) +
            x * y * (1.0 - z) * G3(g, N, N, 0) + x * y * z * G3(g, N, N, N);
        G3(G, i, j, k) = F - E1 - E2 - E3 + C;
      }
    }
  }
}

/* lapl_4ord_inCube: E2G/main.cpp:1566-1594 */
void or_lapl_4ord_incube(int N, const double* G, double* rhs) {
  for (int i = 1; i < N; i++)
    for (int j = 1; j < N; j++)
      for (int k = 1; k < N; k++) {
        size_t ijk = ((size_t)(i - 1) * (N - 1) + j - 1) * (N - 1) + k - 1;
        double lap7 = G3(G, i + 1, j, k) + G3(G, i - 1, j, k) + G3(G, i, j + 1, k) +
                      G3(G, i, j - 1, k) + G3(G, i, j, k + 1) + G3(G, i, j, k - 1) -
                      6.0 * G3(G, i, j, k);
        double temp1 = G3(G, i + 1, j + 1, k + 1) + G3(G, i + 1, j - 1, k + 1) +
                       G3(G, i - 1, j + 1, k + 1) + G3(G, i - 1, j - 1, k + 1) -
                       4.0 * G3(G, i, j, k);
        double temp2 = G3(G, i + 1, j + 1, k - 1) + G3(G, i + 1, j - 1, k - 1) +
                       G3(G, i - 1, j + 1, k - 1) + G3(G, i - 1, j - 1, k - 1) -
                       4.0 * G3(G, i, j, k);
        rhs[ijk] = -2.0 / 3.0 * (lap7 + (temp1 + temp2) / 8.0);
      }
}

/* lapl_4ord_nearSurfc: E2G/main.cpp:1598-1637 (mask = BAND2 points) */
void or_lapl_4ord_band2(int N, const unsigned char* band2, const double* u, double* rhs) {
  for (int i = 1; i < N; i++)
    for (int j = 1; j < N; j++)
      for (int k = 1; k < N; k++) {
        if (!G3(band2, i, j, k)) continue;
        size_t ijk = ((size_t)(i - 1) * (N - 1) + j - 1) * (N - 1) + k - 1;
        double lap7 = G3(u, i + 1, j, k) + G3(u, i - 1, j, k) + G3(u, i, j + 1, k) +
                      G3(u, i, j - 1, k) + G3(u, i, j, k + 1) + G3(u, i, j, k - 1) -
                      6.0 * G3(u, i, j, k);
        double temp1 = G3(u, i + 1, j + 1, k + 1) + G3(u, i + 1, j - 1, k + 1) +
                       G3(u, i - 1, j + 1, k + 1) + G3(u, i - 1, j - 1, k + 1) -
                       4.0 * G3(u, i, j, k);
        double temp2 = G3(u, i + 1, j + 1, k - 1) + G3(u, i + 1, j - 1, k - 1) +
                       G3(u, i - 1, j + 1, k - 1) + G3(u, i - 1, j - 1, k - 1) -
                       4.0 * G3(u, i, j, k);
        rhs[ijk] += 2.0 / 3.0 * (lap7 + (temp1 + temp2) / 8.0);
      }
}

/* dp_dx_4ord / dp_dy_4ord / dp_dz_4ord: E2G/main.cpp:1641-1823
 * (mask = exterior points outside BAND2). */
void or_dp_4ord(int N, double h, int axis, const unsigned char* outmask, const double* p,
                double* rhs) {
  for (int i = 1; i < N; i++)
    for (int j = 1; j < N; j++)
      for (int k = 1; k < N; k++) {
        if (!G3(outmask, i, j, k)) continue;
        size_t ijk = ((size_t)(i - 1) * (N - 1) + j - 1) * (N - 1) + k - 1;
        int c = axis == 0 ? i : (axis == 1 ? j : k);
        int di = axis == 0, dj = axis == 1, dk = axis == 2;
#define PP(o) G3(p, i + (o)*di, j + (o)*dj, k + (o)*dk)
        double d;
        if (c == 0 || c == 1) {
          d = -(25.0 / 12.0) * PP(0) + 4.0 * PP(1) - 3.0 * PP(2) + (4.0 / 3.0) * PP(3) -
              0.25 * PP(4);
        } else if (c == N || c == (N - 1)) {
          d = (25.0 / 12.0) * PP(0) - 4.0 * PP(-1) + 3.0 * PP(-2) - (4.0 / 3.0) * PP(-3) +
              0.25 * PP(-4);
        } else {
          d = -PP(2) + 8.0 * PP(1) - 8.0 * PP(-1) + PP(-2);
          d /= 12.0;
        }
#undef PP
        rhs[ijk] += d * h;
      }
}

/* FFTW RODFT00 definition, applied on each axis of a row-major n^3 array */
void or_dst1_3d(int n, double* a) {
  double* S = (double*)malloc(sizeof(double) * (size_t)n * n);
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++)
      S[(size_t)k * n + j] = 2.0 * sin(PI_ * (double)((long)(j + 1) * (k + 1)) / (double)(n + 1));
  long strides[3] = {(long)n * n, n, 1};
  for (int ax = 2; ax >= 0; ax--) {
    long sa = strides[ax];
    int o1 = (ax + 1) % 3, o2 = (ax + 2) % 3;
#pragma omp parallel
    {
      double* line = (double*)malloc(sizeof(double) * n);
      double* res = (double*)malloc(sizeof(double) * n);
#pragma omp for collapse(2)
      for (int u = 0; u < n; u++)
        for (int v = 0; v < n; v++) {
          double* base = a + (long)u * strides[o1] + (long)v * strides[o2];
          for (int j = 0; j < n; j++) line[j] = base[(long)j * sa];
          for (int k = 0; k < n; k++) {
            double s = 0.0;
            const double* row = &S[(size_t)k * n];
            for (int j = 0; j < n; j++) s += row[j] * line[j];
            res[k] = s;
          }
          for (int k = 0; k < n; k++) base[(long)k * sa] = res[k];
        }
      free(line);
      free(res);
    }
  }
  free(S);
}

/* fftw_DST_Poisson3d_FD: E2G/main.cpp:1423-1489 */
void or_dst_poisson(int N, double* f) {
  or_dst1_3d(N, f);
  double pi_over_n = PI_ / (N + 1);
  for (int i = 0; i < N; i++) {
    double c1 = cos((i + 1) * pi_over_n);
    double s1 = sin((i + 1) * pi_over_n / 2.0);
    s1 *= -2.0 * s1;
    for (int j = 0; j < N; j++) {
      double c2 = cos((j + 1) * pi_over_n);
      double s2 = sin((j + 1) * pi_over_n / 2.0);
      s2 *= -2.0 * s2;
      for (int k = 0; k < N; k++) {
        double c3 = cos((k + 1) * pi_over_n);
        double s3 = sin((k + 1) * pi_over_n / 2.0);
        s3 *= -2.0 * s3;
        size_t ind = ((size_t)i * N + j) * N + k;
        double lap7 = s1 + s2 + s3;
        double sum8 = c1 * c2 * c3;
        double factor = 2.0 / 3.0 * (2.0 * lap7 + sum8 - 1.0);
        if (fabs(factor) > 1.e-14) f[ind] /= factor;
        else f[ind] = 0.0;
      }
    }
  }
  or_dst1_3d(N, f);
  double scale = 1. / pow(2 * (N + 1), 3);
  for (size_t i = 0; i < (size_t)N * N * N; i++) f[i] *= scale;
}

/* solve_Poisson: E2G/main.cpp:969-1044 */
void or_solve_poisson(int N, double L, double h, const unsigned char* band2,
                      const unsigned char* outmask, const double* p, double* u, int variable) {
  size_t m = (size_t)(N + 1) * (N + 1) * (N + 1);
  size_t n3 = (size_t)(N - 1) * (N - 1) * (N - 1);
  double* w = (double*)malloc(sizeof(double) * m);
  double* rhs = (double*)calloc(n3, sizeof(double));
  or_extend_into_cube(N, L, h, u, w);
  or_lapl_4ord_incube(N, w, rhs);
  or_lapl_4ord_band2(N, band2, u, rhs);
  if (variable >= 1 && variable <= 3) or_dp_4ord(N, h, variable - 1, outmask, p, rhs);
  or_dst_poisson(N - 1, rhs);
  memcpy(u, w, sizeof(double) * m);
  for (int i = 1; i < N; i++)
    for (int j = 1; j < N; j++)
      for (int k = 1; k < N; k++) {
        size_t ijk = ((size_t)(i - 1) * (N - 1) + j - 1) * (N - 1) + k - 1;
        G3(u, i, j, k) += rhs[ijk];
      }
  free(w);
  free(rhs);
}
#undef G3
