// hr_eval.cu — the boundary-sum kernel family.
//
// One CTA owns one block of 128 spatially sorted targets (one target per
// thread, FP64 accumulators in registers) and walks that block's interaction
// entries in a fixed order, so every result is deterministic:
//   * near entry  -> direct sum over the node's member sources, staged in
//                    shared memory in tiles of 256 (Call_Ds_*, 2S/KITC.cpp:807-1062;
//                    in direct mode the single node holds all sources, i.e.
//                    eval_Stokes_*_{on,off}Surf of 2S/stokeslets.cpp and
//                    2S/stresslets.cpp, and the sums of E2G/stokes.cpp);
//   * far entry   -> the node's (P+1)^3 proxy points with their moments staged
//                    in shared memory (Call_Treecode_*, 2S/KITC.cpp:671-777).
// A warp whose mask word is zero for an entry skips the arithmetic entirely.
//
// Precision. FP64: every pair in FP64. MIXED: every pair with r > 3 delta is
// evaluated in FP32 from centre-relative FP32 coordinates (the plain kernels
// of far targets, the regularized kernels with erff/expf for 3 delta < r <=
// 8 delta, the subtraction forms of near targets, and all proxy
// interactions), summed per 16 terms in FP32 and added to the FP64
// per-target accumulators; the r <= 3 delta pairs, where the smoothing
// brackets cancel, stay in FP64.
#include <cstdio>

#include "hr_device.h"
#include "hr_pairs.cuh"

namespace hr {

namespace {

#define HR_SMOOTH_STORAGE __device__ const
#include "hr_smoothing_tables.inc"

// On-surface smoothing factors without erf / exp / rsqrt: for r <= 8 delta,
// s1 = G1(s) / delta, s2 = G2(s) / delta^3, s3 = G3(s) / delta^5 with
// s = r^2 / delta^2, each G a piecewise polynomial (64 pieces uniform in
// r/delta, degree 11 in s - centre) fitted in 80-digit arithmetic to the
// reference's formulas (2S/utilities.cpp:211-254, :292-323) with ~1e-16
// relative error; G(0) is the reference's r -> 0 value. The table of a kernel
// family is staged in shared memory once per CTA.
constexpr int kSmoothN = HR_SMOOTH_PIECES * (HR_SMOOTH_DEG + 2);

__device__ __forceinline__ double smooth_eval(const double* __restrict__ tab, double s) {
  int i = (int)(sqrtf((float)s) * (HR_SMOOTH_PIECES / 8.0f));
  i = min(max(i, 0), HR_SMOOTH_PIECES - 1);
  const double* p = tab + i * (HR_SMOOTH_DEG + 2);
  const double t = s - p[0];
  double v = p[HR_SMOOTH_DEG + 1];
#pragma unroll
  for (int k = HR_SMOOTH_DEG; k >= 1; k--) v = fma(v, t, p[k]);
  return v;
}

constexpr int kNT = 256;         // sources per shared-memory tile
constexpr int kSmem = 10 * kNT;  // doubles: 10 SoA arrays of a source tile
constexpr int kMaxP1 = 16;

struct Tgt {
  double px, py, pz;
  double b;
  int near;
  double f0n0;
  double x0[3], n0[3], g0[3];
  double n0xf0[3];
  Coef c;
};

struct Tgt32 {
  float px, py, pz;  // relative to the source surface centre
  float f0n0;        // 0 for targets without subtraction
  float g0[3];
  float n0xf0[3];
  float b;
  float x0[3];       // relative to the source surface centre
  float n0[3];
  CoefF c;
};

template <int KIND>
__device__ __forceinline__ void load_target(const EvalTask& T, int t, bool valid, Tgt& S,
                                            Tgt32& F) {
  S.px = S.py = S.pz = 0.0;
  S.b = 0.0;
  S.f0n0 = 0.0;
  for (int k = 0; k < 3; k++) S.x0[k] = S.n0[k] = S.g0[k] = S.n0xf0[k] = 0.0;
  S.c.c1 = S.c.c2 = S.c.c3 = 0.0;
  // regularized-kernel kinds: on-surface sums and the E2G band sums
  S.near = (KIND == K_SL_ON || KIND == K_DL_ON || KIND == K_E2G_SL7 || KIND == K_E2G_P7) ? 1 : 0;
  if (valid) {
    S.px = T.txyz[3 * t];
    S.py = T.txyz[3 * t + 1];
    S.pz = T.txyz[3 * t + 2];
    if (KIND == K_SL_ON) {
      // f0_dot_n0 = Surfc[i].f . Surfc[i].Nrml  (2S/KITC.cpp:1461, 2S/stokeslets.cpp:167)
      S.f0n0 = T.tq[3 * t] * T.tnrm[3 * t] + T.tq[3 * t + 1] * T.tnrm[3 * t + 1] +
               T.tq[3 * t + 2] * T.tnrm[3 * t + 2];
    } else if (KIND == K_SL_OFF || KIND == K_E2G_SL7) {
      S.b = T.tb[t];
      if (KIND == K_SL_OFF) S.near = T.tnear[t];
      // f0_dot_n0 = nrst_f . nrst_Nrml  (2S/KITC.cpp:1568, E2G/main.cpp:1338)
      S.f0n0 = T.tf0[3 * t] * T.tn0[3 * t] + T.tf0[3 * t + 1] * T.tn0[3 * t + 1] +
               T.tf0[3 * t + 2] * T.tn0[3 * t + 2];
      if (S.near) S.c = reg_coeff(S.b / T.DEL);
    } else if (KIND == K_DL_ON) {
      for (int k = 0; k < 3; k++) S.g0[k] = T.tq[3 * t + k];
    } else if (KIND == K_DL_OFF) {
      S.b = T.tb[t];
      S.near = T.tnear[t];
      for (int k = 0; k < 3; k++) {
        S.x0[k] = T.tx0[3 * t + k];
        S.n0[k] = T.tn0[3 * t + k];
        S.g0[k] = T.tg0[3 * t + k];
      }
      if (S.near) S.c = reg_coeff(S.b / T.DEL);
    } else if (KIND == K_E2G_P7) {
      S.b = T.tb[t];
      double f0[3], n0[3];
      for (int k = 0; k < 3; k++) {
        f0[k] = T.tf0[3 * t + k];
        n0[k] = T.tn0[3 * t + k];
      }
      // E2G/stokes.cpp:144-145
      S.f0n0 = f0[0] * n0[0] + f0[1] * n0[1] + f0[2] * n0[2];
      S.n0xf0[0] = n0[1] * f0[2] - n0[2] * f0[1];
      S.n0xf0[1] = n0[2] * f0[0] - n0[0] * f0[2];
      S.n0xf0[2] = n0[0] * f0[1] - n0[1] * f0[0];
      S.c = reg_coeff(S.b / T.DEL);
    }
  }
  F.px = (float)(S.px - T.ctr[0]);
  F.py = (float)(S.py - T.ctr[1]);
  F.pz = (float)(S.pz - T.ctr[2]);
  // the direct sum of a far Stokeslet target has no subtraction (2S/KITC.cpp:856-882),
  // nor has the plain stresslet of a far target (2S/KITC.cpp:970-995)
  F.f0n0 = (KIND == K_SL_OFF && !S.near) ? 0.0f : (float)S.f0n0;
  const bool no_g0 = KIND == K_DL_OFF && !S.near;
  for (int k = 0; k < 3; k++) {
    F.g0[k] = no_g0 ? 0.0f : (float)S.g0[k];
    F.n0xf0[k] = (float)S.n0xf0[k];
    F.x0[k] = (float)(S.x0[k] - T.ctr[k]);
    F.n0[k] = (float)S.n0[k];
  }
  F.b = (float)S.b;
  F.c.c1 = (float)S.c.c1;
  F.c.c2 = (float)S.c.c2;
  F.c.c3 = (float)S.c.c3;
}

// ---------------------------------------------------------------- FP64 pairs

// One FP64 pair; returns true if the smoothed (erf) branch was taken.
template <int KIND>
__device__ __forceinline__ bool pair64(const double* __restrict__ sm, int j, const Tgt& S,
                                       const Reg& g, const double* __restrict__ stab, double& a0,
                                       double& a1, double& a2) {
  const double* X = sm;
  const double* Y = sm + kNT;
  const double* Z = sm + 2 * kNT;
  const double* NX = sm + 3 * kNT;
  const double* NY = sm + 4 * kNT;
  const double* NZ = sm + 5 * kNT;
  const double* A = sm + 6 * kNT;
  const double* QX = sm + 7 * kNT;
  const double* QY = sm + 8 * kNT;
  const double* QZ = sm + 9 * kNT;
  const double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
  const double r2 = dx * dx + dy * dy + dz * dz;
  constexpr bool kTab = (KIND == K_SL_ON || KIND == K_DL_ON);  // tabulated smoothing, rsqrt only if r > 8 delta
  const double rinv = kTab ? 0.0 : rsqrt(r2);
  bool reg = false;
  if (KIND == K_SL_ON) {
    // Call_Ds_SL_onSurf (2S/KITC.cpp:807-846) with Stokes_SL_7ord_onSurf (2S/utilities.cpp:211)
    const double area = A[j];
    const double fx = QX[j] - S.f0n0 * NX[j];
    const double fy = QY[j] - S.f0n0 * NY[j];
    const double fz = QZ[j] - S.f0n0 * NZ[j];
    const double fdd = fx * dx + fy * dy + fz * dz;
    double H1, H2;
    if (r2 > g.d64) {
      const double ri = rsqrt(r2);
      H1 = ri;
      H2 = ri * ri * ri;
    } else {
      const double sq = r2 * g.inv_d2;
      H1 = smooth_eval(stab, sq) * g.inv_d;
      H2 = smooth_eval(stab + kSmoothN, sq) * g.inv_d3;
      reg = r2 >= g.r0sq;
    }
    H1 *= area;
    H2 *= area * fdd;
    a0 += fx * H1 + dx * H2;
    a1 += fy * H1 + dy * H2;
    a2 += fz * H1 + dz * H2;
  } else if ((KIND == K_SL_OFF || KIND == K_E2G_SL7) && S.near) {
    // Call_Ds_SL regularized branch (2S/KITC.cpp:847) / stokes_SL_7ord (E2G/stokes.cpp:53)
    const double area = A[j];
    const double fx = QX[j] - S.f0n0 * NX[j];
    const double fy = QY[j] - S.f0n0 * NY[j];
    const double fz = QZ[j] - S.f0n0 * NZ[j];
    const double fdd = fx * dx + fy * dy + fz * dz;
    double H1, H2;
    reg = sl_7ord(r2, rinv, g, S.c, H1, H2);
    H1 *= area;
    H2 *= area * fdd;
    a0 += fx * H1 + dx * H2;
    a1 += fy * H1 + dy * H2;
    a2 += fz * H1 + dz * H2;
  } else if (KIND == K_SL_OFF || KIND == K_E2G_SL_AWAY) {
    // plain Stokeslet without subtraction (2S/KITC.cpp:856-882, E2G/stokes.cpp:22-40)
    const double fx = QX[j], fy = QY[j], fz = QZ[j];
    const double fdd = fx * dx + fy * dy + fz * dz;
    const double H1 = A[j] * rinv;
    const double H2 = fdd * H1 * (rinv * rinv);
    a0 += fx * H1 + dx * H2;
    a1 += fy * H1 + dy * H2;
    a2 += fz * H1 + dz * H2;
  } else if (KIND == K_DL_ON) {
    // Call_Ds_DL_onSurf (2S/KITC.cpp:921-957)
    const double gx = QX[j] - S.g0[0];
    const double gy = QY[j] - S.g0[1];
    const double gz = QZ[j] - S.g0[2];
    const double gdd = gx * dx + gy * dy + gz * dz;
    const double ndd = NX[j] * dx + NY[j] * dy + NZ[j] * dz;
    double H3;
    if (r2 > g.d64) {
      const double ri = rsqrt(r2), ri2 = ri * ri;
      H3 = ri2 * ri2 * ri;
    } else {
      H3 = smooth_eval(stab, r2 * g.inv_d2) * g.inv_d5;
      reg = r2 >= g.r0sq;
    }
    const double kernel = ndd * gdd * H3 * A[j];
    a0 += dx * kernel;
    a1 += dy * kernel;
    a2 += dz * kernel;
  } else if (KIND == K_DL_OFF) {
    if (S.near) {
      // Call_Ds_DL regularized branch (2S/KITC.cpp:996-1059), stokes_DL_7ord
      const double b = S.b;
      const double xh0 = X[j] - S.x0[0];
      const double xh1 = Y[j] - S.x0[1];
      const double xh2 = Z[j] - S.x0[2];
      const double gx = QX[j] - S.g0[0];
      const double gy = QY[j] - S.g0[1];
      const double gz = QZ[j] - S.g0[2];
      const double sig_sq = (xh0 * xh0 + xh1 * xh1 + xh2 * xh2) -
                            2.0 * b * (xh0 * S.n0[0] + xh1 * S.n0[1] + xh2 * S.n0[2]);
      const double g_dot_n0 = gx * S.n0[0] + gy * S.n0[1] + gz * S.n0[2];
      const double g_dot_xh = gx * xh0 + gy * xh1 + gz * xh2;
      const double n0_dot_n = S.n0[0] * NX[j] + S.n0[1] * NY[j] + S.n0[2] * NZ[j];
      const double xh_dot_n = xh0 * NX[j] + xh1 * NY[j] + xh2 * NZ[j];
      const double c_m1a = g_dot_n0 * n0_dot_n;
      const double c_m1b = g_dot_xh * n0_dot_n + g_dot_n0 * xh_dot_n;
      const double c_m2a = g_dot_xh * xh_dot_n;
      const double c_m2b = b * c_m1b;
      double H2, H3;
      reg = dl_7ord(r2, rinv, g, S.c, H2, H3);
      const double area = A[j];
      H2 *= area;
      H3 *= area;
      double m1 = dx * c_m1a - S.n0[0] * c_m1b;
      double m2 = -sig_sq * m1 + dx * c_m2a + xh0 * c_m2b;
      a0 += m1 * H2 + m2 * H3;
      m1 = dy * c_m1a - S.n0[1] * c_m1b;
      m2 = -sig_sq * m1 + dy * c_m2a + xh1 * c_m2b;
      a1 += m1 * H2 + m2 * H3;
      m1 = dz * c_m1a - S.n0[2] * c_m1b;
      m2 = -sig_sq * m1 + dz * c_m2a + xh2 * c_m2b;
      a2 += m1 * H2 + m2 * H3;
    } else {
      // plain stresslet (2S/KITC.cpp:970-995)
      const double gdd = QX[j] * dx + QY[j] * dy + QZ[j] * dz;
      const double ndd = NX[j] * dx + NY[j] * dy + NZ[j] * dz;
      const double rinv2 = rinv * rinv;
      const double kernel = gdd * ndd * (rinv2 * rinv2 * rinv) * A[j];
      a0 += dx * kernel;
      a1 += dy * kernel;
      a2 += dz * kernel;
    }
  } else if (KIND == K_E2G_P_AWAY) {
    // stokes_pressure_away (E2G/stokes.cpp:108-121)
    const double H2 = (QX[j] * dx + QY[j] * dy + QZ[j] * dz) * (rinv * rinv * rinv);
    a0 += H2 * A[j];
  } else if (KIND == K_E2G_P7) {
    // stokes_pressure_7ord (E2G/stokes.cpp:151-194)
    double H2;
    reg = lapl_dl_7ord(r2, rinv, g, S.c, H2);
    const double n0 = NX[j], n1 = NY[j], n2 = NZ[j];
    const double f0 = QX[j], f1 = QY[j], f2 = QZ[j];
    const double f_dot_n = f0 * n0 + f1 * n1 + f2 * n2;
    const double ncf0 = (n1 * f2 - n2 * f1) - S.n0xf0[0];
    const double ncf1 = (n2 * f0 - n0 * f2) - S.n0xf0[1];
    const double ncf2 = (n0 * f1 - n1 * f0) - S.n0xf0[2];
    const double n_dot_dx = n0 * dx + n1 * dy + n2 * dz;
    const double ncd0 = n1 * dz - n2 * dy;
    const double ncd1 = n2 * dx - n0 * dz;
    const double ncd2 = n0 * dy - n1 * dx;
    const double normal = -(f_dot_n - S.f0n0) * n_dot_dx;
    const double tangential = -(ncf0 * ncd0 + ncf1 * ncd1 + ncf2 * ncd2);
    a0 += (normal + tangential) * H2 * A[j];
  }
  return reg;
}

// ------------------------------------------------------- FP32 plain pairs
// The singular kernel of each kind (the r/delta > 8 branch of the reference),
// from FP32 centre-relative coordinates.
template <int KIND>
__device__ __forceinline__ void pair32(const float* __restrict__ sf, int j, const Tgt32& F,
                                       float& p0, float& p1, float& p2) {
  const float* X = sf;
  const float* Y = sf + kNT;
  const float* Z = sf + 2 * kNT;
  const float* NX = sf + 3 * kNT;
  const float* NY = sf + 4 * kNT;
  const float* NZ = sf + 5 * kNT;
  const float* A = sf + 6 * kNT;
  const float* QX = sf + 7 * kNT;
  const float* QY = sf + 8 * kNT;
  const float* QZ = sf + 9 * kNT;
  const float dx = F.px - X[j], dy = F.py - Y[j], dz = F.pz - Z[j];
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float rinv = rsqrtf(r2);
  const float rinv2 = rinv * rinv;
  if (KIND == K_E2G_SL_AWAY) {
    // plain Stokeslet, no subtraction; the face sums stage no normals
    const float fx = QX[j], fy = QY[j], fz = QZ[j];
    const float fdd = fx * dx + fy * dy + fz * dz;
    const float H1 = A[j] * rinv;
    const float H2 = fdd * H1 * rinv2;
    p0 += fx * H1 + dx * H2;
    p1 += fy * H1 + dy * H2;
    p2 += fz * H1 + dz * H2;
  } else if (KIND == K_SL_ON || KIND == K_SL_OFF || KIND == K_E2G_SL7) {
    const float fx = QX[j] - F.f0n0 * NX[j];
    const float fy = QY[j] - F.f0n0 * NY[j];
    const float fz = QZ[j] - F.f0n0 * NZ[j];
    const float fdd = fx * dx + fy * dy + fz * dz;
    const float H1 = A[j] * rinv;
    const float H2 = fdd * H1 * rinv2;
    p0 += fx * H1 + dx * H2;
    p1 += fy * H1 + dy * H2;
    p2 += fz * H1 + dz * H2;
  } else if (KIND == K_DL_ON || KIND == K_DL_OFF) {
    const float gx = QX[j] - F.g0[0];
    const float gy = QY[j] - F.g0[1];
    const float gz = QZ[j] - F.g0[2];
    const float gdd = gx * dx + gy * dy + gz * dz;
    const float ndd = NX[j] * dx + NY[j] * dy + NZ[j] * dz;
    const float kernel = ndd * gdd * (rinv2 * rinv2 * rinv) * A[j];
    p0 += dx * kernel;
    p1 += dy * kernel;
    p2 += dz * kernel;
  } else if (KIND == K_E2G_P_AWAY) {
    p0 += (QX[j] * dx + QY[j] * dy + QZ[j] * dz) * (rinv2 * rinv) * A[j];
  } else if (KIND == K_E2G_P7) {
    const float n0 = NX[j], n1 = NY[j], n2 = NZ[j];
    const float f0 = QX[j], f1 = QY[j], f2 = QZ[j];
    const float f_dot_n = f0 * n0 + f1 * n1 + f2 * n2;
    const float ncf0 = (n1 * f2 - n2 * f1) - F.n0xf0[0];
    const float ncf1 = (n2 * f0 - n0 * f2) - F.n0xf0[1];
    const float ncf2 = (n0 * f1 - n1 * f0) - F.n0xf0[2];
    const float n_dot_dx = n0 * dx + n1 * dy + n2 * dz;
    const float ncd0 = n1 * dz - n2 * dy;
    const float ncd1 = n2 * dx - n0 * dz;
    const float ncd2 = n0 * dy - n1 * dx;
    const float normal = -(f_dot_n - F.f0n0) * n_dot_dx;
    const float tangential = -(ncf0 * ncd0 + ncf1 * ncd1 + ncf2 * ncd2);
    p0 += (normal + tangential) * (rinv2 * rinv) * A[j];
  }
}

// ------------------------------------------------ FP32 pairs, r > 3 delta
// The full kernel of a target that uses the regularized forms (the smoothed
// branch for r <= 8 delta, the singular one beyond, with the target's
// subtraction), in FP32 for pairs with r > 3 delta. Returns true if the
// smoothed branch was taken.
template <int KIND>
__device__ __forceinline__ bool pair32r(const float* __restrict__ sf, int j, const Tgt32& F, const RegF& gf,
                                        float& p0, float& p1, float& p2) {
  const float* X = sf;
  const float* Y = sf + kNT;
  const float* Z = sf + 2 * kNT;
  const float* NX = sf + 3 * kNT;
  const float* NY = sf + 4 * kNT;
  const float* NZ = sf + 5 * kNT;
  const float* A = sf + 6 * kNT;
  const float* QX = sf + 7 * kNT;
  const float* QY = sf + 8 * kNT;
  const float* QZ = sf + 9 * kNT;
  const float dx = F.px - X[j], dy = F.py - Y[j], dz = F.pz - Z[j];
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float rinv = rsqrtf(r2);
  const bool reg = r2 <= gf.d64;
  if (KIND == K_SL_ON || KIND == K_SL_OFF || KIND == K_E2G_SL7) {
    const float fx = QX[j] - F.f0n0 * NX[j];
    const float fy = QY[j] - F.f0n0 * NY[j];
    const float fz = QZ[j] - F.f0n0 * NZ[j];
    const float fdd = fx * dx + fy * dy + fz * dz;
    float H1, H2;
    if (KIND == K_SL_ON) sl_7ord_onsurf_f(r2, rinv, gf, H1, H2);
    else sl_7ord_f(r2, rinv, gf, F.c, H1, H2);
    H1 *= A[j];
    H2 *= A[j] * fdd;
    p0 += fx * H1 + dx * H2;
    p1 += fy * H1 + dy * H2;
    p2 += fz * H1 + dz * H2;
  } else if (KIND == K_DL_ON) {
    const float gx = QX[j] - F.g0[0];
    const float gy = QY[j] - F.g0[1];
    const float gz = QZ[j] - F.g0[2];
    const float gdd = gx * dx + gy * dy + gz * dz;
    const float ndd = NX[j] * dx + NY[j] * dy + NZ[j] * dz;
    float H3;
    dl_7ord_onsurf_f(r2, rinv, gf, H3);
    const float kernel = ndd * gdd * H3 * A[j];
    p0 += dx * kernel;
    p1 += dy * kernel;
    p2 += dz * kernel;
  } else if (KIND == K_DL_OFF) {
    // the subtraction form of a near target (2S/KITC.cpp:996-1059)
    const float b = F.b;
    const float xh0 = X[j] - F.x0[0], xh1 = Y[j] - F.x0[1], xh2 = Z[j] - F.x0[2];
    const float gx = QX[j] - F.g0[0], gy = QY[j] - F.g0[1], gz = QZ[j] - F.g0[2];
    const float sig_sq = (xh0 * xh0 + xh1 * xh1 + xh2 * xh2) - 2.0f * b * (xh0 * F.n0[0] + xh1 * F.n0[1] + xh2 * F.n0[2]);
    const float g_dot_n0 = gx * F.n0[0] + gy * F.n0[1] + gz * F.n0[2];
    const float g_dot_xh = gx * xh0 + gy * xh1 + gz * xh2;
    const float n0_dot_n = F.n0[0] * NX[j] + F.n0[1] * NY[j] + F.n0[2] * NZ[j];
    const float xh_dot_n = xh0 * NX[j] + xh1 * NY[j] + xh2 * NZ[j];
    const float c_m1a = g_dot_n0 * n0_dot_n;
    const float c_m1b = g_dot_xh * n0_dot_n + g_dot_n0 * xh_dot_n;
    const float c_m2a = g_dot_xh * xh_dot_n;
    const float c_m2b = b * c_m1b;
    float H2, H3;
    dl_7ord_f(r2, rinv, gf, F.c, H2, H3);
    H2 *= A[j];
    H3 *= A[j];
    float m1 = dx * c_m1a - F.n0[0] * c_m1b;
    float m2 = -sig_sq * m1 + dx * c_m2a + xh0 * c_m2b;
    p0 += m1 * H2 + m2 * H3;
    m1 = dy * c_m1a - F.n0[1] * c_m1b;
    m2 = -sig_sq * m1 + dy * c_m2a + xh1 * c_m2b;
    p1 += m1 * H2 + m2 * H3;
    m1 = dz * c_m1a - F.n0[2] * c_m1b;
    m2 = -sig_sq * m1 + dz * c_m2a + xh2 * c_m2b;
    p2 += m1 * H2 + m2 * H3;
  } else if (KIND == K_E2G_P7) {
    float H2;
    lapl_dl_7ord_f(r2, rinv, gf, F.c, H2);
    const float n0 = NX[j], n1 = NY[j], n2 = NZ[j];
    const float f0 = QX[j], f1 = QY[j], f2 = QZ[j];
    const float f_dot_n = f0 * n0 + f1 * n1 + f2 * n2;
    const float ncf0 = (n1 * f2 - n2 * f1) - F.n0xf0[0];
    const float ncf1 = (n2 * f0 - n0 * f2) - F.n0xf0[1];
    const float ncf2 = (n0 * f1 - n1 * f0) - F.n0xf0[2];
    const float n_dot_dx = n0 * dx + n1 * dy + n2 * dz;
    const float ncd0 = n1 * dz - n2 * dy;
    const float ncd1 = n2 * dx - n0 * dz;
    const float ncd2 = n0 * dy - n1 * dx;
    const float normal = -(f_dot_n - F.f0n0) * n_dot_dx;
    const float tangential = -(ncf0 * ncd0 + ncf1 * ncd1 + ncf2 * ncd2);
    p0 += (normal + tangential) * H2 * A[j];
  }
  return reg;
}

// ------------------------------------------------------------ proxy tiles

template <bool DL>
__device__ __forceinline__ void proxies64(const double* __restrict__ sm, int PT, int cnt, int kk0,
                                          int P1, const double* __restrict__ cheb, const Tgt& S,
                                          double& a0, double& a1, double& a2) {
  int rem = kk0 % (P1 * P1);
  int pi = kk0 / (P1 * P1), pj = rem / P1, pk = rem % P1;
  for (int i = 0; i < cnt; i++) {
    const double dx0 = S.px - cheb[pi];
    const double dx1 = S.py - cheb[P1 + pj];
    const double dx2 = S.pz - cheb[2 * P1 + pk];
    const double r2 = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
    const double rinv = rsqrt(r2);
    const double rinv2 = rinv * rinv;
    if (!DL) {
      // Call_Treecode_SL (2S/KITC.cpp:700-714)
      const double m0 = sm[i] - S.f0n0 * sm[3 * PT + i];
      const double m1 = sm[PT + i] - S.f0n0 * sm[4 * PT + i];
      const double m2 = sm[2 * PT + i] - S.f0n0 * sm[5 * PT + i];
      const double temp = (m0 * dx0 + m1 * dx1 + m2 * dx2) * (rinv2 * rinv);
      a0 += m0 * rinv + temp * dx0;
      a1 += m1 * rinv + temp * dx1;
      a2 += m2 * rinv + temp * dx2;
    } else {
      // Call_Treecode_DL (2S/KITC.cpp:753-771)
      const double M9 = sm[9 * PT + i], M10 = sm[10 * PT + i], M11 = sm[11 * PT + i];
      double tl[3];
#pragma unroll
      for (int l = 0; l < 3; l++) {
        const double ta = sm[(3 * l) * PT + i] - S.g0[l] * M9;
        const double tb = sm[(3 * l + 1) * PT + i] - S.g0[l] * M10;
        const double tc = sm[(3 * l + 2) * PT + i] - S.g0[l] * M11;
        tl[l] = ta * dx0 + tb * dx1 + tc * dx2;
      }
      const double kernel = (tl[0] * dx0 + tl[1] * dx1 + tl[2] * dx2) * (rinv2 * rinv2 * rinv);
      a0 += dx0 * kernel;
      a1 += dx1 * kernel;
      a2 += dx2 * kernel;
    }
    if (++pk == P1) {
      pk = 0;
      if (++pj == P1) {
        pj = 0;
        ++pi;
      }
    }
  }
}

template <bool DL>
__device__ __forceinline__ void proxies32(const float* __restrict__ sf, int PT, int cnt, int kk0,
                                          int P1, const float* __restrict__ chebf, const Tgt32& F,
                                          float& p0, float& p1, float& p2) {
  int rem = kk0 % (P1 * P1);
  int pi = kk0 / (P1 * P1), pj = rem / P1, pk = rem % P1;
  for (int i = 0; i < cnt; i++) {
    const float dx0 = F.px - chebf[pi];
    const float dx1 = F.py - chebf[P1 + pj];
    const float dx2 = F.pz - chebf[2 * P1 + pk];
    const float r2 = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
    const float rinv = rsqrtf(r2);
    const float rinv2 = rinv * rinv;
    if (!DL) {
      const float m0 = sf[i] - F.f0n0 * sf[3 * PT + i];
      const float m1 = sf[PT + i] - F.f0n0 * sf[4 * PT + i];
      const float m2 = sf[2 * PT + i] - F.f0n0 * sf[5 * PT + i];
      const float temp = (m0 * dx0 + m1 * dx1 + m2 * dx2) * (rinv2 * rinv);
      p0 += m0 * rinv + temp * dx0;
      p1 += m1 * rinv + temp * dx1;
      p2 += m2 * rinv + temp * dx2;
    } else {
      const float M9 = sf[9 * PT + i], M10 = sf[10 * PT + i], M11 = sf[11 * PT + i];
      float tl[3];
#pragma unroll
      for (int l = 0; l < 3; l++) {
        const float ta = sf[(3 * l) * PT + i] - F.g0[l] * M9;
        const float tb = sf[(3 * l + 1) * PT + i] - F.g0[l] * M10;
        const float tc = sf[(3 * l + 2) * PT + i] - F.g0[l] * M11;
        tl[l] = ta * dx0 + tb * dx1 + tc * dx2;
      }
      const float kernel = (tl[0] * dx0 + tl[1] * dx1 + tl[2] * dx2) * (rinv2 * rinv2 * rinv);
      p0 += dx0 * kernel;
      p1 += dx1 * kernel;
      p2 += dx2 * kernel;
    }
    if (++pk == P1) {
      pk = 0;
      if (++pj == P1) {
        pj = 0;
        ++pi;
      }
    }
  }
}

template <int KIND, bool MIXED>
__device__ __forceinline__ void run_item(const EvalTask& T, const BlockRef& it,
                                         const Seg* __restrict__ segs, double* sm, float* sf,
                                         double* cheb, float* chebf, const double* stab) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int blk = it.blk;
  const int k = blk * kTB + tid;
  const bool valid = k < T.nt;
  const int t = valid ? T.tord[k] : 0;
  Tgt S;
  Tgt32 F;
  load_target<KIND>(T, t, valid, S, F);
  const Reg g = make_reg(T.DEL);
  RegF gf;
  gf.inv_d = (float)g.inv_d;
  gf.d64 = (float)g.d64;
  // FP64 below, FP32 above: (3 delta)^2 in the mixed mode; in the all-FP32 mode
  // only the r < 1e-14 limits of the reference stay in FP64
  const float cut2f = T.mixed == 2 ? 1e-28f : (float)(9.0 * T.DEL * T.DEL);
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  unsigned long long creg = 0, cplain = 0, cfar = 0, cprox = 0;
  constexpr bool kSrcNrm = !(KIND == K_E2G_SL_AWAY || KIND == K_E2G_P_AWAY);
  // which path a target takes through a source tile
  constexpr bool kPerPairSplit = (KIND == K_SL_ON || KIND == K_DL_ON || KIND == K_SL_OFF || KIND == K_DL_OFF ||
                                   KIND == K_E2G_SL7 || KIND == K_E2G_P7);
  const bool all32 = MIXED && (KIND == K_E2G_SL_AWAY || KIND == K_E2G_P_AWAY ||
                               ((KIND == K_SL_OFF || KIND == K_DL_OFF) && !S.near));
  for (int q = it.seg0; q < it.seg1; q++) {
    const Seg sg = segs[q];
    const Entry E = T.entries[sg.entry];
    const uint32_t wm = E.mask[warp];
    const bool act = valid && ((wm >> lane) & 1u);
    if (E.type == 1) {
      const int m0 = sg.s0, m1 = sg.s1 - 1;
      for (int s0 = m0; s0 <= m1; s0 += kNT) {
        const int cnt = min(kNT, m1 - s0 + 1);
        __syncthreads();
        for (int i = tid; i < cnt; i += kTB) {
          const int s = s0 + i;
          sm[i] = T.sx[s];
          sm[kNT + i] = T.sy[s];
          sm[2 * kNT + i] = T.sz[s];
          if (kSrcNrm) {
            sm[3 * kNT + i] = T.snx[s];
            sm[4 * kNT + i] = T.sny[s];
            sm[5 * kNT + i] = T.snz[s];
          }
          sm[6 * kNT + i] = T.sa[s];
          sm[7 * kNT + i] = T.qx[s];
          sm[8 * kNT + i] = T.qy[s];
          sm[9 * kNT + i] = T.qz[s];
          if (MIXED) {
            sf[i] = T.fx[s];
            sf[kNT + i] = T.fy[s];
            sf[2 * kNT + i] = T.fz[s];
            if (kSrcNrm) {
              sf[3 * kNT + i] = T.fnx[s];
              sf[4 * kNT + i] = T.fny[s];
              sf[5 * kNT + i] = T.fnz[s];
            }
            sf[6 * kNT + i] = T.fa[s];
            sf[7 * kNT + i] = T.fqx[s];
            sf[8 * kNT + i] = T.fqy[s];
            sf[9 * kNT + i] = T.fqz[s];
          }
        }
        __syncthreads();
        if (wm != 0u && act) {
          if (all32) {
            for (int j0 = 0; j0 < cnt; j0 += 16) {
              float p0 = 0.f, p1 = 0.f, p2 = 0.f;
              const int j1 = min(cnt, j0 + 16);
              for (int j = j0; j < j1; j++) pair32<KIND>(sf, j, F, p0, p1, p2);
              a0 += (double)p0;
              a1 += (double)p1;
              a2 += (double)p2;
            }
            if (S.near) cplain += cnt;
            else cfar += cnt;
          } else if (MIXED && kPerPairSplit && S.near) {
            unsigned cr = 0;
            for (int j0 = 0; j0 < cnt; j0 += 16) {
              float p0 = 0.f, p1 = 0.f, p2 = 0.f;
              const int j1 = min(cnt, j0 + 16);
              for (int j = j0; j < j1; j++) {
                const float dx = F.px - sf[j], dy = F.py - sf[kNT + j], dz = F.pz - sf[2 * kNT + j];
                if (dx * dx + dy * dy + dz * dz > cut2f) cr += pair32r<KIND>(sf, j, F, gf, p0, p1, p2);
                else cr += pair64<KIND>(sm, j, S, g, stab, a0, a1, a2);
              }
              a0 += (double)p0;
              a1 += (double)p1;
              a2 += (double)p2;
            }
            creg += cr;
            cplain += cnt - cr;
          } else {
            unsigned cr = 0;
#pragma unroll 2
            for (int j = 0; j < cnt; j++) cr += pair64<KIND>(sm, j, S, g, stab, a0, a1, a2);
            if (S.near) {
              creg += cr;
              cplain += cnt - cr;
            } else {
              cfar += cnt;
            }
          }
        }
      }
    } else if (KIND == K_SL_ON || KIND == K_SL_OFF || KIND == K_DL_ON || KIND == K_DL_OFF) {
      constexpr bool DL = (KIND == K_DL_ON || KIND == K_DL_OFF);
      const int P1 = T.P1, Pf = T.Pf, C = T.C;
      const int PT = (kSmem / C) & ~31;
      __syncthreads();
      if (tid < 3 * P1) {
        const double v = T.tcheb[(size_t)E.node * 3 * P1 + tid];
        cheb[tid] = v;
        if (MIXED) chebf[tid] = (float)(v - T.ctr[tid / P1]);
      }
      const double* M = T.mom + (size_t)E.node * C * Pf;
      for (int kk0 = 0; kk0 < Pf; kk0 += PT) {
        const int cnt = min(PT, Pf - kk0);
        __syncthreads();
        for (int c = 0; c < C; c++)
          for (int i = tid; i < cnt; i += kTB) {
            const double v = M[(size_t)c * Pf + kk0 + i];
            if (MIXED) sf[c * PT + i] = (float)v;
            else sm[c * PT + i] = v;
          }
        __syncthreads();
        if (wm != 0u && act) {
          if (MIXED) {
            for (int i0 = 0; i0 < cnt; i0 += 16) {
              float p0 = 0.f, p1 = 0.f, p2 = 0.f;
              proxies32<DL>(sf + i0, PT, min(16, cnt - i0), kk0 + i0, P1, chebf, F, p0, p1, p2);
              a0 += (double)p0;
              a1 += (double)p1;
              a2 += (double)p2;
            }
          } else {
            proxies64<DL>(sm, PT, cnt, kk0, P1, cheb, S, a0, a1, a2);
          }
          cprox += cnt;
        }
      }
    }
  }
  // partial sums of this item
  double* o = T.partial + ((size_t)it.slot * kTB + tid) * 3;
  o[0] = a0;
  o[1] = a1;
  o[2] = a2;
  // Work counters (pair kinds actually evaluated), one atomic per warp.
  if (T.counters) {
    for (int off = 16; off > 0; off >>= 1) {
      creg += __shfl_down_sync(0xffffffffu, creg, off);
      cplain += __shfl_down_sync(0xffffffffu, cplain, off);
      cfar += __shfl_down_sync(0xffffffffu, cfar, off);
      cprox += __shfl_down_sync(0xffffffffu, cprox, off);
    }
    if (lane == 0) {
      if (creg) atomicAdd(&T.counters[0], creg);
      if (cplain) atomicAdd(&T.counters[1], cplain);
      if (cfar) atomicAdd(&T.counters[2], cfar);
      if (cprox) atomicAdd(&T.counters[3], cprox);
    }
  }
}

template <int FAM, bool MIXED>
__global__ void __launch_bounds__(kTB, 4) eval_kernel(const EvalTask* __restrict__ tasks,
                                                      const BlockRef* __restrict__ items,
                                                      const Seg* __restrict__ segs) {
  __shared__ double sm[kSmem];
  __shared__ float sf[MIXED ? kSmem : 1];
  __shared__ double cheb[3 * kMaxP1];
  __shared__ float chebf[3 * kMaxP1];
  __shared__ EvalTask sT;
  // smoothing tables: G1, G2 for the Stokeslet family, G3 for the stresslet family
  __shared__ double stab[FAM == F_SL ? 2 * kSmoothN : (FAM == F_DL ? kSmoothN : 1)];
  const BlockRef it = items[blockIdx.x];
  if (threadIdx.x == 0) sT = tasks[it.task];
  if (FAM == F_SL) {
    for (int i = threadIdx.x; i < kSmoothN; i += blockDim.x) {
      stab[i] = kSmoothG1[i];
      stab[kSmoothN + i] = kSmoothG2[i];
    }
  } else if (FAM == F_DL) {
    for (int i = threadIdx.x; i < kSmoothN; i += blockDim.x) stab[i] = kSmoothG3[i];
  }
  __syncthreads();
  const int kind = sT.kind;
  if (FAM == F_SL) {
    if (kind == K_SL_ON) run_item<K_SL_ON, MIXED>(sT, it, segs, sm, sf, cheb, chebf, stab);
    else run_item<K_SL_OFF, MIXED>(sT, it, segs, sm, sf, cheb, chebf, stab);
  } else if (FAM == F_DL) {
    if (kind == K_DL_ON) run_item<K_DL_ON, MIXED>(sT, it, segs, sm, sf, cheb, chebf, stab);
    else run_item<K_DL_OFF, MIXED>(sT, it, segs, sm, sf, cheb, chebf, stab);
  } else {
    switch (kind) {
      case K_E2G_SL_AWAY: run_item<K_E2G_SL_AWAY, MIXED>(sT, it, segs, sm, sf, cheb, chebf, stab); break;
      case K_E2G_P_AWAY: run_item<K_E2G_P_AWAY, MIXED>(sT, it, segs, sm, sf, cheb, chebf, stab); break;
      case K_E2G_SL7: run_item<K_E2G_SL7, MIXED>(sT, it, segs, sm, sf, cheb, chebf, stab); break;
      default: run_item<K_E2G_P7, MIXED>(sT, it, segs, sm, sf, cheb, chebf, stab); break;
    }
  }
}

// Sums a target block's item partials in slot order and applies the
// reference drivers' per-target epilogue (scale and jump terms).
__global__ void __launch_bounds__(kTB) reduce_kernel(const EvalTask* __restrict__ tasks,
                                                     const int2* __restrict__ task_blocks) {
  const int2 tb = task_blocks[blockIdx.x];  // (task, block)
  const EvalTask& T = tasks[tb.x];
  const int blk = tb.y, tid = threadIdx.x;
  const int k = blk * kTB + tid;
  if (k >= T.nt) return;
  const int t = T.tord[k];
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  const int s0 = T.item_start[blk], s1 = T.item_start[blk + 1];
  for (int s = s0; s < s1; s++) {
    const double* p = T.partial + ((size_t)s * kTB + tid) * 3;
    a0 += p[0];
    a1 += p[1];
    a2 += p[2];
  }
  const double sc = T.scale;
  double* o = T.out;
  const int kind = T.kind;
  if (kind == K_SL_ON || kind == K_SL_OFF || kind == K_E2G_SL_AWAY || kind == K_E2G_SL7) {
    o[3 * t] = a0 * sc;
    o[3 * t + 1] = a1 * sc;
    o[3 * t + 2] = a2 * sc;
  } else if (kind == K_DL_ON) {
    // DL[3i+k] = u[k] * EightPI6 + 0.5 * g0[k]   (2S/KITC.cpp:1693, 2S/stresslets.cpp:271-278)
    const double* g0 = T.tq + 3 * t;
    o[3 * t] = a0 * sc + 0.5 * g0[0];
    o[3 * t + 1] = a1 * sc + 0.5 * g0[1];
    o[3 * t + 2] = a2 * sc + 0.5 * g0[2];
  } else if (kind == K_DL_OFF) {
    const double b = T.tb[t];
    const double* g0 = T.tg0 + 3 * t;
    double xi = 0.0;
    if (T.jump_mode == 0) {
      // tree: xi = 1/2 on the surface, 1 inside (2S/KITC.cpp:1805-1815)
      if (fabs(b) < 1.0e-12) xi = 0.5;
      else if (b < 0.0) xi = 1.0;
    } else {
      // direct: + g0 inside or on the surface, near targets only (2S/stresslets.cpp:174-178)
      if (T.tnear[t] && ((b < 0.0) || (fabs(b) < 1.0e-14))) xi = 1.0;
    }
    o[3 * t] = a0 * sc + xi * g0[0];
    o[3 * t + 1] = a1 * sc + xi * g0[1];
    o[3 * t + 2] = a2 * sc + xi * g0[2];
  } else if (kind == K_E2G_P_AWAY) {
    o[t] = a0 * sc;
  } else {
    // p *= -denom_FourPI; inside: p -= f0.n0 (E2G/stokes.cpp:196-200)
    double p = a0 * sc;
    if (T.tb[t] < -1.e-12) {
      const double* f0 = T.tf0 + 3 * t;
      const double* n0 = T.tn0 + 3 * t;
      p -= f0[0] * n0[0] + f0[1] * n0[1] + f0[2] * n0[2];
    }
    o[t] = p;
  }
}

}  // namespace

void launch_eval(int family, const EvalTask* d_tasks, const BlockRef* d_items, const Seg* d_segs,
                 int nitems, int ntask_blocks, const int2* d_task_blocks, cudaStream_t st,
                 bool mixed) {
  if (nitems > 0) {
    if (!mixed) {
      if (family == F_SL) eval_kernel<F_SL, false><<<nitems, kTB, 0, st>>>(d_tasks, d_items, d_segs);
      else if (family == F_DL) eval_kernel<F_DL, false><<<nitems, kTB, 0, st>>>(d_tasks, d_items, d_segs);
      else eval_kernel<F_E2G, false><<<nitems, kTB, 0, st>>>(d_tasks, d_items, d_segs);
    } else {
      if (family == F_SL) eval_kernel<F_SL, true><<<nitems, kTB, 0, st>>>(d_tasks, d_items, d_segs);
      else if (family == F_DL) eval_kernel<F_DL, true><<<nitems, kTB, 0, st>>>(d_tasks, d_items, d_segs);
      else eval_kernel<F_E2G, true><<<nitems, kTB, 0, st>>>(d_tasks, d_items, d_segs);
    }
  }
  if (ntask_blocks > 0) reduce_kernel<<<ntask_blocks, kTB, 0, st>>>(d_tasks, d_task_blocks);
}

}  // namespace hr
