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
// Precision. FP64: every pair in FP64. MIXED: FP32 pairs from FP32
// coordinates relative to the target block's first target, summed per 16
// terms in FP32 and added to the FP64 per-target accumulators:
//   * on-surface kinds: every pair, the smoothing factors from FP32
//     piecewise polynomials in s = r^2/delta^2 (no erf / exp, and no
//     cancellation at any r);
//   * off-surface kinds: pairs with r > 3 delta (the plain kernels of far
//     targets, the regularized kernels with erff / expf, the subtraction
//     forms) in FP32; pairs with r <= 3 delta, where the erf / exp brackets
//     with the target's coefficients cancel, in FP64;
//   * all proxy interactions in FP32.
// FP32 (all pairs): as MIXED with every off-surface pair in FP32 too.
#include <cstdio>

#include "hr_device.h"
#include "hr_pairs.cuh"

namespace hr {

namespace {

#define HR_SMOOTH_STORAGE __device__ const
#include "hr_smoothing_tables.inc"

// On-surface smoothing factors without erf / exp / rsqrt: for r <= 8 delta,
// s1 = G1(s) / delta, s2 = G2(s) / delta^3, s3 = G3(s) / delta^5 with
// s = r^2 / delta^2, each G a piecewise polynomial fitted in 80-digit
// arithmetic to the reference's formulas (2S/utilities.cpp:211-254,
// :292-323) with ~1e-16 relative error; G(0) is the reference's r -> 0 value.
// Piece i of a table is centred at s = i w (w = 64 / NI; G1, G2: NI = 64,
// degree 13; G3: NI = 256, degree 9), so the piece of s is
// round-to-nearest(s / w), formed with one fused multiply-add (adding
// 1.5 * 2^52 leaves the rounded integer in the low word), and t = s - i w
// follows from the same sum without a stored centre. The tables of a kernel
// family are staged in shared memory once per CTA, with the powers of
// 1/delta folded into the coefficients.
template <int NI, int DEG>
struct SmoothTab {
  static constexpr int kPieces = NI;
  static constexpr int kCoef = DEG + 1;  // coefficients per piece (even: whole double2s)
  static constexpr int kLen = (NI + 1) * kCoef;
  static_assert(kCoef % 2 == 0, "a piece must be whole double2s");
};
using TabG1 = SmoothTab<HR_SMOOTHS_G1_PIECES, HR_SMOOTHS_G1_DEG>;
using TabG2 = SmoothTab<HR_SMOOTHS_G2_PIECES, HR_SMOOTHS_G2_DEG>;
using TabG3 = SmoothTab<HR_SMOOTHS_G3_PIECES, HR_SMOOTHS_G3_DEG>;
static_assert(TabG1::kPieces == TabG2::kPieces && TabG1::kLen == TabG2::kLen, "G1 and G2 share their pieces");
static_assert((TabG1::kLen * 8) % 16 == 0, "the G2 table must start on a double2");

constexpr double kRoundMagic = 6755399441055744.0;  // 1.5 * 2^52

// Piece index and offset of s >= 0 (s <= 64) on the grid of NI pieces.
template <int NI>
__device__ __forceinline__ int smooth_piece(double s, double& t) {
  const double f = fma(s, NI / 64.0, kRoundMagic);  // kRoundMagic + round(s NI / 64), exact
  t = fma(kRoundMagic - f, 64.0 / NI, s);           // s - i w
  return min(__double2loint(f), NI);
}

template <class TAB>
__device__ __forceinline__ double smooth_horner(const double* __restrict__ tab, int i, double t) {
  const double2* p2 = reinterpret_cast<const double2*>(tab + i * TAB::kCoef);
  double e[TAB::kCoef];
#pragma unroll
  for (int k = 0; k < TAB::kCoef / 2; k++) {
    const double2 v = p2[k];
    e[2 * k] = v.x;
    e[2 * k + 1] = v.y;
  }
  double v = e[TAB::kCoef - 1];
#pragma unroll
  for (int k = TAB::kCoef - 2; k >= 0; k--) v = fma(v, t, e[k]);
  return v;
}

constexpr int kSmooth32N = HR_SMOOTH32_PIECES * 8;  // floats per FP32 table

// FP32 piece: (centre, c0, c1, c2) (c3, c4, c5, 0); index floor(s * pieces / 64)
// for 0 <= s <= 64, formed on the FMA / ALU pipes: adding 1.5 * 2^23 to
// s * pieces / 64 - 1/2 leaves round-to-nearest of it, i.e. the floor (a tie
// picks the lower piece, whose polynomial covers its right end), in the low
// mantissa bits.
__device__ __forceinline__ float smooth_eval_f(const float4* __restrict__ tab, float s) {
  const float f = fmaf(s, HR_SMOOTH32_PIECES / 64.0f, -0.5f) + 12582912.0f;
  const int i = min(__float_as_int(f) - 0x4B400000, HR_SMOOTH32_PIECES - 1);
  const float4 a = tab[2 * i], b = tab[2 * i + 1];
  const float t = s - a.x;
  return fmaf(fmaf(fmaf(fmaf(fmaf(b.z, t, b.y), t, b.x), t, a.w), t, a.z), t, a.y);
}

constexpr int kWarps = kTB / 32;     // warps per CTA, each with its own tiles
constexpr int kNT = 64;              // sources per (per-warp) shared-memory tile
constexpr int kWarpSm = 10 * kNT;    // doubles per warp: a source tile, 10 values per source
constexpr int kSmem = kWarps * kWarpSm;
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
  float px, py, pz;  // relative to the FP32 origin of the target block
  float f0n0;        // 0 for targets without subtraction
  float g0[3];
  float n0xf0[3];
  float b;
  float x0[3];       // relative to the FP32 origin of the target block
  float n0[3];
  CoefF c;
};

template <int KIND>
__device__ __forceinline__ void load_target(const EvalTask& T, int t, bool valid, const double* cb, Tgt& S,
                                            Tgt32& F) {
  S.px = S.py = S.pz = 0.0;
  S.b = 0.0;
  S.f0n0 = 0.0;
  for (int k = 0; k < 3; k++) S.x0[k] = S.n0[k] = S.g0[k] = S.n0xf0[k] = 0.0;
  S.c.c1 = S.c.c2 = S.c.c3 = 0.0;
  // regularized-kernel kinds: on-surface sums and the E2G band sums
  S.near = (KIND == K_SL_ON || KIND == K_DL_ON || KIND == K_E2G_SL7 || KIND == K_E2G_P7 || KIND == K_E2G_UP7) ? 1 : 0;
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
    } else if (KIND == K_E2G_P7 || KIND == K_E2G_UP7) {
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
  F.px = (float)(S.px - cb[0]);
  F.py = (float)(S.py - cb[1]);
  F.pz = (float)(S.pz - cb[2]);
  // the direct sum of a far Stokeslet target has no subtraction (2S/KITC.cpp:856-882),
  // nor has the plain stresslet of a far target (2S/KITC.cpp:970-995)
  F.f0n0 = (KIND == K_SL_OFF && !S.near) ? 0.0f : (float)S.f0n0;
  const bool no_g0 = KIND == K_DL_OFF && !S.near;
  for (int k = 0; k < 3; k++) {
    F.g0[k] = no_g0 ? 0.0f : (float)S.g0[k];
    F.n0xf0[k] = (float)S.n0xf0[k];
    F.x0[k] = (float)(S.x0[k] - cb[k]);
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
  // source j of the warp's tile: (x, y) (z, area) (nx, ny) (nz, qx) (qy, qz)
  const double2* s2 = reinterpret_cast<const double2*>(sm) + 5 * j;
  const double2 v0 = s2[0], v1 = s2[1], v2 = s2[2], v3 = s2[3], v4 = s2[4];
  const double Xj = v0.x, Yj = v0.y, Zj = v1.x, Aj = v1.y;
  const double NXj = v2.x, NYj = v2.y, NZj = v3.x, QXj = v3.y, QYj = v4.x, QZj = v4.y;
  const double dx = S.px - Xj, dy = S.py - Yj, dz = S.pz - Zj;
  const double r2 = dx * dx + dy * dy + dz * dz;
  constexpr bool kTab = (KIND == K_SL_ON || KIND == K_DL_ON);  // tabulated smoothing, rsqrt only if r > 8 delta
  const double rinv = kTab ? 0.0 : rsqrt(r2);
  bool reg = false;
  if (KIND == K_SL_ON) {
    // Call_Ds_SL_onSurf (2S/KITC.cpp:807-846) with Stokes_SL_7ord_onSurf (2S/utilities.cpp:211);
    // the tile holds area x density and area x normal for this kind, so f is area x (f - f0n0 n)
    const double fx = QXj - S.f0n0 * NXj;
    const double fy = QYj - S.f0n0 * NYj;
    const double fz = QZj - S.f0n0 * NZj;
    const double fdd = fx * dx + fy * dy + fz * dz;
    double H1, H2;
    if (r2 > g.dplain) {
      const double ri = rsqrt(r2);
      H1 = ri;
      H2 = ri * ri * ri;
    } else {
      double t;
      const int i = smooth_piece<TabG1::kPieces>(r2 * g.inv_d2, t);
      H1 = smooth_horner<TabG1>(stab, i, t);
      H2 = smooth_horner<TabG2>(stab + TabG1::kLen, i, t);
    }
    reg = r2 <= g.d64 && r2 >= g.r0sq;  // the reference's branch (work counters)
    H2 *= fdd;
    a0 += fx * H1 + dx * H2;
    a1 += fy * H1 + dy * H2;
    a2 += fz * H1 + dz * H2;
  } else if ((KIND == K_SL_OFF || KIND == K_E2G_SL7) && S.near) {
    // Call_Ds_SL regularized branch (2S/KITC.cpp:847) / stokes_SL_7ord (E2G/stokes.cpp:53)
    const double area = Aj;
    const double fx = QXj - S.f0n0 * NXj;
    const double fy = QYj - S.f0n0 * NYj;
    const double fz = QZj - S.f0n0 * NZj;
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
    const double fx = QXj, fy = QYj, fz = QZj;
    const double fdd = fx * dx + fy * dy + fz * dz;
    const double H1 = Aj * rinv;
    const double H2 = fdd * H1 * (rinv * rinv);
    a0 += fx * H1 + dx * H2;
    a1 += fy * H1 + dy * H2;
    a2 += fz * H1 + dz * H2;
  } else if (KIND == K_DL_ON) {
    // Call_Ds_DL_onSurf (2S/KITC.cpp:921-957); the tile holds area x normal for this kind
    const double gx = QXj - S.g0[0];
    const double gy = QYj - S.g0[1];
    const double gz = QZj - S.g0[2];
    const double gdd = gx * dx + gy * dy + gz * dz;
    const double ndd = NXj * dx + NYj * dy + NZj * dz;
    double H3;
    if (r2 > g.dplain) {
      const double ri = rsqrt(r2), ri2 = ri * ri;
      H3 = ri2 * ri2 * ri;
    } else {
      double t;
      const int i = smooth_piece<TabG3::kPieces>(r2 * g.inv_d2, t);
      H3 = smooth_horner<TabG3>(stab, i, t);
    }
    reg = r2 <= g.d64 && r2 >= g.r0sq;  // the reference's branch (work counters)
    const double kernel = ndd * gdd * H3;
    a0 += dx * kernel;
    a1 += dy * kernel;
    a2 += dz * kernel;
  } else if (KIND == K_DL_OFF) {
    if (S.near) {
      // Call_Ds_DL regularized branch (2S/KITC.cpp:996-1059), stokes_DL_7ord
      const double b = S.b;
      const double xh0 = Xj - S.x0[0];
      const double xh1 = Yj - S.x0[1];
      const double xh2 = Zj - S.x0[2];
      const double gx = QXj - S.g0[0];
      const double gy = QYj - S.g0[1];
      const double gz = QZj - S.g0[2];
      const double sig_sq = (xh0 * xh0 + xh1 * xh1 + xh2 * xh2) -
                            2.0 * b * (xh0 * S.n0[0] + xh1 * S.n0[1] + xh2 * S.n0[2]);
      const double g_dot_n0 = gx * S.n0[0] + gy * S.n0[1] + gz * S.n0[2];
      const double g_dot_xh = gx * xh0 + gy * xh1 + gz * xh2;
      const double n0_dot_n = S.n0[0] * NXj + S.n0[1] * NYj + S.n0[2] * NZj;
      const double xh_dot_n = xh0 * NXj + xh1 * NYj + xh2 * NZj;
      const double c_m1a = g_dot_n0 * n0_dot_n;
      const double c_m1b = g_dot_xh * n0_dot_n + g_dot_n0 * xh_dot_n;
      const double c_m2a = g_dot_xh * xh_dot_n;
      const double c_m2b = b * c_m1b;
      double H2, H3;
      reg = dl_7ord(r2, rinv, g, S.c, H2, H3);
      const double area = Aj;
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
      const double gdd = QXj * dx + QYj * dy + QZj * dz;
      const double ndd = NXj * dx + NYj * dy + NZj * dz;
      const double rinv2 = rinv * rinv;
      const double kernel = gdd * ndd * (rinv2 * rinv2 * rinv) * Aj;
      a0 += dx * kernel;
      a1 += dy * kernel;
      a2 += dz * kernel;
    }
  } else if (KIND == K_E2G_P_AWAY) {
    // stokes_pressure_away (E2G/stokes.cpp:108-121)
    const double H2 = (QXj * dx + QYj * dy + QZj * dz) * (rinv * rinv * rinv);
    a0 += H2 * Aj;
  } else if (KIND == K_E2G_P7) {
    // stokes_pressure_7ord (E2G/stokes.cpp:151-194)
    double H2;
    reg = lapl_dl_7ord(r2, rinv, g, S.c, H2);
    const double n0 = NXj, n1 = NYj, n2 = NZj;
    const double f0 = QXj, f1 = QYj, f2 = QZj;
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
    a0 += (normal + tangential) * H2 * Aj;
  }
  return reg;
}

// The box-face sums of one target in one pass (K_E2G_UP_AWAY):
// stokes_SL_away and stokes_pressure_away (E2G/stokes.cpp:13-45, 102-126)
// share the offset, the distance and f.dx, and each keeps the expression of
// its own kind above; a3 collects the pressure.
__device__ __forceinline__ void pair64_face(const double* __restrict__ sm, int j, const Tgt& S, double& a0,
                                            double& a1, double& a2, double& a3) {
  const double2* s2 = reinterpret_cast<const double2*>(sm) + 5 * j;
  const double2 v0 = s2[0], v1 = s2[1], v3 = s2[3], v4 = s2[4];
  const double Xj = v0.x, Yj = v0.y, Zj = v1.x, Aj = v1.y;
  const double QXj = v3.y, QYj = v4.x, QZj = v4.y;
  const double dx = S.px - Xj, dy = S.py - Yj, dz = S.pz - Zj;
  const double r2 = dx * dx + dy * dy + dz * dz;
  const double rinv = rsqrt(r2);
  const double fdd = QXj * dx + QYj * dy + QZj * dz;
  const double H1 = Aj * rinv;
  const double H2 = fdd * H1 * (rinv * rinv);
  a0 += QXj * H1 + dx * H2;
  a1 += QYj * H1 + dy * H2;
  a2 += QZj * H1 + dz * H2;
  a3 += (fdd * (rinv * rinv * rinv)) * Aj;
}

// The band sums of one target in one pass (K_E2G_UP7): stokes_SL_7ord and
// stokes_pressure_7ord (E2G/stokes.cpp:53-97, 134-203) share the offset, the
// distance and the regularized factors' erf and exp (sl_lapl_7ord); each
// keeps the expressions of its own kind above; a3 collects the pressure.
// Returns true if the smoothed branch was taken.
__device__ __forceinline__ bool pair64_band(const double* __restrict__ sm, int j, const Tgt& S, const Reg& g,
                                            double& a0, double& a1, double& a2, double& a3) {
  const double2* s2v = reinterpret_cast<const double2*>(sm) + 5 * j;
  const double2 v0 = s2v[0], v1 = s2v[1], v2 = s2v[2], v3 = s2v[3], v4 = s2v[4];
  const double Xj = v0.x, Yj = v0.y, Zj = v1.x, Aj = v1.y;
  const double NXj = v2.x, NYj = v2.y, NZj = v3.x, QXj = v3.y, QYj = v4.x, QZj = v4.y;
  const double dx = S.px - Xj, dy = S.py - Yj, dz = S.pz - Zj;
  const double r2 = dx * dx + dy * dy + dz * dz;
  const double rinv = rsqrt(r2);
  double H1, H2, H2p;
  const bool reg = sl_lapl_7ord(r2, rinv, g, S.c, H1, H2, H2p);
  {
    const double area = Aj;
    const double fx = QXj - S.f0n0 * NXj;
    const double fy = QYj - S.f0n0 * NYj;
    const double fz = QZj - S.f0n0 * NZj;
    const double fdd = fx * dx + fy * dy + fz * dz;
    H1 *= area;
    H2 *= area * fdd;
    a0 += fx * H1 + dx * H2;
    a1 += fy * H1 + dy * H2;
    a2 += fz * H1 + dz * H2;
  }
  {
    const double n0 = NXj, n1 = NYj, n2 = NZj;
    const double f0 = QXj, f1 = QYj, f2 = QZj;
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
    a3 += (normal + tangential) * H2p * Aj;
  }
  return reg;
}

// ------------------------------------------------------- FP32 plain pairs
// The singular kernel of each kind (the r/delta > 8 branch of the reference),
// from FP32 centre-relative coordinates.
template <int KIND>
__device__ __forceinline__ void pair32(const float4* __restrict__ s4, int j, const Tgt32& F,
                                       float& p0, float& p1, float& p2) {
  constexpr bool kNrm = !(KIND == K_E2G_SL_AWAY || KIND == K_E2G_P_AWAY);
  const float4 P = s4[j];  // x, y, z, area
  const float4 N = kNrm ? s4[kNT + j] : make_float4(0.f, 0.f, 0.f, 0.f);
  const float4 Q = s4[2 * kNT + j];
  const float dx = F.px - P.x, dy = F.py - P.y, dz = F.pz - P.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float rinv = rsqrtf(r2);
  const float rinv2 = rinv * rinv;
  if (KIND == K_E2G_SL_AWAY) {
    // plain Stokeslet, no subtraction; the face sums stage no normals
    const float fx = Q.x, fy = Q.y, fz = Q.z;
    const float fdd = fx * dx + fy * dy + fz * dz;
    const float H1 = P.w * rinv;
    const float H2 = fdd * H1 * rinv2;
    p0 += fx * H1 + dx * H2;
    p1 += fy * H1 + dy * H2;
    p2 += fz * H1 + dz * H2;
  } else if (KIND == K_SL_ON || KIND == K_SL_OFF || KIND == K_E2G_SL7) {
    const float fx = Q.x - F.f0n0 * N.x;
    const float fy = Q.y - F.f0n0 * N.y;
    const float fz = Q.z - F.f0n0 * N.z;
    const float fdd = fx * dx + fy * dy + fz * dz;
    const float H1 = P.w * rinv;
    const float H2 = fdd * H1 * rinv2;
    p0 += fx * H1 + dx * H2;
    p1 += fy * H1 + dy * H2;
    p2 += fz * H1 + dz * H2;
  } else if (KIND == K_DL_ON || KIND == K_DL_OFF) {
    const float gx = Q.x - F.g0[0];
    const float gy = Q.y - F.g0[1];
    const float gz = Q.z - F.g0[2];
    const float gdd = gx * dx + gy * dy + gz * dz;
    const float ndd = N.x * dx + N.y * dy + N.z * dz;
    const float kernel = ndd * gdd * (rinv2 * rinv2 * rinv) * P.w;
    p0 += dx * kernel;
    p1 += dy * kernel;
    p2 += dz * kernel;
  } else if (KIND == K_E2G_P_AWAY) {
    p0 += (Q.x * dx + Q.y * dy + Q.z * dz) * (rinv2 * rinv) * P.w;
  } else if (KIND == K_E2G_P7) {
    const float n0 = N.x, n1 = N.y, n2 = N.z;
    const float f0 = Q.x, f1 = Q.y, f2 = Q.z;
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
    p0 += (normal + tangential) * (rinv2 * rinv) * P.w;
  }
}

// The box-face sums in FP32 in one pass (as pair32 of K_E2G_SL_AWAY and of
// K_E2G_P_AWAY, sharing the offset, the distance and f.dx).
__device__ __forceinline__ void pair32_face(const float4* __restrict__ s4, int j, const Tgt32& F, float& p0,
                                            float& p1, float& p2, float& p3) {
  const float4 P = s4[j];  // x, y, z, area
  const float4 Q = s4[2 * kNT + j];
  const float dx = F.px - P.x, dy = F.py - P.y, dz = F.pz - P.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float rinv = rsqrtf(r2);
  const float rinv2 = rinv * rinv;
  const float fdd = Q.x * dx + Q.y * dy + Q.z * dz;
  const float H1 = P.w * rinv;
  const float H2 = fdd * H1 * rinv2;
  p0 += Q.x * H1 + dx * H2;
  p1 += Q.y * H1 + dy * H2;
  p2 += Q.z * H1 + dz * H2;
  p3 += fdd * (rinv2 * rinv) * P.w;
}

// The band sums in FP32 in one pass, for pairs with r > 3 delta (as pair32r
// of K_E2G_SL7 and of K_E2G_P7, sharing sl_lapl_7ord_f).
__device__ __forceinline__ bool pair32r_band(const float4* __restrict__ s4, int j, const Tgt32& F, const RegF& gf,
                                             float& p0, float& p1, float& p2, float& p3) {
  const float4 P = s4[j];  // x, y, z, area
  const float4 N = s4[kNT + j];
  const float4 Q = s4[2 * kNT + j];
  const float dx = F.px - P.x, dy = F.py - P.y, dz = F.pz - P.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float rinv = rsqrtf(r2);
  const bool reg = r2 <= gf.d64;
  float H1, H2, H2p;
  sl_lapl_7ord_f(r2, rinv, gf, F.c, H1, H2, H2p);
  {
    const float fx = Q.x - F.f0n0 * N.x;
    const float fy = Q.y - F.f0n0 * N.y;
    const float fz = Q.z - F.f0n0 * N.z;
    const float fdd = fx * dx + fy * dy + fz * dz;
    H1 *= P.w;
    H2 *= P.w * fdd;
    p0 += fx * H1 + dx * H2;
    p1 += fy * H1 + dy * H2;
    p2 += fz * H1 + dz * H2;
  }
  {
    const float n0 = N.x, n1 = N.y, n2 = N.z;
    const float f0 = Q.x, f1 = Q.y, f2 = Q.z;
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
    p3 += (normal + tangential) * H2p * P.w;
  }
  return reg;
}

// ------------------------------------- FP32 on-surface pairs, all distances
// Call_Ds_SL_onSurf / Call_Ds_DL_onSurf (2S/KITC.cpp:807-846, 921-957) in
// FP32: the smoothing factor from the FP32 table for s = r^2/delta^2 <= 64,
// the singular kernel beyond (a branch that only warps at the 8 delta
// boundary split on).
template <int KIND>
__device__ __forceinline__ void pair32tab_src(const float4& P, const float4& N, const float4& Q, const Tgt32& F,
                                              const RegF& gf, const float4* __restrict__ tab, float& p0, float& p1,
                                              float& p2) {
  const float dx = F.px - P.x, dy = F.py - P.y, dz = F.pz - P.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float sq = r2 * gf.inv_d2;
  if (KIND == K_SL_ON) {
    const float fx = Q.x - F.f0n0 * N.x;
    const float fy = Q.y - F.f0n0 * N.y;
    const float fz = Q.z - F.f0n0 * N.z;
    const float fdd = fx * dx + fy * dy + fz * dz;
    float H1, H2;
    if (sq <= kPlainOnSurf32) {
      H1 = smooth_eval_f(tab, sq);
      H2 = smooth_eval_f(tab + kSmooth32N / 4, sq);
    } else {
      H1 = rsqrtf(r2);
      H2 = H1 * H1 * H1;
    }
    const float h2 = H2 * fdd;  // the tile holds area x density and area x normal
    p0 += fx * H1 + dx * h2;
    p1 += fy * H1 + dy * h2;
    p2 += fz * H1 + dz * h2;
  } else {  // K_DL_ON
    const float gx = Q.x - F.g0[0];
    const float gy = Q.y - F.g0[1];
    const float gz = Q.z - F.g0[2];
    const float gdd = gx * dx + gy * dy + gz * dz;
    const float ndd = N.x * dx + N.y * dy + N.z * dz;
    float H3;
    if (sq <= kPlainOnSurf32) {
      H3 = smooth_eval_f(tab, sq);
    } else {
      const float ri = rsqrtf(r2), ri2 = ri * ri;
      H3 = ri2 * ri2 * ri;
    }
    const float kernel = ndd * gdd * H3;  // the tile holds area x normal
    p0 += dx * kernel;
    p1 += dy * kernel;
    p2 += dz * kernel;
  }
}

template <int KIND>
__device__ __forceinline__ void pair32tab(const float4* __restrict__ s4, int j, const Tgt32& F, const RegF& gf,
                                          const float4* __restrict__ tab, float& p0, float& p1, float& p2) {
  // source j: (x, y, z, area), area x normal, density (area x density for the Stokeslet)
  pair32tab_src<KIND>(s4[j], s4[kNT + j], s4[2 * kNT + j], F, gf, tab, p0, p1, p2);
}

// ------------------------------------------------ FP32 pairs, r > 3 delta
// The full kernel of a target that uses the regularized forms (the smoothed
// branch for r <= 8 delta, the singular one beyond, with the target's
// subtraction), in FP32 for pairs with r > 3 delta. Returns true if the
// smoothed branch was taken.
template <int KIND>
__device__ __forceinline__ bool pair32r(const float4* __restrict__ s4, int j, const Tgt32& F, const RegF& gf,
                                        float& p0, float& p1, float& p2) {
  const float4 P = s4[j];  // x, y, z, area
  const float4 N = s4[kNT + j];
  const float4 Q = s4[2 * kNT + j];
  const float dx = F.px - P.x, dy = F.py - P.y, dz = F.pz - P.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const float rinv = rsqrtf(r2);
  const bool reg = r2 <= gf.d64;
  if (KIND == K_SL_ON || KIND == K_SL_OFF || KIND == K_E2G_SL7) {
    const float fx = Q.x - F.f0n0 * N.x;
    const float fy = Q.y - F.f0n0 * N.y;
    const float fz = Q.z - F.f0n0 * N.z;
    const float fdd = fx * dx + fy * dy + fz * dz;
    float H1, H2;
    if (KIND == K_SL_ON) sl_7ord_onsurf_f(r2, rinv, gf, H1, H2);
    else sl_7ord_f(r2, rinv, gf, F.c, H1, H2);
    H1 *= P.w;
    H2 *= P.w * fdd;
    p0 += fx * H1 + dx * H2;
    p1 += fy * H1 + dy * H2;
    p2 += fz * H1 + dz * H2;
  } else if (KIND == K_DL_ON) {
    const float gx = Q.x - F.g0[0];
    const float gy = Q.y - F.g0[1];
    const float gz = Q.z - F.g0[2];
    const float gdd = gx * dx + gy * dy + gz * dz;
    const float ndd = N.x * dx + N.y * dy + N.z * dz;
    float H3;
    dl_7ord_onsurf_f(r2, rinv, gf, H3);
    const float kernel = ndd * gdd * H3 * P.w;
    p0 += dx * kernel;
    p1 += dy * kernel;
    p2 += dz * kernel;
  } else if (KIND == K_DL_OFF) {
    // the subtraction form of a near target (2S/KITC.cpp:996-1059)
    const float b = F.b;
    const float xh0 = P.x - F.x0[0], xh1 = P.y - F.x0[1], xh2 = P.z - F.x0[2];
    const float gx = Q.x - F.g0[0], gy = Q.y - F.g0[1], gz = Q.z - F.g0[2];
    const float sig_sq = (xh0 * xh0 + xh1 * xh1 + xh2 * xh2) - 2.0f * b * (xh0 * F.n0[0] + xh1 * F.n0[1] + xh2 * F.n0[2]);
    const float g_dot_n0 = gx * F.n0[0] + gy * F.n0[1] + gz * F.n0[2];
    const float g_dot_xh = gx * xh0 + gy * xh1 + gz * xh2;
    const float n0_dot_n = F.n0[0] * N.x + F.n0[1] * N.y + F.n0[2] * N.z;
    const float xh_dot_n = xh0 * N.x + xh1 * N.y + xh2 * N.z;
    const float c_m1a = g_dot_n0 * n0_dot_n;
    const float c_m1b = g_dot_xh * n0_dot_n + g_dot_n0 * xh_dot_n;
    const float c_m2a = g_dot_xh * xh_dot_n;
    const float c_m2b = b * c_m1b;
    float H2, H3;
    dl_7ord_f(r2, rinv, gf, F.c, H2, H3);
    H2 *= P.w;
    H3 *= P.w;
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
    const float n0 = N.x, n1 = N.y, n2 = N.z;
    const float f0 = Q.x, f1 = Q.y, f2 = Q.z;
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
    p0 += (normal + tangential) * H2 * P.w;
  }
  return reg;
}

// ------------------------------------------------------------ proxy tiles



// Asynchronous copy of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) from global to shared memory by the 32 lanes of a warp.
__device__ __forceinline__ void warp_copy_async(void* dst, const void* src, int bytes, int lane) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  const char* s = static_cast<const char*>(src);
  for (int o = lane * 16; o < bytes; o += 32 * 16)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;\n" ::"r"(d + o), "l"(s + o) : "memory");
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void copy_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Proxy interactions of a run of Chebyshev rows (row r = i (P+1) + j holds
// proxies (i, j, 0..P)) from the warp's shared copy of the node's proxy-major
// moments: FP64 as double2 (DL 5, SL 3 per proxy), FP32 as float4 (DL 3, SL 2).
// Stresslet per proxy: S = (M00, M11, M22, M01 + M10, M02 + M20, M12 + M21),
// Mn (and padding); Stokeslet: f, n. Every lane reads the same proxy (a
// shared-memory broadcast). The stresslet kernel uses
//   sum_l (sum_k (M[3l+k] - g0_l Mn_k) d_k) d_l = d.M.d - (g0.d)(Mn.d),
// the reference's proxy sum (Call_Treecode_DL, 2S/KITC.cpp:753-771)
// regrouped, with d.M.d from the symmetric part and the products of d0, d1
// taken once per row; Call_Treecode_SL (2S/KITC.cpp:700-714) as written.
template <bool DL, int P1C>
__device__ __forceinline__ void proxies64_rows(const double2* __restrict__ s2, int row0, int nrows, int P1rt,
                                               const double* __restrict__ cheb, const Tgt& S, double& a0,
                                               double& a1, double& a2) {
  constexpr int W = DL ? 5 : 3;  // double2 per proxy
  const int P1 = P1C > 0 ? P1C : P1rt;
  for (int r = 0; r < nrows; r++) {
    const int pi = (row0 + r) / P1, pj = (row0 + r) - pi * P1;
    const double d0 = S.px - cheb[pi];
    const double d1 = S.py - cheb[P1 + pj];
    const double r01 = d0 * d0 + d1 * d1;
    const double d00 = d0 * d0, d11 = d1 * d1, d01 = d0 * d1;
    const double g0r = S.g0[0] * d0 + S.g0[1] * d1;
    const double2* row = s2 + r * P1 * W;
#pragma unroll
    for (int pk = 0; pk < (P1C > 0 ? P1C : P1); pk++) {
      const double d2 = S.pz - cheb[2 * P1 + pk];
      const double rinv = rsqrt(fma(d2, d2, r01));
      const double2* m = row + pk * W;
      if (DL) {
        const double2 s01 = m[0], s23 = m[1], s45 = m[2], n01 = m[3], n2 = m[4];
        const double dmd = s01.x * d00 + s01.y * d11 + s23.x * (d2 * d2) + s23.y * d01 + s45.x * (d0 * d2) +
                           s45.y * (d1 * d2);
        const double mnd = n01.x * d0 + n01.y * d1 + n2.x * d2;
        const double g0d = fma(S.g0[2], d2, g0r);
        const double ri2 = rinv * rinv;
        const double kernel = (dmd - g0d * mnd) * (ri2 * ri2 * rinv);
        a0 += d0 * kernel;
        a1 += d1 * kernel;
        a2 += d2 * kernel;
      } else {
        const double2 m01 = m[0], m23 = m[1], m45 = m[2];
        const double q0 = m01.x - S.f0n0 * m23.y;
        const double q1 = m01.y - S.f0n0 * m45.x;
        const double q2 = m23.x - S.f0n0 * m45.y;
        const double temp = (q0 * d0 + q1 * d1 + q2 * d2) * (rinv * rinv * rinv);
        a0 += q0 * rinv + temp * d0;
        a1 += q1 * rinv + temp * d1;
        a2 += q2 * rinv + temp * d2;
      }
    }
  }
}

// FP32 proxies, FP64 accumulation per Chebyshev row. P1C > 0 compiles the
// row length (the proxy loop unrolls and the z coordinates stay in
// registers); P1C = 0 takes any P1.
template <bool DL, int P1C>
__device__ __forceinline__ void proxies32_rows(const float4* __restrict__ s4, int row0, int nrows, int P1rt,
                                               const float* __restrict__ chebf, const Tgt32& F, double& a0,
                                               double& a1, double& a2) {
  constexpr int W = DL ? 3 : 2;  // float4 per proxy
  const int P1 = P1C > 0 ? P1C : P1rt;
  float dz[P1C > 0 ? P1C : 1];
  if constexpr (P1C > 0) {
#pragma unroll
    for (int pk = 0; pk < P1C; pk++) dz[pk] = F.pz - chebf[2 * P1C + pk];
  }
  for (int r = 0; r < nrows; r++) {
    const int pi = (row0 + r) / P1, pj = (row0 + r) - pi * P1;
    const float d0 = F.px - chebf[pi];
    const float d1 = F.py - chebf[P1 + pj];
    const float r01 = d0 * d0 + d1 * d1;
    const float d00 = d0 * d0, d11 = d1 * d1, d01 = d0 * d1;
    const float g0r = F.g0[0] * d0 + F.g0[1] * d1;
    const float4* row = s4 + r * P1 * W;
    float p0 = 0.f, p1 = 0.f, p2 = 0.f;
#pragma unroll
    for (int pk = 0; pk < (P1C > 0 ? P1C : P1); pk++) {
      const float d2 = P1C > 0 ? dz[pk] : F.pz - chebf[2 * P1 + pk];
      const float rinv = rsqrtf(fmaf(d2, d2, r01));
      const float4 A = row[pk * W];
      const float4 B = row[pk * W + 1];
      if (DL) {
        const float Cx = reinterpret_cast<const float*>(row + pk * W + 2)[0];
        const float dmd = A.x * d00 + A.y * d11 + A.z * (d2 * d2) + A.w * d01 + B.x * (d0 * d2) + B.y * (d1 * d2);
        const float mnd = B.z * d0 + B.w * d1 + Cx * d2;
        const float g0d = fmaf(F.g0[2], d2, g0r);
        const float ri2 = rinv * rinv;
        const float kernel = (dmd - g0d * mnd) * (ri2 * ri2 * rinv);
        p0 += d0 * kernel;
        p1 += d1 * kernel;
        p2 += d2 * kernel;
      } else {
        const float m0 = A.x - F.f0n0 * A.w;
        const float m1 = A.y - F.f0n0 * B.x;
        const float m2 = A.z - F.f0n0 * B.y;
        const float temp = (m0 * d0 + m1 * d1 + m2 * d2) * (rinv * rinv * rinv);
        p0 += m0 * rinv + temp * d0;
        p1 += m1 * rinv + temp * d1;
        p2 += m2 * rinv + temp * d2;
      }
    }
    a0 += (double)p0;
    a1 += (double)p1;
    a2 += (double)p2;
  }
}

template <bool DL>
__device__ __forceinline__ void proxies64_any(const double2* __restrict__ s2, int row0, int nrows, int P1,
                                              const double* __restrict__ cheb, const Tgt& S, double& a0, double& a1,
                                              double& a2) {
  switch (P1) {  // the treecode degrees in use: P = 6 (h = 1/64), 10 (h = 1/256)
    case 7: proxies64_rows<DL, 7>(s2, row0, nrows, P1, cheb, S, a0, a1, a2); break;
    case 11: proxies64_rows<DL, 11>(s2, row0, nrows, P1, cheb, S, a0, a1, a2); break;
    default: proxies64_rows<DL, 0>(s2, row0, nrows, P1, cheb, S, a0, a1, a2);
  }
}

template <bool DL>
__device__ __forceinline__ void proxies32_any(const float4* __restrict__ s4, int row0, int nrows, int P1,
                                              const float* __restrict__ chebf, const Tgt32& F, double& a0,
                                              double& a1, double& a2) {
  switch (P1) {  // the treecode degrees in use: P = 5 (inner), 6 (h = 1/64), 10 (h = 1/256)
    case 6: proxies32_rows<DL, 6>(s4, row0, nrows, P1, chebf, F, a0, a1, a2); break;
    case 7: proxies32_rows<DL, 7>(s4, row0, nrows, P1, chebf, F, a0, a1, a2); break;
    case 11: proxies32_rows<DL, 11>(s4, row0, nrows, P1, chebf, F, a0, a1, a2); break;
    default: proxies32_rows<DL, 0>(s4, row0, nrows, P1, chebf, F, a0, a1, a2);
  }
}

template <int KIND, bool MIXED, bool COUNT>
__device__ __forceinline__ void run_item(const EvalTask& T, const BlockRef& it,
                                         const Seg* __restrict__ segs, double* sm, float4* s4,
                                         double* cheb, float* chebf, const double* stab,
                                         const float4* stab32) {
  // work counters (per-branch pair counts) come from FP64 launches made to
  // count them; the other launches skip the branch tests they need
  constexpr bool kCount = !MIXED && COUNT;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int blk = it.blk;
  const int k = blk * kTB + tid;
  const bool valid = k < T.nt;
  const int t = valid ? T.tord[k] : 0;
  // origin of the FP32 coordinates: the block's first target (the sources a
  // block meets lie within a few leaf sizes of it, so FP32 offsets stay small)
  double cb[3];
  {
    const int t0 = T.tord[blk * kTB];
    cb[0] = T.txyz[3 * t0];
    cb[1] = T.txyz[3 * t0 + 1];
    cb[2] = T.txyz[3 * t0 + 2];
  }
  Tgt S;
  Tgt32 F;
  load_target<KIND>(T, t, valid, cb, S, F);
  const Reg g = make_reg(T.DEL);
  RegF gf;
  gf.inv_d = (float)g.inv_d;
  gf.d64 = (float)g.d64;
  gf.inv_d2 = (float)g.inv_d2;
  gf.inv_d3 = (float)g.inv_d3;
  gf.inv_d5 = (float)g.inv_d5;
  // on-surface kinds in the reduced-precision modes: every pair in FP32
  constexpr bool kOn32 = MIXED && (KIND == K_SL_ON || KIND == K_DL_ON);
  // FP64 below, FP32 above: (3 delta)^2 in the mixed mode; in the all-FP32 mode
  // only the r < 1e-14 limits of the reference stay in FP64
  const float cut2f = T.mixed == 2 ? 1e-28f : (float)(9.0 * T.DEL * T.DEL);
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;  // a3: the pressure of K_E2G_UP_AWAY
  unsigned long long creg = 0, cplain = 0, cfar = 0, cprox = 0;
  constexpr bool kFace = KIND == K_E2G_UP_AWAY;
  constexpr bool kSrcNrm = !(KIND == K_E2G_SL_AWAY || KIND == K_E2G_P_AWAY || kFace);
  // which path a target takes through a source tile
  constexpr bool kPerPairSplit = (KIND == K_SL_ON || KIND == K_DL_ON || KIND == K_SL_OFF || KIND == K_DL_OFF ||
                                   KIND == K_E2G_SL7 || KIND == K_E2G_P7 || KIND == K_E2G_UP7);
  constexpr bool kBand = KIND == K_E2G_UP7;
  const bool all32 = MIXED && (KIND == K_E2G_SL_AWAY || KIND == K_E2G_P_AWAY || kFace ||
                               ((KIND == K_SL_OFF || KIND == K_DL_OFF) && !S.near));
  // Each warp walks the item's segments on its own: its own source tiles in
  // shared memory, __syncwarp only, and an entry whose mask is zero for this
  // warp is skipped outright.
  double* wsm = sm + warp * kWarpSm;
  float4* ws4 = s4 + warp * 3 * kNT;
  double* wcheb = cheb + warp * 3 * kMaxP1;
  float* wchebf = chebf + warp * 3 * kMaxP1;
  for (int q = it.seg0; q < it.seg1; q++) {
    const Seg sg = segs[q];
    const Entry E = T.entries[sg.entry];
    const uint32_t wm = E.mask[warp];
    if (wm == 0u) continue;
    const bool act = valid && ((wm >> lane) & 1u);
    if (E.type == 1) {
      const int m0 = sg.s0, m1 = sg.s1 - 1;
      for (int s0 = m0; s0 <= m1; s0 += kNT) {
        const int cnt = min(kNT, m1 - s0 + 1);
        __syncwarp();
        for (int i = lane; i < cnt; i += 32) {
          const int s = s0 + i;
          const double x = T.sx[s], y = T.sy[s], z = T.sz[s];
          // on-surface kinds: area folded into the normal (and, for the
          // Stokeslet, the density), which they only use multiplied by it
          constexpr bool kAreaN = (KIND == K_SL_ON || KIND == K_DL_ON), kAreaQ = (KIND == K_SL_ON);
          if (!kOn32) {
            double2* w2 = reinterpret_cast<double2*>(wsm) + 5 * i;
            const double as = T.sa[s];
            const double an = kAreaN ? as : 1.0, aq = kAreaQ ? as : 1.0;
            w2[0] = make_double2(x, y);
            w2[1] = make_double2(z, as);
            w2[2] = kSrcNrm ? make_double2(an * T.snx[s], an * T.sny[s]) : make_double2(0.0, 0.0);
            w2[3] = make_double2(kSrcNrm ? an * T.snz[s] : 0.0, aq * T.qx[s]);
            w2[4] = make_double2(aq * T.qy[s], aq * T.qz[s]);
          }
          if (MIXED) {
            ws4[i] = make_float4((float)(x - cb[0]), (float)(y - cb[1]), (float)(z - cb[2]), T.fa[s]);
            if (kAreaN) {
              const double as = T.sa[s];
              ws4[kNT + i] = make_float4((float)(as * T.snx[s]), (float)(as * T.sny[s]), (float)(as * T.snz[s]), 0.f);
              if (kAreaQ)
                ws4[2 * kNT + i] = make_float4((float)(as * T.qx[s]), (float)(as * T.qy[s]), (float)(as * T.qz[s]), 0.f);
              else
                ws4[2 * kNT + i] = make_float4(T.fqx[s], T.fqy[s], T.fqz[s], 0.f);
            } else {
              if (kSrcNrm) ws4[kNT + i] = make_float4(T.fnx[s], T.fny[s], T.fnz[s], 0.f);
              ws4[2 * kNT + i] = make_float4(T.fqx[s], T.fqy[s], T.fqz[s], 0.f);
            }
          }
        }
        __syncwarp();
        if (!act) continue;
        if (kOn32) {
          for (int j0 = 0; j0 < cnt; j0 += 16) {
            float p0 = 0.f, p1 = 0.f, p2 = 0.f;
            const int j1 = min(cnt, j0 + 16);
#pragma unroll 4
            for (int j = j0; j < j1; j++) pair32tab<KIND>(ws4, j, F, gf, stab32, p0, p1, p2);
            a0 += (double)p0;
            a1 += (double)p1;
            a2 += (double)p2;
          }
        } else if (kFace && all32) {
          for (int j0 = 0; j0 < cnt; j0 += 16) {
            float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
            const int j1 = min(cnt, j0 + 16);
            if (j1 - j0 == 16) {
#pragma unroll 4
              for (int j = j0; j < j0 + 16; j++) pair32_face(ws4, j, F, p0, p1, p2, p3);
            } else {
              for (int j = j0; j < j1; j++) pair32_face(ws4, j, F, p0, p1, p2, p3);
            }
            a0 += (double)p0;
            a1 += (double)p1;
            a2 += (double)p2;
            a3 += (double)p3;
          }
        } else if (all32) {
          for (int j0 = 0; j0 < cnt; j0 += 16) {
            float p0 = 0.f, p1 = 0.f, p2 = 0.f;
            const int j1 = min(cnt, j0 + 16);
            if (j1 - j0 == 16) {  // a full run: a compile-time trip count
#pragma unroll 4
              for (int j = j0; j < j0 + 16; j++) pair32<KIND>(ws4, j, F, p0, p1, p2);
            } else {
              for (int j = j0; j < j1; j++) pair32<KIND>(ws4, j, F, p0, p1, p2);
            }
            a0 += (double)p0;
            a1 += (double)p1;
            a2 += (double)p2;
          }
        } else if (MIXED && kPerPairSplit && S.near) {
          for (int j0 = 0; j0 < cnt; j0 += 16) {
            float p0 = 0.f, p1 = 0.f, p2 = 0.f;
            const int j1 = min(cnt, j0 + 16);
            float p3 = 0.f;
            for (int j = j0; j < j1; j++) {
              const float4 Pj = ws4[j];
              const float dx = F.px - Pj.x, dy = F.py - Pj.y, dz = F.pz - Pj.z;
              if (kBand) {
                if (dx * dx + dy * dy + dz * dz > cut2f) pair32r_band(ws4, j, F, gf, p0, p1, p2, p3);
                else pair64_band(wsm, j, S, g, a0, a1, a2, a3);
              } else {
                if (dx * dx + dy * dy + dz * dz > cut2f) pair32r<KIND>(ws4, j, F, gf, p0, p1, p2);
                else pair64<KIND>(wsm, j, S, g, stab, a0, a1, a2);
              }
            }
            a0 += (double)p0;
            a1 += (double)p1;
            a2 += (double)p2;
            a3 += (double)p3;
          }
        } else if (kBand) {
          unsigned cr = 0;
          if (cnt == kNT) {
#pragma unroll 2
            for (int j = 0; j < kNT; j++) cr += pair64_band(wsm, j, S, g, a0, a1, a2, a3);
          } else {
            for (int j = 0; j < cnt; j++) cr += pair64_band(wsm, j, S, g, a0, a1, a2, a3);
          }
          if (kCount) {  // two sums' pairs
            creg += 2 * cr;
            cplain += 2 * (cnt - cr);
          }
        } else if (kFace) {
          if (cnt == kNT) {
#pragma unroll 4
            for (int j = 0; j < kNT; j++) pair64_face(wsm, j, S, a0, a1, a2, a3);
          } else {
#pragma unroll 2
            for (int j = 0; j < cnt; j++) pair64_face(wsm, j, S, a0, a1, a2, a3);
          }
          if (kCount) cfar += 2 * cnt;  // two sums' pairs
        } else {
          unsigned cr = 0;
          if (cnt == kNT) {  // a full tile: a compile-time trip count
#pragma unroll 4
            for (int j = 0; j < kNT; j++) cr += pair64<KIND>(wsm, j, S, g, stab, a0, a1, a2);
          } else {
#pragma unroll 2
            for (int j = 0; j < cnt; j++) cr += pair64<KIND>(wsm, j, S, g, stab, a0, a1, a2);
          }
          if (kCount) {
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
      // The node's proxy-major moments stream through the warp's tile in
      // runs of whole Chebyshev rows, double-buffered: the asynchronous copy
      // of the next run overlaps the interactions of this one.
      constexpr int kBpp = MIXED ? (DL ? 48 : 32) : (DL ? 80 : 48);  // bytes per proxy
      constexpr int kHalf = kWarpSm * 4;                              // bytes per buffer
      const char* src = MIXED ? reinterpret_cast<const char*>(T.momf + (size_t)E.node * Pf * (DL ? 12 : 8))
                              : reinterpret_cast<const char*>(T.mom + (size_t)E.node * Pf * C);
      char* buf = reinterpret_cast<char*>(wsm);
      const int rowb = P1 * kBpp;
      const int nr = max(1, kHalf / rowb);
      const int nrow_all = P1 * P1;
      const int nch = (nrow_all + nr - 1) / nr;
      __syncwarp();
      for (int i = lane; i < 3 * P1; i += 32) {
        const double v = T.tcheb[(size_t)E.node * 3 * P1 + i];
        wcheb[i] = v;
        if (MIXED) wchebf[i] = (float)(v - cb[i / P1]);
      }
      warp_copy_async(buf, src, min(nr, nrow_all) * rowb, lane);
      for (int ch = 0; ch < nch; ch++) {
        const int row0 = ch * nr, rows = min(nr, nrow_all - row0);
        if (ch + 1 < nch) {
          const int r1 = row0 + nr;
          warp_copy_async(buf + ((ch + 1) & 1) * kHalf, src + (size_t)r1 * rowb, min(nr, nrow_all - r1) * rowb,
                          lane);
          copy_async_wait<1>();
        } else {
          copy_async_wait<0>();
        }
        __syncwarp();
        if (act) {
          const char* cur = buf + (ch & 1) * kHalf;
          if (MIXED)
            proxies32_any<DL>(reinterpret_cast<const float4*>(cur), row0, rows, P1, wchebf, F, a0, a1, a2);
          else
            proxies64_any<DL>(reinterpret_cast<const double2*>(cur), row0, rows, P1, wcheb, S, a0, a1, a2);
        }
        __syncwarp();
      }
      if (kCount && act) cprox += Pf;
    }
  }
  // partial sums of this item
  double* o = T.partial + ((size_t)it.slot * kTB + tid) * kPartComps;
  o[0] = a0;
  o[1] = a1;
  o[2] = a2;
  o[3] = a3;
  // Work counters (pair kinds actually evaluated), one atomic per warp.
  if (kCount && T.counters) {
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

// ------------------------------------- two targets per thread (mixed, on-surface)

// FP32 proxies of a run of Chebyshev rows for two targets: each shared-memory
// read of a proxy serves both. Sums per row go to acc (FP64). P1C as in
// proxies32_rows.
template <bool DL, int P1C>
__device__ __forceinline__ void proxies32_rows2(const float4* __restrict__ s4, int row0, int nrows, int P1rt,
                                                const float* __restrict__ chebf, const Tgt32 (&F)[2],
                                                double (&acc)[2][3]) {
  constexpr int W = DL ? 3 : 2;  // float4 per proxy
  const int P1 = P1C > 0 ? P1C : P1rt;
  float czr[P1C > 0 ? P1C : 1];
  if constexpr (P1C > 0) {
#pragma unroll
    for (int pk = 0; pk < P1C; pk++) czr[pk] = chebf[2 * P1C + pk];
  }
  for (int r = 0; r < nrows; r++) {
    const int pi = (row0 + r) / P1, pj = (row0 + r) - pi * P1;
    const float cx = chebf[pi], cy = chebf[P1 + pj];
    float d0[2], d1[2], r01[2], d00[2], d11[2], d01[2], g0r[2];
    float p[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};
#pragma unroll
    for (int q = 0; q < 2; q++) {
      d0[q] = F[q].px - cx;
      d1[q] = F[q].py - cy;
      r01[q] = d0[q] * d0[q] + d1[q] * d1[q];
      d00[q] = d0[q] * d0[q];
      d11[q] = d1[q] * d1[q];
      d01[q] = d0[q] * d1[q];
      g0r[q] = F[q].g0[0] * d0[q] + F[q].g0[1] * d1[q];
    }
    const float4* row = s4 + r * P1 * W;
#pragma unroll
    for (int pk = 0; pk < (P1C > 0 ? P1C : P1); pk++) {
      const float cz = P1C > 0 ? czr[pk] : chebf[2 * P1 + pk];
      const float4 A = row[pk * W];
      const float4 B = row[pk * W + 1];
      const float Cx = DL ? reinterpret_cast<const float*>(row + pk * W + 2)[0] : 0.f;
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const float d2 = F[q].pz - cz;
        const float rinv = rsqrtf(fmaf(d2, d2, r01[q]));
        if (DL) {
          const float dmd = A.x * d00[q] + A.y * d11[q] + A.z * (d2 * d2) + A.w * d01[q] + B.x * (d0[q] * d2) +
                            B.y * (d1[q] * d2);
          const float mnd = B.z * d0[q] + B.w * d1[q] + Cx * d2;
          const float g0d = fmaf(F[q].g0[2], d2, g0r[q]);
          const float ri2 = rinv * rinv;
          const float kernel = (dmd - g0d * mnd) * (ri2 * ri2 * rinv);
          p[q][0] += d0[q] * kernel;
          p[q][1] += d1[q] * kernel;
          p[q][2] += d2 * kernel;
        } else {
          const float m0 = A.x - F[q].f0n0 * A.w;
          const float m1 = A.y - F[q].f0n0 * B.x;
          const float m2 = A.z - F[q].f0n0 * B.y;
          const float temp = (m0 * d0[q] + m1 * d1[q] + m2 * d2) * (rinv * rinv * rinv);
          p[q][0] += m0 * rinv + temp * d0[q];
          p[q][1] += m1 * rinv + temp * d1[q];
          p[q][2] += m2 * rinv + temp * d2;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 2; q++)
      for (int c = 0; c < 3; c++) acc[q][c] += (double)p[q][c];
  }
}

template <bool DL>
__device__ __forceinline__ void proxies32_any2(const float4* __restrict__ s4, int row0, int nrows, int P1,
                                               const float* __restrict__ chebf, const Tgt32 (&F)[2],
                                               double (&acc)[2][3]) {
  switch (P1) {  // the treecode degrees in use: P = 5 (inner), 6 (h = 1/64), 10 (h = 1/256)
    case 6: proxies32_rows2<DL, 6>(s4, row0, nrows, P1, chebf, F, acc); break;
    case 7: proxies32_rows2<DL, 7>(s4, row0, nrows, P1, chebf, F, acc); break;
    case 11: proxies32_rows2<DL, 11>(s4, row0, nrows, P1, chebf, F, acc); break;
    default: proxies32_rows2<DL, 0>(s4, row0, nrows, P1, chebf, F, acc);
  }
}

// The reduced-precision on-surface items (K_SL_ON / K_DL_ON, every pair in
// FP32 with the tabulated smoothing factors) with two targets per thread: a
// CTA of kTB2 = 64 threads covers the block's 128 targets — warp w holds
// targets 64 w + lane and 64 w + 32 + lane, i.e. mask words 2 w and 2 w + 1 —
// so every source and proxy read from shared memory serves two pairs.
constexpr int kTB2 = 64;
template <int KIND>
__device__ __forceinline__ void run_item_on2(const EvalTask& T, const BlockRef& it, const Seg* __restrict__ segs,
                                             double* sm, float4* s4, float* chebf, const float4* stab32) {
  constexpr bool DL = (KIND == K_DL_ON);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int blk = it.blk;
  double cb[3];
  {
    const int t0 = T.tord[blk * kTB];
    cb[0] = T.txyz[3 * t0];
    cb[1] = T.txyz[3 * t0 + 1];
    cb[2] = T.txyz[3 * t0 + 2];
  }
  Tgt32 F[2];
  bool valid[2];
#pragma unroll
  for (int q = 0; q < 2; q++) {
    const int k = blk * kTB + warp * 64 + q * 32 + lane;
    valid[q] = k < T.nt;
    Tgt S;
    load_target<KIND>(T, valid[q] ? T.tord[k] : 0, valid[q], cb, S, F[q]);
  }
  const Reg g = make_reg(T.DEL);
  RegF gf;
  gf.inv_d = (float)g.inv_d;
  gf.d64 = (float)g.d64;
  gf.inv_d2 = (float)g.inv_d2;
  gf.inv_d3 = (float)g.inv_d3;
  gf.inv_d5 = (float)g.inv_d5;
  double a[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  double* wsm = sm + warp * kWarpSm;
  float4* ws4 = s4 + warp * 3 * kNT;
  float* wchebf = chebf + warp * 3 * kMaxP1;
  for (int qs = it.seg0; qs < it.seg1; qs++) {
    const Seg sg = segs[qs];
    const Entry E = T.entries[sg.entry];
    const uint32_t mA = E.mask[2 * warp], mB = E.mask[2 * warp + 1];
    if ((mA | mB) == 0u) continue;
    const bool actA = valid[0] && ((mA >> lane) & 1u);
    const bool actB = valid[1] && ((mB >> lane) & 1u);
    if (E.type == 1) {
      const int m0 = sg.s0, m1 = sg.s1 - 1;
      for (int s0 = m0; s0 <= m1; s0 += kNT) {
        const int cnt = min(kNT, m1 - s0 + 1);
        __syncwarp();
        for (int i = lane; i < cnt; i += 32) {
          const int s = s0 + i;
          const double as = T.sa[s];
          ws4[i] = make_float4((float)(T.sx[s] - cb[0]), (float)(T.sy[s] - cb[1]), (float)(T.sz[s] - cb[2]),
                               (float)as);
          ws4[kNT + i] = make_float4((float)(as * T.snx[s]), (float)(as * T.sny[s]), (float)(as * T.snz[s]), 0.f);
          if (KIND == K_SL_ON)
            ws4[2 * kNT + i] = make_float4((float)(as * T.qx[s]), (float)(as * T.qy[s]), (float)(as * T.qz[s]), 0.f);
          else
            ws4[2 * kNT + i] = make_float4(T.fqx[s], T.fqy[s], T.fqz[s], 0.f);
        }
        __syncwarp();
        if (!actA && !actB) continue;
        for (int j0 = 0; j0 < cnt; j0 += 16) {
          float pA[3] = {0.f, 0.f, 0.f}, pB[3] = {0.f, 0.f, 0.f};
          const int j1 = min(cnt, j0 + 16);
          if (j1 - j0 == 16) {  // a full run: a compile-time trip count
#pragma unroll 4
            for (int j = j0; j < j0 + 16; j++) {
              const float4 P = ws4[j], N = ws4[kNT + j], Q = ws4[2 * kNT + j];
              pair32tab_src<KIND>(P, N, Q, F[0], gf, stab32, pA[0], pA[1], pA[2]);
              pair32tab_src<KIND>(P, N, Q, F[1], gf, stab32, pB[0], pB[1], pB[2]);
            }
          } else {
#pragma unroll 2
            for (int j = j0; j < j1; j++) {
              const float4 P = ws4[j], N = ws4[kNT + j], Q = ws4[2 * kNT + j];
              pair32tab_src<KIND>(P, N, Q, F[0], gf, stab32, pA[0], pA[1], pA[2]);
              pair32tab_src<KIND>(P, N, Q, F[1], gf, stab32, pB[0], pB[1], pB[2]);
            }
          }
          if (actA)
            for (int c = 0; c < 3; c++) a[0][c] += (double)pA[c];
          if (actB)
            for (int c = 0; c < 3; c++) a[1][c] += (double)pB[c];
        }
      }
    } else {
      // far node: the proxy-major FP32 moments through the warp's tile, double-buffered
      const int P1 = T.P1, Pf = T.Pf;
      constexpr int kBpp = DL ? 48 : 32;  // bytes per proxy
      constexpr int kHalf = kWarpSm * 4;  // bytes per buffer
      const char* src = reinterpret_cast<const char*>(T.momf + (size_t)E.node * Pf * (DL ? 12 : 8));
      char* buf = reinterpret_cast<char*>(wsm);
      const int rowb = P1 * kBpp;
      const int nr = max(1, kHalf / rowb);
      const int nrow_all = P1 * P1;
      const int nch = (nrow_all + nr - 1) / nr;
      __syncwarp();
      for (int i = lane; i < 3 * P1; i += 32)
        wchebf[i] = (float)(T.tcheb[(size_t)E.node * 3 * P1 + i] - cb[i / P1]);
      warp_copy_async(buf, src, min(nr, nrow_all) * rowb, lane);
      double acc[2][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
      for (int ch = 0; ch < nch; ch++) {
        const int row0 = ch * nr, rows = min(nr, nrow_all - row0);
        if (ch + 1 < nch) {
          const int r1 = row0 + nr;
          warp_copy_async(buf + ((ch + 1) & 1) * kHalf, src + (size_t)r1 * rowb, min(nr, nrow_all - r1) * rowb,
                          lane);
          copy_async_wait<1>();
        } else {
          copy_async_wait<0>();
        }
        __syncwarp();
        if (actA || actB)
          proxies32_any2<DL>(reinterpret_cast<const float4*>(buf + (ch & 1) * kHalf), row0, rows, P1, wchebf, F,
                              acc);
        __syncwarp();
      }
      if (actA)
        for (int c = 0; c < 3; c++) a[0][c] += acc[0][c];
      if (actB)
        for (int c = 0; c < 3; c++) a[1][c] += acc[1][c];
    }
  }
#pragma unroll
  for (int q = 0; q < 2; q++) {
    double* o = T.partial + ((size_t)it.slot * kTB + warp * 64 + q * 32 + lane) * kPartComps;
    o[0] = a[q][0];
    o[1] = a[q][1];
    o[2] = a[q][2];
    o[3] = 0.0;
  }
}

template <int FAM>
__global__ void __launch_bounds__(kTB2, 8) eval_kernel_on2(const EvalTask* __restrict__ tasks,
                                                           const BlockRef* __restrict__ items,
                                                           const Seg* __restrict__ segs) {
  constexpr int kW2 = kTB2 / 32;
  __shared__ __align__(16) double sm[kW2 * kWarpSm];
  __shared__ float4 sf[kW2 * 3 * kNT];
  __shared__ float chebf[kW2 * 3 * kMaxP1];
  __shared__ EvalTask sT;
  __shared__ float4 stab32[FAM == F_SL ? 2 * kSmooth32N / 4 : kSmooth32N / 4];
  const BlockRef it = items[blockIdx.x];
  if (threadIdx.x == 0) sT = tasks[it.task];
  {
    // FP32 tables with the powers of 1/delta in the coefficients (as in eval_kernel)
    const Reg gs = make_reg(tasks[it.task].DEL);
    float* t32 = reinterpret_cast<float*>(stab32);
    for (int i = threadIdx.x; i < kSmooth32N; i += blockDim.x) {
      const bool centre = (i & 7) == 0;
      if (FAM == F_SL) {
        t32[i] = kSmooth32G1[i] * (centre ? 1.0f : (float)gs.inv_d);
        t32[kSmooth32N + i] = kSmooth32G2[i] * (centre ? 1.0f : (float)gs.inv_d3);
      } else {
        t32[i] = kSmooth32G3[i] * (centre ? 1.0f : (float)gs.inv_d5);
      }
    }
  }
  __syncthreads();
  if (FAM == F_SL) run_item_on2<K_SL_ON>(sT, it, segs, sm, sf, chebf, stab32);
  else run_item_on2<K_DL_ON>(sT, it, segs, sm, sf, chebf, stab32);
}

// ON = true: the batch's lean items only — on-surface kinds (K_SL_ON / K_DL_ON)
// or, for the extend-to-grid family, the plain box-face sums (K_E2G_*_AWAY).
// Their code path needs fewer registers than the others' (no nearest-point
// data, no per-target regularization coefficients), so it runs with more
// resident CTAs per SM: six (80 registers) for the Stokeslet and box-face
// sums, five (96) for the stresslet, whose larger smoothing table fills the
// shared memory of a sixth (its degree-11 table that would fit measured
// slower). The FP64 off-surface Stokeslet items fit 96 registers without
// spills and run five CTAs per SM; the other off-surface kernels four.
template <int FAM, bool MIXED, bool ON, bool COUNT>
__global__ void __launch_bounds__(kTB, ON ? (FAM == F_DL ? 5 : 6) : ((FAM == F_SL && !MIXED) ? 5 : 4))
    eval_kernel(const EvalTask* __restrict__ tasks, const BlockRef* __restrict__ items,
                const Seg* __restrict__ segs) {
  __shared__ __align__(16) double sm[kSmem];
  // per-warp FP32 source tiles: (x, y, z, area), (n, 0), (q, 0) per source
  __shared__ float4 sf[MIXED ? kWarps * 3 * kNT : 1];
  __shared__ double cheb[kWarps * 3 * kMaxP1];
  __shared__ float chebf[kWarps * 3 * kMaxP1];
  __shared__ EvalTask sT;
  // smoothing tables: G1, G2 for the Stokeslet family, G3 for the stresslet family
  __shared__ __align__(16) double stab[(FAM == F_SL && ON) ? TabG1::kLen + TabG2::kLen
                                                            : ((FAM == F_DL && ON) ? TabG3::kLen : 2)];
  __shared__ float4 stab32[MIXED ? (FAM == F_SL ? 2 * kSmooth32N / 4 : (FAM == F_DL ? kSmooth32N / 4 : 1)) : 1];
  const BlockRef it = items[blockIdx.x];
  if (threadIdx.x == 0) sT = tasks[it.task];
  // The tables carry the powers of 1/delta of the factors they give: every
  // coefficient is scaled by 1/delta, 1/delta^3 (G1, G2) or 1/delta^5 (G3)
  // while they are staged.
  if ((FAM == F_SL || FAM == F_DL) && ON) {
    const Reg gs = make_reg(tasks[it.task].DEL);
    if (FAM == F_SL) {
      for (int i = threadIdx.x; i < TabG1::kLen; i += blockDim.x) {
        stab[i] = kSmoothSG1[i] * gs.inv_d;
        stab[TabG1::kLen + i] = kSmoothSG2[i] * gs.inv_d3;
      }
    } else {
      for (int i = threadIdx.x; i < TabG3::kLen; i += blockDim.x) stab[i] = kSmoothSG3[i] * gs.inv_d5;
    }
    if (MIXED) {
      float* t32 = reinterpret_cast<float*>(stab32);
      for (int i = threadIdx.x; i < kSmooth32N; i += blockDim.x) {
        const bool centre = (i & 7) == 0;
        if (FAM == F_SL) {
          t32[i] = kSmooth32G1[i] * (centre ? 1.0f : (float)gs.inv_d);
          t32[kSmooth32N + i] = kSmooth32G2[i] * (centre ? 1.0f : (float)gs.inv_d3);
        } else {
          t32[i] = kSmooth32G3[i] * (centre ? 1.0f : (float)gs.inv_d5);
        }
      }
    }
  }
  __syncthreads();
  const int kind = sT.kind;
  if (FAM == F_SL) {
    if (ON) run_item<K_SL_ON, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
    else run_item<K_SL_OFF, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
  } else if (FAM == F_DL) {
    if (ON) run_item<K_DL_ON, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
    else run_item<K_DL_OFF, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
  } else if (ON) {  // extend-to-grid: the plain box-face sums
    if (kind == K_E2G_UP_AWAY) run_item<K_E2G_UP_AWAY, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
    else if (kind == K_E2G_SL_AWAY) run_item<K_E2G_SL_AWAY, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
    else run_item<K_E2G_P_AWAY, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
  } else {  // extend-to-grid: the regularized band sums
    if (kind == K_E2G_UP7) run_item<K_E2G_UP7, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
    else if (kind == K_E2G_SL7) run_item<K_E2G_SL7, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
    else run_item<K_E2G_P7, MIXED, COUNT>(sT, it, segs, sm, sf, cheb, chebf, stab, stab32);
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
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  const int s0 = T.item_start[blk], s1 = T.item_start[blk + 1];
  for (int s = s0; s < s1; s++) {
    const double* p = T.partial + ((size_t)s * kTB + tid) * kPartComps;
    a0 += p[0];
    a1 += p[1];
    a2 += p[2];
    a3 += p[3];
  }
  const double sc = T.scale;
  double* o = T.out;
  const int kind = T.kind;
  if (kind == K_SL_ON || kind == K_SL_OFF || kind == K_E2G_SL_AWAY || kind == K_E2G_SL7) {
    o[3 * t] = a0 * sc;
    o[3 * t + 1] = a1 * sc;
    o[3 * t + 2] = a2 * sc;
  } else if (kind == K_E2G_UP_AWAY) {
    o[3 * t] = a0 * sc;
    o[3 * t + 1] = a1 * sc;
    o[3 * t + 2] = a2 * sc;
    T.out2[t] = a3 * T.scale2;
  } else if (kind == K_E2G_UP7) {
    o[3 * t] = a0 * sc;
    o[3 * t + 1] = a1 * sc;
    o[3 * t + 2] = a2 * sc;
    // p *= -denom_FourPI (scale2); inside: p -= f0.n0 (E2G/stokes.cpp:196-200)
    double p = a3 * T.scale2;
    if (T.tb[t] < -1.e-12) {
      const double* f0 = T.tf0 + 3 * t;
      const double* n0 = T.tn0 + 3 * t;
      p -= f0[0] * n0[0] + f0[1] * n0[1] + f0[2] * n0[2];
    }
    T.out2[t] = p;
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

template <int FAM, bool MIXED, bool COUNT>
void launch_family(const EvalTask* d_tasks, const BlockRef* d_items, const Seg* d_segs, int nitems, int n_on,
                   cudaStream_t st, cudaStream_t side, cudaEvent_t fork, cudaEvent_t join) {
  const bool two = n_on > 0 && nitems > n_on && side;
  cudaStream_t s2 = two ? side : st;
  if (two) {
    cudaEventRecord(fork, st);
    cudaStreamWaitEvent(side, fork, 0);
  }
  if (n_on > 0) {
    if constexpr (MIXED && FAM != F_E2G) eval_kernel_on2<FAM><<<n_on, kTB2, 0, st>>>(d_tasks, d_items, d_segs);
    else eval_kernel<FAM, MIXED, true, COUNT><<<n_on, kTB, 0, st>>>(d_tasks, d_items, d_segs);
  }
  if (nitems > n_on)
    eval_kernel<FAM, MIXED, false, COUNT><<<nitems - n_on, kTB, 0, s2>>>(d_tasks, d_items + n_on, d_segs);
  if (two) {
    cudaEventRecord(join, side);
    cudaStreamWaitEvent(st, join, 0);
  }
}

template <int FAM>
void launch_family_any(bool mixed, bool count, const EvalTask* d_tasks, const BlockRef* d_items, const Seg* d_segs,
                       int nitems, int n_on, cudaStream_t st, cudaStream_t side, cudaEvent_t fork,
                       cudaEvent_t join) {
  if (mixed) launch_family<FAM, true, false>(d_tasks, d_items, d_segs, nitems, n_on, st, side, fork, join);
  else if (count) launch_family<FAM, false, true>(d_tasks, d_items, d_segs, nitems, n_on, st, side, fork, join);
  else launch_family<FAM, false, false>(d_tasks, d_items, d_segs, nitems, n_on, st, side, fork, join);
}

void launch_eval(int family, const EvalTask* d_tasks, const BlockRef* d_items, const Seg* d_segs,
                 int nitems, int n_on, int ntask_blocks, const int2* d_task_blocks, cudaStream_t st,
                 cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, bool mixed, bool count) {
  if (nitems > 0) {
    // the extend-to-grid tasks carry no counters
    if (family == F_SL)
      launch_family_any<F_SL>(mixed, count, d_tasks, d_items, d_segs, nitems, n_on, st, side, fork, join);
    else if (family == F_DL)
      launch_family_any<F_DL>(mixed, count, d_tasks, d_items, d_segs, nitems, n_on, st, side, fork, join);
    else if (mixed)
      launch_family<F_E2G, true, false>(d_tasks, d_items, d_segs, nitems, n_on, st, side, fork, join);
    else
      launch_family<F_E2G, false, false>(d_tasks, d_items, d_segs, nitems, n_on, st, side, fork, join);
  }
  if (ntask_blocks > 0) reduce_kernel<<<ntask_blocks, kTB, 0, st>>>(d_tasks, d_task_blocks);
}

}  // namespace hr
