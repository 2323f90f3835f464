// hr_eval.cu — the boundary-sum kernel family.
//
// One CTA owns one block of 128 spatially sorted targets (one target per
// thread, FP64 accumulators in registers) and walks that block's interaction
// entries in a fixed order, so every result is deterministic:
//   * near entry  -> direct sum over the node's member sources, staged in
//                    shared memory in tiles of 256 (Call_Ds_*, 2S/KITC.cpp:807-1062;
//                    in direct mode the single node holds all sources, i.e.
//                    eval_Stokes_*_{on,off}Surf, 2S/stokeslets.cpp, 2S/stresslets.cpp,
//                    and the E2G sums of E2G/stokes.cpp);
//   * far entry   -> the node's (P+1)^3 proxy points with their moments staged
//                    in shared memory (Call_Treecode_*, 2S/KITC.cpp:671-777).
// A warp whose mask word is zero for an entry skips the arithmetic entirely.
// The per-pair formulas are those of hr_pairs.cuh; the per-target epilogues
// (scale and jump terms) are those of the reference drivers cited below.
#include <cstdio>

#include "hr_device.h"
#include "hr_pairs.cuh"

namespace hr {

namespace {

constexpr int kNT = 256;               // sources per shared-memory tile
constexpr int kSmem = 10 * kNT;        // doubles: 10 SoA arrays of a source tile
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

template <int KIND>
__device__ __forceinline__ void load_target(const EvalTask& T, int t, bool valid, Tgt& S) {
  S.px = S.py = S.pz = 0.0;
  S.b = 0.0;
  S.f0n0 = 0.0;
  for (int k = 0; k < 3; k++) S.x0[k] = S.n0[k] = S.g0[k] = S.n0xf0[k] = 0.0;
  S.c.c1 = S.c.c2 = S.c.c3 = 0.0;
  // regularized-kernel kinds: on-surface sums and the E2G band sums
  S.near = (KIND == K_SL_ON || KIND == K_DL_ON || KIND == K_E2G_SL7 || KIND == K_E2G_P7) ? 1 : 0;
  if (!valid) return;
  S.px = T.txyz[3 * t];
  S.py = T.txyz[3 * t + 1];
  S.pz = T.txyz[3 * t + 2];
  if (KIND == K_SL_ON) {
    // f0_dot_n0 = Surfc[i].f . Surfc[i].Nrml  (2S/KITC.cpp:1461, 2S/stokeslets.cpp:167)
    S.f0n0 = T.tq[3 * t] * T.tnrm[3 * t] + T.tq[3 * t + 1] * T.tnrm[3 * t + 1] +
             T.tq[3 * t + 2] * T.tnrm[3 * t + 2];
  } else if (KIND == K_SL_OFF || KIND == K_E2G_SL7) {
    S.b = T.tb[t];
    S.near = T.tnear[t];
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

// Direct sum of one staged tile for one target.
template <int KIND>
__device__ __forceinline__ void tile_pairs(const double* __restrict__ sm, int cnt, double DEL,
                                           double d64, const Tgt& S, double& a0, double& a1,
                                           double& a2, unsigned long long& creg,
                                           unsigned long long& cplain) {
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
  if (KIND == K_SL_ON) {
    // Call_Ds_SL_onSurf (2S/KITC.cpp:807-844)
    for (int j = 0; j < cnt; j++) {
      double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
      double r2 = dx * dx + dy * dy + dz * dz;
      double r = sqrt(r2);
      double area = A[j];
      double fx = QX[j] - S.f0n0 * NX[j];
      double fy = QY[j] - S.f0n0 * NY[j];
      double fz = QZ[j] - S.f0n0 * NZ[j];
      double fdd = fx * dx + fy * dy + fz * dz;
      double H1, H2;
      sl_7ord_onsurf(r, DEL, H1, H2);
      creg += (r2 <= d64);
      H1 *= area;
      H2 *= area * fdd;
      a0 += fx * H1 + dx * H2;
      a1 += fy * H1 + dy * H2;
      a2 += fz * H1 + dz * H2;
    }
    cplain += cnt;
  } else if (KIND == K_SL_OFF || KIND == K_E2G_SL7) {
    if (S.near) {
      // Call_Ds_SL regularized branch (2S/KITC.cpp:883-915), stokes_SL_7ord
      for (int j = 0; j < cnt; j++) {
        double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2);
        double area = A[j];
        double fx = QX[j] - S.f0n0 * NX[j];
        double fy = QY[j] - S.f0n0 * NY[j];
        double fz = QZ[j] - S.f0n0 * NZ[j];
        double fdd = fx * dx + fy * dy + fz * dz;
        double H1, H2;
        sl_7ord(r, DEL, S.c, H1, H2);
        creg += (r2 <= d64);
        H1 *= area;
        H2 *= fdd * area;
        a0 += fx * H1 + dx * H2;
        a1 += fy * H1 + dy * H2;
        a2 += fz * H1 + dz * H2;
      }
    } else {
      // far target: plain Stokeslet without subtraction (2S/KITC.cpp:856-882)
      for (int j = 0; j < cnt; j++) {
        double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2);
        double area = A[j];
        double fx = QX[j], fy = QY[j], fz = QZ[j];
        double fdd = fx * dx + fy * dy + fz * dz;
        double H1 = area / r;
        double H2 = fdd * area / (r2 * r);
        a0 += fx * H1 + dx * H2;
        a1 += fy * H1 + dy * H2;
        a2 += fz * H1 + dz * H2;
      }
    }
    cplain += cnt;
  } else if (KIND == K_DL_ON) {
    // Call_Ds_DL_onSurf (2S/KITC.cpp:921-957)
    for (int j = 0; j < cnt; j++) {
      double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
      double r2 = dx * dx + dy * dy + dz * dz;
      double r = sqrt(r2);
      double gx = QX[j] - S.g0[0];
      double gy = QY[j] - S.g0[1];
      double gz = QZ[j] - S.g0[2];
      double gdd = gx * dx + gy * dy + gz * dz;
      double ndd = NX[j] * dx + NY[j] * dy + NZ[j] * dz;
      double H3 = dl_7ord_onsurf(r, DEL);
      creg += (r2 <= d64);
      double kernel = ndd * gdd * H3 * A[j];
      a0 += dx * kernel;
      a1 += dy * kernel;
      a2 += dz * kernel;
    }
    cplain += cnt;
  } else if (KIND == K_DL_OFF) {
    if (S.near) {
      // Call_Ds_DL regularized branch (2S/KITC.cpp:996-1059), stokes_DL_7ord
      const double b = S.b;
      for (int j = 0; j < cnt; j++) {
        double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2);
        double xh0 = X[j] - S.x0[0];
        double xh1 = Y[j] - S.x0[1];
        double xh2 = Z[j] - S.x0[2];
        double gx = QX[j] - S.g0[0];
        double gy = QY[j] - S.g0[1];
        double gz = QZ[j] - S.g0[2];
        double sig_sq = (xh0 * xh0 + xh1 * xh1 + xh2 * xh2) -
                        2.0 * b * (xh0 * S.n0[0] + xh1 * S.n0[1] + xh2 * S.n0[2]);
        double g_dot_n0 = gx * S.n0[0] + gy * S.n0[1] + gz * S.n0[2];
        double g_dot_xh = gx * xh0 + gy * xh1 + gz * xh2;
        double n0_dot_n = S.n0[0] * NX[j] + S.n0[1] * NY[j] + S.n0[2] * NZ[j];
        double xh_dot_n = xh0 * NX[j] + xh1 * NY[j] + xh2 * NZ[j];
        double c_m1a = g_dot_n0 * n0_dot_n;
        double c_m1b = g_dot_xh * n0_dot_n + g_dot_n0 * xh_dot_n;
        double c_m2a = g_dot_xh * xh_dot_n;
        double c_m2b = b * c_m1b;
        double H2, H3;
        dl_7ord(r, DEL, S.c, H2, H3);
        creg += (r2 <= d64);
        double area = A[j];
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
      }
    } else {
      // far target: plain stresslet (2S/KITC.cpp:970-995)
      for (int j = 0; j < cnt; j++) {
        double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double r = sqrt(r2);
        double gdd = QX[j] * dx + QY[j] * dy + QZ[j] * dz;
        double ndd = NX[j] * dx + NY[j] * dy + NZ[j] * dz;
        double kernel = gdd * ndd / (r2 * r2 * r) * A[j];
        a0 += dx * kernel;
        a1 += dy * kernel;
        a2 += dz * kernel;
      }
    }
    cplain += cnt;
  } else if (KIND == K_E2G_SL_AWAY) {
    // stokes_SL_away (E2G/stokes.cpp:22-40)
    for (int j = 0; j < cnt; j++) {
      double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
      double r2 = dx * dx + dy * dy + dz * dz;
      double fdd = QX[j] * dx + QY[j] * dy + QZ[j] * dz;
      double H1 = 1.0 / sqrt(r2) * A[j];
      double H2 = H1 / r2 * fdd;
      a0 += QX[j] * H1 + dx * H2;
      a1 += QY[j] * H1 + dy * H2;
      a2 += QZ[j] * H1 + dz * H2;
    }
    cplain += cnt;
  } else if (KIND == K_E2G_P_AWAY) {
    // stokes_pressure_away (E2G/stokes.cpp:108-121)
    for (int j = 0; j < cnt; j++) {
      double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
      double r2 = dx * dx + dy * dy + dz * dz;
      double H2 = 1.0 / (r2 * sqrt(r2));
      H2 *= QX[j] * dx + QY[j] * dy + QZ[j] * dz;
      a0 += H2 * A[j];
    }
    cplain += cnt;
  } else if (KIND == K_E2G_P7) {
    // stokes_pressure_7ord (E2G/stokes.cpp:151-194)
    for (int j = 0; j < cnt; j++) {
      double dx = S.px - X[j], dy = S.py - Y[j], dz = S.pz - Z[j];
      double r2 = dx * dx + dy * dy + dz * dz;
      double r = sqrt(r2);
      double H2 = lapl_dl_7ord(r, DEL, S.c);
      creg += (r2 <= d64);
      double n0 = NX[j], n1 = NY[j], n2 = NZ[j];
      double f0 = QX[j], f1 = QY[j], f2 = QZ[j];
      double f_dot_n = f0 * n0 + f1 * n1 + f2 * n2;
      double ncf0 = (n1 * f2 - n2 * f1) - S.n0xf0[0];
      double ncf1 = (n2 * f0 - n0 * f2) - S.n0xf0[1];
      double ncf2 = (n0 * f1 - n1 * f0) - S.n0xf0[2];
      double n_dot_dx = n0 * dx + n1 * dy + n2 * dz;
      double ncd0 = n1 * dz - n2 * dy;
      double ncd1 = n2 * dx - n0 * dz;
      double ncd2 = n0 * dy - n1 * dx;
      double normal = -(f_dot_n - S.f0n0) * n_dot_dx;
      double tangential = -(ncf0 * ncd0 + ncf1 * ncd1 + ncf2 * ncd2);
      a0 += (normal + tangential) * H2 * A[j];
    }
    cplain += cnt;
  }
}

// Proxy-point (far-field) sum of one staged moment tile.
template <bool DL>
__device__ __forceinline__ void tile_proxies(const double* __restrict__ sm, int PT, int cnt,
                                             int kk0, int P1, const double* __restrict__ cheb,
                                             const Tgt& S, double& a0, double& a1, double& a2) {
  int rem = kk0 % (P1 * P1);
  int pi = kk0 / (P1 * P1), pj = rem / P1, pk = rem % P1;
  for (int i = 0; i < cnt; i++) {
    double dx0 = S.px - cheb[pi];
    double dx1 = S.py - cheb[P1 + pj];
    double dx2 = S.pz - cheb[2 * P1 + pk];
    double r2 = dx0 * dx0 + dx1 * dx1 + dx2 * dx2;
    double r = sqrt(r2);
    if (!DL) {
      // Call_Treecode_SL (2S/KITC.cpp:700-714)
      double m0 = sm[i] - S.f0n0 * sm[3 * PT + i];
      double m1 = sm[PT + i] - S.f0n0 * sm[4 * PT + i];
      double m2 = sm[2 * PT + i] - S.f0n0 * sm[5 * PT + i];
      double temp = (m0 * dx0 + m1 * dx1 + m2 * dx2) / (r2 * r);
      a0 += m0 / r + temp * dx0;
      a1 += m1 / r + temp * dx1;
      a2 += m2 / r + temp * dx2;
    } else {
      // Call_Treecode_DL (2S/KITC.cpp:753-771)
      double M9 = sm[9 * PT + i], M10 = sm[10 * PT + i], M11 = sm[11 * PT + i];
      double tl[3];
#pragma unroll
      for (int l = 0; l < 3; l++) {
        double ta = sm[(3 * l) * PT + i] - S.g0[l] * M9;
        double tb = sm[(3 * l + 1) * PT + i] - S.g0[l] * M10;
        double tc = sm[(3 * l + 2) * PT + i] - S.g0[l] * M11;
        tl[l] = ta * dx0 + tb * dx1 + tc * dx2;
      }
      double kernel = (tl[0] * dx0 + tl[1] * dx1 + tl[2] * dx2) / (r2 * r2 * r);
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

template <int KIND>
__device__ __forceinline__ void run_block(const EvalTask& T, int blk, double* sm, double* cheb) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int k = blk * kTB + tid;
  const bool valid = k < T.nt;
  const int t = valid ? T.tord[k] : 0;
  Tgt S;
  load_target<KIND>(T, t, valid, S);
  const double DEL = T.DEL;
  const double d64 = 64.0 * DEL * DEL;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  unsigned long long creg = 0, cplain = 0, cfar = 0, cprox = 0;
  const int e0 = T.blk_start[blk], e1 = T.blk_start[blk + 1];
  constexpr bool kSrcNrm = !(KIND == K_E2G_SL_AWAY || KIND == K_E2G_P_AWAY);
  for (int e = e0; e < e1; e++) {
    const Entry E = T.entries[e];
    const uint32_t wm = E.mask[warp];
    const bool act = valid && ((wm >> lane) & 1u);
    if (E.type == 1) {
      const int m0 = T.node_m0[E.node], m1 = T.node_m1[E.node];
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
        }
        __syncthreads();
        if (wm != 0u && act) {
          unsigned long long cr = 0, cp = 0;
          tile_pairs<KIND>(sm, cnt, DEL, d64, S, a0, a1, a2, cr, cp);
          if (S.near) {
            creg += cr;
            cplain += cp - cr;
          } else {
            cfar += cp;
          }
        }
      }
    } else if (KIND == K_SL_ON || KIND == K_SL_OFF || KIND == K_DL_ON || KIND == K_DL_OFF) {
      constexpr bool DL = (KIND == K_DL_ON || KIND == K_DL_OFF);
      const int P1 = T.P1, Pf = T.Pf, C = T.C;
      const int PT = (kSmem / C) & ~31;
      __syncthreads();
      if (tid < 3 * P1) cheb[tid] = T.tcheb[(size_t)E.node * 3 * P1 + tid];
      const double* M = T.mom + (size_t)E.node * C * Pf;
      for (int kk0 = 0; kk0 < Pf; kk0 += PT) {
        const int cnt = min(PT, Pf - kk0);
        __syncthreads();
        for (int c = 0; c < C; c++)
          for (int i = tid; i < cnt; i += kTB) sm[c * PT + i] = M[(size_t)c * Pf + kk0 + i];
        __syncthreads();
        if (wm != 0u && act) {
          tile_proxies<DL>(sm, PT, cnt, kk0, P1, cheb, S, a0, a1, a2);
          cprox += cnt;
        }
      }
    }
  }
  // Per-target epilogue.
  if (valid) {
    const double sc = T.scale;
    double* o = T.out;
    if (KIND == K_SL_ON || KIND == K_SL_OFF || KIND == K_E2G_SL_AWAY || KIND == K_E2G_SL7) {
      o[3 * t] = a0 * sc;
      o[3 * t + 1] = a1 * sc;
      o[3 * t + 2] = a2 * sc;
    } else if (KIND == K_DL_ON) {
      // DL[3i+k] = u[k] * EightPI6 + 0.5 * g0[k]   (2S/KITC.cpp:1693, 2S/stresslets.cpp:271-278)
      o[3 * t] = a0 * sc + 0.5 * S.g0[0];
      o[3 * t + 1] = a1 * sc + 0.5 * S.g0[1];
      o[3 * t + 2] = a2 * sc + 0.5 * S.g0[2];
    } else if (KIND == K_DL_OFF) {
      double xi = 0.0;
      if (T.jump_mode == 0) {
        // tree: xi = 1/2 on the surface, 1 inside (2S/KITC.cpp:1805-1815)
        if (fabs(S.b) < 1.0e-12) xi = 0.5;
        else if (S.b < 0.0) xi = 1.0;
      } else {
        // direct: + g0 inside or on the surface, near targets only (2S/stresslets.cpp:174-178)
        if (S.near && ((S.b < 0.0) || (fabs(S.b) < 1.0e-14))) xi = 1.0;
      }
      o[3 * t] = a0 * sc + xi * S.g0[0];
      o[3 * t + 1] = a1 * sc + xi * S.g0[1];
      o[3 * t + 2] = a2 * sc + xi * S.g0[2];
    } else if (KIND == K_E2G_P_AWAY) {
      o[t] = a0 * sc;
    } else if (KIND == K_E2G_P7) {
      // p *= -denom_FourPI; inside: p -= f0.n0 (E2G/stokes.cpp:196-200)
      double p = a0 * sc;
      if (S.b < -1.e-12) p -= S.f0n0;
      o[t] = p;
    }
  }
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

template <int FAM>
__global__ void __launch_bounds__(kTB) eval_kernel(const EvalTask* __restrict__ tasks,
                                                   const BlockRef* __restrict__ blocks) {
  __shared__ double sm[kSmem];
  __shared__ double cheb[3 * kMaxP1];
  __shared__ EvalTask sT;
  const BlockRef br = blocks[blockIdx.x];
  if (threadIdx.x == 0) sT = tasks[br.task];
  __syncthreads();
  const int kind = sT.kind;
  if (FAM == F_SL) {
    if (kind == K_SL_ON) run_block<K_SL_ON>(sT, br.blk, sm, cheb);
    else run_block<K_SL_OFF>(sT, br.blk, sm, cheb);
  } else if (FAM == F_DL) {
    if (kind == K_DL_ON) run_block<K_DL_ON>(sT, br.blk, sm, cheb);
    else run_block<K_DL_OFF>(sT, br.blk, sm, cheb);
  } else {
    switch (kind) {
      case K_E2G_SL_AWAY: run_block<K_E2G_SL_AWAY>(sT, br.blk, sm, cheb); break;
      case K_E2G_P_AWAY: run_block<K_E2G_P_AWAY>(sT, br.blk, sm, cheb); break;
      case K_E2G_SL7: run_block<K_E2G_SL7>(sT, br.blk, sm, cheb); break;
      default: run_block<K_E2G_P7>(sT, br.blk, sm, cheb); break;
    }
  }
}

}  // namespace

void launch_eval(int family, const EvalTask* d_tasks, const BlockRef* d_blocks, int nblocks,
                 cudaStream_t st) {
  if (nblocks <= 0) return;
  if (family == F_SL) eval_kernel<F_SL><<<nblocks, kTB, 0, st>>>(d_tasks, d_blocks);
  else if (family == F_DL) eval_kernel<F_DL><<<nblocks, kTB, 0, st>>>(d_tasks, d_blocks);
  else eval_kernel<F_E2G><<<nblocks, kTB, 0, st>>>(d_tasks, d_blocks);
}

}  // namespace hr
