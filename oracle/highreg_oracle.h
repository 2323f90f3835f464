/*
 * highreg_oracle.h — CPU restatement of the reference's hot path, used ONLY as
 * the oracle by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg. It is never linked into the product library.
 *
 * Conventions (same as the reference): vector fields and points are
 * interleaved xyz arrays (v[3*j+k]); scalar per-point arrays have length n.
 * All arithmetic is FP64 in the reference's operation order.
 */
#ifndef HIGHREG_ORACLE_H
#define HIGHREG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- scalar kernels (2S/utilities.cpp:163-337, E2G/utilities.cpp:174-257) */
void or_reg_coeff(double lam, double c[3]);
void or_sl_7ord(double r, double d, const double c[3], double s[2]);
void or_sl_7ord_onsurf(double r, double d, double s[2]);
void or_dl_7ord(double r, double d, const double c[3], double s[2]);
double or_dl_7ord_onsurf(double r, double d);
double or_lapl_dl_7ord(double r, double d, const double c[3]);

/* ---- direct boundary sums (2S/stokeslets.cpp, 2S/stresslets.cpp) */
void or_sl_offsurf_direct(double DEL, int nq, const double* xq, const double* nq_, const double* aq,
                          const double* f, int nt, const double* xt, const double* b,
                          const double* f0, const double* n0, double* out);
void or_sl_onsurf_direct(double DEL, int nq, const double* xq, const double* nq_, const double* aq,
                         const double* f, double* out);
void or_dl_offsurf_direct(double DEL, int nq, const double* xq, const double* nq_, const double* aq,
                          const double* g, int nt, const double* xt, const double* b,
                          const double* x0, const double* n0, const double* g0, double* out);
void or_dl_onsurf_direct(double DEL, int nq, const double* xq, const double* nq_, const double* aq,
                         const double* g, double* out);

/* ---- extend-to-grid per-target sums (E2G/stokes.cpp) */
void or_e2g_sl_away(int nq, const double* xq, const double* aq, const double* f, int nt,
                    const double* xt, double* out);
double or_e2g_p_away_one(int nq, const double* xq, const double* aq, const double* f, double x,
                         double y, double z);
void or_e2g_p_away(int nq, const double* xq, const double* aq, const double* f, int nt,
                   const double* xt, double* out);
void or_e2g_sl_7ord(double DEL, int nq, const double* xq, const double* nq_, const double* aq,
                    const double* f, int nt, const double* xt, const double* b,
                    const double* f0, const double* n0, double* out);
void or_e2g_p_7ord(double DEL, int nq, const double* xq, const double* nq_, const double* aq,
                   const double* f, int nt, const double* xt, const double* b, const double* f0,
                   const double* n0, double* out);

/* ---- KITC treecode (2S/KITC.cpp). kind: 0 SL on-surface, 1 SL off-surface,
 *      2 DL on-surface, 3 DL off-surface. For on-surface kinds the targets are
 *      the quadrature points themselves (nt == nq, xt == xq).
 *      dens0: SL off -> nearest force f0 (3nt, with n0); DL off -> g0 (3nt).
 *      stats (optional, 4 longs): direct pairs, proxy pairs, far nodes, leaves. */
int or_kitc_eval(int kind, int P, int N0, double theta, const double ctr[3], double DEL, int nq,
                 const double* xq, const double* nq_, const double* aq, const double* dens, int nt,
                 const double* xt, const double* b, const double* x0, const double* n0,
                 const double* dens0, double* out, long* stats);

/* ---- DL density interpolation at nearest points (2S/main.cpp:682-1046).
 *      ctr: centre of the source surface; nrst: reference flag/index (0 = skip). */
void or_interp_dl_density(double h, const double ctr[3], int nq, const double* xq,
                          const double* g, int nt, const int* nrst, const double* x0,
                          const int* i123, double* g0_out);

/* ---- two-surface matvec u_out = u_in - 2/3 DL[u_in] (2S/main.cpp:541-677).
 *      tree = 1 uses the treecode with (P, N0, theta), 0 the direct sums. */
typedef struct {
  int nq[2];
  const double* xq[2];
  const double* nrm[2];
  const double* area[2];
  double ctr[2][3];
  /* target set t = quadrature points of surface t, nearest data w.r.t. surface 1-t */
  const double* b[2];
  const double* x0[2];
  const double* n0[2];
  const int* nrst[2];
  const int* i123[2];
  const double* f0[2]; /* nearest force (SL right-hand side) */
  double h, DEL;
  int tree, P, N0;
  double theta;
} or_scene2s;

void or_matvec_2s(const or_scene2s* sc, const double* u_in, double* u_out);
/* b = -(2/3) SL[f] (2S/main.cpp:186-207, 421-537); f[s] = force on surface s */
void or_rhs_2s(const or_scene2s* sc, const double* f1, const double* f2, double* bvec);
/* GMRES(im) with modified Gram-Schmidt + Givens as in 2S/main.cpp:236-416,
 * but with the true restart residual r0 = b - A x0 and x accumulated across
 * cycles. x: in = initial guess, out = solution. Returns iterations. */
int or_gmres_2s(const or_scene2s* sc, const double* bvec, double* x, int im, int iter_max,
                double tol, double* resid_hist);

/* ---- extend-to-grid Poisson path (E2G/main.cpp:969-1044, 1423-1823).
 *      Grids are row-major (N+1)^3; rhs / DST arrays row-major (N-1)^3. */
void or_extend_into_cube(int N, double L, double h, const double* g, double* G);
void or_lapl_4ord_incube(int N, const double* G, double* rhs);
void or_lapl_4ord_band2(int N, const unsigned char* band2_mask, const double* u, double* rhs);
void or_dp_4ord(int N, double h, int axis, const unsigned char* outside_band2_mask,
                const double* p, double* rhs);
void or_dst1_3d(int n, double* a); /* unnormalised DST-I (FFTW RODFT00) on each axis */
void or_dst_poisson(int n, double* f);
void or_solve_poisson(int N, double L, double h, const unsigned char* band2_mask,
                      const unsigned char* outside_band2_mask, const double* p, double* u,
                      int variable);

#ifdef __cplusplus
}
#endif
#endif
