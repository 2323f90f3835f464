/*
 * highreg_b200.h — C ABI of the B200 (sm_100a) implementation of the
 * regularized Stokeslet / stresslet boundary sums of Beale & Tlupova's
 * high-order regularization (reference: stlupova/high-order-regularization).
 *
 * Plain pointers and sizes only. Unless an entry point says otherwise,
 * pointers are HOST pointers, arrays of points / vector fields are
 * interleaved xyz (v[3*j+k], as the reference's f[3*j+k]), results are
 * written into caller-owned buffers, and every call is synchronous at return.
 * Every function returns HR_OK (0) or a nonzero status; hr_last_error() gives
 * the message. A context is not thread-safe; use one context per thread.
 *
 * Reference citations are file:line within the reference project
 * (2S = highreg_stokes_2surf, E2G = highreg_stokes_extend_to_grid).
 */
#ifndef HIGHREG_B200_H
#define HIGHREG_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HR_OK 0
#define HR_ERR_ARG 1           /* bad argument (size, null pointer, unsupported option) */
#define HR_ERR_CUDA 2          /* CUDA / cuFFT runtime failure */
#define HR_ERR_NAN 3           /* non-finite value detected in an input or output */
#define HR_ERR_NOT_CONVERGED 4 /* GMRES hit its iteration cap or stagnated */
#define HR_ERR_NO_DEVICE 5     /* no usable sm_100 device */
#define HR_ERR_STATE 6         /* object used in the wrong state */

/* evaluation mode and precision */
#define HR_DIRECT 0 /* all-pairs sums: eval_Stokes_*_{on,off}Surf (2S/stokeslets.cpp, 2S/stresslets.cpp) */
#define HR_TREE 1   /* KITC treecode: eval_Stokes_*_tree (2S/KITC.cpp:1389-1830) */
#define HR_FP64 0   /* all pairs in FP64 */
#define HR_MIXED 1  /* pairs with r > 3 delta and proxy interactions in FP32, FP64 per-target accumulation */
#define HR_FP32 2   /* every pair in FP32 (the r < 1e-14 limits excepted), FP64 per-target accumulation */

typedef struct hr_ctx hr_ctx;

/* A quadrature surface: grid-line-intersection points with partition-of-unity
 * area weights (the reference's vector<Surf_point>, 2S/utilities.h:30-39),
 * as host SoA arrays in the reference's order. */
typedef struct {
  int n;
  const double* xyz;    /* 3n points */
  const double* nrml;   /* 3n unit normals */
  const double* area;   /* n area elements h^2 sigma_i(n)/|n_i| */
  const int* plane;     /* n grid-line family of each point (0,1,2), may be NULL */
  double center[3];     /* surface centre: the treecode root box is centre + [-1,1]^3 */
} hr_surface;

/* Target points with their nearest-surface data (the reference's
 * vector<Target_point>, 2S/utilities.h:41-53). For on-surface sums the
 * targets are the surface's own points and only xyz is read. */
typedef struct {
  int n;
  const double* xyz;  /* 3n target points */
  const double* b;    /* n signed distance to the source surface */
  const double* x0;   /* 3n nearest surface point */
  const double* n0;   /* 3n unit normal at x0 */
  const int* nrst;    /* n reference flag: 0 = no subtraction / no interpolation
                         (|b|/delta > 8), else the nearest quadrature index */
  const int* i123;    /* 3n Monge-patch indices (ind1, ind2, ind3) of each target */
} hr_targets;

typedef struct {
  int mode;      /* HR_DIRECT or HR_TREE */
  int P;         /* treecode interpolation degree (2S/KITC.h:14) */
  int N0;        /* treecode leaf size (2S/KITC.h:16) */
  double theta;  /* treecode MAC parameter, sq_theta = theta^2 (2S/KITC.h:17) */
  int precision; /* HR_FP64, HR_MIXED or HR_FP32 */
} hr_eval_opts;

/* ---------------------------------------------------------------- context */
int hr_ctx_create(int device, hr_ctx** out);
void hr_ctx_destroy(hr_ctx* ctx);
const char* hr_last_error(const hr_ctx* ctx);
/* number of kernel launches issued by this context so far */
long long hr_ctx_launch_count(const hr_ctx* ctx);

/* ------------------------------------------------- boundary sums (drop-in) */
/* eval_Stokes_SL_onSurf[_tree]: 2S/stokeslets.cpp:141-180, 2S/KITC.cpp:1389-1492.
 * f: 3n density on S; out: 3n Stokeslet sum at S's own points. */
int hr_stokes_sl_onsurf(hr_ctx* ctx, const hr_eval_opts* opt, double delta, const hr_surface* S,
                        const double* f, double* out);
/* eval_Stokes_SL_offSurf[_tree]: 2S/stokeslets.cpp:12-86, 2S/KITC.cpp:1496-1602.
 * f0: 3nt force at each target's nearest point (Target_point::nrst_f). */
int hr_stokes_sl_offsurf(hr_ctx* ctx, const hr_eval_opts* opt, double delta, const hr_surface* S,
                         const double* f, const hr_targets* T, const double* f0, double* out);
/* eval_Stokes_DL_onSurf[_tree]: 2S/stresslets.cpp:186-228, 2S/KITC.cpp:1606-1709. */
int hr_stokes_dl_onsurf(hr_ctx* ctx, const hr_eval_opts* opt, double delta, const hr_surface* S,
                        const double* g, double* out);
/* eval_Stokes_DL_offSurf[_tree]: 2S/stresslets.cpp:13-96, 2S/KITC.cpp:1712-1830.
 * g0: 3nt density at the nearest points (Target_point::nrst_g). The jump term
 * follows the mode's reference: tree adds g0/2 on the surface and g0 inside,
 * direct adds g0 inside or when |b| < 1e-14. */
int hr_stokes_dl_offsurf(hr_ctx* ctx, const hr_eval_opts* opt, double delta, const hr_surface* S,
                         const double* g, const hr_targets* T, const double* g0, double* out);

/* interpolate_DL_density: 2S/main.cpp:916-1046. Six-point tensor Lagrange
 * interpolation of g at each target's nearest point x0, on the grid lines of
 * the Monge plane (i123) of the source surface with spacing h.
 * S->center is the source surface centre; S->plane is required. */
int hr_interpolate_dl_density(hr_ctx* ctx, double h, const hr_surface* S, const double* g,
                              const hr_targets* T, double* g0);

/* ------------------------------------------------ extend-to-grid (E2G) sums */
/* stokes_SL_away: E2G/stokes.cpp:13-45 (plain Stokeslet, nt targets xyz). */
int hr_e2g_stokeslet_away(hr_ctx* ctx, const hr_surface* S, const double* f, int nt,
                          const double* xyz, double* out3);
/* stokes_pressure_away: E2G/stokes.cpp:102-126. */
int hr_e2g_pressure_away(hr_ctx* ctx, const hr_surface* S, const double* f, int nt,
                         const double* xyz, double* out1);
/* stokes_SL_7ord at band targets: E2G/stokes.cpp:53-97 with f0 = the exact
 * density at x0 (E2G/main.cpp:1330-1345). f0: 3nt. */
int hr_e2g_stokeslet_7ord(hr_ctx* ctx, double delta, const hr_surface* S, const double* f,
                          const hr_targets* T, const double* f0, double* out3);
/* stokes_pressure_7ord: E2G/stokes.cpp:134-203. */
int hr_e2g_pressure_7ord(hr_ctx* ctx, double delta, const hr_surface* S, const double* f,
                         const hr_targets* T, const double* f0, double* out1);

/* fftw_DST_Poisson3d_FD: E2G/main.cpp:1423-1489. In place on a row-major
 * n^3 host array: DST-I, divide by the eigenvalues of the 4th-order compact
 * Laplacian, DST-I, scale 1/(2(n+1))^3. */
int hr_dst_poisson3d(hr_ctx* ctx, int n, double* f);
/* A plain 3D DST-I, FFTW's RODFT00 on all three axes, unnormalised
 * (Y = 2 sum X_j sin(pi (j+1)(k+1)/(n+1)) per axis), of a row-major n^3 host
 * array: what fftw_plan_r2r_3d(n, n, n, in, out, FFTW_RODFT00 x3, ...) +
 * fftw_execute compute in E2G/main.cpp:1429-1471. The plan keeps its device
 * tables and buffers; each execute copies in, runs three fused DST passes and
 * copies out (in == out allowed). n + 1 must be even (the grids' N = n + 1). */
typedef struct hr_dst1_plan hr_dst1_plan;
int hr_dst1_plan_create(hr_ctx* ctx, int n, hr_dst1_plan** out);
int hr_dst1_execute(hr_dst1_plan* p, const double* in, double* out);
void hr_dst1_plan_destroy(hr_dst1_plan* p);
/* Page-locked host memory (cudaHostAlloc / cudaFreeHost), for callers that
 * stage arrays to the library without linking the CUDA runtime themselves
 * (the FFTW-API layer's fftw_malloc / fftw_free). */
int hr_host_alloc(size_t bytes, void** out);
void hr_host_free(void* p);

/* solve_Poisson: E2G/main.cpp:969-1044. Grids are row-major (N+1)^3.
 * band2: 1 at BAND2 points; outside: 1 at exterior points outside BAND2
 * (phi > 0 and not in BAND2). u is in/out; p is read when variable = 1..3. */
int hr_e2g_solve_poisson(hr_ctx* ctx, int N, double L, const uint8_t* band2,
                         const uint8_t* outside, const double* p, double* u, int variable);

/* ---------------------------------------------- extend-to-grid pipeline */
/* The whole extend-to-grid computation of test_Stokes_Poisson3d_FD
 * (E2G/main.cpp:107-424) for the translating prolate spheroid on [0, 3]^3,
 * h = 3/N: host setup (Generate_Surface, find_nrst_surfc with BAND1 = 4,
 * BAND2 = 2, exact density) at create time; on the device, the face and band
 * pressure / velocity sums in one batched launch, then the four Poisson
 * extensions (p, then u with the extended p). N must be even and >= 36. */
typedef struct hr_e2g hr_e2g;
typedef struct {
  int N;
  double L, h, delta;
  int nq;        /* quadrature points */
  int n_tagged;  /* grid points within BAND1 of the surface */
  int n_band;    /* tagged interior points outside or on the surface (evaluated) */
  int n_face;    /* box-face grid points */
  long long pairs;
} hr_e2g_info;
typedef struct {
  double seconds_sums;     /* the four boundary sums */
  double seconds_poisson;  /* the four Poisson extensions */
  double seconds_total;
  long long pairs;
} hr_e2g_report;
int hr_e2g_create(hr_ctx* ctx, int N, hr_e2g** out);
int hr_e2g_get_info(const hr_e2g* e, hr_e2g_info* info);
int hr_e2g_run(hr_e2g* e, int precision, hr_e2g_report* rep);
/* which: 0 p after the sums, 1 u after the sums (3 grids), 2 extended p,
 * 3 extended u (3 grids); grids row-major (N+1)^3 */
int hr_e2g_get(hr_e2g* e, int which, double* out);
/* which: 0 quadrature (3nq xyz, 3nq nrml, nq area, 3nq f), 1 nrst grid (int,
 * (N+1)^3), 2 tagged targets (b, 3 x0, 3 n0, band2) as doubles */
int hr_e2g_scene(const hr_e2g* e, int which, void* out);
void hr_e2g_destroy(hr_e2g* e);
/* Error norms of the last hr_e2g_run, computed on the device: extended p and
 * u against the exact solution over the whole grid (exact outside or on the
 * surface, p = 0 and u = (1, 0, 0) inside; the reference's tables,
 * E2G/main.cpp:236-259, 470-497), the band velocity after the sums against
 * the exact solution (E2G/main.cpp:1359-1405), and, after hr_e2g_snapshot,
 * the extended grids against the snapshot: max |x - ref| / max |ref| and
 * ||x - ref||_2 / ||ref||_2 (-1 without a snapshot). u errors use |u| (the
 * Euclidean norm of the vector at a point). */
typedef struct {
  double p_max, p_rms, u_max, u_rms;
  double band_u_max, band_u_rms;
  double ref_p_max_rel, ref_p_rel_l2, ref_u_max_rel, ref_u_rel_l2;
} hr_e2g_errors;
/* keeps the current extended p and u grids (device copies) as the comparison reference */
int hr_e2g_snapshot(hr_e2g* e);
int hr_e2g_error_norms(hr_e2g* e, hr_e2g_errors* out);
/* exact translating-spheroid solution (E2G/utilities.cpp:294-411) */
double hr_e2g_p_exact(double x, double y, double z);
void hr_e2g_u_exact(double x, double y, double z, double* u);

/* --------------------------------------------------- two-surface problem */
/* The two-surface boundary integral equation (I - 2/3 D) u = b
 * (2S/main.cpp:140-417). Target set s is the quadrature points of surface s
 * with nearest data relative to the OTHER surface. */
typedef struct {
  hr_surface surf[2];
  hr_targets tgt[2];
  const double* f0[2]; /* 3n force at each target's nearest point (for the RHS) */
  double h;            /* grid spacing */
  double delta;        /* regularization length */
} hr_scene2s;

typedef struct {
  int restart;         /* GMRES restart length (reference: 15, 2S/main.cpp:213) */
  int max_iter;        /* iteration cap (reference: 100) */
  double tol;          /* relative residual tolerance (reference: 1e-10) */
  int precision;       /* HR_FP64, or HR_MIXED / HR_FP32: reduced-precision matvecs (below) */
  int use_guess;       /* 1: x holds an initial guess on input */
  int true_residual;   /* 1: check ||b - A x|| / ||b|| with an FP64 matvec at the end */
  /* HR_MIXED / HR_FP32 solve by iterative refinement: every Krylov matvec
   * in the reduced precision, each GMRES cycle run until its residual falls
   * by 10 x mixed_accuracy (or below tol / 2), then the FP64 true residual
   * b - A x starts the next cycle; the solve ends when that FP64 residual
   * meets tol. mixed_accuracy: relative accuracy of a reduced-precision
   * matvec (0 = 3e-7 for HR_MIXED, whose measured max-norm relative error
   * is 2.7e-7, and 1e-6 for HR_FP32; with an inner treecode,
   * hr_plan2s_set_inner_tree, at least its measured accuracy). With
   * use_guess, the guess's first residual comes from the reduced-precision
   * operator, and a guess that already meets tol is confirmed in FP64. */
  double mixed_accuracy;
} hr_gmres_opts;

typedef struct {
  int iterations;
  int restarts;
  int matvecs_fp64;
  int matvecs_mixed;
  double residual;       /* final Arnoldi relative residual */
  double true_residual;  /* FP64 ||b - A x|| / ||b|| (if requested, else -1) */
  double seconds;        /* device time of the solve */
  int guess_rejected;    /* 1 if the initial guess was worse than zero and was dropped */
  double resid_hist[512];
} hr_gmres_report;

typedef struct hr_plan2s hr_plan2s;

/* Uploads the scene, builds both treecodes, interaction lists and density
 * interpolation stencils. Geometry-only work: done once per scene. */
int hr_plan2s_create(hr_ctx* ctx, const hr_scene2s* scene, const hr_eval_opts* opt,
                     hr_plan2s** out);
void hr_plan2s_destroy(hr_plan2s* plan);
/* y = (I - 2/3 D) x (2S/main.cpp:541-677); host buffers of 3(n1+n2). */
int hr_plan2s_matvec(hr_plan2s* plan, const double* x, double* y);
/* b = -2/3 S[f] (2S/main.cpp:186-207, 421-537); f1, f2 host 3n_s forces. */
int hr_plan2s_rhs(hr_plan2s* plan, const double* f1, const double* f2, double* b);
/* GMRES solve; x in/out (host). */
int hr_plan2s_solve(hr_plan2s* plan, const hr_gmres_opts* opt, const double* b, double* x,
                    hr_gmres_report* rep);
/* Device-pointer variants (buffers already in HBM, on the context's stream). */
int hr_plan2s_matvec_dev(hr_plan2s* plan, const double* x_dev, double* y_dev, int precision);
int hr_plan2s_rhs_dev(hr_plan2s* plan, const double* f1_dev, const double* f2_dev, double* b_dev);
int hr_plan2s_solve_dev(hr_plan2s* plan, const hr_gmres_opts* opt, const double* b_dev,
                        double* x_dev, hr_gmres_report* rep);
/* Work counts of one matvec: pair evaluations (direct + proxy), by kind. */
typedef struct {
  long long direct_pairs_near; /* regularized (r <= 8 delta candidates) target x source pairs */
  long long direct_pairs_far;  /* plain-kernel target x source pairs (far targets) */
  long long proxy_pairs;       /* target x proxy-point evaluations */
  long long moment_terms;      /* proxy x source terms of the upward pass */
  long long flops;             /* algorithmic flops by the fixed per-pair convention */
} hr_work;
/* which 2: the inner treecode's stresslet batch (hr_plan2s_set_inner_tree),
 * counted from its interaction lists without a launch: direct pairs of
 * regularized-branch targets in direct_pairs_near, of the others in
 * direct_pairs_far; flops is 0. */
int hr_plan2s_work(hr_plan2s* plan, int which /*0 matvec, 1 rhs, 2 inner*/, hr_work* w);
/* Self-check of the reduced-precision upward pass: for density x (host, n),
 * the proxy moments of both trees from the tensor-core 3xTF32 kernel against
 * the FP64 ones; max over nodes and channels of max |difference| / max |FP64
 * moment|. HR_TREE plans only. */
int hr_plan2s_check_upward_pass(hr_plan2s* plan, const double* x, double* max_rel_err);
/* Gives the reduced-precision inner operator of GMRES-IR (HR_MIXED and
 * HR_FP32 solves) a treecode of its own: KITC with degree P, leaf size N0 and
 * MAC theta over the same surfaces, targets and density stencils. The inner
 * Krylov cycles then apply this cheaper operator, while every FP64 true
 * residual, and with it the stopping test, still applies the plan's own
 * treecode: the converged answer meets the same residual tolerance. The
 * inner operator's relative L2 error against the plan's FP64 one, on a fixed
 * pseudo-random density, is measured here (written to *rel_err if not NULL)
 * and is the default mixed_accuracy of later solves. P = 0 removes it.
 * HR_TREE plans only. */
int hr_plan2s_set_inner_tree(hr_plan2s* plan, int P, int N0, double theta, double* rel_err);
/* the plan's stream (cudaStream_t) for callers that enqueue their own work */
void* hr_plan2s_stream(hr_plan2s* plan);
/* Times `iters` back-to-back launches of one boundary-sum batch with CUDA
 * events on the plan's stream (inputs as left by the last matvec / RHS):
 * which 0 = stresslet batch (matvec, FP64), 1 = Stokeslet batch (RHS),
 * 2 = stresslet batch (mixed precision), 3 = the inner treecode's mixed
 * stresslet batch. Returns milliseconds per launch. */
int hr_plan2s_time_batch(hr_plan2s* plan, int which, int iters, double* ms_per_launch);

/* ------------------------------------------- two-surface geometry setup */
/* Host setup producing an hr_scene2s: Generate_Surface (2S/surface.cpp:13-71),
 * Compute_nearest_data (2S/surface.cpp:450-526) and surfc_force
 * (2S/surface.cpp:530-559), parameterized. Default parameters reproduce the
 * reference's scene (2S/utilities.h:15-26, 2S/utilities.cpp:10-40,
 * 2S/main.cpp:147-157) bit for bit. */
typedef struct {
  double axes[3];       /* spheroid semi-axes (ellipse_a, ellipse_b, ellipse_c) */
  double center[2][3];  /* centres of surfaces 1 and 2 */
  double unrot[2][9];   /* row-major "un-rotation" R: body coordinates = R (x - centre) */
  int rotated[2];       /* 1: the level set uses unrot (the reference's rotated flag) */
  double kappa0, q;     /* delta = kappa0 (1/64)^(1-q) h^q */
  int tension_body;     /* surface tension gamma = 1 + z^2: 0 = z - centre_z (the reference),
                           1 = the body-frame z of unrot (the same for an unrotated surface or
                           a rotation about z, as in the reference's scene) */
} hr_geom2s_params;

typedef struct hr_geom2s hr_geom2s;
int hr_geom2s_default_params(hr_geom2s_params* p);
/* h = 1/N on the box [-1, 1]^3 around each centre */
int hr_geom2s_generate(const hr_geom2s_params* p, int N, hr_geom2s** out);
/* Borrowed views (valid until destroy): the scene and the interfacial force
 * f = 2 H gamma n - grad_s gamma, gamma = 1 + z^2, at every quadrature point. */
int hr_geom2s_view(const hr_geom2s* g, hr_scene2s* scene, const double** force);
void hr_geom2s_destroy(hr_geom2s* g);
/* Wall seconds of the set-up phases of hr_geom2s_generate: [0] quadrature
 * points of both surfaces, [1] interfacial forces, [2] / [3] nearest data
 * (nearest-point search, Newton projection, Monge patch, forces at the
 * nearest points) of target sets 0 / 1. */
int hr_geom2s_phase_seconds(const hr_geom2s* g, double* out4);

/* ------------------------------------------------- learned warm start */
/* No counterpart in the reference (its GMRES starts from zero,
 * 2S/main.cpp:1067-1075). A pointwise MLP maps local geometry to an initial
 * guess for the two-surface solve; hr_plan2s_solve with use_guess = 1 takes
 * it and falls back to the zero guess when ||b - A x0|| > ||b||, so the
 * converged answer is the zero-guess method's. */

/* Seeded two-surface instance: the reference's spheroid (axes 1, .5, .5) at
 * the origin, a second one rotated by a uniform random rotation (Shoemake
 * quaternion) and offset along a uniform random direction so that the solids
 * are `gap` apart, gap uniform in [0.02, 0.3] x 2 (the major diameter), and a
 * background rigid motion u(x) = U + Omega x (x - xmid) with |U| = |Omega| = 1.
 * Instance `index` is the index-th draw of std::mt19937_64(seed). The
 * right-hand side of an instance is hr_plan2s_rhs(force) + 2/3 u: rigid
 * motions satisfy (I - 2/3 D) u = 2/3 u, so its solution is u plus the
 * response to the interfacial force. */
typedef struct {
  hr_geom2s_params geom; /* for hr_geom2s_generate */
  double U[3], Omega[3], xmid[3];
  double gap;            /* distance between the two solids */
} hr_warm_instance;
int hr_warm_instance_make(unsigned long long seed, int index, hr_warm_instance* out);
/* u(x) at n points (3 doubles each). */
int hr_warm_imposed_velocity(const hr_warm_instance* w, const double* xyz, int n, double* u);

#define HR_WARM_NFEAT 12
/* Features of every quadrature point, surface 0 then surface 1 (the GMRES
 * vector's order), 12 floats each: unit normal (3), principal curvatures
 * k1 >= k2 (2), distance to the other solid (1), unit direction to its nearest
 * point (3), imposed velocity u(x) (3). Vectors are in the body frame of the
 * point's own surface (v_body = R v, R = geom.unrot of that surface, or the
 * identity when it is not rotated). u_imposed (optional): u(x) in FP64, world
 * frame, 3 per point. */
int hr_warm_features(const hr_scene2s* scene, const hr_warm_instance* w, float* feat, double* u_imposed);
/* The two body frames (18 doubles: R of surface 0, R of surface 1, row-major,
 * v_body = R v_world) for hr_mlp_infer_frames. */
int hr_warm_frames(const hr_warm_instance* w, double* rot);

/* The network 12 -> 64 -> 64 -> 64 -> 3 (SiLU, FP32), trained and applied
 * on the device. Parameters: W1[12][64] b1[64] W2[64][64] b2[64] W3[64][64]
 * b3[64] W4[64][3] b4[3] (9347 floats), W[i][j] = input i to output j. */
typedef struct hr_mlp hr_mlp;
int hr_mlp_nparams(void);
/* Glorot-uniform weights from `seed`, zero biases, identity normalization. */
int hr_mlp_create(hr_ctx* ctx, unsigned long long seed, hr_mlp** out);
void hr_mlp_destroy(hr_mlp* m);
/* Input normalization x' = (x - mean) / std (12 each) and output scale. */
int hr_mlp_set_normalization(hr_mlp* m, const float* mean, const float* stdv, float out_scale);
int hr_mlp_get_params(hr_mlp* m, float* host);
/* Also resets the Adam moments and step count. */
int hr_mlp_set_params(hr_mlp* m, const float* host);
/* One Adam step (lr, beta 0.9 / 0.999, eps 1e-8) on the mean squared error
 * of MLP(X) against T / out_scale over a batch of `batch` samples of the
 * device arrays X (n x 12) and T (n x 3): random = 1 draws the batch by a
 * hash of (seed, step, slot), random = 0 takes samples 0..batch-1. lr = 0
 * computes the gradient only. loss (optional): the batch's mean loss. */
int hr_mlp_train_step(hr_mlp* m, const float* X_dev, const float* T_dev, long n, int batch, int random,
                      unsigned long long seed, float lr, double* loss);
/* Gradient of the mean loss over samples 0..batch-1, to the host. */
int hr_mlp_gradient(hr_mlp* m, const float* X_dev, const float* T_dev, int batch, float* grad_host,
                    double* loss);
/* out[s] = base[s] + out_scale * MLP(X[s]) (FP64, 3 per sample; base may be
 * NULL); raw (optional, FP32): the network output before scaling. */
int hr_mlp_infer(hr_mlp* m, const float* X_dev, long n, const double* base_dev, double* out_dev,
                 float* raw_dev);
/* The same with the output in body frames: samples frame_start[f] ..
 * frame_start[f+1]-1 (host array, nframes + 1 entries, nframes <= 8) use
 * rot[9 f ..] (host, row-major, v_body = R v_world) and get
 * out[s] = base[s] + out_scale * R^T MLP(X[s]). */
int hr_mlp_infer_frames(hr_mlp* m, const float* X_dev, long n, const double* base_dev, double* out_dev,
                        int nframes, const long* frame_start, const double* rot);
/* Weights file: "HRMLP001", layer widths (5 int32), 12 means, 12 stds,
 * out_scale, 9347 FP32 parameters, FNV-1a 64-bit checksum of the rest. A
 * file with another header, shape or checksum is rejected (HR_ERR_ARG). */
int hr_mlp_save(hr_mlp* m, const char* path);
int hr_mlp_load(hr_mlp* m, const char* path);

/* -------------------------------------------------- measured FP64 peak */
/* Runs an FP64 FMA throughput loop on the device; returns FLOP/s. */
int hr_measure_fp64_peak(hr_ctx* ctx, double* flops_per_s);
/* The same with FP32 FMAs (16 independent chains per thread). */
int hr_measure_fp32_peak(hr_ctx* ctx, double* flops_per_s);

/* -------------------------------------- allocation-free Stokeslet sum */
/* No counterpart in the reference. The plain Stokeslet sum of
 * hr_e2g_stokeslet_away (all pairs, scaled by 1/(8 pi)) on caller-owned
 * DEVICE buffers, with no device allocation and no context: for callers that
 * cannot call cudaMalloc (a memory pool or framework allocator owns the
 * device, or the path must not synchronize the device as cudaMalloc/cudaFree
 * may). Its only scratch, 3 doubles per (target, source chunk), is a
 * file-scope __device__ array of 4 Mi doubles (32 MiB per device), so nt is
 * limited to hr_stokeslet_away_noalloc_max_targets() = 1,398,101; larger nt
 * returns HR_ERR_ARG. The first call on a device (that device current) looks
 * the array up once; make it before any stream capture. All calls share the
 * array and leave their partial sums in it; every slot read is written
 * first, so nothing needs clearing, but calls that overlap on the GPU race.
 * The looked-up address belongs to the device's primary context: do not call
 * this again after cudaDeviceReset on that device. Launch errors are reported
 * with cudaPeekAtLastError (the thread's last error is left as it is). nq
 * above 715,827,882 returns HR_ERR_ARG (int source indices).
 * Enqueued on `stream` (a cudaStream_t, NULL = legacy default stream). */
int hr_stokeslet_away_noalloc(const double* xyz_src_dev, const double* area_dev, const double* f_dev, int nq,
                              const double* xyz_tgt_dev, int nt, double* out_dev, void* stream);
long long hr_stokeslet_away_noalloc_max_targets(void);

/* ------------------------------------------------------------ output */
/* Writes a float64 array as a NumPy .npy file (version 1.0, little-endian, C
 * order), the binary form of the reference's text dumps (vel1 / vel2,
 * 2S/main.cpp:258-270; mid-plane slices, E2G/main.cpp:115-118). */
int hr_write_npy(const char* path, const double* data, int ndim, const long long* shape);
/* Mid-plane y = 1.5 (j = N/2) slices of the last hr_e2g_run, gathered on the
 * device (the reference's p_midY / err_p_midY / err_u_midY files,
 * E2G/main.cpp:297-300, 546): out holds 4 x (N+1)^2 doubles in (i, k) order:
 * extended p; |p - p_exact| outside or on the surface (0 inside); |u -
 * u_exact| likewise; p_exact likewise. */
int hr_e2g_midplane(hr_e2g* e, double* out);

#ifdef __cplusplus
}
#endif
#endif
