// hr_capi.cu — the C ABI (include/highreg_b200.h): context, drop-in boundary
// sums, density interpolation, the two-surface plan (matvec, RHS, GMRES) and
// the FP64 peak measurement.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <exception>
#include <random>
#include <thread>
#include <vector>

#include <omp.h>

#include "hr_runtime.h"

using namespace hr;

namespace hr {
// implemented in hr_poisson.cu
void dst_poisson3d_dev(Ctx& C, int n, double* f_dev);
struct Dst1Plan;
Dst1Plan* dst1_plan_create(Ctx& C, int n);
void dst1_plan_destroy(Dst1Plan* D);
void dst1_execute(Ctx& C, Dst1Plan* D, const double* in_host, double* out_host);

}  // namespace hr

namespace {

constexpr double kPI = 3.14159265358979323846;
// 1/(8 pi): EightPI (2S/KITC.cpp:1395) and denom_EightPI (2S/utilities.h:11)
inline double sl_scale() { return 1.0 / (8.0 * kPI); }
// -6/(8 pi) as the tree drivers write it (2S/KITC.cpp:1612, 1718)
inline double dl_scale_tree() { return -6.0 / (8.0 * kPI); }
// -6 * denom_EightPI as the direct sums write it (2S/stresslets.cpp:66, 170, 271)
inline double dl_scale_direct() { return -6.0 * (1.0 / (8.0 * kPI)); }
// 1/(4 pi) (E2G/utilities.h:9)
inline double p_scale() { return 1.0 / (4.0 * kPI); }

template <class F>
int guard(hr_ctx* ctx, F&& f) {
  try {
    f();
    return HR_OK;
  } catch (const hr::Error& e) {
    if (ctx) ctx->c.err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    if (ctx) ctx->c.err = e.what();
    return HR_ERR_CUDA;
  }
}

void check_opts(const hr_eval_opts* o) {
  HR_REQUIRE(o, "options missing");
  HR_REQUIRE(o->mode == HR_DIRECT || o->mode == HR_TREE, "mode must be HR_DIRECT or HR_TREE");
  HR_REQUIRE(o->precision == HR_FP64 || o->precision == HR_MIXED || o->precision == HR_FP32, "unknown precision");
  if (o->mode == HR_TREE) {
    HR_REQUIRE(o->P >= 1 && o->P <= 15, "P must be in [1, 15]");
    HR_REQUIRE(o->N0 >= 1, "N0 must be >= 1");
    HR_REQUIRE(o->theta > 0.0, "theta must be > 0");
  }
}

void check_finite(const double* a, size_t n, const char* what) {
  for (size_t i = 0; i < n; i++)
    if (!std::isfinite(a[i])) throw hr::Error(HR_ERR_NAN, std::string("non-finite value in ") + what);
}

// Monge-patch axes (ind1, ind2, ind3) of every interpolating target must be
// coordinate indices 0..2.
void check_i123(int n, const int* nrst, const int* i123) {
  for (int i = 0; i < n; i++)
    if (nrst[i] != 0)
      for (int k = 0; k < 3; k++)
        if (i123[3 * i + k] < 0 || i123[3 * i + k] > 2)
          throw hr::Error(HR_ERR_ARG, "i123 entries must be 0, 1 or 2");
}

// near = the regularized branch: |b| / delta <= 8 (2S/KITC.cpp:856, 970; 2S/stokeslets.cpp:40)
std::vector<uint8_t> near_flags(int n, const double* b, double delta) {
  std::vector<uint8_t> v(n, 1);
  if (b)
    for (int i = 0; i < n; i++) v[i] = (fabs(b[i]) / delta > 8.0) ? 0 : 1;
  return v;
}

void upload_targets(DevTargets& tg, int n, const double* xyz, const double* b, const double* x0,
                    const double* n0, const double* f0, const double* nrm,
                    const std::vector<uint8_t>& near, cudaStream_t st) {
  tg.n = n;
  tg.xyz.upload(xyz, 3 * (size_t)n, st);
  if (b) tg.b.upload(b, n, st);
  else {
    tg.b.alloc(n);
    tg.b.zero(st);
  }
  if (x0) tg.x0.upload(x0, 3 * (size_t)n, st);
  else {
    tg.x0.alloc(3 * (size_t)n);
    tg.x0.zero(st);
  }
  if (n0) tg.n0.upload(n0, 3 * (size_t)n, st);
  else {
    tg.n0.alloc(3 * (size_t)n);
    tg.n0.zero(st);
  }
  if (f0) tg.f0.upload(f0, 3 * (size_t)n, st);
  else {
    tg.f0.alloc(3 * (size_t)n);
    tg.f0.zero(st);
  }
  tg.g0.alloc(3 * (size_t)n);
  tg.g0.zero(st);
  if (nrm) tg.nrm.upload(nrm, 3 * (size_t)n, st);
  else {
    tg.nrm.alloc(3 * (size_t)n);
    tg.nrm.zero(st);
  }
  tg.near.upload(near, st);
}

// Flop convention per evaluated pair (counts of the cited reference lines).
struct Flops {
  double reg, near_plain, far_target, proxy;
};
Flops flops_of(int kind) {
  switch (kind) {
    case K_SL_ON: return {57, 37, 37, 29};
    case K_SL_OFF: return {59, 37, 31, 29};
    case K_DL_ON: return {50, 35, 35, 50};
    case K_DL_OFF: return {129, 103, 31, 50};
    case K_E2G_SL_AWAY: return {31, 31, 31, 0};
    case K_E2G_P_AWAY: return {18, 18, 18, 0};
    case K_E2G_UP_AWAY: return {24.5, 24.5, 24.5, 0};  // per counted pair: each fused pair counts twice
    case K_E2G_UP7: return {61.5, 42, 42, 0};
    case K_E2G_SL7: return {59, 37, 37, 0};
    default: return {64, 47, 47, 0};
  }
}

// One self-contained boundary sum (the stateless drop-in entry points).
void single_eval(Ctx& C, int kind, const hr_eval_opts* opt, double delta, const hr_surface* S,
                 const double* dens, int nt, const double* txyz, const double* b,
                 const double* x0, const double* n0, const double* dens0, double* out, int odim) {
  cudaStream_t st = C.stream;
  HR_REQUIRE(S && S->n >= 0, "surface missing");
  HR_REQUIRE(delta > 0.0 || kind == K_E2G_SL_AWAY || kind == K_E2G_P_AWAY, "delta must be > 0");
  HR_REQUIRE(out, "output missing");
  const bool direct = !opt || opt->mode == HR_DIRECT;
  const int P = opt ? opt->P : 6, N0 = opt ? opt->N0 : 1000;
  const double theta = opt ? opt->theta : 0.6;
  const bool on = (kind == K_SL_ON || kind == K_DL_ON);
  const bool dl = (kind == K_DL_ON || kind == K_DL_OFF);
  if (on) {
    nt = S->n;
    txyz = S->xyz;
  }
  HR_REQUIRE(nt >= 0 && (nt == 0 || txyz), "targets missing");
  if (S->n == 0 || nt == 0) {
    std::fill(out, out + (size_t)odim * nt, 0.0);
    // an empty surface contributes nothing; DL jump terms still apply
    if (nt > 0 && dl && dens0 && !on) {
      for (int t = 0; t < nt; t++) {
        double xi = 0.0;
        if (direct) xi = (fabs(b[t]) / delta <= 8.0 && (b[t] < 0.0 || fabs(b[t]) < 1e-14)) ? 1.0 : 0.0;
        else xi = fabs(b[t]) < 1e-12 ? 0.5 : (b[t] < 0.0 ? 1.0 : 0.0);
        for (int k = 0; k < 3; k++) out[3 * t + k] = xi * dens0[3 * t + k];
      }
    }
    return;
  }
  HR_REQUIRE(dens, "density missing");
  DevTree tree;
  tree.build(*S, P, N0, theta, direct, st);
  DBuf<double> q3;
  q3.upload(dens, 3 * (size_t)S->n, st);
  tree.set_density(C, q3.p, dl, !direct, opt && opt->precision != HR_FP64);
  std::vector<uint8_t> near =
      (kind == K_SL_OFF || kind == K_DL_OFF) ? near_flags(nt, b, delta) : std::vector<uint8_t>(nt, 1);
  DevTargets tg;
  upload_targets(tg, nt, txyz, on ? nullptr : b, x0, n0,
                 (kind == K_SL_OFF || kind == K_E2G_SL7 || kind == K_E2G_P7) ? dens0 : nullptr,
                 on ? S->nrml : nullptr, near, st);
  if (kind == K_DL_OFF && dens0) tg.g0.upload(dens0, 3 * (size_t)nt, st);
  DevLists L;
  L.build(tree.host, nt, txyz, near.data(), st);
  DBuf<double> d_out;
  d_out.alloc((size_t)odim * nt);
  double scale;
  switch (kind) {
    case K_DL_ON:
    case K_DL_OFF: scale = direct ? dl_scale_direct() : dl_scale_tree(); break;
    case K_E2G_P_AWAY: scale = p_scale(); break;
    case K_E2G_P7: scale = -p_scale(); break;
    default: scale = sl_scale();
  }
  EvalTask task = make_task(kind, delta, scale, tree, L, tg, d_out.p);
  task.jump_mode = direct ? 1 : 0;
  task.mixed = opt ? opt->precision : 0;
  if (on) task.tq = q3.p;
  Batch B;
  B.family = dl ? F_DL : ((kind <= K_DL_OFF) ? F_SL : F_E2G);
  B.tasks.push_back(task);
  B.lists.push_back(&L.host);
  B.trees.push_back(&tree.host);
  B.finalize(st, C.num_sms);
  B.launch(C);
  HR_CHECK_CUDA(cudaGetLastError());
  HR_CHECK_CUDA(cudaMemcpyAsync(out, d_out.p, sizeof(double) * odim * nt, cudaMemcpyDeviceToHost, st));
  HR_CHECK_CUDA(cudaStreamSynchronize(st));
  if (opt && opt->precision != HR_FP64) C.check_tc();
}

}  // namespace

// ----------------------------------------------------------------- context
extern "C" int hr_ctx_create(int device, hr_ctx** out) {
  if (!out) return HR_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return HR_ERR_NO_DEVICE;
  if (device < 0 || device >= ndev) return HR_ERR_ARG;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return HR_ERR_NO_DEVICE;
  if (prop.major != 10) return HR_ERR_NO_DEVICE;  // built for sm_100a only
  std::unique_ptr<hr_ctx> ctx(new hr_ctx);
  int rc = guard(ctx.get(), [&] {
    ctx->c.device = device;
    ctx->c.num_sms = prop.multiProcessorCount;
    HR_CHECK_CUDA(cudaSetDevice(device));
    HR_CHECK_CUDA(cudaStreamCreateWithFlags(&ctx->c.stream, cudaStreamNonBlocking));
    HR_CHECK_CUDA(cudaStreamCreateWithFlags(&ctx->c.side, cudaStreamNonBlocking));
    HR_CHECK_CUDA(cudaEventCreateWithFlags(&ctx->c.ev_fork, cudaEventDisableTiming));
    HR_CHECK_CUDA(cudaEventCreateWithFlags(&ctx->c.ev_join, cudaEventDisableTiming));
    ctx->c.counters.alloc(64);
    ctx->c.counters.zero(ctx->c.stream);
  });
  if (rc != HR_OK) return rc;
  *out = ctx.release();
  return HR_OK;
}

extern "C" void hr_ctx_destroy(hr_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->c.device);
  if (ctx->c.side) {
    cudaStreamSynchronize(ctx->c.side);
    cudaStreamDestroy(ctx->c.side);
  }
  if (ctx->c.stream) {
    cudaStreamSynchronize(ctx->c.stream);
    ctx->c.counters.release();
    cudaStreamDestroy(ctx->c.stream);
  }
  if (ctx->c.ev_fork) cudaEventDestroy(ctx->c.ev_fork);
  if (ctx->c.ev_join) cudaEventDestroy(ctx->c.ev_join);
  for (auto& e : ctx->c.pin_ev)
    if (e) cudaEventDestroy(e);
  if (ctx->c.pin) cudaFreeHost(ctx->c.pin);
  delete ctx;
}

extern "C" const char* hr_last_error(const hr_ctx* ctx) { return ctx ? ctx->c.err.c_str() : "no context"; }

extern "C" long long hr_ctx_launch_count(const hr_ctx* ctx) { return ctx ? ctx->c.launches : 0; }

// ---------------------------------------------------------- boundary sums
extern "C" int hr_stokes_sl_onsurf(hr_ctx* ctx, const hr_eval_opts* opt, double delta,
                                   const hr_surface* S, const double* f, double* out) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    check_opts(opt);
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    single_eval(ctx->c, K_SL_ON, opt, delta, S, f, 0, nullptr, nullptr, nullptr, nullptr, nullptr,
                out, 3);
  });
}

extern "C" int hr_stokes_sl_offsurf(hr_ctx* ctx, const hr_eval_opts* opt, double delta,
                                    const hr_surface* S, const double* f, const hr_targets* T,
                                    const double* f0, double* out) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    check_opts(opt);
    HR_REQUIRE(T && T->n >= 0, "targets missing");
    HR_REQUIRE(T->n == 0 || (T->xyz && T->b && T->n0 && f0), "target arrays missing");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    single_eval(ctx->c, K_SL_OFF, opt, delta, S, f, T->n, T->xyz, T->b, T->x0, T->n0, f0, out, 3);
  });
}

extern "C" int hr_stokes_dl_onsurf(hr_ctx* ctx, const hr_eval_opts* opt, double delta,
                                   const hr_surface* S, const double* g, double* out) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    check_opts(opt);
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    single_eval(ctx->c, K_DL_ON, opt, delta, S, g, 0, nullptr, nullptr, nullptr, nullptr, nullptr,
                out, 3);
  });
}

extern "C" int hr_stokes_dl_offsurf(hr_ctx* ctx, const hr_eval_opts* opt, double delta,
                                    const hr_surface* S, const double* g, const hr_targets* T,
                                    const double* g0, double* out) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    check_opts(opt);
    HR_REQUIRE(T && T->n >= 0, "targets missing");
    HR_REQUIRE(T->n == 0 || (T->xyz && T->b && T->x0 && T->n0 && g0), "target arrays missing");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    single_eval(ctx->c, K_DL_OFF, opt, delta, S, g, T->n, T->xyz, T->b, T->x0, T->n0, g0, out, 3);
  });
}

extern "C" int hr_e2g_stokeslet_away(hr_ctx* ctx, const hr_surface* S, const double* f, int nt,
                                     const double* xyz, double* out3) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    single_eval(ctx->c, K_E2G_SL_AWAY, nullptr, 1.0, S, f, nt, xyz, nullptr, nullptr, nullptr,
                nullptr, out3, 3);
  });
}

extern "C" int hr_e2g_pressure_away(hr_ctx* ctx, const hr_surface* S, const double* f, int nt,
                                    const double* xyz, double* out1) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    single_eval(ctx->c, K_E2G_P_AWAY, nullptr, 1.0, S, f, nt, xyz, nullptr, nullptr, nullptr,
                nullptr, out1, 1);
  });
}

extern "C" int hr_e2g_stokeslet_7ord(hr_ctx* ctx, double delta, const hr_surface* S,
                                     const double* f, const hr_targets* T, const double* f0,
                                     double* out3) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_REQUIRE(T && T->n >= 0, "targets missing");
    HR_REQUIRE(T->n == 0 || (T->xyz && T->b && T->n0 && f0), "target arrays missing");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    single_eval(ctx->c, K_E2G_SL7, nullptr, delta, S, f, T->n, T->xyz, T->b, T->x0, T->n0, f0,
                out3, 3);
  });
}

extern "C" int hr_e2g_pressure_7ord(hr_ctx* ctx, double delta, const hr_surface* S,
                                    const double* f, const hr_targets* T, const double* f0,
                                    double* out1) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_REQUIRE(T && T->n >= 0, "targets missing");
    HR_REQUIRE(T->n == 0 || (T->xyz && T->b && T->n0 && f0), "target arrays missing");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    single_eval(ctx->c, K_E2G_P7, nullptr, delta, S, f, T->n, T->xyz, T->b, T->x0, T->n0, f0,
                out1, 1);
  });
}

extern "C" int hr_interpolate_dl_density(hr_ctx* ctx, double h, const hr_surface* S,
                                         const double* g, const hr_targets* T, double* g0) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_REQUIRE(S && T && g0, "arguments missing");
    HR_REQUIRE(h > 0.0, "h must be > 0");
    HR_REQUIRE(T->n == 0 || (T->x0 && T->nrst && T->i123), "target nearest data missing");
    HR_REQUIRE(S->n == 0 || (S->xyz && g), "surface arrays missing");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    cudaStream_t st = ctx->c.stream;
    check_i123(T->n, T->nrst, T->i123);
    Stencils s = build_stencils(h, S->center, S->n, S->xyz, T->n, T->nrst, T->x0, T->i123);
    if (S->n == 0) {
      for (size_t e = 0; e < s.tgt.size(); e++) HR_REQUIRE(false, "interpolation from an empty surface");
    }
    DevStencils ds;
    ds.build(s, st);
    DBuf<double> dg, dg0;
    dg.upload(g, 3 * (size_t)std::max(1, S->n), st);
    dg0.alloc(3 * (size_t)std::max(1, T->n));
    dg0.zero(st);
    launch_interp(ds.ne, ds.tgt.p, ds.idx.p, ds.pq.p, dg.p, dg0.p, st);
    ctx->c.launches++;
    HR_CHECK_CUDA(cudaGetLastError());
    HR_CHECK_CUDA(cudaMemcpyAsync(g0, dg0.p, sizeof(double) * 3 * T->n, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
}

extern "C" int hr_dst_poisson3d(hr_ctx* ctx, int n, double* f) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_REQUIRE(n >= 1 && f, "bad DST arguments");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    cudaStream_t st = ctx->c.stream;
    size_t m = (size_t)n * n * n;
    DBuf<double> d;
    d.upload(f, m, st);
    dst_poisson3d_dev(ctx->c, n, d.p);
    HR_CHECK_CUDA(cudaMemcpyAsync(f, d.p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
}

struct hr_dst1_plan {
  hr_ctx* ctx = nullptr;
  hr::Dst1Plan* d = nullptr;
  ~hr_dst1_plan() {
    if (d) hr::dst1_plan_destroy(d);
  }
};

extern "C" int hr_dst1_plan_create(hr_ctx* ctx, int n, hr_dst1_plan** out) {
  if (!ctx || !out) return HR_ERR_ARG;
  *out = nullptr;
  return guard(ctx, [&] {
    HR_REQUIRE(n >= 1 && (n + 1) % 2 == 0, "3D DST-I length n must have n + 1 even");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    std::unique_ptr<hr_dst1_plan> p(new hr_dst1_plan);
    p->ctx = ctx;
    p->d = dst1_plan_create(ctx->c, n);
    *out = p.release();
  });
}

extern "C" int hr_dst1_execute(hr_dst1_plan* p, const double* in, double* out) {
  if (!p || !in || !out) return HR_ERR_ARG;
  return guard(p->ctx, [&] {
    HR_CHECK_CUDA(cudaSetDevice(p->ctx->c.device));
    dst1_execute(p->ctx->c, p->d, in, out);
  });
}

extern "C" int hr_host_alloc(size_t bytes, void** out) {
  if (!out) return HR_ERR_ARG;
  *out = nullptr;
  if (cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    *out = nullptr;
    return HR_ERR_CUDA;
  }
  return HR_OK;
}

extern "C" void hr_host_free(void* p) {
  if (p) cudaFreeHost(p);
}

extern "C" void hr_dst1_plan_destroy(hr_dst1_plan* p) {
  if (!p) return;
  cudaSetDevice(p->ctx->c.device);
  cudaStreamSynchronize(p->ctx->c.stream);
  delete p;
}

extern "C" int hr_e2g_solve_poisson(hr_ctx* ctx, int N, double L, const uint8_t* band2,
                                    const uint8_t* outside, const double* p, double* u,
                                    int variable) {
  if (!ctx) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_REQUIRE(N >= 6 && L > 0 && band2 && outside && u, "bad Poisson arguments");
    HR_REQUIRE(!(variable >= 1 && variable <= 3) || p, "pressure grid missing");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    cudaStream_t st = ctx->c.stream;
    size_t m = (size_t)(N + 1) * (N + 1) * (N + 1);
    DBuf<uint8_t> db, dout;
    DBuf<double> dp, du;
    db.upload(band2, m, st);
    dout.upload(outside, m, st);
    if (p) dp.upload(p, m, st);
    du.upload(u, m, st);
    solve_poisson_dev(ctx->c, N, L, db.p, dout.p, p ? dp.p : nullptr, du.p, variable);
    HR_CHECK_CUDA(cudaMemcpyAsync(u, du.p, m * sizeof(double), cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
}

// ------------------------------------------------------------ two surfaces
struct hr_plan2s {
  hr_ctx* owner = nullptr;
  Ctx* C = nullptr;
  int nq[2] = {0, 0};
  int off[2] = {0, 0};  // offsets of each surface in the 3n vector
  int n = 0;
  double h = 0, delta = 0;
  hr_eval_opts opt;
  DevTree tree[2];
  DevTargets tg[2];
  DevLists Lon[2], Loff[2];  // Loff[t]: tree of surface 1-t at target set t
  DevStencils sten[2];       // sten[t]: density of surface 1-t at target set t's x0
  DBuf<double> out_on[2], out_off[2];
  DBuf<double> xin, fin;
  DBuf<unsigned long long> counters;  // 4 per task: reg, near-plain, far-target, proxy
  Batch dl[3];                         // by precision: [0] FP64, [1] mixed, [2] all FP32
  Batch sl;
  // GMRES work space
  int Vcols = 0;
  DBuf<double> V, r, bsave, partial, hbuf, ybuf;
  // Optional treecode of the reduced-precision inner operator of GMRES-IR:
  // trees and interaction lists of its own over the same targets, stencils
  // and output buffers.
  struct Inner {
    int P = 0, N0 = 0;
    double theta = 0.0;
    DevTree tree[2];
    DevLists Lon[2], Loff[2];
    Batch dl[3];  // [1] mixed, [2] all FP32 ([0] unused)
    double accuracy = 0.0;  // measured ||A_inner u - A u|| / ||A u|| (mixed precision)
  };
  std::unique_ptr<Inner> inner;
  // host copies of the surfaces and near flags, for building an inner treecode later
  std::vector<double> hxyz[2], hnrml[2], harea[2];
  std::vector<uint8_t> near_host[2];
  hr_surface surf_host[2];
  // the density-interpolation stencils' inputs per target set (the caller's
  // scene need not outlive the plan's creation); built on dl_thread, then freed
  std::vector<int> hnrst[2], hi123[2];
  std::vector<double> hx0[2];
  // The density-interpolation stencils are built and the FP64 stresslet batch
  // segmented on a host thread of its own while the caller goes on (to the
  // right-hand side, which needs only the Stokeslet batch), their uploads on a
  // stream of its own; every other use of the plan first waits for it
  // (plan_ready).
  std::thread dl_thread;
  std::mutex dl_mu;  // one joiner, if two host threads reach plan_ready at once
  std::exception_ptr dl_error;
  cudaStream_t up = nullptr;
  cudaEvent_t up_done = nullptr;
  ~hr_plan2s() {
    if (dl_thread.joinable()) dl_thread.join();
    if (up_done) cudaEventDestroy(up_done);
    if (up) cudaStreamDestroy(up);
  }
};

namespace {

// Runs a() on a second host thread (with `device` current there) and b() on
// this one, each with half of the host's cores for its OpenMP loops (so the
// two teams do not oversubscribe them); rethrows the exception of either
// (b's first).
template <class A, class B>
void run_both(int device, A&& a, B&& b) {
  const int half = std::max(1, omp_get_num_procs() / 2);
  const int before = omp_get_max_threads();
  std::exception_ptr ea, eb;
  std::thread th([&] {
    try {
      omp_set_num_threads(half);
      HR_CHECK_CUDA(cudaSetDevice(device));
      a();
    } catch (...) {
      ea = std::current_exception();
    }
  });
  omp_set_num_threads(half);
  try {
    b();
  } catch (...) {
    eb = std::current_exception();
  }
  omp_set_num_threads(before);
  th.join();
  if (eb) std::rethrow_exception(eb);
  if (ea) std::rethrow_exception(ea);
}

void sl_batch(hr_plan2s& P);

// Stresslet batches of the matvec, one per precision in [prec0, prec1), over
// the given trees and lists (the plan's own, or the inner operator's).
void dl_batches(hr_plan2s& P, DevTree* tree, DevLists* Lon, DevLists* Loff, Batch* dl, int prec0, int prec1,
                bool count, cudaStream_t st) {
  const bool direct = P.opt.mode == HR_DIRECT;
  for (int prec = prec0; prec < prec1; prec++) {
    Batch& B = dl[prec];
    B.family = F_DL;
    B.tasks.clear();
    B.lists.clear();
    B.trees.clear();
    for (int t = 0; t < 2; t++) {
      const int s = t;
      EvalTask on = make_task(K_DL_ON, P.delta, direct ? dl_scale_direct() : dl_scale_tree(),
                              tree[s], Lon[t], P.tg[t], P.out_on[t].p);
      on.tq = P.xin.p + P.off[s];
      on.mixed = prec;
      if (count) on.counters = P.counters.p + 4 * (2 * t);
      EvalTask of = make_task(K_DL_OFF, P.delta, direct ? dl_scale_direct() : dl_scale_tree(),
                              tree[1 - t], Loff[t], P.tg[t], P.out_off[t].p);
      of.jump_mode = direct ? 1 : 0;
      of.mixed = prec;
      if (count) of.counters = P.counters.p + 4 * (2 * t + 1);
      B.tasks.push_back(on);
      B.lists.push_back(&Lon[t].host);
      B.trees.push_back(&tree[s].host);
      B.tasks.push_back(of);
      B.lists.push_back(&Loff[t].host);
      B.trees.push_back(&tree[1 - t].host);
    }
    B.finalize(st, P.C->num_sms);
  }
}

void plan_batches(hr_plan2s& P) {
  cudaStream_t st = P.C->stream;
  P.counters.alloc(4 * 8);
  P.counters.zero(st);
  // the reduced-precision batches are built on first use (plan_matvec); the
  // Stokeslet batch here, the FP64 stresslet batch on a second host thread
  // that outlives the plan's creation
  sl_batch(P);
  HR_CHECK_CUDA(cudaStreamCreateWithFlags(&P.up, cudaStreamNonBlocking));
  HR_CHECK_CUDA(cudaEventCreateWithFlags(&P.up_done, cudaEventDisableTiming));
  const int dev = P.C->device;
  P.dl_thread = std::thread([&P, dev] {
    try {
      HR_CHECK_CUDA(cudaSetDevice(dev));
      for (int t = 0; t < 2; t++) {
        const hr_surface& Ssrc = P.surf_host[1 - t];
        Stencils sv = build_stencils(P.h, Ssrc.center, Ssrc.n, Ssrc.xyz, P.nq[t], P.hnrst[t].data(),
                                     P.hx0[t].data(), P.hi123[t].data());
        P.sten[t].build(sv, P.up);
        std::vector<int>().swap(P.hnrst[t]);
        std::vector<int>().swap(P.hi123[t]);
        std::vector<double>().swap(P.hx0[t]);
      }
      dl_batches(P, P.tree, P.Lon, P.Loff, P.dl, 0, 1, true, P.up);
      HR_CHECK_CUDA(cudaEventRecord(P.up_done, P.up));
    } catch (...) {
      P.dl_error = std::current_exception();
    }
  });
}

// Waits for the FP64 stresslet batch of plan_batches (and orders the plan's
// stream after its uploads); rethrows its error on every use.
void plan_ready(hr_plan2s& P) {
  std::lock_guard<std::mutex> lock(P.dl_mu);
  if (P.dl_thread.joinable()) {
    P.dl_thread.join();
    if (!P.dl_error) HR_CHECK_CUDA(cudaStreamWaitEvent(P.C->stream, P.up_done, 0));
  }
  if (P.dl_error) std::rethrow_exception(P.dl_error);
}

void sl_batch(hr_plan2s& P) {
  cudaStream_t st = P.C->stream;
  Batch& B = P.sl;
  B.family = F_SL;
  for (int t = 0; t < 2; t++) {
    EvalTask on = make_task(K_SL_ON, P.delta, sl_scale(), P.tree[t], P.Lon[t], P.tg[t], P.out_on[t].p);
    on.tq = P.fin.p + P.off[t];
    on.counters = P.counters.p + 4 * (4 + 2 * t);
    EvalTask of = make_task(K_SL_OFF, P.delta, sl_scale(), P.tree[1 - t], P.Loff[t], P.tg[t],
                            P.out_off[t].p);
    of.counters = P.counters.p + 4 * (4 + 2 * t + 1);
    B.tasks.push_back(on);
    B.lists.push_back(&P.Lon[t].host);
    B.trees.push_back(&P.tree[t].host);
    B.tasks.push_back(of);
    B.lists.push_back(&P.Loff[t].host);
    B.trees.push_back(&P.tree[1 - t].host);
  }
  B.finalize(st, P.C->num_sms);
}

void plan_matvec(hr_plan2s& P, const double* x_dev, double* y_dev, int prec) {
  Ctx& C = *P.C;
  cudaStream_t st = C.stream;
  const bool tree = P.opt.mode == HR_TREE;
  if (x_dev != P.xin.p)
    HR_CHECK_CUDA(cudaMemcpyAsync(P.xin.p, x_dev, sizeof(double) * P.n, cudaMemcpyDeviceToDevice, st));
  // the reduced-precision operator runs on the inner treecode when there is one
  hr_plan2s::Inner* in = (prec != HR_FP64 && P.inner) ? P.inner.get() : nullptr;
  DevTree* trees = in ? in->tree : P.tree;
  plan_ready(P);  // the stencils and the FP64 stresslet batch
  for (int s = 0; s < 2; s++) trees[s].set_density(C, P.xin.p + P.off[s], true, tree, prec != HR_FP64);
  for (int t = 0; t < 2; t++) {
    P.tg[t].g0.zero(st);
    launch_interp(P.sten[t].ne, P.sten[t].tgt.p, P.sten[t].idx.p, P.sten[t].pq.p,
                  P.xin.p + P.off[1 - t], P.tg[t].g0.p, st);
    C.launches++;
  }
  if (!in && !P.dl[prec].ready) dl_batches(P, P.tree, P.Lon, P.Loff, P.dl, prec, prec + 1, true, st);
  (in ? in->dl[prec] : P.dl[prec]).launch(C);
  // set 0: u - on*f - comp*f ; set 1: u - comp*f - on*f   (2S/main.cpp:612-676)
  launch_matvec_combine(3 * P.nq[0], 2.0 / 3.0, P.xin.p + P.off[0], P.out_on[0].p, P.out_off[0].p,
                        y_dev + P.off[0], st);
  launch_matvec_combine(3 * P.nq[1], 2.0 / 3.0, P.xin.p + P.off[1], P.out_off[1].p, P.out_on[1].p,
                        y_dev + P.off[1], st);
  C.launches += 2;
  HR_CHECK_CUDA(cudaGetLastError());
}

void plan_rhs(hr_plan2s& P, const double* f1_dev, const double* f2_dev, double* b_dev) {
  Ctx& C = *P.C;
  cudaStream_t st = C.stream;
  const bool tree = P.opt.mode == HR_TREE;
  if (f1_dev != P.fin.p + P.off[0])
    HR_CHECK_CUDA(cudaMemcpyAsync(P.fin.p + P.off[0], f1_dev, sizeof(double) * 3 * P.nq[0],
                                  cudaMemcpyDeviceToDevice, st));
  if (f2_dev != P.fin.p + P.off[1])
    HR_CHECK_CUDA(cudaMemcpyAsync(P.fin.p + P.off[1], f2_dev, sizeof(double) * 3 * P.nq[1],
                                  cudaMemcpyDeviceToDevice, st));
  for (int s = 0; s < 2; s++) P.tree[s].set_density(C, P.fin.p + P.off[s], false, tree);
  P.sl.launch(C);
  // SL_1 = on1 + comp2 ; SL_2 = comp1 + on2 ; b = -SL * 2/3
  launch_rhs_combine(3 * P.nq[0], 2.0 / 3.0, P.out_on[0].p, P.out_off[0].p, b_dev + P.off[0], st);
  launch_rhs_combine(3 * P.nq[1], 2.0 / 3.0, P.out_off[1].p, P.out_on[1].p, b_dev + P.off[1], st);
  C.launches += 2;
  HR_CHECK_CUDA(cudaGetLastError());
}

double dev_norm(hr_plan2s& P, const double* v) {
  Ctx& C = *P.C;
  launch_dots(P.n, 1, v, P.n, v, P.partial.p, C.stream);
  launch_dots_finalize(1, P.partial.p, P.hbuf.p, C.stream);
  C.launches += 2;
  double h;
  HR_CHECK_CUDA(cudaMemcpyAsync(&h, P.hbuf.p, sizeof(double), cudaMemcpyDeviceToHost, C.stream));
  HR_CHECK_CUDA(cudaStreamSynchronize(C.stream));
  return sqrt(h);
}

// GMRES with classical Gram-Schmidt and one re-orthogonalisation, Givens
// rotations on the host, relative residual ||r|| / ||b|| (2S/main.cpp:236-416),
// restarting from the true residual r = b - A x.
// HR_MIXED / HR_FP32 solve by iterative refinement with reduced-precision
// inner GMRES (GMRES-IR): every Krylov matvec is in the reduced precision; a
// cycle stops once its Arnoldi residual has fallen by eta = 10 x
// mixed_accuracy (or below tol / 2); the FP64 true residual r = b - A x then
// starts the next cycle, and the solve ends when that FP64 residual meets
// tol. A cycle that does not halve the true residual sends the rest of the
// solve to FP64 matvecs.
int plan_solve(hr_plan2s& P, const hr_gmres_opts& o, const double* b_dev, double* x_dev,
               hr_gmres_report* rep) {
  Ctx& C = *P.C;
  cudaStream_t st = C.stream;
  const int n = P.n;
  const int m = std::max(1, std::min(o.restart, 60));
  const int max_iter = std::max(0, o.max_iter);
  hr_gmres_report R;
  memset(&R, 0, sizeof(R));
  R.true_residual = -1.0;
  if (P.Vcols < m + 1) {
    P.V.alloc((size_t)(m + 1) * n);
    P.Vcols = m + 1;
  }
  cudaEvent_t e0, e1;
  HR_CHECK_CUDA(cudaEventCreate(&e0));
  HR_CHECK_CUDA(cudaEventCreate(&e1));
  HR_CHECK_CUDA(cudaEventRecord(e0, st));
  // default: the mixed matvec's measured max-norm relative error is 2.7e-7
  // (with an inner treecode, at least its measured accuracy)
  const double mixed_eps =
      o.mixed_accuracy > 0.0
          ? o.mixed_accuracy
          : std::max(o.precision == HR_FP32 ? 1e-6 : 3e-7, P.inner ? P.inner->accuracy : 0.0);
  const bool refine = o.precision != HR_FP64;
  const double eta = std::min(0.1, 10.0 * mixed_eps);
  double b_norm = dev_norm(P, b_dev);
  double bscale = b_norm > 1.e-8 ? b_norm : 1.0;
  double* r = P.r.p;
  // initial residual; with refinement the guess's residual comes from the
  // reduced-precision operator (the first FP64 true residual follows its cycle)
  bool r_true = true;  // r holds the FP64 residual b - A x
  if (o.use_guess) {
    const int p0 = refine ? o.precision : HR_FP64;
    plan_matvec(P, x_dev, r, p0);
    if (p0) R.matvecs_mixed++;
    else R.matvecs_fp64++;
    r_true = p0 == HR_FP64;
    launch_sub(n, b_dev, r, r, st);
    C.launches++;
    double rn = dev_norm(P, r);
    if (!(rn <= b_norm) || !std::isfinite(rn)) {  // worse than the zero guess: drop it
      R.guess_rejected = 1;
      HR_CHECK_CUDA(cudaMemsetAsync(x_dev, 0, sizeof(double) * n, st));
      launch_copy(n, b_dev, r, st);
      C.launches++;
      r_true = true;
    }
  } else {
    HR_CHECK_CUDA(cudaMemsetAsync(x_dev, 0, sizeof(double) * n, st));
    launch_copy(n, b_dev, r, st);
    C.launches++;
  }
  std::vector<double> H((size_t)(m + 1) * m, 0.0), g(m + 1, 0.0), y(m + 1, 0.0), cs(m, 0.0),
      sn(m, 0.0), hh(2 * 64 + 2, 0.0);
  auto Hm = [&](int i, int j) -> double& { return H[(size_t)i * m + j]; };
  int iter = 0;
  double error = 1.0;
  int status = HR_OK;
  bool need_true_check = o.true_residual != 0 || o.precision != HR_FP64;
  int fp64_tail = 0;  // after a refinement cycle that stalled, stay in FP64
  for (;;) {
    double r_norm = dev_norm(P, r);
    error = r_norm / bscale;
    if (!std::isfinite(r_norm)) {
      status = HR_ERR_NAN;
      break;
    }
    if (refine && R.restarts > 0) R.true_residual = error;
    if (error <= o.tol && !r_true) {  // a guess already good enough: confirm in FP64
      plan_matvec(P, x_dev, r, 0);
      R.matvecs_fp64++;
      launch_sub(n, b_dev, r, r, st);
      C.launches++;
      r_true = true;
      R.restarts++;
      continue;
    }
    if (error <= o.tol || iter >= max_iter) break;
    const double err_start = error;
    const double cycle_tol = (refine && !fp64_tail) ? std::max(0.5 * o.tol, eta * err_start) : o.tol;
    launch_copy(n, r, P.V.p, st);
    launch_scale_host(n, 1.0 / r_norm, P.V.p, st);
    C.launches += 2;
    std::fill(g.begin(), g.end(), 0.0);
    g[0] = r_norm;
    int j = -1;
    while (j < m - 1 && error > cycle_tol && iter < max_iter) {
      j++;
      iter++;
      double* vj = P.V.p + (size_t)j * n;
      double* w = P.V.p + (size_t)(j + 1) * n;
      const int prec = (refine && !fp64_tail) ? o.precision : HR_FP64;
      plan_matvec(P, vj, w, prec);
      if (prec) R.matvecs_mixed++;
      else R.matvecs_fp64++;
      // CGS2
      launch_dots(n, j + 1, P.V.p, n, w, P.partial.p, st);
      launch_dots_finalize(j + 1, P.partial.p, P.hbuf.p, st);
      launch_axpy_multi(n, j + 1, P.V.p, n, P.hbuf.p, -1.0, w, st);
      launch_dots(n, j + 1, P.V.p, n, w, P.partial.p, st);
      launch_dots_finalize(j + 1, P.partial.p, P.hbuf.p + 64, st);
      launch_axpy_multi(n, j + 1, P.V.p, n, P.hbuf.p + 64, -1.0, w, st);
      launch_dots(n, 1, w, n, w, P.partial.p, st);
      launch_dots_finalize(1, P.partial.p, P.hbuf.p + 128, st);
      C.launches += 8;
      HR_CHECK_CUDA(cudaMemcpyAsync(hh.data(), P.hbuf.p, sizeof(double) * 129, cudaMemcpyDeviceToHost, st));
      HR_CHECK_CUDA(cudaStreamSynchronize(st));
      for (int i = 0; i <= j; i++) Hm(i, j) = hh[i] + hh[64 + i];
      double v_norm = sqrt(hh[128]);
      Hm(j + 1, j) = v_norm;
      if (v_norm != 0.0) {
        launch_scale_host(n, 1.0 / v_norm, w, st);
        C.launches++;
      }
      for (int i = 0; i <= j - 1; i++) {
        double t = Hm(i, j);
        Hm(i, j) = cs[i] * t + sn[i] * Hm(i + 1, j);
        Hm(i + 1, j) = -sn[i] * t + cs[i] * Hm(i + 1, j);
      }
      double hr_ = sqrt(Hm(j, j) * Hm(j, j) + Hm(j + 1, j) * Hm(j + 1, j));
      if (hr_ == 0.0) hr_ = 1.e-16;
      cs[j] = Hm(j, j) / hr_;
      sn[j] = Hm(j + 1, j) / hr_;
      Hm(j, j) = cs[j] * Hm(j, j) + sn[j] * Hm(j + 1, j);
      Hm(j + 1, j) = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      error = fabs(g[j + 1]) / bscale;
      if (iter - 1 < 512) R.resid_hist[iter - 1] = error;
      if (!std::isfinite(error)) {
        status = HR_ERR_NAN;
        break;
      }
    }
    if (status != HR_OK || j < 0) break;
    // y = R^{-1} g, x += V y
    for (int i = 0; i <= j; i++) y[i] = g[i];
    y[j] = y[j] / Hm(j, j);
    for (int k = j - 1; k >= 0; k--) {
      double t = y[k];
      for (int i = k + 1; i <= j; i++) t -= Hm(k, i) * y[i];
      y[k] = t / Hm(k, k);
    }
    HR_CHECK_CUDA(cudaMemcpyAsync(P.ybuf.p, y.data(), sizeof(double) * (j + 1), cudaMemcpyHostToDevice, st));
    launch_axpy_multi(n, j + 1, P.V.p, n, P.ybuf.p, 1.0, x_dev, st);
    C.launches++;
    R.restarts++;
    const bool converged = error <= o.tol;
    if (converged && !need_true_check) break;
    // true residual r = b - A x (FP64)
    plan_matvec(P, x_dev, r, 0);
    R.matvecs_fp64++;
    launch_sub(n, b_dev, r, r, st);
    C.launches++;
    r_true = true;
    if (refine) {
      const double tr = dev_norm(P, r) / bscale;
      if (!(tr <= 0.5 * err_start)) fp64_tail = 1;  // the reduced-precision cycle stalled
      continue;  // the loop head tests the FP64 residual
    }
    if (converged) {
      double tr = dev_norm(P, r) / bscale;
      R.true_residual = tr;
      if (tr <= o.tol * 10.0 || iter >= max_iter) break;
    }
  }
  if (status == HR_OK && need_true_check && R.true_residual < 0) {
    plan_matvec(P, x_dev, r, 0);
    R.matvecs_fp64++;
    launch_sub(n, b_dev, r, r, st);
    C.launches++;
    R.true_residual = dev_norm(P, r) / bscale;
  }
  HR_CHECK_CUDA(cudaEventRecord(e1, st));
  HR_CHECK_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  C.check_tc();
  R.iterations = iter;
  R.residual = error;
  R.seconds = ms * 1e-3;
  if (rep) *rep = R;
  if (status != HR_OK) return status;
  if (error > o.tol) return HR_ERR_NOT_CONVERGED;
  return HR_OK;
}

}  // namespace

extern "C" int hr_plan2s_create(hr_ctx* ctx, const hr_scene2s* sc, const hr_eval_opts* opt,
                                hr_plan2s** out) {
  if (!ctx || !out) return HR_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<hr_plan2s> P(new hr_plan2s);
  int rc = guard(ctx, [&] {
    check_opts(opt);
    HR_REQUIRE(sc, "scene missing");
    HR_REQUIRE(sc->delta > 0 && sc->h > 0, "h and delta must be > 0");
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    cudaStream_t st = ctx->c.stream;
    P->owner = ctx;
    P->C = &ctx->c;
    P->opt = *opt;
    P->h = sc->h;
    P->delta = sc->delta;
    for (int s = 0; s < 2; s++) {
      const hr_surface& S = sc->surf[s];
      const hr_targets& T = sc->tgt[s];
      HR_REQUIRE(S.n > 0 && S.xyz && S.nrml && S.area && S.plane, "surface arrays missing");
      HR_REQUIRE(T.n == S.n, "target set s must be the points of surface s");
      HR_REQUIRE(T.b && T.x0 && T.n0 && T.nrst && T.i123 && sc->f0[s], "target nearest data missing");
      check_finite(S.xyz, 3 * (size_t)S.n, "surface points");
      check_finite(S.nrml, 3 * (size_t)S.n, "surface normals");
      check_finite(S.area, S.n, "area weights");
      P->nq[s] = S.n;
      P->hxyz[s].assign(S.xyz, S.xyz + 3 * (size_t)S.n);
      P->hnrml[s].assign(S.nrml, S.nrml + 3 * (size_t)S.n);
      P->harea[s].assign(S.area, S.area + S.n);
      hr_surface& H = P->surf_host[s];
      H = S;
      H.xyz = P->hxyz[s].data();
      H.nrml = P->hnrml[s].data();
      H.area = P->harea[s].data();
      H.plane = nullptr;
    }
    P->off[0] = 0;
    P->off[1] = 3 * P->nq[0];
    P->n = 3 * (P->nq[0] + P->nq[1]);
    const bool direct = opt->mode == HR_DIRECT;
    // the two surfaces' host planning runs on two host threads
    run_both(
        ctx->c.device, [&] { P->tree[1].build(sc->surf[1], opt->P, opt->N0, opt->theta, direct, st); },
        [&] { P->tree[0].build(sc->surf[0], opt->P, opt->N0, opt->theta, direct, st); });
    auto per_target_set = [&](int t) {
      const hr_targets& T = sc->tgt[t];
      std::vector<uint8_t> near = near_flags(T.n, T.b, sc->delta);
      P->near_host[t] = near;
      upload_targets(P->tg[t], T.n, sc->surf[t].xyz, T.b, T.x0, T.n0, sc->f0[t], sc->surf[t].nrml,
                     near, st);
      std::vector<uint8_t> all(T.n, 1);
      const std::vector<int> mo = morton_order(T.n, sc->surf[t].xyz);  // shared by both lists
      P->Lon[t].build(P->tree[t].host, T.n, sc->surf[t].xyz, all.data(), st, &mo);
      P->Loff[t].build(P->tree[1 - t].host, T.n, sc->surf[t].xyz, near.data(), st, &mo);
      check_i123(T.n, T.nrst, T.i123);
      P->hnrst[t].assign(T.nrst, T.nrst + T.n);
      P->hi123[t].assign(T.i123, T.i123 + 3 * (size_t)T.n);
      P->hx0[t].assign(T.x0, T.x0 + 3 * (size_t)T.n);
      P->out_on[t].alloc(3 * (size_t)T.n);
      P->out_off[t].alloc(3 * (size_t)T.n);
    };
    run_both(ctx->c.device, [&] { per_target_set(1); }, [&] { per_target_set(0); });
    P->xin.alloc(P->n);
    P->fin.alloc(P->n);
    P->r.alloc(P->n);
    P->partial.alloc((size_t)kRedBlocks * 64);
    P->hbuf.alloc(256);
    P->ybuf.alloc(64);
    plan_batches(*P);
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
  if (rc != HR_OK) return rc;
  *out = P.release();
  return HR_OK;
}

extern "C" void hr_plan2s_destroy(hr_plan2s* plan) {
  if (!plan) return;
  if (plan->C) cudaStreamSynchronize(plan->C->stream);
  delete plan;
}

extern "C" int hr_plan2s_set_inner_tree(hr_plan2s* plan, int P, int N0, double theta, double* rel_err) {
  if (!plan) return HR_ERR_ARG;
  return guard(plan->owner, [&] {
    hr_plan2s& Q = *plan;
    plan_ready(Q);
    HR_REQUIRE(Q.opt.mode == HR_TREE, "an inner treecode needs an HR_TREE plan");
    if (rel_err) *rel_err = 0.0;
    if (P == 0) {
      HR_CHECK_CUDA(cudaStreamSynchronize(Q.C->stream));
      Q.inner.reset();
      return;
    }
    HR_REQUIRE(P >= 1 && P <= 15, "inner treecode degree P must be in [1, 15]");
    HR_REQUIRE(N0 >= 1, "inner treecode leaf size N0 must be >= 1");
    HR_REQUIRE(theta > 0.0 && theta < 1.0, "inner treecode theta must be in (0, 1)");
    cudaStream_t st = Q.C->stream;
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
    std::unique_ptr<hr_plan2s::Inner> in(new hr_plan2s::Inner);
    in->P = P;
    in->N0 = N0;
    in->theta = theta;
    for (int s = 0; s < 2; s++) in->tree[s].build(Q.surf_host[s], P, N0, theta, false, st);
    for (int t = 0; t < 2; t++) {
      std::vector<uint8_t> all(Q.nq[t], 1);
      const std::vector<int> mo = morton_order(Q.nq[t], Q.surf_host[t].xyz);
      in->Lon[t].build(in->tree[t].host, Q.nq[t], Q.surf_host[t].xyz, all.data(), st, &mo);
      in->Loff[t].build(in->tree[1 - t].host, Q.nq[t], Q.surf_host[t].xyz, Q.near_host[t].data(), st, &mo);
    }
    dl_batches(Q, in->tree, in->Lon, in->Loff, in->dl, 1, 3, false, Q.C->stream);
    // accuracy of the inner operator (mixed precision) against the plan's FP64
    // one, on a fixed pseudo-random density
    Q.inner.reset();
    std::vector<double> u(Q.n), y64(Q.n), yin(Q.n);
    std::mt19937_64 rng(20261203);
    std::normal_distribution<double> nd(0.0, 1.0);
    for (auto& v : u) v = nd(rng);
    DBuf<double> du, dy;
    du.upload(u, st);
    dy.alloc(Q.n);
    plan_matvec(Q, du.p, dy.p, HR_FP64);
    HR_CHECK_CUDA(cudaMemcpyAsync(y64.data(), dy.p, sizeof(double) * Q.n, cudaMemcpyDeviceToHost, st));
    Q.inner = std::move(in);
    plan_matvec(Q, du.p, dy.p, HR_MIXED);
    HR_CHECK_CUDA(cudaMemcpyAsync(yin.data(), dy.p, sizeof(double) * Q.n, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
    Q.C->check_tc();
    double num = 0.0, den = 0.0;
    for (int i = 0; i < Q.n; i++) {
      num += (yin[i] - y64[i]) * (yin[i] - y64[i]);
      den += y64[i] * y64[i];
    }
    Q.inner->accuracy = den > 0.0 ? sqrt(num / den) : 0.0;
    if (rel_err) *rel_err = Q.inner->accuracy;
  });
}

extern "C" void* hr_plan2s_stream(hr_plan2s* plan) { return plan ? (void*)plan->C->stream : nullptr; }

static hr_ctx* ctx_of(hr_plan2s* p) { return p->owner; }

extern "C" int hr_plan2s_matvec_dev(hr_plan2s* plan, const double* x_dev, double* y_dev, int precision) {
  if (!plan) return HR_ERR_ARG;
  return guard(ctx_of(plan), [&] {
    HR_REQUIRE(x_dev && y_dev, "null vector");
    HR_REQUIRE(precision == HR_FP64 || precision == HR_MIXED || precision == HR_FP32, "unknown precision");
    plan_matvec(*plan, x_dev, y_dev, precision);
    if (precision != HR_FP64) plan->C->check_tc();
  });
}

extern "C" int hr_plan2s_rhs_dev(hr_plan2s* plan, const double* f1_dev, const double* f2_dev,
                                 double* b_dev) {
  if (!plan) return HR_ERR_ARG;
  return guard(ctx_of(plan), [&] {
    HR_REQUIRE(f1_dev && f2_dev && b_dev, "null vector");
    plan_rhs(*plan, f1_dev, f2_dev, b_dev);
  });
}

extern "C" int hr_plan2s_solve_dev(hr_plan2s* plan, const hr_gmres_opts* opt, const double* b_dev,
                                   double* x_dev, hr_gmres_report* rep) {
  if (!plan || !opt) return HR_ERR_ARG;
  int status = HR_OK;
  int rc = guard(ctx_of(plan), [&] {
    HR_REQUIRE(b_dev && x_dev, "null vector");
    HR_REQUIRE(opt->restart >= 1 && opt->restart <= 60, "restart must be in [1, 60]");
    HR_REQUIRE(opt->tol > 0, "tol must be > 0");
    status = plan_solve(*plan, *opt, b_dev, x_dev, rep);
    if (status == HR_ERR_NOT_CONVERGED) plan->C->err = "GMRES did not reach the tolerance";
    if (status == HR_ERR_NAN) plan->C->err = "non-finite residual in GMRES";
  });
  return rc != HR_OK ? rc : status;
}

extern "C" int hr_plan2s_matvec(hr_plan2s* plan, const double* x, double* y) {
  if (!plan) return HR_ERR_ARG;
  return guard(ctx_of(plan), [&] {
    HR_REQUIRE(x && y, "null vector");
    cudaStream_t st = plan->C->stream;
    DBuf<double> dy;
    dy.alloc(plan->n);
    HR_CHECK_CUDA(cudaMemcpyAsync(plan->xin.p, x, sizeof(double) * plan->n, cudaMemcpyHostToDevice, st));
    plan_matvec(*plan, plan->xin.p, dy.p, 0);
    HR_CHECK_CUDA(cudaMemcpyAsync(y, dy.p, sizeof(double) * plan->n, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
}

extern "C" int hr_plan2s_rhs(hr_plan2s* plan, const double* f1, const double* f2, double* b) {
  if (!plan) return HR_ERR_ARG;
  return guard(ctx_of(plan), [&] {
    HR_REQUIRE(f1 && f2 && b, "null vector");
    cudaStream_t st = plan->C->stream;
    DBuf<double> db;
    db.alloc(plan->n);
    HR_CHECK_CUDA(cudaMemcpyAsync(plan->fin.p, f1, sizeof(double) * 3 * plan->nq[0], cudaMemcpyHostToDevice, st));
    HR_CHECK_CUDA(cudaMemcpyAsync(plan->fin.p + plan->off[1], f2, sizeof(double) * 3 * plan->nq[1],
                                  cudaMemcpyHostToDevice, st));
    plan_rhs(*plan, plan->fin.p, plan->fin.p + plan->off[1], db.p);
    HR_CHECK_CUDA(cudaMemcpyAsync(b, db.p, sizeof(double) * plan->n, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
}

extern "C" int hr_plan2s_solve(hr_plan2s* plan, const hr_gmres_opts* opt, const double* b,
                               double* x, hr_gmres_report* rep) {
  if (!plan || !opt) return HR_ERR_ARG;
  int status = HR_OK;
  int rc = guard(ctx_of(plan), [&] {
    HR_REQUIRE(b && x, "null vector");
    HR_REQUIRE(opt->restart >= 1 && opt->restart <= 60, "restart must be in [1, 60]");
    cudaStream_t st = plan->C->stream;
    DBuf<double> db, dx;
    db.upload(b, plan->n, st);
    dx.upload(x, plan->n, st);
    status = plan_solve(*plan, *opt, db.p, dx.p, rep);
    HR_CHECK_CUDA(cudaMemcpyAsync(x, dx.p, sizeof(double) * plan->n, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
    if (status == HR_ERR_NOT_CONVERGED) plan->C->err = "GMRES did not reach the tolerance";
  });
  return rc != HR_OK ? rc : status;
}

extern "C" int hr_plan2s_work(hr_plan2s* plan, int which, hr_work* w) {
  if (!plan || !w || which < 0 || which > 2) return HR_ERR_ARG;
  return guard(ctx_of(plan), [&] {
    plan_ready(*plan);
    if (which == 2) {
      // the inner treecode's stresslet batch, from its interaction lists (no launch)
      if (!plan->inner) throw Error(HR_ERR_STATE, "the plan has no inner treecode");
      const hr_plan2s::Inner& in = *plan->inner;
      memset(w, 0, sizeof(*w));
      for (int t = 0; t < 2; t++)
        for (const DevLists* L : {&in.Lon[t], &in.Loff[t]}) {
          w->direct_pairs_near += L->host.near_pairs_reg;
          w->direct_pairs_far += L->host.near_pairs_plain;
          w->proxy_pairs += L->host.proxy_pairs;
        }
      for (int s = 0; s < 2; s++) w->moment_terms += in.tree[s].moment_terms;
      w->flops = 0;  // the r <= 8 delta split of the direct pairs is only counted by a launch
      return;
    }
    cudaStream_t st = plan->C->stream;
    plan->counters.zero(st);
    DBuf<double> tmp;
    tmp.alloc(plan->n);
    const Batch* B;
    // one counting launch of the batch (ordinary launches skip the counts)
    struct Counting {
      Ctx& C;
      explicit Counting(Ctx& c) : C(c) { C.count_work = true; }
      ~Counting() { C.count_work = false; }
    } counting(*plan->C);
    if (which == 0) {
      HR_CHECK_CUDA(cudaMemsetAsync(tmp.p, 0, sizeof(double) * plan->n, st));
      plan_matvec(*plan, tmp.p, tmp.p, 0);
      B = &plan->dl[0];
    } else {
      HR_CHECK_CUDA(cudaMemsetAsync(plan->fin.p, 0, sizeof(double) * plan->n, st));
      plan_rhs(*plan, plan->fin.p, plan->fin.p + plan->off[1], tmp.p);
      B = &plan->sl;
    }
    unsigned long long c[32];
    HR_CHECK_CUDA(cudaMemcpyAsync(c, plan->counters.p, sizeof(c), cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
    memset(w, 0, sizeof(*w));
    double fl = 0;
    const int base = which == 0 ? 0 : 4;
    for (int t = 0; t < 4; t++) {
      const unsigned long long* q = c + 4 * (base + t);
      int kind = B->tasks[t].kind;
      Flops F = flops_of(kind);
      w->direct_pairs_near += (long long)(q[0] + q[1]);
      w->direct_pairs_far += (long long)q[2];
      w->proxy_pairs += (long long)q[3];
      fl += q[0] * F.reg + q[1] * F.near_plain + q[2] * F.far_target + q[3] * F.proxy;
    }
    if (plan->opt.mode == HR_TREE) {
      const int C = which == 0 ? 12 : 6;
      for (int s = 0; s < 2; s++) {
        w->moment_terms += plan->tree[s].moment_terms;
        fl += 2.0 * C * (double)plan->tree[s].moment_terms;
      }
    }
    w->flops = (long long)fl;
  });
}

extern "C" int hr_measure_fp64_peak(hr_ctx* ctx, double* flops_per_s) {
  if (!ctx || !flops_per_s) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    cudaStream_t st = ctx->c.stream;
    DBuf<double> o;
    o.alloc(1);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->c.device);
    const int blocks = sms * 8, iters = 1 << 14;
    launch_fma_peak(o.p, 256, blocks, st);  // warm-up
    cudaEvent_t a, b;
    HR_CHECK_CUDA(cudaEventCreate(&a));
    HR_CHECK_CUDA(cudaEventCreate(&b));
    HR_CHECK_CUDA(cudaEventRecord(a, st));
    launch_fma_peak(o.p, iters, blocks, st);
    HR_CHECK_CUDA(cudaEventRecord(b, st));
    HR_CHECK_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ctx->c.launches += 2;
    double fl = 2.0 * 8.0 * (double)iters * blocks * 256;
    *flops_per_s = fl / (ms * 1e-3);
  });
}

extern "C" int hr_plan2s_check_upward_pass(hr_plan2s* plan, const double* x, double* max_rel_err) {
  if (!plan || !x || !max_rel_err) return HR_ERR_ARG;
  return guard(ctx_of(plan), [&] {
    plan_ready(*plan);
    hr_plan2s& P = *plan;
    Ctx& C = *P.C;
    cudaStream_t st = C.stream;
    HR_REQUIRE(P.opt.mode == HR_TREE, "the upward pass exists in tree mode only");
    HR_CHECK_CUDA(cudaMemcpyAsync(P.xin.p, x, sizeof(double) * P.n, cudaMemcpyHostToDevice, st));
    double worst = 0.0;
    for (int s = 0; s < 2; s++) {
      DevTree& T = P.tree[s];
      const size_t m = (size_t)T.nn * 12 * T.Pf;
      std::vector<double> a(m), b(m);
      T.set_density(C, P.xin.p + P.off[s], true, true, false);
      HR_CHECK_CUDA(cudaMemcpyAsync(a.data(), T.mom.p, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
      HR_CHECK_CUDA(cudaStreamSynchronize(st));
      T.set_density(C, P.xin.p + P.off[s], true, true, true);
      HR_CHECK_CUDA(cudaMemcpyAsync(b.data(), T.mom.p, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
      HR_CHECK_CUDA(cudaStreamSynchronize(st));
      C.check_tc();
      // per node and stored channel (the 6 symmetric combinations of g (x) n
      // and n, 10 doubles per proxy), relative to that channel's largest FP64 value
      for (int nd = 0; nd < T.nn; nd++)
        for (int c = 0; c < 9; c++) {
          const double* pa = a.data() + (size_t)nd * 10 * T.Pf + c;
          const double* pb = b.data() + (size_t)nd * 10 * T.Pf + c;
          double mx = 0.0, dif = 0.0;
          for (int k = 0; k < T.Pf; k++) {
            mx = std::max(mx, fabs(pa[10 * k]));
            dif = std::max(dif, fabs(pa[10 * k] - pb[10 * k]));
          }
          if (mx > 0.0) worst = std::max(worst, dif / mx);
        }
    }
    *max_rel_err = worst;
  });
}

extern "C" int hr_measure_fp32_peak(hr_ctx* ctx, double* flops_per_s) {
  if (!ctx || !flops_per_s) return HR_ERR_ARG;
  return guard(ctx, [&] {
    HR_CHECK_CUDA(cudaSetDevice(ctx->c.device));
    cudaStream_t st = ctx->c.stream;
    DBuf<float> o;
    o.alloc(1);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->c.device);
    const int blocks = sms * 8, iters = 1 << 14;
    launch_fma_peak32(o.p, 256, blocks, st);  // warm-up
    cudaEvent_t a, b;
    HR_CHECK_CUDA(cudaEventCreate(&a));
    HR_CHECK_CUDA(cudaEventCreate(&b));
    HR_CHECK_CUDA(cudaEventRecord(a, st));
    launch_fma_peak32(o.p, iters, blocks, st);
    HR_CHECK_CUDA(cudaEventRecord(b, st));
    HR_CHECK_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    ctx->c.launches += 2;
    double fl = 2.0 * 16.0 * (double)iters * blocks * 256;
    *flops_per_s = fl / (ms * 1e-3);
  });
}

extern "C" int hr_plan2s_time_batch(hr_plan2s* plan, int which, int iters, double* ms_per_launch) {
  if (!plan || !ms_per_launch || iters < 1 || which < 0 || which > 3) return HR_ERR_ARG;
  return guard(ctx_of(plan), [&] {
    cudaStream_t st = plan->C->stream;
    HR_REQUIRE(which != 3 || plan->inner, "the plan has no inner treecode");
    plan_ready(*plan);
    if (which == 2 && !plan->dl[1].ready)
      dl_batches(*plan, plan->tree, plan->Lon, plan->Loff, plan->dl, 1, 2, true, plan->C->stream);
    Batch& B = which == 3 ? plan->inner->dl[1] : which == 1 ? plan->sl : plan->dl[which == 2 ? 1 : 0];
    cudaEvent_t a, b;
    HR_CHECK_CUDA(cudaEventCreate(&a));
    HR_CHECK_CUDA(cudaEventCreate(&b));
    B.launch(*plan->C);  // warm-up
    HR_CHECK_CUDA(cudaEventRecord(a, st));
    for (int i = 0; i < iters; i++) B.launch(*plan->C);
    HR_CHECK_CUDA(cudaEventRecord(b, st));
    HR_CHECK_CUDA(cudaEventSynchronize(b));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    HR_CHECK_CUDA(cudaGetLastError());
    *ms_per_launch = ms / iters;
  });
}
