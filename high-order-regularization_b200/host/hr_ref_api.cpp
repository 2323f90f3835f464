// hr_ref_api.cpp — the reference's evaluator signatures (include/highreg_refapi.h)
// implemented over the C ABI. The reference's functions return nothing and
// print their problems; a failure here cannot be reported through the
// signature either, so it prints the library's message and aborts rather
// than return wrong numbers.
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "../../include/highreg_b200.h"
#include "../../include/highreg_refapi.h"

namespace {

struct State {
  hr_ctx* ctx = nullptr;
  int device = 0;
  int P = 6, N0 = 1000;  // 2S/KITC.h:14-16
  double theta = 0.6;    // 2S/KITC.h:17
  // treecode root centres by surf_num (2S/utilities.h:19-26)
  double ctr[3][3] = {{0, 0, 0}, {0, 0, -0.5 - 1.0 / (16.0 * 16.0 * 16.0)}, {0, 0, 0.5}};
};
State g;
std::mutex g_mu;

hr_ctx* context() {
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g.ctx) {
    int rc = hr_ctx_create(g.device, &g.ctx);
    if (rc != HR_OK) {
      fprintf(stderr, "highreg_refapi: no usable B200 (status %d)\n", rc);
      std::abort();
    }
  }
  return g.ctx;
}

void check(int rc) {
  if (rc != HR_OK) {
    fprintf(stderr, "highreg_refapi: %s (status %d)\n", hr_last_error(g.ctx), rc);
    std::abort();
  }
}

struct Soa {
  std::vector<double> xyz, nrml, area, dens;
  hr_surface s;
};

// density: 0 = f, 1 = g
void surface_of(const std::vector<Surf_point>& S, int n, int surf_num, int density, Soa& o) {
  o.xyz.resize(3 * (size_t)n);
  o.nrml.resize(3 * (size_t)n);
  o.area.resize(n);
  o.dens.resize(3 * (size_t)n);
  for (int i = 0; i < n; i++) {
    const std::vector<double>& q = density ? S[i].g : S[i].f;
    for (int k = 0; k < 3; k++) {
      o.xyz[3 * i + k] = S[i].x[k];
      o.nrml[3 * i + k] = S[i].Nrml[k];
      o.dens[3 * i + k] = q[k];
    }
    o.area[i] = S[i].Area;
  }
  o.s.n = n;
  o.s.xyz = o.xyz.data();
  o.s.nrml = o.nrml.data();
  o.s.area = o.area.data();
  o.s.plane = nullptr;
  int c = (surf_num >= 0 && surf_num <= 2) ? surf_num : 0;
  for (int k = 0; k < 3; k++) o.s.center[k] = g.ctr[c][k];
}

struct Tgt {
  std::vector<double> xyz, b, x0, n0, dens0;
  hr_targets t;
};

// dens0: 0 = nrst_f, 1 = nrst_g
void targets_of(const std::vector<Target_point>& T, int n, int dens0, Tgt& o) {
  o.xyz.resize(3 * (size_t)n);
  o.b.resize(n);
  o.x0.resize(3 * (size_t)n);
  o.n0.resize(3 * (size_t)n);
  o.dens0.resize(3 * (size_t)n);
  for (int i = 0; i < n; i++) {
    o.xyz[3 * i] = T[i].x;
    o.xyz[3 * i + 1] = T[i].y;
    o.xyz[3 * i + 2] = T[i].z;
    o.b[i] = T[i].b;
    o.x0[3 * i] = T[i].nrst_x;
    o.x0[3 * i + 1] = T[i].nrst_y;
    o.x0[3 * i + 2] = T[i].nrst_z;
    const std::vector<double>& d = dens0 ? T[i].nrst_g : T[i].nrst_f;
    for (int k = 0; k < 3; k++) {
      o.n0[3 * i + k] = T[i].nrst_Nrml[k];
      o.dens0[3 * i + k] = d[k];
    }
  }
  o.t.n = n;
  o.t.xyz = o.xyz.data();
  o.t.b = o.b.data();
  o.t.x0 = o.x0.data();
  o.t.n0 = o.n0.data();
  o.t.nrst = nullptr;
  o.t.i123 = nullptr;
}

hr_eval_opts opts(int mode) {
  hr_eval_opts o;
  o.mode = mode;
  o.P = g.P;
  o.N0 = g.N0;
  o.theta = g.theta;
  o.precision = HR_FP64;
  return o;
}

// on-surface evaluators: the targets are the quadrature points themselves
void on_surface(int kind, int mode, int surf_num, double DEL, int N_quad,
                const std::vector<Surf_point>& Surfc, int N_target, std::vector<double>& out) {
  if (N_target != N_quad) {
    fprintf(stderr, "highreg_refapi: on-surface targets must be the quadrature points\n");
    std::abort();
  }
  Soa s;
  surface_of(Surfc, N_quad, surf_num, kind, s);
  hr_eval_opts o = opts(mode);
  out.assign(3 * (size_t)N_target, 0.0);
  if (kind == 0) check(hr_stokes_sl_onsurf(context(), &o, DEL, &s.s, s.dens.data(), out.data()));
  else check(hr_stokes_dl_onsurf(context(), &o, DEL, &s.s, s.dens.data(), out.data()));
}

void off_surface(int kind, int mode, int surf_num, double DEL, int N_quad,
                 const std::vector<Surf_point>& Surfc, int N_target,
                 const std::vector<Target_point>& Target, std::vector<double>& out) {
  Soa s;
  surface_of(Surfc, N_quad, surf_num, kind, s);
  Tgt t;
  targets_of(Target, N_target, kind, t);
  hr_eval_opts o = opts(mode);
  out.assign(3 * (size_t)N_target, 0.0);
  if (kind == 0)
    check(hr_stokes_sl_offsurf(context(), &o, DEL, &s.s, s.dens.data(), &t.t, t.dens0.data(), out.data()));
  else
    check(hr_stokes_dl_offsurf(context(), &o, DEL, &s.s, s.dens.data(), &t.t, t.dens0.data(), out.data()));
}

}  // namespace

extern "C" void hr_refapi_set_tree(int P, int N0, double theta) {
  g.P = P;
  g.N0 = N0;
  g.theta = theta;
}
extern "C" void hr_refapi_set_center(int surf_num, double x, double y, double z) {
  if (surf_num < 0 || surf_num > 2) return;
  g.ctr[surf_num][0] = x;
  g.ctr[surf_num][1] = y;
  g.ctr[surf_num][2] = z;
}
extern "C" void hr_refapi_set_device(int device) { g.device = device; }

void eval_Stokes_SL_onSurf_tree(int surf_num, double, double DEL, int N_quad,
                                const std::vector<Surf_point>& Surfc, int N_target,
                                const std::vector<Target_point>&, std::vector<double>& SL) {
  on_surface(0, HR_TREE, surf_num, DEL, N_quad, Surfc, N_target, SL);
}
void eval_Stokes_SL_offSurf_tree(int surf_num, double, double DEL, int N_quad,
                                 const std::vector<Surf_point>& Surfc, int N_target,
                                 const std::vector<Target_point>& Target, std::vector<double>& SL) {
  off_surface(0, HR_TREE, surf_num, DEL, N_quad, Surfc, N_target, Target, SL);
}
void eval_Stokes_DL_onSurf_tree(int surf_num, double, double DEL, int N_quad,
                                const std::vector<Surf_point>& Surfc, int N_target,
                                const std::vector<Target_point>&, std::vector<double>& DL) {
  on_surface(1, HR_TREE, surf_num, DEL, N_quad, Surfc, N_target, DL);
}
void eval_Stokes_DL_offSurf_tree(int surf_num, double, double DEL, int N_quad,
                                 const std::vector<Surf_point>& Surfc, int N_target,
                                 const std::vector<Target_point>& Target, std::vector<double>& DL) {
  off_surface(1, HR_TREE, surf_num, DEL, N_quad, Surfc, N_target, Target, DL);
}
void eval_Stokes_SL_offSurf(double, double DEL, int N_quad, const std::vector<Surf_point>& Surfc,
                            int N_target, const std::vector<Target_point>& Target,
                            std::vector<double>& SL) {
  off_surface(0, HR_DIRECT, 0, DEL, N_quad, Surfc, N_target, Target, SL);
}
void eval_Stokes_SL_onSurf(double DEL, int N_quad, const std::vector<Surf_point>& Surfc, int N_target,
                           const std::vector<Target_point>&, std::vector<double>& SL_vec) {
  on_surface(0, HR_DIRECT, 0, DEL, N_quad, Surfc, N_target, SL_vec);
}
void eval_Stokes_DL_offSurf(double, double DEL, int N_quad, const std::vector<Surf_point>& Surfc,
                            int N_target, std::vector<Target_point>& Target,
                            std::vector<double>& DL_vec) {
  off_surface(1, HR_DIRECT, 0, DEL, N_quad, Surfc, N_target, Target, DL_vec);
}
void eval_Stokes_DL_onSurf(double DEL, int N_quad, const std::vector<Surf_point>& Surfc, int N_target,
                           std::vector<Target_point>&, std::vector<double>& DL_vec) {
  on_surface(1, HR_DIRECT, 0, DEL, N_quad, Surfc, N_target, DL_vec);
}
