// Test-only wrapper: exposes the UNMODIFIED reference two-surface program
// (highreg_stokes_2surf/*.cpp, compiled from where it lies by
// oracle/build_oracle.py) through flat extern "C" entry points, so that the
// oracle can drive the reference's own functions on identical inputs.
//
// It holds one "scene" exactly as 2S/main.cpp:67-130 and
// 2S/main.cpp:147-177 build it (two spheroids, on-surface targets, nearest
// data, interfacial forces) and forwards evaluations to the reference
// functions named in each comment. Nothing here re-implements the math.
//
// This file is oracle infrastructure: the product library never links it.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <unistd.h>

#include "stresslets.h"  // pulls stokeslets.h -> KITC.h -> surface.h -> utilities.h

// Defined in 2S/main.cpp (compiled with its main() renamed).
void test_Integral_Equation_gmres(double h, int N_quad1, vector<Surf_point>& Surfc1,
                                  int N_quad2, vector<Surf_point>& Surfc2, int N_target1,
                                  vector<Target_point>& Target1, int N_target2,
                                  vector<Target_point>& Target2);
void eval_SL(double h, double DEL_on, double DEL_off, int N_quad1, vector<Surf_point>& Surfc1,
             int N_quad2, vector<Surf_point>& Surfc2, int N_target1,
             vector<Target_point>& Target1, int N_target2, vector<Target_point>& Target2,
             vector<double>& SL_1, vector<double>& SL_2);
void solve_IE_1step(double h, double DEL_on, double DEL_off, int N_quad1,
                    vector<Surf_point>& Surfc1, int N_quad2, vector<Surf_point>& Surfc2,
                    int N_target1, vector<Target_point>& Target1, int N_target2,
                    vector<Target_point>& Target2, int n, const vector<double>& u_in,
                    vector<double>& u_out);
void interpolate_DL_density(int surf_num, double h, int N_quad, const vector<Surf_point>& Surfc,
                            int N_target, vector<Target_point>& Target);
void set_surface_force(int surf_num, int N_quad, vector<Surf_point>& Surfc);

namespace {
int g_N = 0;
double g_h = 0, g_DEL = 0;
vector<Surf_point> S[2];
vector<Target_point> T[2];
std::string g_log;

struct CoutCapture {
  std::stringstream ss;
  std::streambuf* old;
  CoutCapture() { old = std::cout.rdbuf(ss.rdbuf()); }
  ~CoutCapture() {
    std::cout.rdbuf(old);
    g_log += ss.str();
  }
};

// delta = kappa * h^q, kappa = kappa0 (1/64)^(1-q): 2S/main.cpp:147-157
double delta_of(double h) {
  double kappa0 = 4.0, q = 5.0 / 7.0;
  double kappa = kappa0 * pow(1.0 / 64.0, 1.0 - q);
  return kappa * pow(h, q);
}
}  // namespace

extern "C" {

const char* ref2s_log() { return g_log.c_str(); }
void ref2s_clear_log() { g_log.clear(); }

// Scene construction as in 2S/main.cpp:67-124 (surfaces at the origin,
// surface 2 rotated, then translated by ctr1/ctr2; targets = quadrature
// points) and 2S/main.cpp:165-174 (nearest data, interfacial force).
int ref2s_setup(int N) {
  CoutCapture cap;
  g_N = N;
  g_h = 1.0 / N;
  g_DEL = delta_of(g_h);
  for (int s = 0; s < 2; s++) {
    S[s].clear();
    T[s].clear();
  }
  Generate_Surface(0, 0, N, g_h, &S[0]);
  Generate_Surface(0, 1, N, g_h, &S[1]);
  for (auto& p : S[0]) { p.x[0] += ctr1_x; p.x[1] += ctr1_y; p.x[2] += ctr1_z; }
  for (auto& p : S[1]) { p.x[0] += ctr2_x; p.x[1] += ctr2_y; p.x[2] += ctr2_z; }
  Generate_Targets_OnSurface((int)S[0].size(), S[0], &T[0]);
  Generate_Targets_OnSurface((int)S[1].size(), S[1], &T[1]);
  Compute_nearest_data(1, 0, g_h, g_DEL, (int)S[0].size(), S[0], (int)T[1].size(), T[1]);
  Compute_nearest_data(2, 1, g_h, g_DEL, (int)S[1].size(), S[1], (int)T[0].size(), T[0]);
  set_surface_force(1, (int)S[0].size(), S[0]);
  set_surface_force(2, (int)S[1].size(), S[1]);
  return 0;
}

void ref2s_counts(int* nq1, int* nq2, double* h, double* delta) {
  *nq1 = (int)S[0].size();
  *nq2 = (int)S[1].size();
  *h = g_h;
  *delta = g_DEL;
}

// s = 0 or 1. Arrays are interleaved xyz (3n) as in the reference's f[3j+k].
void ref2s_get_surface(int s, double* xyz, double* nrml, double* area, int* plane, double* f,
                       double* g) {
  const auto& P = S[s];
  for (size_t i = 0; i < P.size(); i++) {
    for (int k = 0; k < 3; k++) {
      xyz[3 * i + k] = P[i].x[k];
      nrml[3 * i + k] = P[i].Nrml[k];
      f[3 * i + k] = P[i].f[k];
      g[3 * i + k] = P[i].g[k];
    }
    area[i] = P[i].Area;
    plane[i] = P[i].plane;
  }
}

void ref2s_set_f(int s, const double* f) {
  for (size_t i = 0; i < S[s].size(); i++)
    for (int k = 0; k < 3; k++) S[s][i].f[k] = f[3 * i + k];
}
void ref2s_set_g(int s, const double* g) {
  for (size_t i = 0; i < S[s].size(); i++)
    for (int k = 0; k < 3; k++) S[s][i].g[k] = g[3 * i + k];
}

// Target set t holds the quadrature points of surface t; its nearest data
// refers to the OTHER surface (2S/main.cpp:165-166).
void ref2s_get_targets(int t, double* b, double* x0, double* n0, double* f0, double* g0,
                       int* nrst, int* i123) {
  const auto& Q = T[t];
  for (size_t i = 0; i < Q.size(); i++) {
    b[i] = Q[i].b;
    x0[3 * i] = Q[i].nrst_x;
    x0[3 * i + 1] = Q[i].nrst_y;
    x0[3 * i + 2] = Q[i].nrst_z;
    for (int k = 0; k < 3; k++) {
      n0[3 * i + k] = Q[i].nrst_Nrml[k];
      f0[3 * i + k] = Q[i].nrst_f[k];
      g0[3 * i + k] = Q[i].nrst_g[k];
    }
    nrst[i] = Q[i].nrst;
    i123[3 * i] = Q[i].i1;
    i123[3 * i + 1] = Q[i].i2;
    i123[3 * i + 2] = Q[i].i3;
  }
}

void ref2s_set_nrst_g(int t, const double* g0) {
  for (size_t i = 0; i < T[t].size(); i++)
    for (int k = 0; k < 3; k++) T[t][i].nrst_g[k] = g0[3 * i + k];
}

// interpolate_DL_density (2S/main.cpp:916-1046) of surface s's density g at
// the nearest points of the other target set.
void ref2s_interpolate(int s) {
  CoutCapture cap;
  int t = 1 - s;
  interpolate_DL_density(s + 1, g_h, (int)S[s].size(), S[s], (int)T[t].size(), T[t]);
}

// One boundary sum of surface s's density at target set t.
//   kind 0: Stokeslet (f), kind 1: stresslet (g)
//   tree 1: eval_Stokes_*_tree (2S/KITC.cpp:1389-1830); 0: direct
//   (2S/stokeslets.cpp:12-180, 2S/stresslets.cpp:13-228)
void ref2s_eval(int kind, int tree, int s, int t, double* out) {
  CoutCapture cap;
  int nq = (int)S[s].size(), nt = (int)T[t].size();
  vector<double> res(3 * nt, 0.0);
  if (kind == 0) {
    if (s == t) {
      if (tree) eval_Stokes_SL_onSurf_tree(s + 1, g_h, g_DEL, nq, S[s], nt, T[t], res);
      else eval_Stokes_SL_onSurf(g_DEL, nq, S[s], nt, T[t], res);
    } else {
      if (tree) eval_Stokes_SL_offSurf_tree(s + 1, g_h, g_DEL, nq, S[s], nt, T[t], res);
      else eval_Stokes_SL_offSurf(g_h, g_DEL, nq, S[s], nt, T[t], res);
    }
  } else {
    if (s == t) {
      if (tree) eval_Stokes_DL_onSurf_tree(s + 1, g_h, g_DEL, nq, S[s], nt, T[t], res);
      else eval_Stokes_DL_onSurf(g_DEL, nq, S[s], nt, T[t], res);
    } else {
      if (tree) eval_Stokes_DL_offSurf_tree(s + 1, g_h, g_DEL, nq, S[s], nt, T[t], res);
      else eval_Stokes_DL_offSurf(g_h, g_DEL, nq, S[s], nt, T[t], res);
    }
  }
  memcpy(out, res.data(), sizeof(double) * 3 * nt);
}

// Right-hand side b = -(2/3) S[f] (2S/main.cpp:186-207).
void ref2s_rhs(double* b) {
  CoutCapture cap;
  int n1 = (int)T[0].size(), n2 = (int)T[1].size();
  vector<double> SL1(3 * n1, 0), SL2(3 * n2, 0);
  eval_SL(g_h, g_DEL, g_DEL, (int)S[0].size(), S[0], (int)S[1].size(), S[1], n1, T[0], n2, T[1],
          SL1, SL2);
  for (int i = 0; i < 3 * n1; i++) b[i] = -SL1[i] * (2.0 / 3.0);
  for (int i = 0; i < 3 * n2; i++) b[3 * n1 + i] = -SL2[i] * (2.0 / 3.0);
}

// Matrix-vector product u_out = (I - 2/3 D) u_in (2S/main.cpp:541-677).
void ref2s_matvec(const double* u_in, double* u_out) {
  CoutCapture cap;
  int n1 = (int)T[0].size(), n2 = (int)T[1].size();
  int n = 3 * (n1 + n2);
  vector<double> in(u_in, u_in + n), out(n, 0.0);
  solve_IE_1step(g_h, g_DEL, g_DEL, (int)S[0].size(), S[0], (int)S[1].size(), S[1], n1, T[0], n2,
                 T[1], n, in, out);
  memcpy(u_out, out.data(), sizeof(double) * n);
}

// The whole solve (2S/main.cpp:140-417). Writes the reference's vel1/vel2
// files into a scratch directory; returns the solution and the residual
// history parsed from the reference's own "Iteration j residual = r" lines.
int ref2s_solve(double* x_out, double* resid, int max_resid) {
  char tmpl[] = "/tmp/hr_ref2s_XXXXXX";
  char* dir = mkdtemp(tmpl);
  char cwd[4096];
  if (!getcwd(cwd, sizeof(cwd))) return -1;
  if (dir && chdir(dir) != 0) return -1;
  size_t log_start = g_log.size();
  {
    CoutCapture cap;
    int n1 = (int)T[0].size(), n2 = (int)T[1].size();
    test_Integral_Equation_gmres(g_h, (int)S[0].size(), S[0], (int)S[1].size(), S[1], n1, T[0],
                                 n2, T[1]);
    for (int i = 0; i < n1; i++) {
      x_out[3 * i] = T[0][i].u;
      x_out[3 * i + 1] = T[0][i].v;
      x_out[3 * i + 2] = T[0][i].w;
    }
    for (int i = 0; i < n2; i++) {
      x_out[3 * n1 + 3 * i] = T[1][i].u;
      x_out[3 * n1 + 3 * i + 1] = T[1][i].v;
      x_out[3 * n1 + 3 * i + 2] = T[1][i].w;
    }
  }
  if (chdir(cwd) != 0) return -1;
  if (dir) {
    std::string cmd = std::string("rm -rf ") + dir;
    if (system(cmd.c_str()) != 0) { /* scratch cleanup only */ }
  }
  int count = 0;
  std::istringstream in(g_log.substr(log_start));
  std::string line;
  while (std::getline(in, line)) {
    size_t p = line.find("Iteration ");
    size_t q = line.find("residual = ");
    if (p == 0 && q != std::string::npos && count < max_resid) {
      resid[count++] = atof(line.c_str() + q + 11);
    }
  }
  return count;
}

// Loads surface s and target set s from arrays instead of building them (the
// reference's own set-up scans every quadrature point per target and takes
// hours at h = 1/256). Layouts as in ref2s_get_surface / ref2s_get_targets;
// the target set s holds surface s's quadrature points with nearest data on
// the other surface. h and delta are the scene's.
void ref2s_load(int s, int n, const double* xyz, const double* nrml, const double* area,
                const double* f, const double* g, const double* b, const double* x0,
                const double* n0, const double* f0, const int* nrst_idx, const int* i123,
                double h, double delta) {
  g_h = h;
  g_DEL = delta;
  g_N = (int)lround(1.0 / h);
  S[s].assign(n, Surf_point());
  T[s].assign(n, Target_point());
  for (int i = 0; i < n; i++) {
    for (int k = 0; k < 3; k++) {
      S[s][i].x[k] = xyz[3 * i + k];
      S[s][i].Nrml[k] = nrml[3 * i + k];
      S[s][i].f[k] = f[3 * i + k];
      S[s][i].g[k] = g[3 * i + k];
      T[s][i].nrst_Nrml[k] = n0[3 * i + k];
      T[s][i].nrst_f[k] = f0[3 * i + k];
    }
    S[s][i].Area = area[i];
    T[s][i].x = xyz[3 * i];
    T[s][i].y = xyz[3 * i + 1];
    T[s][i].z = xyz[3 * i + 2];
    T[s][i].b = b[i];
    T[s][i].nrst_x = x0[3 * i];
    T[s][i].nrst_y = x0[3 * i + 1];
    T[s][i].nrst_z = x0[3 * i + 2];
    T[s][i].nrst = nrst_idx[i];
    T[s][i].i1 = i123[3 * i];
    T[s][i].i2 = i123[3 * i + 1];
    T[s][i].i3 = i123[3 * i + 2];
  }
}

// Direct (use_tree = 0) boundary sums of surface s's density at a sample of
// target set t, through the reference's own functions:
//   kind 0 Stokeslet, kind 1 stresslet;
//   s != t: eval_Stokes_SL_offSurf / eval_Stokes_DL_offSurf
//     (2S/stokeslets.cpp:12-86, 2S/stresslets.cpp:13-96) on the sampled
//     targets; for the stresslet, interpolate_DL_density (2S/main.cpp:916-1046)
//     first fills their nearest-point densities g0 (also written to g0_out);
//   s == t: the per-target on-surface sums stokes_SL_7ord_onSurf /
//     stokes_DL_7ord_onSurf (2S/stokeslets.cpp:188-225,
//     2S/stresslets.cpp:236-279) with the subtraction data the drivers
//     eval_Stokes_*_onSurf take from Surfc[i] (2S/stokeslets.cpp:167,
//     2S/stresslets.cpp:215-217).
void ref2s_sample_eval(int kind, int s, int t, int n, const int* idx, double* out, double* g0_out) {
  CoutCapture cap;
  int nq = (int)S[s].size();
  if (s != t) {
    vector<Target_point> sub(n);
    for (int i = 0; i < n; i++) sub[i] = T[t][idx[i]];
    vector<double> res(3 * n, 0.0);
    if (kind == 0) {
      eval_Stokes_SL_offSurf(g_h, g_DEL, nq, S[s], n, sub, res);
    } else {
      interpolate_DL_density(s + 1, g_h, nq, S[s], n, sub);
      if (g0_out)
        for (int i = 0; i < n; i++)
          for (int k = 0; k < 3; k++) g0_out[3 * i + k] = sub[i].nrst_g[k];
      eval_Stokes_DL_offSurf(g_h, g_DEL, nq, S[s], n, sub, res);
    }
    memcpy(out, res.data(), sizeof(double) * 3 * n);
    return;
  }
  vector<double> q(3 * nq);
  for (int j = 0; j < nq; j++)
    for (int k = 0; k < 3; k++) q[3 * j + k] = kind == 0 ? S[s][j].f[k] : S[s][j].g[k];
#pragma omp parallel
  {
    vector<double> res(3, 0.0);
#pragma omp for schedule(dynamic, 4)
    for (int m = 0; m < n; m++) {
      const int i = idx[m];
      const Surf_point& P = S[s][i];
      if (kind == 0) {
        double f0_dot_n0 = dot_product(P.f, P.Nrml);
        stokes_SL_7ord_onSurf(g_DEL, nq, S[s], q, f0_dot_n0, P.x[0], P.x[1], P.x[2], res);
      } else {
        stokes_DL_7ord_onSurf(g_DEL, nq, S[s], q, P.g, P.x[0], P.x[1], P.x[2], res);
      }
      for (int k = 0; k < 3; k++) out[3 * m + k] = res[k];
    }
  }
}

// Scalar kernels for kernel-level checks (2S/utilities.cpp:163-337).
void ref2s_reg_coeff(double lam, double* c) { get_reg_coeff_7ord(lam, c[0], c[1], c[2]); }
void ref2s_sl_7ord(double r, double d, const double* c, double* s) {
  Stokes_SL_7ord(r, d, c[0], c[1], c[2], s[0], s[1]);
}
void ref2s_sl_7ord_onsurf(double r, double d, double* s) { Stokes_SL_7ord_onSurf(r, d, s[0], s[1]); }
void ref2s_dl_7ord(double r, double d, const double* c, double* s) {
  Stokes_DL_7ord(r, d, c[0], c[1], c[2], s[0], s[1]);
}
void ref2s_dl_7ord_onsurf(double r, double d, double* s) { Stokes_DL_7ord_onSurf(r, d, s[0]); }

}  // extern "C"
