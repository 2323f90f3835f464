// Test-only wrapper: exposes the UNMODIFIED reference extend-to-grid program
// (highreg_stokes_extend_to_grid/*.cpp, compiled from where it lies by
// oracle/build_oracle.py, its main() renamed, FFTW replaced by the test-only
// DST-I stand-in in oracle/fftw_standin/fftw3.h) through flat extern "C"
// entry points. Grids are exchanged as row-major (N+1)^3 arrays, index
// (i*(N+1)+j)*(N+1)+k, matching the reference's g[i][j][k].
//
// The scene follows E2G/main.cpp:66-165: L = 3, h = L/N, delta = kappa h^q,
// BAND1 = 4, BAND2 = 2, the exact translating-spheroid density.
//
// This file is oracle infrastructure: the product library never links it.
#include <cstring>
#include <sstream>
#include <string>

#include "stokes.h"  // pulls surface.h -> utilities.h

void solve_Poisson(int N, double L, double h, int*** nrst, int N_target,
                   const vector<Target_point>& Target, double*** p, double*** u, int variable);
void eval_p_BI_cubeEdges(int N, double h, int N_quad, const vector<Surf_point>& Surfc,
                         const vector<double>& f_ex, double*** p_bi);
void eval_p_BI_nearSurfc(int N, double h, double DEL, int N_quad, const vector<Surf_point>& Surfc,
                         int*** nrst, int N_target, const vector<Target_point>& Target,
                         const vector<double>& f_ex, double*** p_bi);
void eval_u_BI_cubeEdges(int N, double h, int N_quad, const vector<Surf_point>& Surfc,
                         const vector<double>& f_ex, double*** ux_bi, double*** uy_bi,
                         double*** uz_bi);
void eval_u_BI_nearSurfc(int N, double h, double DEL, int N_quad, const vector<Surf_point>& Surfc,
                         int*** nrst, int N_target, const vector<Target_point>& Target,
                         const vector<double>& f_ex, double*** ux_bi, double*** uy_bi,
                         double*** uz_bi);
void fftw_DST_Poisson3d_FD(int N, double* f);
void test_Stokes_Poisson3d_FD(double L, int N, double h, double DEL);

namespace {
int g_N = 0;
double g_L = 3.0, g_h = 0, g_DEL = 0;
vector<Surf_point> Surfc;
vector<double> f_ex;
vector<Target_point> Target;
int*** nrst = nullptr;
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

template <class T>
T*** alloc3(int N) {
  T*** a = new T**[N + 1];
  for (int i = 0; i <= N; i++) {
    a[i] = new T*[N + 1];
    for (int j = 0; j <= N; j++) a[i][j] = new T[N + 1]();
  }
  return a;
}
template <class T>
void free3(T*** a, int N) {
  if (!a) return;
  for (int i = 0; i <= N; i++) {
    for (int j = 0; j <= N; j++) delete[] a[i][j];
    delete[] a[i];
  }
  delete[] a;
}
template <class T>
void to3(const T* flat, T*** a, int N) {
  size_t m = N + 1;
  for (int i = 0; i <= N; i++)
    for (int j = 0; j <= N; j++) memcpy(a[i][j], flat + (i * m + j) * m, sizeof(T) * m);
}
template <class T>
void from3(T*** a, T* flat, int N) {
  size_t m = N + 1;
  for (int i = 0; i <= N; i++)
    for (int j = 0; j <= N; j++) memcpy(flat + (i * m + j) * m, a[i][j], sizeof(T) * m);
}
}  // namespace

extern "C" {

const char* refe2g_log() { return g_log.c_str(); }
void refe2g_clear_log() { g_log.clear(); }

// E2G/main.cpp:72-80 (h, delta) and 112-159 (surface, density, band tagging)
int refe2g_setup(int N) {
  CoutCapture cap;
  if (nrst) free3(nrst, g_N);
  g_N = N;
  g_L = 3.0;
  g_h = g_L / N;
  double kappa0 = 4.0, q = 5.0 / 7.0;
  double kappa = kappa0 * pow(1.0 / 64.0, 1.0 - q);
  g_DEL = kappa * pow(g_h, q);
  Surfc.clear();
  Target.clear();
  Generate_Surface(N, g_h, &Surfc);
  int nq = (int)Surfc.size();
  f_ex.assign(3 * nq, 0.0);
  for (int i = 0; i < nq; i++) {
    vector<double> fe = stokeslet_density(Surfc[i].x);
    for (int k = 0; k < 3; k++) f_ex[3 * i + k] = fe[k];
  }
  nrst = alloc3<int>(N);
  find_nrst_surfc(N, g_h, 4.0, 2.0, nq, Surfc, nrst, &Target);
  return 0;
}

void refe2g_counts(int* nq, int* nt, double* h, double* delta) {
  *nq = (int)Surfc.size();
  *nt = (int)Target.size();
  *h = g_h;
  *delta = g_DEL;
}

void refe2g_get_surface(double* xyz, double* nrml, double* area, double* f) {
  for (size_t i = 0; i < Surfc.size(); i++) {
    for (int k = 0; k < 3; k++) {
      xyz[3 * i + k] = Surfc[i].x[k];
      nrml[3 * i + k] = Surfc[i].Nrml[k];
      f[3 * i + k] = f_ex[3 * i + k];
    }
    area[i] = Surfc[i].Area;
  }
}

void refe2g_set_f(const double* f) { memcpy(f_ex.data(), f, sizeof(double) * f_ex.size()); }

void refe2g_get_targets(double* b, double* x0, double* n0, int* band2) {
  for (size_t i = 0; i < Target.size(); i++) {
    b[i] = Target[i].b;
    x0[3 * i] = Target[i].nrst_x;
    x0[3 * i + 1] = Target[i].nrst_y;
    x0[3 * i + 2] = Target[i].nrst_z;
    for (int k = 0; k < 3; k++) n0[3 * i + k] = Target[i].nrst_Nrml[k];
    band2[i] = Target[i].band2 ? 1 : 0;
  }
}

void refe2g_get_nrst(int* out) { from3(nrst, out, g_N); }

// E2G/main.cpp:1049-1116 — plain pressure on the six box faces, zero elsewhere.
void refe2g_eval_p_faces(double* p) {
  CoutCapture cap;
  double*** a = alloc3<double>(g_N);
  eval_p_BI_cubeEdges(g_N, g_h, (int)Surfc.size(), Surfc, f_ex, a);
  from3(a, p, g_N);
  free3(a, g_N);
}

// E2G/main.cpp:1120-1213 — regularized pressure at band points with b >= 0
// (in/out: other entries pass through).
void refe2g_eval_p_band(double* p) {
  CoutCapture cap;
  double*** a = alloc3<double>(g_N);
  to3(p, a, g_N);
  eval_p_BI_nearSurfc(g_N, g_h, g_DEL, (int)Surfc.size(), Surfc, nrst, (int)Target.size(), Target,
                      f_ex, a);
  from3(a, p, g_N);
  free3(a, g_N);
}

// E2G/main.cpp:1218-1299 — plain Stokeslet on the faces; (1,0,0) elsewhere.
void refe2g_eval_u_faces(double* ux, double* uy, double* uz) {
  CoutCapture cap;
  double ***a = alloc3<double>(g_N), ***b = alloc3<double>(g_N), ***c = alloc3<double>(g_N);
  eval_u_BI_cubeEdges(g_N, g_h, (int)Surfc.size(), Surfc, f_ex, a, b, c);
  from3(a, ux, g_N);
  from3(b, uy, g_N);
  from3(c, uz, g_N);
  free3(a, g_N);
  free3(b, g_N);
  free3(c, g_N);
}

// E2G/main.cpp:1303-1406 — regularized Stokeslet at band points with b >= 0.
void refe2g_eval_u_band(double* ux, double* uy, double* uz) {
  CoutCapture cap;
  double ***a = alloc3<double>(g_N), ***b = alloc3<double>(g_N), ***c = alloc3<double>(g_N);
  to3(ux, a, g_N);
  to3(uy, b, g_N);
  to3(uz, c, g_N);
  eval_u_BI_nearSurfc(g_N, g_h, g_DEL, (int)Surfc.size(), Surfc, nrst, (int)Target.size(), Target,
                      f_ex, a, b, c);
  from3(a, ux, g_N);
  from3(b, uy, g_N);
  from3(c, uz, g_N);
  free3(a, g_N);
  free3(b, g_N);
  free3(c, g_N);
}

// E2G/main.cpp:969-1044 — extension + 4th-order RHS + DST solve; u in/out.
void refe2g_solve_poisson(int variable, const double* p, double* u) {
  CoutCapture cap;
  double ***pa = alloc3<double>(g_N), ***ua = alloc3<double>(g_N);
  to3(p, pa, g_N);
  to3(u, ua, g_N);
  solve_Poisson(g_N, g_L, g_h, nrst, (int)Target.size(), Target, variable == 0 ? ua : pa, ua,
                variable);
  from3(ua, u, g_N);
  free3(pa, g_N);
  free3(ua, g_N);
}

// E2G/main.cpp:1423-1489 — DST-I Poisson solve of an n^3 row-major array.
void refe2g_dst_poisson(int n, double* f) { fftw_DST_Poisson3d_FD(n, f); }

// The whole driver E2G/main.cpp:107-964 (writes its slice files into cwd).
void refe2g_run(void) {
  CoutCapture cap;
  test_Stokes_Poisson3d_FD(g_L, g_N, g_h, g_DEL);
}

// Loads a scene from arrays instead of building it (the reference's own
// set-up at N = 384 takes minutes of serial work): quadrature points, the
// density, the tagged targets and the (N+1)^3 nearest-point index grid, in
// the layouts of refe2g_get_surface / refe2g_get_targets / refe2g_get_nrst.
void refe2g_load(int N, int nq, const double* xyz, const double* nrml, const double* area,
                 const double* f, int nt, const double* b, const double* x0, const double* n0,
                 const int* band2, const int* nrst_grid) {
  if (nrst) free3(nrst, g_N);
  g_N = N;
  g_L = 3.0;
  g_h = g_L / N;
  double kappa0 = 4.0, q = 5.0 / 7.0;
  double kappa = kappa0 * pow(1.0 / 64.0, 1.0 - q);
  g_DEL = kappa * pow(g_h, q);
  Surfc.assign(nq, Surf_point());
  f_ex.assign(f, f + 3 * (size_t)nq);
  for (int i = 0; i < nq; i++) {
    for (int k = 0; k < 3; k++) {
      Surfc[i].x[k] = xyz[3 * i + k];
      Surfc[i].Nrml[k] = nrml[3 * i + k];
    }
    Surfc[i].Area = area[i];
  }
  Target.assign(nt, Target_point());
  for (int i = 0; i < nt; i++) {
    Target[i].b = b[i];
    Target[i].nrst_x = x0[3 * i];
    Target[i].nrst_y = x0[3 * i + 1];
    Target[i].nrst_z = x0[3 * i + 2];
    for (int k = 0; k < 3; k++) Target[i].nrst_Nrml[k] = n0[3 * i + k];
    Target[i].band2 = band2[i] != 0;
  }
  nrst = alloc3<int>(N);
  to3(nrst_grid, nrst, N);
}

// Replaces the nearest-point index grid (e.g. one that keeps a sample of the
// tagged grid points and sets the rest to -1, so that the reference's band
// drivers evaluate only the sample).
void refe2g_set_nrst(const int* nrst_grid) { to3(nrst_grid, nrst, g_N); }

// The reference's plain sums (stokes_SL_away, stokes_pressure_away;
// E2G/stokes.cpp:13-45, 102-126) at arbitrary points, as its box-face drivers
// call them (E2G/main.cpp:1049-1116, 1218-1299): u (3 per point) and p.
void refe2g_away_points(int n, const double* xyz, double* u, double* p) {
  int nq = (int)Surfc.size();
#pragma omp parallel
  {
    vector<double> SL(3, 0.0);
#pragma omp for schedule(dynamic, 4)
    for (int i = 0; i < n; i++) {
      stokes_SL_away(nq, Surfc, f_ex, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2], SL);
      for (int k = 0; k < 3; k++) u[3 * i + k] = SL[k];
      p[i] = stokes_pressure_away(nq, Surfc, f_ex, xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]);
    }
  }
}

double refe2g_p_exact(double x, double y, double z) { return p_exact(x, y, z); }
void refe2g_u_exact(double x, double y, double z, double* u) {
  vector<double> v = SL_exact(x, y, z);
  u[0] = v[0];
  u[1] = v[1];
  u[2] = v[2];
}

void refe2g_lapl_dl_7ord(double r, double d, const double* c, double* s2) {
  Lapl_DL_7ord(r, d, c[0], c[1], c[2], *s2);
}

}  // extern "C"
