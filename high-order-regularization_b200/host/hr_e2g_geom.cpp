// hr_e2g_geom.cpp — host setup of the extend-to-grid problem: the translating
// prolate spheroid of highreg_stokes_extend_to_grid (semi-axes 1, .5, .5,
// centre (1.5, 1.5, 1.5), box [0, 3]^3, h = 3/N):
//   * quadrature points on grid-line crossings (Generate_Surface,
//     E2G/surface.cpp:12-66, grid offset by the centre),
//   * the exact surface force of the translating body (stokeslet_density,
//     E2G/utilities.cpp:267-285) and the exact pressure and velocity
//     (p_exact, SL_exact: E2G/utilities.cpp:294-411),
//   * the BAND1 = 4h / BAND2 = 2h tagging of grid points with their nearest
//     surface point and signed distance (find_nrst_surfc, E2G/surface.cpp:303-392).
// The reference tags grid points while scanning quadrature points in order,
// so the target numbering is "by first claiming quadrature point, then i, j,
// k"; the same numbering is produced here with a parallel first-claim pass.
#include <algorithm>
#include <atomic>
#include <memory>
#include <cmath>
#include <cstring>
#include <vector>

#include "hr_e2g_geom.h"

namespace e2g_setup {

constexpr double kPI = 3.14159265358979323846;
constexpr double kCtr = 1.5;                   // E2G/utilities.h:19
const double kAx[3] = {1.0, 0.5, 0.5};         // E2G/utilities.h:12-14

inline double phi(const double* y) {
  double x0 = y[0] - kCtr, x1 = y[1] - kCtr, x2 = y[2] - kCtr;
  return x0 * x0 / (kAx[0] * kAx[0]) + x1 * x1 / (kAx[1] * kAx[1]) + x2 * x2 / (kAx[2] * kAx[2]) - 1.0;
}
inline double dphi(int i, const double* y) { return 2.0 * (y[i] - kCtr) / (kAx[i] * kAx[i]); }

// stokeslet_density: E2G/utilities.cpp:267-285
void stokeslet_density(const double* pt, double* f) {
  double x = pt[0] - kCtr;
  double a = kAx[0], b = kAx[1];
  double a_sq = a * a, b_sq = b * b;
  double x_sq = x * x;
  double e_sq = 1.0 - b_sq / a_sq;
  double e = sqrt(e_sq);
  double Le = log((1.0 + e) / (1.0 - e));
  f[0] = 4.0 * e_sq * e * a / b / ((1.0 + e_sq) * Le - 2.0 * e) / sqrt(a_sq - e_sq * x_sq);
  f[1] = 0.0;
  f[2] = 0.0;
}

// p_exact: E2G/utilities.cpp:294-321
double p_exact(double xi, double yi, double zi) {
  double x = xi - kCtr, y = yi - kCtr, z = zi - kCtr;
  double a_sq = kAx[0] * kAx[0], b_sq = kAx[1] * kAx[1];
  double r_sq = y * y + z * z;
  double c = sqrt(a_sq - b_sq);
  double R1 = sqrt((x + c) * (x + c) + r_sq);
  double R2 = sqrt((x - c) * (x - c) + r_sq);
  double dB1dx = 1.0 / R1 - 1.0 / R2;
  double e = c / kAx[0];
  double Le = log((1.0 + e) / (1.0 - e));
  double a1 = e * e / ((1.0 + e * e) * Le - 2.0 * e);
  return -2.0 * a1 * dB1dx;
}

// SL_exact: E2G/utilities.cpp:360-411
void u_exact(double xi, double yi, double zi, double* u) {
  double x = xi - kCtr, y = yi - kCtr, z = zi - kCtr;
  double a_sq = kAx[0] * kAx[0], b_sq = kAx[1] * kAx[1];
  double r_sq = y * y + z * z;
  double c = sqrt(a_sq - b_sq);
  double R1 = sqrt((x + c) * (x + c) + r_sq);
  double R2 = sqrt((x - c) * (x - c) + r_sq);
  double R1c = R1 - (x + c);
  double R2c = R2 - (x - c);
  double B10;
  if (r_sq < 1.e-14) {
    if (x < 0) B10 = log((x - c) / (x + c));
    else B10 = log((x + c) / (x - c));
  } else {
    B10 = log(R2c / R1c);
  }
  double B30 = (x + c) / R1 - (x - c) / R2;
  double dB1dx = 1.0 / R1 - 1.0 / R2;
  double dB1dyz = 0.0;
  if (r_sq > 1.e-14) dB1dyz = 1.0 / R2 / R2c - 1.0 / R1 / R1c;
  double dB3dyz = 1.0 / R2 - 1.0 / R1 + x * dB1dyz;
  double e = c / kAx[0];
  double Le = log((1.0 + e) / (1.0 - e));
  double a1 = e * e / ((1.0 + e * e) * Le - 2.0 * e);
  double b1 = a1 * (1.0 - e * e) / (2.0 * e * e);
  u[0] = 2.0 * a1 * B10 - a1 * B30 + 2.0 * b1 * ((x - c) / R2 - (x + c) / R1 + B10 + x * dB1dx);
  double Er = a1 * (1.0 / R2 - 1.0 / R1) + 2.0 * b1 * dB3dyz;
  u[1] = Er * y;
  u[2] = Er * z;
}

namespace {
constexpr double kTol = 1e-14;
const double kTheta = 70.0 * kPI / 180.0;

double bump(double r) {
  double b = 0.0;
  if (fabs(r) < 1.0) {
    double r2 = r * r;
    b = exp(2.0 * r2 / (r2 - 1.0));
  }
  return b;
}
double part_unity(int i, const double* n) {
  double v[3] = {bump(acos(fabs(n[0])) / kTheta), bump(acos(fabs(n[1])) / kTheta),
                 bump(acos(fabs(n[2])) / kTheta)};
  double vs = v[0] + v[1] + v[2];
  return v[i] / vs;
}

double bisection(const double* PT, double H, int i, double a, double b) {
  double xl[3] = {PT[0], PT[1], PT[2]}, xr[3] = {PT[0], PT[1], PT[2]}, xm[3] = {PT[0], PT[1], PT[2]};
  xl[i] += a * H;
  xr[i] += b * H;
  if (phi(xl) * phi(xr) > 0.0) return 0.0;
  if (fabs(phi(xl)) <= kTol) return a;
  if (fabs(phi(xr)) <= kTol) return b;
  double p = (a + b) / 2;
  xm[i] = PT[i] + p * H;
  double pm = phi(xm);
  int guard = 0;
  while (fabs(pm) > kTol && guard++ < 2000) {
    if (phi(xl) * phi(xm) < 0.0) b = p;
    else {
      a = p;
      memcpy(xl, xm, sizeof(xl));
    }
    p = (a + b) / 2;
    xm[i] = PT[i] + p * H;
    pm = phi(xm);
  }
  return p;
}

// Newton: E2G/surface.cpp:88-128
double newton(const double* PT, double H, int i, double a, double b) {
  double xl[3] = {PT[0], PT[1], PT[2]}, xr[3] = {PT[0], PT[1], PT[2]}, xn[3] = {PT[0], PT[1], PT[2]};
  xl[i] += a * H;
  xr[i] += b * H;
  int n = 0;
  if (phi(xl) * phi(xr) > 0.0) return 0.0;
  if (fabs(phi(xl)) <= kTol) return a;
  if (fabs(phi(xr)) <= kTol) return b;
  double p = (a + b) / 2;
  xn[i] = PT[i] + p * H;
  double ph = phi(xn), dph = dphi(i, xn) * H;
  while ((fabs(ph) > kTol) && (fabs(dph) > kTol) && (n < 100)) {
    p -= ph / dph;
    xn[i] = PT[i] + p * H;
    n = n + 1;
    ph = phi(xn);
    dph = dphi(i, xn) * H;
  }
  if ((n >= 100) || (fabs(dph) <= kTol)) p = bisection(PT, H, i, a, b);
  return p;
}

int lu4(double A[4][4], int p[4]) {
  for (int j = 0; j < 4; j++) p[j] = j;
  for (int j = 0; j < 4; j++) {
    int k = j;
    double m = A[p[j]][j];
    for (int i = j + 1; i < 4; i++)
      if (fabs(A[p[i]][j]) > fabs(m)) {
        m = A[p[i]][j];
        k = i;
      }
    if (k != j) std::swap(p[j], p[k]);
    double ajj = A[p[j]][j];
    if (fabs(ajj) < 1.0e-15) return -1;
    for (int i = j + 1; i < 4; i++) {
      double lij = A[p[i]][j] / ajj;
      A[p[i]][j] = lij;
      for (int kk = j + 1; kk < 4; kk++) A[p[i]][kk] -= lij * A[p[j]][kk];
    }
  }
  return 0;
}
void lu4_solve(const double A[4][4], const int p[4], const double b[4], double x[4]) {
  x[0] = b[p[0]];
  for (int i = 1; i < 4; i++) {
    x[i] = b[p[i]];
    double rs = 0.0;
    for (int j = 0; j < i; j++) rs += A[p[i]][j] * x[j];
    x[i] -= rs;
  }
  x[3] = x[3] / A[p[3]][3];
  for (int i = 2; i >= 0; i--) {
    double rs = 0.0;
    for (int j = 3; j > i; j--) rs += A[p[i]][j] * x[j];
    x[i] = (x[i] - rs) / A[p[i]][i];
  }
}

// find_Nearest: E2G/surface.cpp:204-295
int find_nearest(const double* pt, const double* start, double* x0, double* n0, double* lam_out = nullptr) {
  double x[3] = {start[0], start[1], start[2]};
  double F[4] = {phi(x), x[0] - pt[0], x[1] - pt[1], x[2] - pt[2]};
  double Fn = F[0] * F[0] + F[1] * F[1] + F[2] * F[2] + F[3] * F[3];
  int n = 0;
  double lam = 0.0;
  const double H00 = 2.0 / (kAx[0] * kAx[0]), H11 = 2.0 / (kAx[1] * kAx[1]), H22 = 2.0 / (kAx[2] * kAx[2]);
  while ((Fn > kTol) && (n <= 100)) {
    double p1 = dphi(0, x), p2 = dphi(1, x), p3 = dphi(2, x);
    F[0] = phi(x);
    F[1] = x[0] - pt[0] + lam * p1;
    F[2] = x[1] - pt[1] + lam * p2;
    F[3] = x[2] - pt[2] + lam * p3;
    Fn = F[0] * F[0] + F[1] * F[1] + F[2] * F[2] + F[3] * F[3];
    double J[4][4] = {{0.0, p1, p2, p3},
                      {p1, 1.0 + lam * H00, lam * 0.0, lam * 0.0},
                      {p2, lam * 0.0, 1.0 + lam * H11, lam * 0.0},
                      {p3, lam * 0.0, lam * 0.0, 1.0 + lam * H22}};
    int perm[4];
    if (lu4(J, perm) == -1) return -1;
    double sol[4];
    lu4_solve(J, perm, F, sol);
    lam = lam - sol[0];
    for (int i = 0; i < 3; i++) x[i] = x[i] - sol[i + 1];
    n = n + 1;
  }
  if (n > 100) return -1;
  if (lam_out) *lam_out = lam;
  for (int k = 0; k < 3; k++) x0[k] = x[k];
  double a = dphi(0, x), b = dphi(1, x), c = dphi(2, x);
  double nn = sqrt(a * a + b * b + c * c);
  n0[0] = a / nn;
  n0[1] = b / nn;
  n0[2] = c / nn;
  return 0;
}
}  // namespace

// Generate_Surface (E2G/surface.cpp:12-66) + stokeslet_density + find_nrst_surfc.
void build(Scene& S, int N, double band1, double band2) {
  S.N = N;
  S.L = 3.0;
  S.h = S.L / N;
  const double h = S.h;
  const double kappa0 = 4.0, q = 5.0 / 7.0;  // E2G/main.cpp:76-80
  double kappa = kappa0 * pow(1.0 / 64.0, 1.0 - q);
  S.delta = kappa * pow(h, q);
  // quadrature points
  std::vector<std::vector<double>> per(3 * (2 * N + 1));
  const double cth = cos(kTheta);
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int i = 0; i < 3; i++)
    for (int l1 = -N; l1 <= N; l1++) {
      std::vector<double>& out = per[i * (2 * N + 1) + (l1 + N)];
      int i1 = i == 0 ? 1 : 0, i2 = i == 2 ? 1 : 2;
      double A[3] = {0, 0, 0}, B[3] = {0, 0, 0};
      for (int l2 = -N; l2 <= N; l2++) {
        A[i1] = l1 * h + kCtr;
        A[i2] = l2 * h + kCtr;
        B[i1] = l1 * h + kCtr;
        B[i2] = l2 * h + kCtr;
        // phi along the line is a quadratic in j, (j h / a_i)^2 + R: its sign
        // can change only within a few segments of the roots +-j*. Rounding
        // moves a sign change by far less than a segment, so the reference's
        // scan of every segment (E2G/surface.cpp:26-64) is run over windows of
        // 7 segments around the roots, in increasing j, with its own tests.
        double y0[3] = {A[0], A[1], A[2]};
        y0[i] = kCtr;
        const double R = phi(y0);
        if (R > 1e-10) continue;  // the line misses the surface
        const double root = R < 0.0 ? sqrt(-R) * kAx[i] / h : 0.0;
        const int ra = (int)floor(-root), rb = (int)floor(root);
        const int lo1 = std::max(-N, ra - 3), hi1 = std::min(N, ra + 3);
        const int lo2 = std::max(-N, std::max(rb - 3, hi1 + 1)), hi2 = std::min(N, rb + 3);
        const int win[2][2] = {{lo1, hi1}, {lo2, hi2}};
        for (const auto& wj : win)
          for (int j = wj[0]; j <= wj[1]; j++) {
            A[i] = j * h + kCtr;
            B[i] = A[i] + h;
            int sa = phi(A) < 0.0 ? -1 : 1, sb = phi(B) < 0.0 ? -1 : 1;
            if (sa * sb < 0) {
              double tau = newton(A, h, i, 0, 1);
              double x[3] = {A[0], A[1], A[2]};
              x[i] += tau * h;
              double nv[3];
              for (int k = 0; k < 3; k++) nv[k] = dphi(k, x);
              double nn = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
              for (int k = 0; k < 3; k++) nv[k] /= nn;
              if (fabs(nv[i]) >= cth) {
                double ar = h * h * part_unity(i, nv) / fabs(nv[i]);
                out.insert(out.end(), {x[0], x[1], x[2], nv[0], nv[1], nv[2], ar});
              }
            }
          }
      }
    }
  for (auto& v : per)
    for (size_t k = 0; k < v.size(); k += 7) {
      S.xq.insert(S.xq.end(), {v[k], v[k + 1], v[k + 2]});
      S.nrm.insert(S.nrm.end(), {v[k + 3], v[k + 4], v[k + 5]});
      S.area.push_back(v[k + 6]);
    }
  const int nq = (int)S.area.size();
  S.f.resize(3 * (size_t)nq);
  for (int j = 0; j < nq; j++) stokeslet_density(&S.xq[3 * j], &S.f[3 * j]);
  // band tagging: first quadrature point (in order) within (BAND1+1)h of a grid point
  const long M = N + 1;
  // (C++17: new std::atomic<int>[] leaves the values for the parallel fill)
  std::unique_ptr<std::atomic<int>[]> claim(new std::atomic<int>[M * M * M]);
#pragma omp parallel for schedule(static)
  for (long g = 0; g < M * M * M; g++) claim[g].store(nq, std::memory_order_relaxed);
  const double tol = 1.e-12;
  const int width = (int)ceil(band1);
#pragma omp parallel for schedule(dynamic, 256)
  for (int q2 = 0; q2 < nq; q2++) {
    const double* xs = &S.xq[3 * q2];
    int i0 = (int)floor(xs[0] / h - band1) - 1;
    int j0 = (int)floor(xs[1] / h - band1) - 1;
    int k0 = (int)floor(xs[2] / h - band1) - 1;
    // the reference's cube of grid points, each row (i, j) cut to the k that
    // can pass the distance test below (a slightly larger radius and one
    // point of slack on each side; the test itself is unchanged)
    const double rr = ((band1 + 1) * h + tol) * (1.0 + 1e-12) + 1e-15;
    for (int i = i0; i <= i0 + 2 * width + 3; i++)
      for (int j = j0; j <= j0 + 2 * width + 3; j++) {
        const double dx = i * h - xs[0], dy = j * h - xs[1];
        const double rem = rr * rr - dx * dx - dy * dy;
        if (rem < 0.0) continue;
        const double half = sqrt(rem);
        const int klo = std::max(k0, (int)floor((xs[2] - half) / h) - 1);
        const int khi = std::min(k0 + 2 * width + 3, (int)ceil((xs[2] + half) / h) + 1);
        for (int k = klo; k <= khi; k++) {
          if (i < 0 || j < 0 || k < 0 || i > N || j > N || k > N) continue;
          double pt[3] = {i * h, j * h, k * h};
          double d_sq = (pt[0] - xs[0]) * (pt[0] - xs[0]) + (pt[1] - xs[1]) * (pt[1] - xs[1]) +
                        (pt[2] - xs[2]) * (pt[2] - xs[2]);
          if (sqrt(d_sq) <= ((band1 + 1) * h + tol)) {
            std::atomic<int>& c = claim[((long)i * M + j) * M + k];
            int cur = c.load(std::memory_order_relaxed);
            while (q2 < cur && !c.compare_exchange_weak(cur, q2, std::memory_order_relaxed)) {
            }
          }
        }
      }
  }
  struct Tag {
    int q;
    long g;
    double b, x0[3], n0[3];
  };
  // claimed grid points in grid order: counted per i-plane, then filled
  std::vector<long> cand;
  {
    std::vector<long> cnt(M + 1, 0);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; i++) {
      long c = 0;
      for (long g = i * M * M; g < (i + 1) * M * M; g++) c += claim[g].load(std::memory_order_relaxed) < nq;
      cnt[i + 1] = c;
    }
    for (long i = 0; i < M; i++) cnt[i + 1] += cnt[i];
    cand.resize(cnt[M]);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; i++) {
      long o = cnt[i];
      for (long g = i * M * M; g < (i + 1) * M * M; g++)
        if (claim[g].load(std::memory_order_relaxed) < nq) cand[o++] = g;
    }
  }
  // quadrature points bucketed by grid cell (dense CSR table over the cells
  // the surface occupies, ascending point index per cell), for the retries below
  long cmin[3] = {0, 0, 0}, cmax[3] = {-1, -1, -1};
  std::vector<long> qcell(3 * (size_t)nq);
  for (int q2 = 0; q2 < nq; q2++)
    for (int d = 0; d < 3; d++) {
      const long c = (long)floor(S.xq[3 * q2 + d] / h);
      qcell[3 * q2 + d] = c;
      if (q2 == 0 || c < cmin[d]) cmin[d] = c;
      if (q2 == 0 || c > cmax[d]) cmax[d] = c;
    }
  const long cn[3] = {cmax[0] - cmin[0] + 1, cmax[1] - cmin[1] + 1, cmax[2] - cmin[2] + 1};
  auto cell_of = [&](long a, long b2, long c) -> long {
    if (a < cmin[0] || a > cmax[0] || b2 < cmin[1] || b2 > cmax[1] || c < cmin[2] || c > cmax[2]) return -1;
    return ((a - cmin[0]) * cn[1] + (b2 - cmin[1])) * cn[2] + (c - cmin[2]);
  };
  const long ncell = nq > 0 ? cn[0] * cn[1] * cn[2] : 0;
  std::vector<int> cstart(ncell + 1, 0), citems(nq);
  for (int q2 = 0; q2 < nq; q2++) cstart[cell_of(qcell[3 * q2], qcell[3 * q2 + 1], qcell[3 * q2 + 2]) + 1]++;
  for (long c = 0; c < ncell; c++) cstart[c + 1] += cstart[c];
  {
    std::vector<int> fill(cstart.begin(), cstart.end() - 1);
    for (int q2 = 0; q2 < nq; q2++) citems[fill[cell_of(qcell[3 * q2], qcell[3 * q2 + 1], qcell[3 * q2 + 2])]++] = q2;
  }
  std::vector<Tag> tags(cand.size());
  std::vector<uint8_t> ok(cand.size(), 0);
#pragma omp parallel for schedule(dynamic, 256)
  for (long c = 0; c < (long)cand.size(); c++) {
    long g = cand[c];
    int i = (int)(g / (M * M)), j = (int)((g / M) % M), k = (int)(g % M);
    double pt[3] = {i * h, j * h, k * h};
    // A point farther from the surface than the band can be tagged from no
    // start: find_nearest stops at a critical point of the distance (pt - x0
    // along the normal, to ~1e-14), whose |b| is then at least the distance d.
    // phi is quadratic with Hessian diag(2/a_i^2) <= 8, so |phi(pt)| <=
    // |grad phi(pt)| d + 4 d^2 bounds d from below, and such points (a fifth of
    // the candidates at N = 384, each tried from ~17 starts) are skipped with
    // the outcome every attempt would give.
    {
      const double g0 = dphi(0, pt), g1 = dphi(1, pt), g2 = dphi(2, pt);
      const double gn = sqrt(g0 * g0 + g1 * g1 + g2 * g2);
      const double dlow = (sqrt(gn * gn + 16.0 * fabs(phi(pt))) - gn) / 8.0;
      if (dlow > band1 * h + tol + 1e-10 * h) continue;
    }
    Tag t;
    t.g = g;
    t.q = claim[g].load(std::memory_order_relaxed);
    double lam = 0.0;
    bool converged = false;
    auto attempt = [&](int q2) {
      converged = false;
      if (find_nearest(pt, &S.xq[3 * q2], t.x0, t.n0, &lam) != 0) return false;
      converged = true;
      t.b = (pt[0] - t.x0[0]) * t.n0[0] + (pt[1] - t.x0[1]) * t.n0[1] + (pt[2] - t.x0[2]) * t.n0[2];
      return fabs(t.b) <= (band1 * h + tol);
    };
    bool tagged = attempt(t.q);
    // At a converged point pt - x0 = lam grad phi(x0); on this ellipsoid the
    // nearest surface point is the one critical point with 2 lam > -min a_i^2
    // (x0_i - c_i = a_i^2 (pt_i - c_i) / (a_i^2 + 2 lam), the root of a
    // decreasing function there), and |b| = |pt - x0| is then the distance.
    // When it already exceeds the band, every start ends at a point at least
    // as far, so the later attempts below would all fail.
    const bool nearest = converged && 2.0 * lam > -0.25 * (1.0 - 1e-6);  // min a_i^2 = 0.25
    if (!tagged && nearest && fabs(t.b) > band1 * h + tol + 1e-10 * h) continue;
    if (!tagged) {
      // The reference leaves the point untagged and tries again from every
      // later quadrature point whose neighbourhood contains it
      // (E2G/surface.cpp:325-358): same candidates, same order.
      std::vector<int> later;
      for (long a = i - 7; a <= i + 7; a++)
        for (long b2 = j - 7; b2 <= j + 7; b2++)
          for (long c2 = k - 7; c2 <= k + 7; c2++) {
            const long cell = cell_of(a, b2, c2);
            if (cell < 0) continue;
            for (int e = cstart[cell]; e < cstart[cell + 1]; e++) {
              int q2 = citems[e];
              if (q2 <= t.q) continue;
              const double* xs = &S.xq[3 * q2];
              double d_sq = (pt[0] - xs[0]) * (pt[0] - xs[0]) + (pt[1] - xs[1]) * (pt[1] - xs[1]) +
                            (pt[2] - xs[2]) * (pt[2] - xs[2]);
              if (sqrt(d_sq) <= ((band1 + 1) * h + tol)) later.push_back(q2);
            }
          }
      std::sort(later.begin(), later.end());
      for (int q2 : later) {
        if (attempt(q2)) {
          t.q = q2;
          tagged = true;
          break;
        }
      }
    }
    if (tagged) {
      tags[c] = t;
      ok[c] = 1;
    }
  }
  // reference order: by claiming quadrature point, then the i, j, k loop. The
  // candidates are in grid order, so a stable counting sort by q gives it.
  std::vector<long> qstart(nq + 1, 0);
  for (size_t c = 0; c < cand.size(); c++)
    if (ok[c]) qstart[tags[c].q + 1]++;
  for (int q2 = 0; q2 < nq; q2++) qstart[q2 + 1] += qstart[q2];
  const long nkept = qstart[nq];
  std::vector<Tag> kept(nkept);
  for (size_t c = 0; c < cand.size(); c++)
    if (ok[c]) kept[qstart[tags[c].q]++] = tags[c];
  S.nrst.resize(M * M * M);
#pragma omp parallel for schedule(static)
  for (long g = 0; g < M * M * M; g++) S.nrst[g] = -1;
  S.b.resize(nkept);
  S.x0.resize(3 * nkept);
  S.n0.resize(3 * nkept);
  S.band2.resize(nkept);
  S.g.resize(nkept);
#pragma omp parallel for schedule(static)
  for (long t = 0; t < nkept; t++) {
    const Tag& T = kept[t];
    S.nrst[T.g] = (int)t;
    S.g[t] = T.g;
    S.b[t] = T.b;
    for (int d = 0; d < 3; d++) {
      S.x0[3 * t + d] = T.x0[d];
      S.n0[3 * t + d] = T.n0[d];
    }
    S.band2[t] = fabs(T.b) <= band2 * h + tol ? 1 : 0;
  }
}

}  // namespace e2g_setup
