// hr_geometry.cpp — host setup that produces the boundary sums' inputs for the
// two-surface problem: quadrature points on grid-line crossings with
// partition-of-unity weights, nearest-point data of each surface's points
// with respect to the other surface, and the interfacial force.
//
// Follows 2S/surface.cpp and 2S/utilities.cpp, parameterized so that the
// spheroids' axes, centres and rotations can be chosen freely (the reference
// hard-codes them: 2S/utilities.h:15-26, 2S/utilities.cpp:10-40). With the
// default parameters every floating-point expression is the reference's, so
// the generated scene matches the reference bit for bit.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

#include <omp.h>

#include "../../include/highreg_b200.h"

namespace {

constexpr double kPI = 3.14159265358979323846;
constexpr double kTol = 1e-14;                   // 2S/utilities.h:14
const double kTheta = 70.0 * kPI / 180.0;        // 2S/utilities.h:13

struct Spheroid {
  double a2[3];
  double ctr[3];
  double R[3][3];  // un-rotation: body coordinates = R (x - ctr)
  bool rotated;
  bool centered;   // generation uses the uncentred level set (surf_num = 0)

  // phi: 2S/utilities.cpp:58-86
  double phi(const double* x) const {
    double xx[3] = {x[0], x[1], x[2]};
    if (centered)
      for (int k = 0; k < 3; k++) xx[k] = x[k] - ctr[k];
    if (rotated) {
      double u[3] = {0, 0, 0};
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) u[i] += R[i][j] * xx[j];
      return u[0] * u[0] / a2[0] + u[1] * u[1] / a2[1] + u[2] * u[2] / a2[2] - 1.0;
    }
    return xx[0] * xx[0] / a2[0] + xx[1] * xx[1] / a2[1] + xx[2] * xx[2] / a2[2] - 1.0;
  }
  // Dphi: 2S/utilities.cpp:91-121
  double dphi(int i, const double* x) const {
    double xx[3] = {x[0], x[1], x[2]};
    if (centered)
      for (int k = 0; k < 3; k++) xx[k] = x[k] - ctr[k];
    if (rotated) {
      double u[3] = {0, 0, 0};
      for (int r = 0; r < 3; r++)
        for (int j = 0; j < 3; j++) u[r] += R[r][j] * xx[j];
      double d[3] = {2.0 * u[0] / a2[0], 2.0 * u[1] / a2[1], 2.0 * u[2] / a2[2]};
      return d[0] * R[0][i] + d[1] * R[1][i] + d[2] * R[2][i];
    }
    return 2.0 * xx[i] / a2[i];
  }
  // D2phi: 2S/utilities.cpp:126-158
  void d2phi(double H[3][3]) const {
    if (rotated) {
      double A0 = 2.0 / a2[0], A1 = 2.0 / a2[1], A2 = 2.0 / a2[2];
      for (int i = 0; i < 3; i++)
        for (int j = i; j < 3; j++)
          H[i][j] = A0 * R[0][i] * R[0][j] + A1 * R[1][i] * R[1][j] + A2 * R[2][i] * R[2][j];
      H[1][0] = H[0][1];
      H[2][0] = H[0][2];
      H[2][1] = H[1][2];
    } else {
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) H[i][j] = 0.0;
      H[0][0] = 2.0 / a2[0];
      H[1][1] = 2.0 / a2[1];
      H[2][2] = 2.0 / a2[2];
    }
  }
};

// bump, Part_Unity: 2S/surface.cpp:181-207
double bump(double r) {
  if (fabs(r) < 1.0) {
    double r2 = r * r;
    return exp(2.0 * r2 / (r2 - 1.0));
  }
  return 0.0;
}
double part_unity(int i, const double* n) {
  double v0 = bump(acos(fabs(n[0])) / kTheta);
  double v1 = bump(acos(fabs(n[1])) / kTheta);
  double v2 = bump(acos(fabs(n[2])) / kTheta);
  double vs = v0 + v1 + v2;
  double v[3] = {v0, v1, v2};
  return v[i] / vs;
}

// bisection: 2S/surface.cpp:139-174
double bisection(const Spheroid& S, const double* PT, double H, int i, double a, double b) {
  double xl[3] = {PT[0], PT[1], PT[2]}, xr[3] = {PT[0], PT[1], PT[2]}, xm[3] = {PT[0], PT[1], PT[2]};
  xl[i] += a * H;
  xr[i] += b * H;
  double p = 0.0;
  if (S.phi(xl) * S.phi(xr) > 0.0) return p;
  if (fabs(S.phi(xl)) <= kTol) return a;
  if (fabs(S.phi(xr)) <= kTol) return b;
  p = (a + b) / 2;
  xm[i] = PT[i] + p * H;
  double pm = S.phi(xm);
  int guard = 0;
  while (fabs(pm) > kTol && guard++ < 2000) {
    if (S.phi(xl) * S.phi(xm) < 0.0) b = p;
    else {
      a = p;
      memcpy(xl, xm, sizeof(xl));
    }
    p = (a + b) / 2;
    xm[i] = PT[i] + p * H;
    pm = S.phi(xm);
  }
  return p;
}

// Newton: 2S/surface.cpp:95-135
double newton(const Spheroid& S, const double* PT, double H, int i, double a, double b) {
  const int n_max = 100;
  double xl[3] = {PT[0], PT[1], PT[2]}, xr[3] = {PT[0], PT[1], PT[2]}, xn[3] = {PT[0], PT[1], PT[2]};
  xl[i] += a * H;
  xr[i] += b * H;
  int n = 0;
  double p = 0.0;
  if (S.phi(xl) * S.phi(xr) > 0.0) return p;
  if (fabs(S.phi(xl)) <= kTol) return a;
  if (fabs(S.phi(xr)) <= kTol) return b;
  p = (a + b) / 2;
  xn[i] = PT[i] + p * H;
  double ph = S.phi(xn);
  double dph = S.dphi(i, xn) * H;
  while ((fabs(ph) > kTol) && (fabs(dph) > kTol) && (n < n_max)) {
    p -= ph / dph;
    xn[i] = PT[i] + p * H;
    n = n + 1;
    ph = S.phi(xn);
    dph = S.dphi(i, xn) * H;
  }
  if ((n >= n_max) || (fabs(dph) <= kTol)) p = bisection(S, PT, H, i, a, b);
  return p;
}

struct QPoint {
  double x[3], n[3], area;
  int plane;
};

// Segments of grid line {A + t h e_i} (j = t) on which the reference's scan
// (Generate_Surface, 2S/surface.cpp:26-66) can see a sign change of phi.
// Along the line phi is the quadratic alpha j^2 + beta j + gamma (alpha > 0):
// rounding (~1e-14 here) can flip its sign only where |phi| < 1e-13, i.e.
// within a tiny distance of a real root or of the vertex of a quadratic whose
// minimum is below 1e-12. Windows of 7 segments around the two roots (or the
// vertex) keep every sign change; the scan runs over them in increasing j with
// the reference's own tests. Returns false when the line misses the surface.
bool line_windows(const Spheroid& S, const double* A, int i, double h, double off_i, int N, int lo[2],
                  int hi[2]) {
  double x0[3] = {A[0], A[1], A[2]};
  x0[i] = off_i;
  if (S.centered)
    for (int k = 0; k < 3; k++) x0[k] -= S.ctr[k];
  double u0[3], r[3];
  for (int k = 0; k < 3; k++) {
    if (S.rotated) {
      u0[k] = S.R[k][0] * x0[0] + S.R[k][1] * x0[1] + S.R[k][2] * x0[2];
      r[k] = S.R[k][i];
    } else {
      u0[k] = x0[k];
      r[k] = k == i ? 1.0 : 0.0;
    }
  }
  double alpha = 0.0, beta = 0.0, gamma = -1.0;
  for (int k = 0; k < 3; k++) {
    alpha += h * h * r[k] * r[k] / S.a2[k];
    beta += 2.0 * h * u0[k] * r[k] / S.a2[k];
    gamma += u0[k] * u0[k] / S.a2[k];
  }
  const double v = -beta / (2.0 * alpha);
  const double minval = gamma - beta * beta / (4.0 * alpha);
  if (minval > 1e-12) return false;
  const double half = sqrt(std::max(0.0, -minval / alpha));
  const int ra = (int)std::max(-1e9, std::min(1e9, floor(v - half)));
  const int rb = (int)std::max(-1e9, std::min(1e9, floor(v + half)));
  lo[0] = std::max(-N, ra - 3);
  hi[0] = std::min(N, ra + 3);
  lo[1] = std::max(-N, std::max(rb - 3, hi[0] + 1));
  hi[1] = std::min(N, rb + 3);
  return true;
}

// Generate_Surface: 2S/surface.cpp:13-71 (grid at origin + offset; points
// translated by shift afterwards).
std::vector<QPoint> generate_surface(const Spheroid& S, int N, double h, const double off[3],
                                     const double shift[3]) {
  std::vector<std::vector<QPoint>> per(3 * (2 * N + 1));
  const double cth = cos(kTheta);
#pragma omp parallel for schedule(dynamic, 1) collapse(2)
  for (int i = 0; i < 3; i++) {
    for (int l1 = -N; l1 <= N; l1++) {
      std::vector<QPoint>& out = per[i * (2 * N + 1) + (l1 + N)];
      double A[3] = {0, 0, 0}, B[3] = {0, 0, 0};
      int i1 = i == 0 ? 1 : 0, i2 = i == 2 ? 1 : 2;
      for (int l2 = -N; l2 <= N; l2++) {
        A[i1] = l1 * h + off[i1];
        A[i2] = l2 * h + off[i2];
        B[i1] = l1 * h + off[i1];
        B[i2] = l2 * h + off[i2];
        int lo[2], hi[2];
        if (!line_windows(S, A, i, h, off[i], N, lo, hi)) continue;  // the line misses the surface
        for (int w = 0; w < 2; w++)
          for (int j = lo[w]; j <= hi[w]; j++) {
            A[i] = j * h + off[i];
            B[i] = A[i] + h;
            int sa = S.phi(A) < 0.0 ? -1 : 1, sb = S.phi(B) < 0.0 ? -1 : 1;
            if (sa * sb < 0) {
              double tau = newton(S, A, h, i, 0, 1);
              QPoint q;
              q.x[0] = A[0];
              q.x[1] = A[1];
              q.x[2] = A[2];
              q.x[i] += tau * h;
              for (int k = 0; k < 3; k++) q.n[k] = S.dphi(k, q.x);
              double nn = sqrt(q.n[0] * q.n[0] + q.n[1] * q.n[1] + q.n[2] * q.n[2]);
              for (int k = 0; k < 3; k++) q.n[k] /= nn;
              if (fabs(q.n[i]) >= cth) {
                q.area = h * h * part_unity(i, q.n) / fabs(q.n[i]);
                q.plane = i;
                out.push_back(q);
              }
            }
          }
      }
    }
  }
  std::vector<QPoint> all;
  for (auto& v : per)
    for (auto& q : v) {
      for (int k = 0; k < 3; k++) q.x[k] += shift[k];
      all.push_back(q);
    }
  return all;
}

// LU_factorization + solveByLU: 2S/utilities.cpp:361-431 (4x4)
int lu4(double A[4][4], int p[4]) {
  const int n = 4;
  for (int j = 0; j < n; j++) p[j] = j;
  for (int j = 0; j < n; j++) {
    int k = j;
    double m = A[p[j]][j];
    for (int i = j + 1; i < n; i++)
      if (fabs(A[p[i]][j]) > fabs(m)) {
        m = A[p[i]][j];
        k = i;
      }
    if (k != j) std::swap(p[j], p[k]);
    double ajj = A[p[j]][j];
    if (fabs(ajj) < 1.0e-15) return -1;
    for (int i = j + 1; i < n; i++) {
      double lij = A[p[i]][j] / ajj;
      A[p[i]][j] = lij;
      for (int kk = j + 1; kk < n; kk++) A[p[i]][kk] -= lij * A[p[j]][kk];
    }
  }
  return 0;
}
void lu4_solve(const double A[4][4], const int p[4], const double b[4], double x[4]) {
  const int n = 4;
  x[0] = b[p[0]];
  for (int i = 1; i < n; i++) {
    x[i] = b[p[i]];
    double rs = 0.0;
    for (int j = 0; j < i; j++) rs += A[p[i]][j] * x[j];
    x[i] -= rs;
  }
  x[n - 1] = x[n - 1] / A[p[n - 1]][n - 1];
  for (int i = n - 2; i >= 0; i--) {
    double rs = 0.0;
    for (int j = n - 1; j > i; j--) rs += A[p[i]][j] * x[j];
    x[i] = (x[i] - rs) / A[p[i]][i];
  }
}

// find_Nearest_Start: 2S/surface.cpp:277-365 (Newton on the Lagrange system)
int nearest_point(const Spheroid& S, const double* pt, const double* start, double* x0,
                  double* n0) {
  const int n_max = 100;
  double x[3] = {start[0], start[1], start[2]};
  double lam = 0.0;
  int n = 0;
  double F[4];
  F[0] = S.phi(x);
  F[1] = x[0] - pt[0];
  F[2] = x[1] - pt[1];
  F[3] = x[2] - pt[2];
  double Fn = F[0] * F[0] + F[1] * F[1] + F[2] * F[2] + F[3] * F[3];
  double H[3][3];
  S.d2phi(H);
  while ((Fn > kTol) && (n <= n_max)) {
    double p1 = S.dphi(0, x), p2 = S.dphi(1, x), p3 = S.dphi(2, x);
    F[0] = S.phi(x);
    F[1] = x[0] - pt[0] + lam * p1;
    F[2] = x[1] - pt[1] + lam * p2;
    F[3] = x[2] - pt[2] + lam * p3;
    Fn = F[0] * F[0] + F[1] * F[1] + F[2] * F[2] + F[3] * F[3];
    double J[4][4] = {{0.0, p1, p2, p3},
                      {p1, 1.0 + lam * H[0][0], lam * H[0][1], lam * H[0][2]},
                      {p2, lam * H[1][0], 1.0 + lam * H[1][1], lam * H[1][2]},
                      {p3, lam * H[2][0], lam * H[2][1], 1.0 + lam * H[2][2]}};
    int perm[4];
    if (lu4(J, perm) == -1) return -1;
    double sol[4];
    lu4_solve(J, perm, F, sol);
    lam = lam - sol[0];
    for (int i = 0; i < 3; i++) x[i] = x[i] - sol[i + 1];
    n = n + 1;
  }
  if (n > n_max) return -1;
  for (int k = 0; k < 3; k++) x0[k] = x[k];
  double a = S.dphi(0, x), b = S.dphi(1, x), c = S.dphi(2, x);
  double nn = sqrt(a * a + b * b + c * c);
  n0[0] = a / nn;
  n0[1] = b / nn;
  n0[2] = c / nn;
  return 0;
}

// select_Monge_Patch: 2S/surface.cpp:395-431
void monge(const Spheroid& S, const double* x, int& i1, int& i2, int& i3) {
  double nx = fabs(S.dphi(0, x)), ny = fabs(S.dphi(1, x)), nz = fabs(S.dphi(2, x));
  if (nx >= ny) {
    if (nx >= nz) {
      i1 = 1;
      i2 = 2;
      i3 = 0;
    } else {
      i1 = 0;
      i2 = 1;
      i3 = 2;
    }
  } else {
    if (ny >= nz) {
      i1 = 0;
      i2 = 2;
      i3 = 1;
    } else {
      i1 = 0;
      i2 = 1;
      i3 = 2;
    }
  }
}

// mean_curvature (spheroid formula): 2S/surface.cpp:214-248
double mean_curvature(const Spheroid& S, const double axes[3], const double* x) {
  double a = axes[1], c = axes[0];
  double a_sq = a * a;
  double xx[3] = {x[0] - S.ctr[0], x[1] - S.ctr[1], x[2] - S.ctr[2]};
  double cos_sq;
  if (S.rotated) {
    double u[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) u[i] += S.R[i][j] * xx[j];
    cos_sq = (u[1] * u[1] + u[2] * u[2]) / a_sq;
  } else {
    cos_sq = (xx[1] * xx[1] + xx[2] * xx[2]) / a_sq;
  }
  double temp = a_sq + (c * c - a_sq) * cos_sq;
  return c * (a_sq + temp) / (2.0 * a * sqrt(temp * temp * temp));
}

// surfc_force: 2S/surface.cpp:530-559 (gamma = 1 + z^2, f = 2 H gamma n - grad_s gamma).
// body_z: z is the body-frame coordinate (row 2 of the un-rotation), so the
// tension field turns with the surface; otherwise the reference's z - centre_z.
void surface_force(const Spheroid& S, const double axes[3], const double* x0, const double* n0,
                   double* f, bool body_z = false) {
  double H = mean_curvature(S, axes, x0);
  double zz = x0[2] - S.ctr[2];
  double Dgx = 0.0, Dgy = 0.0, Dgz = 2.0 * zz;
  if (body_z && S.rotated) {
    zz = S.R[2][0] * (x0[0] - S.ctr[0]) + S.R[2][1] * (x0[1] - S.ctr[1]) + S.R[2][2] * (x0[2] - S.ctr[2]);
    Dgx = 2.0 * zz * S.R[2][0];
    Dgy = 2.0 * zz * S.R[2][1];
    Dgz = 2.0 * zz * S.R[2][2];
  }
  double gamma = 1.0 + zz * zz;
  double Dgn = Dgx * n0[0] + Dgy * n0[1] + Dgz * n0[2];
  double sg0 = Dgx - Dgn * n0[0], sg1 = Dgy - Dgn * n0[1], sg2 = Dgz - Dgn * n0[2];
  gamma *= 2.0 * H;
  f[0] = gamma * n0[0] - sg0;
  f[1] = gamma * n0[1] - sg1;
  f[2] = gamma * n0[2] - sg2;
}

// find_Nearest_grid (2S/surface.cpp:370-390): nearest quadrature point of a
// plane family, first index on ties, none beyond distance^2 = 100. A k-d
// tree over each family's points (median splits on the widest axis, leaves of
// at most kLeaf points, tight bounding boxes) is searched nearer child first;
// a subtree is skipped only when the squared distance from the point to its
// box exceeds the best squared distance found so far by more than a 1e-12
// relative margin (for rounding), so every point at the best distance is met
// and the lowest index among equals wins: the same index as the reference's
// linear scan.
struct PointTree {
  static constexpr int kLeaf = 16;
  struct Node {
    double lo[3], hi[3];
    int child[2];  // -1 for a leaf
    int begin, end;
  };
  std::vector<Node> nodes[3];  // per plane family; node 0 is the root
  std::vector<int> ids[3];     // point indices in leaf order
  std::vector<double> pts[3];  // their coordinates, packed in the same order

  int make(int f, const std::vector<QPoint>& P, int b, int e) {
    Node nd;
    for (int k = 0; k < 3; k++) {
      nd.lo[k] = 1e300;
      nd.hi[k] = -1e300;
    }
    for (int i = b; i < e; i++)
      for (int k = 0; k < 3; k++) {
        nd.lo[k] = std::min(nd.lo[k], P[ids[f][i]].x[k]);
        nd.hi[k] = std::max(nd.hi[k], P[ids[f][i]].x[k]);
      }
    nd.child[0] = nd.child[1] = -1;
    nd.begin = b;
    nd.end = e;
    const int me = (int)nodes[f].size();
    nodes[f].push_back(nd);
    if (e - b > kLeaf) {
      int ax = 0;
      for (int k = 1; k < 3; k++)
        if (nd.hi[k] - nd.lo[k] > nd.hi[ax] - nd.lo[ax]) ax = k;
      const int mid = (b + e) / 2;
      std::nth_element(ids[f].begin() + b, ids[f].begin() + mid, ids[f].begin() + e,
                       [&](int u, int v) { return P[u].x[ax] < P[v].x[ax]; });
      const int l = make(f, P, b, mid);
      const int r = make(f, P, mid, e);
      nodes[f][me].child[0] = l;
      nodes[f][me].child[1] = r;
    }
    return me;
  }

  void build(const std::vector<QPoint>& P) {
    for (int f = 0; f < 3; f++) {
      ids[f].clear();
      nodes[f].clear();
      for (size_t j = 0; j < P.size(); j++)
        if (P[j].plane == f) ids[f].push_back((int)j);
      if (!ids[f].empty()) make(f, P, 0, (int)ids[f].size());
      pts[f].resize(3 * ids[f].size());
      for (size_t i = 0; i < ids[f].size(); i++)
        for (int k = 0; k < 3; k++) pts[f][3 * i + k] = P[ids[f][i]].x[k];
    }
  }

  static double box_d2(const Node& nd, const double* pt) {
    double d2 = 0;
    for (int k = 0; k < 3; k++) {
      double d = 0;
      if (pt[k] < nd.lo[k]) d = nd.lo[k] - pt[k];
      else if (pt[k] > nd.hi[k]) d = pt[k] - nd.hi[k];
      d2 += d * d;
    }
    return d2;
  }

  int nearest(const double* pt, int f) const {
    if (nodes[f].empty()) return -1;
    int i0 = -1;
    double best = 100.0;
    int stack[128];
    int top = 0;
    stack[top++] = 0;
    while (top > 0) {
      const Node& nd = nodes[f][stack[--top]];
      if (box_d2(nd, pt) > best * (1.0 + 1e-12) + 1e-300) continue;
      if (nd.child[0] < 0) {
        for (int i = nd.begin; i < nd.end; i++) {
          const double* x = &pts[f][3 * i];
          const int j = ids[f][i];
          double dist = (pt[0] - x[0]) * (pt[0] - x[0]) + (pt[1] - x[1]) * (pt[1] - x[1]) +
                        (pt[2] - x[2]) * (pt[2] - x[2]);
          if (dist < best || (dist == best && i0 >= 0 && j < i0)) {
            best = dist;
            i0 = j;
          }
        }
        continue;
      }
      // push the farther child first so the nearer one is searched first
      const int a = nd.child[0], b = nd.child[1];
      const bool a_near = box_d2(nodes[f][a], pt) <= box_d2(nodes[f][b], pt);
      stack[top++] = a_near ? b : a;
      stack[top++] = a_near ? a : b;
    }
    return i0;
  }
};

}  // namespace

struct hr_geom2s {
  hr_geom2s_params prm;
  int N = 0;
  double h = 0, delta = 0;
  std::vector<double> xyz[2], nrm[2], area[2], f[2];
  std::vector<int> plane[2];
  std::vector<double> b[2], x0[2], n0[2], f0[2];
  std::vector<int> nrst[2], i123[2];
  // wall seconds of the set-up phases: quadrature (both surfaces), forces,
  // nearest data of target sets 0 and 1
  double phase_s[4] = {0, 0, 0, 0};
};

extern "C" int hr_geom2s_default_params(hr_geom2s_params* p) {
  if (!p) return HR_ERR_ARG;
  memset(p, 0, sizeof(*p));
  // 2S/utilities.h:15-26
  p->axes[0] = 1.0;
  p->axes[1] = 0.5;
  p->axes[2] = 0.5;
  p->center[0][2] = -0.5 - 1.0 / (16.0 * 16.0 * 16.0);
  p->center[1][2] = 0.5;
  // make_rot_mat with alpha = beta = 0, gamma = 30 deg: 2S/utilities.cpp:10-40
  double alpha = 0.0, beta = 0.0, gam = 30.0 * kPI / 180.0;
  double ca = cos(alpha), sa = sin(alpha), cb = cos(beta), sb = sin(beta), cg = cos(gam),
         sg = sin(gam);
  double* R = p->unrot[1];
  R[0] = cb * cg;
  R[1] = cb * sg;
  R[2] = -sb;
  R[3] = sa * sb * cg - ca * sg;
  R[4] = sa * sb * sg + ca * cg;
  R[5] = sa * cb;
  R[6] = ca * sb * cg + sa * sg;
  R[7] = ca * sb * sg - sa * cg;
  R[8] = ca * cb;
  for (int k = 0; k < 9; k++) p->unrot[0][k] = (k % 4 == 0) ? 1.0 : 0.0;
  p->rotated[0] = 0;
  p->rotated[1] = 1;
  p->kappa0 = 4.0;  // 2S/main.cpp:147-148
  p->q = 5.0 / 7.0;
  return HR_OK;
}

extern "C" int hr_geom2s_generate(const hr_geom2s_params* prm, int N, hr_geom2s** out) {
  if (!prm || !out || N < 2) return HR_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<hr_geom2s> G(new hr_geom2s);
  G->prm = *prm;
  G->N = N;
  G->h = 1.0 / N;  // L = 1 (2S/main.cpp:68-70)
  double kappa = prm->kappa0 * pow(1.0 / 64.0, 1.0 - prm->q);  // 2S/main.cpp:155-157
  G->delta = kappa * pow(G->h, prm->q);
  Spheroid gen[2], cen[2];
  for (int s = 0; s < 2; s++) {
    for (int k = 0; k < 3; k++) {
      gen[s].a2[k] = prm->axes[k] * prm->axes[k];
      gen[s].ctr[k] = prm->center[s][k];
    }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) gen[s].R[i][j] = prm->unrot[s][3 * i + j];
    gen[s].rotated = prm->rotated[s] != 0;
    gen[s].centered = false;
    cen[s] = gen[s];
    cen[s].centered = true;
  }
  std::vector<QPoint> P[2];
  const double zero[3] = {0, 0, 0};
  double t0 = omp_get_wtime();
  for (int s = 0; s < 2; s++) P[s] = generate_surface(gen[s], N, G->h, zero, prm->center[s]);
  double t1 = omp_get_wtime();
  G->phase_s[0] = t1 - t0;
  for (int s = 0; s < 2; s++) {
    const int n = (int)P[s].size();
    G->xyz[s].resize(3 * n);
    G->nrm[s].resize(3 * n);
    G->area[s].resize(n);
    G->plane[s].resize(n);
    G->f[s].resize(3 * n);
#pragma omp parallel for schedule(static, 256)
    for (int i = 0; i < n; i++) {
      for (int k = 0; k < 3; k++) {
        G->xyz[s][3 * i + k] = P[s][i].x[k];
        G->nrm[s][3 * i + k] = P[s][i].n[k];
      }
      G->area[s][i] = P[s][i].area;
      G->plane[s][i] = P[s][i].plane;
      // set_surface_force (2S/main.cpp:1050-1059)
      surface_force(cen[s], prm->axes, P[s][i].x, P[s][i].n, &G->f[s][3 * i], prm->tension_body != 0);
    }
  }
  t0 = omp_get_wtime();
  G->phase_s[1] = t0 - t1;
  // Compute_nearest_data: 2S/surface.cpp:450-526 (targets of set t vs surface 1-t)
  for (int t = 0; t < 2; t++) {
    const int src = 1 - t;
    const Spheroid& S = cen[src];
    PointTree CI;
    CI.build(P[src]);
    const int n = (int)P[t].size();
    G->b[t].assign(n, 0.0);
    G->x0[t].assign(3 * n, 0.0);
    G->n0[t].assign(3 * n, 0.0);
    G->f0[t].assign(3 * n, 0.0);
    G->nrst[t].assign(n, 0);
    G->i123[t].assign(3 * n, 0);
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
      const double* pt = P[t][i].x;
      int i1, i2, i3;
      monge(S, pt, i1, i2, i3);
      int nrst_i = CI.nearest(pt, i3);
      G->nrst[t][i] = nrst_i;
      if (nrst_i < 0) continue;
      double x0[3], n0[3];
      if (nearest_point(S, pt, P[src][nrst_i].x, x0, n0) != 0) continue;
      for (int k = 0; k < 3; k++) {
        G->x0[t][3 * i + k] = x0[k];
        G->n0[t][3 * i + k] = n0[k];
      }
      G->i123[t][3 * i] = i1;
      G->i123[t][3 * i + 1] = i2;
      G->i123[t][3 * i + 2] = i3;
      double b = (pt[0] - x0[0]) * n0[0] + (pt[1] - x0[1]) * n0[1] + (pt[2] - x0[2]) * n0[2];
      G->b[t][i] = b;
      if (fabs(b) / G->delta > 8.0) {
        G->nrst[t][i] = 0;
        continue;
      }
      surface_force(S, prm->axes, x0, n0, &G->f0[t][3 * i], prm->tension_body != 0);
    }
    t1 = omp_get_wtime();
    G->phase_s[2 + t] = t1 - t0;
    t0 = t1;
  }
  *out = G.release();
  return HR_OK;
}

extern "C" int hr_geom2s_view(const hr_geom2s* G, hr_scene2s* sc, const double** force) {
  if (!G || !sc) return HR_ERR_ARG;
  memset(sc, 0, sizeof(*sc));
  for (int s = 0; s < 2; s++) {
    hr_surface& S = sc->surf[s];
    S.n = (int)G->area[s].size();
    S.xyz = G->xyz[s].data();
    S.nrml = G->nrm[s].data();
    S.area = G->area[s].data();
    S.plane = G->plane[s].data();
    for (int k = 0; k < 3; k++) S.center[k] = G->prm.center[s][k];
    hr_targets& T = sc->tgt[s];
    T.n = S.n;
    T.xyz = G->xyz[s].data();
    T.b = G->b[s].data();
    T.x0 = G->x0[s].data();
    T.n0 = G->n0[s].data();
    T.nrst = G->nrst[s].data();
    T.i123 = G->i123[s].data();
    sc->f0[s] = G->f0[s].data();
    if (force) force[s] = G->f[s].data();
  }
  sc->h = G->h;
  sc->delta = G->delta;
  return HR_OK;
}

extern "C" int hr_geom2s_phase_seconds(const hr_geom2s* G, double* out4) {
  if (!G || !out4) return HR_ERR_ARG;
  for (int k = 0; k < 4; k++) out4[k] = G->phase_s[k];
  return HR_OK;
}

extern "C" void hr_geom2s_destroy(hr_geom2s* G) { delete G; }
