// hr_warm.cpp — host side of the learned GMRES warm start: seeded two-surface
// instances (random gap, relative orientation and imposed rigid motion) and
// the 12 pointwise geometry features the warm-start network reads.
//
// Instances reuse the two-surface scene generator (the reference's spheroid,
// grid-line quadrature and force law, 2S/surface.cpp:13-71 and :530-559) with
// the second spheroid rotated and placed so that the two solids are `gap`
// apart; its surface tension 1 + z^2 is taken in its own body frame, so the
// rotated drop is the reference's drop turned as a whole (for the unrotated
// first surface this is the reference's law). The vector features and the
// network's output are expressed in the body frame of the point's own
// surface: with the tension attached to the body, the response of a drop on
// its own is then a function of the body-frame normal alone (the Gauss map of
// a convex surface is one to one), which world-frame features cannot give for
// a randomly turned drop. The imposed velocity is a background rigid motion
// u(x) = U + Omega x (x - xmid). Rigid motions satisfy (I - 2/3 D) u = 2/3 u on
// the union of the two closed surfaces, so with right-hand side
// b = -2/3 S[f] + 2/3 u the solution is u plus the response to the force f;
// the network predicts that response.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/highreg_b200.h"

namespace {

constexpr double kPI = 3.14159265358979323846;

// Uniform double in [0, 1) from the top 53 bits of one mt19937_64 draw.
double unif(std::mt19937_64& g) { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }

struct Ellipsoid {
  double a[3];     // semi-axes
  double c[3];     // centre
  double R[3][3];  // body = R (x - c)
  void body(const double* x, double* u) const {
    double d[3] = {x[0] - c[0], x[1] - c[1], x[2] - c[2]};
    for (int i = 0; i < 3; i++) u[i] = R[i][0] * d[0] + R[i][1] * d[1] + R[i][2] * d[2];
  }
  // a vector (not a point) in body coordinates
  void to_body(const double* v, double* u) const {
    for (int i = 0; i < 3; i++) u[i] = R[i][0] * v[0] + R[i][1] * v[1] + R[i][2] * v[2];
  }
  void world(const double* u, double* x) const {
    for (int j = 0; j < 3; j++) x[j] = c[j] + R[0][j] * u[0] + R[1][j] * u[1] + R[2][j] * u[2];
  }
  double phi(const double* x) const {
    double u[3];
    body(x, u);
    return u[0] * u[0] / (a[0] * a[0]) + u[1] * u[1] / (a[1] * a[1]) + u[2] * u[2] / (a[2] * a[2]) - 1.0;
  }
  // Closest point of the solid ellipsoid to y (y itself when inside): the
  // nearest surface point x_i = a_i^2 v_i / (t + a_i^2) with t > 0 the root of
  // sum (a_i v_i / (t + a_i^2))^2 = 1 (Eberly, "Distance from a point to an
  // ellipse, an ellipsoid, or a hyperellipsoid", 2013), found by bisection.
  void project(const double* y, double* x) const {
    double v[3];
    body(y, v);
    double F0 = 0.0;
    for (int i = 0; i < 3; i++) F0 += (v[i] / a[i]) * (v[i] / a[i]);
    if (F0 <= 1.0) {
      for (int k = 0; k < 3; k++) x[k] = y[k];
      return;
    }
    double amax = fmax(a[0], fmax(a[1], a[2]));
    double vn = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    double lo = 0.0, hi = vn * amax;
    for (int it = 0; it < 200; it++) {
      double t = 0.5 * (lo + hi);
      if (t <= lo || t >= hi) break;
      double F = -1.0;
      for (int i = 0; i < 3; i++) {
        double r = a[i] * v[i] / (t + a[i] * a[i]);
        F += r * r;
      }
      if (F > 0.0) lo = t;
      else hi = t;
    }
    double t = 0.5 * (lo + hi), u[3];
    for (int i = 0; i < 3; i++) u[i] = a[i] * a[i] * v[i] / (t + a[i] * a[i]);
    world(u, x);
  }
  // Principal curvatures (k1 >= k2, positive for the convex body with the
  // outward normal) at a surface point: eigenvalues of the shape operator
  // P Hess(phi) P / |grad phi| restricted to the tangent plane.
  void curvatures(const double* x, double* k1, double* k2) const {
    double u[3], gb[3], g[3], H[3][3];
    body(x, u);
    for (int i = 0; i < 3; i++) gb[i] = 2.0 * u[i] / (a[i] * a[i]);
    for (int j = 0; j < 3; j++) g[j] = R[0][j] * gb[0] + R[1][j] * gb[1] + R[2][j] * gb[2];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double s = 0.0;
        for (int k = 0; k < 3; k++) s += R[k][i] * (2.0 / (a[k] * a[k])) * R[k][j];
        H[i][j] = s;
      }
    double gn = sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2]);
    double n[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
    double P[3][3], PH[3][3], S[3][3];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) P[i][j] = (i == j ? 1.0 : 0.0) - n[i] * n[j];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double s = 0.0;
        for (int k = 0; k < 3; k++) s += P[i][k] * H[k][j];
        PH[i][j] = s;
      }
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) {
        double s = 0.0;
        for (int k = 0; k < 3; k++) s += PH[i][k] * P[k][j];
        S[i][j] = s / gn;
      }
    double tr = S[0][0] + S[1][1] + S[2][2];
    double tr2 = 0.0;
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) tr2 += S[i][j] * S[j][i];
    double Hm = 0.5 * tr, K = 0.5 * (tr * tr - tr2);
    double disc = sqrt(fmax(Hm * Hm - K, 0.0));
    *k1 = Hm + disc;
    *k2 = Hm - disc;
  }
};

Ellipsoid from_params(const hr_geom2s_params& p, int s) {
  Ellipsoid E;
  for (int k = 0; k < 3; k++) {
    E.a[k] = p.axes[k];
    E.c[k] = p.center[s][k];
  }
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) E.R[i][j] = p.rotated[s] ? p.unrot[s][3 * i + j] : (i == j ? 1.0 : 0.0);
  return E;
}

// Distance between the two solids by alternating projections (convex sets:
// von Neumann / Cheney-Goldstein); 0 when they overlap.
double solid_distance(const Ellipsoid& A, const Ellipsoid& B) {
  double p1[3] = {A.c[0], A.c[1], A.c[2]}, p2[3];
  for (int it = 0; it < 20000; it++) {
    B.project(p1, p2);
    double q[3];
    A.project(p2, q);
    double dq = fabs(q[0] - p1[0]) + fabs(q[1] - p1[1]) + fabs(q[2] - p1[2]);
    for (int k = 0; k < 3; k++) p1[k] = q[k];
    if (dq < 1e-15) break;
  }
  B.project(p1, p2);
  double d[3] = {p2[0] - p1[0], p2[1] - p1[1], p2[2] - p1[2]};
  return sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
}

void unit_vector(std::mt19937_64& g, double* d) {
  double z = 2.0 * unif(g) - 1.0, ph = 2.0 * kPI * unif(g), r = sqrt(fmax(0.0, 1.0 - z * z));
  d[0] = r * cos(ph);
  d[1] = r * sin(ph);
  d[2] = z;
}

}  // namespace

extern "C" int hr_warm_instance_make(unsigned long long seed, int index, hr_warm_instance* out) {
  if (!out || index < 0) return HR_ERR_ARG;
  std::mt19937_64 g(seed);
  double gap = 0, q[4] = {0, 0, 0, 1}, dir[3] = {0, 0, 1}, U[3] = {0, 0, 0}, W[3] = {0, 0, 0};
  for (int i = 0; i <= index; i++) {
    // gap uniform in [0.02, 0.3] x diameter (2, the major axis)
    gap = (0.02 + 0.28 * unif(g)) * 2.0;
    // uniform rotation: Shoemake's quaternion from three uniforms
    double u1 = unif(g), u2 = unif(g), u3 = unif(g);
    q[0] = sqrt(1.0 - u1) * sin(2.0 * kPI * u2);
    q[1] = sqrt(1.0 - u1) * cos(2.0 * kPI * u2);
    q[2] = sqrt(u1) * sin(2.0 * kPI * u3);
    q[3] = sqrt(u1) * cos(2.0 * kPI * u3);
    unit_vector(g, dir);
    unit_vector(g, U);
    unit_vector(g, W);
  }
  hr_warm_instance& w = *out;
  memset(&w, 0, sizeof(w));
  hr_geom2s_default_params(&w.geom);
  for (int s = 0; s < 2; s++)
    for (int k = 0; k < 3; k++) w.geom.center[s][k] = 0.0;
  for (int k = 0; k < 9; k++) w.geom.unrot[0][k] = (k % 4 == 0) ? 1.0 : 0.0;
  w.geom.rotated[0] = 0;
  // rotation matrix of the unit quaternion (x, y, z, w) = q
  const double x = q[0], y = q[1], z = q[2], s = q[3];
  double* R = w.geom.unrot[1];
  R[0] = 1 - 2 * (y * y + z * z);
  R[1] = 2 * (x * y - z * s);
  R[2] = 2 * (x * z + y * s);
  R[3] = 2 * (x * y + z * s);
  R[4] = 1 - 2 * (x * x + z * z);
  R[5] = 2 * (y * z - x * s);
  R[6] = 2 * (x * z - y * s);
  R[7] = 2 * (y * z + x * s);
  R[8] = 1 - 2 * (x * x + y * y);
  w.geom.rotated[1] = 1;
  w.geom.tension_body = 1;
  // place the second centre along dir so that the solids are `gap` apart;
  // the distance is convex in the offset and zero while they overlap
  Ellipsoid A = from_params(w.geom, 0);
  double lo = 0.0, hi = 2.0 + gap + 1.0;
  for (int it = 0; it < 60; it++) {
    double t = 0.5 * (lo + hi);
    for (int k = 0; k < 3; k++) w.geom.center[1][k] = t * dir[k];
    Ellipsoid B = from_params(w.geom, 1);
    if (solid_distance(A, B) < gap) lo = t;
    else hi = t;
  }
  for (int k = 0; k < 3; k++) w.geom.center[1][k] = hi * dir[k];
  w.gap = solid_distance(A, from_params(w.geom, 1));
  for (int k = 0; k < 3; k++) {
    w.U[k] = U[k];
    w.Omega[k] = W[k];
    w.xmid[k] = 0.5 * (w.geom.center[0][k] + w.geom.center[1][k]);
  }
  return HR_OK;
}

extern "C" int hr_warm_imposed_velocity(const hr_warm_instance* w, const double* xyz, int n, double* u) {
  if (!w || n < 0 || (n > 0 && (!xyz || !u))) return HR_ERR_ARG;
  for (int i = 0; i < n; i++) {
    const double* x = xyz + 3 * i;
    double r[3] = {x[0] - w->xmid[0], x[1] - w->xmid[1], x[2] - w->xmid[2]};
    u[3 * i] = w->U[0] + w->Omega[1] * r[2] - w->Omega[2] * r[1];
    u[3 * i + 1] = w->U[1] + w->Omega[2] * r[0] - w->Omega[0] * r[2];
    u[3 * i + 2] = w->U[2] + w->Omega[0] * r[1] - w->Omega[1] * r[0];
  }
  return HR_OK;
}

extern "C" int hr_warm_features(const hr_scene2s* sc, const hr_warm_instance* w, float* feat, double* u_imposed) {
  if (!sc || !w || !feat) return HR_ERR_ARG;
  Ellipsoid E[2] = {from_params(w->geom, 0), from_params(w->geom, 1)};
  long off = 0;
  for (int s = 0; s < 2; s++) {
    const hr_surface& S = sc->surf[s];
    if (S.n < 0 || (S.n > 0 && (!S.xyz || !S.nrml))) return HR_ERR_ARG;
    const Ellipsoid& self = E[s];
    const Ellipsoid& other = E[1 - s];
    std::vector<double> uimp(3 * (size_t)S.n);
    hr_warm_imposed_velocity(w, S.xyz, S.n, uimp.data());
#pragma omp parallel for schedule(static)
    for (int i = 0; i < S.n; i++) {
      const double* x = S.xyz + 3 * i;
      float* f = feat + (off + i) * HR_WARM_NFEAT;
      double k1, k2, x0[3];
      self.curvatures(x, &k1, &k2);
      other.project(x, x0);
      double d[3] = {x0[0] - x[0], x0[1] - x[1], x0[2] - x[2]};
      double b = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
      double inv = b > 0.0 ? 1.0 / b : 0.0;
      for (int k = 0; k < 3; k++) d[k] *= inv;
      double nb[3], db[3], ub[3];
      self.to_body(S.nrml + 3 * i, nb);
      self.to_body(d, db);
      self.to_body(&uimp[3 * i], ub);
      for (int k = 0; k < 3; k++) f[k] = (float)nb[k];
      f[3] = (float)k1;
      f[4] = (float)k2;
      f[5] = (float)b;
      for (int k = 0; k < 3; k++) f[6 + k] = (float)db[k];
      for (int k = 0; k < 3; k++) f[9 + k] = (float)ub[k];
    }
    if (u_imposed)
      for (long k = 0; k < 3L * S.n; k++) u_imposed[3 * off + k] = uimp[k];
    off += S.n;
  }
  return HR_OK;
}

extern "C" int hr_warm_frames(const hr_warm_instance* w, double* rot) {
  if (!w || !rot) return HR_ERR_ARG;
  for (int s = 0; s < 2; s++) {
    Ellipsoid E = from_params(w->geom, s);
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) rot[9 * s + 3 * i + j] = E.R[i][j];
  }
  return HR_OK;
}
