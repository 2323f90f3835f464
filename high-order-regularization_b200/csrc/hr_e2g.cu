// hr_e2g.cu — the extend-to-grid pipeline on the device
// (test_Stokes_Poisson3d_FD, E2G/main.cpp:107-424):
//   1. pressure and velocity boundary integrals at the six box faces with the
//      plain kernels and at the BAND1 grid points outside or on the surface
//      with the 7th-order regularized kernels and subtraction (one batched
//      launch of the four sums, E2G/main.cpp:1049-1406, as two passes: velocity
//      and pressure at the same targets share each pair's distance and
//      smoothing factors);
//   2. p = 0 and u = (1, 0, 0) elsewhere, then the four Poisson extensions:
//      p first (variable 0), then u_x, u_y, u_z with the extended p
//      (E2G/main.cpp:195-200, 403-424).
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "../host/hr_e2g_geom.h"
#include "hr_runtime.h"

using namespace hr;

namespace {

__global__ void fill_kernel(long n, double v, double* a) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) a[i] = v;
}

__global__ void scatter_kernel(int n, int comps, const long* __restrict__ gi,
                               const double* __restrict__ v, double* g0, double* g1, double* g2) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  long g = gi[t];
  if (comps == 1) {
    g0[g] = v[t];
  } else {
    g0[g] = v[3 * t];
    g1[g] = v[3 * t + 1];
    g2[g] = v[3 * t + 2];
  }
}

// The Poisson masks (E2G/main.cpp:1611-1614, 1654-1672): band2 is set
// beforehand at the BAND2 points (scattered from the tagged targets); a point
// is exterior when phi(x) > 0 and it is not in BAND2. The level set is formed
// with unfused operations in the order the host's expression
// u0 u0 / 1 + u1 u1 / 0.25 + u2 u2 / 0.25 - 1 evaluates (dividing by 0.25 is
// multiplying by 4 exactly), so the sign test is the host's.
__global__ void exterior_mask_kernel(int M, double h, const uint8_t* __restrict__ band2, uint8_t* __restrict__ om) {
  const long m3 = (long)M * M * M;
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < m3; g += (long)gridDim.x * blockDim.x) {
    const int i = (int)(g / ((long)M * M)), j = (int)((g / M) % M), k = (int)(g % M);
    const double u0 = __dsub_rn(__dmul_rn((double)i, h), 1.5);
    const double u1 = __dsub_rn(__dmul_rn((double)j, h), 1.5);
    const double u2 = __dsub_rn(__dmul_rn((double)k, h), 1.5);
    const double levl = __dsub_rn(__dadd_rn(__dadd_rn(__dmul_rn(u0, u0), __dmul_rn(__dmul_rn(u1, u1), 4.0)),
                                            __dmul_rn(__dmul_rn(u2, u2), 4.0)),
                                  1.0);
    om[g] = (levl > 0.0 && !band2[g]) ? 1 : 0;
  }
}

__global__ void set_points_kernel(int n, const long* __restrict__ gi, uint8_t* __restrict__ mask) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) mask[gi[t]] = 1;
}

constexpr double kPI = 3.14159265358979323846;

// ---------------------------------------------------------------- error norms
// The exact solution of the translating prolate spheroid (semi-axes 1, .5, .5,
// centre (1.5, 1.5, 1.5)): p_exact and SL_exact, E2G/utilities.cpp:294-321 and
// :360-411, evaluated per grid point on the device.
__device__ void exact_pu(double xi, double yi, double zi, double& p, double u[3]) {
  const double x = xi - 1.5, y = yi - 1.5, z = zi - 1.5;
  const double a_sq = 1.0, b_sq = 0.25;
  const double r_sq = y * y + z * z;
  const double c = sqrt(a_sq - b_sq);
  const double R1 = sqrt((x + c) * (x + c) + r_sq);
  const double R2 = sqrt((x - c) * (x - c) + r_sq);
  const double R1c = R1 - (x + c);
  const double R2c = R2 - (x - c);
  double B10;
  if (r_sq < 1.e-14) B10 = (x < 0) ? log((x - c) / (x + c)) : log((x + c) / (x - c));
  else B10 = log(R2c / R1c);
  const double B30 = (x + c) / R1 - (x - c) / R2;
  const double dB1dx = 1.0 / R1 - 1.0 / R2;
  double dB1dyz = 0.0;
  if (r_sq > 1.e-14) dB1dyz = 1.0 / R2 / R2c - 1.0 / R1 / R1c;
  const double dB3dyz = 1.0 / R2 - 1.0 / R1 + x * dB1dyz;
  const double e = c / 1.0;
  const double Le = log((1.0 + e) / (1.0 - e));
  const double a1 = e * e / ((1.0 + e * e) * Le - 2.0 * e);
  const double b1 = a1 * (1.0 - e * e) / (2.0 * e * e);
  p = -2.0 * a1 * dB1dx;
  u[0] = 2.0 * a1 * B10 - a1 * B30 + 2.0 * b1 * ((x - c) / R2 - (x + c) / R1 + B10 + x * dB1dx);
  const double Er = a1 * (1.0 / R2 - 1.0 / R1) + 2.0 * b1 * dB3dyz;
  u[1] = Er * y;
  u[2] = Er * z;
}

// The grids' values where the reference compares (E2G/main.cpp:236-259, 470-497):
// the exact solution outside or on the surface, p = 0 and u = (1, 0, 0) inside.
__device__ void grid_exact(int N, double h, long g, double& p, double u[3]) {
  const long M = N + 1;
  const int i = (int)(g / (M * M)), j = (int)((g / M) % M), k = (int)(g % M);
  const double x = i * h, y = j * h, z = k * h;
  const double lv = (x - 1.5) * (x - 1.5) + (y - 1.5) * (y - 1.5) / 0.25 + (z - 1.5) * (z - 1.5) / 0.25 - 1.0;
  if (lv > 0.0 || fabs(lv) < 1e-12) {
    exact_pu(x, y, z, p, u);
  } else {
    p = 0.0;
    u[0] = 1.0;
    u[1] = u[2] = 0.0;
  }
}

// Mid-plane j = N/2 (y = 1.5) slices: extended p, |p - p_exact|, |u - u_exact|
// and p_exact, the last three outside or on the surface only (0 inside), as
// the reference's slice files (E2G/main.cpp:221-224, 297-300, 505-546).
__global__ void midplane_kernel(int N, double h, const double* __restrict__ p, const double* __restrict__ u,
                                double* __restrict__ out) {
  const long M = N + 1, m3 = M * M * M, mm = M * M;
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= mm) return;
  const int i = (int)(e / M), k = (int)(e % M), j = N / 2;
  const long g = ((long)i * M + j) * M + k;
  const double x = i * h, y = j * h, z = k * h;
  const double lv = (x - 1.5) * (x - 1.5) + (y - 1.5) * (y - 1.5) / 0.25 + (z - 1.5) * (z - 1.5) / 0.25 - 1.0;
  double pe = 0.0, dp = 0.0, du = 0.0;
  if (lv > 0.0 || fabs(lv) < 1e-12) {
    double ue[3];
    exact_pu(x, y, z, pe, ue);
    dp = fabs(p[g] - pe);
    const double d0 = u[g] - ue[0], d1 = u[m3 + g] - ue[1], d2 = u[2 * m3 + g] - ue[2];
    du = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  }
  out[e] = p[g];
  out[mm + e] = dp;
  out[2 * mm + e] = du;
  out[3 * mm + e] = pe;
}

constexpr int kErrBlocks = 148 * 4, kErrThreads = 256, kErrVals = 12;

// Per-block maxima and sums (fixed grid-stride assignment, so the final
// in-order reduction is deterministic):
//  0 max|p - pex|  1 sum (p - pex)^2  2 max|u - uex|  3 sum |u - uex|^2
//  4 max|p - pref| 5 sum (p - pref)^2 6 max|pref|     7 sum pref^2
//  8 max|u - uref| 9 sum |u - uref|^2 10 max|uref|    11 sum |uref|^2
__global__ void __launch_bounds__(kErrThreads) grid_errors_kernel(int N, double h, const double* __restrict__ p,
                                                                  const double* __restrict__ u,
                                                                  const double* __restrict__ pref,
                                                                  const double* __restrict__ uref,
                                                                  double* __restrict__ part) {
  const long M = N + 1, m3 = M * M * M;
  double v[kErrVals];
  for (int q = 0; q < kErrVals; q++) v[q] = 0.0;
  for (long g = (long)blockIdx.x * blockDim.x + threadIdx.x; g < m3; g += (long)gridDim.x * blockDim.x) {
    double pe, ue[3];
    grid_exact(N, h, g, pe, ue);
    const double uu[3] = {u[g], u[m3 + g], u[2 * m3 + g]};
    const double dp = fabs(p[g] - pe);
    const double du2 = (uu[0] - ue[0]) * (uu[0] - ue[0]) + (uu[1] - ue[1]) * (uu[1] - ue[1]) +
                       (uu[2] - ue[2]) * (uu[2] - ue[2]);
    v[0] = fmax(v[0], dp);
    v[1] += dp * dp;
    v[2] = fmax(v[2], sqrt(du2));
    v[3] += du2;
    if (pref) {
      const double rp = fabs(p[g] - pref[g]);
      const double r0 = uref[g], r1 = uref[m3 + g], r2 = uref[2 * m3 + g];
      const double ru2 = (uu[0] - r0) * (uu[0] - r0) + (uu[1] - r1) * (uu[1] - r1) + (uu[2] - r2) * (uu[2] - r2);
      const double un2 = r0 * r0 + r1 * r1 + r2 * r2;
      v[4] = fmax(v[4], rp);
      v[5] += rp * rp;
      v[6] = fmax(v[6], fabs(pref[g]));
      v[7] += pref[g] * pref[g];
      v[8] = fmax(v[8], sqrt(ru2));
      v[9] += ru2;
      v[10] = fmax(v[10], sqrt(un2));
      v[11] += un2;
    }
  }
  __shared__ double red[kErrThreads / 32][kErrVals];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int q = 0; q < kErrVals; q++) {
    const bool is_max = (q % 2 == 0);
    double x = v[q];
    for (int off = 16; off > 0; off >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, off);
      x = is_max ? fmax(x, y) : x + y;
    }
    if (lane == 0) red[warp][q] = x;
  }
  __syncthreads();
  if (threadIdx.x < kErrVals) {
    const int q = threadIdx.x;
    double x = red[0][q];
    for (int w = 1; w < kErrThreads / 32; w++) x = (q % 2 == 0) ? fmax(x, red[w][q]) : x + red[w][q];
    part[(size_t)blockIdx.x * kErrVals + q] = x;
  }
}

// Band velocity after the sums vs the exact solution at the band targets
// (E2G/main.cpp:1359-1405): one thread per target, per-block max and sum.
__global__ void __launch_bounds__(kErrThreads) band_errors_kernel(int N, double h, int nb, const long* __restrict__ gb,
                                                                  const double* __restrict__ u,
                                                                  double* __restrict__ part) {
  const long M = N + 1, m3 = M * M * M;
  double mx = 0.0, sq = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nb; t += gridDim.x * blockDim.x) {
    const long g = gb[t];
    double pe, ue[3];
    grid_exact(N, h, g, pe, ue);
    const double d0 = u[g] - ue[0], d1 = u[m3 + g] - ue[1], d2 = u[2 * m3 + g] - ue[2];
    const double d = d0 * d0 + d1 * d1 + d2 * d2;
    mx = fmax(mx, sqrt(d));
    sq += d;
  }
  for (int off = 16; off > 0; off >>= 1) {
    mx = fmax(mx, __shfl_down_sync(0xffffffffu, mx, off));
    sq += __shfl_down_sync(0xffffffffu, sq, off);
  }
  __shared__ double red[kErrThreads / 32][2];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[warp][0] = mx;
    red[warp][1] = sq;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < kErrThreads / 32; w++) {
      mx = fmax(mx, red[w][0]);
      sq += red[w][1];
    }
    part[2 * blockIdx.x] = mx;
    part[2 * blockIdx.x + 1] = sq;
  }
}

}  // namespace

struct hr_e2g {
  hr_ctx* owner = nullptr;
  e2g_setup::Scene S;
  int nface = 0, nband = 0;
  DevTree tree;
  DBuf<double> q3;
  DevTargets tf, tb;
  DevLists Lf, Lb;
  DBuf<double> pf, uf, pb, ub;
  DBuf<long> gf, gb;
  DBuf<uint8_t> mband2, mout;
  DBuf<double> p_bi, u_bi, p_ext, u_ext;  // grids
  DBuf<double> p_ref, u_ref;              // snapshot of the extended grids for comparisons
  bool have_ref = false;
  bool ran = false;                       // hr_e2g_run has filled the grids
  Batch batch[3];                         // by precision: FP64, mixed, all FP32
  long long pairs = 0;
  PoissonWork* pw = nullptr;              // FFT plan and grid buffers of the four Poisson solves
  ~hr_e2g() { poisson_work_destroy(pw); }
};

// The four sums of one run in one batch, in precision prec.
static void e2g_batch(hr_e2g& E, int prec, Ctx& C) {
  const double p_scale = 1.0 / (4.0 * kPI), sl_scale = 1.0 / (8.0 * kPI);
  const double delta = E.S.delta;
  Batch& B = E.batch[prec];
  B.family = F_E2G;
  // the two box-face sums (velocity and pressure at the same targets) in one pass
  EvalTask a = make_task(K_E2G_UP_AWAY, delta, sl_scale, E.tree, E.Lf, E.tf, E.uf.p);
  a.out2 = E.pf.p;
  a.scale2 = p_scale;
  // and the two band sums likewise
  EvalTask c = make_task(K_E2G_UP7, delta, sl_scale, E.tree, E.Lb, E.tb, E.ub.p);
  c.out2 = E.pb.p;
  c.scale2 = -p_scale;
  for (EvalTask* t : {&a, &c}) {
    t->mixed = prec;
    t->jump_mode = 1;
  }
  B.tasks = {a, c};
  B.lists = {&E.Lf.host, &E.Lb.host};
  B.trees = {&E.tree.host, &E.tree.host};
  B.finalize(C.stream, C.num_sms);
}

extern "C" int hr_e2g_create(hr_ctx* ctx, int N, hr_e2g** out) {
  if (!ctx || !out || N < 36 || N % 2 != 0) return HR_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<hr_e2g> E(new hr_e2g);
  E->owner = ctx;
  Ctx& C = ctx->c;
  try {
    HR_CHECK_CUDA(cudaSetDevice(C.device));
    cudaStream_t st = C.stream;
    e2g_setup::build(E->S, N, 4.0, 2.0);  // BAND1, BAND2: E2G/main.cpp:112-113
    const auto& S = E->S;
    const int M = N + 1;
    const double h = S.h;
    // surface (direct sums: a single node holding every source)
    hr_surface surf;
    memset(&surf, 0, sizeof(surf));
    surf.n = (int)S.area.size();
    surf.xyz = S.xq.data();
    surf.nrml = S.nrm.data();
    surf.area = S.area.data();
    surf.center[0] = surf.center[1] = surf.center[2] = 1.5;
    E->tree.build(surf, 6, 1000, 0.6, true, st);
    E->q3.upload(S.f, st);
    E->tree.set_density(C, E->q3.p, false, false);
    // face targets in the reference loop order (E2G/main.cpp:1058-1075)
    std::vector<double> fx;
    std::vector<long> fg;
    for (int i = 0; i <= N; i++)
      for (int j = 0; j <= N; j++) {
        // an (i, j) column off the box's i and j faces meets the box only at k = 0 and k = N
        const bool all = (i == 0 || i == N || j == 0 || j == N);
        for (int k = 0; k <= N; k += (all || k == N) ? 1 : N) {
          fx.insert(fx.end(), {i * h, j * h, k * h});
          fg.push_back(((long)i * M + j) * M + k);
        }
      }
    // band targets outside or on the surface (E2G/main.cpp:1133-1162)
    // (one i-slab per OpenMP iteration, slabs concatenated in i order)
    std::vector<double> bx, bb, bx0, bn0, bf0;
    std::vector<long> bg;
    {
      struct Slab {
        std::vector<double> x, b, x0, n0, f0;
        std::vector<long> g;
      };
      std::vector<Slab> slab(N + 1);
#pragma omp parallel for schedule(dynamic, 4)
      for (int i = 1; i < N; i++) {
        Slab& L = slab[i];
        for (int j = 1; j < N; j++)
          for (int k = 1; k < N; k++) {
            long g = ((long)i * M + j) * M + k;
            int ind = S.nrst[g];
            if (ind == -1) continue;
            double b = S.b[ind];
            if ((b > 0.0) || (fabs(b) < 1.e-12)) {
              L.x.insert(L.x.end(), {i * h, j * h, k * h});
              L.b.push_back(b);
              const double* x0 = &S.x0[3 * ind];
              L.x0.insert(L.x0.end(), {x0[0], x0[1], x0[2]});
              L.n0.insert(L.n0.end(), {S.n0[3 * ind], S.n0[3 * ind + 1], S.n0[3 * ind + 2]});
              double f0[3];
              e2g_setup::stokeslet_density(x0, f0);
              L.f0.insert(L.f0.end(), {f0[0], f0[1], f0[2]});
              L.g.push_back(g);
            }
          }
      }
      for (const Slab& L : slab) {
        bx.insert(bx.end(), L.x.begin(), L.x.end());
        bb.insert(bb.end(), L.b.begin(), L.b.end());
        bx0.insert(bx0.end(), L.x0.begin(), L.x0.end());
        bn0.insert(bn0.end(), L.n0.begin(), L.n0.end());
        bf0.insert(bf0.end(), L.f0.begin(), L.f0.end());
        bg.insert(bg.end(), L.g.begin(), L.g.end());
      }
    }
    E->nface = (int)fg.size();
    E->nband = (int)bg.size();
    auto up = [&](DevTargets& T, int n, const std::vector<double>& x, const double* b,
                  const double* x0, const double* n0, const double* f0) {
      T.n = n;
      T.xyz.upload(x.data(), 3 * (size_t)n, st);
      if (b) T.b.upload(b, n, st);
      else {
        T.b.alloc(n);
        T.b.zero(st);
      }
      T.x0.alloc(3 * (size_t)n);
      if (x0) T.x0.upload(x0, 3 * (size_t)n, st);
      T.n0.alloc(3 * (size_t)n);
      if (n0) T.n0.upload(n0, 3 * (size_t)n, st);
      else T.n0.zero(st);
      T.f0.alloc(3 * (size_t)n);
      if (f0) T.f0.upload(f0, 3 * (size_t)n, st);
      else T.f0.zero(st);
      T.g0.alloc(3 * (size_t)n);
      T.nrm.alloc(3 * (size_t)n);
      std::vector<uint8_t> nr(n, 1);
      T.near.upload(nr, st);
    };
    up(E->tf, E->nface, fx, nullptr, nullptr, nullptr, nullptr);
    up(E->tb, E->nband, bx, bb.data(), bx0.data(), bn0.data(), bf0.data());
    E->Lf.build(E->tree.host, E->nface, fx.data(), nullptr, st);
    E->Lb.build(E->tree.host, E->nband, bx.data(), nullptr, st);
    E->gf.upload(fg, st);
    E->gb.upload(bg, st);
    E->pf.alloc(E->nface);
    E->uf.alloc(3 * (size_t)E->nface);
    E->pb.alloc(std::max(1, E->nband));
    E->ub.alloc(3 * (size_t)std::max(1, E->nband));
    e2g_batch(*E, HR_FP64, C);  // the reduced-precision batches are built on first use
    E->pairs = 2LL * (E->nface + E->nband) * (long long)surf.n;
    // masks: BAND2 points, and exterior points outside BAND2, built on the
    // device from the BAND2 targets' grid indices
    const size_t mm = (size_t)M * M * M;
    std::vector<long> g2;
    for (size_t t = 0; t < S.band2.size(); t++)
      if (S.band2[t]) g2.push_back(S.g[t]);
    DBuf<long> dg2;
    dg2.upload(g2, st);
    E->mband2.alloc(mm);
    E->mband2.zero(st);
    E->mout.alloc(mm);
    if (!g2.empty())
      set_points_kernel<<<(unsigned)((g2.size() + 255) / 256), 256, 0, st>>>((int)g2.size(), dg2.p, E->mband2.p);
    exterior_mask_kernel<<<4 * C.num_sms, 256, 0, st>>>(M, h, E->mband2.p, E->mout.p);
    C.launches += 2;
    HR_CHECK_CUDA(cudaGetLastError());
    size_t m3 = (size_t)M * M * M;
    E->p_bi.alloc(m3);
    E->u_bi.alloc(3 * m3);
    E->p_ext.alloc(m3);
    E->u_ext.alloc(3 * m3);
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  } catch (const hr::Error& e) {
    C.err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    C.err = e.what();
    return HR_ERR_CUDA;
  }
  *out = E.release();
  return HR_OK;
}

extern "C" int hr_e2g_get_info(const hr_e2g* E, hr_e2g_info* info) {
  if (!E || !info) return HR_ERR_ARG;
  info->N = E->S.N;
  info->L = E->S.L;
  info->h = E->S.h;
  info->delta = E->S.delta;
  info->nq = (int)E->S.area.size();
  info->n_tagged = (int)E->S.b.size();
  info->n_band = E->nband;
  info->n_face = E->nface;
  info->pairs = E->pairs;
  return HR_OK;
}

extern "C" int hr_e2g_run(hr_e2g* E, int precision, hr_e2g_report* rep) {
  if (!E) return HR_ERR_ARG;
  Ctx& C = E->owner->c;
  try {
    HR_CHECK_CUDA(cudaSetDevice(C.device));
    cudaStream_t st = C.stream;
    const int N = E->S.N, M = N + 1;
    const long m3 = (long)M * M * M;
    HR_REQUIRE(precision == HR_FP64 || precision == HR_MIXED || precision == HR_FP32, "unknown precision");
    if (!E->batch[precision].ready) e2g_batch(*E, precision, C);  // before the timed region
    cudaEvent_t ev[4];
    for (auto& e : ev) HR_CHECK_CUDA(cudaEventCreate(&e));
    HR_CHECK_CUDA(cudaEventRecord(ev[0], st));
    E->batch[precision].launch(C);
    E->ran = true;
    HR_CHECK_CUDA(cudaEventRecord(ev[1], st));
    // grids: p = 0, u = (1, 0, 0) off the evaluated points (E2G/main.cpp:1062, 1234-1236)
    int fb = 148 * 8;
    fill_kernel<<<fb, 256, 0, st>>>(m3, 0.0, E->p_bi.p);
    fill_kernel<<<fb, 256, 0, st>>>(m3, 1.0, E->u_bi.p);
    fill_kernel<<<fb, 256, 0, st>>>(2 * m3, 0.0, E->u_bi.p + m3);
    double *ux = E->u_bi.p, *uy = ux + m3, *uz = uy + m3;
    scatter_kernel<<<(E->nface + 255) / 256, 256, 0, st>>>(E->nface, 1, E->gf.p, E->pf.p, E->p_bi.p,
                                                           nullptr, nullptr);
    scatter_kernel<<<(E->nface + 255) / 256, 256, 0, st>>>(E->nface, 3, E->gf.p, E->uf.p, ux, uy, uz);
    if (E->nband > 0) {
      scatter_kernel<<<(E->nband + 255) / 256, 256, 0, st>>>(E->nband, 1, E->gb.p, E->pb.p, E->p_bi.p,
                                                             nullptr, nullptr);
      scatter_kernel<<<(E->nband + 255) / 256, 256, 0, st>>>(E->nband, 3, E->gb.p, E->ub.p, ux, uy, uz);
    }
    C.launches += 7;
    HR_CHECK_CUDA(cudaGetLastError());
    HR_CHECK_CUDA(cudaEventRecord(ev[2], st));
    // Poisson extensions: p (variable 0) then u_x, u_y, u_z with the extended p
    HR_CHECK_CUDA(cudaMemcpyAsync(E->p_ext.p, E->p_bi.p, sizeof(double) * m3, cudaMemcpyDeviceToDevice, st));
    if (!E->pw) E->pw = poisson_work_create(C, N);
    solve_poisson_dev(C, N, E->S.L, E->mband2.p, E->mout.p, nullptr, E->p_ext.p, 0, E->pw);
    HR_CHECK_CUDA(cudaMemcpyAsync(E->u_ext.p, E->u_bi.p, sizeof(double) * 3 * m3, cudaMemcpyDeviceToDevice, st));
    for (int v = 0; v < 3; v++)
      solve_poisson_dev(C, N, E->S.L, E->mband2.p, E->mout.p, E->p_ext.p, E->u_ext.p + v * m3, v + 1, E->pw);
    HR_CHECK_CUDA(cudaEventRecord(ev[3], st));
    HR_CHECK_CUDA(cudaEventSynchronize(ev[3]));
    float t01 = 0, t23 = 0, t03 = 0;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    cudaEventElapsedTime(&t23, ev[2], ev[3]);
    cudaEventElapsedTime(&t03, ev[0], ev[3]);
    for (auto& e : ev) cudaEventDestroy(e);
    if (rep) {
      memset(rep, 0, sizeof(*rep));
      rep->seconds_sums = t01 * 1e-3;
      rep->seconds_poisson = t23 * 1e-3;
      rep->seconds_total = t03 * 1e-3;
      rep->pairs = E->pairs;
    }
  } catch (const hr::Error& e) {
    C.err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    C.err = e.what();
    return HR_ERR_CUDA;
  }
  return HR_OK;
}

// which: 0 p after the sums, 1 u after the sums (3 grids), 2 extended p, 3 extended u (3 grids)
extern "C" int hr_e2g_get(hr_e2g* E, int which, double* out) {
  if (!E || !out || which < 0 || which > 3) return HR_ERR_ARG;
  Ctx& C = E->owner->c;
  try {
    HR_CHECK_CUDA(cudaSetDevice(C.device));
    const long M = E->S.N + 1, m3 = M * M * M;
    const double* src = which == 0 ? E->p_bi.p : which == 1 ? E->u_bi.p : which == 2 ? E->p_ext.p : E->u_ext.p;
    long n = (which == 1 || which == 3) ? 3 * m3 : m3;
    d2h_staged(C, out, src, sizeof(double) * n);
  } catch (const hr::Error& e) {
    C.err = e.what();
    return e.code;
  }
  return HR_OK;
}

// scene data for checks: which 0 = quadrature (3nq xyz, 3nq nrml, nq area, 3nq f),
// 1 = nrst grid (int), 2 = tagged targets (b, x0, n0, band2 as double)
extern "C" int hr_e2g_scene(const hr_e2g* E, int which, void* out) {
  if (!E || !out) return HR_ERR_ARG;
  const auto& S = E->S;
  if (which == 0) {
    double* o = (double*)out;
    size_t nq = S.area.size();
    memcpy(o, S.xq.data(), 3 * nq * sizeof(double));
    memcpy(o + 3 * nq, S.nrm.data(), 3 * nq * sizeof(double));
    memcpy(o + 6 * nq, S.area.data(), nq * sizeof(double));
    memcpy(o + 7 * nq, S.f.data(), 3 * nq * sizeof(double));
  } else if (which == 1) {
    memcpy(out, S.nrst.data(), S.nrst.size() * sizeof(int));
  } else if (which == 2) {
    double* o = (double*)out;
    size_t nt = S.b.size();
    memcpy(o, S.b.data(), nt * sizeof(double));
    memcpy(o + nt, S.x0.data(), 3 * nt * sizeof(double));
    memcpy(o + 4 * nt, S.n0.data(), 3 * nt * sizeof(double));
    for (size_t t = 0; t < nt; t++) o[7 * nt + t] = S.band2[t];
  } else {
    return HR_ERR_ARG;
  }
  return HR_OK;
}

extern "C" void hr_e2g_destroy(hr_e2g* E) {
  if (!E) return;
  cudaStreamSynchronize(E->owner->c.stream);
  delete E;
}

extern "C" double hr_e2g_p_exact(double x, double y, double z) { return e2g_setup::p_exact(x, y, z); }
extern "C" void hr_e2g_u_exact(double x, double y, double z, double* u) { e2g_setup::u_exact(x, y, z, u); }

extern "C" int hr_e2g_snapshot(hr_e2g* E) {
  if (!E) return HR_ERR_ARG;
  Ctx& C = E->owner->c;
  try {
    const long M = E->S.N + 1, m3 = M * M * M;
    cudaStream_t st = C.stream;
    if (!E->have_ref) {
      E->p_ref.alloc(m3);
      E->u_ref.alloc(3 * m3);
    }
    HR_CHECK_CUDA(cudaMemcpyAsync(E->p_ref.p, E->p_ext.p, sizeof(double) * m3, cudaMemcpyDeviceToDevice, st));
    HR_CHECK_CUDA(cudaMemcpyAsync(E->u_ref.p, E->u_ext.p, sizeof(double) * 3 * m3, cudaMemcpyDeviceToDevice, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
    E->have_ref = true;
  } catch (const hr::Error& e) {
    C.err = e.what();
    return e.code;
  }
  return HR_OK;
}

extern "C" int hr_e2g_midplane(hr_e2g* E, double* out) {
  if (!E || !out) return HR_ERR_ARG;
  Ctx& C = E->owner->c;
  try {
    cudaStream_t st = C.stream;
    if (!E->ran) throw Error(HR_ERR_STATE, "hr_e2g_midplane needs a completed hr_e2g_run");
    const int N = E->S.N;
    const long M = N + 1, mm = M * M;
    DBuf<double> d;
    d.alloc(4 * (size_t)mm);
    midplane_kernel<<<(unsigned)((mm + 255) / 256), 256, 0, st>>>(N, E->S.h, E->p_ext.p, E->u_ext.p, d.p);
    C.launches++;
    HR_CHECK_CUDA(cudaGetLastError());
    HR_CHECK_CUDA(cudaMemcpyAsync(out, d.p, sizeof(double) * 4 * mm, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  } catch (const Error& e) {
    C.err = e.what();
    return e.code;
  }
  return HR_OK;
}

extern "C" int hr_e2g_error_norms(hr_e2g* E, hr_e2g_errors* out) {
  if (!E || !out) return HR_ERR_ARG;
  Ctx& C = E->owner->c;
  try {
    cudaStream_t st = C.stream;
    const int N = E->S.N;
    const long M = N + 1, m3 = M * M * M;
    DBuf<double> part, bpart;
    part.alloc((size_t)kErrBlocks * kErrVals);
    bpart.alloc(2 * (size_t)kErrBlocks);
    grid_errors_kernel<<<kErrBlocks, kErrThreads, 0, st>>>(N, E->S.h, E->p_ext.p, E->u_ext.p,
                                                           E->have_ref ? E->p_ref.p : nullptr,
                                                           E->have_ref ? E->u_ref.p : nullptr, part.p);
    band_errors_kernel<<<kErrBlocks, kErrThreads, 0, st>>>(N, E->S.h, E->nband, E->gb.p, E->u_bi.p, bpart.p);
    C.launches += 2;
    HR_CHECK_CUDA(cudaGetLastError());
    std::vector<double> h((size_t)kErrBlocks * kErrVals), hb(2 * (size_t)kErrBlocks);
    HR_CHECK_CUDA(cudaMemcpyAsync(h.data(), part.p, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaMemcpyAsync(hb.data(), bpart.p, sizeof(double) * hb.size(), cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
    double v[kErrVals] = {0};
    double bm = 0.0, bs = 0.0;
    for (int b = 0; b < kErrBlocks; b++) {
      for (int q = 0; q < kErrVals; q++) {
        const double x = h[(size_t)b * kErrVals + q];
        v[q] = (q % 2 == 0) ? std::max(v[q], x) : v[q] + x;
      }
      bm = std::max(bm, hb[2 * b]);
      bs += hb[2 * b + 1];
    }
    out->p_max = v[0];
    out->p_rms = sqrt(v[1] / (double)m3);
    out->u_max = v[2];
    out->u_rms = sqrt(v[3] / (double)m3);
    out->band_u_max = bm;
    out->band_u_rms = E->nband > 0 ? sqrt(bs / (double)E->nband) : 0.0;
    if (E->have_ref) {
      out->ref_p_max_rel = v[6] > 0 ? v[4] / v[6] : 0.0;
      out->ref_p_rel_l2 = v[7] > 0 ? sqrt(v[5] / v[7]) : 0.0;
      out->ref_u_max_rel = v[10] > 0 ? v[8] / v[10] : 0.0;
      out->ref_u_rel_l2 = v[11] > 0 ? sqrt(v[9] / v[11]) : 0.0;
    } else {
      out->ref_p_max_rel = out->ref_p_rel_l2 = out->ref_u_max_rel = out->ref_u_rel_l2 = -1.0;
    }
  } catch (const hr::Error& e) {
    C.err = e.what();
    return e.code;
  }
  return HR_OK;
}
