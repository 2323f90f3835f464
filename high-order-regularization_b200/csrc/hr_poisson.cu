// hr_poisson.cu — the extend-to-grid Poisson solve on the device
// (solve_Poisson + fftw_DST_Poisson3d_FD, E2G/main.cpp:969-1044, 1423-1823).
//
// DST-I (FFTW RODFT00, unnormalised) of length n along one axis is computed
// from a real FFT of length N = n + 1 with the classical sine-transform
// pre/post-processing (the auxiliary-array method for the sine transform,
// e.g. Press et al., Numerical Recipes, "sinft"):
//   y_0 = 0,  y_j = sin(j pi/N) (x_j + x_{N-j}) + (x_j - x_{N-j}) / 2,
//   Y_k = sum_j y_j e^{-2 pi i jk/N} = R_k + i I_k,
//   F_{2k} = -I_k,  F_1 = R_0 / 2,  F_{2k+1} = F_{2k-1} + R_k,
// where F_k = sum_j x_j sin(pi jk/N) and RODFT00 returns 2 F_{k}, k = 1..n.
// Each pass transforms along the contiguous axis and its post kernel writes
// the result with the axes rotated ([a][b][c] -> [c][a][b]), so three passes
// cover the three axes and restore the layout. The last forward pass divides
// by the eigenvalues of the 4th-order compact Laplacian; the last inverse
// pass applies the 1/(2(n+1))^3 scale and adds the extension w into u.
#include <cufft.h>

#include <cmath>
#include <memory>
#include <vector>

#include "hr_runtime.h"

namespace hr {

namespace {

#define HR_CHECK_CUFFT(call)                                                       \
  do {                                                                             \
    cufftResult r_ = (call);                                                       \
    if (r_ != CUFFT_SUCCESS)                                                       \
      throw ::hr::Error(HR_ERR_CUDA, std::string(#call) + ": cufft error " + std::to_string((int)r_)); \
  } while (0)

// y[l][j] = sin(j pi/N)(x_j + x_{N-j}) + (x_j - x_{N-j})/2, x_j = in[l][j-1]
__global__ void dst_pre_kernel(long lines, int n, const double* __restrict__ in,
                               const double* __restrict__ sintab, double* __restrict__ y) {
  const int N = n + 1;
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long total = lines * N;
  for (; idx < total; idx += (long)gridDim.x * blockDim.x) {
    long l = idx / N;
    int j = (int)(idx - l * N);
    double v = 0.0;
    if (j > 0) {
      const double* row = in + l * n;
      double xj = row[j - 1];
      double xm = (N - j - 1 < n && N - j - 1 >= 0 && N - j != N) ? row[N - j - 1] : 0.0;
      v = sintab[j] * (xj + xm) + 0.5 * (xj - xm);
    }
    y[idx] = v;
  }
}

// mode 0: plain; mode 1: divide by eigenvalue (i,j,k) = (k_line, line -> (j,k));
// mode 2: scale and add into u grid (N+1)^3 at interior offset, u pre-filled with w.
__global__ void dst_post_kernel(long lines, int n, const double2* __restrict__ Z,
                                double* __restrict__ out, int mode, const double* __restrict__ evc,
                                const double* __restrict__ evs, double scale,
                                const double* __restrict__ w, double* __restrict__ u) {
  const int N = n + 1;
  const int H = N / 2;
  long l = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= lines) return;
  const double2* z = Z + l * (H + 1);
  // line l of the input [a][b][c] layout is (a, b) = (l / nb, l % nb) with
  // nb = n; the output position of element k is out[k][l].
  const long L = lines;
  int ja = 0, jb = 0;
  double sa = 0, ca = 0, sb = 0, cb = 0;
  if (mode != 0) {
    ja = (int)(l / n);
    jb = (int)(l % n);
    ca = evc[ja];
    sa = evs[ja];
    cb = evc[jb];
    sb = evs[jb];
  }
  auto emit = [&](int k, double F2) {
    // F2 = 2 F_{k+1}: RODFT00 output index k
    if (mode == 0) {
      out[(long)k * L + l] = F2;
    } else if (mode == 1) {
      // factor for (i, j, k) = (k, ja, jb) (E2G/main.cpp:1447-1476)
      double c1 = evc[k], s1 = evs[k];
      double lap7 = s1 + sa + sb;
      double sum8 = c1 * ca * cb;
      double factor = 2.0 / 3.0 * (2.0 * lap7 + sum8 - 1.0);
      double v = F2;
      if (fabs(factor) > 1.e-14) v /= factor;
      else v = 0.0;
      out[(long)k * L + l] = v;
    } else {
      const int M = n + 2;  // grid size N_grid + 1
      long gi = ((long)(k + 1) * M + (ja + 1)) * M + (jb + 1);
      u[gi] = w[gi] + F2 * scale;
    }
  };
  double2 z0 = z[0];
  double Fodd = z0.x;  // 2 F_1 = R_0
  emit(0, Fodd);
  for (int k = 1; k < H; k++) {
    double2 zk = z[k];
    emit(2 * k - 1, -2.0 * zk.y);  // 2 F_{2k} = -2 I_k
    Fodd += 2.0 * zk.x;            // 2 F_{2k+1} = 2 F_{2k-1} + 2 R_k
    if (2 * k < n) emit(2 * k, Fodd);
  }
}

// Transfinite (Coons) extension of the boundary values (extend_into_cube,
// E2G/main.cpp:1494-1527).
__global__ void extend_kernel(int N, double L, double h, const double* __restrict__ g,
                              double* __restrict__ G) {
  const long M = N + 1;
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= M * M * M) return;
  int i = (int)(idx / (M * M)), j = (int)((idx / M) % M), k = (int)(idx % M);
  auto at = [&](int a, int b, int c) { return g[((long)a * M + b) * M + c]; };
  double x = i * h / L, y = j * h / L, z = k * h / L;
  double F, E1, E2, E3, C;
  F = x * at(N, j, k) + (1.0 - x) * at(0, j, k);
  F += y * at(i, N, k) + (1.0 - y) * at(i, 0, k);
  F += z * at(i, j, N) + (1.0 - z) * at(i, j, 0);
  E1 = (1.0 - y) * (1.0 - z) * at(i, 0, 0) + (1.0 - y) * z * at(i, 0, N) +
       y * (1.0 - z) * at(i, N, 0) + y * z * at(i, N, N);
  E2 = (1.0 - x) * (1.0 - z) * at(0, j, 0) + (1.0 - x) * z * at(0, j, N) +
       x * (1.0 - z) * at(N, j, 0) + x * z * at(N, j, N);
  E3 = (1.0 - x) * (1.0 - y) * at(0, 0, k) + (1.0 - x) * y * at(0, N, k) +
       x * (1.0 - y) * at(N, 0, k) + x * y * at(N, N, k);
  C = (1.0 - x) * (1.0 - y) * (1.0 - z) * at(0, 0, 0) + (1.0 - x) * (1.0 - y) * z * at(0, 0, N) +
      (1.0 - x) * y * (1.0 - z) * at(0, N, 0) + (1.0 - x) * y * z * at(0, N, N) +
      x * (1.0 - y) * (1.0 - z) * at(N, 0, 0) + x * (1.0 - y) * z * at(N, 0, N) +
      x * y * (1.0 - z) * at(N, N, 0) + x * y * z * at(N, N, N);
  G[idx] = F - E1 - E2 - E3 + C;
}

// 4th-order compact Laplacian RHS (lapl_4ord_inCube, lapl_4ord_nearSurfc,
// dp_d{x,y,z}_4ord: E2G/main.cpp:1566-1823), one fused pass over the interior.
__global__ void rhs_kernel(int N, double h, const double* __restrict__ Gw,
                           const double* __restrict__ u, const uint8_t* __restrict__ band2,
                           const uint8_t* __restrict__ outside, const double* __restrict__ p,
                           int axis, double* __restrict__ rhs) {
  const long M = N + 1;
  const long n = N - 1;
  long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n * n * n) return;
  int i = (int)(idx / (n * n)) + 1, j = (int)((idx / n) % n) + 1, k = (int)(idx % n) + 1;
  auto G = [&](const double* a, int ii, int jj, int kk) { return a[((long)ii * M + jj) * M + kk]; };
  auto lap = [&](const double* a) {
    double lap7 = G(a, i + 1, j, k) + G(a, i - 1, j, k) + G(a, i, j + 1, k) + G(a, i, j - 1, k) +
                  G(a, i, j, k + 1) + G(a, i, j, k - 1) - 6.0 * G(a, i, j, k);
    double temp1 = G(a, i + 1, j + 1, k + 1) + G(a, i + 1, j - 1, k + 1) +
                   G(a, i - 1, j + 1, k + 1) + G(a, i - 1, j - 1, k + 1) - 4.0 * G(a, i, j, k);
    double temp2 = G(a, i + 1, j + 1, k - 1) + G(a, i + 1, j - 1, k - 1) +
                   G(a, i - 1, j + 1, k - 1) + G(a, i - 1, j - 1, k - 1) - 4.0 * G(a, i, j, k);
    return lap7 + (temp1 + temp2) / 8.0;
  };
  double r = -2.0 / 3.0 * lap(Gw);
  const long gi = ((long)i * M + j) * M + k;
  if (band2[gi]) r += 2.0 / 3.0 * lap(u);
  if (axis >= 0 && outside[gi]) {
    const int c = axis == 0 ? i : (axis == 1 ? j : k);
    const int di = axis == 0, dj = axis == 1, dk = axis == 2;
    auto P = [&](int o) { return G(p, i + o * di, j + o * dj, k + o * dk); };
    double d;
    if (c == 0 || c == 1) {
      d = -(25.0 / 12.0) * P(0) + 4.0 * P(1) - 3.0 * P(2) + (4.0 / 3.0) * P(3) - 0.25 * P(4);
    } else if (c == N || c == (N - 1)) {
      d = (25.0 / 12.0) * P(0) - 4.0 * P(-1) + 3.0 * P(-2) - (4.0 / 3.0) * P(-3) + 0.25 * P(-4);
    } else {
      d = -P(2) + 8.0 * P(1) - 8.0 * P(-1) + P(-2);
      d /= 12.0;
    }
    r += d * h;
  }
  rhs[idx] = r;
}

struct DstPlan {
  int n = 0;
  cufftHandle plan = 0;
  DBuf<double> y, sintab, evc, evs;
  DBuf<double2> z;
  DBuf<double> tmp;
  void make(Ctx& C, int n_) {
    n = n_;
    const int N = n + 1;
    HR_REQUIRE(N % 2 == 0, "DST-I via real FFT needs n + 1 even");
    const long lines = (long)n * n;
    int dims[1] = {N};
    int inembed[1] = {N}, onembed[1] = {N / 2 + 1};
    HR_CHECK_CUFFT(cufftPlanMany(&plan, 1, dims, inembed, 1, N, onembed, 1, N / 2 + 1, CUFFT_D2Z,
                                 (int)lines));
    HR_CHECK_CUFFT(cufftSetStream(plan, C.stream));
    y.alloc((size_t)lines * N);
    z.alloc((size_t)lines * (N / 2 + 1));
    tmp.alloc((size_t)n * n * n);
    std::vector<double> st(N), c(n), s(n);
    for (int j = 0; j < N; j++) st[j] = sin(j * 3.14159265358979323846 / N);
    // eigenvalue factors exactly as E2G/main.cpp:1445-1460 evaluates them
    const double PI = 3.14159265358979323846;
    double pi_over_n = PI / (n + 1);
    for (int i = 0; i < n; i++) {
      c[i] = cos((i + 1) * pi_over_n);
      double s1 = sin((i + 1) * pi_over_n / 2.0);
      s1 *= -2.0 * s1;
      s[i] = s1;
    }
    sintab.upload(st, C.stream);
    evc.upload(c, C.stream);
    evs.upload(s, C.stream);
  }
  ~DstPlan() {
    if (plan) cufftDestroy(plan);
  }
  // one pass: in [n][n][n] -> out rotated
  void pass(Ctx& C, const double* in, double* out, int mode, double scale, const double* w,
            double* u) {
    const long lines = (long)n * n;
    const int N = n + 1;
    long tot = lines * N;
    int blocks = (int)std::min<long>((tot + 255) / 256, 148L * 32);
    dst_pre_kernel<<<blocks, 256, 0, C.stream>>>(lines, n, in, sintab.p, y.p);
    HR_CHECK_CUFFT(cufftExecD2Z(plan, y.p, (cufftDoubleComplex*)z.p));
    dst_post_kernel<<<(int)((lines + 127) / 128), 128, 0, C.stream>>>(lines, n, z.p, out, mode,
                                                                      evc.p, evs.p, scale, w, u);
    C.launches += 3;
    HR_CHECK_CUDA(cudaGetLastError());
  }
  // 3D DST-I of a (in place through tmp); last pass uses mode/scale/w/u
  void dst3(Ctx& C, double* a, int last_mode, double scale, const double* w, double* u) {
    pass(C, a, tmp.p, 0, 0, nullptr, nullptr);
    pass(C, tmp.p, a, 0, 0, nullptr, nullptr);
    pass(C, a, tmp.p, last_mode, scale, w, u);
    if (last_mode != 2)
      HR_CHECK_CUDA(cudaMemcpyAsync(a, tmp.p, sizeof(double) * (size_t)n * n * n,
                                    cudaMemcpyDeviceToDevice, C.stream));
  }
};

}  // namespace

void dst_poisson3d_dev(Ctx& C, int n, double* f_dev) {
  DstPlan P;
  P.make(C, n);
  P.dst3(C, f_dev, 1, 0.0, nullptr, nullptr);
  P.dst3(C, f_dev, 0, 0.0, nullptr, nullptr);
  double scale = 1. / pow(2 * (n + 1), 3);
  launch_scale_host(n * n * n, scale, f_dev, C.stream);
  C.launches++;
  HR_CHECK_CUDA(cudaGetLastError());
}

// The FFT plan, twiddle tables and grid work buffers of one grid size, kept
// across solves (a pipeline runs four solves per evaluation).
struct PoissonWork {
  int N = 0;
  DstPlan P;
  DBuf<double> w, rhs;
};

PoissonWork* poisson_work_create(Ctx& C, int N) {
  std::unique_ptr<PoissonWork> W(new PoissonWork);
  W->N = N;
  const long M = N + 1;
  const int n = N - 1;
  W->w.alloc(M * M * M);
  W->rhs.alloc((size_t)n * n * n);
  W->P.make(C, n);
  return W.release();
}

void poisson_work_destroy(PoissonWork* W) { delete W; }

void solve_poisson_dev(Ctx& C, int N, double L, const uint8_t* band2_dev, const uint8_t* out_dev,
                       const double* p_dev, double* u_dev, int variable, PoissonWork* work) {
  std::unique_ptr<PoissonWork> own;
  if (!work || work->N != N) {
    own.reset(poisson_work_create(C, N));
    work = own.get();
  }
  const double h = L / N;
  const long M = N + 1;
  const long m3 = M * M * M;
  const int n = N - 1;
  DBuf<double>& w = work->w;
  DBuf<double>& rhs = work->rhs;
  extend_kernel<<<(int)((m3 + 255) / 256), 256, 0, C.stream>>>(N, L, h, u_dev, w.p);
  const int axis = (variable >= 1 && variable <= 3) ? variable - 1 : -1;
  long n3 = (long)n * n * n;
  rhs_kernel<<<(int)((n3 + 255) / 256), 256, 0, C.stream>>>(N, h, w.p, u_dev, band2_dev, out_dev,
                                                            p_dev, axis, rhs.p);
  C.launches += 2;
  HR_CHECK_CUDA(cudaGetLastError());
  DstPlan& P = work->P;
  P.dst3(C, rhs.p, 1, 0.0, nullptr, nullptr);
  // u = w everywhere, then the interior gets w + scaled solution
  HR_CHECK_CUDA(cudaMemcpyAsync(u_dev, w.p, sizeof(double) * m3, cudaMemcpyDeviceToDevice, C.stream));
  double scale = 1. / pow(2 * (n + 1), 3);
  P.dst3(C, rhs.p, 2, scale, w.p, u_dev);
  // a temporary work area is freed at return; its buffers must be idle first
  if (own) HR_CHECK_CUDA(cudaStreamSynchronize(C.stream));
}

}  // namespace hr
