// hr_aux.cu — upward pass, density interpolation, permutations, combines and
// the deterministic vector kernels used by GMRES.
#include "hr_device.h"
#include "hr_pairs.cuh"

namespace hr {

namespace {

constexpr int kMomThreads = 384;
constexpr int kMomTile = 64;  // sources staged per sub-tile
static_assert(kMomThreads >= 4 * kMomTile, "a thread per (axis, source) and per source for the channels");
constexpr int kMaxP1 = 16;

// Upward pass of one (node, source range) item: the barycentric Lagrange
// proxy moments of Panel_Moments_SL / Panel_Moments_DL (2S/KITC.cpp:351-668):
//   M[c][ijk] = sum_s L_i(x_s) L_j(y_s) L_k(z_s) A_s q_c(s),
//   L_i(x) = (w_i / (x - t_i)) / sum_m (w_m / (x - t_m)),  w_j = (-1)^j d_j,
// with the removable singularity |x - t_j| < 1e-7 handled as in the reference.
// SL channels: f (3), n (3). DL channels: g (x) n (9, g-major), n (3).
template <bool DL>
__global__ void __launch_bounds__(kMomThreads) moments_kernel(
    const MomItem* __restrict__ items, int P1, const double* __restrict__ tcheb,
    const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
    const double* __restrict__ nx, const double* __restrict__ ny, const double* __restrict__ nz,
    const double* __restrict__ a, const double* __restrict__ qx, const double* __restrict__ qy,
    const double* __restrict__ qz, double* __restrict__ partial) {
  constexpr int C = DL ? 12 : 6;
  __shared__ double sL[3][kMaxP1][kMomTile];  // normalized Lagrange values per axis
  __shared__ double sA[kMomTile];
  __shared__ double sQ[C][kMomTile];
  __shared__ double sT[3 * kMaxP1];
  const MomItem it = items[blockIdx.x];
  const int Pf = P1 * P1 * P1;
  const int tid = threadIdx.x;
  if (tid < 3 * P1) sT[tid] = tcheb[(size_t)it.node * 3 * P1 + tid];
  // barycentric weights w_j = (-1)^j d_j, d_0 = d_P = 1/2 (2S/KITC.cpp:365-375)
  __syncthreads();
  for (int kk0 = 0; kk0 < Pf; kk0 += kMomThreads) {
    const int kk = kk0 + tid;
    const int i = kk / (P1 * P1), j = (kk / P1) % P1, k = kk % P1;
    double acc[C];
#pragma unroll
    for (int c = 0; c < C; c++) acc[c] = 0.0;
    for (int s0 = it.s0; s0 < it.s1; s0 += kMomTile) {
      const int cnt = min(kMomTile, it.s1 - s0);
      __syncthreads();
      // threads 0..191: the Lagrange values of one (axis, source) each,
      // normalized by their own axis sum; threads 192..255: area and channel
      // values of one source each
      if (tid < 3 * kMomTile) {
        const int ax = tid / kMomTile, src = tid - ax * kMomTile;
        if (src < cnt) {
          const int s = s0 + src;
          const double pc = ax == 0 ? x[s] : (ax == 1 ? y[s] : z[s]);
          double L[kMaxP1];
          int flag = -1;
          double S = 0.0;
          for (int jj = 0; jj < P1; jj++) {
            const double w = ((jj % 2 == 0) ? 1.0 : -1.0) * ((jj == 0 || jj == P1 - 1) ? 0.5 : 1.0);
            const double d = pc - sT[ax * P1 + jj];
            if (fabs(d) < 1.e-07) {
              flag = jj;
              L[jj] = 0.0;
            } else {
              L[jj] = w / d;
              S += L[jj];
            }
          }
          const double inv = 1.0 / S;
          for (int jj = 0; jj < P1; jj++)
            sL[ax][jj][src] = (flag > -1) ? (jj == flag ? 1.0 : 0.0) : L[jj] * inv;
        }
      } else if (tid < 4 * kMomTile) {
        const int src = tid - 3 * kMomTile;
        if (src < cnt) {
          const int s = s0 + src;
          sA[src] = a[s];
          const double n3[3] = {nx[s], ny[s], nz[s]};
          const double q3[3] = {qx[s], qy[s], qz[s]};
          if (DL) {
            for (int l = 0; l < 3; l++)
              for (int m = 0; m < 3; m++) sQ[3 * l + m][src] = q3[l] * n3[m];
            for (int m = 0; m < 3; m++) sQ[9 + m][src] = n3[m];
          } else {
            for (int m = 0; m < 3; m++) {
              sQ[m][src] = q3[m];
              sQ[3 + m][src] = n3[m];
            }
          }
        }
      }
      __syncthreads();
      if (kk < Pf) {
        for (int s = 0; s < cnt; s++) {
          const double v = sL[0][i][s] * sL[1][j][s] * sL[2][k][s] * sA[s];
#pragma unroll
          for (int c = 0; c < C; c++) acc[c] += v * sQ[c][s];
        }
      }
    }
    if (kk < Pf) {
#pragma unroll
      for (int c = 0; c < C; c++) partial[((size_t)it.out * C + c) * Pf + kk] = acc[c];
    }
  }
}

// Sums the partial moments of each node in item order (deterministic) and
// stores them proxy-major. The stresslet's 12 channels
// (g (x) n, g-major, then n) enter the far field only through
//   d.M.d = M00 d0^2 + M11 d1^2 + M22 d2^2 + (M01 + M10) d0 d1
//         + (M02 + M20) d0 d2 + (M12 + M21) d1 d2   and   Mn.d,
// so they are stored as those 6 symmetric combinations and Mn: FP64 10
// doubles per proxy (the last one zero), FP32 12 floats (the last three zero).
// The Stokeslet's 6 channels (f, n) are stored as they are: FP64 6 doubles,
// FP32 8 floats (the last two zero).
__global__ void moments_reduce_kernel(int C, int Pf, const int* __restrict__ item_start,
                                      const double* __restrict__ partial, double* __restrict__ mom,
                                      float* __restrict__ momf) {
  // one thread per (node, proxy, stored value): a value is one channel, or for
  // the stresslet's symmetric combinations the sum of two, each summed over
  // the node's items in item order
  const int node = blockIdx.y, o = blockIdx.z;
  const int kk = blockIdx.x * blockDim.x + threadIdx.x;
  if (kk >= Pf) return;
  const bool dl = C == 12;
  int c0 = o, c1 = -1;
  if (dl) {
    const int first[10] = {0, 4, 8, 1, 2, 5, 9, 10, 11, -1};
    const int second[10] = {-1, -1, -1, 3, 6, 7, -1, -1, -1, -1};
    c0 = first[o];
    c1 = second[o];
  }
  const int a = item_start[node], b = item_start[node + 1];
  double s0 = 0.0, s1 = 0.0;
  if (c0 >= 0)
    for (int q = a; q < b; q++) s0 += partial[((size_t)q * C + c0) * Pf + kk];
  if (c1 >= 0)
    for (int q = a; q < b; q++) s1 += partial[((size_t)q * C + c1) * Pf + kk];
  const double v = c1 >= 0 ? s0 + s1 : s0;
  const size_t k = (size_t)node * Pf + kk;
  if (dl) {
    mom[k * 10 + o] = v;  // o = 9: the zero pad
    momf[k * 12 + o] = (float)v;
    if (o == 9) momf[k * 12 + 10] = momf[k * 12 + 11] = 0.f;
  } else {
    mom[k * 6 + o] = v;
    momf[k * 8 + o] = (float)v;
    if (o == 5) momf[k * 8 + 6] = momf[k * 8 + 7] = 0.f;
  }
}

__global__ void permute_kernel(int n, const int* __restrict__ perm, const double* __restrict__ q3,
                               double* __restrict__ qx, double* __restrict__ qy,
                               double* __restrict__ qz, float* __restrict__ fqx,
                               float* __restrict__ fqy, float* __restrict__ fqz) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  int o = perm[p];
  const double a = q3[3 * o], b = q3[3 * o + 1], c = q3[3 * o + 2];
  qx[p] = a;
  qy[p] = b;
  qz[p] = c;
  fqx[p] = (float)a;
  fqy[p] = (float)b;
  fqz[p] = (float)c;
}

__global__ void permute_soa_kernel(int n, const int* __restrict__ perm,
                                   const double* __restrict__ src, double* __restrict__ dst) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  dst[p] = src[perm[p]];
}

// sixPoint_coeff (2S/main.cpp:750-757)
__device__ __forceinline__ void six_coeff(double p, double c[6]) {
  c[0] = -p * (p * p - 1.0) * (p - 2.0) * (p - 3.0) / 120.0;
  c[1] = p * (p - 1.0) * (p * p - 4.0) * (p - 3.0) / 24.0;
  c[2] = -(p * p - 1.0) * (p * p - 4.0) * (p - 3.0) / 12.0;
  c[3] = p * (p + 1.0) * (p * p - 4.0) * (p - 3.0) / 12.0;
  c[4] = -p * (p * p - 1.0) * (p + 2.0) * (p - 3.0) / 24.0;
  c[5] = p * (p * p - 1.0) * (p * p - 4.0) / 120.0;
}

// sixPointInterpolate over the precomputed stencil (2S/main.cpp:759-778, 1019-1039)
__global__ void interp_kernel(int ne, const int* __restrict__ tgt, const int* __restrict__ idx,
                              const double* __restrict__ pq, const double* __restrict__ g,
                              double* __restrict__ g0) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ne) return;
  double a[6], b[6];
  six_coeff(pq[2 * e], a);
  six_coeff(pq[2 * e + 1], b);
  const int* st = idx + 36 * (size_t)e;
  const int t = tgt[e];
  for (int comp = 0; comp < 3; comp++) {
    double ft[6];
    for (int jj = 0; jj < 6; jj++) {
      double s = 0.0;
      for (int ii = 0; ii < 6; ii++) s += a[ii] * g[3 * st[6 * ii + jj] + comp];
      ft[jj] = s;
    }
    double v = 0.0;
    for (int jj = 0; jj < 6; jj++) v += b[jj] * ft[jj];
    g0[3 * t + comp] = v;
  }
}

// u_out = u_in - on*factor; u_out -= comp*factor   (2S/main.cpp:612-676)
__global__ void matvec_combine_kernel(int n, double factor, const double* __restrict__ x,
                                      const double* __restrict__ on,
                                      const double* __restrict__ comp, double* __restrict__ y) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = x[i] - on[i] * factor;
  v -= comp[i] * factor;
  y[i] = v;
}

// SL = on; SL += comp; b = -SL * factor   (2S/main.cpp:202-207, 478-536)
__global__ void rhs_combine_kernel(int n, double factor, const double* __restrict__ on,
                                   const double* __restrict__ comp, double* __restrict__ b) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = on[i];
  s += comp[i];
  b[i] = -s * factor;
}

constexpr int kDotThreads = 256;
constexpr int kMaxCols = 64;

// partial[blk][c] = sum over this block's strided range of V[c][i] * w[i]
__global__ void __launch_bounds__(kDotThreads) dots_kernel(int n, int ncols,
                                                           const double* __restrict__ V, long ldv,
                                                           const double* __restrict__ w,
                                                           double* __restrict__ partial) {
  __shared__ double red[kDotThreads / 32][kMaxCols];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int c0 = 0; c0 < ncols; c0 += 8) {
    double acc[8];
#pragma unroll
    for (int q = 0; q < 8; q++) acc[q] = 0.0;
    for (int i = blockIdx.x * kDotThreads + tid; i < n; i += gridDim.x * kDotThreads) {
      const double wi = w[i];
#pragma unroll
      for (int q = 0; q < 8; q++)
        if (c0 + q < ncols) acc[q] += V[(size_t)(c0 + q) * ldv + i] * wi;
    }
#pragma unroll
    for (int q = 0; q < 8; q++) {
      double v = acc[q];
      for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
      if (lane == 0 && c0 + q < ncols) red[warp][c0 + q] = v;
    }
  }
  __syncthreads();
  if (tid < ncols) {
    double s = 0.0;
    for (int wq = 0; wq < kDotThreads / 32; wq++) s += red[wq][tid];
    partial[(size_t)blockIdx.x * kMaxCols + tid] = s;
  }
}

// One warp per column: lane l sums blocks l, l + 32, ... in order, then a
// fixed shuffle tree adds the lanes (deterministic).
__global__ void dots_finalize_kernel(int ncols, int nblk, const double* __restrict__ partial,
                                     double* __restrict__ out) {
  const int c = blockIdx.x, lane = threadIdx.x;
  if (c >= ncols) return;
  double s = 0.0;
  for (int b = lane; b < nblk; b += 32) s += partial[(size_t)b * kMaxCols + c];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if (lane == 0) out[c] = s;
}

// w += sign * sum_c coef[c] V[c]
__global__ void axpy_multi_kernel(int n, int ncols, const double* __restrict__ V, long ldv,
                                  const double* __restrict__ coef, double sign,
                                  double* __restrict__ w) {
  __shared__ double sc[kMaxCols];
  if (threadIdx.x < ncols) sc[threadIdx.x] = coef[threadIdx.x];
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = w[i];
    for (int c = 0; c < ncols; c++) v += sign * sc[c] * V[(size_t)c * ldv + i];
    w[i] = v;
  }
}

__global__ void scale_dev_kernel(int n, const double* __restrict__ s, double* __restrict__ w) {
  const double f = 1.0 / s[0];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] *= f;
}
__global__ void scale_kernel(int n, double s, double* __restrict__ w) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] *= s;
}
__global__ void sub_kernel(int n, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ o) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    o[i] = a[i] - b[i];
}
__global__ void copy_kernel(int n, const double* __restrict__ a, double* __restrict__ o) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) o[i] = a[i];
}

// FP64 FMA throughput loop: 8 independent chains per thread.
__global__ void fma_peak_kernel(double* out, int iters) {
  double a[8];
  for (int q = 0; q < 8; q++) a[q] = 1.0 + 1e-9 * (threadIdx.x + q);
  const double m = 0.999999999, c = 1e-12;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int q = 0; q < 8; q++) a[q] = fma(a[q], m, c);
  }
  double s = 0;
  for (int q = 0; q < 8; q++) s += a[q];
  if (s == 12345.678) out[0] = s;  // keeps the loop alive
}

// FP32 counterpart: 16 independent FMA chains per thread.
__global__ void fma_peak32_kernel(float* out, int iters) {
  float a[16];
  for (int q = 0; q < 16; q++) a[q] = 1.0f + 1e-6f * (threadIdx.x + q);
  const float m = 0.9999999f, c = 1e-7f;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int q = 0; q < 16; q++) a[q] = fmaf(a[q], m, c);
  }
  float s = 0;
  for (int q = 0; q < 16; q++) s += a[q];
  if (s == 12345.678f) out[0] = s;  // keeps the loop alive
}

inline int nblk(long n, int t) { return (int)std::min<long>((n + t - 1) / t, 148L * 16); }

}  // namespace

void launch_moments(int dl, const MomItem* d_items, int nitems, int P1, const double* tcheb,
                    const double* x, const double* y, const double* z, const double* nx,
                    const double* ny, const double* nz, const double* a, const double* qx,
                    const double* qy, const double* qz, double* partial, cudaStream_t st) {
  if (nitems <= 0) return;
  if (dl)
    moments_kernel<true><<<nitems, kMomThreads, 0, st>>>(d_items, P1, tcheb, x, y, z, nx, ny, nz, a,
                                                         qx, qy, qz, partial);
  else
    moments_kernel<false><<<nitems, kMomThreads, 0, st>>>(d_items, P1, tcheb, x, y, z, nx, ny, nz,
                                                          a, qx, qy, qz, partial);
}

void launch_moments_reduce(int C, int Pf, int nnodes_out, const int* d_item_start,
                           const double* partial, double* mom, float* momf, cudaStream_t st) {
  if (nnodes_out <= 0) return;
  dim3 grid((Pf + 127) / 128, nnodes_out, C == 12 ? 10 : 6);
  moments_reduce_kernel<<<grid, 128, 0, st>>>(C, Pf, d_item_start, partial, mom, momf);
}

void launch_permute(int n, const int* perm, const double* q3, double* qx, double* qy, double* qz,
                    float* fqx, float* fqy, float* fqz, cudaStream_t st) {
  if (n <= 0) return;
  permute_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, perm, q3, qx, qy, qz, fqx, fqy, fqz);
}

void launch_permute_soa(int n, const int* perm, const double* src, double* dst, cudaStream_t st) {
  if (n <= 0) return;
  permute_soa_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, perm, src, dst);
}

void launch_interp(int ne, const int* tgt, const int* idx, const double* pq, const double* g,
                   double* g0, cudaStream_t st) {
  if (ne <= 0) return;
  interp_kernel<<<(ne + 127) / 128, 128, 0, st>>>(ne, tgt, idx, pq, g, g0);
}

void launch_matvec_combine(int n, double factor, const double* x, const double* on,
                           const double* comp, double* y, cudaStream_t st) {
  if (n <= 0) return;
  matvec_combine_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, factor, x, on, comp, y);
}

void launch_rhs_combine(int n, double factor, const double* on, const double* comp, double* b,
                        cudaStream_t st) {
  if (n <= 0) return;
  rhs_combine_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, factor, on, comp, b);
}

void launch_dots(int n, int ncols, const double* V, long ldv, const double* w, double* partial,
                 cudaStream_t st) {
  dots_kernel<<<kRedBlocks, kDotThreads, 0, st>>>(n, ncols, V, ldv, w, partial);
}

void launch_dots_finalize(int ncols, const double* partial, double* out, cudaStream_t st) {
  dots_finalize_kernel<<<ncols, 32, 0, st>>>(ncols, kRedBlocks, partial, out);
}

void launch_axpy_multi(int n, int ncols, const double* V, long ldv, const double* coef,
                       double sign, double* w, cudaStream_t st) {
  axpy_multi_kernel<<<nblk(n, 256), 256, 0, st>>>(n, ncols, V, ldv, coef, sign, w);
}

void launch_scale(int n, const double* s_dev, double* w, cudaStream_t st) {
  scale_dev_kernel<<<nblk(n, 256), 256, 0, st>>>(n, s_dev, w);
}
void launch_scale_host(int n, double s, double* w, cudaStream_t st) {
  scale_kernel<<<nblk(n, 256), 256, 0, st>>>(n, s, w);
}
void launch_sub(int n, const double* a, const double* b, double* out, cudaStream_t st) {
  sub_kernel<<<nblk(n, 256), 256, 0, st>>>(n, a, b, out);
}
void launch_copy(int n, const double* a, double* out, cudaStream_t st) {
  copy_kernel<<<nblk(n, 256), 256, 0, st>>>(n, a, out);
}

void launch_fma_peak(double* out, int iters, int blocks, cudaStream_t st) {
  fma_peak_kernel<<<blocks, 256, 0, st>>>(out, iters);
}

void launch_fma_peak32(float* out, int iters, int blocks, cudaStream_t st) {
  fma_peak32_kernel<<<blocks, 256, 0, st>>>(out, iters);
}

}  // namespace hr
