// hr_noalloc.cu — an all-pairs plain Stokeslet sum on caller-owned device
// buffers that performs no device allocation at all.
//
// Some callers cannot call cudaMalloc: code that runs while a memory pool or
// framework allocator owns the device memory, code on a path that must not
// synchronize the device (cudaMalloc/cudaFree can), or a callback with no
// allocator of its own. For them this entry point keeps its only scratch,
// the per-chunk partial sums of the split-source sum, in a fixed-size
// file-scope __device__ array that every GPU loading the library holds until
// the process exits.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress and caches it for that
// device; make that first call before any stream capture. The cached address
// belongs to the device's primary context: after cudaDeviceReset on that
// device the entry point must not be called again in this process. Every call shares
// the array and leaves the last call's partial sums in it; each call writes
// every slot it later reads, so nothing needs clearing, but two calls that
// overlap on the GPU (different streams, no ordering) race on the array.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/highreg_b200.h"

namespace {

// 4 Mi doubles = 32 MiB of partial sums: 3 doubles per (target, source chunk).
constexpr long kScratchDoubles = 4L << 20;
constexpr int kThreads = 128;
constexpr int kTile = 256;
constexpr int kChunk = 2048;  // sources per chunk
constexpr int kMaxChunks = 64;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_dev[64] = {nullptr};  // per device ordinal, set on first use

// Partial sums of one (target block, source chunk): the plain Stokeslet of
// the sum kernel family, H1 = A/r, H2 = (f.dx) A / r^3, from interleaved
// device arrays staged through shared memory.
__global__ void __launch_bounds__(kThreads) away_partial_kernel(
    const double* __restrict__ xs, const double* __restrict__ area, const double* __restrict__ f,
    int nq, const double* __restrict__ xt, int nt, int chunk, double* __restrict__ partial) {
  __shared__ double s[7][kTile];
  const int t = blockIdx.x * kThreads + threadIdx.x;
  const bool valid = t < nt;
  const double px = valid ? xt[3 * t] : 0.0, py = valid ? xt[3 * t + 1] : 0.0,
               pz = valid ? xt[3 * t + 2] : 0.0;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  const int c = blockIdx.y;
  const int j0 = c * chunk, j1 = min(nq, j0 + chunk);
  for (int s0 = j0; s0 < j1; s0 += kTile) {
    const int cnt = min(kTile, j1 - s0);
    __syncthreads();
    for (int i = threadIdx.x; i < cnt; i += kThreads) {
      const int j = s0 + i;
      s[0][i] = xs[3 * j];
      s[1][i] = xs[3 * j + 1];
      s[2][i] = xs[3 * j + 2];
      s[3][i] = area[j];
      s[4][i] = f[3 * j];
      s[5][i] = f[3 * j + 1];
      s[6][i] = f[3 * j + 2];
    }
    __syncthreads();
    if (valid) {
#pragma unroll 2
      for (int i = 0; i < cnt; i++) {
        const double dx = px - s[0][i], dy = py - s[1][i], dz = pz - s[2][i];
        const double r2 = dx * dx + dy * dy + dz * dz;
        const double rinv = rsqrt(r2);
        const double fdd = s[4][i] * dx + s[5][i] * dy + s[6][i] * dz;
        const double H1 = s[3][i] * rinv;
        const double H2 = fdd * H1 * (rinv * rinv);
        a0 += s[4][i] * H1 + dx * H2;
        a1 += s[5][i] * H1 + dy * H2;
        a2 += s[6][i] * H1 + dz * H2;
      }
    }
  }
  if (valid) {
    double* o = partial + ((size_t)c * nt + t) * 3;
    o[0] = a0;
    o[1] = a1;
    o[2] = a2;
  }
}

// out = scale * sum over chunks, in chunk order (deterministic).
__global__ void away_reduce_kernel(const double* __restrict__ partial, int nt, int nchunks,
                                   double scale, double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int c = 0; c < nchunks; c++) {
    const double* p = partial + ((size_t)c * nt + t) * 3;
    a0 += p[0];
    a1 += p[1];
    a2 += p[2];
  }
  out[3 * t] = a0 * scale;
  out[3 * t + 1] = a1 * scale;
  out[3 * t + 2] = a2 * scale;
}

}  // namespace

extern "C" long long hr_stokeslet_away_noalloc_max_targets(void) { return kScratchDoubles / 3; }

extern "C" int hr_stokeslet_away_noalloc(const double* xyz_src_dev, const double* area_dev,
                                         const double* f_dev, int nq, const double* xyz_tgt_dev,
                                         int nt, double* out_dev, void* stream) {
  if (nq < 0 || nt < 0) return HR_ERR_ARG;
  // interleaved source and target indices (3 j + k) are int arithmetic
  if (3LL * nq > 2147483647LL) return HR_ERR_ARG;
  if (nt == 0) return HR_OK;
  if ((long long)3 * nt > kScratchDoubles) return HR_ERR_ARG;  // beyond the scratch array
  if (!xyz_tgt_dev || !out_dev || (nq > 0 && (!xyz_src_dev || !area_dev || !f_dev))) return HR_ERR_ARG;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return HR_ERR_CUDA;
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_dev[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return HR_ERR_CUDA;
      g_scratch_dev[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_dev[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double scale = 1.0 / (8.0 * 3.14159265358979323846);
  int nchunks = nq > 0 ? (nq + kChunk - 1) / kChunk : 1;
  long long fit = kScratchDoubles / (3LL * nt);
  if (nchunks > kMaxChunks) nchunks = kMaxChunks;
  if (nchunks > fit) nchunks = (int)fit;
  const int chunk = nq > 0 ? (nq + nchunks - 1) / nchunks : 0;
  dim3 grid((nt + kThreads - 1) / kThreads, nchunks);
  away_partial_kernel<<<grid, kThreads, 0, st>>>(xyz_src_dev, area_dev, f_dev, nq, xyz_tgt_dev, nt,
                                                 chunk, scratch);
  away_reduce_kernel<<<(nt + 255) / 256, 256, 0, st>>>(scratch, nt, nchunks, scale, out_dev);
  // peek, not get: a launch error stays visible to the caller's own error
  // handling, and an earlier error of the caller's is not consumed here
  if (cudaPeekAtLastError() != cudaSuccess) return HR_ERR_CUDA;
  return HR_OK;
}
