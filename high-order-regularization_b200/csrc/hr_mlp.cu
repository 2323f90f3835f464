// hr_mlp.cu — the learned GMRES warm start: a pointwise MLP
// 12 -> 64 -> 64 -> 64 -> 3 with SiLU hidden activations and FP32 weights,
// trained on the GPU by these kernels (forward, backward, Adam) and applied by
// an inference kernel that writes an FP64 initial guess.
//
// Parameter layout (flat, 9347 floats): W1[12][64] b1[64] W2[64][64] b2[64]
// W3[64][64] b3[64] W4[64][3] b4[3]; W[i][j] is the weight from input i to
// output j. Inputs are normalized in the kernels: x' = (x - mean) / std; the
// output is scaled by out_scale.
//
// Kernels:
//   fwd_bwd_kernel   one thread per sample: forward, loss, backward deltas.
//                    Weights live in shared memory (broadcast reads, 128-bit
//                    rows); each thread's hidden activations are a column of a
//                    shared array, so layer loops never index registers
//                    dynamically. Pre-activations and deltas go to global
//                    memory feature-major ([feature][batch], coalesced).
//   grad_kernel      parameter gradients as the batch contraction
//                    dW = A^T Delta, split over chunks of 32 samples staged in
//                    shared memory; each thread owns ~37 parameters.
//   grad_reduce      sums the chunk partials in chunk order (deterministic).
//   adam_kernel      Adam with bias correction (Kingma & Ba 2015).
//   infer_kernel     guess = base + out_scale * MLP(x), FP64 out.
// The network is FP32 SIMT arithmetic: about 55 kflop per training sample, so
// a whole training run is a small fraction of the solves that produce its data.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "hr_runtime.h"

namespace {

constexpr int kIn = 12, kH = 64, kOut = 3;
constexpr int oW1 = 0, ob1 = oW1 + kIn * kH, oW2 = ob1 + kH, ob2 = oW2 + kH * kH, oW3 = ob2 + kH,
              ob3 = oW3 + kH * kH, oW4 = ob3 + kH, ob4 = oW4 + kH * kOut, kNP = ob4 + kOut;
static_assert(kNP == 9347, "parameter count");
constexpr int kZ = 3 * kH;            // stored pre-activations per sample: z1, z2, z3
constexpr int kD = 3 * kH + kOut;     // stored deltas per sample: d1, d2, d3, d4
constexpr int kA = kIn + 3 * kH + 1;  // activation row in the gradient: x', s(z1), s(z2), s(z3), 1
constexpr int kThreads = 128;
constexpr int kGradThreads = 256;
constexpr int kPerThread = (kNP + kGradThreads - 1) / kGradThreads;  // 37
constexpr int kChunk = 32;
constexpr int kPpad = (kNP + 3) & ~3;

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigm(z);
  return s * (1.0f + z * (1.0f - s));
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  // splitmix64 finalizer (Steele, Lea, Flood 2014)
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

struct Norm {
  float mean[kIn], inv_std[kIn];
  float out_scale;
};

// Batch sample s: s itself (in-order batches) or a hash of (seed, step, s).
__device__ __forceinline__ long sample_index(long s, long n, unsigned long long seed, long step, int random) {
  if (!random) return s;
  const unsigned long long h = mix64(seed ^ mix64(((unsigned long long)step << 32) ^ (unsigned long long)s));
  return (long)(h % (unsigned long long)n);
}

// z[j] = bias[j] + sum_i col[i] * W[i][j], col = this thread's activation column.
__device__ __forceinline__ void dense64(const float* __restrict__ P, int oW, int ob, const float* col,
                                        float z[kH]) {
#pragma unroll
  for (int j = 0; j < kH; j++) z[j] = P[ob + j];
#pragma unroll 2
  for (int i = 0; i < kH; i++) {
    const float ai = col[i * kThreads];
    const float4* w = reinterpret_cast<const float4*>(P + oW + i * kH);
#pragma unroll
    for (int j4 = 0; j4 < kH / 4; j4++) {
      const float4 v = w[j4];
      z[4 * j4] += ai * v.x;
      z[4 * j4 + 1] += ai * v.y;
      z[4 * j4 + 2] += ai * v.z;
      z[4 * j4 + 3] += ai * v.w;
    }
  }
}

// Forward of one sample; on return z holds z3 and col holds s(z3).
// Zs (optional): feature-major store of z1, z2, z3 at column s of a batch of B.
__device__ __forceinline__ void forward(const float* __restrict__ P, const float* __restrict__ xin,
                                        const Norm& nm, float* col, float z[kH], float y[kOut],
                                        float* __restrict__ Zs, long s, long B) {
  float x[kIn];
#pragma unroll
  for (int i = 0; i < kIn; i++) x[i] = (xin[i] - nm.mean[i]) * nm.inv_std[i];
#pragma unroll
  for (int j = 0; j < kH; j++) z[j] = P[ob1 + j];
#pragma unroll
  for (int i = 0; i < kIn; i++) {
    const float4* w = reinterpret_cast<const float4*>(P + oW1 + i * kH);
#pragma unroll
    for (int j4 = 0; j4 < kH / 4; j4++) {
      const float4 v = w[j4];
      z[4 * j4] += x[i] * v.x;
      z[4 * j4 + 1] += x[i] * v.y;
      z[4 * j4 + 2] += x[i] * v.z;
      z[4 * j4 + 3] += x[i] * v.w;
    }
  }
  for (int layer = 0; layer < 3; layer++) {
#pragma unroll
    for (int j = 0; j < kH; j++) {
      if (Zs) Zs[(size_t)(layer * kH + j) * B + s] = z[j];
      col[j * kThreads] = silu(z[j]);
    }
    if (layer < 2) dense64(P, layer == 0 ? oW2 : oW3, layer == 0 ? ob2 : ob3, col, z);
  }
#pragma unroll
  for (int j = 0; j < kOut; j++) y[j] = P[ob4 + j];
#pragma unroll 4
  for (int i = 0; i < kH; i++) {
    const float ai = col[i * kThreads];
#pragma unroll
    for (int j = 0; j < kOut; j++) y[j] += ai * P[oW4 + i * kOut + j];
  }
}

__device__ __forceinline__ void load_params(float* P, const float* __restrict__ params) {
  for (int i = threadIdx.x; i < kNP; i += blockDim.x) P[i] = params[i];
}

// Training pass over a batch: forward, squared-error loss (mean over batch and
// components of (y - t / out_scale)^2), backward deltas.
__global__ void __launch_bounds__(kThreads) fwd_bwd_kernel(
    const float* __restrict__ params, Norm nm, const float* __restrict__ X, const float* __restrict__ T,
    long n, int batch, unsigned long long seed, long step, int random, long* __restrict__ idx_out,
    float* __restrict__ Zs, float* __restrict__ Ds, double* __restrict__ loss_part) {
  extern __shared__ __align__(16) float sm[];
  float* P = sm;              // kNP weights (padded)
  float* cols = sm + kPpad;   // kH x kThreads activation / delta columns
  __shared__ double red[kThreads / 32];
  load_params(P, params);
  __syncthreads();
  float* col = cols + threadIdx.x;
  const int s = blockIdx.x * kThreads + threadIdx.x;
  double l2 = 0.0;
  if (s < batch) {
    const long g = sample_index(s, n, seed, step, random);
    idx_out[s] = g;
    const long B = batch;
    float z[kH], y[kOut];
    forward(P, X + g * kIn, nm, col, z, y, Zs, s, B);
    float d4[kOut];
    const float inv = 2.0f / (float)((long)batch * kOut);
#pragma unroll
    for (int j = 0; j < kOut; j++) {
      const float e = y[j] - T[g * kOut + j] / nm.out_scale;
      l2 += (double)e * (double)e;
      d4[j] = e * inv;
      Ds[(size_t)(3 * kH + j) * B + s] = d4[j];
    }
    // d3 = (W4 d4) * s'(z3), z3 still in registers
    float d[kH];
#pragma unroll
    for (int i = 0; i < kH; i++) {
      float t = 0.f;
#pragma unroll
      for (int j = 0; j < kOut; j++) t += P[oW4 + i * kOut + j] * d4[j];
      d[i] = t * dsilu(z[i]);
      Ds[(size_t)(2 * kH + i) * B + s] = d[i];
    }
    // d2 = (W3 d3) * s'(z2), then d1 = (W2 d2) * s'(z1)
    for (int layer = 1; layer >= 0; layer--) {
      const int oW = layer == 1 ? oW3 : oW2;
#pragma unroll 2
      for (int i = 0; i < kH; i++) {
        const float4* w = reinterpret_cast<const float4*>(P + oW + i * kH);
        float t = 0.f;
#pragma unroll
        for (int j4 = 0; j4 < kH / 4; j4++) {
          const float4 v = w[j4];
          t += v.x * d[4 * j4] + v.y * d[4 * j4 + 1] + v.z * d[4 * j4 + 2] + v.w * d[4 * j4 + 3];
        }
        const float di = t * dsilu(Zs[(size_t)(layer * kH + i) * B + s]);
        col[i * kThreads] = di;
        Ds[(size_t)(layer * kH + i) * B + s] = di;
      }
#pragma unroll
      for (int i = 0; i < kH; i++) d[i] = col[i * kThreads];
    }
  }
  for (int off = 16; off > 0; off >>= 1) l2 += __shfl_down_sync(0xffffffffu, l2, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = l2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < kThreads / 32; w++) t += red[w];
    loss_part[blockIdx.x] = t;
  }
}

// Activation-row and delta-row index of parameter p, packed (a | d << 16).
__device__ __forceinline__ int param_rows(int p) {
  int a, d;
  if (p < ob1) { a = (p - oW1) / kH; d = (p - oW1) % kH; }
  else if (p < oW2) { a = kA - 1; d = p - ob1; }
  else if (p < ob2) { a = kIn + (p - oW2) / kH; d = kH + (p - oW2) % kH; }
  else if (p < oW3) { a = kA - 1; d = kH + (p - ob2); }
  else if (p < ob3) { a = kIn + kH + (p - oW3) / kH; d = 2 * kH + (p - oW3) % kH; }
  else if (p < oW4) { a = kA - 1; d = 2 * kH + (p - ob3); }
  else if (p < ob4) { a = kIn + 2 * kH + (p - oW4) / kOut; d = 3 * kH + (p - oW4) % kOut; }
  else { a = kA - 1; d = 3 * kH + (p - ob4); }
  return a | (d << 16);
}

// Partial gradient of every parameter over one chunk of samples.
__global__ void __launch_bounds__(kGradThreads) grad_kernel(Norm nm, const float* __restrict__ X, int batch,
                                                            const long* __restrict__ idx,
                                                            const float* __restrict__ Zs,
                                                            const float* __restrict__ Ds,
                                                            float* __restrict__ partial) {
  extern __shared__ __align__(16) float gsm[];
  float* sAct = gsm;                 // kChunk x kA
  float* sDel = gsm + kChunk * kA;   // kChunk x kD
  const int s0 = blockIdx.x * kChunk;
  const int cs = min(kChunk, batch - s0);
  for (int e = threadIdx.x; e < kChunk * kA; e += kGradThreads) {
    const int s = e % kChunk, a = e / kChunk;
    float v = 0.f;
    if (s < cs) {
      const long g = s0 + s;
      if (a < kIn) v = (X[idx[g] * kIn + a] - nm.mean[a]) * nm.inv_std[a];
      else if (a < kA - 1) v = silu(Zs[(size_t)(a - kIn) * batch + g]);
      else v = 1.0f;
    }
    sAct[s * kA + a] = v;
  }
  for (int e = threadIdx.x; e < kChunk * kD; e += kGradThreads) {
    const int s = e % kChunk, d = e / kChunk;
    sDel[s * kD + d] = s < cs ? Ds[(size_t)d * batch + s0 + s] : 0.f;
  }
  __syncthreads();
  int rows[kPerThread];
  float acc[kPerThread];
#pragma unroll
  for (int k = 0; k < kPerThread; k++) {
    const int p = threadIdx.x + k * kGradThreads;
    rows[k] = p < kNP ? param_rows(p) : (kA - 1);
    acc[k] = 0.f;
  }
  for (int s = 0; s < cs; s++) {
    const float* a = sAct + s * kA;
    const float* dd = sDel + s * kD;
#pragma unroll
    for (int k = 0; k < kPerThread; k++) acc[k] += a[rows[k] & 0xffff] * dd[rows[k] >> 16];
  }
  float* out = partial + (size_t)blockIdx.x * kNP;
#pragma unroll
  for (int k = 0; k < kPerThread; k++) {
    const int p = threadIdx.x + k * kGradThreads;
    if (p < kNP) out[p] = acc[k];
  }
}

__global__ void grad_reduce_kernel(const float* __restrict__ partial, int nchunks, float* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNP) return;
  float s = 0.f;
  for (int c = 0; c < nchunks; c++) s += partial[(size_t)c * kNP + p];
  grad[p] = s;
}

__global__ void adam_kernel(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNP) return;
  const float g = grad[p];
  const float mm = b1 * m[p] + (1.0f - b1) * g;
  const float vv = b2 * v[p] + (1.0f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  params[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

// Output frames of inference: samples start[f] .. start[f+1]-1 are rotated
// by R[f]^T (v_body = R v_world); n = 0 leaves the output as it is.
constexpr int kMaxFrames = 8;
struct Frames {
  int n;
  long start[kMaxFrames + 1];
  double R[kMaxFrames][9];
};

__global__ void __launch_bounds__(kThreads) infer_kernel(const float* __restrict__ params, Norm nm,
                                                         const float* __restrict__ X, long n,
                                                         const double* __restrict__ base,
                                                         double* __restrict__ out, float* __restrict__ raw,
                                                         Frames fr) {
  extern __shared__ __align__(16) float sm[];
  float* P = sm;
  float* cols = sm + kPpad;
  load_params(P, params);
  __syncthreads();
  const long s = (long)blockIdx.x * kThreads + threadIdx.x;
  if (s >= n) return;
  float z[kH], y[kOut];
  forward(P, X + s * kIn, nm, cols + threadIdx.x, z, y, nullptr, 0, 0);
  double v[kOut] = {y[0], y[1], y[2]};
  for (int f = 0; f < fr.n; f++) {
    if (s >= fr.start[f] && s < fr.start[f + 1]) {
      const double* R = fr.R[f];
      v[0] = R[0] * y[0] + R[3] * y[1] + R[6] * y[2];
      v[1] = R[1] * y[0] + R[4] * y[1] + R[7] * y[2];
      v[2] = R[2] * y[0] + R[5] * y[1] + R[8] * y[2];
    }
  }
#pragma unroll
  for (int j = 0; j < kOut; j++) {
    if (raw) raw[s * kOut + j] = y[j];
    if (out) out[s * kOut + j] = (base ? base[s * kOut + j] : 0.0) + (double)nm.out_scale * v[j];
  }
}

__global__ void sum_kernel(const double* __restrict__ part, int n, double* out) {
  double s = 0.0;
  for (int i = 0; i < n; i++) s += part[i];
  *out = s;
}

constexpr size_t kFwdSmem = sizeof(float) * ((size_t)kPpad + (size_t)kH * kThreads);
constexpr size_t kGradSmem = sizeof(float) * (size_t)kChunk * (kA + kD);

}  // namespace

struct hr_mlp {
  hr_ctx* owner = nullptr;
  Norm nm;
  hr::DBuf<float> params, grad, m, v, partial;
  hr::DBuf<float> Zs, Ds;
  hr::DBuf<long> idx;
  hr::DBuf<double> loss_part, loss;
  int cap = 0;
  long step = 0;
  void ensure(int batch) {
    if (batch <= cap) return;
    Zs.alloc((size_t)batch * kZ);
    Ds.alloc((size_t)batch * kD);
    idx.alloc(batch);
    loss_part.alloc((batch + kThreads - 1) / kThreads);
    partial.alloc((size_t)((batch + kChunk - 1) / kChunk) * kNP);
    cap = batch;
  }
};

namespace {

template <class F>
int mlp_guard(hr_mlp* M, F&& f) {
  try {
    f();
    return HR_OK;
  } catch (const hr::Error& e) {
    if (M && M->owner) M->owner->c.err = e.what();
    return e.code;
  } catch (const std::exception& e) {
    if (M && M->owner) M->owner->c.err = e.what();
    return HR_ERR_CUDA;
  }
}

void set_smem_attrs() {
  static bool done = false;
  if (done) return;
  HR_CHECK_CUDA(cudaFuncSetAttribute(fwd_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem));
  HR_CHECK_CUDA(cudaFuncSetAttribute(infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFwdSmem));
  HR_CHECK_CUDA(cudaFuncSetAttribute(grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGradSmem));
  done = true;
}

// FNV-1a 64-bit over a byte string.
unsigned long long fnv1a(const unsigned char* p, size_t n) {
  unsigned long long h = 1469598103934665603ULL;
  for (size_t i = 0; i < n; i++) {
    h ^= p[i];
    h *= 1099511628211ULL;
  }
  return h;
}

}  // namespace

extern "C" int hr_mlp_nparams(void) { return kNP; }

extern "C" int hr_mlp_create(hr_ctx* ctx, unsigned long long seed, hr_mlp** out) {
  if (!ctx || !out) return HR_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<hr_mlp> M(new hr_mlp);
  M->owner = ctx;
  int rc = mlp_guard(M.get(), [&] {
    cudaStream_t st = ctx->c.stream;
    set_smem_attrs();
    // Glorot-uniform weights, zero biases; uniforms from splitmix64 of (seed, index)
    std::vector<float> p(kNP, 0.0f);
    auto fill = [&](int off, int fan_in, int fan_out) {
      const double lim = sqrt(6.0 / (double)(fan_in + fan_out));
      for (int k = 0; k < fan_in * fan_out; k++) {
        unsigned long long h = seed + 0x9e3779b97f4a7c15ULL * (unsigned long long)(off + k + 1);
        h = (h ^ (h >> 30)) * 0xbf58476d1ce4e5b9ULL;
        h = (h ^ (h >> 27)) * 0x94d049bb133111ebULL;
        h ^= h >> 31;
        const double u = (double)(h >> 11) / 9007199254740992.0;
        p[off + k] = (float)((2.0 * u - 1.0) * lim);
      }
    };
    fill(oW1, kIn, kH);
    fill(oW2, kH, kH);
    fill(oW3, kH, kH);
    fill(oW4, kH, kOut);
    M->params.upload(p, st);
    M->grad.alloc(kNP);
    M->m.alloc(kNP);
    M->v.alloc(kNP);
    M->m.zero(st);
    M->v.zero(st);
    M->loss.alloc(1);
    for (int i = 0; i < kIn; i++) {
      M->nm.mean[i] = 0.f;
      M->nm.inv_std[i] = 1.f;
    }
    M->nm.out_scale = 1.f;
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
  if (rc != HR_OK) return rc;
  *out = M.release();
  return HR_OK;
}

// Frees the network's device buffers (cudaFree waits for work using them);
// it does not touch the owning context, which may already be gone.
extern "C" void hr_mlp_destroy(hr_mlp* M) { delete M; }

extern "C" int hr_mlp_set_normalization(hr_mlp* M, const float* mean, const float* stdv, float out_scale) {
  if (!M || !mean || !stdv || !(out_scale > 0)) return HR_ERR_ARG;
  for (int i = 0; i < kIn; i++)
    if (!(stdv[i] > 0)) return HR_ERR_ARG;
  for (int i = 0; i < kIn; i++) {
    M->nm.mean[i] = mean[i];
    M->nm.inv_std[i] = 1.0f / stdv[i];
  }
  M->nm.out_scale = out_scale;
  return HR_OK;
}

extern "C" int hr_mlp_get_params(hr_mlp* M, float* host) {
  if (!M || !host) return HR_ERR_ARG;
  return mlp_guard(M, [&] {
    cudaStream_t st = M->owner->c.stream;
    HR_CHECK_CUDA(cudaMemcpyAsync(host, M->params.p, sizeof(float) * kNP, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
}

extern "C" int hr_mlp_set_params(hr_mlp* M, const float* host) {
  if (!M || !host) return HR_ERR_ARG;
  return mlp_guard(M, [&] {
    cudaStream_t st = M->owner->c.stream;
    HR_CHECK_CUDA(cudaMemcpyAsync(M->params.p, host, sizeof(float) * kNP, cudaMemcpyHostToDevice, st));
    M->m.zero(st);
    M->v.zero(st);
    M->step = 0;
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
}

extern "C" int hr_mlp_train_step(hr_mlp* M, const float* X_dev, const float* T_dev, long n, int batch,
                                 int random, unsigned long long seed, float lr, double* loss) {
  if (!M || !X_dev || !T_dev || n < 1 || batch < 1 || (!random && batch > n) || !(lr >= 0)) return HR_ERR_ARG;
  return mlp_guard(M, [&] {
    hr::Ctx& C = M->owner->c;
    cudaStream_t st = C.stream;
    set_smem_attrs();
    M->ensure(batch);
    const int nb = (batch + kThreads - 1) / kThreads;
    const int nchunks = (batch + kChunk - 1) / kChunk;
    const long step = M->step + 1;
    fwd_bwd_kernel<<<nb, kThreads, kFwdSmem, st>>>(M->params.p, M->nm, X_dev, T_dev, n, batch, seed, step, random,
                                                    M->idx.p, M->Zs.p, M->Ds.p, M->loss_part.p);
    grad_kernel<<<nchunks, kGradThreads, kGradSmem, st>>>(M->nm, X_dev, batch, M->idx.p, M->Zs.p, M->Ds.p, M->partial.p);
    grad_reduce_kernel<<<(kNP + 255) / 256, 256, 0, st>>>(M->partial.p, nchunks, M->grad.p);
    C.launches += 3;
    if (lr > 0) {
      M->step = step;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
      adam_kernel<<<(kNP + 255) / 256, 256, 0, st>>>(M->params.p, M->grad.p, M->m.p, M->v.p, lr, b1, b2, 1e-8f, c1,
                                                      c2);
      C.launches++;
    }
    HR_CHECK_CUDA(cudaGetLastError());
    if (loss) {
      sum_kernel<<<1, 1, 0, st>>>(M->loss_part.p, nb, M->loss.p);
      C.launches++;
      double l = 0;
      HR_CHECK_CUDA(cudaMemcpyAsync(&l, M->loss.p, sizeof(double), cudaMemcpyDeviceToHost, st));
      HR_CHECK_CUDA(cudaStreamSynchronize(st));
      *loss = l / (double)((long)batch * kOut);
    }
  });
}

extern "C" int hr_mlp_gradient(hr_mlp* M, const float* X_dev, const float* T_dev, int batch, float* grad_host,
                               double* loss) {
  if (!M || !grad_host) return HR_ERR_ARG;
  int rc = hr_mlp_train_step(M, X_dev, T_dev, batch, batch, 0, 0, 0.0f, loss);
  if (rc != HR_OK) return rc;
  return mlp_guard(M, [&] {
    cudaStream_t st = M->owner->c.stream;
    HR_CHECK_CUDA(cudaMemcpyAsync(grad_host, M->grad.p, sizeof(float) * kNP, cudaMemcpyDeviceToHost, st));
    HR_CHECK_CUDA(cudaStreamSynchronize(st));
  });
}

static int infer(hr_mlp* M, const float* X_dev, long n, const double* base_dev, double* out_dev, float* raw_dev,
                 const Frames& fr) {
  if (!M || n < 0 || (n > 0 && !X_dev)) return HR_ERR_ARG;
  if (n == 0) return HR_OK;
  return mlp_guard(M, [&] {
    hr::Ctx& C = M->owner->c;
    set_smem_attrs();
    infer_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, kFwdSmem, C.stream>>>(
        M->params.p, M->nm, X_dev, n, base_dev, out_dev, raw_dev, fr);
    C.launches++;
    HR_CHECK_CUDA(cudaGetLastError());
  });
}

extern "C" int hr_mlp_infer(hr_mlp* M, const float* X_dev, long n, const double* base_dev, double* out_dev,
                            float* raw_dev) {
  Frames fr;
  memset(&fr, 0, sizeof(fr));
  return infer(M, X_dev, n, base_dev, out_dev, raw_dev, fr);
}

extern "C" int hr_mlp_infer_frames(hr_mlp* M, const float* X_dev, long n, const double* base_dev, double* out_dev,
                                   int nframes, const long* frame_start, const double* rot) {
  if (nframes < 0 || nframes > kMaxFrames || (nframes > 0 && (!frame_start || !rot))) return HR_ERR_ARG;
  Frames fr;
  memset(&fr, 0, sizeof(fr));
  fr.n = nframes;
  for (int f = 0; f <= nframes; f++) fr.start[f] = frame_start[f];
  for (int f = 0; f < nframes; f++) {
    if (fr.start[f + 1] < fr.start[f]) return HR_ERR_ARG;
    for (int k = 0; k < 9; k++) fr.R[f][k] = rot[9 * f + k];
  }
  return infer(M, X_dev, n, base_dev, out_dev, nullptr, fr);
}

// Weights file: "HRMLP001", layer widths (5 x int32), 12 input means, 12 input
// stds, out_scale, the 9347 parameters (FP32), FNV-1a 64 of everything before.
extern "C" int hr_mlp_save(hr_mlp* M, const char* path) {
  if (!M || !path) return HR_ERR_ARG;
  std::vector<float> p(kNP);
  int rc = hr_mlp_get_params(M, p.data());
  if (rc != HR_OK) return rc;
  std::vector<unsigned char> buf;
  auto put = [&](const void* d, size_t n) {
    const unsigned char* c = (const unsigned char*)d;
    buf.insert(buf.end(), c, c + n);
  };
  put("HRMLP001", 8);
  const int shape[5] = {kIn, kH, kH, kH, kOut};
  put(shape, sizeof(shape));
  float stdv[kIn];
  for (int i = 0; i < kIn; i++) stdv[i] = 1.0f / M->nm.inv_std[i];
  put(M->nm.mean, sizeof(float) * kIn);
  put(stdv, sizeof(float) * kIn);
  put(&M->nm.out_scale, 4);
  put(p.data(), sizeof(float) * kNP);
  const unsigned long long h = fnv1a(buf.data(), buf.size());
  put(&h, 8);
  FILE* f = fopen(path, "wb");
  if (!f) {
    M->owner->c.err = std::string("cannot open ") + path;
    return HR_ERR_ARG;
  }
  const size_t w = fwrite(buf.data(), 1, buf.size(), f);
  fclose(f);
  return w == buf.size() ? HR_OK : HR_ERR_ARG;
}

extern "C" int hr_mlp_load(hr_mlp* M, const char* path) {
  if (!M || !path) return HR_ERR_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) {
    M->owner->c.err = std::string("cannot open ") + path;
    return HR_ERR_ARG;
  }
  std::vector<unsigned char> buf;
  unsigned char tmp[4096];
  size_t r;
  while ((r = fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + r);
  fclose(f);
  const size_t need = 8 + 5 * 4 + 4 * (2 * kIn + 1) + 4 * (size_t)kNP + 8;
  const int shape[5] = {kIn, kH, kH, kH, kOut};
  unsigned long long h = 0;
  if (buf.size() == need) memcpy(&h, buf.data() + need - 8, 8);
  if (buf.size() != need || memcmp(buf.data(), "HRMLP001", 8) != 0 || memcmp(buf.data() + 8, shape, 20) != 0 ||
      h != fnv1a(buf.data(), need - 8)) {
    M->owner->c.err = std::string("not a 12-64-64-64-3 warm-start weights file (header, shape or checksum): ") + path;
    return HR_ERR_ARG;
  }
  float mean[kIn], stdv[kIn], sc;
  memcpy(mean, buf.data() + 28, 4 * kIn);
  memcpy(stdv, buf.data() + 28 + 4 * kIn, 4 * kIn);
  memcpy(&sc, buf.data() + 28 + 8 * kIn, 4);
  const int rc = hr_mlp_set_normalization(M, mean, stdv, sc);
  if (rc != HR_OK) return rc;
  std::vector<float> p(kNP);
  memcpy(p.data(), buf.data() + 32 + 8 * kIn, 4 * (size_t)kNP);
  return hr_mlp_set_params(M, p.data());
}
