// hr_moments_tc.cu — the treecode's upward pass on the 5th-generation tensor
// cores (tcgen05, kind::tf32) for the reduced-precision operator.
//
// The proxy charges of a node (Panel_Moments_SL / _DL, 2S/KITC.cpp:351-668),
//   M[c][(i,j,k)] = sum_s L_i(x_s) L_j(y_s) L_k(z_s) a_s q_c(s),
// are the GEMM
//   D[(j,k), (c,i)] = sum_s A[(j,k), s] B[(c,i), s],
//   A[(j,k), s] = L_j(y_s) L_k(z_s),   B[(c,i), s] = L_i(x_s) a_s q_c(s),
// with M = (P+1)^2 <= 128 rows (padded to 128), N = C (P+1) columns (padded to
// a multiple of 16) and K = the node's sources. One CTA of 128 threads per
// work item (a node and up to 512 of its sources):
//   * threads 0..95 evaluate the barycentric Lagrange values of a tile of 32
//     sources, one (axis, source) each (offsets in FP64 for the reference's
//     removable-singularity rule, quotients in FP32), threads 96..127 the
//     channel values a_s q_c(s);
//   * all threads form the A and B tiles in shared memory, K-major, in the
//     no-swizzle canonical layout (8-row x 16-byte core matrices; K-chunk
//     stride 128 B, 8-row-group stride 1024 B), each value split into TF32
//     hi = tf32(v) and lo = tf32(v - hi);
//   * one thread issues, per K-step of 8, the three tcgen05.mma of the split
//     product A_hi B_hi + A_hi B_lo + A_lo B_hi into an FP32 accumulator in
//     tensor memory, and commits them to an mbarrier; the next tile's Lagrange
//     values are computed while they run;
//   * each warp reads its 32 accumulator rows (tcgen05.ld 32x32b) and writes
//     the item's partial moments as FP64 in the layout of the FP64 upward
//     pass, whose in-order reduction follows.
// 3xTF32 keeps ~FP32 accuracy (the dropped lo x lo term is ~2^-22 relative);
// the moments feed only the FP32 far field of the reduced-precision operator.
//
// Every wait on the mbarrier is bounded: past the limit the kernel sets the
// error flag, waits (bounded) once more for its own MMAs, frees its tensor
// memory and returns.
#include <cuda_runtime.h>

#include <cstdint>

#include "hr_device.h"

namespace hr {

namespace {

constexpr int kTcThreads = 128;
constexpr int kTcK = 32;          // sources per K tile
static_assert(kTcThreads == 4 * kTcK, "three warps of Lagrange values and one of channel values per tile");
constexpr int kTcMaxP1 = 11;      // (P+1)^2 <= 128
constexpr long kWaitLimit = 1L << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_rna(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// Shared-memory matrix descriptor, K-major, no swizzle: start address, leading
// byte offset (between the two 16-byte K chunks of one instruction), stride
// byte offset (between 8-row groups), descriptor version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred P1;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
      "selp.b32 %0, 1, 0, P1;\n\t}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for completion phase `parity`; false if the limit was hit.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  for (long it = 0; it < kWaitLimit; it++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

struct TcShape {
  int P1, C, M2;   // M2 = P1^2 rows used
  int Npad, cols;  // padded N, allocated TMEM columns
};

template <bool DL>
__global__ void __launch_bounds__(kTcThreads) moments_tc_kernel(
    const MomItem* __restrict__ items, TcShape sh, const double* __restrict__ tcheb,
    const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
    const double* __restrict__ nx, const double* __restrict__ ny, const double* __restrict__ nz,
    const double* __restrict__ a, const double* __restrict__ qx, const double* __restrict__ qy,
    const double* __restrict__ qz, double* __restrict__ partial, int* __restrict__ err) {
  constexpr int C = DL ? 12 : 6;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int P1 = sh.P1, M2 = sh.M2, Npad = sh.Npad, Pf = P1 * P1 * P1;
  float* Ahi = reinterpret_cast<float*>(smem);
  float* Alo = Ahi + 128 * kTcK;
  float* Bhi = Alo + 128 * kTcK;
  float* Blo = Bhi + Npad * kTcK;
  float* sL = Blo + Npad * kTcK;       // [3][kTcMaxP1][kTcK] normalized Lagrange values
  float* sAQ = sL + 3 * kTcMaxP1 * kTcK;  // [C][kTcK] a_s q_c(s)
  double* sT = reinterpret_cast<double*>(sAQ + 12 * kTcK);  // Chebyshev points, 3 P1
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sT + 3 * kTcMaxP1 + 1);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 1);
  int* sflag = reinterpret_cast<int*>(tslot + 1);

  const MomItem it = items[blockIdx.x];
  const int ntile = (it.s1 - it.s0 + kTcK - 1) / kTcK;
  if (ntile <= 0) {  // no sources: zero moments
    for (int e = tid; e < C * Pf; e += kTcThreads) partial[(size_t)it.out * C * Pf + e] = 0.0;
    return;
  }
  if (tid < 3 * P1) sT[tid] = tcheb[(size_t)it.node * 3 * P1 + tid];
  // zero the operand tiles once: padding rows and columns stay zero
  for (int e = tid; e < (2 * 128 + 2 * Npad) * kTcK; e += kTcThreads) Ahi[e] = 0.f;
  if (tid == 0) {
    *sflag = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1u) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"((uint32_t)sh.cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t bar = smem_u32(mbar);
  // instruction descriptor: D FP32, A and B TF32, both K-major, N, M = 128
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(Npad >> 3) << 17) | ((128u >> 4) << 24);
  bool ok = true;

  for (int kt = 0; kt < ntile && ok; kt++) {
    const int s0 = it.s0 + kt * kTcK;
    // Lagrange values of this tile's sources (overlaps the previous tile's MMAs):
    // threads 0..95 one (axis, source) each — the offset from each Chebyshev
    // point in FP64 (for the reference's removable-singularity test), the
    // barycentric quotients in FP32, which is all the TF32 split keeps —
    // and threads 96..127 the channel values a_s q_c(s) of one source each
    if (tid < 3 * kTcK) {
      const int ax = tid / kTcK, src = tid - ax * kTcK;
      const int s = s0 + src;
      const bool valid = s < it.s1;
      const double pc = valid ? (ax == 0 ? x[s] : (ax == 1 ? y[s] : z[s])) : 0.0;
      float L[kTcMaxP1];
      int flag = -1;
      float S = 0.f;
      for (int jj = 0; jj < P1; jj++) {
        // w_j = (-1)^j d_j, d_0 = d_P = 1/2 (2S/KITC.cpp:365-375)
        const float w = ((jj % 2 == 0) ? 1.f : -1.f) * ((jj == 0 || jj == P1 - 1) ? 0.5f : 1.f);
        const double d = pc - sT[ax * P1 + jj];
        if (fabs(d) < 1.e-07) {
          flag = jj;
          L[jj] = 0.f;
        } else {
          L[jj] = w / (float)d;
          S += L[jj];
        }
      }
      const float inv = 1.f / S;
      for (int jj = 0; jj < P1; jj++) {
        const float v = (flag > -1) ? (jj == flag ? 1.f : 0.f) : L[jj] * inv;
        sL[(ax * kTcMaxP1 + jj) * kTcK + src] = valid ? v : 0.f;
      }
    } else {
      const int src = tid - 3 * kTcK;
      const int s = s0 + src;
      const bool valid = s < it.s1;
      const double as = valid ? a[s] : 0.0;
      const double n3[3] = {valid ? nx[s] : 0.0, valid ? ny[s] : 0.0, valid ? nz[s] : 0.0};
      const double q3[3] = {valid ? qx[s] : 0.0, valid ? qy[s] : 0.0, valid ? qz[s] : 0.0};
      if (DL) {
        for (int l = 0; l < 3; l++)
          for (int m = 0; m < 3; m++) sAQ[(3 * l + m) * kTcK + src] = (float)(as * q3[l] * n3[m]);
        for (int m = 0; m < 3; m++) sAQ[(9 + m) * kTcK + src] = (float)(as * n3[m]);
      } else {
        for (int m = 0; m < 3; m++) {
          sAQ[m * kTcK + src] = (float)(as * q3[m]);
          sAQ[(3 + m) * kTcK + src] = (float)(as * n3[m]);
        }
      }
    }
    // the previous tile's MMAs must be done reading the operand tiles; the
    // outcome is made uniform across the CTA before anyone acts on it
    bool mine = true;
    if (kt > 0) mine = mbar_wait(bar, (uint32_t)((kt - 1) & 1));
    ok = __syncthreads_and(mine) != 0;
    if (!ok) {
      if (tid == 0) atomicExch(err, 1);
      break;
    }
    // operand tiles: thread -> (row r0 of a core matrix, K chunk kc)
    {
      const int r0 = tid & 7, kc = (tid >> 3) & 7, g0 = tid >> 6;
      for (int rg = g0; rg < 16; rg += 2) {
        const int m = rg * 8 + r0;
        if (m >= M2) continue;
        const int j = m / P1, k = m - j * P1;
        float h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int sc = kc * 4 + e;
          const float v = sL[(1 * kTcMaxP1 + j) * kTcK + sc] * sL[(2 * kTcMaxP1 + k) * kTcK + sc];
          h[e] = tf32_rna(v);
          l[e] = tf32_rna(v - h[e]);
        }
        const int off = (rg * 8 + kc) * 32 + r0 * 4;
        *reinterpret_cast<float4*>(Ahi + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(Alo + off) = make_float4(l[0], l[1], l[2], l[3]);
      }
      const int NG = Npad / 8, CN = C * P1;
      for (int rg = g0; rg < NG; rg += 2) {
        const int n = rg * 8 + r0;
        if (n >= CN) continue;
        const int c = n / P1, i = n - c * P1;
        float h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; e++) {
          const int sc = kc * 4 + e;
          const float v = sL[(0 * kTcMaxP1 + i) * kTcK + sc] * sAQ[c * kTcK + sc];
          h[e] = tf32_rna(v);
          l[e] = tf32_rna(v - h[e]);
        }
        const int off = (rg * 8 + kc) * 32 + r0 * 4;
        *reinterpret_cast<float4*>(Bhi + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(Blo + off) = make_float4(l[0], l[1], l[2], l[3]);
      }
    }
    // generic-proxy writes -> visible to the tensor core's async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t aH = smem_u32(Ahi), aL = smem_u32(Alo), bH = smem_u32(Bhi), bL = smem_u32(Blo);
#pragma unroll
      for (int ks = 0; ks < kTcK / 8; ks++) {
        const uint32_t o = ks * 2 * 128;  // two 16-byte K chunks per K-step of 8
        const uint64_t dAh = make_desc(aH + o, 128, 1024), dAl = make_desc(aL + o, 128, 1024);
        const uint64_t dBh = make_desc(bH + o, 128, 1024), dBl = make_desc(bL + o, 128, 1024);
        mma_tf32(tmem, dAh, dBh, idesc, (kt > 0 || ks > 0) ? 1u : 0u);
        mma_tf32(tmem, dAh, dBl, idesc, 1u);
        mma_tf32(tmem, dAl, dBh, idesc, 1u);
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                   : "memory");
    }
  }
  // the last commit: accumulator complete (uniform outcome, as above)
  const int last = ntile - 1;
  if (ok) {
    ok = __syncthreads_and(mbar_wait(bar, (uint32_t)(last & 1))) != 0;
    if (!ok && tid == 0) atomicExch(err, 1);
  }
  if (!ok) {
    // a wait ran out: give the MMAs in flight one more bounded chance before freeing
    mbar_wait(bar, (uint32_t)(last & 1));
  } else {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int m = warp * 32 + lane;  // accumulator row of this thread
    const int CN = C * P1;
    for (int col0 = 0; col0 < Npad; col0 += 16) {
      uint32_t v[16];
      const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, "
          "%13, %14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
            "=r"(v[15])
          : "r"(ta));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < M2) {
#pragma unroll
        for (int q = 0; q < 16; q++) {
          const int n = col0 + q;
          if (n < CN) {
            const int c = n / P1, i = n - c * P1;
            partial[((size_t)it.out * C + c) * Pf + (size_t)i * M2 + m] = (double)__uint_as_float(v[q]);
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)sh.cols)
                 : "memory");
  }
}

}  // namespace

bool moments_tc_supported(int P1) { return P1 >= 2 && P1 <= kTcMaxP1; }

size_t moments_tc_smem(int dl, int P1, int* npad, int* cols) {
  const int C = dl ? 12 : 6;
  const int N = C * P1;
  const int Np = (N + 15) / 16 * 16;
  int c = 32;
  while (c < Np) c *= 2;
  size_t need = sizeof(float) * ((size_t)(2 * 128 + 2 * Np) * kTcK + 3 * kTcMaxP1 * kTcK + 12 * kTcK) +
                sizeof(double) * (3 * kTcMaxP1 + 1) + 64;
  // at most 512 / cols resident CTAs per SM, so every allocation of tensor
  // memory succeeds at once: ask for enough shared memory to cap occupancy
  const size_t sm_total = 233472;  // shared memory per SM
  const size_t cap = sm_total * (size_t)c / 512;
  if (need < cap) need = cap;
  need = (need + 1023) / 1024 * 1024;
  if (npad) *npad = Np;
  if (cols) *cols = c;
  return need;
}

void launch_moments_tc(int dl, const MomItem* d_items, int nitems, int P1, const double* tcheb, const double* x,
                       const double* y, const double* z, const double* nx, const double* ny, const double* nz,
                       const double* a, const double* qx, const double* qy, const double* qz, double* partial,
                       int* err, cudaStream_t st) {
  if (nitems <= 0) return;
  TcShape sh;
  sh.P1 = P1;
  sh.C = dl ? 12 : 6;
  sh.M2 = P1 * P1;
  const size_t smem = moments_tc_smem(dl, P1, &sh.Npad, &sh.cols);
  if (dl) {
    cudaFuncSetAttribute(moments_tc_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    moments_tc_kernel<true><<<nitems, kTcThreads, smem, st>>>(d_items, sh, tcheb, x, y, z, nx, ny, nz, a, qx, qy,
                                                              qz, partial, err);
  } else {
    cudaFuncSetAttribute(moments_tc_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    moments_tc_kernel<false><<<nitems, kTcThreads, smem, st>>>(d_items, sh, tcheb, x, y, z, nx, ny, nz, a, qx, qy,
                                                               qz, partial, err);
  }
}

}  // namespace hr
