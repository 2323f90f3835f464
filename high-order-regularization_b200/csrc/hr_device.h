// hr_device.h — device task descriptors and kernel launchers (internal).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "hr_engine.h"

namespace hr {

// One boundary sum: a source surface (tree order SoA) evaluated at a target
// set (reference order). All pointers are device pointers.
// doubles per target in a work item's partial sums (3 velocity + 1 pressure)
constexpr int kPartComps = 4;

struct EvalTask {
  int kind;       // Kind
  int jump_mode;  // DL kinds: 0 = treecode convention, 1 = direct-sum convention
  int P1, Pf;     // treecode degree + 1 and (P+1)^3
  int C;          // FP64 moment values stored per proxy (6 SL, 10 DL)
  int nt;         // number of targets
  int mixed;      // 0 FP64; 1: pairs beyond 3 delta and proxies in FP32 (FP64 accumulation); 2: all pairs FP32
  int pad;
  double DEL;     // regularization length delta
  double scale;   // final factor of the sum (1/8pi, -6/8pi, ...)
  const double *sx, *sy, *sz, *snx, *sny, *snz, *sa;  // sources, tree order
  const double *qx, *qy, *qz;                         // density, tree order
  double ctr[3];                                      // source surface centre (FP32 frame origin)
  // FP32 copies for the mixed-precision far field: positions relative to ctr
  const float *fx, *fy, *fz, *fnx, *fny, *fnz, *fa, *fqx, *fqy, *fqz;
  const int *node_m0, *node_m1;                       // inclusive member ranges
  const double* tcheb;                                // 3*P1 per node
  const double* mom;                                  // Pf*C per node, proxy-major
  const float* momf;                                  // Pf*W32 per node (W32 = 12 DL, 8 SL)
  const int* tord;                                    // target order -> target index
  const double* txyz;                                 // 3nt targets
  const double* tb;                                   // nt signed distances
  const uint8_t* tnear;                               // nt regularized-branch flag
  const double* tf0;                                  // 3nt nearest force (SL off, E2G)
  const double *tx0, *tn0, *tg0;                      // 3nt nearest point, normal, density
  const double *tq, *tnrm;                            // 3nt own density and normal (on-surface)
  double* out;                                        // 3nt (or nt for pressure)
  double* out2;                                       // nt pressure of K_E2G_UP_AWAY (scaled by scale2)
  double scale2;
  const Entry* entries;                               // interaction entries
  const int* blk_start;                               // per target block, into entries
  unsigned long long* counters;  // [0] regularized pairs [1] near-target plain [2] far-target [3] proxy
  const int* item_start;  // per target block: its work items' partial slots [start, end)
  double* partial;        // 3 x 128 doubles per work item
};

// A piece of one entry: a near entry's source sub-range [s0, s1), or a whole
// far entry (proxy points).
struct Seg {
  int entry;
  int s0, s1;
};

// One CTA's work: a run of consecutive segments of one target block. Each
// item writes its partial sums into its own slot; the reduce kernel adds the
// slots of a block in order, so results do not depend on scheduling.
struct BlockRef {
  int task;
  int blk;
  int seg0, seg1;
  int slot;
};

enum Family : int { F_SL = 0, F_DL = 1, F_E2G = 2 };

// Evaluates every work item of a combined list — the first n_on items (lean:
// on-surface tasks, or the extend-to-grid box-face sums) in one launch on st,
// the rest in another on `side` (forked from and joined back to st with the
// two events; on st as well when side is null) — then reduces the partial sums
// per target (deterministic order) and applies the epilogue. With count, the
// FP64 launches also add their per-branch pair counts to the tasks' counters.
void launch_eval(int family, const EvalTask* d_tasks, const BlockRef* d_items, const Seg* d_segs,
                 int nitems, int n_on, int ntask_blocks, const int2* d_task_blocks, cudaStream_t st,
                 cudaStream_t side, cudaEvent_t fork, cudaEvent_t join, bool mixed, bool count);

// Upward pass: proxy moments of every non-root node of a tree.
struct MomItem {
  int node;
  int s0;  // first source (tree order)
  int s1;  // one past last source
  int out; // partial slot
};
// Poisson extension (solve_Poisson, E2G/main.cpp:969-1044) with a reusable
// work area (FFT plan, tables, grid buffers) for one grid size N.
struct PoissonWork;
PoissonWork* poisson_work_create(struct Ctx& C, int N);
void poisson_work_destroy(PoissonWork* w);
void solve_poisson_dev(struct Ctx& C, int N, double L, const uint8_t* band2_dev, const uint8_t* out_dev,
                       const double* p_dev, double* u_dev, int variable, PoissonWork* work = nullptr);

// Tensor-core (tcgen05, 3xTF32) upward pass for the reduced-precision operator:
// same items and partial layout as launch_moments; a timed-out wait sets *err.
bool moments_tc_supported(int P1);
size_t moments_tc_smem(int dl, int P1, int* npad, int* cols);
void launch_moments_tc(int dl, const MomItem* d_items, int nitems, int P1, const double* tcheb, const double* x,
                       const double* y, const double* z, const double* nx, const double* ny, const double* nz,
                       const double* a, const double* qx, const double* qy, const double* qz, double* partial,
                       int* err, cudaStream_t st);
void launch_moments(int dl, const MomItem* d_items, int nitems, int P1, const double* tcheb,
                    const double* x, const double* y, const double* z, const double* nx,
                    const double* ny, const double* nz, const double* a, const double* qx,
                    const double* qy, const double* qz, double* partial, cudaStream_t st);
void launch_moments_reduce(int C, int Pf, int nnodes_out, const int* d_item_start,
                           const double* partial, double* mom, float* momf, cudaStream_t st);

// Gathers interleaved reference-order density into tree-order SoA.
void launch_permute(int n, const int* perm, const double* q3, double* qx, double* qy, double* qz,
                    float* fqx, float* fqy, float* fqz, cudaStream_t st);
void launch_permute_soa(int n, const int* perm, const double* src, double* dst, cudaStream_t st);

// Six-point density interpolation at nearest points.
void launch_interp(int ne, const int* tgt, const int* idx, const double* pq, const double* g,
                   double* g0, cudaStream_t st);

// Two-surface combine steps.
void launch_matvec_combine(int n, double factor, const double* x, const double* on,
                           const double* comp, double* y, cudaStream_t st);
void launch_rhs_combine(int n, double factor, const double* on, const double* comp, double* b,
                        cudaStream_t st);

// Vector kernels for GMRES (deterministic reductions).
constexpr int kRedBlocks = 296;
void launch_dots(int n, int ncols, const double* V, long ldv, const double* w, double* partial,
                 cudaStream_t st);
void launch_dots_finalize(int ncols, const double* partial, double* out, cudaStream_t st);
void launch_axpy_multi(int n, int ncols, const double* V, long ldv, const double* coef,
                       double sign, double* w, cudaStream_t st);
void launch_scale(int n, const double* s_dev, double* w, cudaStream_t st);
void launch_scale_host(int n, double s, double* w, cudaStream_t st);
void launch_sub(int n, const double* a, const double* b, double* out, cudaStream_t st);
void launch_copy(int n, const double* a, double* out, cudaStream_t st);

// FP64 FMA peak loop.
void launch_fma_peak(double* out, int iters, int blocks, cudaStream_t st);
void launch_fma_peak32(float* out, int iters, int blocks, cudaStream_t st);

}  // namespace hr
