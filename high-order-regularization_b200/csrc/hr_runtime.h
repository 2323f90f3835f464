// hr_runtime.h — context, device buffers and the device-resident objects the
// C ABI is built from (internal).
#pragma once
#include <cuda_runtime.h>

#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/highreg_b200.h"
#include "hr_device.h"
#include "hr_engine.h"

namespace hr {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define HR_CHECK_CUDA(call)                                                                  \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      throw ::hr::Error(HR_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));    \
  } while (0)

#define HR_REQUIRE(cond, msg)                                   \
  do {                                                          \
    if (!(cond)) throw ::hr::Error(HR_ERR_ARG, std::string(msg)); \
  } while (0)

// The library's device buffers come from one stream-ordered memory pool per
// device that keeps freed blocks mapped (up to a few GiB), so building and
// destroying plans does not map and unmap pages for every buffer. dev_alloc
// returns memory that every stream may use at once; dev_free first waits for
// the pointer's device to go idle, as cudaFree does, and never throws.
void* dev_alloc(size_t bytes);
void dev_free(void* p) noexcept;

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0;
  DBuf() = default;
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), n(o.n) {
    o.p = nullptr;
    o.n = 0;
  }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      n = o.n;
      o.p = nullptr;
      o.n = 0;
    }
    return *this;
  }
  ~DBuf() { release(); }
  void release() {
    if (p) dev_free(p);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    p = static_cast<T*>(dev_alloc(count * sizeof(T)));
    n = count;
  }
  void upload(const T* h, size_t count, cudaStream_t st) {
    alloc(count);
    if (h && count) HR_CHECK_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st));
  }
  void upload(const std::vector<T>& v, cudaStream_t st) { upload(v.data(), v.size(), st); }
  void zero(cudaStream_t st) {
    if (p) HR_CHECK_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), st));
  }
};

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  // a second stream forked from and joined back to `stream` around the two
  // launches of a boundary-sum batch, so that each fills the other's tail
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  std::string err;
  long long launches = 0;
  int num_sms = 148;
  // while set, FP64 boundary-sum launches record their per-branch pair counts
  // (the tasks' work counters); other launches skip the tests
  bool count_work = false;
  DBuf<unsigned long long> counters;  // [0] reg pairs [1] plain pairs [2] proxies
  DBuf<int> tc_err;                   // set by a tensor-core kernel whose bounded wait ran out
  // two pinned host buffers of kPinChunk bytes for staged reads (d2h_staged),
  // allocated on first use, and the events that mark each one filled
  void* pin = nullptr;
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  // throws if a tensor-core kernel of this context reported a timed-out wait
  void check_tc();
};

// Bytes of one pinned staging buffer of d2h_staged.
constexpr size_t kPinChunk = size_t(16) << 20;

// Reads `bytes` from device memory into (pageable) host memory through the
// context's two pinned buffers: the copy of chunk k + 1 runs while host threads
// move chunk k into place. Returns when all of it has arrived. Reads of up to
// two chunks go straight to `dst`.
void d2h_staged(Ctx& C, void* dst, const void* src, size_t bytes);

// A surface on the device: sources in tree order, its tree, density buffers
// and the upward-pass work items.
struct DevTree {
  Tree host;
  int n = 0, nn = 0, P1 = 0, Pf = 0;
  DBuf<double> x, y, z, nx, ny, nz, a;
  DBuf<int> perm, m0, m1;
  DBuf<double> tcheb;
  DBuf<double> qx, qy, qz;
  DBuf<float> fx, fy, fz, fnx, fny, fnz, fa, fqx, fqy, fqz;  // FP32 copies, centre-relative
  double ctr[3] = {0, 0, 0};
  DBuf<double> mom;  // nn * Pf * C, proxy-major (C = 10 DL symmetric form, 6 SL)
  DBuf<float> momf;  // nn * Pf * W32 FP32 copy (W32 = 12 DL, 8 SL)
  DBuf<MomItem> items;
  DBuf<int> item_start;
  DBuf<double> partial;
  int nitems = 0;
  long long moment_terms = 0;  // sum over non-root nodes of Pf * members
  void build(const hr_surface& S, int P, int N0, double theta, bool direct, cudaStream_t st);
  // density (reference order, interleaved, device) -> tree-order SoA (+ moments)
  // tc: the upward pass on the tensor cores (reduced-precision operator)
  void set_density(Ctx& C, const double* q3_dev, bool dl, bool moments, bool tc = false);
};

// Target data on the device, reference order.
struct DevTargets {
  int n = 0;
  DBuf<double> xyz, b, x0, n0, f0, g0;
  DBuf<uint8_t> near;
  DBuf<double> nrm;  // own normals for on-surface targets
};

struct DevLists {
  Lists host;
  DBuf<int> tord, blk_start;
  DBuf<Entry> entries;
  void build(const Tree& T, int nt, const double* txyz, const uint8_t* near, cudaStream_t st,
             const std::vector<int>* morton = nullptr);
};

struct DevStencils {
  int ne = 0;
  DBuf<int> tgt, idx;
  DBuf<double> pq;
  void build(const Stencils& S, cudaStream_t st);
};

// A batch of boundary sums evaluated together (one or two kernel launches and
// one reduction).
struct Batch {
  int family = F_SL;
  std::vector<EvalTask> tasks;
  std::vector<const Lists*> lists;
  std::vector<const Tree*> trees;  // source tree of each task (member ranges of near entries)
  DBuf<EvalTask> d_tasks;
  DBuf<BlockRef> d_items;
  DBuf<Seg> d_segs;
  DBuf<int> d_item_start;
  DBuf<int2> d_task_blocks;
  DBuf<double> d_partial;
  int nitems = 0, ntask_blocks = 0;
  int n_on = 0;  // leading lean items (on-surface / box-face tasks, launched on their own)
  bool ready = false;  // finalize has run
  // builds the segments and cost-balanced work items of all tasks
  void finalize(cudaStream_t st, int num_sms = 148);
  void launch(Ctx& C);
};

EvalTask make_task(int kind, double DEL, double scale, const DevTree& T, const DevLists& L,
                   const DevTargets& tg, double* out);

}  // namespace hr

// The C ABI's opaque context.
struct hr_ctx {
  hr::Ctx c;
};
