// hr_fftw_shim.cpp — libhighreg_fftw.so: FFTW 3's r2r interface, as far as
// the reference's extend-to-grid Poisson solve uses it
// (fftw_DST_Poisson3d_FD, E2G/main.cpp:1423-1489), on the B200 through the
// C ABI's 3D DST-I plans (hr_dst1_*, the fused dst_pass_kernel).
//
// A relinked reference driver calls, per Poisson solve: fftw_malloc x2,
// fftw_plan_r2r_3d x2 (forward in place, backward out of place), fftw_execute
// x2 with its eigenvalue divide between them on the host, fftw_destroy_plan x2,
// fftw_cleanup. Each fftw_plan holds one device plan (tables and two n^3
// device buffers); all plans share one library context on device
// $HR_FFTW_DEVICE (default 0), created with the first plan. Each
// fftw_execute reads the plan's input array and writes its output array (host
// memory, in == out allowed) synchronously. fftw_cleanup releases the context
// once no plan is left. Errors are reported on stderr and leave the output
// array untouched; plan creation fails (NULL) for shapes or kinds other than
// n^3 RODFT00 with n + 1 even.
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <set>

#include "fftw_shim/fftw3.h"
#include "highreg_b200.h"

struct fftw_plan_s {
  int n = 0;
  double* in = nullptr;
  double* out = nullptr;
  hr_dst1_plan* p = nullptr;
};

namespace {

std::mutex g_mu;
hr_ctx* g_ctx = nullptr;
int g_plans = 0;
std::set<void*> g_pinned;

hr_ctx* shared_ctx() {
  if (!g_ctx) {
    const char* d = std::getenv("HR_FFTW_DEVICE");
    const int dev = d ? std::atoi(d) : 0;
    if (hr_ctx_create(dev, &g_ctx) != HR_OK) {
      std::fprintf(stderr, "fftw (B200 layer): no context on device %d\n", dev);
      g_ctx = nullptr;
    }
  }
  return g_ctx;
}

}  // namespace

extern "C" {

void* fftw_malloc(size_t n) {
  void* p = nullptr;
  if (hr_host_alloc(n ? n : 1, &p) == HR_OK) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_pinned.insert(p);
    return p;
  }
  // page-locked memory unavailable: plain aligned memory
  if (posix_memalign(&p, 64, n ? n : 1) != 0) return nullptr;
  return p;
}

void fftw_free(void* p) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_pinned.find(p);
    if (it != g_pinned.end()) {
      g_pinned.erase(it);
      hr_host_free(p);
      return;
    }
  }
  std::free(p);
}

fftw_plan fftw_plan_r2r_3d(int n0, int n1, int n2, double* in, double* out, fftw_r2r_kind kind0,
                           fftw_r2r_kind kind1, fftw_r2r_kind kind2, unsigned flags) {
  (void)flags;
  if (n0 < 1 || n0 != n1 || n0 != n2 || kind0 != FFTW_RODFT00 || kind1 != FFTW_RODFT00 ||
      kind2 != FFTW_RODFT00 || (n0 + 1) % 2 != 0 || !in || !out) {
    std::fprintf(stderr, "fftw (B200 layer): only n^3 RODFT00 plans with n + 1 even are supported\n");
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  hr_ctx* ctx = shared_ctx();
  if (!ctx) return nullptr;
  fftw_plan P = new fftw_plan_s;
  P->n = n0;
  P->in = in;
  P->out = out;
  if (hr_dst1_plan_create(ctx, n0, &P->p) != HR_OK) {
    std::fprintf(stderr, "fftw (B200 layer): %s\n", hr_last_error(ctx));
    delete P;
    return nullptr;
  }
  g_plans++;
  return P;
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  if (hr_dst1_execute(p->p, p->in, p->out) != HR_OK) {
    std::lock_guard<std::mutex> lock(g_mu);
    std::fprintf(stderr, "fftw (B200 layer): execute failed: %s\n", g_ctx ? hr_last_error(g_ctx) : "");
  }
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  hr_dst1_plan_destroy(p->p);
  delete p;
  std::lock_guard<std::mutex> lock(g_mu);
  g_plans--;
}

void fftw_cleanup(void) {
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_ctx && g_plans == 0) {
    hr_ctx_destroy(g_ctx);
    g_ctx = nullptr;
  }
}

}  // extern "C"
