/*
 * Test-only stand-in for the small part of the FFTW3 API that the reference's
 * extend-to-grid driver uses (highreg_stokes_extend_to_grid/main.cpp:1423-1489):
 * fftw_malloc, fftw_plan_r2r_3d with FFTW_RODFT00 on all three axes,
 * fftw_execute, fftw_destroy_plan, fftw_cleanup.
 *
 * FFTW itself is a third-party dependency that the reference does not vendor
 * (its makefile links -lfftw3 with no pinned version) and it is not installed
 * here. This header implements the published definition of FFTW's RODFT00
 * (DST-I, unnormalised):  Y_k = 2 * sum_{j=0}^{n-1} X_j sin(pi (j+1)(k+1) / (n+1)),
 * applied separably along the three axes of a row-major n*n*n array, by dense
 * sine-matrix products (O(n^4) work: fine for the oracle sizes, n <= 95).
 *
 * It is part of the oracle (test infrastructure) and is never linked into the
 * product library.
 */
#ifndef HR_FFTW_STANDIN_H
#define HR_FFTW_STANDIN_H

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#define FFTW_RODFT00 7
#define FFTW_ESTIMATE (1U << 6)

typedef int fftw_r2r_kind;

struct hr_standin_plan {
  int n0, n1, n2;
  double* in;
  double* out;
};
typedef hr_standin_plan* fftw_plan;

static inline void* fftw_malloc(size_t bytes) { return std::malloc(bytes); }
static inline void fftw_free(void* p) { std::free(p); }

static inline fftw_plan fftw_plan_r2r_3d(int n0, int n1, int n2, double* in, double* out,
                                         fftw_r2r_kind, fftw_r2r_kind, fftw_r2r_kind,
                                         unsigned) {
  fftw_plan p = new hr_standin_plan;
  p->n0 = n0; p->n1 = n1; p->n2 = n2; p->in = in; p->out = out;
  return p;
}

/* one DST-I along an axis with the given element stride, over all lines */
static inline void hr_standin_dst_axis(double* a, int n, int n_lines_outer, int n_lines_inner,
                                       long stride_axis, long stride_outer, long stride_inner) {
  std::vector<double> S((size_t)n * n);
  for (int k = 0; k < n; k++)
    for (int j = 0; j < n; j++)
      S[(size_t)k * n + j] = 2.0 * std::sin(M_PI * (double)((long)(j + 1) * (k + 1)) / (double)(n + 1));
#pragma omp parallel
  {
    std::vector<double> line(n), res(n);
#pragma omp for collapse(2)
    for (int o = 0; o < n_lines_outer; o++) {
      for (int in_ = 0; in_ < n_lines_inner; in_++) {
        double* base = a + (long)o * stride_outer + (long)in_ * stride_inner;
        for (int j = 0; j < n; j++) line[j] = base[(long)j * stride_axis];
        for (int k = 0; k < n; k++) {
          double s = 0.0;
          const double* row = &S[(size_t)k * n];
          for (int j = 0; j < n; j++) s += row[j] * line[j];
          res[k] = s;
        }
        for (int k = 0; k < n; k++) base[(long)k * stride_axis] = res[k];
      }
    }
  }
}

static inline void fftw_execute(const fftw_plan p) {
  const int n0 = p->n0, n1 = p->n1, n2 = p->n2;
  const size_t total = (size_t)n0 * n1 * n2;
  if (p->out != p->in) std::memcpy(p->out, p->in, total * sizeof(double));
  double* a = p->out;
  /* axis 2 (contiguous), axis 1, axis 0 of the row-major [n0][n1][n2] array */
  hr_standin_dst_axis(a, n2, n0, n1, 1, (long)n1 * n2, n2);
  hr_standin_dst_axis(a, n1, n0, n2, n2, (long)n1 * n2, 1);
  hr_standin_dst_axis(a, n0, n1, n2, (long)n1 * n2, n2, 1);
}

static inline void fftw_destroy_plan(fftw_plan p) { delete p; }
static inline void fftw_cleanup(void) {}

#endif
