/*
 * fftw3.h of the FFTW-API layer (libhighreg_fftw.so): the part of FFTW 3's
 * public interface that the reference's extend-to-grid driver calls
 * (highreg_stokes_extend_to_grid/main.cpp:6, 1423-1489), so that driver
 * compiles and links unmodified with its Poisson transforms on the B200.
 *
 * Names, the plan handle, the r2r kind and flag values and the signatures are
 * FFTW's (an interface that has to be alike for a drop-in: a caller compiled
 * against either header gets the same calls); the implementation is this
 * repository's (host/hr_fftw_shim.cpp over hr_dst1_* of libhighreg_b200.so).
 *
 * Supported: fftw_plan_r2r_3d with FFTW_RODFT00 on all three axes and
 * n0 = n1 = n2 = n with n + 1 even (other kinds or shapes return NULL, as
 * FFTW's planner does for a plan it cannot make); planner flags are accepted
 * and ignored. fftw_malloc returns page-locked host memory (fast copies to the
 * GPU), fftw_free releases it.
 */
#ifndef HR_FFTW_SHIM_FFTW3_H
#define HR_FFTW_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* the r2r kind is an int-sized enum; the layer implements RODFT00 (DST-I),
 * whose value is FFTW's, so that callers built against FFTW's header pass
 * the same number */
typedef enum hr_fftw_r2r_kind { FFTW_RODFT00 = 7 } fftw_r2r_kind;

/* planner flag used by the reference (accepted and ignored) */
#define FFTW_ESTIMATE (1U << 6)

typedef struct fftw_plan_s* fftw_plan;

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_r2r_3d(int n0, int n1, int n2, double* in, double* out, fftw_r2r_kind kind0,
                           fftw_r2r_kind kind1, fftw_r2r_kind kind2, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void fftw_cleanup(void);

#ifdef __cplusplus
}
#endif
#endif
