/* Test infrastructure (oracle only): the subset of the FFTW 2.1.5 real
 * multi-dimensional interface that the reference calls:
 *   rfftw3d_create_plan        fmm3d/matmgnt3d.cpp:58-59
 *   rfftw2d_create_plan        common/vecmatop.cpp:599-600 (linked, never run)
 *   rfftwnd_real_to_complex    fmm3d/matmgnt3d.cpp:239,324
 *   rfftwnd_complex_to_real    fmm3d/matmgnt3d.cpp:269
 *   rfftwnd_destroy_plan       fmm3d/matmgnt3d.cpp:35-36
 * Semantics follow FFTW2's documented conventions: row-major arrays, the
 * last dimension halved to n/2+1 complex outputs, unnormalised transforms,
 * and (howmany, stride, dist) addressing.  Implemented in fftw_shim.c. */
#ifndef KIFMM_ORACLE_RFFTW_SHIM_H
#define KIFMM_ORACLE_RFFTW_SHIM_H

#include "fftw.h"

#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_REAL_TO_COMPLEX FFTW_FORWARD
#define FFTW_COMPLEX_TO_REAL FFTW_BACKWARD

typedef struct rfftwnd_plan_s* rfftwnd_plan;

rfftwnd_plan rfftw2d_create_plan(int nx, int ny, fftw_direction dir, int flags);
rfftwnd_plan rfftw3d_create_plan(int nx, int ny, int nz, fftw_direction dir, int flags);
void rfftwnd_destroy_plan(rfftwnd_plan plan);
void rfftwnd_real_to_complex(rfftwnd_plan plan, int howmany,
                             fftw_real* in, int istride, int idist,
                             fftw_complex* out, int ostride, int odist);
void rfftwnd_complex_to_real(rfftwnd_plan plan, int howmany,
                             fftw_complex* in, int istride, int idist,
                             fftw_real* out, int ostride, int odist);

#ifdef __cplusplus
}
#endif
#endif
