/* Test infrastructure (oracle only): a minimal stand-in for the FFTW 2.1.5
 * complex-FFT header, so that the reference KIFMM sources compile here
 * without FFTW installed.  Only the names the reference uses are declared
 * (common/commoninc.hpp:42 includes "fftw.h"; fmm3d/matmgnt3d.cpp uses
 * fftw_complex with .re/.im fields at :345-347,422-432).
 *
 * The transforms themselves are written from the DFT definition in
 * fftw_shim.c; no FFTW source is used.  Never linked into the product. */
#ifndef KIFMM_ORACLE_FFTW_SHIM_H
#define KIFMM_ORACLE_FFTW_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_real;
typedef struct { fftw_real re, im; } fftw_complex;

/* FFTW2 sign convention: forward = exp(-2 pi i jk/n), backward = exp(+...). */
typedef enum { FFTW_FORWARD = -1, FFTW_BACKWARD = 1 } fftw_direction;

#define FFTW_ESTIMATE     (0)
#define FFTW_MEASURE      (1)
#define FFTW_OUT_OF_PLACE (0)
#define FFTW_IN_PLACE     (8)

#ifdef __cplusplus
}
#endif
#endif
