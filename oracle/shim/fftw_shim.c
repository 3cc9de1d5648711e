/* Test infrastructure (oracle only).  A small mixed-radix FFT behind the
 * FFTW 2.1.5 rfftwnd interface declared in rfftw.h, so the reference KIFMM
 * (which calls rfftwnd_* at fmm3d/matmgnt3d.cpp:58-59,239,269,324) builds
 * and runs as the CPU oracle and CPU baseline.  Written from the DFT
 * definition X[k] = sum_j x[j] exp(sign * 2 pi i jk / n):
 *   - complex 1-D transforms: recursive decimation in time, smallest prime
 *     factor first (radix 4 preferred, then 2, 3, 5, ..., generic DFT for
 *     any remaining prime), twiddles from one table per length;
 *   - real -> complex n-D: complex transform of each last-axis line with
 *     zero imaginary part, keep n/2+1 outputs, then complex transforms along
 *     the remaining axes;
 *   - complex -> real n-D: complex inverse transforms along the leading
 *     axes, then each last-axis line is completed by Hermitian symmetry and
 *     the real part of its inverse transform is kept (the imaginary parts of
 *     the self-conjugate entries are ignored, as FFTW2 does).
 * Unnormalised in both directions, like FFTW2.  Never linked into the
 * product library. */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "rfftw.h"

typedef struct {
  int n;
  int sign;      /* -1 forward, +1 backward */
  double* twr;   /* exp(sign*2*pi*i*j/n), j = 0..n-1 */
  double* twi;
} cplan1d;

struct rfftwnd_plan_s {
  int rank;
  int dims[3];
  int sign;
  cplan1d ax[3];       /* complex plans per axis (same sign) */
  double* work;        /* scratch: one full complex array */
  double* line;        /* scratch: 2 lines of max length, complex */
};

static void cplan_init(cplan1d* p, int n, int sign) {
  p->n = n;
  p->sign = sign;
  p->twr = (double*)malloc(sizeof(double) * (size_t)n);
  p->twi = (double*)malloc(sizeof(double) * (size_t)n);
  for (int j = 0; j < n; j++) {
    double a = 2.0 * M_PI * (double)j / (double)n;
    p->twr[j] = cos(a);
    p->twi[j] = (double)sign * sin(a);
  }
}

static void cplan_free(cplan1d* p) {
  free(p->twr);
  free(p->twi);
}

static int smallest_factor(int n) {
  if (n % 4 == 0) return 4;
  if (n % 2 == 0) return 2;
  for (int f = 3; f * f <= n; f += 2)
    if (n % f == 0) return f;
  return n;
}

/* Transform n points read from (xr,xi) at stride `s` into (outr,outi)
 * contiguous.  `tstep` = N_top / n so that the twiddle of this sub-length is
 * tw[j * tstep]. */
static void fft_rec(const cplan1d* p, int n, const double* xr, const double* xi, int s,
                    double* outr, double* outi, int tstep) {
  if (n == 1) {
    outr[0] = xr[0];
    outi[0] = xi[0];
    return;
  }
  int f = smallest_factor(n);
  int m = n / f;
  for (int r = 0; r < f; r++)
    fft_rec(p, m, xr + (size_t)r * s, xi + (size_t)r * s, s * f, outr + (size_t)r * m,
            outi + (size_t)r * m, tstep * f);
  /* butterflies: X[k1 + m*k2] = sum_r (w_n^{r k1} Y_r[k1]) w_f^{r k2} */
  double tr[64], ti[64];
  double* br = tr;
  double* bi = ti;
  double* heap = NULL;
  if (f > 64) {
    heap = (double*)malloc(sizeof(double) * 2 * (size_t)f);
    br = heap;
    bi = heap + f;
  }
  const int N = p->n;
  for (int k1 = 0; k1 < m; k1++) {
    for (int r = 0; r < f; r++) {
      double yr = outr[r * m + k1], yi = outi[r * m + k1];
      int t = (int)(((long)r * k1 * tstep) % N);
      double wr = p->twr[t], wi = p->twi[t];
      br[r] = yr * wr - yi * wi;
      bi[r] = yr * wi + yi * wr;
    }
    if (f == 2) {
      outr[k1] = br[0] + br[1];
      outi[k1] = bi[0] + bi[1];
      outr[k1 + m] = br[0] - br[1];
      outi[k1 + m] = bi[0] - bi[1];
    } else if (f == 4) {
      /* w_4 = exp(sign * i pi/2) = sign*i */
      double s0r = br[0] + br[2], s0i = bi[0] + bi[2];
      double d0r = br[0] - br[2], d0i = bi[0] - bi[2];
      double s1r = br[1] + br[3], s1i = bi[1] + bi[3];
      double d1r = br[1] - br[3], d1i = bi[1] - bi[3];
      double sg = (double)p->sign;
      /* (sign*i) * d1 = (-sign*d1i, sign*d1r) */
      double jd1r = -sg * d1i, jd1i = sg * d1r;
      outr[k1] = s0r + s1r;
      outi[k1] = s0i + s1i;
      outr[k1 + m] = d0r + jd1r;
      outi[k1 + m] = d0i + jd1i;
      outr[k1 + 2 * m] = s0r - s1r;
      outi[k1 + 2 * m] = s0i - s1i;
      outr[k1 + 3 * m] = d0r - jd1r;
      outi[k1 + 3 * m] = d0i - jd1i;
    } else {
      int ws = N / f; /* w_f = tw[ws] */
      for (int k2 = 0; k2 < f; k2++) {
        double ar = 0.0, ai = 0.0;
        for (int r = 0; r < f; r++) {
          int t = (int)(((long)r * k2 % f) * ws);
          double wr = p->twr[t], wi = p->twi[t];
          ar += br[r] * wr - bi[r] * wi;
          ai += br[r] * wi + bi[r] * wr;
        }
        outr[k1 + m * k2] = ar;
        outi[k1 + m * k2] = ai;
      }
    }
  }
  free(heap);
}

/* In-place complex transform of n points at (re,im) with stride s (elements
 * of interleaved complex array: re at 2*idx, im at 2*idx+1). */
static void cfft_strided(const cplan1d* p, double* a, int s, double* line) {
  int n = p->n;
  double* xr = line;
  double* xi = line + n;
  double* yr = line + 2 * n;
  double* yi = line + 3 * n;
  for (int j = 0; j < n; j++) {
    xr[j] = a[2 * (size_t)j * s];
    xi[j] = a[2 * (size_t)j * s + 1];
  }
  fft_rec(p, n, xr, xi, 1, yr, yi, 1);
  for (int j = 0; j < n; j++) {
    a[2 * (size_t)j * s] = yr[j];
    a[2 * (size_t)j * s + 1] = yi[j];
  }
}

static rfftwnd_plan make_plan(int rank, const int* dims, fftw_direction dir) {
  rfftwnd_plan p = (rfftwnd_plan)calloc(1, sizeof(*p));
  p->rank = rank;
  p->sign = (dir == FFTW_FORWARD) ? -1 : 1;
  int maxn = 1;
  size_t total = 1;
  for (int d = 0; d < rank; d++) {
    p->dims[d] = dims[d];
    cplan_init(&p->ax[d], dims[d], p->sign);
    if (dims[d] > maxn) maxn = dims[d];
    total *= (size_t)(d == rank - 1 ? dims[d] / 2 + 1 : dims[d]);
  }
  p->work = (double*)malloc(sizeof(double) * 2 * total);
  p->line = (double*)malloc(sizeof(double) * 4 * (size_t)maxn);
  return p;
}

rfftwnd_plan rfftw2d_create_plan(int nx, int ny, fftw_direction dir, int flags) {
  (void)flags;
  int d[2] = {nx, ny};
  return make_plan(2, d, dir);
}

rfftwnd_plan rfftw3d_create_plan(int nx, int ny, int nz, fftw_direction dir, int flags) {
  (void)flags;
  int d[3] = {nx, ny, nz};
  return make_plan(3, d, dir);
}

void rfftwnd_destroy_plan(rfftwnd_plan p) {
  if (!p) return;
  for (int d = 0; d < p->rank; d++) cplan_free(&p->ax[d]);
  free(p->work);
  free(p->line);
  free(p);
}

/* Transform the complex work array (dims[0..rank-2] full, last = nh) along
 * every axis except the last. */
static void leading_axes(rfftwnd_plan p, int nh) {
  int rank = p->rank;
  for (int ax = 0; ax < rank - 1; ax++) {
    int n = p->dims[ax];
    size_t inner = (size_t)nh;
    for (int d = ax + 1; d < rank - 1; d++) inner *= (size_t)p->dims[d];
    size_t outer = 1;
    for (int d = 0; d < ax; d++) outer *= (size_t)p->dims[d];
    for (size_t o = 0; o < outer; o++)
      for (size_t i = 0; i < inner; i++)
        cfft_strided(&p->ax[ax], p->work + 2 * (o * (size_t)n * inner + i), (int)inner, p->line);
  }
}

void rfftwnd_real_to_complex(rfftwnd_plan p, int howmany, fftw_real* in, int istride, int idist,
                             fftw_complex* out, int ostride, int odist) {
  int rank = p->rank;
  int nl = p->dims[rank - 1];
  int nh = nl / 2 + 1;
  size_t nlines = 1;
  for (int d = 0; d < rank - 1; d++) nlines *= (size_t)p->dims[d];
  const cplan1d* pl = &p->ax[rank - 1];
  double* xr = p->line;
  double* xi = p->line + nl;
  double* yr = p->line + 2 * nl;
  double* yi = p->line + 3 * nl;
  for (int h = 0; h < howmany; h++) {
    const double* src = in + (size_t)h * idist;
    for (size_t L = 0; L < nlines; L++) {
      for (int j = 0; j < nl; j++) {
        xr[j] = src[(L * nl + j) * (size_t)istride];
        xi[j] = 0.0;
      }
      fft_rec(pl, nl, xr, xi, 1, yr, yi, 1);
      for (int k = 0; k < nh; k++) {
        p->work[2 * (L * nh + k)] = yr[k];
        p->work[2 * (L * nh + k) + 1] = yi[k];
      }
    }
    leading_axes(p, nh);
    fftw_complex* dst = out + (size_t)h * odist;
    for (size_t e = 0; e < nlines * nh; e++) {
      dst[e * (size_t)ostride].re = p->work[2 * e];
      dst[e * (size_t)ostride].im = p->work[2 * e + 1];
    }
  }
}

void rfftwnd_complex_to_real(rfftwnd_plan p, int howmany, fftw_complex* in, int istride, int idist,
                             fftw_real* out, int ostride, int odist) {
  int rank = p->rank;
  int nl = p->dims[rank - 1];
  int nh = nl / 2 + 1;
  size_t nlines = 1;
  for (int d = 0; d < rank - 1; d++) nlines *= (size_t)p->dims[d];
  const cplan1d* pl = &p->ax[rank - 1];
  double* xr = p->line;
  double* xi = p->line + nl;
  double* yr = p->line + 2 * nl;
  double* yi = p->line + 3 * nl;
  for (int h = 0; h < howmany; h++) {
    const fftw_complex* src = in + (size_t)h * idist;
    for (size_t e = 0; e < nlines * nh; e++) {
      p->work[2 * e] = src[e * (size_t)istride].re;
      p->work[2 * e + 1] = src[e * (size_t)istride].im;
    }
    leading_axes(p, nh);
    double* dst = out + (size_t)h * odist;
    for (size_t L = 0; L < nlines; L++) {
      for (int k = 0; k < nh; k++) {
        xr[k] = p->work[2 * (L * nh + k)];
        xi[k] = p->work[2 * (L * nh + k) + 1];
      }
      for (int k = nh; k < nl; k++) {
        xr[k] = xr[nl - k];
        xi[k] = -xi[nl - k];
      }
      xi[0] = 0.0;
      if (nl % 2 == 0) xi[nl / 2] = 0.0;
      fft_rec(pl, nl, xr, xi, 1, yr, yi, 1);
      for (int j = 0; j < nl; j++) dst[(L * nl + j) * (size_t)ostride] = yr[j];
    }
  }
}
