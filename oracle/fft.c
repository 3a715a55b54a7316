/*
 * ORACLE (test infrastructure only).
 *
 * A small FFT used in place of FFTW3, which is absent from this image, when
 * the reference's C library is compiled for the oracle (shims/fftw3.h maps
 * the two FFTW calls the reference makes, src/wavemoth.c:828-831 and
 * :1181/:1185, onto these functions).  Only the semantics FFTW documents for
 * an unnormalised complex-to-real transform are reproduced: the imaginary
 * parts of the DC and (even n) Nyquist inputs are ignored, the output is
 * sum_j X_j e^{+2 pi i j p / n} over the Hermitian completion of X.
 *
 * Algorithm: radix-2 iterative FFT for power-of-two lengths and Bluestein's
 * chirp-z reformulation (a power-of-two convolution) for every other length.
 * Results are labelled "not FFTW" wherever they are timed.
 */
#define _USE_MATH_DEFINES
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

typedef struct { double re, im; } cplx;

typedef struct {
  int n;           /* transform length */
  int pow2;        /* 1 if n is a power of two */
  int M;           /* convolution length (Bluestein) or n */
  cplx *tw;        /* twiddles for the length-M radix-2 FFT: e^{-2 pi i k / M}, k < M/2 */
  cplx *chirp;     /* w_k = e^{+i pi k^2 / n} (Bluestein, sign for the inverse DFT) */
  cplx *filt;      /* FFT of the Bluestein filter */
  cplx *work;      /* scratch of length M (not thread safe; one plan per thread) */
} or_fft_plan;

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

/* in-place radix-2 DIT, forward sign (e^{-2 pi i ...}) using tw of length M/2 */
static void fft_pow2(cplx *x, int M, const cplx *tw, int inverse) {
  for (int i = 1, j = 0; i < M; ++i) {
    int bit = M >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) { cplx t = x[i]; x[i] = x[j]; x[j] = t; }
  }
  for (int len = 2; len <= M; len <<= 1) {
    int step = M / len;
    for (int i = 0; i < M; i += len) {
      for (int k = 0; k < len / 2; ++k) {
        cplx w = tw[k * step];
        if (inverse) w.im = -w.im;
        cplx u = x[i + k], v = x[i + k + len / 2];
        cplx t = { v.re * w.re - v.im * w.im, v.re * w.im + v.im * w.re };
        x[i + k].re = u.re + t.re; x[i + k].im = u.im + t.im;
        x[i + k + len / 2].re = u.re - t.re; x[i + k + len / 2].im = u.im - t.im;
      }
    }
  }
}

or_fft_plan *or_fft_plan_create(int n) {
  or_fft_plan *p = calloc(1, sizeof(or_fft_plan));
  if (!p || n <= 0) { free(p); return NULL; }
  p->n = n;
  p->pow2 = is_pow2(n);
  if (p->pow2) {
    p->M = n;
  } else {
    p->M = 1;
    while (p->M < 2 * n - 1) p->M <<= 1;
  }
  int M = p->M;
  p->tw = malloc(sizeof(cplx) * (M / 2 + 1));
  p->work = malloc(sizeof(cplx) * M);
  for (int k = 0; k < M / 2 + 1; ++k) {
    double a = -2.0 * M_PI * (double)k / (double)M;
    p->tw[k].re = cos(a); p->tw[k].im = sin(a);
  }
  if (!p->pow2) {
    p->chirp = malloc(sizeof(cplx) * n);
    p->filt = calloc(M, sizeof(cplx));
    for (int k = 0; k < n; ++k) {
      /* k^2 mod 2n keeps the angle argument exact */
      int64_t k2 = ((int64_t)k * k) % (2 * (int64_t)n);
      double a = M_PI * (double)k2 / (double)n;
      p->chirp[k].re = cos(a); p->chirp[k].im = sin(a);
    }
    /* inverse DFT: X_p = sum_j x_j e^{+2pi i jp/n}; jp = (j^2 + p^2 - (p-j)^2)/2
       => X_p = w_p sum_j (x_j w_j) conj(w_{p-j}) ... with w_k = e^{i pi k^2/n} */
    for (int k = 0; k < n; ++k) {
      cplx c = { p->chirp[k].re, -p->chirp[k].im };
      p->filt[k] = c;
      if (k > 0) p->filt[M - k] = c;
    }
    fft_pow2(p->filt, M, p->tw, 0);
  }
  return p;
}

void or_fft_plan_destroy(or_fft_plan *p) {
  if (!p) return;
  free(p->tw); free(p->work); free(p->chirp); free(p->filt); free(p);
}

/* x (length n) <- sum_j x_j e^{+2 pi i j p / n} (unnormalised inverse DFT) */
void or_fft_inverse(or_fft_plan *p, cplx *x) {
  int n = p->n, M = p->M;
  if (p->pow2) { fft_pow2(x, n, p->tw, 1); return; }
  cplx *w = p->work;
  for (int k = 0; k < n; ++k) {
    cplx c = p->chirp[k];
    w[k].re = x[k].re * c.re - x[k].im * c.im;
    w[k].im = x[k].re * c.im + x[k].im * c.re;
  }
  for (int k = n; k < M; ++k) { w[k].re = 0; w[k].im = 0; }
  fft_pow2(w, M, p->tw, 0);
  for (int k = 0; k < M; ++k) {
    cplx a = w[k], b = p->filt[k];
    w[k].re = a.re * b.re - a.im * b.im;
    w[k].im = a.re * b.im + a.im * b.re;
  }
  fft_pow2(w, M, p->tw, 1);
  double inv = 1.0 / (double)M;
  for (int k = 0; k < n; ++k) {
    cplx c = p->chirp[k], a = { w[k].re * inv, w[k].im * inv };
    x[k].re = a.re * c.re - a.im * c.im;
    x[k].im = a.re * c.im + a.im * c.re;
  }
}

/* Unnormalised c2r of length n for `howmany` interleaved transforms.
   in:  complex element j of transform t at in[j*istride + t*idist] (j <= n/2)
   out: real element q of transform t at out[q*ostride + t*odist]
   in and out may alias (FFTW in-place use). */
void or_fft_c2r_many(or_fft_plan *p, int howmany, const double *in, int istride,
                     int idist, double *out, int ostride, int odist) {
  int n = p->n, h = n / 2;
  cplx *all = malloc(sizeof(cplx) * (size_t)n * howmany);
  for (int t = 0; t < howmany; ++t) {
    cplx *z = all + (size_t)t * n;
    for (int j = 0; j <= h; ++j) {
      const double *c = in + 2 * ((size_t)j * istride + (size_t)t * idist);
      z[j].re = c[0]; z[j].im = c[1];
    }
    z[0].im = 0;
    if (n % 2 == 0) z[h].im = 0;
    for (int j = h + 1; j < n; ++j) { z[j].re = z[n - j].re; z[j].im = -z[n - j].im; }
  }
  for (int t = 0; t < howmany; ++t) {
    cplx *z = all + (size_t)t * n;
    or_fft_inverse(p, z);
    for (int q = 0; q < n; ++q) out[(size_t)q * ostride + (size_t)t * odist] = z[q].re;
  }
  free(all);
}
