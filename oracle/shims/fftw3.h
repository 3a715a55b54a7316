/* ORACLE shim: the two FFTW3 entry points the reference's C library calls
   (src/wavemoth.c:828-831, :1181, :1185), mapped onto oracle/fft.c.  FFTW3 is
   not installed in this image; transforms computed through this shim are
   labelled "not FFTW" wherever they are timed. */
#ifndef ORACLE_FFTW3_SHIM_H
#define ORACLE_FFTW3_SHIM_H
typedef double fftw_complex[2];
typedef struct or_fftw_plan_s *fftw_plan;
#define FFTW_MEASURE (0U)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_ESTIMATE (1U << 6)
fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out);
void fftw_destroy_plan(fftw_plan p);
#endif
