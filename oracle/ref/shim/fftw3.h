/*
 * FFTW3-API-compatible header for the reference CPU build (test
 * infrastructure only).  FFTW is not installed in this image; the reference's
 * math/fft.c only needs the subset declared here.  The implementation in
 * fftw_shim.c is a project-written mixed-radix DFT derived from the DFT
 * definition  X[k] = sum_j x[j] exp(sign * 2*pi*i*j*k/n)  (no scaling), which is
 * the convention FFTW documents for FFTW_FORWARD (-1) and FFTW_BACKWARD (+1).
 * It is not FFTW code.
 */
#ifndef MAOSREF_SHIM_FFTW3_H
#define MAOSREF_SHIM_FFTW3_H
#include <stdio.h>
#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)
#define FFTW_EXHAUSTIVE (1U << 3)
#define FFTW_UNALIGNED (1U << 1)

typedef enum { FFTW_R2HC = 0, FFTW_HC2R = 1 } fftw_r2r_kind;
typedef fftw_r2r_kind fftwf_r2r_kind;

typedef struct { int n, is, os; } fftw_iodim;
typedef fftw_iodim fftwf_iodim;

typedef double fftw_complex[2];
typedef float fftwf_complex[2];

typedef struct maosref_fft_plan *fftw_plan;
typedef struct maosref_fft_plan *fftwf_plan;

/* double precision */
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed, int istride, int idist,
                             fftw_complex *out, const int *onembed, int ostride, int odist,
                             int sign, unsigned flags);
fftw_plan fftw_plan_guru_split_dft(int rank, const fftw_iodim *dims, int howmany_rank,
                                   const fftw_iodim *howmany_dims, double *ri, double *ii,
                                   double *ro, double *io, unsigned flags);
fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);
void fftw_cleanup(void);
int fftw_import_wisdom_from_file(FILE *f);
void fftw_export_wisdom_to_file(FILE *f);

/* single precision */
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_many_dft(int rank, const int *n, int howmany,
                               fftwf_complex *in, const int *inembed, int istride, int idist,
                               fftwf_complex *out, const int *onembed, int ostride, int odist,
                               int sign, unsigned flags);
fftwf_plan fftwf_plan_guru_split_dft(int rank, const fftwf_iodim *dims, int howmany_rank,
                                     const fftwf_iodim *howmany_dims, float *ri, float *ii,
                                     float *ro, float *io, unsigned flags);
fftwf_plan fftwf_plan_r2r_1d(int n, float *in, float *out, fftwf_r2r_kind kind, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup_threads(void);
void fftwf_cleanup(void);
int fftwf_import_wisdom_from_file(FILE *f);
void fftwf_export_wisdom_to_file(FILE *f);

#ifdef __cplusplus
}
#endif
#endif
