/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Minimal FFTW3 API stand-in so that the reference's unmodified
 * 4_fbe/amber_funcs.c builds here (FFTW is not installed).  Declares only the
 * calls amber uses: fftw_plan_dft_c2r_2d, fftw_execute, fftw_destroy_plan,
 * fftw_init_threads, fftw_plan_with_nthreads.  The arithmetic is our own
 * FP64 mixed-radix DFT (oracle/fft64.c); it is NOT FFTW, so agreement with a
 * real FFTW build is to FP64 rounding only ("parity unpinned" at this edge).
 */
#ifndef AMBER_ORACLE_FFTW3_SHIM_H
#define AMBER_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int nthreads);
void fftw_cleanup_threads(void);

#ifdef __cplusplus
}
#endif
#endif
