/* ORACLE / TEST INFRASTRUCTURE ONLY: FP64 reference DFTs (see fft64.c). */
#ifndef AMBER_ORACLE_FFT64_H
#define AMBER_ORACLE_FFT64_H

typedef struct fft64_plan1d fft64_plan1d;

fft64_plan1d *fft64_plan1d_create(int n);
void fft64_plan1d_destroy(fft64_plan1d *p);
/* in/out: n interleaved (re, im) pairs; sign = +1 (inverse, unnormalised) or -1. */
void fft64_exec1d(const fft64_plan1d *p, int sign, const double *in_ri, double *out_ri);

/* Unnormalised 2D complex-to-real, exponent +1.  in_ri: n0 × (n1/2+1) complex
 * (interleaved).  out: n0 rows of n1 reals, row stride out_stride doubles.  in
 * and out may alias (FFTW in-place layout: out_stride = 2(n1/2+1)). */
void fft64_c2r_2d(int n0, int n1, const double *in_ri, double *out, long out_stride, int nthreads);

#endif
