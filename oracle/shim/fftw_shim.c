/*
 * ORACLE / TEST INFRASTRUCTURE ONLY: FFTW3-API shim over oracle/fft64.c.
 * The plan records the arrays; fftw_execute runs the unnormalised c2r with
 * the convention stated in fft64.c.  In-place plans (out == in, as every
 * amber call site uses, amber_funcs.c:990-991) write rows with FFTW's padded
 * stride 2(n1/2+1); out-of-place plans write n1 reals per row.
 */
#include <stdlib.h>
#include "fftw3.h"
#include "../fft64.h"

struct fftw_plan_s {
    int n0, n1;
    fftw_complex *in;
    double *out;
    int nthreads;
};

static int g_nthreads = 1;

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags)
{
    (void)flags;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->n0 = n0;
    p->n1 = n1;
    p->in = in;
    p->out = out;
    p->nthreads = g_nthreads;
    return p;
}

void fftw_execute(const fftw_plan p)
{
    long stride = ((void *)p->out == (void *)p->in) ? 2L * (p->n1 / 2 + 1) : p->n1;
    fft64_c2r_2d(p->n0, p->n1, (const double *)p->in, p->out, stride, p->nthreads);
}

void fftw_destroy_plan(fftw_plan p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { g_nthreads = nthreads > 0 ? nthreads : 1; }
void fftw_cleanup_threads(void) {}
