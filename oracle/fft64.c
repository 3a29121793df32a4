/*
 * ORACLE / TEST INFRASTRUCTURE ONLY — never linked into libamber_cuda.
 *
 * Plain FP64 discrete Fourier transforms for the CPU oracle and for the
 * FFTW-API shim that lets the reference's own sources build here.
 *
 * 1D: recursive mixed-radix Cooley–Tukey (decimation in time) for ANY length;
 * each prime factor p is combined with a direct p-point DFT, so lengths such
 * as 380 = 2·2·5·19 or 740 = 2·2·5·37 need no padding.  Twiddles come from
 * one table w[j] = exp(sign·2πi·j/N) of the full length.
 *
 * 2D c2r (the only transform amber uses: fftw_plan_dft_c2r_2d,
 * 4_fbe/amber_funcs.c:402,990,1116): unnormalised, exponent +1.
 * Convention (documented because the reference feeds a j=0 column that is not
 * Hermitian, amber_funcs.c:581-592): complex inverse DFT along axis 0 for every
 * stored column j ≤ n1/2, then a 1D c2r along axis 1 that ignores the
 * imaginary parts of bin 0 and (n1 even) bin n1/2 — the half-complex layout of
 * a 1D c2r has no slot for them.  Columns that are entirely zero are skipped.
 */
#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fft64.h"

typedef double complex cplx;

struct fft64_plan1d {
    int n;
    int nf;
    int f[64];
    cplx *w; /* w[j] = exp(+2πi j/n) */
};

static int factorize(int n, int *f)
{
    int nf = 0;
    /* radix 4 first keeps the recursion shallow; then 2, 3, 5, ... */
    while (n % 4 == 0) { f[nf++] = 4; n /= 4; }
    while (n % 2 == 0) { f[nf++] = 2; n /= 2; }
    for (int p = 3; (long)p * p <= n; p += 2)
        while (n % p == 0) { f[nf++] = p; n /= p; }
    if (n > 1) f[nf++] = n;
    return nf;
}

fft64_plan1d *fft64_plan1d_create(int n)
{
    fft64_plan1d *p = (fft64_plan1d *)calloc(1, sizeof(*p));
    p->n = n;
    p->nf = factorize(n, p->f);
    p->w = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    for (int j = 0; j < n; ++j) {
        /* reduce to the first octant-free form: angle = 2π j / n in long double */
        long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)j / (long double)n;
        p->w[j] = (double)cosl(a) + I * (double)sinl(a);
    }
    return p;
}

void fft64_plan1d_destroy(fft64_plan1d *p)
{
    if (!p) return;
    free(p->w);
    free(p);
}

/* out[k] = Σ_t in[t·is] · exp(sign·2πi t k / n), n = product of f[0..nf) ; stride into
 * the base table is ws = N/n. */
static void rec(const fft64_plan1d *pl, int sign, int n, const int *f, int nf, const cplx *in, long is,
                cplx *out, int ws, cplx *scratch)
{
    if (n == 1) { out[0] = in[0]; return; }
    int p = f[0];
    int m = n / p;
    for (int r = 0; r < p; ++r)
        rec(pl, sign, m, f + 1, nf - 1, in + r * is, is * p, out + (long)r * m, ws * p, scratch + n);
    /* combine: X[k + q m] = Σ_r Y_r[k] · W_n^{r (k + q m)} */
    const int N = pl->n;
    for (int k = 0; k < m; ++k) {
        for (int r = 0; r < p; ++r) scratch[r] = out[(long)r * m + k];
        for (int q = 0; q < p; ++q) {
            long kk = k + (long)q * m;
            cplx s = scratch[0];
            for (int r = 1; r < p; ++r) {
                long e = ((long)r * kk) % n;
                cplx tw = pl->w[(e * ws) % N];
                if (sign < 0) tw = conj(tw);
                s += scratch[r] * tw;
            }
            out[kk] = s;
        }
    }
}

void fft64_exec1d(const fft64_plan1d *p, int sign, const double *in_ri, double *out_ri)
{
    const int n = p->n;
    cplx *tmp = (cplx *)malloc(sizeof(cplx) * (size_t)n);
    cplx *scr = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * n + 64));
    rec(p, sign, n, p->f, p->nf, (const cplx *)in_ri, 1, tmp, 1, scr);
    memcpy(out_ri, tmp, sizeof(cplx) * (size_t)n);
    free(tmp);
    free(scr);
}

void fft64_c2r_2d(int n0, int n1, const double *in_ri, double *out, long out_stride, int nthreads)
{
    const int h = n1 / 2 + 1;
    fft64_plan1d *p0 = fft64_plan1d_create(n0);
    fft64_plan1d *p1 = fft64_plan1d_create(n1);
    cplx *mid = (cplx *)calloc((size_t)n0 * h, sizeof(cplx));
    const cplx *X = (const cplx *)in_ri;
    (void)nthreads;

#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1)
    {
        cplx *col = (cplx *)malloc(sizeof(cplx) * (size_t)(n0 > n1 ? n0 : n1));
        cplx *res = (cplx *)malloc(sizeof(cplx) * (size_t)(n0 > n1 ? n0 : n1));
        cplx *scr = (cplx *)malloc(sizeof(cplx) * (size_t)(2 * (n0 > n1 ? n0 : n1) + 64));
#pragma omp for schedule(static)
        for (int j = 0; j < h; ++j) {
            int nz = 0;
            for (int i = 0; i < n0; ++i) {
                col[i] = X[(long)i * h + j];
                nz |= (col[i] != 0);
            }
            if (!nz) continue; /* mid is already zero */
            rec(p0, +1, n0, p0->f, p0->nf, col, 1, res, 1, scr);
            for (int i = 0; i < n0; ++i) mid[(long)i * h + j] = res[i];
        }
#pragma omp for schedule(static)
        for (int i = 0; i < n0; ++i) {
            const cplx *row = mid + (long)i * h;
            for (int k = 0; k < h && k < n1; ++k) col[k] = row[k];
            col[0] = creal(col[0]);
            if (n1 % 2 == 0) col[n1 / 2] = creal(col[n1 / 2]);
            for (int k = h; k < n1; ++k) col[k] = conj(row[n1 - k]);
            rec(p1, +1, n1, p1->f, p1->nf, col, 1, res, 1, scr);
            for (int k = 0; k < n1; ++k) out[(long)i * out_stride + k] = creal(res[k]);
        }
        free(col);
        free(res);
        free(scr);
    }
    free(mid);
    fft64_plan1d_destroy(p0);
    fft64_plan1d_destroy(p1);
}
