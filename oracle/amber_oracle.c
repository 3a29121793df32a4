/*
 * ORACLE / TEST INFRASTRUCTURE ONLY — a plain FP64 CPU restatement of the
 * AMBER estimator hot path, used by tests/, smoke() and bench.py's CPU
 * baseline as the checker.  Nothing in libamber_cuda links or calls this.
 *
 * Each function follows the reference line by line in arithmetic order (file:line
 * cited per function) but computes in double where the reference used float for
 * the maps and the triple-product sums, so it is the "FP64 oracle of the plain
 * method".  It is pinned against the reference's own sources built with
 * -Dfloat=double (oracle/_ref/ref_amber64) and, for gridding, against the
 * reference's own vcg (oracle/_ref/ref_vcg); see tests/test_oracle_pins.py.
 *
 * Layouts (all row-major, the file order of the reference):
 *   grid  re_im[cell][nc][2], cell = ii·(N1/2+1) + jj
 *   count ntig[cell][nc]
 *   maps  m[p][x], x = ii·Ng1 + jj over the Ng1 × Ng1 grid
 *   lags  bldnu[(Δ2+nc10)·nclen + (Δ3+nc10)]
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "fft64.h"

#define ORC_EXPORT __attribute__((visibility("default")))

/* ---- a1: gridding, 3_vcg/tgefuncs.c:377-505 (flag_key 1) and 511-621 (flag_key 0) ----
 * randpar [G][npar] (u/ν0, v/ν0, ...), data [G][nc][nstokes][3] (re, im, wt);
 * only Stokes 0 (RR) reaches the output files (tgefuncs.c:480-493, 645-655).
 * Returns 0, or -1 if a record lands outside the NN × (NN/2+1) grid (the
 * reference would write out of bounds there). */
ORC_EXPORT int orc_grid_vis(long NN, long nc, double dU, double Umax, float nu_chan0, int flag_key, long G,
                            long npar, long nstokes, const float *randpar, const float *data, double *re_im,
                            double *ntig)
{
    const long H = NN / 2 + 1;
    for (long g = 0; g < G; ++g) {
        const float *rp = randpar + g * npar;
        float signv = (rp[1] < 0.f) ? -1.f : 1.f; /* tgefuncs.c:400 */
        float u1 = nu_chan0 * signv * rp[0];     /* 402 */
        float v1 = nu_chan0 * signv * rp[1];     /* 403 */
        float s = u1 * u1 + v1 * v1;
        double Uval = sqrt((double)s); /* 405 */
        if (!(Uval <= Umax)) continue;
        int ii = (int)round(u1 / dU); /* 466-468 */
        ii = (ii < 0) ? (int)(NN + ii) : ii;
        int jj = (int)round(v1 / dU);
        if (ii < 0 || ii >= NN || jj < 0 || jj >= H) return -1;
        long index = (long)ii * H + jj; /* 483 */
        const float *d = data + g * nc * nstokes * 3;
        for (long nn = 0; nn < nc; ++nn) {
            const float *rr = d + nn * nstokes * 3;
            float re, im, n;
            if (flag_key == 1) { /* 418-431 */
                if (rr[2] > 0.f) { re = rr[0]; im = signv * rr[1]; n = 1.f; }
                else { re = 0.f; im = 0.f; n = 0.f; }
            } else { /* 564-566, 608 */
                re = rr[0]; im = signv * rr[1]; n = 1.f;
            }
            re_im[(index * nc + nn) * 2 + 0] += re;
            re_im[(index * nc + nn) * 2 + 1] += im;
            ntig[index * nc + nn] += n;
        }
    }
    return 0;
}

/* ---- a3: normalize_data, 4_fbe/amber_funcs.c:1946-1978 ---- */
ORC_EXPORT void orc_normalize(long ncell, long nc, double *re_im, double *ntig)
{
    for (long i = 0; i < ncell * nc; ++i)
        if (ntig[i] > 0) { re_im[2 * i] /= ntig[i]; re_im[2 * i + 1] /= ntig[i]; }
    for (long i = 0; i < ncell * nc; ++i)
        if (ntig[i] > 0) ntig[i] = 1;
}

/* ---- a4: ring geometry and closed triangles ---- */
ORC_EXPORT void orc_uavg(int Nr, const double *lo, const double *hi, double *uavg)
{
    for (int i = 0; i < Nr; ++i) /* amber_funcs.c:2065 */
        uavg[i] = (2. / 3.) * (pow(hi[i], 3.) - pow(lo[i], 3.)) / (pow(hi[i], 2.) - pow(lo[i], 2.));
}

/* Closed-triangle rule of calCR, amber_funcs.c:439-449; order r1 ↑, r2 ≤ r1 ↑, r3 ≤ r2 ↑.
 * tri may be NULL (count only). */
ORC_EXPORT int orc_triangles(int Nr, const double *Uavg, int *tri, int maxtri)
{
    int n = 0;
    for (int r1 = 0; r1 < Nr; ++r1)
        for (int r2 = 0; r2 <= r1; ++r2) {
            double tt = Uavg[r2] / Uavg[r1];
            if (tt >= 0.5 && tt <= 1.0)
                for (int r3 = 0; r3 <= r2; ++r3) {
                    double mu = 0.5 * (tt + 1. / tt - (Uavg[r3] / Uavg[r1]) * (Uavg[r3] / Uavg[r2]));
                    if (mu >= 0.5 / tt && mu <= 1.0) {
                        if (tri && n < maxtri) { tri[3 * n] = r1; tri[3 * n + 1] = r2; tri[3 * n + 2] = r3; }
                        ++n;
                    }
                }
        }
    return n;
}

/* Padded map side, 4_fbe/amber.c:193-197. */
ORC_EXPORT long orc_ng1(double uhigh, double Du)
{
    double umax = uhigh + 3;
    long nmax = (long)(umax / Du);
    long ng1 = (long)(3 * nmax);
    return (ng1 % 2 == 0) ? ng1 + 2 : ng1 + 3;
}

/* calCR, amber_funcs.c:389-491: ring-masked channel-5 sampling mask on the
 * N1 grid (j < N1/3, |ia| folded), c2r, then Num = Σ II_r1·II_r2·II_r3.
 * rdata[4·t] = {r1, r2, r3, Num}.  Returns rcount. */
ORC_EXPORT int orc_calcr(long N1, long nc, const double *ntig, int Nr, const double *lo, const double *hi,
                         const double *Uavg, double *rdata, int maxtri, int nthreads)
{
    const long H = N1 / 2 + 1, K = N1 * N1;
    const int plane = 5; /* amber_funcs.c:427 */
    double *II = (double *)malloc(sizeof(double) * (size_t)(Nr * K));
    double *AA = (double *)malloc(sizeof(double) * (size_t)(N1 * H * 2));
    for (int r = 0; r < Nr; ++r) {
        memset(AA, 0, sizeof(double) * (size_t)(N1 * H * 2));
        for (long i = 0; i < N1; ++i) {
            long ia = (i > N1 / 2) ? (N1 - i) : i;
            for (long j = 0; j < N1 / 3; ++j) {
                long index = i * H + j;
                double uu = sqrt(1.0 * (ia * ia + j * j));
                if (uu >= lo[r] && uu < hi[r] && uu > 0.0) {
                    AA[2 * index] = ntig[index * nc + plane];
                    AA[2 * index + 1] = 0.0;
                }
            }
        }
        fft64_c2r_2d((int)N1, (int)N1, AA, II + (long)r * K, N1, nthreads);
    }
    int n = 0;
    for (int r1 = 0; r1 < Nr; ++r1)
        for (int r2 = 0; r2 <= r1; ++r2) {
            double tt = Uavg[r2] / Uavg[r1];
            if (tt >= 0.5 && tt <= 1.0)
                for (int r3 = 0; r3 <= r2; ++r3) {
                    double mu = 0.5 * (tt + 1. / tt - (Uavg[r3] / Uavg[r1]) * (Uavg[r3] / Uavg[r2]));
                    if (mu >= 0.5 / tt && mu <= 1.0) {
                        const double *a = II + (long)r1 * K, *b = II + (long)r2 * K, *c = II + (long)r3 * K;
                        double Num = 0.0;
                        for (long x = 0; x < K; ++x) Num += a[x] * b[x] * c[x];
                        if (n < maxtri) {
                            rdata[4 * n] = r1; rdata[4 * n + 1] = r2; rdata[4 * n + 2] = r3; rdata[4 * n + 3] = Num;
                        }
                        ++n;
                    }
                }
        }
    free(II);
    free(AA);
    return n;
}

/* ---- a6/a7: Dfg / Ifg + c2r, amber_funcs.c:573-621 (FP64 maps; the reference
 * casts them to float, amber_funcs.c:992-999).  src: complex grid (mask == 0)
 * or sampling mask (mask == 1, imaginary part 0).  out: Ng1 × Ng1. ---- */
static int ring_map(long N1, long nc, const double *src, int mask, double lo, double hi, long Ng1, int plane,
                    double *out, int nthreads)
{
    const long H1 = N1 / 2 + 1, Hg = Ng1 / 2 + 1;
    double *buf = (double *)calloc((size_t)(Ng1 * Hg * 2), sizeof(double));
    for (long ia = -Ng1 / 2 + 1; ia < Ng1 / 2 + 1; ++ia)
        for (long j = 0; j < Ng1 / 3; ++j) {
            long iN = (ia < 0) ? (N1 + ia) : ia;
            long iNg = (ia < 0) ? (Ng1 + ia) : ia;
            double uu = sqrt(1. * (ia * ia + j * j));
            if (uu >= lo && uu < hi && uu > 0.0) {
                if (iN < 0 || iN >= N1 || j >= H1) { free(buf); return -1; }
                long idxN = iN * H1 + j, idxG = iNg * Hg + j;
                if (mask) {
                    buf[2 * idxG] = src[idxN * nc + plane];
                    buf[2 * idxG + 1] = 0.;
                } else {
                    buf[2 * idxG] = src[(idxN * nc + plane) * 2];
                    buf[2 * idxG + 1] = src[(idxN * nc + plane) * 2 + 1];
                }
            }
        }
    fft64_c2r_2d((int)Ng1, (int)Ng1, buf, out, Ng1, nthreads);
    free(buf);
    return 0;
}

ORC_EXPORT int orc_ring_map(long N1, long nc, const double *re_im, double lo, double hi, long Ng1, int plane,
                            double *out, int nthreads)
{
    return ring_map(N1, nc, re_im, 0, lo, hi, Ng1, plane, out, nthreads);
}

ORC_EXPORT int orc_ring_mask_map(long N1, long nc, const double *ntig, double lo, double hi, long Ng1, int plane,
                                 double *out, int nthreads)
{
    return ring_map(N1, nc, ntig, 1, lo, hi, Ng1, plane, out, nthreads);
}

/* ---- a5 + a8/a9: channel-triplet enumeration (precompute_vcp_dnu,
 * amber_funcs.c:2264-2310, when uf_nc == 0; precompute_unflg_vcp, 2207-2259,
 * otherwise) and the triple-product loop of amber.c:247-266 /
 * amber_v2.c:243-270, in FP64.  Maps m1/m2/m3 (and i1/i2/i3 for v2, else
 * NULL) are [nc][K].  Per-anchor partial lag arrays are summed in anchor
 * order, so the result is deterministic.  Returns total_vcp. ---- */
ORC_EXPORT long orc_triangle(long K, long nc, int nc10, int uf_nc, const int *uf_chans, const double *m1,
                             const double *m2, const double *m3, const double *i1, const double *i2,
                             const double *i3, double *bldnu, int64_t *numdnu, double *numtri, int nthreads)
{
    const int nclen = 2 * nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    const int n = uf_nc > 0 ? uf_nc : (int)nc;
    double *pb = (double *)calloc((size_t)(n * ncsize), sizeof(double));
    double *pn = (double *)calloc((size_t)(n * ncsize), sizeof(double));
    int64_t *pc = (int64_t *)calloc((size_t)(n * ncsize), sizeof(int64_t));
    long total = 0;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : total)
    for (int a = 0; a < n; ++a) {
        int p1 = uf_nc > 0 ? uf_chans[a] : a;
        for (int b = 0; b < n; ++b) {
            int p2 = uf_nc > 0 ? uf_chans[b] : b;
            if (abs(p2 - p1) > nc10) continue;
            for (int c = 0; c < n; ++c) {
                int p3 = uf_nc > 0 ? uf_chans[c] : c;
                if (abs(p3 - p1) > nc10) continue;
                long idx = (long)(p2 - p1 + nc10) * nclen + (p3 - p1 + nc10);
                const double *x1 = m1 + (long)p1 * K, *x2 = m2 + (long)p2 * K, *x3 = m3 + (long)p3 * K;
                double s = 0.;
                for (long x = 0; x < K; ++x) s += x1[x] * x2[x] * x3[x];
                pb[(long)a * ncsize + idx] += s;
                if (i1) {
                    const double *y1 = i1 + (long)p1 * K, *y2 = i2 + (long)p2 * K, *y3 = i3 + (long)p3 * K;
                    double t = 0.;
                    for (long x = 0; x < K; ++x) t += y1[x] * y2[x] * y3[x];
                    pn[(long)a * ncsize + idx] += t;
                }
                pc[(long)a * ncsize + idx] += 1;
                ++total;
            }
        }
    }
    for (long i = 0; i < ncsize; ++i) {
        double sb = 0., sn = 0.;
        int64_t sc = 0;
        for (int a = 0; a < n; ++a) {
            sb += pb[(long)a * ncsize + i];
            sn += pn[(long)a * ncsize + i];
            sc += pc[(long)a * ncsize + i];
        }
        bldnu[i] = sb;
        if (numdnu) numdnu[i] = sc;
        if (numtri) numtri[i] = sn;
    }
    free(pb);
    free(pn);
    free(pc);
    return total;
}

/* Σ|products| per lag cell — the scale against which mixed-precision error
 * is measured.  Same enumeration as orc_triangle. */
ORC_EXPORT void orc_triangle_absscale(long K, long nc, int nc10, int uf_nc, const int *uf_chans, const double *m1,
                                      const double *m2, const double *m3, double *absscale, int nthreads)
{
    const int nclen = 2 * nc10 + 1;
    const long ncsize = (long)nclen * nclen;
    const int n = uf_nc > 0 ? uf_nc : (int)nc;
    double *pb = (double *)calloc((size_t)(n * ncsize), sizeof(double));
#pragma omp parallel for schedule(dynamic) num_threads(nthreads > 0 ? nthreads : 1)
    for (int a = 0; a < n; ++a) {
        int p1 = uf_nc > 0 ? uf_chans[a] : a;
        for (int b = 0; b < n; ++b) {
            int p2 = uf_nc > 0 ? uf_chans[b] : b;
            if (abs(p2 - p1) > nc10) continue;
            for (int c = 0; c < n; ++c) {
                int p3 = uf_nc > 0 ? uf_chans[c] : c;
                if (abs(p3 - p1) > nc10) continue;
                long idx = (long)(p2 - p1 + nc10) * nclen + (p3 - p1 + nc10);
                const double *x1 = m1 + (long)p1 * K, *x2 = m2 + (long)p2 * K, *x3 = m3 + (long)p3 * K;
                double s = 0.;
                for (long x = 0; x < K; ++x) s += fabs(x1[x] * x2[x] * x3[x]);
                pb[(long)a * ncsize + idx] += s;
            }
        }
    }
    for (long i = 0; i < ncsize; ++i) {
        double sb = 0.;
        for (int a = 0; a < n; ++a) sb += pb[(long)a * ncsize + i];
        absscale[i] = sb;
    }
    free(pb);
}

/* ---- f3: MAPS two-point function, amber_funcs.c:1418-1488 (cl_dnu) driven as
 * 4_fbe/maps.c:179-210 does: for every channel pair nn1 <= nn2, per log bin of
 * U = |(ia, j)|·Du in [umin, umax):
 *   no    = Σ NTiG[nn1],  pksum = Σ (Re1·Re2 + Im1·Im2)·NTiG[nn1],  usum = Σ U·NTiG[nn1]
 * (cells in index order), binps = pksum/no, binu = usum/no where no != 0; then
 * cldnu[b][nn2−nn1] += binps (nn1 ascending) and numdnu[nn2−nn1] += 1.  binu and
 * num are what the last pair (nn1 = nn2 = nc−1) leaves, as maps.c prints them.
 * The grid is the normalised one (normalize_data).  A cell whose bin index
 * rounds to NB (U just below umax) is skipped; the reference would write past
 * its arrays there.  cldnu_abs (may be NULL) is the same sum over |terms|. */
ORC_EXPORT void orc_cl_dnu(long N1, long nc, double Du, const double *re_im, const double *ntig, int NB, double umin,
                           double umax, double *cldnu, double *cldnu_abs, double *numdnu, double *binu, int *num)
{
    const long H = N1 / 2 + 1;
    double *usum = (double *)calloc(NB, sizeof(double));
    double *pksum = (double *)calloc(NB, sizeof(double));
    double *pkabs = (double *)calloc(NB, sizeof(double));
    int *no = (int *)calloc(NB, sizeof(int));
    const double binsiz = log10(umax / umin) / (1. * NB);
    memset(cldnu, 0, sizeof(double) * NB * nc);
    if (cldnu_abs) memset(cldnu_abs, 0, sizeof(double) * NB * nc);
    memset(numdnu, 0, sizeof(double) * nc);
    for (long n1 = 0; n1 < nc; ++n1)
        for (long n2 = n1; n2 < nc; ++n2) {
            for (int i = 0; i < NB; ++i) {
                no[i] = 0;
                usum[i] = pksum[i] = pkabs[i] = 0.0;
            }
            for (long i = 0; i < N1; ++i)
                for (long j = 0; j < H; ++j) {
                    const long index = i * H + j;
                    const long ia = (i > N1 / 2) ? (N1 - i) : i;
                    const double uu = sqrt(1. * (ia * ia + j * j)) * Du;
                    if (uu >= umin && uu < umax) {
                        const double *a = re_im + 2 * (index * nc + n1), *b = re_im + 2 * (index * nc + n2);
                        double numer = a[0] * b[0] + a[1] * b[1];
                        const double w = ntig[index * nc + n1];
                        numer *= w;
                        const int tmp = (int)floor(log10(uu / umin) / binsiz);
                        if (tmp < 0 || tmp >= NB) continue;
                        no[tmp] += w;
                        pksum[tmp] += numer;
                        pkabs[tmp] += fabs(numer);
                        usum[tmp] += uu * w;
                    }
                }
            for (int i = 0; i < NB; ++i)
                if (no[i] != 0) {
                    usum[i] /= (1. * no[i]);
                    pksum[i] /= (1. * no[i]);
                    pkabs[i] /= (1. * no[i]);
                }
            numdnu[n2 - n1] += 1.;
            for (int i = 0; i < NB; ++i) {
                cldnu[i * nc + (n2 - n1)] += pksum[i];
                if (cldnu_abs) cldnu_abs[i * nc + (n2 - n1)] += pkabs[i];
            }
        }
    for (int i = 0; i < NB; ++i) {
        binu[i] = usum[i];
        num[i] = no[i];
    }
    free(usum);
    free(pksum);
    free(pkabs);
    free(no);
}
