/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Driver that runs the reference's OWN estimator functions, compiled unchanged
 * from 4_fbe/amber_funcs.c and 4_fbe/vars.c, on parameters instead of the
 * constants hard-coded in 4_fbe/amber.c:43-54,187 and annular_rings
 * (amber_funcs.c:2022-2094).  The control flow follows amber.c:21-335 (v1) and
 * amber_v2.c:21-345 (v2): read_inputs_ess → initialize → ReadGVnAC_gridding →
 * normalize_data → rings → calCR → read_rings → uf_chans / vcp table → per
 * triangle: fill_s2d_float (+ fill_s2I) ×3 → OpenMP triple-product loop → file.
 *
 * Built twice by oracle/Makefile: as shipped (float maps and accumulators —
 * the byte-format reference and the timed CPU baseline) and with
 * -Dfloat=double (the FP64 reference).
 *
 * usage: ref_amber <Rlzn> <v1|v2> <nc10> <uf_nc> <rings_file> <rp_begin> <rp_end>
 *                  <nthreads> <res_path> <input_params_ess>
 * rings_file: "Nr" then Nr lines "ULow UHigh" (text, %lf).
 * Prints one JSON line with timings (accumulation timed like amber.c:230,285).
 */
#include <math.h>
#include <omp.h>
#include <stdalign.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"
#include "mabs_funcs.h"
#include "vars.h"

static double ng1_of(double uhigh, double du, long *ng1_out)
{
    /* amber.c:193-197 */
    double umax = uhigh + 3;
    long nmax = (long)(umax / du);
    long ng1 = (long)(3 * nmax);
    ng1 = (ng1 % 2 == 0) ? ng1 + 2 : ng1 + 3;
    *ng1_out = ng1;
    return umax;
}

int main(int argc, char **argv)
{
    if (argc != 11) {
        fprintf(stderr,
                "usage: %s <Rlzn> <v1|v2> <nc10> <uf_nc> <rings_file> <rp_begin> <rp_end> <nthreads> "
                "<res_path> <input_params_ess>\n",
                argv[0]);
        return 1;
    }
    int Rlzn = atoi(argv[1]);
    int v2 = strcmp(argv[2], "v2") == 0;
    int rp_begin = atoi(argv[6]), rp_end = atoi(argv[7]);
    int nthreads = atoi(argv[8]);
    NRi = Rlzn;
    nc10 = atoi(argv[3]);
    uf_nc = atoi(argv[4]);
    snprintf(res_path, sizeof(res_path), "%s", argv[9]);
    read_inputs_ess(argv[10]);

    FILE *fr = fopen(argv[5], "r");
    if (!fr || fscanf(fr, "%d", &Nr) != 1 || Nr <= 0) {
        fprintf(stderr, "bad rings file\n");
        return 1;
    }
    Umin = 1.;
    int nclen = 2 * nc10 + 1;
    int ncsize = nclen * nclen;
    Nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();

    double t_all = omp_get_wtime();
    initialize();
    ReadGVnAC_gridding();
    normalize_data();
    for (int i = 0; i < Nr; ++i)
        if (fscanf(fr, "%lf %lf", &ULow[i], &UHigh[i]) != 2) {
            fprintf(stderr, "bad rings file\n");
            return 1;
        }
    fclose(fr);
    for (int i = 0; i < Nr; ++i) /* bin average, amber_funcs.c:2065 */
        Uavg[i] = (2. / 3.) * (pow(UHigh[i], 3.) - pow(ULow[i], 3.)) / (pow(UHigh[i], 2.) - pow(ULow[i], 2.));

    long sd_size;
    Umax = ng1_of(UHigh[Nr - 1], Du, &Ng1);
    Ng2 = Ng1;
    sd_size = Ng1 * Ng2;
    float **sd1 = allocate_2d_float_aligned(nc, sd_size);
    float **sd2 = allocate_2d_float_aligned(nc, sd_size);
    float **sd3 = allocate_2d_float_aligned(nc, sd_size);
    float **sI1 = NULL, **sI2 = NULL, **sI3 = NULL;
    if (v2) {
        sI1 = allocate_2d_float_aligned(nc, sd_size);
        sI2 = allocate_2d_float_aligned(nc, sd_size);
        sI3 = allocate_2d_float_aligned(nc, sd_size);
    }
    fftw_init_threads();
    fftw_plan_with_nthreads(Nthreads);
    omp_set_num_threads(Nthreads);

    calCR();
    int rcount;
    double *rdata;
    read_rings(&rcount, &rdata);

    int *vcp = NULL, total_vcp = 0;
    if (flag_key == 1) {
        if (get_uf_chans("uf_chans.txt") != 0) {
            fprintf(stderr, "uf_chans.txt unreadable\n");
            return 1;
        }
        total_vcp = precompute_unflg_vcp(nc10, &vcp);
    } else if (flag_key == 0) {
        total_vcp = precompute_vcp_dnu(nc, nc10, &vcp);
    } else {
        fprintf(stderr, "bad flag_key %d\n", flag_key);
        return 1;
    }

    float *bldnu = (float *)aligned_alloc(64, ncsize * sizeof(float));
    int *numdnu_i = (int *)aligned_alloc(64, ncsize * sizeof(int));
    float *numdnu_f = (float *)aligned_alloc(64, ncsize * sizeof(float));
    double t_acc = 0, t_maps = 0, products = 0;
    if (rp_end > rcount || rp_end < 0) rp_end = rcount;

    for (int rp = rp_begin; rp < rp_end; ++rp) {
        int r1 = (int)rdata[rp * 4 + 0], r2 = (int)rdata[rp * 4 + 1], r3 = (int)rdata[rp * 4 + 2];
        Umax = ng1_of(UHigh[r1], Du, &Ng1);
        Ng2 = Ng1;
        double gfact = (1. * Ng1) / (1. * N1);
        double Num = gfact * gfact * rdata[rp * 4 + 3];
        double inv_Ng1_Ng2 = 1.0 / (Ng1 * Ng2 * 1.);
        sd_size = Ng1 * Ng2;

        double t0 = omp_get_wtime();
        fill_s2d_float(sd1, r1, 1, 1);
        fill_s2d_float(sd2, r2, 1, 1);
        fill_s2d_float(sd3, r3, 1, 1);
        if (v2) {
            fill_s2I(sI1, r1);
            fill_s2I(sI2, r2);
            fill_s2I(sI3, r3);
        }
        t_maps += omp_get_wtime() - t0;

        memset(bldnu, 0, ncsize * sizeof(float));
        memset(numdnu_i, 0, ncsize * sizeof(int));
        memset(numdnu_f, 0, ncsize * sizeof(float));
        t0 = omp_get_wtime();
        /* triple-product lag accumulation: the loop of amber.c:234-283 and
         * amber_v2.c:230-288 — per-thread lag buffers, dynamic schedule over
         * the vcp tuples, merged under a critical section. */
#pragma omp parallel num_threads(Nthreads)
        {
            float *my_b = (float *)calloc(ncsize, sizeof(float));
            int *my_ni = (int *)calloc(ncsize, sizeof(int));
            float *my_nf = (float *)calloc(ncsize, sizeof(float));
#pragma omp for schedule(dynamic) nowait
            for (int t = 0; t < total_vcp; ++t) {
                const int *tu = vcp + 6 * (long)t;
                const float *restrict a = sd1[tu[0]];
                const float *restrict b = sd2[tu[1]];
                const float *restrict c = sd3[tu[2]];
                float acc = 0.;
                for (long x = 0; x < sd_size; ++x) acc += a[x] * b[x] * c[x];
                my_b[tu[5]] += acc;
                if (v2) {
                    const float *restrict ia = sI1[tu[0]];
                    const float *restrict ib = sI2[tu[1]];
                    const float *restrict ic = sI3[tu[2]];
                    float nt = 0.;
                    for (long x = 0; x < sd_size; ++x) nt += ia[x] * ib[x] * ic[x];
                    my_nf[tu[5]] += nt;
                } else {
                    my_ni[tu[5]] += 1;
                }
            }
#pragma omp critical
            {
                for (int i = 0; i < ncsize; ++i) {
                    bldnu[i] += my_b[i];
                    numdnu_i[i] += my_ni[i];
                    numdnu_f[i] += my_nf[i];
                }
            }
            free(my_b);
            free(my_ni);
            free(my_nf);
        }
        t_acc += omp_get_wtime() - t0;
        products += (double)total_vcp * (double)sd_size;

        char fname[1024];
        FILE *fo;
        if (v2) {
            snprintf(fname, sizeof(fname), "%s/bsout_final2_ra%d_rb%d_rc%d_R%d", res_path, r1, r2, r3, Rlzn);
            fo = fopen(fname, "wb");
            if (!fo) { perror("fopen"); return 1; }
            fwrite(&inv_Ng1_Ng2, sizeof(double), 1, fo);
            fwrite(bldnu, sizeof(float), ncsize, fo);
            fwrite(numdnu_f, sizeof(float), ncsize, fo);
        } else {
            double Ntri = Num * inv_Ng1_Ng2;
            snprintf(fname, sizeof(fname), "%s/bsout_final_ra%d_rb%d_rc%d_R%d", res_path, r1, r2, r3, Rlzn);
            fo = fopen(fname, "wb");
            if (!fo) { perror("fopen"); return 1; }
            fwrite(&Ntri, sizeof(double), 1, fo);
            fwrite(&Num, sizeof(double), 1, fo);
            fwrite(bldnu, sizeof(float), ncsize, fo);
            fwrite(numdnu_i, sizeof(int), ncsize, fo);
        }
        fclose(fo);
    }
    printf("AMBER_REF_JSON {\"rcount\": %d, \"total_vcp\": %d, \"rp_begin\": %d, \"rp_end\": %d, \"threads\": %d, "
           "\"accum_s\": %.6f, \"maps_s\": %.6f, \"products\": %.17g, \"total_s\": %.6f, \"float_bytes\": %d}\n",
           rcount, total_vcp, rp_begin, rp_end, Nthreads, t_acc, t_maps, products, omp_get_wtime() - t_all,
           (int)sizeof(float));
    return 0;
}
