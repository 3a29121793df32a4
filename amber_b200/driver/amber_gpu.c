/*
 * amber_gpu — drop-in for 4_fbe/amber (v1) and 4_fbe/amber_v2 (v2) on a B200.
 *
 * Same inputs as the reference: input_params_ess ("nu0 dnu chan0 data_path",
 * amber_funcs.c:175-188), <data_path>/GV_data_<R> and <data_path>/sampling
 * (amber_funcs.c:1720-1941), <data_path>/uf_chans.txt when the GV header's
 * flag_key is 1 (amber_funcs.c:2485-2508).  Same outputs: <res_path>/closed_rings
 * and rcount (calCR, amber_funcs.c:406-483) and one file per closed triangle,
 * v1 bsout_final_ra{r1}_rb{r2}_rc{r3}_R{R} = {f64 Ntri, f64 Num, f32 bldnu[nclen²],
 * i32 numdnu[nclen²]} (amber.c:287-304), v2 bsout_final2_… = {f64 1/Ng1²,
 * f32 bldnu, f32 numdnu} (amber_v2.c:295-309).  The constants the reference
 * hard-codes (amber.c:43-54,187 and the ring edges of annular_rings) are
 * optional arguments here whose defaults are the reference's own: v1, nc10 =
 * 383 (amber.c:46) and the 22 annular_rings edges (amber_funcs.c:2022-2062,
 * amber.c:44-45), so `amber_gpu <Rlzn>` runs what `amber <Rlzn>` runs.  Errors
 * keep the reference's behaviour: perror/fprintf + exit.
 *
 * usage: amber_gpu <Rlzn> [v1|v2] [nc10|-] [rings_file|-] [rp_begin] [rp_end] [res_path]
 *                  [input_params_ess] [mixed|fp64]
 *        amber_gpu --default-rings      (print the default ring edges and exit)
 * Under RANK / WORLD_SIZE / LOCAL_RANK (one process per GPU) each process takes its share of
 * the closed triangles (amber_cuda_shard_plan) on GPU LOCAL_RANK and writes their files; rank 0
 * also writes closed_rings and rcount.  The files are those of a single-process run.
 * rings_file: "Nr" then Nr lines "ULow UHigh"; "-" keeps the default.
 */
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>

#include "amber_cuda.h"

static void die(const char *what)
{
    perror(what);
    exit(EXIT_FAILURE);
}

static void check(amber_cuda_ctx *ctx, int rc, const char *what)
{
    if (rc != AMBER_OK) {
        fprintf(stderr, "%s failed (%d): %s\n", what, rc, amber_cuda_last_error(ctx));
        exit(EXIT_FAILURE);
    }
}

/* The reference's ring edges (annular_rings, amber_funcs.c:2022-2062): lower edges on a
 * piecewise-uniform ladder, 0-50 in steps of 5, 50-100 in 10, 100-200 in 20, 200-270 in 35,
 * each ring's upper edge the next ring's lower one, then the first lower edge raised to 1
 * and the last upper edge set to 270.  DEFAULT_NR = 22 is the bin count of amber.c:44-45. */
#define DEFAULT_NR 22
static void default_rings(double *ulow, double *uhigh)
{
    static const int ladder[4][3] = {{0, 50, 5}, {50, 100, 10}, {100, 200, 20}, {200, 270, 35}};
    int n = 0;
    for (int k = 0; k < 4; ++k)
        for (int e = ladder[k][0]; e < ladder[k][1] && n < DEFAULT_NR; e += ladder[k][2]) {
            ulow[n] = e;
            if (n > 0) uhigh[n - 1] = e;
            ++n;
        }
    ulow[0] = 1.0;
    uhigh[DEFAULT_NR - 1] = 270.0;
}

int main(int argc, char **argv)
{
    if (argc == 2 && strcmp(argv[1], "--default-rings") == 0) {
        double lo[DEFAULT_NR], hi[DEFAULT_NR];
        default_rings(lo, hi);
        printf("%d\n", DEFAULT_NR);
        for (int i = 0; i < DEFAULT_NR; ++i) printf("%.17g %.17g\n", lo[i], hi[i]);
        return 0;
    }
    if (argc < 2) {
        printf("Usage: %s <Rlzn> [v1|v2] [nc10|-] [rings_file|-] [rp_begin] [rp_end] [res_path] [input_params_ess] "
               "[mixed|fp64]\n",
               argv[0]);
        return 1;
    }
    const int rlzn = atoi(argv[1]);
    const int v2 = argc > 2 && strcmp(argv[2], "v2") == 0;
    const int nc10 = (argc > 3 && strcmp(argv[3], "-") != 0) ? atoi(argv[3]) : 383;  /* amber.c:46 */
    const char *rings_file = (argc > 4 && strcmp(argv[4], "-") != 0) ? argv[4] : NULL;
    int rp_begin = argc > 5 ? atoi(argv[5]) : 0;
    int rp_end = argc > 6 ? atoi(argv[6]) : -1;
    const char *res_path = argc > 7 ? argv[7] : (v2 ? "results/v2" : "results/v1");
    const char *params = argc > 8 ? argv[8] : "input_params_ess";
    const int precision = (argc > 9 && strcmp(argv[9], "fp64") == 0) ? AMBER_PREC_FP64 : AMBER_PREC_MIXED;

    /* input_params_ess: nu0 dnu chan0 data_path */
    double nu0, dnu, chan0;
    char data_path[512];
    FILE *fp = fopen(params, "r");
    if (!fp) die("Error opening file: input_params_ess");
    if (fscanf(fp, "%lf%lf%lf%511s", &nu0, &dnu, &chan0, data_path) != 4) {
        fprintf(stderr, "input_params_ess: expected nu0 dnu chan0 data_path\n");
        exit(EXIT_FAILURE);
    }
    fclose(fp);

    /* GV_data_<R>: {int64 NN; int64 nc; f64 Du; int32 flag_key} then re/im per cell and channel */
    char path[1024];
    snprintf(path, sizeof(path), "%s/GV_data_%d", data_path, rlzn);
    fp = fopen(path, "rb");
    if (!fp) die("Error opening file: GV_data");
    int64_t NN, nc;
    double Du;
    int32_t flag_key;
    if (fread(&NN, 8, 1, fp) != 1 || fread(&nc, 8, 1, fp) != 1 || fread(&Du, 8, 1, fp) != 1 ||
        fread(&flag_key, 4, 1, fp) != 1) {
        fprintf(stderr, "GV_data: short header\n");
        exit(EXIT_FAILURE);
    }
    /* the gridding stage writes an even NN = 2·ceil(Umax/dU) and Du > 0; the bounds keep the
     * buffer sizes below from wrapping on a file that is not a grid */
    if (NN <= 0 || NN % 2 || NN > (1 << 20) || nc <= 0 || nc > (1 << 20) || !(Du > 0)) {
        fprintf(stderr, "GV_data: bad header (NN %lld, nc %lld, Du %g)\n", (long long)NN, (long long)nc, Du);
        exit(EXIT_FAILURE);
    }
    const size_t ncell = (size_t)NN * (NN / 2 + 1);
    double *re_im = (double *)malloc(sizeof(double) * 2 * ncell * nc);
    double *ntig = (double *)malloc(sizeof(double) * ncell * nc);
    if (!re_im || !ntig) die("malloc");
    if (fread(re_im, sizeof(double), 2 * ncell * nc, fp) != 2 * ncell * nc) {
        fprintf(stderr, "GV_data: truncated grid\n");
        exit(EXIT_FAILURE);
    }
    fclose(fp);
    snprintf(path, sizeof(path), "%s/sampling", data_path);
    fp = fopen(path, "rb");
    if (!fp) die("Error opening file: sampling");
    if (fread(ntig, sizeof(double), ncell * nc, fp) != ncell * nc) {
        fprintf(stderr, "sampling: truncated\n");
        exit(EXIT_FAILURE);
    }
    fclose(fp);

    /* rings: the file's, or the reference's own edges */
    int Nr = DEFAULT_NR;
    double *ulow, *uhigh;
    if (rings_file) {
        fp = fopen(rings_file, "r");
        if (!fp) die("Error opening rings file");
        if (fscanf(fp, "%d", &Nr) != 1 || Nr <= 0) {
            fprintf(stderr, "rings file: bad count\n");
            exit(EXIT_FAILURE);
        }
        ulow = (double *)malloc(sizeof(double) * Nr);
        uhigh = (double *)malloc(sizeof(double) * Nr);
        if (!ulow || !uhigh) die("malloc");
        for (int i = 0; i < Nr; ++i)
            if (fscanf(fp, "%lf %lf", &ulow[i], &uhigh[i]) != 2) {
                fprintf(stderr, "rings file: bad edges\n");
                exit(EXIT_FAILURE);
            }
        fclose(fp);
    } else {
        ulow = (double *)malloc(sizeof(double) * Nr);
        uhigh = (double *)malloc(sizeof(double) * Nr);
        if (!ulow || !uhigh) die("malloc");
        default_rings(ulow, uhigh);
    }

    /* uf_chans.txt when the data are flagged: one integer per unflagged channel */
    int uf_nc = 0;
    int *uf = NULL;
    if (flag_key == 1) {
        snprintf(path, sizeof(path), "%s/uf_chans.txt", data_path);
        fp = fopen(path, "r");
        if (!fp) die("Error opening file");
        int cap = 64, v;
        uf = (int *)malloc(sizeof(int) * cap);
        if (!uf) die("malloc");
        while (fscanf(fp, "%d", &v) == 1) {
            if (uf_nc == cap) {
                int *grown = (int *)realloc(uf, sizeof(int) * (cap *= 2));
                if (!grown) die("realloc");
                uf = grown;
            }
            uf[uf_nc++] = v;
        }
        fclose(fp);
        if (uf_nc == 0) {
            fprintf(stderr, "uf_chans.txt: no channels\n");
            exit(EXIT_FAILURE);
        }
    }

    amber_cuda_opts opts;
    amber_cuda_default_opts(&opts);
    /* one process per GPU under a launcher that sets RANK / WORLD_SIZE / LOCAL_RANK (torchrun,
     * mpirun wrappers): this process's GPU, and its share of the closed triangles below */
    const char *env_rank = getenv("RANK"), *env_world = getenv("WORLD_SIZE"), *env_local = getenv("LOCAL_RANK");
    const int world = env_world ? atoi(env_world) : 1;
    const int rank = (world > 1 && env_rank) ? atoi(env_rank) : 0;
    if (world < 1 || rank < 0 || rank >= world) {
        fprintf(stderr, "RANK=%d outside WORLD_SIZE=%d\n", rank, world);
        exit(EXIT_FAILURE);
    }
    if (world > 1 && env_local) opts.device = atoi(env_local);
    opts.precision = precision;
    amber_cuda_ctx *ctx = NULL;
    int rc = amber_cuda_create(&opts, &ctx);
    if (rc != AMBER_OK) {
        fprintf(stderr, "amber_cuda_create failed (%d): no usable sm_100 GPU\n", rc);
        exit(EXIT_FAILURE);
    }
    check(ctx, amber_cuda_load_grid_packed(ctx, NN, nc, Du, flag_key, re_im, ntig), "load grid");
    check(ctx, amber_cuda_set_rings(ctx, Nr, ulow, uhigh), "set rings");
    check(ctx, amber_cuda_set_channels(ctx, nc10, uf_nc, uf), "set channels");
    printf("NN=%ld, nc=%ld, Du=%lf, Flag=%d, nc10=%d, Unflagged Channels=%d\n", (long)NN, (long)nc, Du, flag_key,
           nc10, uf_nc);

    int rcount = 0;
    check(ctx, amber_cuda_calcr(ctx, 0, &rcount, NULL), "calCR");
    double *rdata = (double *)malloc(sizeof(double) * 4 * (rcount > 0 ? rcount : 1));
    check(ctx, amber_cuda_calcr(ctx, rcount, &rcount, rdata), "calCR");
    mkdir(res_path, 0755);
    if (rank == 0) {  /* the shared files: one writer */
        snprintf(path, sizeof(path), "%s/closed_rings", res_path);
        fp = fopen(path, "wb");
        if (!fp) die("Error opening file: closed_rings");
        fwrite(rdata, sizeof(double), 4 * (size_t)rcount, fp);
        fclose(fp);
        snprintf(path, sizeof(path), "%s/rcount", res_path);
        fp = fopen(path, "w");
        if (!fp) die("Error opening file: rcount");
        fprintf(fp, "%d", rcount);
        fclose(fp);
    }
    printf("Total combinations of rings on a plane forming closed triangle = %d\n", rcount);

    if (rp_end < 0 || rp_end > rcount) rp_end = rcount;
    if (rp_begin < 0) rp_begin = 0;
    const int nrange = rp_end > rp_begin ? rp_end - rp_begin : 0;
    /* this process's triangles of the range: all of them, or its share under the shard plan
     * (amber_cuda_shard_plan: whole triangles, so its files are the single-process ones) */
    int *rps = (int *)malloc(sizeof(int) * (nrange > 0 ? nrange : 1));
    int ntri = 0;
    if (world > 1 && nrange > 0) {
        int *r1s = (int *)malloc(sizeof(int) * nrange), *owner = (int *)malloc(sizeof(int) * nrange);
        long *ngs = (long *)malloc(sizeof(long) * nrange);
        if (!r1s || !owner || !ngs) die("malloc");
        for (int t = 0; t < nrange; ++t) {
            r1s[t] = (int)rdata[4 * (rp_begin + t)];
            ngs[t] = amber_cuda_ng1(ctx, r1s[t]);
        }
        check(ctx, amber_cuda_shard_plan(nrange, r1s, ngs, world, owner), "shard plan");
        for (int t = 0; t < nrange; ++t)
            if (owner[t] == rank) rps[ntri++] = rp_begin + t;
        free(r1s);
        free(owner);
        free(ngs);
    } else {
        for (int t = 0; t < nrange; ++t) rps[ntri++] = rp_begin + t;
    }
    const int nclen = 2 * nc10 + 1;
    const size_t ncsize = (size_t)nclen * nclen;
    int *tri = (int *)malloc(sizeof(int) * 3 * (ntri > 0 ? ntri : 1));
    for (int t = 0; t < ntri; ++t)
        for (int j = 0; j < 3; ++j) tri[3 * t + j] = (int)rdata[4 * rps[t] + j];
    double *bl = (double *)malloc(sizeof(double) * ncsize * (ntri > 0 ? ntri : 1));
    double *nt = v2 ? (double *)malloc(sizeof(double) * ncsize * (ntri > 0 ? ntri : 1)) : NULL;
    int64_t *nd = (int64_t *)malloc(sizeof(int64_t) * ncsize * (ntri > 0 ? ntri : 1));
    if (ntri > 0) check(ctx, amber_cuda_triangles(ctx, ntri, tri, v2, bl, nd, nt), "triangles");
    double products = 0, ms = 0;
    amber_cuda_last_run_stats(ctx, &products, &ms);

    float *fb = (float *)malloc(sizeof(float) * ncsize);
    float *fn = (float *)malloc(sizeof(float) * ncsize);
    int32_t *in = (int32_t *)malloc(sizeof(int32_t) * ncsize);
    for (int t = 0; t < ntri; ++t) {
        const int rp = rps[t], r1 = tri[3 * t], r2 = tri[3 * t + 1], r3 = tri[3 * t + 2];
        const long ng = amber_cuda_ng1(ctx, r1);
        const double gfact = (1. * ng) / (1. * NN), inv = 1.0 / (ng * ng * 1.);
        const double Num = gfact * gfact * rdata[4 * rp + 3];
        for (size_t i = 0; i < ncsize; ++i) fb[i] = (float)bl[t * ncsize + i];
        FILE *fo;
        if (v2) {
            for (size_t i = 0; i < ncsize; ++i) fn[i] = (float)nt[t * ncsize + i];
            snprintf(path, sizeof(path), "%s/bsout_final2_ra%d_rb%d_rc%d_R%d", res_path, r1, r2, r3, rlzn);
            fo = fopen(path, "wb");
            if (!fo) die("fopen");
            fwrite(&inv, sizeof(double), 1, fo);
            if (fwrite(fb, sizeof(float), ncsize, fo) != ncsize) die("fwrite bldnu");
            if (fwrite(fn, sizeof(float), ncsize, fo) != ncsize) die("fwrite numdnu");
        } else {
            for (size_t i = 0; i < ncsize; ++i) {
                if (nd[t * ncsize + i] > INT32_MAX) {
                    fprintf(stderr, "numdnu overflows int32 at lag cell %zu\n", i);
                    exit(EXIT_FAILURE);
                }
                in[i] = (int32_t)nd[t * ncsize + i];
            }
            const double Ntri = Num * inv;
            snprintf(path, sizeof(path), "%s/bsout_final_ra%d_rb%d_rc%d_R%d", res_path, r1, r2, r3, rlzn);
            fo = fopen(path, "wb");
            if (!fo) die("fopen");
            fwrite(&Ntri, sizeof(double), 1, fo);
            fwrite(&Num, sizeof(double), 1, fo);
            if (fwrite(fb, sizeof(float), ncsize, fo) != ncsize) die("fwrite bldnu");
            if (fwrite(in, sizeof(int32_t), ncsize, fo) != ncsize) die("fwrite numdnu");
        }
        fclose(fo);
    }
    printf("AMBER_GPU_JSON {\"triangles\": %d, \"products\": %.17g, \"device_ms\": %.3f, \"rank\": %d, "
           "\"world\": %d}\n",
           ntri, products, ms, rank, world);
    amber_cuda_destroy(ctx);
    return 0;
}
