/*
 * maps_gpu — the MAPS executable (4_fbe/maps.c) on libamber_cuda.
 *
 *   maps_gpu <Rlzn> <GV> [input_params] [NB Umin Umax]
 *
 * As maps.c: <Rlzn> selects <data_path>/GV_data_<Rlzn>; <GV> is read and not
 * used (maps.c:68-69); the parameters file (default "input_params", read as
 * read_inputs does, amber_funcs.c:159-173: "NN Du nu0 dnu chan0 nc data_path")
 * gives data_path, and the grid size, channel count and Du come from the GV
 * file's header (initialize, amber_funcs.c:1720-1745).  The grid is normalised
 * (maps.c:113-139) and C_l(Δν) is computed for every channel pair with maps.c's
 * bins (NB = 15 from Umin1 = 1 to Umax1 = 500, maps.c:161-163; the optional
 * arguments override them) by amber_cuda_cl_dnu, whose sums are bit-identical
 * to the reference's cl_dnu loop.  The result goes to results/cldnu in maps.c's
 * layout (maps.c:195-206): one line "bin binu Δ cldnu numdnu num" per bin and Δ.
 *
 * A machine-readable summary line "MAPS_GPU_JSON {...}" goes to stdout.
 */
#include <errno.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "amber_cuda.h"

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void die(const char *what)
{
    perror(what);
    exit(EXIT_FAILURE);
}

int main(int argc, char *argv[])
{
    if (argc != 3 && argc != 4 && argc != 7) {
        printf("Usage: %s <Rlzn> <GV> [input_params] [NB Umin Umax]\n", argv[0]);
        return 1;
    }
    const int rlzn = atoi(argv[1]);
    const char *params = argc >= 4 ? argv[3] : "input_params";
    int NB = 15;
    double umin = 1., umax = 500.;
    if (argc == 7) {
        NB = atoi(argv[4]);
        umin = atof(argv[5]);
        umax = atof(argv[6]);
    }
    long NN_in = 0, nc_in = 0;
    double Du_in = 0, nu0 = 0, dnu = 0, chan0 = 0;
    char data_path[512];
    FILE *fp = fopen(params, "r");
    if (!fp) die("Error opening file: input_params");
    if (fscanf(fp, "%ld%lf%lf%lf%lf%ld%511s", &NN_in, &Du_in, &nu0, &dnu, &chan0, &nc_in, data_path) != 7) {
        fprintf(stderr, "input_params: expected NN Du nu0 dnu chan0 nc data_path\n");
        return 1;
    }
    fclose(fp);

    const double t0 = now_s();
    char path[1100];
    snprintf(path, sizeof(path), "%s/GV_data_%d", data_path, rlzn);
    fp = fopen(path, "rb");
    if (!fp) die("Error opening file: GV_data");
    int64_t NN = 0, nc = 0;
    double Du = 0;
    int32_t flag_key = 0;
    if (fread(&NN, 8, 1, fp) != 1 || fread(&nc, 8, 1, fp) != 1 || fread(&Du, 8, 1, fp) != 1 ||
        fread(&flag_key, 4, 1, fp) != 1 || NN <= 0 || NN % 2 || NN > (1 << 20) || nc <= 0 || nc > (1 << 20) ||
        !(Du > 0)) {
        fprintf(stderr, "GV_data: bad header\n");
        return 1;
    }
    const size_t cells = (size_t)NN * (size_t)(NN / 2 + 1) * (size_t)nc;
    double *re_im = (double *)malloc(sizeof(double) * 2 * cells);
    double *ntig = (double *)malloc(sizeof(double) * cells);
    if (!re_im || !ntig) {
        fprintf(stderr, "out of host memory\n");
        return 1;
    }
    if (fread(re_im, sizeof(double), 2 * cells, fp) != 2 * cells) {
        fprintf(stderr, "GV_data: truncated grid\n");
        return 1;
    }
    fclose(fp);
    snprintf(path, sizeof(path), "%s/sampling", data_path);
    fp = fopen(path, "rb");
    if (!fp) die("Error opening file: sampling");
    if (fread(ntig, sizeof(double), cells, fp) != cells) {
        fprintf(stderr, "sampling: truncated\n");
        return 1;
    }
    fclose(fp);
    const double t_read = now_s() - t0;

    amber_cuda_opts o;
    amber_cuda_default_opts(&o);
    amber_cuda_ctx *ctx = NULL;
    if (amber_cuda_create(&o, &ctx) != AMBER_OK) {
        fprintf(stderr, "amber_cuda_create failed (an sm_100 GPU is required)\n");
        return 1;
    }
    double *cldnu = (double *)malloc(sizeof(double) * (size_t)NB * nc);
    double *numdnu = (double *)malloc(sizeof(double) * nc);
    double *binu = (double *)malloc(sizeof(double) * NB);
    int *num = (int *)malloc(sizeof(int) * NB);
    if (!cldnu || !numdnu || !binu || !num) {
        fprintf(stderr, "out of host memory\n");
        return 1;
    }
    const double t1 = now_s();
    int rc = amber_cuda_load_grid_packed(ctx, NN, nc, Du, flag_key, re_im, ntig);
    if (rc == AMBER_OK) rc = amber_cuda_cl_dnu(ctx, NB, umin, umax, cldnu, numdnu, binu, num);
    const double t_gpu = now_s() - t1;
    if (rc != AMBER_OK) {
        fprintf(stderr, "MAPS failed (%d): %s\n", rc, amber_cuda_last_error(ctx));
        amber_cuda_destroy(ctx);
        return 1;
    }
    amber_cuda_destroy(ctx);

    if (mkdir("results", 0755) != 0 && errno != EEXIST) die("results");
    fp = fopen("results/cldnu", "w");
    if (!fp) die("results/cldnu");
    for (int i = 0; i < NB; ++i)
        for (long j = 0; j < nc; ++j)
            fprintf(fp, "%d\t%e\t%ld\t%e\t%e\t%d\n", i, binu[i], j, cldnu[(size_t)i * nc + j], numdnu[j], num[i]);
    if (fclose(fp) != 0) die("results/cldnu");
    printf("MAPS_GPU_JSON {\"NN\": %ld, \"nc\": %ld, \"NB\": %d, \"pairs\": %ld, \"read_s\": %.6f, \"gpu_s\": %.6f}\n",
           (long)NN, (long)nc, NB, (long)(nc * (nc + 1) / 2), t_read, t_gpu);
    free(re_im);
    free(ntig);
    free(cldnu);
    free(numdnu);
    free(binu);
    free(num);
    return 0;
}
