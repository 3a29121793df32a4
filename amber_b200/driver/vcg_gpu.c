/*
 * vcg_gpu — the gridding stage's executable (3_vcg/main.c:13-77) on libamber_cuda.
 *
 *   vcg_gpu <input visibilities> <input parameters file> <output GV file>
 *           <flagging 0|1> <collapse 0|1> <want sampling file 0|1> <output sampling file>
 *
 * Same arguments and the same output files as the reference:
 *   - parameters file: "nc Umax FWHM f" (read_inputs, 3_vcg/tgefuncs.c:30-38;
 *     f is read and not used by the gridding);
 *   - grid size as initialize_gridding (tgefuncs.c:302-312):
 *     θ0 = 0.6·FWHM·π/(180·60), dU = √(ln 2)/(π·θ0), Ng = ⌈Umax/dU⌉, NN = 2·Ng;
 *   - flagging 1 grids channels with wt > 0 (group_loop_gridding, 377-505),
 *     0 every channel (group_loop_gridding_without_flag, 511-621);
 *   - collapse 1 sums groups of 4 channels (collapse_channels, 816-838; main.c:31);
 *   - GV file (WriteGVnAC_gridding 628-690 / WriteGVnAC_coll 693-724):
 *     int64 NN, int64 nc, f64 dU, int32 flag_key, then for every cell
 *     (ii < NN, jj < NN/2+1) and channel f64 re, f64 im;
 *   - sampling file (Write_NTiG 728-748 / Write_NTiG_coll 752-770): f64 count
 *     per cell and channel, same order, no header.
 * One difference: a flagging or collapse key other than 0 or 1 is an error here
 * (the reference prints a warning and writes an all-zero grid or no GV file).
 *
 * The visibilities come through a reader interface (vis_reader).  UVFITS and
 * CFITSIO are absent from this build, so the reader built in parses the
 * synthetic random-groups file "AMBRVIS1" (int64 gcount, pcount, nstokes,
 * nchan; float nu_chan0, del_chan, chan0, pad; then per group float
 * randpar[pcount] and float data[nchan][nstokes][3] = (re, im, wt)); a UVFITS
 * reader (read_fits_header / read_ranpar / read_data of
 * 3_vcg/read_fits_funcmfs.c) fills the same struct.  The first nc channels of
 * every record are gridded, as the reference's loop walks them.
 *
 * A machine-readable summary line "VCG_GPU_JSON {...}" goes to stdout.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "amber_cuda.h"

typedef struct vis_reader {
    long gcount, pcount, nstokes, nchan;
    float nu_chan0, del_chan, chan0;
    void *state;
    /* every record: randpar [gcount][pcount], data [gcount][nchan][nstokes][3]; 0 on success */
    int (*read_all)(struct vis_reader *r, float *randpar, float *data);
    void (*close)(struct vis_reader *r);
} vis_reader;

static int synth_read_all(vis_reader *r, float *randpar, float *data)
{
    FILE *fp = (FILE *)r->state;
    const long nel = r->nchan * r->nstokes * 3;
    for (long g = 0; g < r->gcount; ++g) {
        if (fread(randpar + g * r->pcount, sizeof(float), (size_t)r->pcount, fp) != (size_t)r->pcount) return -1;
        if (fread(data + g * nel, sizeof(float), (size_t)nel, fp) != (size_t)nel) return -1;
    }
    return 0;
}

static void synth_close(vis_reader *r)
{
    if (r->state) fclose((FILE *)r->state);
    r->state = NULL;
}

static int open_synthetic(const char *path, vis_reader *r)
{
    FILE *fp = fopen(path, "rb");
    if (!fp) return -1;
    char magic[8];
    int64_t h[4];
    float f[4];
    /* records, random parameters, Stokes and channels; the upper bounds keep every buffer size
     * below 2^56 bytes, so nothing computed from them wraps */
    if (fread(magic, 1, 8, fp) != 8 || memcmp(magic, "AMBRVIS1", 8) != 0 || fread(h, 8, 4, fp) != 4 ||
        fread(f, 4, 4, fp) != 4 || h[0] < 0 || h[0] > ((int64_t)1 << 32) || h[1] < 2 || h[1] > 64 || h[2] < 1 ||
        h[2] > 16 || h[3] < 1 || h[3] > (1 << 16)) {
        fclose(fp);
        return -2;
    }
    r->gcount = (long)h[0];
    r->pcount = (long)h[1];
    r->nstokes = (long)h[2];
    r->nchan = (long)h[3];
    r->nu_chan0 = f[0];
    r->del_chan = f[1];
    r->chan0 = f[2];
    r->state = fp;
    r->read_all = synth_read_all;
    r->close = synth_close;
    return 0;
}

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static int write_all(const char *path, const void *head, size_t head_bytes, const double *v, size_t n)
{
    FILE *fp = fopen(path, "wb");
    if (!fp) return -1;
    int ok = (!head_bytes || fwrite(head, 1, head_bytes, fp) == head_bytes) && fwrite(v, sizeof(double), n, fp) == n;
    return (fclose(fp) == 0 && ok) ? 0 : -1;
}

int main(int argc, char *argv[])
{
    if (argc != 8) {
        printf("Usage: %s <input visibilities> <input parameters file> <output GV file> <flagging?> <Collapse?> "
               "<want sampling_fle?> <output sampling_file>\n",
               argv[0]);
        return 1;
    }
    const char *vis_path = argv[1], *param_path = argv[2], *gv_path = argv[3], *ntig_path = argv[7];
    const int flag_key = atoi(argv[4]), coll_key = atoi(argv[5]), key_ntig = atoi(argv[6]);
    if ((flag_key != 0 && flag_key != 1) || (coll_key != 0 && coll_key != 1)) {
        fprintf(stderr, "flagging and collapse keys are 0 or 1\n");
        return 1;
    }
    const long n_collapse = coll_key ? 4 : 1;

    int nc = 0;
    double Umax = 0, FWHM = 0, f = 0;
    FILE *pf = fopen(param_path, "r");
    if (!pf || fscanf(pf, "%d%lf%lf%lf", &nc, &Umax, &FWHM, &f) != 4) {
        fprintf(stderr, "cannot read nc Umax FWHM f from %s\n", param_path);
        return 1;
    }
    fclose(pf);
    const double theta_0 = 0.6 * FWHM * M_PI / (180. * 60.);
    const double dU = sqrt(log(2)) / (M_PI * theta_0);
    const int Ng = (int)ceil(Umax / dU);
    const long NN = (long)2 * Ng;
    if (nc <= 0 || NN <= 0) {
        fprintf(stderr, "bad parameters: nc=%d NN=%ld\n", nc, NN);
        return 1;
    }

    vis_reader rd;
    memset(&rd, 0, sizeof(rd));
    int st = open_synthetic(vis_path, &rd);
    if (st) {
        fprintf(stderr, "%s: %s\n", vis_path, st == -1 ? "cannot open" : "not a visibility file");
        return 1;
    }
    if (nc > rd.nchan) {
        fprintf(stderr, "nc=%d channels asked for, the file holds %ld\n", nc, rd.nchan);
        rd.close(&rd);
        return 1;
    }
    const double t0 = now_s();
    const long G = rd.gcount, nel = rd.nchan * rd.nstokes * 3;
    float *randpar = (float *)malloc(sizeof(float) * (size_t)(G > 0 ? G : 1) * rd.pcount);
    float *data = (float *)malloc(sizeof(float) * (size_t)(G > 0 ? G : 1) * nel);
    if (!randpar || !data || rd.read_all(&rd, randpar, data)) {
        fprintf(stderr, "%s: short read\n", vis_path);
        return 1;
    }
    rd.close(&rd);
    if (rd.nchan != nc) {  // keep the first nc channels of each record, in place
        const long keep = (long)nc * rd.nstokes * 3;
        for (long g = 0; g < G; ++g) memmove(data + g * keep, data + g * nel, sizeof(float) * keep);
    }
    const double t_read = now_s() - t0;

    amber_cuda_opts o;
    amber_cuda_default_opts(&o);
    amber_cuda_ctx *ctx = NULL;
    if (amber_cuda_create(&o, &ctx) != AMBER_OK) {
        fprintf(stderr, "amber_cuda_create failed (an sm_100 GPU is required)\n");
        return 1;
    }
    const long H = NN / 2 + 1, ncoll = nc / n_collapse;
    const size_t ncells = (size_t)NN * H * ncoll;
    double *re_im = (double *)malloc(sizeof(double) * 2 * ncells);
    double *ntig = (double *)malloc(sizeof(double) * ncells);
    if (!re_im || !ntig) {
        fprintf(stderr, "out of host memory for a %ld x %ld x %ld grid\n", NN, H, ncoll);
        return 1;
    }
    const double t1 = now_s();
    int rc = amber_cuda_grid_vis_collapsed(ctx, NN, nc, dU, Umax, rd.nu_chan0, flag_key, G, rd.pcount, rd.nstokes,
                                           randpar, data, n_collapse, re_im, ntig);
    const double t_grid = now_s() - t1;
    if (rc != AMBER_OK) {
        fprintf(stderr, "gridding failed (%d): %s\n", rc, amber_cuda_last_error(ctx));
        amber_cuda_destroy(ctx);
        return 1;
    }
    amber_cuda_destroy(ctx);

    const double t2 = now_s();
    unsigned char head[28];
    const int64_t nn64 = NN, nc64 = ncoll;
    const int32_t fk = flag_key;
    memcpy(head, &nn64, 8);
    memcpy(head + 8, &nc64, 8);
    memcpy(head + 16, &dU, 8);
    memcpy(head + 24, &fk, 4);
    if (write_all(gv_path, head, sizeof(head), re_im, 2 * ncells)) {
        perror(gv_path);
        return 1;
    }
    if (key_ntig == 1 && write_all(ntig_path, NULL, 0, ntig, ncells)) {
        perror(ntig_path);
        return 1;
    }
    const double t_write = now_s() - t2;
    printf("VCG_GPU_JSON {\"NN\": %ld, \"nc\": %d, \"nc_out\": %ld, \"dU\": %.17g, \"records\": %ld, "
           "\"read_s\": %.6f, \"grid_s\": %.6f, \"write_s\": %.6f}\n",
           NN, nc, ncoll, dU, G, t_read, t_grid, t_write);
    free(randpar);
    free(data);
    free(re_im);
    free(ntig);
    return 0;
}
