/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Stand-in for the reference's UVFITS reader (3_vcg/read_fits_funcmfs.c:29-127)
 * so that the reference's unmodified gridding stage (3_vcg/main.c +
 * 3_vcg/tgefuncs.c) runs on synthetic visibility records: CFITSIO and UVFITS
 * data are absent here.  It exports the same four calls and the same globals
 * that tgefuncs.c reads (gcount, nstokes, nchan, randpar, data, nu_chan0,
 * del_chan, chan0), filled from a plain binary file instead of a FITS file.
 *
 * File layout (little-endian, written by amber_b200.synth):
 *   char magic[8] = "AMBRVIS1"
 *   int64 gcount, pcount, nstokes, nchan
 *   float nu_chan0, del_chan, chan0, pad
 *   gcount × { float randpar[pcount]; float data[nchan][nstokes][3] }
 * with data[c][s] = (re, im, wt) exactly like a random-groups UVFITS row.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

long gcount, pcount, nstokes, nchan, ncmplx;
float *data;
float *randpar;
float chan0, nu_chan0, del_chan;

static FILE *g_fp;
static long g_nel;
static long g_hdr = 8 + 4 * 8 + 4 * 4;

void printerror(int status)
{
    if (status) {
        fprintf(stderr, "synthetic visibility reader: status %d\n", status);
        exit(status);
    }
}

int read_fits_header(char *in_file)
{
    char magic[8];
    long long h[4];
    float f[4];
    g_fp = fopen(in_file, "rb");
    if (!g_fp) { fprintf(stderr, "unable to open %s\n", in_file); exit(1); }
    if (fread(magic, 1, 8, g_fp) != 8 || memcmp(magic, "AMBRVIS1", 8) != 0) { fprintf(stderr, "bad magic\n"); exit(1); }
    if (fread(h, 8, 4, g_fp) != 4 || fread(f, 4, 4, g_fp) != 4) { fprintf(stderr, "short header\n"); exit(1); }
    gcount = h[0]; pcount = h[1]; nstokes = h[2]; nchan = h[3];
    nu_chan0 = f[0]; del_chan = f[1]; chan0 = f[2];
    ncmplx = 3;
    randpar = (float *)calloc(pcount, sizeof(float));
    g_nel = ncmplx * nstokes * nchan;
    data = (float *)calloc(g_nel, sizeof(float));
    return 0;
}

static long rec_bytes(void) { return (long)sizeof(float) * (pcount + g_nel); }

int read_ranpar(long grp)
{
    fseek(g_fp, g_hdr + (grp - 1) * rec_bytes(), SEEK_SET);
    if (fread(randpar, sizeof(float), pcount, g_fp) != (size_t)pcount) printerror(107);
    return 0;
}

int read_data(long group)
{
    fseek(g_fp, g_hdr + (group - 1) * rec_bytes() + (long)sizeof(float) * pcount, SEEK_SET);
    if (fread(data, sizeof(float), g_nel, g_fp) != (size_t)g_nel) printerror(107);
    return 0;
}

int close_fits(void)
{
    if (g_fp) fclose(g_fp);
    g_fp = NULL;
    return 0;
}
