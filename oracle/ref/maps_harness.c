/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Runs the reference's OWN two-point (MAPS) function cl_dnu, compiled
 * unchanged from 4_fbe/amber_funcs.c and 4_fbe/vars.c, the way 4_fbe/maps.c's
 * main drives it (maps.c:90-210).  maps.c itself does not build as shipped (its
 * makefile target compiles a mabs_funcs.c that does not exist, and it defines
 * the globals vars.c also defines), so this harness restates its main with the
 * constants it hard-codes (NB = 15, Umax1 = 500, Umin1 = 1) as parameters:
 * read_inputs_ess → initialize → ReadGVnAC_gridding → normalize_data (the same
 * loops maps.c inlines at 113-139) → cl_dnu for every pair nn1 <= nn2 →
 * results file.  The text file has maps.c's layout (maps.c:197-205); the
 * binary file holds cldnu [NB][nc], numdnu [nc], binu [NB] (f64) and num [NB]
 * (int32) at full precision.  The time of the pair loop (one host thread, as
 * in maps.c) is printed as "MAPS_REF_JSON {...}".
 *
 * usage: ref_maps <Rlzn> <input_params_ess> <NB> <umin> <umax> <text out> <binary out>
 */
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include "fftw3.h"
#include "mabs_funcs.h"
#include "vars.h"

void cl_dnu(int nn1, int nn2, int NB, double umax, double umin, double *usum, double *pksum, int *no);

int main(int argc, char **argv)
{
    if (argc != 8) {
        fprintf(stderr, "usage: %s <Rlzn> <input_params_ess> <NB> <umin> <umax> <text out> <binary out>\n", argv[0]);
        return 1;
    }
    NRi = atoi(argv[1]);
    read_inputs_ess(argv[2]);
    const int NB = atoi(argv[3]);
    const double Umin1 = atof(argv[4]), Umax1 = atof(argv[5]);
    Nr = 1;
    uf_nc = 0;
    initialize();
    ReadGVnAC_gridding();
    normalize_data();

    int *num = (int *)calloc(NB, sizeof(int));
    double *binu = (double *)calloc(NB, sizeof(double));
    double *binps = (double *)calloc(NB, sizeof(double));
    double *cldnu = (double *)calloc((size_t)NB * nc, sizeof(double));
    double *numdnu = (double *)calloc(nc, sizeof(double));
    const double t0 = omp_get_wtime();
    for (int nn1 = 0; nn1 < nc; ++nn1)
        for (int nn2 = nn1; nn2 < nc; ++nn2) {
            cl_dnu(nn1, nn2, NB, Umax1, Umin1, binu, binps, num);
            numdnu[nn2 - nn1] += 1.;
            for (int i = 0; i < NB; ++i) cldnu[(size_t)i * nc + (nn2 - nn1)] += binps[i];
        }
    const double t_pairs = omp_get_wtime() - t0;
    FILE *fp = fopen(argv[6], "w");
    if (!fp) return 1;
    for (int i = 0; i < NB; ++i)
        for (long j = 0; j < nc; ++j)
            fprintf(fp, "%d\t%e\t%ld\t%e\t%e\t%d\n", i, binu[i], j, cldnu[(size_t)i * nc + j], numdnu[j], num[i]);
    fclose(fp);
    fp = fopen(argv[7], "wb");
    if (!fp) return 1;
    fwrite(cldnu, sizeof(double), (size_t)NB * nc, fp);
    fwrite(numdnu, sizeof(double), nc, fp);
    fwrite(binu, sizeof(double), NB, fp);
    fwrite(num, sizeof(int), NB, fp);
    fclose(fp);
    printf("\nMAPS_REF_JSON {\"pairs_s\": %.6f, \"pairs\": %ld}\n", t_pairs, (long)nc * (nc + 1) / 2);
    return 0;
}
