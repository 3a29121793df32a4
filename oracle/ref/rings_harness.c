/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Prints the ring edges of the reference's own annular_rings()
 * (4_fbe/amber_funcs.c:2022-2062, compiled unchanged) for Nr = 22, the bin count
 * 4_fbe/amber.c:44-45 and amber_v2.c:44-45 hard-code: "Nr" then Nr lines
 * "ULow UHigh" with 17 significant digits.
 *
 * usage: ref_rings [Nr]
 */
#include <stdio.h>
#include <stdlib.h>
#include "fftw3.h"
#include "mabs_funcs.h"
#include "vars.h"

int main(int argc, char **argv)
{
    Nr = argc > 1 ? atoi(argv[1]) : 22;
    ULow = (double *)calloc(Nr, sizeof(double));
    UHigh = (double *)calloc(Nr, sizeof(double));
    Uavg = (double *)calloc(Nr, sizeof(double));
    if (!ULow || !UHigh || !Uavg) return 1;
    annular_rings();
    printf("%d\n", Nr);
    for (int i = 0; i < Nr; ++i) printf("%.17g %.17g\n", ULow[i], UHigh[i]);
    return 0;
}
