/*
 * ORACLE / TEST INFRASTRUCTURE ONLY.
 * CFITSIO stand-in: CFITSIO is not installed here and no UVFITS data exists.
 * The amber side only calls these from dead code (read_uvdata,
 * 4_fbe/amber_funcs.c:1551-1716); every stub returns a nonzero status.
 */
#ifndef AMBER_ORACLE_FITSIO_SHIM_H
#define AMBER_ORACLE_FITSIO_SHIM_H
#include <stdio.h>

typedef struct fitsfile_s fitsfile;

#define READONLY 0
#define TFLOAT 42
#define TDOUBLE 82
#define FLEN_KEYWORD 75
#define FLEN_VALUE 71
#define FLEN_COMMENT 73

int fits_open_file(fitsfile **f, const char *name, int mode, int *status);
int fits_close_file(fitsfile *f, int *status);
int fits_read_keys_lng(fitsfile *f, const char *key, int n0, int nkeys, long *v, int *nfound, int *status);
int fits_read_keys_dbl(fitsfile *f, const char *key, int n0, int nkeys, double *v, int *nfound, int *status);
int fits_read_subset(fitsfile *f, int dtype, long *fp, long *lp, long *inc, void *nulval, void *arr,
                     int *anynul, int *status);
void fits_report_error(FILE *stream, int status);
#endif
