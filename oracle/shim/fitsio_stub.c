/* ORACLE / TEST INFRASTRUCTURE ONLY: CFITSIO stubs (see fitsio.h). */
#include "fitsio.h"

int fits_open_file(fitsfile **f, const char *name, int mode, int *status)
{ (void)f; (void)name; (void)mode; return *status = 104; }
int fits_close_file(fitsfile *f, int *status) { (void)f; return *status = 104; }
int fits_read_keys_lng(fitsfile *f, const char *k, int a, int b, long *v, int *n, int *status)
{ (void)f; (void)k; (void)a; (void)b; (void)v; (void)n; return *status = 104; }
int fits_read_keys_dbl(fitsfile *f, const char *k, int a, int b, double *v, int *n, int *status)
{ (void)f; (void)k; (void)a; (void)b; (void)v; (void)n; return *status = 104; }
int fits_read_subset(fitsfile *f, int t, long *a, long *b, long *c, void *d, void *e, int *g, int *status)
{ (void)f; (void)t; (void)a; (void)b; (void)c; (void)d; (void)e; (void)g; return *status = 104; }
void fits_report_error(FILE *s, int status) { fprintf(s, "cfitsio stub: status %d\n", status); }
