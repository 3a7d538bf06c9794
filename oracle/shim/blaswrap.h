/*
 * Stand-in for the blaswrap header used by the wbfmm reference sources.
 * Only the routines the reference calls are declared; they are implemented
 * as plain loops in glib_shim.c.  Test infrastructure only.
 */
#ifndef WBFMM_ORACLE_BLASWRAP_SHIM_H
#define WBFMM_ORACLE_BLASWRAP_SHIM_H

void blaswrap_daxpy(int n, double a, double *x, int incx, double *y, int incy);
void blaswrap_saxpy(int n, float a, float *x, int incx, float *y, int incy);
void zgemm_(const char *ta, const char *tb, int *m, int *n, int *k,
            double *al, double *A, int *lda, double *B, int *ldb,
            double *bt, double *C, int *ldc);
void cgemm_(const char *ta, const char *tb, int *m, int *n, int *k,
            float *al, float *A, int *lda, float *B, int *ldb,
            float *bt, float *C, int *ldc);

#endif
