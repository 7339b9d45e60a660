/* cblas_shim.c -- libasd_cblas.so: cblas_dgemm (the BLAS call of the
 * reference's plain path, gemm/llg_sqt_mkl.c:378) forwarded to
 * asd_cblas_dgemm of libasd_b200.so.  Kept apart from libasd_b200.so, so that
 * only a program that asks for it gets a GPU cblas_dgemm. */
#include <stdio.h>

#include "../../include/asd_b200.h"
#include "../../include/asd_cblas.h"

static long g_calls;

void cblas_dgemm(int order, int transa, int transb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb, double beta, double *c,
                 int ldc) {
    __atomic_add_fetch(&g_calls, 1, __ATOMIC_RELAXED);
    if (asd_cblas_dgemm(order, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc) !=
        ASD_OK)
        fprintf(stderr, "libasd_cblas cblas_dgemm: %s\n", asd_last_error());
}

long asd_cblas_calls(void) { return __atomic_load_n(&g_calls, __ATOMIC_RELAXED); }
