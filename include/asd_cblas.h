/*
 * asd_cblas.h -- libasd_cblas.so, the BLAS symbol of the reference's plain
 * S(q,t) path on the GPU.
 *
 * The reference's gemm program calls cblas_dgemm from MKL or OpenBLAS once
 * per step for the correlation matrix (gemm/llg_sqt_mkl.c:378).  This small
 * library exports that symbol and forwards every call to asd_cblas_dgemm of
 * libasd_b200.so (include/asd_b200.h): link it ahead of the CPU BLAS
 * (gcc ... -lasd_cblas -lopenblas), or load it before the program's BLAS, and
 * the program's GEMM runs on the B200 unchanged.  The parameters are those of
 * CBLAS, with its enumerations passed as int (CblasRowMajor 101,
 * CblasColMajor 102, CblasNoTrans 111, CblasTrans 112, CblasConjTrans 113).
 * As BLAS does, invalid arguments are reported on stderr and the call
 * returns without touching C.  A program that already includes a cblas.h
 * needs no declaration from here.
 */
#ifndef ASD_CBLAS_H
#define ASD_CBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

/* gemm/llg_sqt_mkl.c:378 -- C = alpha op(A) op(B) + beta C. */
void cblas_dgemm(int order, int transa, int transb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb, double beta, double *c,
                 int ldc);

/* Calls of cblas_dgemm this library served in this process (no counterpart in
 * the reference; tests use it to show which BLAS a program reached). */
long asd_cblas_calls(void);

#ifdef __cplusplus
}
#endif
#endif
