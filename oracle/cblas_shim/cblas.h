/* Minimal CBLAS declarations so that the reference's gemm/llg_sqt_mkl.c, which
 * includes "cblas.h", compiles against the OpenBLAS shared library found in
 * this image (the image ships the library without its header).  Test
 * infrastructure only. */
#ifndef ASD_ORACLE_CBLAS_SHIM_H
#define ASD_ORACLE_CBLAS_SHIM_H
enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
void cblas_dgemm(enum CBLAS_ORDER order, enum CBLAS_TRANSPOSE transa, enum CBLAS_TRANSPOSE transb,
                 int m, int n, int k, double alpha, const double *a, int lda, const double *b,
                 int ldb, double beta, double *c, int ldc);
#endif
