// fp64_gemm.h -- arguments of the FP64 CUDA-core GEMM (fp64_gemm.cu).
#pragma once
#include <cuda_runtime.h>

namespace asd {

struct Fp64GemmArgs {
    int dropin;           // 1: fused_dgemm semantics; 0: S(q,t) phase epilogue
    long m, n, k;         // C is m x n, contraction over k
    const double *a;      // A(i,k) = a[i*sai + k*sak]
    long sai, sak;
    int a_k_fast;         // 1 when sak == 1 (k is the contiguous axis)
    const double *b;      // B(k,j) = b[k*sbk + j*sbj]
    long sbk, sbj;
    int b_k_fast;
    double alpha;
    // DROPIN
    double *c;            // interleaved re/im, ldc
    const double *q;
    long ldc;
    long m4, n2;          // rows/cols the reference updates
    // PHASE
    const double *mrow, *zcol;       // [m][3], [n][3]
    const double2 *uphase, *wphase;  // [m], [n]
    // both: partial sums, one per block (DROPIN: per block and K block)
    double2 *part;
};

long fp64_gemm_num_parts(const Fp64GemmArgs &p);
cudaError_t launch_fp64_gemm(const Fp64GemmArgs &p, cudaStream_t st);

}  // namespace asd
