// fp64_gemm.h -- arguments of the GPU fused_dgemm (fp64_gemm.cu).
#pragma once
#include <cuda_runtime.h>

namespace asd {

struct Fp64GemmArgs {
    long m, n, k;         // C is m x n, contraction over k
    const double *a;      // A(i,k) = a[i*sai + k*sak]
    long sai, sak;
    int a_k_fast;         // 1 when sak == 1 (k is the contiguous axis)
    const double *b;      // B(k,j) = b[k*sbk + j*sbj]
    long sbk, sbj;
    int b_k_fast;
    double alpha;
    double *c;            // interleaved re/im, ldc
    const double *q;
    long ldc;
    long m4, n2;          // rows/cols the reference updates
    double2 *part;        // sums of the updated C, one per block and K block
};

long fp64_gemm_num_parts(const Fp64GemmArgs &p);
cudaError_t launch_fp64_gemm(const Fp64GemmArgs &p, cudaStream_t st);

}  // namespace asd
