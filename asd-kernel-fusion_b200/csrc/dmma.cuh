// dmma.cuh -- FP64 tensor-core MMA (mma.sync m16n8k8 .f64) and the
// fragment layout this library relies on.
//
// One warp computes D(16x8) = A(16x8) * B(8x8) + C(16x8) in FP64.  With
// g = lane / 4 and t = lane % 4 a thread holds
//   A: a0 = A[g][t],   a1 = A[g+8][t],   a2 = A[g][t+4],   a3 = A[g+8][t+4]
//   B: b0 = B[t][g],   b1 = B[t+4][g]
//   C, D: c0 = C[g][2t], c1 = C[g][2t+1], c2 = C[g+8][2t], c3 = C[g+8][2t+1]
// (asd_check_dmma_layout tests exactly this against a host product).
//
// The contraction index k is summed, so any permutation of k applied to A's
// columns and B's rows alike leaves D unchanged.  The GEMMs here use the
// permutation that gives thread t the physical k = 2t and 2t + 1 in place of
// the logical t and t + 4: a0/a2 (and a1/a3, b0/b1) are then two consecutive
// doubles, one 16-byte shared-memory load.
#pragma once
#include <cuda_runtime.h>

namespace asd {
namespace dmma {

__device__ __forceinline__ void mma_m16n8k8(double (&d)[4], const double (&a)[4],
                                            const double (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

}  // namespace dmma
}  // namespace asd
