// fp64_gemm.cu -- the reference's fused_dgemm on the GPU (FP64 CUDA cores),
// for the drop-in entry point (dropin.cu).
//
// Semantics of kernel_fusion/gemm_kernel.h:355-422: alpha folded into A, K in
// blocks of 240, per element a sequential FMA chain over k (the AVX2
// micro-kernel's order, :9-35), then C = fma(q, acc, C) on the interleaved
// re/im layout and the updated values summed once per K block (:39-88).
// Because the per-element arithmetic is the same chain of correctly rounded
// FMAs, C is bit-identical to the reference's.  (S(q,t) in FP64 does not come
// here: it runs on the FP64 tensor cores, dmma_sqt.cu.)
//
// Tile 64 x 64, 256 threads, 4 x 4 results per thread, k staged through
// shared memory 16 at a time (240 = 15 * 16, so K blocks never straddle a
// stage).
#include "asd_internal.h"
#include "fp64_gemm.h"

namespace asd {
namespace {

constexpr int TB = 64;
constexpr int TK = 16;

__device__ __forceinline__ long row_re(long i) { return (i / 4) * 8 + (i % 4); }

// A(i,k) = a[i*sai + k*sak], B(k,j) = b[k*sbk + j*sbj].
__global__ void __launch_bounds__(256) fp64_gemm_kernel(Fp64GemmArgs p) {
    __shared__ double As[TK][TB + 1];
    __shared__ double Bs[TK][TB + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const long i0 = (long)blockIdx.y * TB, j0 = (long)blockIdx.x * TB;
    double acc[4][4];
    const long kblk = 240;
    int kb_index = 0;
    for (long kbeg = 0; kbeg < p.k; kbeg += kblk, ++kb_index) {
        const long kend = min(kbeg + kblk, (long)p.k);
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
        for (long k0 = kbeg; k0 < kend; k0 += TK) {
            const int kcnt = (int)min((long)TK, kend - k0);
            // stage A: 64 rows x 16 k; B: 16 k x 64 cols (4 elements each per thread)
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int idx = threadIdx.x + q * 256;
                int ii, kk;
                if (p.a_k_fast) { kk = idx & 15; ii = idx >> 4; }
                else { ii = idx & 63; kk = idx >> 6; }
                const long gi = i0 + ii, gk = k0 + kk;
                double v = 0.0;
                if (gi < p.m && kk < kcnt) {
                    v = p.a[gi * p.sai + gk * p.sak];
                    v = __dmul_rn(v, p.alpha);  // dgemm_tcopy_4 (:238)
                }
                As[kk][ii] = v;
                int jj, kk2;
                if (p.b_k_fast) { kk2 = idx & 15; jj = idx >> 4; }
                else { jj = idx & 63; kk2 = idx >> 6; }
                const long gj = j0 + jj, gk2 = k0 + kk2;
                double w = 0.0;
                if (gj < p.n && kk2 < kcnt) w = p.b[gk2 * p.sbk + gj * p.sbj];
                Bs[kk2][jj] = w;
            }
            __syncthreads();
            for (int kk = 0; kk < kcnt; ++kk) {
                double av[4], bv[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) av[r] = As[kk][ty + 16 * r];
#pragma unroll
                for (int c = 0; c < 4; ++c) bv[c] = Bs[kk][tx + 16 * c];
#pragma unroll
                for (int r = 0; r < 4; ++r)
#pragma unroll
                    for (int c = 0; c < 4; ++c) acc[r][c] = __fma_rn(av[r], bv[c], acc[r][c]);
            }
            __syncthreads();
        }
        // C = fma(q, acc, C) and the K-block sum, rows < m4, cols < n2 only
        double bre = 0.0, bim = 0.0;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const long i = i0 + ty + 16 * r;
            if (i >= p.m4) continue;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const long j = j0 + tx + 16 * c;
                if (j >= p.n2) continue;
                const long ir = row_re(i) + j * p.ldc;
                const double cr = __fma_rn(p.q[ir], acc[r][c], p.c[ir]);
                const double ci = __fma_rn(p.q[ir + 4], acc[r][c], p.c[ir + 4]);
                p.c[ir] = cr;
                p.c[ir + 4] = ci;
                bre += cr;
                bim += ci;
            }
        }
        // per-block reduction of this K block's sum
        __shared__ double red[2][256];
        red[0][threadIdx.x] = bre;
        red[1][threadIdx.x] = bim;
        __syncthreads();
        for (int s = 128; s > 0; s >>= 1) {
            if (threadIdx.x < s) {
                red[0][threadIdx.x] += red[0][threadIdx.x + s];
                red[1][threadIdx.x] += red[1][threadIdx.x + s];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            const long nblk = (long)gridDim.x * gridDim.y;
            const long b = (long)blockIdx.y * gridDim.x + blockIdx.x;
            p.part[(long)kb_index * nblk + b] = make_double2(red[0][0], red[1][0]);
        }
        __syncthreads();
    }
}

}  // namespace

long fp64_gemm_num_parts(const Fp64GemmArgs &p) {
    const long nbx = (p.n + TB - 1) / TB, nby = (p.m + TB - 1) / TB;
    const long nkb = (p.k + 239) / 240;
    return nbx * nby * nkb;
}

cudaError_t launch_fp64_gemm(const Fp64GemmArgs &p, cudaStream_t st) {
    dim3 grid((unsigned)((p.n + TB - 1) / TB), (unsigned)((p.m + TB - 1) / TB));
    if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
    fp64_gemm_kernel<<<grid, 256, 0, st>>>(p);
    return cudaGetLastError();
}

}  // namespace asd
