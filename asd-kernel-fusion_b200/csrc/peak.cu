// peak.cu -- measured FP64 throughput of the GPU, the denominators of the
// FP64 roofline fractions (the one-launch RK4 step is bound by FP64 issue on
// the CUDA cores, the plain S(q,t) GEMM by the FP64 tensor cores), and the
// check of the FP64 MMA fragment layout (dmma.cuh).  Diagnostics; no
// counterpart in the reference.
#include <cuda_runtime.h>

#include "asd_internal.h"
#include "dmma.cuh"

namespace asd {
namespace {

constexpr int kChains = 8;     // independent FMA chains per thread
constexpr int kFmaIters = 16384;
constexpr int kMmaTiles = 16;  // independent accumulator tiles per warp
constexpr int kMmaIters = 256;

// Where the peak kernels would store a result that cannot occur: the stores
// keep the compiler from dropping the arithmetic.
__device__ double g_peak_sink[1024];

// kChains independent chains x = fma(x, a, b) per thread; a < 1 keeps x
// bounded.  The result is stored only when it is impossible, so the compiler
// keeps every FMA and nothing is written in practice.
__global__ void __launch_bounds__(256) fma_peak_kernel(double a, double b) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (double)(threadIdx.x + c);
#pragma unroll 1
    for (int it = 0; it < kFmaIters; it += 8) {
#pragma unroll
        for (int u = 0; u < 8; ++u)
#pragma unroll
            for (int c = 0; c < kChains; ++c) x[c] = __fma_rn(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == -1.2345e300) g_peak_sink[blockIdx.x & 1023] = s;
}

// kMmaTiles independent m16n8k8 accumulators per warp, the operands constant.
__global__ void __launch_bounds__(256) dmma_peak_kernel() {
    const int lane = threadIdx.x & 31;
    double a[4], b[2], d[kMmaTiles][4];
#pragma unroll
    for (int e = 0; e < 4; ++e) a[e] = 1e-3 * (lane + e);
    b[0] = 1e-3 * lane;
    b[1] = -1e-3 * lane;
#pragma unroll
    for (int t = 0; t < kMmaTiles; ++t)
#pragma unroll
        for (int e = 0; e < 4; ++e) d[t][e] = 0.0;
#pragma unroll 1
    for (int it = 0; it < kMmaIters; ++it)
#pragma unroll
        for (int t = 0; t < kMmaTiles; ++t) dmma::mma_m16n8k8(d[t], a, b);
    double s = 0.0;
#pragma unroll
    for (int t = 0; t < kMmaTiles; ++t) s += d[t][0] + d[t][1] + d[t][2] + d[t][3];
    if (s == -1.2345e300) g_peak_sink[blockIdx.x & 1023] = s;
}

// One warp: D = A * B with A[16][8] and B[8][8] row-major in global memory,
// fragments loaded per the layout stated in dmma.cuh, D[16][8] row-major.
__global__ void dmma_layout_kernel(const double *A, const double *B, double *D) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    double a[4] = {A[g * 8 + t], A[(g + 8) * 8 + t], A[g * 8 + t + 4], A[(g + 8) * 8 + t + 4]};
    double b[2] = {B[t * 8 + g], B[(t + 4) * 8 + g]};
    double d[4] = {0.0, 0.0, 0.0, 0.0};
    dmma::mma_m16n8k8(d, a, b);
    D[g * 8 + 2 * t] = d[0];
    D[g * 8 + 2 * t + 1] = d[1];
    D[(g + 8) * 8 + 2 * t] = d[2];
    D[(g + 8) * 8 + 2 * t + 1] = d[3];
}

}  // namespace
}  // namespace asd

extern "C" int asd_measure_fp64_peak(int which, double *tflops, double *ms, void *stream) {
    using namespace asd;
    if (!tflops || !ms || (which != 0 && which != 1))
        return fail(ASD_ERR_INVALID, "which must be 0 (FMA) or 1 (DMMA), outputs non-NULL");
    int dev = 0, sms = 0;
    ASD_CUDA_TRY(cudaGetDevice(&dev));
    ASD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaStream_t st = (cudaStream_t)stream;
    const int blocks = sms * 4;  // 32 warps per SM
    cudaEvent_t e0, e1;
    ASD_CUDA_TRY(cudaEventCreate(&e0));
    ASD_CUDA_TRY(cudaEventCreate(&e1));
    double flops = 0.0;
    cudaError_t err = cudaSuccess;
    for (int rep = 0; rep < 2 && err == cudaSuccess; ++rep) {  // the first launch warms up
        cudaEventRecord(e0, st);
        if (which == 0) {
            fma_peak_kernel<<<blocks, 256, 0, st>>>(0.999999, 1e-7);
            flops = 2.0 * kChains * kFmaIters * 256.0 * blocks;
        } else {
            dmma_peak_kernel<<<blocks, 256, 0, st>>>();
            flops = 2.0 * 16 * 8 * 8 * (double)kMmaTiles * kMmaIters * 8.0 * blocks;
        }
        cudaEventRecord(e1, st);
        err = cudaGetLastError();
        if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    }
    float t = 0.f;
    if (err == cudaSuccess) err = cudaEventElapsedTime(&t, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (err != cudaSuccess) return cuda_fail(err, "fp64 peak kernel");
    *ms = t;
    *tflops = flops / (t * 1e-3) / 1e12;
    return ASD_OK;
}

extern "C" int asd_check_dmma_layout(const double *A, const double *B, double *D, void *stream) {
    using namespace asd;
    if (!A || !B || !D) return fail(ASD_ERR_INVALID, "NULL argument");
    dmma_layout_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(A, B, D);
    ASD_CUDA_TRY(cudaGetLastError());
    return ASD_OK;
}
