// sqt_kernels.cu -- the memory-bound pieces around the S(q,t) correlation
// GEMM: replica means, operand splitting, the FP64 phase epilogue of the
// plain path, and the deterministic final reduction.
//
// S(q,t) = (1/M) sum_ij u_i w_j (C_ij - m_i . z_j),  C = (1/nfile) A B^T,
// with u_i = e^{-i q.r_i}, w_j = e^{+i q.r_j} (so u_i w_j is the reference's
// qmat entry e^{-i q.(r_i - r_j)}, gemm/llg_sqt_mkl.c:290-300), m_i the
// replica mean at t (fint_avg, :349-366) and z_j the mean at t = 0
// (zerot_avg, llg_sqt_baseline.c:240-259).
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cmath>

#include "asd_internal.h"

namespace asd {
namespace {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// One warp per site: mean over replicas of the 3 components.
__global__ void __launch_bounds__(256) site_mean_kernel(const double *__restrict__ state, long M,
                                                        int nfile,
                                                        const double2 *__restrict__ phase,
                                                        double *__restrict__ mean,
                                                        float4 *__restrict__ vec4,
                                                        float *__restrict__ vec1) {
    const long site = (long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (site >= M) return;
    const double *p = state + site * 3L * nfile;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int f = lane; f < nfile; f += 32) {
        sx += p[3 * f];
        sy += p[3 * f + 1];
        sz += p[3 * f + 2];
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    sz = warp_sum(sz);
    if (lane == 0) {
        const double mx = sx / nfile, my = sy / nfile, mz = sz / nfile;
        mean[site * 3] = mx;
        mean[site * 3 + 1] = my;
        mean[site * 3 + 2] = mz;
        const double2 ph = phase[site];
        vec4[site] = make_float4((float)mx, (float)my, (float)mz, (float)ph.x);
        vec1[site] = (float)ph.y;
    }
}

// One warp per site: the sum over this context's replicas of the 3
// components (lane l adds replicas l, l + 32, ..., as site_mean_kernel).
__global__ void __launch_bounds__(256) site_sum_kernel(const double *__restrict__ state, long M,
                                                       int nfile, double *__restrict__ sums) {
    const long site = (long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (site >= M) return;
    const double *p = state + site * 3L * nfile;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int f = lane; f < nfile; f += 32) {
        sx += p[3 * f];
        sy += p[3 * f + 1];
        sz += p[3 * f + 2];
    }
    sx = warp_sum(sx);
    sy = warp_sum(sy);
    sz = warp_sum(sz);
    if (lane == 0) {
        sums[site * 3] = sx;
        sums[site * 3 + 1] = sy;
        sums[site * 3 + 2] = sz;
    }
}

// S(q,t) of a replica-sharded ensemble from the all-reduced shard values:
// part = (1/M) sum_ij u_i w_j alpha C_ij over all shards, sums / zsums = the
// ensemble's site sums at t and at the origin.  The connected-part term
// (1/M) sum_ij u_i w_j m_i . z_j factorises as (1/M) sum_c U_c W_c with
// U_c = sum_i u_i m_ic, W_c = sum_j w_j z_jc.  One block, fixed order.
__global__ void __launch_bounds__(1024) shard_finish_kernel(
    long M, double inv_nf, const double *__restrict__ part, const double *__restrict__ sums,
    const double *__restrict__ zsums, const double2 *__restrict__ u,
    const double2 *__restrict__ w, double *__restrict__ out) {
    __shared__ double red[12][1024 / 32];
    double v[12] = {};
    for (long i = threadIdx.x; i < M; i += 1024) {
        const double2 ui = u[i], wi = w[i];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const double m = sums[i * 3 + c] * inv_nf, z = zsums[i * 3 + c] * inv_nf;
            v[4 * c] += ui.x * m;
            v[4 * c + 1] += ui.y * m;
            v[4 * c + 2] += wi.x * z;
            v[4 * c + 3] += wi.y * z;
        }
    }
#pragma unroll
    for (int q = 0; q < 12; ++q) v[q] = warp_sum(v[q]);
    const int lane = threadIdx.x & 31, wid = threadIdx.x / 32;
    if (lane == 0)
#pragma unroll
        for (int q = 0; q < 12; ++q) red[q][wid] = v[q];
    __syncthreads();
    if (threadIdx.x == 0) {
        double t[12];
        for (int q = 0; q < 12; ++q) {
            t[q] = 0.0;
            for (int k = 0; k < 1024 / 32; ++k) t[q] += red[q][k];
        }
        double ore = 0.0, oim = 0.0;
        for (int c = 0; c < 3; ++c) {
            const double ur = t[4 * c], ui = t[4 * c + 1], wr = t[4 * c + 2], wi = t[4 * c + 3];
            ore += ur * wr - ui * wi;
            oim += ur * wi + ui * wr;
        }
        out[0] = part[0] - ore / (double)M;
        out[1] = part[1] - oim / (double)M;
    }
}

// hi = round(x), lo = round(x - hi), each to the operand format.
__device__ __forceinline__ void split_tf32(double x, float &hi, float &lo) {
    uint32_t h, l;
    const float xf = (float)x;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(xf));
    hi = __uint_as_float(h);
    const float rf = (float)(x - (double)hi);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(rf));
    lo = __uint_as_float(l);
}

// Both split kernels convert columns [kbeg, kend) of every row (kbeg and kend
// even; columns K..Kp-1 are the zero padding), one thread per column pair.
__global__ void __launch_bounds__(256) split_tf32_kernel(const double *__restrict__ s, long M,
                                                         int K, int Kp, int kbeg, int kend,
                                                         float2 *__restrict__ hi,
                                                         float2 *__restrict__ lo) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pairs = (kend - kbeg) / 2;
    if (t >= M * pairs) return;
    const long row = t / pairs;
    const int k = kbeg + (int)(t - row * pairs) * 2;
    float2 h = make_float2(0.f, 0.f), l = make_float2(0.f, 0.f);
    if (k < K) split_tf32(s[row * K + k], h.x, l.x);
    if (k + 1 < K) split_tf32(s[row * K + k + 1], h.y, l.y);
    const long o = row * (Kp / 2) + k / 2;
    hi[o] = h;
    lo[o] = l;
}

__global__ void __launch_bounds__(256) split_bf16_kernel(const double *__restrict__ s, long M,
                                                         int K, int Kp, int kbeg, int kend,
                                                         __nv_bfloat162 *__restrict__ hi,
                                                         __nv_bfloat162 *__restrict__ lo) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pairs = (kend - kbeg) / 2;
    if (t >= M * pairs) return;
    const long row = t / pairs;
    const int k = kbeg + (int)(t - row * pairs) * 2;
    double x0 = 0.0, x1 = 0.0;
    if (k < K) x0 = s[row * K + k];
    if (k + 1 < K) x1 = s[row * K + k + 1];
    const __nv_bfloat16 h0 = __double2bfloat16(x0), h1 = __double2bfloat16(x1);
    const __nv_bfloat16 l0 = __double2bfloat16(x0 - (double)__bfloat162float(h0));
    const __nv_bfloat16 l1 = __double2bfloat16(x1 - (double)__bfloat162float(h1));
    const long o = row * (Kp / 2) + k / 2;
    hi[o] = __halves2bfloat162(h0, h1);
    lo[o] = __halves2bfloat162(l0, l1);
}

// FP16 split of scale * x (scale a power of two, so the product is exact):
// hi and lo each round to nearest even, and lo is formed from the exact FP64
// difference.  FP16 has TF32's 11-bit significand, so hi + lo carry 22 bits.
__global__ void __launch_bounds__(256) split_f16_kernel(const double *__restrict__ s, long M,
                                                        int K, int Kp, int kbeg, int kend,
                                                        double scale, __half2 *__restrict__ hi,
                                                        __half2 *__restrict__ lo) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const int pairs = (kend - kbeg) / 2;
    if (t >= M * pairs) return;
    const long row = t / pairs;
    const int k = kbeg + (int)(t - row * pairs) * 2;
    double x0 = 0.0, x1 = 0.0;
    if (k < K) x0 = s[row * K + k] * scale;
    if (k + 1 < K) x1 = s[row * K + k + 1] * scale;
    const __half h0 = __double2half(x0), h1 = __double2half(x1);
    const __half l0 = __double2half(x0 - (double)__half2float(h0));
    const __half l1 = __double2half(x1 - (double)__half2float(h1));
    const long o = row * (Kp / 2) + k / 2;
    hi[o] = __halves2half2(h0, h1);
    lo[o] = __halves2half2(l0, l1);
}


// Separable 2-D DFT of the displacement histogram: T[dr][b] = sum_dc G[dr][dc]
// e^{-2 pi i b dc / N}, then S[a][b] = scale * sum_dr T[dr][b] e^{-2 pi i a dr / N}.
__global__ void grid_dft_rows_kernel(const double *__restrict__ G, int N,
                                     double2 *__restrict__ T) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * N) return;
    const int dr = t / N, b = t % N;
    double re = 0.0, im = 0.0;
    for (int dc = 0; dc < N; ++dc) {
        double sn, cs;
        sincospi(2.0 * (double)((b * dc) % N) / (double)N, &sn, &cs);
        const double g = G[dr * N + dc];
        re += g * cs;
        im -= g * sn;
    }
    T[t] = make_double2(re, im);
}

__global__ void grid_dft_cols_kernel(const double2 *__restrict__ T, int N, double scale,
                                     double *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= N * N) return;
    const int a = t / N, b = t % N;
    double re = 0.0, im = 0.0;
    for (int dr = 0; dr < N; ++dr) {
        double sn, cs;
        sincospi(2.0 * (double)((a * dr) % N) / (double)N, &sn, &cs);
        const double2 v = T[dr * N + b];
        // (v.x + i v.y) (cs - i sn)
        re += v.x * cs + v.y * sn;
        im += v.y * cs - v.x * sn;
    }
    out[2 * t] = re * scale;
    out[2 * t + 1] = im * scale;
}

// Single block, fixed summation order: thread t sums t, t+256, ... then a
// shared-memory tree.
__global__ void __launch_bounds__(256) finalize_kernel(const double2 *__restrict__ part,
                                                       int nparts, double scale,
                                                       double *__restrict__ out) {
    __shared__ double sre[256], sim[256];
    double a = 0.0, b = 0.0;
    for (int k = threadIdx.x; k < nparts; k += 256) {
        a += part[k].x;
        b += part[k].y;
    }
    sre[threadIdx.x] = a;
    sim[threadIdx.x] = b;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sre[threadIdx.x] += sre[threadIdx.x + s];
            sim[threadIdx.x] += sim[threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = sre[0] * scale;
        out[1] = sim[0] * scale;
    }
}

}  // namespace

cudaError_t launch_site_mean(const double *state, long M, int nfile, const double2 *phase,
                             double *mean, float4 *vec4, float *vec1, cudaStream_t st) {
    const unsigned blocks = (unsigned)((M + 7) / 8);
    site_mean_kernel<<<blocks, 256, 0, st>>>(state, M, nfile, phase, mean, vec4, vec1);
    return cudaGetLastError();
}

cudaError_t launch_site_sum(const double *state, long M, int nfile, double *sums,
                            cudaStream_t st) {
    site_sum_kernel<<<(unsigned)((M + 7) / 8), 256, 0, st>>>(state, M, nfile, sums);
    return cudaGetLastError();
}

cudaError_t launch_shard_finish(long M, int nfile_total, const double *part, const double *sums,
                                const double *zsums, const double2 *u, const double2 *w,
                                double *out, cudaStream_t st) {
    shard_finish_kernel<<<1, 1024, 0, st>>>(M, 1.0 / (double)nfile_total, part, sums, zsums, u, w,
                                            out);
    return cudaGetLastError();
}

cudaError_t launch_split_range(int kind, const double *state, long M, int K, int Kp, int kbeg,
                               int kend, void *hi, void *lo, double scale, cudaStream_t st) {
    if (kbeg < 0 || kend > Kp || kbeg >= kend || (kbeg | kend | Kp) & 1 || kind < 1 || kind > 3)
        return cudaErrorInvalidValue;
    const long total = M * ((kend - kbeg) / 2);
    const unsigned blocks = (unsigned)((total + 255) / 256);
    if (kind == 1)
        split_tf32_kernel<<<blocks, 256, 0, st>>>(state, M, K, Kp, kbeg, kend, (float2 *)hi,
                                                  (float2 *)lo);
    else if (kind == 2)
        split_bf16_kernel<<<blocks, 256, 0, st>>>(state, M, K, Kp, kbeg, kend,
                                                  (__nv_bfloat162 *)hi, (__nv_bfloat162 *)lo);
    else
        split_f16_kernel<<<blocks, 256, 0, st>>>(state, M, K, Kp, kbeg, kend, scale,
                                                 (__half2 *)hi, (__half2 *)lo);
    return cudaGetLastError();
}

cudaError_t launch_split(int kind, const double *state, long M, int K, int Kp, void *hi, void *lo,
                         double scale, cudaStream_t st) {
    return launch_split_range(kind, state, M, K, Kp, 0, Kp, hi, lo, scale, st);
}

double split_scale(int kind, double spin_len) {
    if (kind != 3 || !(spin_len > 0.0) || !(spin_len < 1e300)) return 1.0;
    return ldexp(1.0, 12 - ilogb(spin_len));
}




cudaError_t launch_grid_dft(const double *G, int lat_n, double scale, double2 *tmp, double *out,
                            cudaStream_t st) {
    const int n = lat_n * lat_n;
    grid_dft_rows_kernel<<<(n + 127) / 128, 128, 0, st>>>(G, lat_n, tmp);
    grid_dft_cols_kernel<<<(n + 127) / 128, 128, 0, st>>>(tmp, lat_n, scale, out);
    return cudaGetLastError();
}

cudaError_t launch_finalize(const double2 *part, int nparts, double scale, double *out,
                            cudaStream_t st) {
    finalize_kernel<<<1, 256, 0, st>>>(part, nparts, scale, out);
    return cudaGetLastError();
}

}  // namespace asd
