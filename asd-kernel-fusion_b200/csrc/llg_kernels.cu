// llg_kernels.cu -- RK4 time stepping of the LLG equation on the GPU, FP64.
//
// Arithmetic contract: every operation is an explicitly rounded FP64
// intrinsic (__dmul_rn, __dadd_rn, __dsub_rn, __ddiv_rn, __dsqrt_rn), in the
// order the reference writes it, so the compiler cannot contract a*b+c into
// an FMA.  With alpha = J2 = h = 0 the trajectory is therefore bit-identical
// to the reference's euler / runge_kutta / renormalisation built with
// -ffp-contract=off (llg_sqt_baseline.c:29-142, :298-309).
#include <cstdlib>

#include "asd_internal.h"

namespace asd {
namespace {

#include "llg_math.cuh"

// One fused RK4 stage, site-major layout.  Thread t handles replica
// f = t % nfile of site t / nfile, so a warp touches 32 consecutive 24-byte
// records (768 contiguous bytes) of each operand.  The combination order
// reproduces runge_kutta's final sum spin + k1/6 + k2/3 + k3/3 + k4/6
// evaluated left to right (llg_sqt_baseline.c:138), carried in acc.
template <int STAGE, bool J2, bool H, bool DAMP>
__global__ void __launch_bounds__(256) llg_stage_kernel(LLGArgs a, const double *__restrict__ y,
                                                        const double *__restrict__ ys,
                                                        double *__restrict__ acc,
                                                        double *__restrict__ out) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long total = a.M * a.nc;
    if (t >= total) return;
    const long site = t / a.nc;
    const int f = a.f0 + (int)(t - site * a.nc);
    const int row = (int)(site / a.N), col = (int)(site - (long)row * a.N);
    const long sstride = 3L * a.nfile;
    const long off = 3L * f;
    const V3 d = llg_rhs<J2, H, DAMP>(ys, sstride, off, a.N, row, col, a);
    const long e = site * sstride + off;
    const double k0 = dm(d.x, a.dt), k1 = dm(d.y, a.dt), k2 = dm(d.z, a.dt);
    if (STAGE == 1) {
        const double y0 = y[e], y1 = y[e + 1], y2 = y[e + 2];
        out[e] = da(y0, half(k0));
        out[e + 1] = da(y1, half(k1));
        out[e + 2] = da(y2, half(k2));
        acc[e] = da(y0, div6(k0));
        acc[e + 1] = da(y1, div6(k1));
        acc[e + 2] = da(y2, div6(k2));
    } else if (STAGE == 2 || STAGE == 3) {
        const double y0 = y[e], y1 = y[e + 1], y2 = y[e + 2];
        if (STAGE == 2) {
            out[e] = da(y0, half(k0));
            out[e + 1] = da(y1, half(k1));
            out[e + 2] = da(y2, half(k2));
        } else {
            out[e] = da(y0, k0);
            out[e + 1] = da(y1, k1);
            out[e + 2] = da(y2, k2);
        }
        acc[e] = da(acc[e], div3(k0));
        acc[e + 1] = da(acc[e + 1], div3(k1));
        acc[e + 2] = da(acc[e + 2], div3(k2));
    } else {
        const double o0 = da(acc[e], div6(k0));
        const double o1 = da(acc[e + 1], div6(k1));
        const double o2 = da(acc[e + 2], div6(k2));
        // llg_sqt_baseline.c:301-308 / llg_sqt_fusion.c:353-360
        const double nrm = __dsqrt_rn(da(da(dm(o0, o0), dm(o1, o1)), dm(o2, o2)));
        out[e] = dq(dm(a.spin_len, o0), nrm);
        out[e + 1] = dq(dm(a.spin_len, o1), nrm);
        out[e + 2] = dq(dm(a.spin_len, o2), nrm);
    }
}

template <int STAGE>
cudaError_t launch_stage_t(const LLGArgs &a, const double *y, const double *ys, double *acc,
                           double *out, cudaStream_t st) {
    if (a.f0 < 0 || a.nc < 1 || a.f0 + a.nc > a.nfile) return cudaErrorInvalidValue;
    const long total = a.M * a.nc;
    const int threads = 256;
    const unsigned blocks = (unsigned)((total + threads - 1) / threads);
    const int sel = (a.use_j2 ? 4 : 0) | (a.use_h ? 2 : 0) | (a.use_damp ? 1 : 0);
#define ASD_STAGE_CASE(S, J, Hh, D)                                                            \
    case S:                                                                                    \
        llg_stage_kernel<STAGE, J, Hh, D><<<blocks, threads, 0, st>>>(a, y, ys, acc, out);     \
        break;
    switch (sel) {
        ASD_STAGE_CASE(0, false, false, false)
        ASD_STAGE_CASE(1, false, false, true)
        ASD_STAGE_CASE(2, false, true, false)
        ASD_STAGE_CASE(3, false, true, true)
        ASD_STAGE_CASE(4, true, false, false)
        ASD_STAGE_CASE(5, true, false, true)
        ASD_STAGE_CASE(6, true, true, false)
        ASD_STAGE_CASE(7, true, true, true)
    }
#undef ASD_STAGE_CASE
    return cudaGetLastError();
}

// ------------------------------------------------ temporally blocked step
// One RK4 step per launch.  A CTA owns a 16 x 16 core of sites for F
// replicas and loads the 24 x 24 patch around it (a halo of 4 sites, one per
// stage) into shared memory.  Stage s then runs on the region within
// distance 4 - s of the core (Chebyshev distance, which also covers the
// diagonal J2 neighbours), so stage 4 produces exactly the core.  Stage
// inputs ping-pong between two shared buffers; the base state and the
// running combination of each (site, replica) stay in the registers of the
// thread that owns it.  Only y is read and only the renormalised core is
// written: 48 bytes of DRAM traffic per site-step instead of 384.  The
// arithmetic per (site, replica) is the stage kernels' (bit-identical).
constexpr int FT = 16;              // core side
constexpr int FH = 4;               // halo = number of stages
constexpr int FP = FT + 2 * FH;     // patch side
constexpr int FR1 = (FT + 6) * (FT + 6);  // sites of the stage-1 region

// Site of the patch for the idx-th entry of the region list: the core in
// row-major order first, then the rings at distance 1, 2, 3.  So the first
// 256, 324, 400, 484 entries are the regions of stages 4, 3, 2, 1.
__device__ __forceinline__ void region_site(int idx, int &r, int &c) {
    if (idx < FT * FT) {
        r = FH + idx / FT;
        c = FH + idx % FT;
        return;
    }
    idx -= FT * FT;
    int d = 1;
    for (; d < 3; ++d) {
        const int cnt = 4 * (FT + 2 * d) - 4;
        if (idx < cnt) break;
        idx -= cnt;
    }
    const int L = FT + 2 * d;
    if (idx < L) { r = FH - d; c = FH - d + idx; return; }
    idx -= L;
    if (idx < L) { r = FH + FT - 1 + d; c = FH - d + idx; return; }
    idx -= L;
    if (idx < L - 2) { r = FH - d + 1 + idx; c = FH - d; return; }
    idx -= L - 2;
    r = FH - d + 1 + idx;
    c = FH + FT - 1 + d;
}

template <int F, int NT, bool J2, bool H, bool DAMP>
// At most 64 registers per thread so that four CTAs share an SM: the stages
// are separated by barriers, and more resident CTAs hide them (measured:
// 0.60 ms per step at 128x128x500 with four CTAs per SM, 0.83 ms with two).
__global__ void __launch_bounds__(NT, 4 * 256 / NT) llg_step_fused_kernel(LLGArgs a, int tiles_x,
                                                            const double *__restrict__ y,
                                                            double *__restrict__ yout) {
    extern __shared__ double fsm[];
    constexpr int SLOT = 3 * F;                      // doubles per patch site
    constexpr int NITEM = (FR1 * F + NT - 1) / NT;   // items owned per thread
    double *bufA = fsm;
    double *bufB = fsm + FP * FP * SLOT;
    const int tile = blockIdx.x;
    const int R0 = (tile / tiles_x) * FT, C0 = (tile % tiles_x) * FT;
    const int f0 = blockIdx.y * F;
    const int N = a.N;
    const long K = 3L * a.nfile;
    const int nf = min(F, a.nfile - f0);  // replicas present in this chunk

    // load the patch (periodic wrap), zero for replicas past nfile
    for (int e = threadIdx.x; e < FP * FP * SLOT; e += NT) {
        const int slot = e / SLOT, w = e - slot * SLOT;
        const int pr = slot / FP, pc = slot - pr * FP;
        const int gr = ((R0 + pr - FH) % N + N) % N;
        const int gc = ((C0 + pc - FH) % N + N) % N;
        double v = 0.0;
        if (w < 3 * nf) v = y[((long)gr * N + gc) * K + 3L * f0 + w];
        bufA[e] = v;
    }
    __syncthreads();

    double yb[NITEM][3], acc[NITEM][3];
    int slot_of[NITEM];
#pragma unroll
    for (int j = 0; j < NITEM; ++j) {
        const int it = threadIdx.x + j * NT;
        slot_of[j] = -1;
        if (it < FR1 * F) {
            int r, c;
            region_site(it / F, r, c);
            slot_of[j] = r * FP + c;
            const double *p = bufA + slot_of[j] * SLOT + (it % F) * 3;
            yb[j][0] = p[0];
            yb[j][1] = p[1];
            yb[j][2] = p[2];
        }
    }
    // The region list covers each stage's sites first (see region_site).
    const int stage_items[4] = {FR1 * F, (FT + 4) * (FT + 4) * F, (FT + 2) * (FT + 2) * F,
                                FT * FT * F};
    double *in = bufA, *out = bufB;
#pragma unroll
    for (int s = 1; s <= 4; ++s) {
        const int lim = stage_items[s - 1];
        // phase 1: every owned item's increment k = dt * f(stage input), all
        // loads from `in` before any store to `out`
        double kv[NITEM][3];
#pragma unroll
        for (int j = 0; j < NITEM; ++j) {
            const int it = threadIdx.x + j * NT;
            const int f = it % F;
            kv[j][0] = kv[j][1] = kv[j][2] = 0.0;
            if (it >= lim || f >= nf) continue;
            const int slot = slot_of[j];
            const V3 d = llg_rhs<J2, H, DAMP>(in, SLOT, 3L * f, FP, slot / FP, slot % FP, a);
            kv[j][0] = dm(d.x, a.dt);
            kv[j][1] = dm(d.y, a.dt);
            kv[j][2] = dm(d.z, a.dt);
        }
        // phase 2: stage combination
#pragma unroll
        for (int j = 0; j < NITEM; ++j) {
            const int it = threadIdx.x + j * NT;
            const int f = it % F;
            if (it >= lim || f >= nf) continue;
            const int slot = slot_of[j];
            const double k0 = kv[j][0], k1 = kv[j][1], k2 = kv[j][2];
            double *o = out + slot * SLOT + 3 * f;
            if (s == 1) {
                o[0] = da(yb[j][0], half(k0));
                o[1] = da(yb[j][1], half(k1));
                o[2] = da(yb[j][2], half(k2));
                acc[j][0] = da(yb[j][0], div6(k0));
                acc[j][1] = da(yb[j][1], div6(k1));
                acc[j][2] = da(yb[j][2], div6(k2));
            } else if (s == 2) {
                o[0] = da(yb[j][0], half(k0));
                o[1] = da(yb[j][1], half(k1));
                o[2] = da(yb[j][2], half(k2));
                acc[j][0] = da(acc[j][0], div3(k0));
                acc[j][1] = da(acc[j][1], div3(k1));
                acc[j][2] = da(acc[j][2], div3(k2));
            } else if (s == 3) {
                o[0] = da(yb[j][0], k0);
                o[1] = da(yb[j][1], k1);
                o[2] = da(yb[j][2], k2);
                acc[j][0] = da(acc[j][0], div3(k0));
                acc[j][1] = da(acc[j][1], div3(k1));
                acc[j][2] = da(acc[j][2], div3(k2));
            } else {
                const double o0 = da(acc[j][0], div6(k0));
                const double o1 = da(acc[j][1], div6(k1));
                const double o2 = da(acc[j][2], div6(k2));
                const double nrm = __dsqrt_rn(da(da(dm(o0, o0), dm(o1, o1)), dm(o2, o2)));
                const int gr = R0 + slot / FP - FH, gc = C0 + slot % FP - FH;
                if (gr < N && gc < N) {
                    double *g = yout + ((long)gr * N + gc) * K + 3L * (f0 + f);
                    g[0] = dq(dm(a.spin_len, o0), nrm);
                    g[1] = dq(dm(a.spin_len, o1), nrm);
                    g[2] = dq(dm(a.spin_len, o2), nrm);
                }
            }
        }
        if (s < 4) {
            __syncthreads();
            double *t = in;
            in = out;
            out = t;
        }
    }
}

template <int F, int NT>
cudaError_t launch_fused_t(const LLGArgs &a, const double *y, double *yout, cudaStream_t st) {
    const int tiles_x = (a.N + FT - 1) / FT;
    dim3 grid((unsigned)(tiles_x * tiles_x), (unsigned)((a.nfile + F - 1) / F));
    if (grid.y > 65535u) return cudaErrorInvalidConfiguration;
    const size_t smem = 2ull * FP * FP * 3 * F * sizeof(double);
    const int sel = (a.use_j2 ? 4 : 0) | (a.use_h ? 2 : 0) | (a.use_damp ? 1 : 0);
    cudaError_t e = cudaSuccess;
#define ASD_FUSED_CASE(S, J, Hh, D)                                                         \
    case S: {                                                                               \
        auto k = llg_step_fused_kernel<F, NT, J, Hh, D>;                                    \
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem); \
        if (e == cudaSuccess) k<<<grid, NT, smem, st>>>(a, tiles_x, y, yout);               \
        break;                                                                              \
    }
    switch (sel) {
        ASD_FUSED_CASE(0, false, false, false)
        ASD_FUSED_CASE(1, false, false, true)
        ASD_FUSED_CASE(2, false, true, false)
        ASD_FUSED_CASE(3, false, true, true)
        ASD_FUSED_CASE(4, true, false, false)
        ASD_FUSED_CASE(5, true, false, true)
        ASD_FUSED_CASE(6, true, true, false)
        ASD_FUSED_CASE(7, true, true, true)
    }
#undef ASD_FUSED_CASE
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

// Tiled transpose between [nfile][M][3] and [M][nfile][3] through shared
// memory: 32 sites x 32 replicas x 3 doubles per block.
template <bool TO_SITEMAJOR>
__global__ void __launch_bounds__(256) transpose_kernel(const double *__restrict__ src,
                                                        double *__restrict__ dst, long M,
                                                        int nfile, int fbeg, int nc) {
    // The AoS side holds replicas [fbeg, fbeg + nc) as [nc][M][3]; the
    // site-major side is the whole [M][nfile][3] array.  lf = local replica.
    __shared__ double tile[32][32 * 3 + 1];
    const long s0 = (long)blockIdx.x * 32;
    const int l0 = blockIdx.y * 32;
    // read
    for (int idx = threadIdx.x; idx < 32 * 96; idx += blockDim.x) {
        const int r = idx / 96, w = idx % 96;
        if (TO_SITEMAJOR) {
            // AoS: for replica l0+r, 96 contiguous doubles of sites s0..s0+31
            const int lf = l0 + r;
            const long s = s0 + w / 3;
            if (lf < nc && s < M) tile[r][w] = src[((long)lf * M + s0) * 3 + w];
        } else {
            // site-major: for site s0+r, 96 contiguous doubles of replicas l0..l0+31
            const long s = s0 + r;
            const int lf = l0 + w / 3;
            if (lf < nc && s < M) tile[r][w] = src[(s * nfile + fbeg + l0) * 3 + w];
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < 32 * 96; idx += blockDim.x) {
        const int r = idx / 96, w = idx % 96;
        const int c = w % 3, q = w / 3;
        if (TO_SITEMAJOR) {
            // write site s0+r, replicas l0..: value from tile[lf-l0][(s-s0)*3+c]
            const long s = s0 + r;
            const int lf = l0 + q;
            if (lf < nc && s < M) dst[(s * nfile + fbeg + lf) * 3 + c] = tile[q][r * 3 + c];
        } else {
            const int lf = l0 + r;
            const long s = s0 + q;
            if (lf < nc && s < M) dst[((long)lf * M + s) * 3 + c] = tile[q][r * 3 + c];
        }
    }
}

// euler on the reference layout: thread t -> site t % M of replica t / M
// (the reference's loop order, llg_sqt_baseline.c:44-48), reference physics.
__global__ void __launch_bounds__(256) euler_aos_kernel(LLGArgs a, const double *__restrict__ y,
                                                        double *__restrict__ d) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.M * a.nfile) return;
    const long f = t / a.M;
    const long site = t - f * a.M;
    const int row = (int)(site / a.N), col = (int)(site - (long)row * a.N);
    const V3 r = llg_rhs<false, false, false>(y, 3, f * a.M * 3, a.N, row, col, a);
    d[t * 3] = r.x;
    d[t * 3 + 1] = r.y;
    d[t * 3 + 2] = r.z;
}

// runge_kutta's element-wise loops (llg_sqt_baseline.c:104-139).
__global__ void rk_pass_kernel(int pass, long n, double dt, const double *__restrict__ spin,
                               double *__restrict__ cur, double *__restrict__ k,
                               const double *__restrict__ k1, const double *__restrict__ k2,
                               const double *__restrict__ k3) {
    const long j = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const double kk = dm(k[j], dt);
    k[j] = kk;
    if (pass == 1 || pass == 2) {
        cur[j] = da(spin[j], half(kk));
    } else if (pass == 3) {
        cur[j] = da(spin[j], kk);
    } else {
        double v = da(spin[j], dq(k1[j], 6.0));
        v = da(v, dq(k2[j], 3.0));
        v = da(v, dq(k3[j], 3.0));
        cur[j] = da(v, dq(kk, 6.0));
    }
}

__global__ void div_check_kernel(const double *__restrict__ x, long n, unsigned long long *bad) {
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const double v = x[i];
        const bool ok3 = __double_as_longlong(div3(v)) == __double_as_longlong(__ddiv_rn(v, 3.0));
        const bool ok6 = __double_as_longlong(div6(v)) == __double_as_longlong(__ddiv_rn(v, 6.0));
        if (!ok3 || !ok6) atomicAdd(bad, 1ull);
    }
}

}  // namespace

cudaError_t launch_div_check(const double *x, long n, unsigned long long *bad, cudaStream_t st) {
    div_check_kernel<<<1184, 256, 0, st>>>(x, n, bad);
    return cudaGetLastError();
}

LLGArgs make_llg_args(const asd_params &p) {
    LLGArgs a;
    a.N = p.N;
    a.nfile = p.nfile;
    a.M = (long)p.N * p.N;
    a.J1 = p.J1;
    a.J2 = p.J2;
    a.hx = p.hx;
    a.hy = p.hy;
    a.hz = p.hz;
    a.alpha = p.alpha;
    a.g = 1.0 / (1.0 + p.alpha * p.alpha);
    a.dt = p.dt;
    a.spin_len = p.spin_len;
    a.use_j2 = p.J2 != 0.0;
    a.use_h = (p.hx != 0.0 || p.hy != 0.0 || p.hz != 0.0);
    a.use_damp = p.alpha != 0.0;
    a.f0 = 0;
    a.nc = p.nfile;
    return a;
}

cudaError_t launch_llg_stage(int stage, const LLGArgs &a, const double *y, const double *ys_in,
                             double *acc, double *ys_out, cudaStream_t st) {
    switch (stage) {
        case 1: return launch_stage_t<1>(a, y, ys_in, acc, ys_out, st);
        case 2: return launch_stage_t<2>(a, y, ys_in, acc, ys_out, st);
        case 3: return launch_stage_t<3>(a, y, ys_in, acc, ys_out, st);
        case 4: return launch_stage_t<4>(a, y, ys_in, acc, ys_out, st);
    }
    return cudaErrorInvalidValue;
}

cudaError_t launch_llg_step_fused(const LLGArgs &a, const double *y, double *yout,
                                  cudaStream_t st) {
    // 2 replicas per CTA, 256 threads (55 KB of shared memory, 4 CTAs per SM)
    return launch_fused_t<2, 256>(a, y, yout, st);
}

cudaError_t launch_aos_to_sitemajor_range(const double *aos, double *sm, long M, int nfile,
                                          int f0, int nc, cudaStream_t st) {
    if (f0 < 0 || nc < 1 || f0 + nc > nfile) return cudaErrorInvalidValue;
    dim3 grid((unsigned)((M + 31) / 32), (unsigned)((nc + 31) / 32));
    transpose_kernel<true><<<grid, 256, 0, st>>>(aos, sm, M, nfile, f0, nc);
    return cudaGetLastError();
}

cudaError_t launch_sitemajor_to_aos_range(const double *sm, double *aos, long M, int nfile,
                                          int f0, int nc, cudaStream_t st) {
    if (f0 < 0 || nc < 1 || f0 + nc > nfile) return cudaErrorInvalidValue;
    dim3 grid((unsigned)((M + 31) / 32), (unsigned)((nc + 31) / 32));
    transpose_kernel<false><<<grid, 256, 0, st>>>(sm, aos, M, nfile, f0, nc);
    return cudaGetLastError();
}

cudaError_t launch_aos_to_sitemajor(const double *aos, double *sm, long M, int nfile,
                                    cudaStream_t st) {
    return launch_aos_to_sitemajor_range(aos, sm, M, nfile, 0, nfile, st);
}

cudaError_t launch_sitemajor_to_aos(const double *sm, double *aos, long M, int nfile,
                                    cudaStream_t st) {
    return launch_sitemajor_to_aos_range(sm, aos, M, nfile, 0, nfile, st);
}

cudaError_t launch_euler_aos(const LLGArgs &a, const double *spin, double *deriv,
                             cudaStream_t st) {
    const long total = a.M * a.nfile;
    euler_aos_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a, spin, deriv);
    return cudaGetLastError();
}

cudaError_t launch_rk_pass(int pass, long n, double dt, const double *spin, double *cur,
                           double *k, const double *k1, const double *k2, const double *k3,
                           cudaStream_t st) {
    rk_pass_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pass, n, dt, spin, cur, k, k1,
                                                                 k2, k3);
    return cudaGetLastError();
}

}  // namespace asd

extern "C" int asd_check_const_division(const double *x, long n, unsigned long long *bad,
                                        void *stream) {
    using namespace asd;
    if (!x || !bad || n < 0) return fail(ASD_ERR_INVALID, "bad argument");
    ASD_CUDA_TRY(launch_div_check(x, n, bad, (cudaStream_t)stream));
    return ASD_OK;
}
