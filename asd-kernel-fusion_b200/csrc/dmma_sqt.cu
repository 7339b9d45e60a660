// dmma_sqt.cu -- the plain FP64 S(q,t) path: one FP64 tensor-core GEMM
// (mma.sync m16n8k8 .f64, dmma.cuh) whose epilogue applies the connected-part
// subtraction, the phase and the reduction, so that no C matrix exists.
//
// The reference's plain path is cblas_dgemm of the whole (N^2 x N^2)
// correlation matrix followed by three sweeps over it: the outer-product
// subtraction, the phase product and the sum (gemm/llg_sqt_mkl.c:378-423).
// Here C_ij = alpha * sum_k A_ik B_jk stays in registers: the phase factorises
// as u_i w_j and the outer term is m_i . z_j, so the epilogue needs only
// per-row and per-column vectors, and each CTA leaves one complex partial:
//   part[tile] = sum_{i,j in tile} u_i w_j (alpha C_ij - m_i . z_j)
// (or, for the error scale of S(q,t), sum_{i,j in tile} |alpha C_ij - m_i . z_j|).
// The q-grid epilogue instead leaves, per tile, the sums of
// alpha C_ij - m_i . z_j along each diagonal i - j of the tile, split by
// whether the lattice column of j wraps around (qgrid.cu bins them by
// displacement).  Every sum runs in a fixed order: results repeat bit for bit.
//
// The same main loop with a store epilogue is the plain product behind the
// cblas_dgemm drop-in (C = alpha A B^T + beta C, A [M][K], B [MB][K]).
//
// Operands: A = the state at t, B = the origin, both site-major [M][K] FP64
// (K = 3 * nfile contiguous), i.e. the GEMM is C = A B^T with both operands
// K-major.  Tiles of 128 x 128, K staged 32 at a time through a 3-deep
// cp.async pipeline (16-byte copies when K is even, 8-byte ones otherwise;
// zero fill past M and K); 8 warps of 64 x 32, each a 4 x 4 grid of
// m16n8k8 accumulators (64 FP64 registers).  Shared-memory rows are 256 bytes
// (32 doubles) with the 16-byte chunks of odd rows XOR-ed by 4 (a 64-byte
// shift), so that the 16-byte fragment loads of a quarter warp (two rows) fall
// into different banks.  (K stages of 16 in a 4-deep pipeline took 1.6 %
// longer at 256x256x1000; the k order of every accumulator, and so the result,
// is the same bit for bit.)
#include <cuda_runtime.h>

#include "asd_internal.h"
#include "dmma.cuh"

namespace asd {
namespace {

constexpr int BM = 128, BN = 128, BK = 32, STAGES = 3, THREADS = 256;
constexpr int GROUP_M = 16;  // row tiles per raster group (A bands stay in L2)
constexpr int TILE_DOUBLES = BM * BK;          // one operand tile of one stage
constexpr int STAGE_DOUBLES = (BM + BN) * BK;  // 8192 doubles = 64 KB
constexpr int PIPE_BYTES = STAGES * STAGE_DOUBLES * 8;
constexpr int TSTRIDE = BN + 1;  // q grid: epilogue tile row stride (doubles)
constexpr int GRID_SMEM = BM * TSTRIDE * 8;
constexpr int EPI_PHASE = 0, EPI_GRID = 1, EPI_STORE = 2;
constexpr int KCH = BK / 2;  // 16-byte chunks per shared-memory row
constexpr int LOG_KCH = 4;
static_assert(KCH == (1 << LOG_KCH), "chunks per row");

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
// Offset (doubles) of the 16-byte chunk ch (0..7) of row r in a 16-double row.
__device__ __forceinline__ int chunk_off(int r, int ch) { return r * BK + ((ch ^ ((r & 1) << 2)) << 1); }

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src, int src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_u32(dst)), "l"(src),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void tile_coords(int tile, int num_m, int num_n, int &mb, int &nb) {
    const int per_group = GROUP_M * num_n;
    const int group = tile / per_group;
    const int first_m = group * GROUP_M;
    const int gsz = min(GROUP_M, num_m - first_m);
    const int r = tile - group * per_group;
    mb = first_m + r % gsz;
    nb = r / gsz;
}

// Copies rows [row0, row0 + 128) x k [k0, k0 + 16) of a [M][K] operand into a
// stage tile; VEC = 2: 16-byte copies (K even), VEC = 1: 8-byte copies.
template <int VEC>
__device__ __forceinline__ void load_tile(double *dst, const double *__restrict__ src, long M,
                                          int K, long row0, int k0) {
    if (VEC == 2) {
#pragma unroll
        for (int q = 0; q < (BM * BK / 2) / THREADS; ++q) {
            const int idx = threadIdx.x + q * THREADS;
            const int r = idx >> LOG_KCH, ch = idx & (KCH - 1);
            const long gi = row0 + r;
            const int gk = k0 + 2 * ch;
            const bool ok = (gi < M) && (gk < K);
            const double *s = ok ? src + gi * K + gk : src;
            cp_async16(dst + chunk_off(r, ch), s, ok ? 16 : 0);
        }
    } else {
#pragma unroll
        for (int q = 0; q < (BM * BK) / THREADS; ++q) {
            const int idx = threadIdx.x + q * THREADS;
            const int r = idx >> (LOG_KCH + 1), k = idx & (BK - 1);
            const long gi = row0 + r;
            const int gk = k0 + k;
            const bool ok = (gi < M) && (gk < K);
            const double *s = ok ? src + gi * K + gk : src;
            cp_async8(dst + chunk_off(r, k >> 1) + (k & 1), s, ok ? 8 : 0);
        }
    }
}

template <int VEC, int EPI>
__global__ void __launch_bounds__(THREADS, 1)
    dmma_sqt_kernel(const double *__restrict__ A, const double *__restrict__ B, long M, int K,
                    int num_m, int num_n, double alpha, int outer,
                    const double *__restrict__ mrow, const double *__restrict__ zcol,
                    const double2 *__restrict__ uphase, const double2 *__restrict__ wphase,
                    double2 *__restrict__ part, int lat_n, double *__restrict__ tdiag,
                    int abs_sum, long MB, double *__restrict__ Cst, long ldc, double beta) {
    extern __shared__ __align__(16) double smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm = warp >> 2, wn = warp & 3;  // 2 x 4 warps of 64 x 32
    int mb, nb;
    tile_coords(blockIdx.x, num_m, num_n, mb, nb);
    const long m0 = (long)mb * BM, n0 = (long)nb * BN;
    const int nkb = (K + BK - 1) / BK;
    const long MBr = (EPI == EPI_STORE) ? MB : M;  // rows of B (M for S(q,t))

    double acc[4][4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[a][b][e] = 0.0;

#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < nkb) {
            load_tile<VEC>(smem + s * STAGE_DOUBLES, A, M, K, m0, s * BK);
            load_tile<VEC>(smem + s * STAGE_DOUBLES + TILE_DOUBLES, B, MBr, K, n0, s * BK);
        }
        cp_commit();
    }
#pragma unroll 1
    for (int kb = 0; kb < nkb; ++kb) {
        cp_wait<STAGES - 2>();
        __syncthreads();  // stage kb landed for all; stage kb-1 is free again
        {
            const int kn = kb + STAGES - 1;
            if (kn < nkb) {
                double *st = smem + (kn % STAGES) * STAGE_DOUBLES;
                load_tile<VEC>(st, A, M, K, m0, kn * BK);
                load_tile<VEC>(st + TILE_DOUBLES, B, MBr, K, n0, kn * BK);
            }
            cp_commit();
        }
        const double *sa = smem + (kb % STAGES) * STAGE_DOUBLES;
        const double *sb = sa + TILE_DOUBLES;
#pragma unroll
        for (int kk = 0; kk < BK; kk += 8) {
            const int ch = (kk >> 1) + t;  // physical k = kk + 2t, kk + 2t + 1
            double af[4][4], bf[4][2];
#pragma unroll
            for (int mt = 0; mt < 4; ++mt) {
                const int r = wm * 64 + mt * 16 + g;
                const double2 lo = *reinterpret_cast<const double2 *>(sa + chunk_off(r, ch));
                const double2 hi = *reinterpret_cast<const double2 *>(sa + chunk_off(r + 8, ch));
                af[mt][0] = lo.x;
                af[mt][1] = hi.x;
                af[mt][2] = lo.y;
                af[mt][3] = hi.y;
            }
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
                const int c = wn * 32 + nt * 8 + g;
                const double2 v = *reinterpret_cast<const double2 *>(sb + chunk_off(c, ch));
                bf[nt][0] = v.x;
                bf[nt][1] = v.y;
            }
#pragma unroll
            for (int mt = 0; mt < 4; ++mt)
#pragma unroll
                for (int nt = 0; nt < 4; ++nt) dmma::mma_m16n8k8(acc[mt][nt], af[mt], bf[nt]);
        }
    }
    cp_wait<0>();

    if (EPI == EPI_STORE) {
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long i = m0 + wm * 64 + mt * 16 + g + 8 * h;
                if (i >= M) continue;
#pragma unroll
                for (int nt = 0; nt < 4; ++nt)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const long j = n0 + wn * 32 + nt * 8 + 2 * t + e;
                        if (j >= MBr) continue;
                        double *cp = Cst + i + j * ldc;
                        const double v = alpha * acc[mt][nt][2 * h + e];
                        *cp = (beta != 0.0) ? v + beta * *cp : v;
                    }
            }
    } else if (EPI == EPI_PHASE) {
        // sum over the thread's 8 rows x 8 columns of u_i w_j (alpha C_ij - m_i . z_j)
        double tot_re = 0.0, tot_im = 0.0;
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const long i = m0 + wm * 64 + mt * 16 + g + 8 * h;
                if (i >= M) continue;
                double mx = 0.0, my = 0.0, mz = 0.0;
                if (outer) {
                    mx = mrow[3 * i];
                    my = mrow[3 * i + 1];
                    mz = mrow[3 * i + 2];
                }
                double sre = 0.0, sim = 0.0;
#pragma unroll
                for (int nt = 0; nt < 4; ++nt)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const long j = n0 + wn * 32 + nt * 8 + 2 * t + e;
                        if (j >= M) continue;
                        double v = alpha * acc[mt][nt][2 * h + e];
                        if (outer) v -= mx * zcol[3 * j] + my * zcol[3 * j + 1] + mz * zcol[3 * j + 2];
                        if (abs_sum) {
                            sre += fabs(v);
                        } else {
                            const double2 w = wphase[j];
                            sre += w.x * v;
                            sim += w.y * v;
                        }
                    }
                if (abs_sum) {
                    tot_re += sre;
                } else {
                    const double2 u = uphase[i];
                    tot_re += u.x * sre - u.y * sim;
                    tot_im += u.x * sim + u.y * sre;
                }
            }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            tot_re += __shfl_xor_sync(0xffffffffu, tot_re, o);
            tot_im += __shfl_xor_sync(0xffffffffu, tot_im, o);
        }
        __shared__ double red[2][THREADS / 32];
        if (lane == 0) {
            red[0][warp] = tot_re;
            red[1][warp] = tot_im;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double re = 0.0, im = 0.0;
            for (int w = 0; w < THREADS / 32; ++w) {
                re += red[0][w];
                im += red[1][w];
            }
            part[blockIdx.x] = make_double2(re, im);
        }
    } else {
        // The tile's connected values v_ij into shared memory (zero outside
        // the lattice), then one thread per diagonal d = r - c sums them in
        // row order, split by class: 0 when the lattice column of j is at
        // most that of i (no wrap), 1 otherwise.
        __syncthreads();  // every warp is done reading the pipeline stages
        double *T = smem;
#pragma unroll
        for (int mt = 0; mt < 4; ++mt)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int r = wm * 64 + mt * 16 + g + 8 * h;
                const long i = m0 + r;
                double mx = 0.0, my = 0.0, mz = 0.0;
                if (outer && i < M) {
                    mx = mrow[3 * i];
                    my = mrow[3 * i + 1];
                    mz = mrow[3 * i + 2];
                }
#pragma unroll
                for (int nt = 0; nt < 4; ++nt)
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int c = wn * 32 + nt * 8 + 2 * t + e;
                        const long j = n0 + c;
                        double v = 0.0;
                        if (i < M && j < M) {
                            v = alpha * acc[mt][nt][2 * h + e];
                            if (outer)
                                v -= mx * zcol[3 * j] + my * zcol[3 * j + 1] + mz * zcol[3 * j + 2];
                        }
                        T[r * TSTRIDE + c] = v;
                    }
            }
        __syncthreads();
        constexpr int ND = BM + BN - 1;
        const long tslot = (long)mb * num_n + nb;
        for (int dd = threadIdx.x; dd < ND; dd += THREADS) {
            const int d = dd - (BN - 1);  // r - c
            const int r0 = d > 0 ? d : 0, r1 = (BM - 1 < BN - 1 + d) ? BM - 1 : BN - 1 + d;
            // a = (i - j) mod N, the column displacement; class 0 iff col(i) >= a
            const long delta = m0 - n0 + d;
            long a = delta % lat_n;
            if (a < 0) a += lat_n;
            int xi = (int)((m0 + r0) % lat_n);
            double s0 = 0.0, s1 = 0.0;
            for (int r = r0; r <= r1; ++r) {
                const double v = T[r * TSTRIDE + (r - d)];
                if (xi >= a)
                    s0 += v;
                else
                    s1 += v;
                if (++xi == lat_n) xi = 0;
            }
            tdiag[(tslot * ND + dd) * 2] = s0;
            tdiag[(tslot * ND + dd) * 2 + 1] = s1;
        }
    }
}

// 32 x 32 tiles through shared memory (a padded column avoids bank conflicts).
__global__ void __launch_bounds__(256) transpose_f64_kernel(const double *__restrict__ in,
                                                            long rows, long cols,
                                                            double *__restrict__ out) {
    __shared__ double tile[32][33];
    const long r0 = (long)blockIdx.y * 32, c0 = (long)blockIdx.x * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const long r = r0 + y, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[y][threadIdx.x] = in[r * cols + c];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const long c = c0 + y, r = r0 + threadIdx.x;
        if (r < rows && c < cols) out[c * rows + r] = tile[threadIdx.x][y];
    }
}

__global__ void scale_f64_kernel(double *c, long m, long n, long ldc, double beta) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m * n) return;
    const long j = t / m, i = t - j * m;
    double *p = c + i + j * ldc;
    *p = (beta == 0.0) ? 0.0 : beta * *p;
}

}  // namespace

cudaError_t launch_transpose_f64(const double *in, long rows, long cols, double *out,
                                 cudaStream_t st) {
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    const long gx = (cols + 31) / 32, gy = (rows + 31) / 32;
    if (gx > 0x7fffffffL || gy > 65535) return cudaErrorInvalidConfiguration;
    transpose_f64_kernel<<<dim3((unsigned)gx, (unsigned)gy), dim3(32, 8), 0, st>>>(in, rows, cols,
                                                                                   out);
    return cudaGetLastError();
}

cudaError_t launch_scale_f64(double *c, long m, long n, long ldc, double beta, cudaStream_t st) {
    if (m <= 0 || n <= 0) return cudaSuccess;
    const long blocks = (m * n + 255) / 256;
    if (blocks > 0x7fffffffL) return cudaErrorInvalidConfiguration;
    scale_f64_kernel<<<(unsigned)blocks, 256, 0, st>>>(c, m, n, ldc, beta);
    return cudaGetLastError();
}

long dmma_sqt_tiles(long M) {
    const long nm = (M + BM - 1) / BM;
    return nm * nm;
}

int dmma_sqt_diagonals() { return BM + BN - 1; }

int launch_dmma_sqt(const DmmaSqtArgs &p, cudaStream_t st) {
    const bool store = (p.C != nullptr);
    const long MB = store ? p.MB : p.M;
    if (p.M <= 0 || MB <= 0 || p.K <= 0) return fail(ASD_ERR_INVALID, "empty GEMM");
    if (store && (p.tdiag || p.ldc < p.M)) return fail(ASD_ERR_INVALID, "store: bad ldc or q grid");
    const long nm = (p.M + BM - 1) / BM, nn = (MB + BN - 1) / BN;
    if (nm * nn > 0x7fffffffL) return fail(ASD_ERR_UNSUPPORTED, "too many tiles");
    const int num_m = (int)nm, num_n = (int)nn;
    const bool grid = (p.tdiag != nullptr);
    if (grid && (p.lat_n < 1 || (long)p.lat_n * p.lat_n != p.M))
        return fail(ASD_ERR_INVALID, "q grid needs M = N*N");
    const bool vec2 = (p.K % 2 == 0) && (((uintptr_t)p.A | (uintptr_t)p.B) & 15) == 0;
    const int smem = (grid && GRID_SMEM > PIPE_BYTES) ? GRID_SMEM : PIPE_BYTES;
    auto go = [&](auto kern) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        kern<<<(unsigned)(nm * nn), THREADS, smem, st>>>(p.A, p.B, p.M, p.K, num_m, num_n, p.alpha,
                                                          p.outer, p.mrow, p.zcol, p.uphase,
                                                          p.wphase, p.part, p.lat_n, p.tdiag,
                                                          p.abs_sum, MB, p.C, p.ldc, p.beta);
        return cudaGetLastError();
    };
    cudaError_t e;
    if (store)
        e = vec2 ? go(dmma_sqt_kernel<2, EPI_STORE>) : go(dmma_sqt_kernel<1, EPI_STORE>);
    else if (grid)
        e = vec2 ? go(dmma_sqt_kernel<2, EPI_GRID>) : go(dmma_sqt_kernel<1, EPI_GRID>);
    else
        e = vec2 ? go(dmma_sqt_kernel<2, EPI_PHASE>) : go(dmma_sqt_kernel<1, EPI_PHASE>);
    if (e != cudaSuccess) return cuda_fail(e, "dmma_sqt launch");
    return ASD_OK;
}

}  // namespace asd
