// umma_sqt.cu -- S(q,t) as one persistent tcgen05 GEMM with the phase, the
// connected-part subtraction and the reduction fused into its epilogue.
//
// This is the B200 counterpart of the reference's fused_dgemm + KERNEL
// (kernel_fusion/gemm_kernel.h:1-224, :355-422), which streams the full C
// and qmat matrices (2 N^4 + 2 N^4 doubles) through its store epilogue.
// Here neither C nor qmat exists: the phase factorises as u_i * w_j and the
// outer term as m_i . z_j, so the epilogue needs only per-row and per-column
// vectors, and each CTA leaves one complex partial sum.
//
// Precision (3-term split): A = Ah + Al, B = Bh + Bl in TF32, BF16 or FP16, the
// tensor cores accumulate Ah Bh + Ah Bl + Al Bh in FP32 in TMEM; the epilogue
// works in FP32 per 32-column chunk and accumulates in FP64 across chunks,
// tiles and CTAs.
//
// Roles (one CTA per SM, persistent over 128 x 256 tiles):
//   warp 0      TMA producer (one thread): 4 tiles per k block (Ah, Al, Bh, Bl)
//   warp 1      MMA issuer (one thread): 3 x 4 tcgen05.mma per k block
//   warps 2..   epilogue: TMEM -> registers, phase/outer/reduction.  Eight
//               warps (two per TMEM lane quarter, each taking half of the
//               tile's columns) for the phase epilogue, so that its pass over
//               an accumulation chunk stays shorter than the chunk's MMAs even
//               for small chunks; four for the q-grid epilogue, whose
//               per-warp transposition buffers fill the shared memory.
// TMEM holds two 128 x 256 FP32 accumulators (all 512 columns), so the
// epilogue of one tile overlaps the MMAs of the next.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "asd_internal.h"
#include "ptx_sm100.cuh"

namespace asd {
namespace {

constexpr int BM = 128;
constexpr int BN = 256;
// Epilogue warps of each epilogue kind (EPI_GRID: 4, the others 8) and the
// CTA's threads: the TMA and MMA warps plus those.
__host__ __device__ constexpr int epi_warps(int epi) { return epi == 2 ? 4 : 8; }
__host__ __device__ constexpr int cta_threads(int epi) { return 64 + 32 * epi_warps(epi); }
constexpr int MAX_EPI_WARPS = 8;
constexpr int TMEM_COLS = 512;
constexpr uint32_t WAIT_LIMIT = 1u << 24;
// Row tiles per raster group.  Measured on B200 at 128x128x500 and
// 256x256x1000: groups of 16 keep the DRAM traffic lowest (the group's A
// bands, 24-48 MB, stay in L2 while B streams past once per group).
constexpr int GROUP_M = 16;
// q grid: per warp, a 32 x 32 transposition buffer (FP32) while a tile is
// binned, then the warp's tile-diagonal partials (9 x 32 x 2 FP64) when it is
// combined; the two uses alternate, so they share one region.
constexpr int GRID_DIAG_M = 9;  // diagonals per lane and warp: 32 m + lane, 9 values of m
constexpr int GRID_SCRATCH_BYTES = 4 * GRID_DIAG_M * 32 * 2 * 8;  // >= 4 * 32 * 32 * 4
constexpr int GRID_ND = BM + BN - 1;  // diagonals r - c of a 128 x 256 tile

// Pipeline geometry: 128 bytes of K per operand row per stage (the 128-byte
// swizzle width), two stages of 96 KB (Ah, Al 128 x 128 B; Bh, Bl 256 x 128 B).
// Measured on B200, two 96 KB stages are as fast as or faster than four of
// 48 KB with a 64-byte swizzle (fewer barrier round trips per flop).
struct Geo {
    static constexpr int ROWB = 128;
    static constexpr int STAGES = 2;
    static constexpr int A_TILE = BM * ROWB;
    static constexpr int B_TILE = BN * ROWB;
    static constexpr int STAGE_BYTES = 2 * A_TILE + 2 * B_TILE;
    static constexpr int KSTEPS = ROWB / 32;  // 32-byte MMA k steps per stage
    static constexpr int PIPE_BYTES = STAGES * STAGE_BYTES;
    // epilogue column table: w_j = (Re, Im) and z_j, double-buffered by tile
    static constexpr int TABLE_BYTES = 2 * BN * (int)(sizeof(float2) + sizeof(float4));
};

struct SmemTail {
    uint64_t full[Geo::STAGES];
    uint64_t empty[Geo::STAGES];
    uint64_t tfull[2];
    uint64_t tempty[2];
    uint64_t drain;
    uint64_t ebar;  // epilogue warps' barrier
    uint32_t tmem_base;
    int abort_flag;
    double red[2][MAX_EPI_WARPS];
};

constexpr int smem_bytes() {
    return 1024 /*alignment slack*/ + Geo::PIPE_BYTES + Geo::TABLE_BYTES +
           (int)((sizeof(SmemTail) + 15) & ~size_t(15));
}

// Tile raster: groups of group_m row tiles, each walked over all column tiles
// with the row index fastest, so the concurrent tiles share a few B bands and
// the group's A bands stay in L2 while B streams past once per group.
// The tile index is 64-bit: above N = 2896 (M = N^2 sites) there are more
// than 2^31 tiles of 128 x 256.
__device__ __forceinline__ void tile_coords(long tile, int num_m, int num_n, int group_m, int &mb,
                                            int &nb) {
    const long per_group = (long)group_m * num_n;
    const int group = (int)(tile / per_group);
    const int first_m = group * group_m;
    const int gsz = min(group_m, num_m - first_m);
    const long r = tile - group * per_group;
    mb = first_m + (int)(r % gsz);
    nb = (int)(r / gsz);
}

__device__ __forceinline__ void raise_abort(SmemTail *t, unsigned *status) {
    t->abort_flag = 1;
    if (status) atomicOr(status, (unsigned)kStatusTimeout);
}

// Barrier among the epilogue warps on an mbarrier (one arrival per warp), so
// that the wait is bounded like every other wait here: a warp that gives up,
// or sees the abort flag, leaves instead of hanging.
__device__ __forceinline__ bool epilogue_sync(uint64_t *bar, uint32_t &phase,
                                              volatile int *abort) {
    __syncwarp();
    if ((threadIdx.x & 31) == 0) ptx::mbar_arrive(bar);
    const bool ok = ptx::mbar_wait_bounded(bar, phase, abort, WAIT_LIMIT);
    phase ^= 1u;
    return ok;
}

// q grid: bits l = 0..31 of the rows 32 q + l whose lattice column
// x(l) = (x0 + l) mod N lies below thr, i.e. the rows in class 1 of a
// diagonal whose column displacement is thr.  For N >= 32 the 32 rows wrap
// at most once (at l = N - x0), so the set is at most two runs of bits.
__device__ __forceinline__ uint32_t grid_below_mask(int x0, int thr, int N) {
    auto low = [](int k) -> uint32_t {
        return k >= 32 ? 0xffffffffu : (k <= 0 ? 0u : (1u << k) - 1u);
    };
    if (N >= 32) {
        const int nw = min(32, N - x0);  // rows before the wrap: x = x0 + l
        return low(min(nw, thr - x0)) | (low(thr + N - x0) & ~low(nw));
    }
    uint32_t m = 0;
    int x = x0;
    for (int l = 0; l < 32; ++l) {
        if (x < thr) m |= 1u << l;
        if (++x == N) x = 0;
    }
    return m;
}

// val added to exactly one of the four sums, chosen by (b, c): predicated
// adds, so no lane branches and each sum sees its values in step order.
__device__ __forceinline__ void grid_add4(float &pa0, float &pa1, float &pb0, float &pb1,
                                          float val, uint32_t b, uint32_t c) {
    asm("{\n\t.reg .pred pb, q0, q1, q2, q3;\n\t"
        "setp.ne.u32 pb, %5, 0;\n\t"
        "setp.eq.and.u32 q0, %6, 0, !pb;\n\t"
        "setp.ne.and.u32 q1, %6, 0, !pb;\n\t"
        "setp.eq.and.u32 q2, %6, 0, pb;\n\t"
        "setp.ne.and.u32 q3, %6, 0, pb;\n\t"
        "@q0 add.rn.f32 %0, %0, %4;\n\t"
        "@q1 add.rn.f32 %1, %1, %4;\n\t"
        "@q2 add.rn.f32 %2, %2, %4;\n\t"
        "@q3 add.rn.f32 %3, %3, %4;\n\t}"
        : "+f"(pa0), "+f"(pa1), "+f"(pb0), "+f"(pb1)
        : "f"(val), "r"(b), "r"(c));
}

// q grid: one 32 x 32 block (column group c) of a warp's accumulator rows.
// Lane l holds v[jj] = acc(row 32 q + l, column 32 c + jj).  The block's
// diagonals are lambda = l - jj in [-31, 31]; lane L owns lambda = L (tile
// diagonal 32 (q - c) + L, register gd[8 - c]) and lambda = L - 32 (tile
// diagonal 32 (q - c - 1) + L, gd[7 - c]).  Lane l writes v[jj] to row
// (l - jj) mod 32, column l of the warp's buffer; lane L then reads its row,
// from column L onwards (conflict-free both ways): step s reads column
// l = (L + s) mod 32, which is on lambda = L - 32 iff s >= 32 - L.  The class
// of a step (class 0 iff the row's lattice column x >= a, a = (i - j) mod N
// of the diagonal) comes from two 32-bit masks formed once per block, so a
// step is a shared load and one predicated add to one of four sums.
__device__ __forceinline__ void grid_block(const uint32_t (&v)[32], int c, int lane,
                                           const float4 &r4, const float4 *z_tab, float alpha,
                                           bool last, int x_row, int a_first, int N, float *xp,
                                           double (&gd)[9][2]) {
    const float4 *zq = z_tab + c * 32;
    const int wbase = lane * 33;  // row (lane - jj) mod 32, column lane: (wbase - 32 jj) mod 1024
#pragma unroll
    for (int jj = 0; jj < 32; ++jj) {
        float val = alpha * __uint_as_float(v[jj]);
        if (last) {
            const float4 z = zq[jj];
            float o = r4.x * z.x;
            o = fmaf(r4.y, z.y, o);
            o = fmaf(r4.z, z.z, o);
            val -= o;
        }
        xp[(wbase - 32 * jj) & 1023] = val;
    }
    __syncwarp();
    // diagonal lambda = L of block c: i - j shifted by -32 c from block 0
    int aa = (a_first - ((32 * c) % N)) % N;
    if (aa < 0) aa += N;
    int ab = (aa - (32 % N)) % N;  // lambda = L - 32
    if (ab < 0) ab += N;
    const int x0 = __shfl_sync(0xffffffffu, x_row, 0);  // row 32 q + 0
    // class-1 rows: lambda = L on rows l >= L, lambda = L - 32 on rows l < L;
    // rotated right by L so that bit s is the row read at step s
    const uint32_t lowL = (1u << lane) - 1u;
    const uint32_t cm = (grid_below_mask(x0, aa, N) & ~lowL) | (grid_below_mask(x0, ab, N) & lowL);
    uint32_t cbits = __funnelshift_r(cm, cm, lane);
    uint32_t bbits = __funnelshift_r(lowL, lowL, lane);  // steps on lambda = L - 32
    const float *row = xp + lane * 32;
    float pa0 = 0.f, pa1 = 0.f, pb0 = 0.f, pb1 = 0.f;
#pragma unroll 8
    for (int s = 0; s < 32; ++s) {
        const float val = row[(lane + s) & 31];
        grid_add4(pa0, pa1, pb0, pb1, val, bbits & 1u, cbits & 1u);
        bbits >>= 1;
        cbits >>= 1;
    }
    __syncwarp();  // the buffer is free for the next block
    gd[8 - c][0] += (double)pa0;
    gd[8 - c][1] += (double)pa1;
    gd[7 - c][0] += (double)pb0;  // zero in lane 0, which has no lambda = -32
    gd[7 - c][1] += (double)pb1;
}

// KIND: 1 = TF32x3, 2 = BF16x3, 3 = FP16x3.  EPI selects the epilogue:
//   EPI_PHASE  S(q,t) at one q: per-CTA partial sum of u_i w_j (alpha C - m.z)
//   EPI_STORE  the raw FP32 accumulator to dbg_c[i * dbg_ldc + j] (diagnostic)
//   EPI_GRID   the whole q grid: per tile, the sums of alpha C_ij - m_i.z_j
//              along each diagonal d = r - c of the tile, split by whether
//              the lattice column of j wraps (class 0: col(j) <= col(i)),
//              into tdiag[mb][nb][d + BN - 1][class] (qgrid.cu bins them).
//              Each epilogue lane owns the diagonals d = 32 m + lane of its
//              warp's 32 rows: a 32 x 32 block of the accumulator goes
//              through shared memory transposed along its diagonals (lane l
//              writes its value of column jj to row (l - jj) mod 32), each
//              lane sums its two diagonals of the block in a fixed order
//              (FP32, at most 32 terms) into FP64 registers, and the four
//              warps' registers are combined per tile in warp order.  No
//              atomics: the bins repeat bit for bit.
constexpr int EPI_PHASE = 0, EPI_STORE = 1, EPI_GRID = 2;
static_assert(epi_warps(EPI_GRID) == 4 && epi_warps(EPI_PHASE) == MAX_EPI_WARPS, "warp counts");
template <int KIND, int EPI>
__global__ void __launch_bounds__(cta_threads(EPI), 1)
    umma_sqt_kernel(const __grid_constant__ CUtensorMap tm_ah,
                    const __grid_constant__ CUtensorMap tm_al,
                    const __grid_constant__ CUtensorMap tm_bh,
                    const __grid_constant__ CUtensorMap tm_bl, int num_m, int num_n, int kb_begin,
                    int kb_end, int kb_per_chunk, int outer, const float4 *__restrict__ row4,
                    const float *__restrict__ row1, const float4 *__restrict__ col4,
                    const float *__restrict__ col1, float alpha, double2 *__restrict__ part,
                    unsigned *__restrict__ status, float *__restrict__ dbg_c, long dbg_ldc,
                    int lat_n, double *__restrict__ tdiag, int group_m) {
    using G = Geo;
    constexpr bool STORE = (EPI == EPI_STORE);
    constexpr int EW = epi_warps(EPI);         // epilogue warps
    constexpr int NHALF = EW / 4;              // warps per TMEM lane quarter
    constexpr int GPH = BN / 32 / NHALF;       // 32-column groups per warp
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    float2 *tab_w = reinterpret_cast<float2 *>(smem + G::PIPE_BYTES);           // [2][BN]
    float4 *tab_z = reinterpret_cast<float4 *>(smem + G::PIPE_BYTES + 2 * BN * sizeof(float2));
    SmemTail *tail = reinterpret_cast<SmemTail *>(smem + G::PIPE_BYTES + G::TABLE_BYTES);
    uint8_t *gscr = smem + G::PIPE_BYTES + G::TABLE_BYTES + ((sizeof(SmemTail) + 15) & ~size_t(15));
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    const long num_tiles = (long)num_m * num_n;

    if (threadIdx.x == 0) {
        for (int s = 0; s < G::STAGES; ++s) {
            ptx::mbar_init(&tail->full[s], 1);
            ptx::mbar_init(&tail->empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            ptx::mbar_init(&tail->tfull[b], 1);
            ptx::mbar_init(&tail->tempty[b], EW);  // one arrival per epilogue warp
        }
        ptx::mbar_init(&tail->drain, 1);
        ptx::mbar_init(&tail->ebar, EW);
        tail->abort_flag = 0;
        ptx::fence_mbar_init();
    }
    if (warp == 0) {
        ptx::tmem_alloc(&tail->tmem_base, TMEM_COLS);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tmem_base = tail->tmem_base;
    volatile int *abort_flag = &tail->abort_flag;

    if (warp == 0) {
        if (lane == 0) {
            ptx::tma_prefetch_desc(&tm_ah);
            ptx::tma_prefetch_desc(&tm_al);
            ptx::tma_prefetch_desc(&tm_bh);
            ptx::tma_prefetch_desc(&tm_bl);
            constexpr int KE = G::ROWB / ((KIND == 1) ? 4 : 2);  // elements per stage row
            int stage = 0;
            uint32_t phase = 0;
            bool issued[G::STAGES] = {};
            uint32_t issued_parity[G::STAGES] = {};
            bool ok = true;
            for (long tile = blockIdx.x; tile < num_tiles && ok; tile += gridDim.x) {
                int mb, nb;
                tile_coords(tile, num_m, num_n, group_m, mb, nb);
                const int arow = mb * BM;
                const int brow = nb * BN;
                for (int kb = kb_begin; kb < kb_end; ++kb) {
                    if (!ptx::mbar_wait_bounded(&tail->empty[stage], phase ^ 1u, abort_flag,
                                                WAIT_LIMIT)) {
                        raise_abort(tail, status);
                        ok = false;
                        break;
                    }
                    uint8_t *st = smem + stage * G::STAGE_BYTES;
                    const int x = kb * KE;
                    ptx::mbar_arrive_expect_tx(&tail->full[stage], G::STAGE_BYTES);
                    ptx::tma_load_2d(st, &tm_ah, &tail->full[stage], x, arow);
                    ptx::tma_load_2d(st + G::A_TILE, &tm_al, &tail->full[stage], x, arow);
                    ptx::tma_load_2d(st + 2 * G::A_TILE, &tm_bh, &tail->full[stage], x, brow);
                    ptx::tma_load_2d(st + 2 * G::A_TILE + G::B_TILE, &tm_bl, &tail->full[stage],
                                     x, brow);
                    issued[stage] = true;
                    issued_parity[stage] = phase;
                    if (++stage == G::STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            // Never leave the CTA with bulk copies still landing in shared
            // memory: wait (bounded, ignoring the abort flag) for the last
            // fill of every stage.
            for (int s = 0; s < G::STAGES; ++s) {
                if (!issued[s]) continue;
                uint32_t i = 0;
                while (!ptx::mbar_try_wait(&tail->full[s], issued_parity[s]) && i < WAIT_LIMIT) {
                    ++i;
                    __nanosleep(64);
                }
                if (i >= WAIT_LIMIT && status) atomicOr(status, (unsigned)kStatusTimeout);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // A/B format: TF32 2 (kind::tf32); BF16 1, FP16 0 (kind::f16)
            constexpr uint32_t FMT = KIND == 1 ? 2u : KIND == 2 ? 1u : 0u;
            constexpr uint32_t IDESC = ptx::umma_idesc(FMT, BM, BN);
            int stage = 0;
            uint32_t phase = 0;
            int abuf = 0;
            uint32_t aphase = 0;
            bool ok = true;
            const uint32_t smem_base = ptx::smem_u32(smem);
            for (long tile = blockIdx.x; tile < num_tiles && ok; tile += gridDim.x) {
                // K is accumulated in chunks of kb_per_chunk k blocks, each
                // into a fresh TMEM buffer: the tensor core's FP32
                // accumulation loses precision with the number of
                // accumulation steps, and the epilogue adds the chunks in FP64.
                for (int kb0 = kb_begin; kb0 < kb_end && ok; kb0 += kb_per_chunk) {
                    const int kb1 = min(kb0 + kb_per_chunk, kb_end);
                    if (!ptx::mbar_wait_bounded(&tail->tempty[abuf], aphase ^ 1u, abort_flag,
                                                WAIT_LIMIT)) {
                        raise_abort(tail, status);
                        ok = false;
                        break;
                    }
                    ptx::tc_fence_after();
                    const uint32_t d_tmem = tmem_base + (uint32_t)(abuf * BN);
                    for (int kb = kb0; kb < kb1; ++kb) {
                        if (!ptx::mbar_wait_bounded(&tail->full[stage], phase, abort_flag,
                                                    WAIT_LIMIT)) {
                            raise_abort(tail, status);
                            ok = false;
                            break;
                        }
                        ptx::tc_fence_after();
                        const uint32_t s0 = smem_base + stage * G::STAGE_BYTES;
                        const uint64_t dah = ptx::umma_desc_kmajor<G::ROWB>(s0);
                        const uint64_t dal = ptx::umma_desc_kmajor<G::ROWB>(s0 + G::A_TILE);
                        const uint64_t dbh = ptx::umma_desc_kmajor<G::ROWB>(s0 + 2 * G::A_TILE);
                        const uint64_t dbl =
                            ptx::umma_desc_kmajor<G::ROWB>(s0 + 2 * G::A_TILE + G::B_TILE);
#pragma unroll
                        for (int kk = 0; kk < G::KSTEPS; ++kk) {
                            const uint64_t adv = (uint64_t)(2 * kk);  // 32 bytes per k step
                            const uint32_t accum = (kb > kb0 || kk > 0) ? 1u : 0u;
                            if (KIND != 1) {
                                ptx::umma_f16(d_tmem, dah + adv, dbh + adv, IDESC, accum);
                                ptx::umma_f16(d_tmem, dah + adv, dbl + adv, IDESC, 1u);
                                ptx::umma_f16(d_tmem, dal + adv, dbh + adv, IDESC, 1u);
                            } else {
                                ptx::umma_tf32(d_tmem, dah + adv, dbh + adv, IDESC, accum);
                                ptx::umma_tf32(d_tmem, dah + adv, dbl + adv, IDESC, 1u);
                                ptx::umma_tf32(d_tmem, dal + adv, dbh + adv, IDESC, 1u);
                            }
                        }
                        ptx::umma_commit(&tail->empty[stage]);
                        if (++stage == G::STAGES) {
                            stage = 0;
                            phase ^= 1u;
                        }
                    }
                    if (!ok) break;
                    ptx::umma_commit(&tail->tfull[abuf]);
                    if (++abuf == 2) {
                        abuf = 0;
                        aphase ^= 1u;
                    }
                }
            }
            // Wait for every issued MMA before TMEM can be released.
            ptx::umma_commit(&tail->drain);
            uint32_t i = 0;
            while (!ptx::mbar_try_wait(&tail->drain, 0u) && i < WAIT_LIMIT) {
                ++i;
                __nanosleep(64);
            }
            if (i >= WAIT_LIMIT && status) atomicOr(status, (unsigned)kStatusTimeout);
        }
    } else {
        // Epilogue warps 2.. own TMEM lane quarters (warp % 4) * 32; with
        // eight, warps 2..5 take the column groups [0, 4) and warps 6..9
        // the groups [4, 8) of every chunk.
        const int quarter = warp & 3;
        const int rloc = quarter * 32 + lane;
        const int etid = threadIdx.x - 64;  // 0 .. 32 EW - 1 among the epilogue threads
        const int c_first = ((warp - 2) / 4) * GPH;
        int abuf = 0;
        uint32_t aphase = 0;
        double tot_re = 0.0, tot_im = 0.0;
        int tcount = 0;
        uint32_t ephase = 0;
        float *xpose = reinterpret_cast<float *>(gscr) + quarter * 32 * 32;  // [32][32]
        double *wdiag = reinterpret_cast<double *>(gscr);                       // [4][9][32][2]
        for (long tile = blockIdx.x; tile < num_tiles; tile += gridDim.x, ++tcount) {
            int mb, nb;
            tile_coords(tile, num_m, num_n, group_m, mb, nb);
            const long i = (long)mb * BM + rloc;
            const long j0 = (long)nb * BN;
            const int tb = tcount & 1;
            float2 *w_tab = tab_w + tb * BN;
            float4 *z_tab = tab_z + tb * BN;
            if (!STORE) {
                // Column table of this tile (double-buffered by tile: every
                // epilogue warp finished tile - 2 before it passed the
                // barrier of tile - 1).
#pragma unroll
                for (int h = 0; h < BN / (32 * EW); ++h) {
                    const int jl = etid + 32 * EW * h;
                    const float4 cz = __ldg(&col4[j0 + jl]);
                    w_tab[jl] = make_float2(cz.w, __ldg(&col1[j0 + jl]));
                    z_tab[jl] = make_float4(cz.x, cz.y, cz.z, 0.f);
                }
                if (!epilogue_sync(&tail->ebar, ephase, abort_flag)) {
                    raise_abort(tail, status);
                    break;
                }
            }
            const float4 r4 = STORE ? make_float4(0.f, 0.f, 0.f, 0.f) : row4[i];
            const float ui = STORE ? 0.f : row1[i];
            double s_re = 0.0, s_im = 0.0;
            bool ok = true;
            // q grid: this lane's diagonals d = 32 (quarter - 8 + mm) + lane of
            // the tile, both classes; the column of its own row's site;
            // the columns a = (i - j) mod N of its first block's two diagonals.
            double gd[GRID_DIAG_M][2];
            int x_row = 0, a_first = 0;
            if (EPI == EPI_GRID) {
#pragma unroll
                for (int mm = 0; mm < GRID_DIAG_M; ++mm) gd[mm][0] = gd[mm][1] = 0.0;
                x_row = (int)((mb * (long)BM + quarter * 32 + lane) % lat_n);
                // diagonal d = 32 quarter + lane of block c = 0: i - j = i0 - j0 + d
                long dl = (long)mb * BM - (long)nb * BN + quarter * 32 + lane;
                dl %= lat_n;
                a_first = (int)(dl < 0 ? dl + lat_n : dl);
            }
            for (int kb0 = kb_begin; kb0 < kb_end; kb0 += kb_per_chunk) {
                const bool first = (kb0 == kb_begin);
                // the connected-part term, once per row: in the last chunk
                // of the launch that carries it
                const bool last = outer && (kb0 + kb_per_chunk >= kb_end);
                if (!ptx::mbar_wait_bounded(&tail->tfull[abuf], aphase, abort_flag, WAIT_LIMIT)) {
                    raise_abort(tail, status);
                    ok = false;
                    break;
                }
                ptx::tc_fence_after();
                // Per 32-column group, in FP32: a = sum_j w_j acc_ij and, in the
                // last chunk only, o = sum_j w_j (m_i . z_j); the row sum
                // s_i = alpha * a - o is carried in FP64.  (The q grid unrolls
                // the groups: its per-lane diagonal registers are indexed by c.)
                constexpr int CU = (EPI == EPI_GRID) ? BN / 32 : 1;
#pragma unroll CU
                for (int cc = 0; cc < GPH; ++cc) {
                    const int c = (EPI == EPI_GRID) ? cc : c_first + cc;  // a constant for the grid
                    uint32_t v[32];
                    const uint32_t taddr = tmem_base + ((uint32_t)(quarter * 32) << 16) +
                                           (uint32_t)(abuf * BN + c * 32);
                    ptx::tmem_ld_32x32b_x32(taddr, v);
                    ptx::tmem_ld_wait();
                    if (STORE) {
                        float *dst = dbg_c + i * dbg_ldc + j0 + c * 32;
#pragma unroll
                        for (int jj = 0; jj < 32; ++jj)
                            dst[jj] = (first ? 0.f : dst[jj]) + __uint_as_float(v[jj]);
                        continue;
                    }
                    if (EPI == EPI_GRID) {
                        grid_block(v, c, lane, r4, z_tab, alpha, last, x_row, a_first, lat_n,
                                   xpose, gd);
                        continue;
                    }
                    const float4 *wq = reinterpret_cast<const float4 *>(w_tab + c * 32);
                    float are0 = 0.f, aim0 = 0.f, are1 = 0.f, aim1 = 0.f;
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const float4 w = wq[q];  // (Re w, Im w) of columns 2q, 2q+1
                        const float a0 = __uint_as_float(v[2 * q]);
                        const float a1 = __uint_as_float(v[2 * q + 1]);
                        are0 = fmaf(w.x, a0, are0);
                        aim0 = fmaf(w.y, a0, aim0);
                        are1 = fmaf(w.z, a1, are1);
                        aim1 = fmaf(w.w, a1, aim1);
                    }
                    float ore = 0.f, oim = 0.f;
                    if (last) {
                        const float4 *zq = z_tab + c * 32;
                        const float2 *wv = w_tab + c * 32;
#pragma unroll 8
                        for (int jj = 0; jj < 32; ++jj) {
                            const float4 z = zq[jj];
                            const float2 w = wv[jj];
                            float o = r4.x * z.x;
                            o = fmaf(r4.y, z.y, o);
                            o = fmaf(r4.z, z.z, o);
                            ore = fmaf(w.x, o, ore);
                            oim = fmaf(w.y, o, oim);
                        }
                    }
                    s_re += (double)alpha * (double)(are0 + are1) - (double)ore;
                    s_im += (double)alpha * (double)(aim0 + aim1) - (double)oim;
                }
                ptx::tc_fence_before();
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&tail->tempty[abuf]);
                if (++abuf == 2) {
                    abuf = 0;
                    aphase ^= 1u;
                }
            }
            if (!ok) break;
            if (EPI == EPI_GRID) {
                // the four warps' diagonals -> tdiag[tile], in warp order; the
                // shared region served as transposition buffers until now
                if (!epilogue_sync(&tail->ebar, ephase, abort_flag)) {
                    raise_abort(tail, status);
                    break;
                }
                double *wq = wdiag + quarter * (GRID_DIAG_M * 32 * 2);
#pragma unroll
                for (int mm = 0; mm < GRID_DIAG_M; ++mm) {
                    wq[(mm * 32 + lane) * 2] = gd[mm][0];
                    wq[(mm * 32 + lane) * 2 + 1] = gd[mm][1];
                }
                if (!epilogue_sync(&tail->ebar, ephase, abort_flag)) {
                    raise_abort(tail, status);
                    break;
                }
                double *td = tdiag + ((long)mb * num_n + nb) * GRID_ND * 2;
                for (int idx = etid; idx < GRID_ND * 2; idx += 32 * EW) {
                    const int d = idx / 2 - (BN - 1), cls = idx & 1;
                    const int L = (d + 256) & 31, m = (d - L) / 32;
                    double sum = 0.0;
#pragma unroll
                    for (int w = 0; w < 4; ++w) {
                        const int mm = m - w + 8;
                        if (mm >= 0 && mm < GRID_DIAG_M)
                            sum += wdiag[((w * GRID_DIAG_M + mm) * 32 + L) * 2 + cls];
                    }
                    td[idx] = sum;
                }
                if (!epilogue_sync(&tail->ebar, ephase, abort_flag)) {
                    raise_abort(tail, status);
                    break;
                }
            }
            // u_i * s_i with u_i = (r4.w, ui)
            tot_re += (double)r4.w * s_re - (double)ui * s_im;
            tot_im += (double)r4.w * s_im + (double)ui * s_re;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            tot_re += __shfl_xor_sync(0xffffffffu, tot_re, o);
            tot_im += __shfl_xor_sync(0xffffffffu, tot_im, o);
        }
        if (lane == 0) {
            tail->red[0][warp - 2] = tot_re;
            tail->red[1][warp - 2] = tot_im;
        }
    }

    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (threadIdx.x == 0 && EPI == EPI_PHASE) {
        double re = 0.0, im = 0.0;  // fixed order: the results repeat bit for bit
#pragma unroll
        for (int w = 0; w < EW; ++w) {
            re += tail->red[0][w];
            im += tail->red[1][w];
        }
        part[blockIdx.x] = make_double2(re, im);
    }
    if (warp == 0) ptx::tmem_dealloc(tmem_base, TMEM_COLS);
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Row-major [rows][Kp] operand, box = rowb (128) bytes of K x box_rows rows,
// 128-byte swizzle.
int make_tmap(CUtensorMap *m, const void *base, int kind, long rows, int Kp, int box_rows,
              int rowb) {
    auto enc = get_encode_fn();
    if (!enc) return fail(ASD_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const int esize = split_esize(kind);
    const CUtensorMapDataType dt = kind == 1   ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32
                                   : kind == 2 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                               : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    cuuint64_t gdim[2] = {(cuuint64_t)Kp, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)Kp * esize};
    cuuint32_t box[2] = {(cuuint32_t)(rowb / esize), (cuuint32_t)box_rows};
    cuuint32_t estride[2] = {1, 1};
    CUresult r = enc(m, dt, 2, const_cast<void *>(base), gdim, gstride, box, estride,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(ASD_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return ASD_OK;
}

}  // namespace

long umma_row_pad(long M) { return (M + BN - 1) / BN * BN; }

int umma_tile_rows() { return BM; }
int umma_tile_cols() { return BN; }

long umma_max_grid_for(long M, int num_sms) {
    const long Mp = umma_row_pad(M);
    const long tiles = (Mp / BM) * (Mp / BN);
    return tiles < num_sms ? tiles : num_sms;
}

int launch_umma_sqt(const UmmaSqtArgs &a, cudaStream_t st) {
    const long Mp = umma_row_pad(a.M);
    if (a.kind < 1 || a.kind > 3) return fail(ASD_ERR_INVALID, "split kind %d", a.kind);
    const int esize = split_esize(a.kind);
    if (a.Kp <= 0 || (a.Kp * esize) % Geo::ROWB != 0)
        return fail(ASD_ERR_INVALID, "Kp=%d: rows must be a multiple of 128 bytes", a.Kp);
    if (((uintptr_t)a.a_hi | (uintptr_t)a.a_lo | (uintptr_t)a.b_hi | (uintptr_t)a.b_lo) & 15)
        return fail(ASD_ERR_INVALID, "operand base not 16-byte aligned");
    const int ke = Geo::ROWB / esize;  // K elements per pipeline stage
    CUtensorMap tah, tal, tbh, tbl;
    int rc;
    if ((rc = make_tmap(&tah, a.a_hi, a.kind, Mp, a.Kp, BM, Geo::ROWB)) != ASD_OK) return rc;
    if ((rc = make_tmap(&tal, a.a_lo, a.kind, Mp, a.Kp, BM, Geo::ROWB)) != ASD_OK) return rc;
    if ((rc = make_tmap(&tbh, a.b_hi, a.kind, Mp, a.Kp, BN, Geo::ROWB)) != ASD_OK) return rc;
    if ((rc = make_tmap(&tbl, a.b_lo, a.kind, Mp, a.Kp, BN, Geo::ROWB)) != ASD_OK) return rc;
    const int num_m = (int)(Mp / BM), num_n = (int)(Mp / BN), num_kb = a.Kp / ke;
    const int k_end = a.k_end > 0 ? a.k_end : a.Kp;
    if (a.k_begin < 0 || a.k_begin % ke != 0 || k_end % ke != 0 || k_end > a.Kp ||
        a.k_begin >= k_end)
        return fail(ASD_ERR_INVALID, "K range [%d, %d) is not whole k blocks of %d in [0, %d)",
                    a.k_begin, k_end, ke, a.Kp);
    const int kb_begin = a.k_begin / ke, kb_end = k_end / ke;
    const long tiles = (long)num_m * num_n;
    // k blocks per accumulation chunk: chunk_k elements of K (0 = all of K)
    int kpc = a.chunk_k > 0 ? (a.chunk_k + ke - 1) / ke : num_kb;
    if (kpc < 1) kpc = 1;
    if (kpc > num_kb) kpc = num_kb;
    // One persistent CTA per SM (or per tile, if fewer); every CTA strides
    // over the tiles, so any grid size is correct and a caller's cap (the
    // partials it has room for) only lengthens each CTA's tile list.
    int grid = tiles < a.num_sms ? (int)tiles : a.num_sms;
    if (a.max_grid > 0 && grid > a.max_grid) grid = a.max_grid;
    if (grid < 1) return fail(ASD_ERR_INVALID, "no tiles to launch");
    const int epi = a.dbg_c ? EPI_STORE : (a.tdiag ? EPI_GRID : EPI_PHASE);
    if (epi == EPI_GRID && (a.lat_n < 1 || (long)a.lat_n * a.lat_n != a.M || a.k_begin != 0 ||
                            (a.k_end != 0 && a.k_end != a.Kp)))
        return fail(ASD_ERR_INVALID, "q grid: M must be N*N and K whole");
    const int smem = smem_bytes() + ((epi == EPI_GRID) ? GRID_SCRATCH_BYTES : 0);
    auto go = [&](auto kern) {
        cudaError_t r =
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (r != cudaSuccess) return r;
        kern<<<grid, cta_threads(epi), smem, st>>>(tah, tal, tbh, tbl, num_m, num_n, kb_begin, kb_end,
                                              kpc, a.outer, a.row4, a.row1, a.col4, a.col1,
                                              a.alpha, a.part, a.status, a.dbg_c, a.dbg_ldc,
                                              a.lat_n, a.tdiag, GROUP_M);
        return cudaGetLastError();
    };
    cudaError_t e;
    if (a.kind == 3)
        e = epi == EPI_STORE  ? go(umma_sqt_kernel<3, EPI_STORE>)
            : epi == EPI_GRID ? go(umma_sqt_kernel<3, EPI_GRID>)
                              : go(umma_sqt_kernel<3, EPI_PHASE>);
    else if (a.kind == 2)
        e = epi == EPI_STORE  ? go(umma_sqt_kernel<2, EPI_STORE>)
            : epi == EPI_GRID ? go(umma_sqt_kernel<2, EPI_GRID>)
                              : go(umma_sqt_kernel<2, EPI_PHASE>);
    else
        e = epi == EPI_STORE  ? go(umma_sqt_kernel<1, EPI_STORE>)
            : epi == EPI_GRID ? go(umma_sqt_kernel<1, EPI_GRID>)
                              : go(umma_sqt_kernel<1, EPI_PHASE>);
    if (e != cudaSuccess) return cuda_fail(e, "umma_sqt launch");
    return grid;
}

namespace {
// Waits on an mbarrier that no thread ever arrives at: the bounded wait must
// give up after `limit` polls and record a timeout.
__global__ void mbar_timeout_probe_kernel(uint32_t limit, unsigned *status) {
    __shared__ uint64_t bar;
    __shared__ int abort_flag;
    if (threadIdx.x == 0) {
        ptx::mbar_init(&bar, 1);
        abort_flag = 0;
        ptx::fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0 && !ptx::mbar_wait_bounded(&bar, 0u, &abort_flag, limit))
        atomicOr(status, (unsigned)kStatusTimeout);
}
}  // namespace

cudaError_t launch_mbar_timeout_probe(uint32_t limit, unsigned *status, cudaStream_t st) {
    mbar_timeout_probe_kernel<<<1, 32, 0, st>>>(limit, status);
    return cudaGetLastError();
}

}  // namespace asd

// Diagnostic entry point (declared in include/asd_b200.h): the bare
// split-precision tensor-core product C = Ah Bh^T + Ah Bl^T + Al Bh^T, FP32,
// device pointers, rows a multiple of 256.
extern "C" int asd_umma_gemm_f32(int kind, long rows, int Kp, const void *a_hi, const void *a_lo,
                                 const void *b_hi, const void *b_lo, float *c, long ldc,
                                 int chunk_k, void *stream) {
    using namespace asd;
    if (kind < 1 || kind > 3)
        return fail(ASD_ERR_INVALID, "kind must be 1 (TF32), 2 (BF16) or 3 (FP16)");
    if (rows <= 0 || rows % 256 != 0) return fail(ASD_ERR_INVALID, "rows must be a multiple of 256");
    if (!a_hi || !a_lo || !b_hi || !b_lo || !c || ldc < rows)
        return fail(ASD_ERR_INVALID, "bad pointer or ldc");
    int dev = 0, sms = 0;
    ASD_CUDA_TRY(cudaGetDevice(&dev));
    ASD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    UmmaSqtArgs u{};
    u.kind = kind;
    u.M = rows;
    u.Kp = Kp;
    u.a_hi = a_hi;
    u.a_lo = a_lo;
    u.b_hi = b_hi;
    u.b_lo = b_lo;
    u.num_sms = sms;
    u.dbg_c = c;
    u.dbg_ldc = ldc;
    u.chunk_k = chunk_k;
    const int g = launch_umma_sqt(u, (cudaStream_t)stream);
    return g < 0 ? g : ASD_OK;
}

// ------------------------------------------------ allocation-free variant
// Some hosts cannot call cudaMalloc from the code that evaluates S(q,t):
// applications that hand all device memory to their own pool or caching
// allocator at start-up and keep a fixed budget, and time-step loops that
// must not call cudaMalloc/cudaFree because those calls can synchronise the
// device and stall the other streams.  asd_sqt_split_noalloc serves them: the
// caller passes every input and output buffer, and the only scratch the
// kernels need -- one partial sum per CTA and a status word -- lives in the
// fixed array below, which every GPU that loads this library holds until the
// process exits.
namespace asd {
namespace {

constexpr int kNoAllocMaxCtas = 1024;  // partials: at most one per CTA
constexpr size_t kNoAllocPartBytes = kNoAllocMaxCtas * sizeof(double2);
constexpr size_t kNoAllocScratchBytes = kNoAllocPartBytes + 256;  // + status word
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch in the current device's context.  The
// symbol's name in host code is only a host-side stand-in for it.  The
// address is looked up on every call (a host-side query that allocates
// nothing), so it stays right after cudaDeviceReset, under another context,
// and when the caller switches devices between calls.
int noalloc_scratch(unsigned char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    *out = static_cast<unsigned char *>(p);
    return ASD_OK;
}

// Sum of the per-CTA partials in a fixed order, times scale; NaN when a
// bounded wait in the GEMM gave up (status word non-zero).
__global__ void __launch_bounds__(256) noalloc_finalize_kernel(const double2 *__restrict__ part,
                                                               int nparts, double scale,
                                                               const unsigned *__restrict__ status,
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
        const bool bad = (*status != 0u);
        out[0] = bad ? __longlong_as_double(0x7ff8000000000000ll) : sre[0] * scale;
        out[1] = bad ? __longlong_as_double(0x7ff8000000000000ll) : sim[0] * scale;
    }
}

}  // namespace
}  // namespace asd

extern "C" int asd_sqt_split_noalloc(int kind, long rows, int Kp, const void *a_hi,
                                     const void *a_lo, const void *b_hi, const void *b_lo,
                                     const void *row4, const float *row1, const void *col4,
                                     const float *col1, double alpha, double scale, int chunk_k,
                                     double *d_out, void *stream) {
    using namespace asd;
    if (kind != 1 && kind != 2) return fail(ASD_ERR_INVALID, "kind must be 1 (TF32x3) or 2 (BF16x3)");
    if (rows <= 0 || rows % 256 != 0) return fail(ASD_ERR_INVALID, "rows must be a positive multiple of 256");
    if (!a_hi || !a_lo || !b_hi || !b_lo || !row4 || !row1 || !col4 || !col1 || !d_out)
        return fail(ASD_ERR_INVALID, "NULL buffer");
    if (((uintptr_t)row4 | (uintptr_t)col4) & 15)
        return fail(ASD_ERR_INVALID, "row4/col4 must be 16-byte aligned");
    if (chunk_k < 0) return fail(ASD_ERR_INVALID, "chunk_k < 0");
    int dev = 0, sms = 0, sdev = 0;
    ASD_CUDA_TRY(cudaGetDevice(&dev));
    cudaStream_t st = (cudaStream_t)stream;
    // The scratch address is the current device's; a stream of another
    // device would run the kernels there with this device's address.
    ASD_CUDA_TRY(cudaStreamGetDevice(st, &sdev));
    if (sdev != dev)
        return fail(ASD_ERR_INVALID, "stream belongs to device %d, the current device is %d", sdev,
                    dev);
    ASD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const long ctas = umma_max_grid_for(rows, sms);
    if (ctas > kNoAllocMaxCtas)
        return fail(ASD_ERR_UNSUPPORTED,
                    "the fixed scratch holds %d CTA partials; this launch needs %ld", kNoAllocMaxCtas,
                    ctas);
    unsigned char *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc != ASD_OK) return rc;
    double2 *part = reinterpret_cast<double2 *>(scratch);
    unsigned *status = reinterpret_cast<unsigned *>(scratch + kNoAllocPartBytes);
    // the status word keeps the last call's value: clear it
    ASD_CUDA_TRY(cudaMemsetAsync(status, 0, sizeof(unsigned), st));
    UmmaSqtArgs u{};
    u.kind = kind;
    u.M = rows;
    u.Kp = Kp;
    u.a_hi = a_hi;
    u.a_lo = a_lo;
    u.b_hi = b_hi;
    u.b_lo = b_lo;
    u.row4 = static_cast<const float4 *>(row4);
    u.row1 = row1;
    u.col4 = static_cast<const float4 *>(col4);
    u.col1 = col1;
    u.alpha = (float)alpha;
    u.part = part;
    u.status = status;
    u.num_sms = sms;
    u.max_grid = kNoAllocMaxCtas;  // never more partials than the array holds
    u.chunk_k = chunk_k;
    const int grid = launch_umma_sqt(u, st);
    if (grid < 0) return grid;
    noalloc_finalize_kernel<<<1, 256, 0, st>>>(part, grid, scale, status, d_out);
    ASD_CUDA_TRY(cudaGetLastError());
    return ASD_OK;
}
