// llg_kernels.cu -- RK4 time stepping of the LLG equation on the GPU, FP64.
//
// Arithmetic contract: every operation is an explicitly rounded FP64
// intrinsic (__dmul_rn, __dadd_rn, __dsub_rn, __ddiv_rn, __dsqrt_rn), in the
// order the reference writes it, so the compiler cannot contract a*b+c into
// an FMA.  With alpha = J2 = h = 0 the trajectory is therefore bit-identical
// to the reference's euler / runge_kutta / renormalisation built with
// -ffp-contract=off (llg_sqt_baseline.c:29-142, :298-309).
#include <cstdlib>
#include <type_traits>

#include "asd_internal.h"

namespace asd {
namespace {

#include "llg_math.cuh"

// One fused RK4 stage, site-major layout.  Thread t handles replica
// f = t % nfile of site t / nfile, so a warp touches 32 consecutive 24-byte
// records (768 contiguous bytes) of each operand.  The combination order
// reproduces runge_kutta's final sum spin + k1/6 + k2/3 + k3/3 + k4/6
// evaluated left to right (llg_sqt_baseline.c:138), carried in acc.
//
// Thread mapping.  With fewer than 64 replicas, thread t is (site t / nc,
// replica t % nc).  With 64 or more (ngroups = ceil(nc / 32) groups of 32),
// block b takes a 2 x 4 patch of sites (one per warp) of replica group
// b % ngroups, lane = replica within the group: the warps of a block are
// lattice neighbours, so many of the input vectors a warp reads as
// neighbours are other warps' centres and hit in L1 instead of L2 (the block
// reads 20 distinct site vectors for 8 sites, 24 with J2, instead of 40 / 72).
// Measured on B200 against one thread per (site, replica) in order:
// 256x256x1000 with J2 5.21 vs 6.12-6.21 ms per step of four stages.
// At most 32 registers (8 blocks of 256 threads per SM): stage 4 with J2
// otherwise takes 34 and only 6 blocks fit.
template <int STAGE, bool J2, bool H, bool DAMP>
__global__ void __launch_bounds__(256, 8) llg_stage_kernel(LLGArgs a, const double *__restrict__ y,
                                                        const double *__restrict__ ys,
                                                        double *__restrict__ acc,
                                                        double *__restrict__ out, int ngroups) {
    long site;
    int f;
    if (ngroups > 0) {
        const int g = (int)(blockIdx.x % ngroups);
        const long tile = blockIdx.x / ngroups;
        const int tcols = (a.N + 3) / 4;
        const int w = threadIdx.x >> 5;
        const int trow = (int)(tile / tcols) * 2 + (w >> 2), tcol = (int)(tile % tcols) * 4 + (w & 3);
        const int lf = g * 32 + (threadIdx.x & 31);
        if (trow >= a.N || tcol >= a.N || lf >= a.nc) return;
        site = (long)trow * a.N + tcol;
        f = a.f0 + lf;
    } else {
        const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
        if (t >= a.M * a.nc) return;
        site = t / a.nc;
        f = a.f0 + (int)(t - site * a.nc);
    }
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

__device__ __forceinline__ V3 ld3(const double *p) { return V3{p[0], p[1], p[2]}; }

constexpr int kGroupedMinReplicas = 64;  // below: one thread per (site, replica) in order

template <int STAGE>
cudaError_t launch_stage_t(const LLGArgs &a, const double *y, const double *ys, double *acc,
                           double *out, cudaStream_t st) {
    if (a.f0 < 0 || a.nc < 1 || a.f0 + a.nc > a.nfile) return cudaErrorInvalidValue;
    const long total = a.M * a.nc;
    const int threads = 256;
    const int sel = (a.use_j2 ? 4 : 0) | (a.use_h ? 2 : 0) | (a.use_damp ? 1 : 0);
    // site-grouped mapping when the replica groups of 32 are mostly full
    const int ngroups = (a.nc >= kGroupedMinReplicas) ? (a.nc + 31) / 32 : 0;
    const long gblocks = (long)ngroups * ((a.N + 1) / 2) * ((a.N + 3) / 4);
    if (gblocks > 0x7fffffffL) return cudaErrorInvalidConfiguration;
    const unsigned blocks = ngroups > 0 ? (unsigned)gblocks
                                        : (unsigned)((total + threads - 1) / threads);
#define ASD_STAGE_CASE(S, J, Hh, D)                                                            \
    case S:                                                                                    \
        llg_stage_kernel<STAGE, J, Hh, D><<<blocks, threads, 0, st>>>(a, y, ys, acc, out,      \
                                                                       ngroups);               \
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

// ------------------------------------------------ row-streaming step
// One RK4 step per launch, streamed down the lattice.  The work is a set of
// columns of rows: a band of wc core columns (plus 4 halo columns each side,
// one per stage) for SF replicas, over all N rows.  A persistent grid of
// CTAs splits the band x replica-group x row space evenly, each CTA taking
// one contiguous run of rows that crosses at most a few (band, group)
// boundaries; every piece of a run is streamed on its own.
//
// A piece of rs rows (relative rows 0..rs+7: 4 halo rows above and below)
// is walked once, two phases per iteration j, separated by barriers:
//   phase A: stage 1 on row j-1 (y rows j-2..j), stage 3 on row j-4;
//   phase B: cp.async prefetch of y row j+1, stage 2 on row j-2, stage 4 on
//            row j-5 (renormalised, stored to DRAM).
// Each stage reads only rows written in an earlier phase, and the two stages
// of a phase are independent (twice the instruction-level parallelism of a
// stage-per-phase schedule, half the barriers).  Stage inputs live in rings
// of 3 rows, y in a ring of 5 rows, and the running RK4 combination of the
// five rows in flight in registers.  Halo work is (wc + 8) / wc in columns;
// DRAM traffic: y read once (the halo columns mostly from L2) and y_new
// written once, 48 bytes per site-step.  Per (site, replica) the arithmetic
// is the stage kernels' (bit-identical).
namespace stream {
constexpr int SF = 4;                  // replicas per CTA (96 contiguous bytes per site)
constexpr int WC_MAX = 64;             // core columns per band
constexpr int WT_MAX = WC_MAX + 8;     // columns held per row
constexpr int NT_MAX = WT_MAX * SF;    // threads per CTA at most (288)
constexpr int YR = 5;                  // rows of the y ring
constexpr int ROWS = YR + 3 * 3;       // row buffers in shared memory
constexpr int MIN_RUN = 16;            // fewest rows per CTA
}  // namespace stream

struct StreamGeom {
    int wc;   // core columns per band (a multiple of 8)
    int wt;   // wc + 8 columns held per row
    int nb;   // bands: ceil(N / wc)
    int ng;   // replica groups: ceil(nc / SF)
    int rw;   // doubles per row buffer: wt * SF * 3
    long run; // rows per CTA of the nb * ng * N rows of work
};

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}


// Inputs of one stage at one (site, replica): the centre value, its
// neighbours in llg_rhs's order -- (row+1), (row-1), (col-1), (col+1), then
// the diagonals (+1,+1), (+1,-1), (-1,+1), (-1,-1) -- and the RK4 base y.
struct SIn {
    V3 s, nb[4], n2[4], yb;
};

// Loads record `me` of row buffer `mid` and its neighbours from the rows
// above (`up`, row-1) and below (`dn`, row+1); CS = doubles per column.
template <bool J2>
__device__ __forceinline__ void load_in(const double *up, const double *mid, const double *dn,
                                        int me, SIn &in) {
    constexpr int CS = stream::SF * 3;
    in.s = ld3(mid + me);
    in.nb[0] = ld3(dn + me);
    in.nb[1] = ld3(up + me);
    in.nb[2] = ld3(mid + me - CS);
    in.nb[3] = ld3(mid + me + CS);
    if (J2) {
        in.n2[0] = ld3(dn + me + CS);
        in.n2[1] = ld3(dn + me - CS);
        in.n2[2] = ld3(up + me + CS);
        in.n2[3] = ld3(up + me - CS);
    }
}

template <bool J2, bool H, bool DAMP>
__global__ void __launch_bounds__(stream::NT_MAX, 2)
    llg_step_stream_kernel(LLGArgs a, StreamGeom g, const double *__restrict__ y,
                           double *__restrict__ yout) {
    using namespace stream;
    extern __shared__ double ssm[];
    const int rw = g.rw;
    double *const ybuf = ssm;
    double *const s1 = ssm + YR * rw;
    double *const s2 = s1 + 3 * rw;
    double *const s3 = s2 + 3 * rw;
    const int N = a.N;
    const long K = 3L * a.nfile;
    const int tid = threadIdx.x;
    const int cl = tid / SF, fl = tid - cl * SF;
    const int me = tid * 3;  // == (cl * SF + fl) * 3
    const bool comp = cl >= 1 && cl <= g.wt - 2;
    const double dt = a.dt;

    const long total = (long)g.nb * g.ng * N;
    long b = (long)blockIdx.x * g.run;
    const long e = min(b + g.run, total);
    while (b < e) {
        // piece: rows [R0, R0 + rs) of work column u = band + nb * grp
        const long u = b / N;
        const int R0 = (int)(b - u * N);
        const int rs = (int)min((long)(N - R0), e - b);
        b += rs;
        const int band = (int)(u % g.nb), grp = (int)(u / g.nb);
        const int C0 = band * g.wc;
        const int fbase = a.f0 + grp * SF;
        const int nvalid = min(SF, a.f0 + a.nc - fbase);
        const int gcol = C0 + cl - 4;
        const bool store = cl >= 4 && cl < 4 + g.wc && gcol < N && fl < nvalid;
        const int J = rs + 9;  // iterations: stage 4 reaches relative row rs + 3 at j = rs + 8

        // A row buffer holds rw = 3 * blockDim.x doubles, so each thread
        // copies three of them per row: column c = x / 12 of the band
        // (periodic), value w = x % 12 of its 4 replicas x 3 components.
        // Their offsets within a lattice row are the same for every row of
        // the piece, so they are formed once here, not once per row.
        long goff[3];
        bool gval[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const int x = tid + k * (int)blockDim.x;
            const int c = x / (SF * 3), w = x - c * (SF * 3);
            int gc = (C0 - 4 + c) % N;
            if (gc < 0) gc += N;
            gval[k] = w < 3 * nvalid;
            goff[k] = (long)gc * K + 3L * fbase + w;
        }
        const long row_stride = (long)N * K;
        // y row R0 - 4 + j (periodic) of this band and replica group -> y ring
        auto load_row = [&](int j, int slot) {  // slot = j % YR
            int gr = R0 - 4 + j;  // in [-4, N + 4): at most two wraps for N >= 3
            while (gr < 0) gr += N;
            while (gr >= N) gr -= N;
            const double *src = y + (long)gr * row_stride;
            double *dst = ybuf + slot * rw;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const int x = tid + k * (int)blockDim.x;
                if (gval[k])
                    cp_async8(dst + x, src + goff[k]);
                else
                    dst[x] = 0.0;
            }
        };
        // Stage bodies on relative row r (in y slot r % 5, ring slot r % 3),
        // each split into its shared-memory loads (ld) and its arithmetic and
        // stores (st*), so that the two stages of a phase can issue all their
        // loads before either computes.  The callers pass the ring slots of
        // rows r - 1, r, r + 1 (and of the base row in the y ring, or -1):
        // the y slots are compile-time constants of the unrolled iteration,
        // the 3-row ring slots one of three rotations of a running j % 3.
        auto ld = [&](const double *ring, int su, int sm, int sd, int sb) {
            SIn in;
            load_in<J2>(ring + su * rw, ring + sm * rw, ring + sd * rw, me, in);
            if (sb >= 0) in.yb = ld3(ybuf + sb * rw + me);
            return in;
        };
        auto st1 = [&](const SIn &in, int r3, double *ac) {  // s1 = y + k/2, acc = y + k/6
            const V3 d = llg_rhs_vals<J2, H, DAMP>(in.s, in.nb, in.n2, a);
            const double k0 = dm(d.x, dt), k1 = dm(d.y, dt), k2 = dm(d.z, dt);
            double *o = s1 + r3 * rw + me;
            o[0] = da(in.s.x, half(k0));
            o[1] = da(in.s.y, half(k1));
            o[2] = da(in.s.z, half(k2));
            ac[0] = da(in.s.x, div6(k0));
            ac[1] = da(in.s.y, div6(k1));
            ac[2] = da(in.s.z, div6(k2));
        };
        auto st2 = [&](const SIn &in, int r3, double *ac) {  // s2 = y + k/2, acc += k/3
            const V3 d = llg_rhs_vals<J2, H, DAMP>(in.s, in.nb, in.n2, a);
            const double k0 = dm(d.x, dt), k1 = dm(d.y, dt), k2 = dm(d.z, dt);
            double *o = s2 + r3 * rw + me;
            o[0] = da(in.yb.x, half(k0));
            o[1] = da(in.yb.y, half(k1));
            o[2] = da(in.yb.z, half(k2));
            ac[0] = da(ac[0], div3(k0));
            ac[1] = da(ac[1], div3(k1));
            ac[2] = da(ac[2], div3(k2));
        };
        auto st3 = [&](const SIn &in, int r3, double *ac) {  // s3 = y + k, acc += k/3
            const V3 d = llg_rhs_vals<J2, H, DAMP>(in.s, in.nb, in.n2, a);
            const double k0 = dm(d.x, dt), k1 = dm(d.y, dt), k2 = dm(d.z, dt);
            double *o = s3 + r3 * rw + me;
            o[0] = da(in.yb.x, k0);
            o[1] = da(in.yb.y, k1);
            o[2] = da(in.yb.z, k2);
            ac[0] = da(ac[0], div3(k0));
            ac[1] = da(ac[1], div3(k1));
            ac[2] = da(ac[2], div3(k2));
        };
        auto st4 = [&](const SIn &in, int r, const double *ac) {  // acc + k/6, renormalised
            const V3 d = llg_rhs_vals<J2, H, DAMP>(in.s, in.nb, in.n2, a);
            const double k0 = dm(d.x, dt), k1 = dm(d.y, dt), k2 = dm(d.z, dt);
            const double o0 = da(ac[0], div6(k0));
            const double o1 = da(ac[1], div6(k1));
            const double o2 = da(ac[2], div6(k2));
            const double nrm = __dsqrt_rn(da(da(dm(o0, o0), dm(o1, o1)), dm(o2, o2)));
            if (store) {
                double *gp = yout + ((long)(R0 - 4 + r) * N + gcol) * K + 3L * (fbase + fl);
                gp[0] = dq(dm(a.spin_len, o0), nrm);
                gp[1] = dq(dm(a.spin_len, o1), nrm);
                gp[2] = dq(dm(a.spin_len, o2), nrm);
            }
        };

        double acc[5][3];  // row r's combination in acc[r % 5]
        __syncthreads();   // the previous piece is done with every buffer
        load_row(0, 0);
        cp_async_commit();
        // Iteration j with R = j % 5 known at compile time, so acc[] and the y
        // ring slots are static; m3 = j % 3 runs along, and the 3-row ring
        // slots of rows j - 1 .. j - 6 are its rotations (j-3, j-6: m3;
        // j-2, j-5: m3 + 1; j-1, j-4: m3 + 2, mod 3).  Valid rows: stage s on
        // relative rows s..rs+7-s.
        int m3 = 0;
        auto iter = [&](auto rc, int j) {
            constexpr int R = decltype(rc)::value;
            if (j >= J) return;  // uniform over the CTA
            const int a0 = m3, a1 = (m3 == 2) ? 0 : m3 + 1, a2 = (m3 == 0) ? 2 : m3 - 1;
            m3 = a1;
            cp_async_wait_all();
            __syncthreads();  // phase A: stage 1 on row j-1, stage 3 on row j-4
            if (comp) {
                const bool d1 = j >= 2 && j <= rs + 7, d3 = j >= 7;
                const int y_m2 = (j + 3) % 5, y_m1 = (j + 4) % 5, y_0 = j % 5, y_m4 = (j + 1) % 5;
                if (d1 && d3) {
                    const SIn i1 = ld(ybuf, y_m2, y_m1, y_0, -1), i3 = ld(s2, a1, a2, a0, y_m4);
                    st1(i1, a2, acc[(R + 4) % 5]);
                    st3(i3, a2, acc[(R + 1) % 5]);
                } else if (d1) {
                    st1(ld(ybuf, y_m2, y_m1, y_0, -1), a2, acc[(R + 4) % 5]);
                } else if (d3) {
                    st3(ld(s2, a1, a2, a0, y_m4), a2, acc[(R + 1) % 5]);
                }
            }
            __syncthreads();  // phase B: prefetch, stage 2 on row j-2, stage 4 on row j-5
            if (j + 1 <= rs + 7) load_row(j + 1, (R + 1) % 5);
            cp_async_commit();
            if (comp) {
                const bool d2 = j >= 4 && j <= rs + 7, d4 = j >= 9;
                const int y_m2 = (j + 3) % 5;
                if (d2 && d4) {
                    const SIn i2 = ld(s1, a0, a1, a2, y_m2), i4 = ld(s3, a0, a1, a2, -1);
                    st2(i2, a1, acc[(R + 3) % 5]);
                    st4(i4, j - 5, acc[R]);
                } else if (d2) {
                    st2(ld(s1, a0, a1, a2, y_m2), a1, acc[(R + 3) % 5]);
                } else if (d4) {
                    st4(ld(s3, a0, a1, a2, -1), j - 5, acc[R]);
                }
            }
        };
        for (int j0 = 0; j0 < J; j0 += 5) {
            iter(std::integral_constant<int, 0>{}, j0);
            iter(std::integral_constant<int, 1>{}, j0 + 1);
            iter(std::integral_constant<int, 2>{}, j0 + 2);
            iter(std::integral_constant<int, 3>{}, j0 + 3);
            iter(std::integral_constant<int, 4>{}, j0 + 4);
        }
    }
}

size_t stream_smem_bytes(const StreamGeom &g) {
    return (size_t)stream::ROWS * g.rw * sizeof(double);
}

template <bool J2, bool H, bool DAMP>
cudaError_t launch_stream_t(const LLGArgs &a, const double *y, double *yout, cudaStream_t st) {
    using namespace stream;
    auto k = llg_step_stream_kernel<J2, H, DAMP>;
    StreamGeom g;
    g.nb = (a.N + WC_MAX - 1) / WC_MAX;
    g.wc = ((a.N + g.nb - 1) / g.nb + 7) / 8 * 8;  // wt * SF is a whole number of warps
    g.wt = g.wc + 8;
    g.rw = g.wt * SF * 3;
    g.ng = (a.nc + SF - 1) / SF;
    const int threads = g.wt * SF;
    const size_t smem = stream_smem_bytes(g);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem)) !=
        cudaSuccess)
        return e;
    // One CTA per resident slot, each with an equal run of the rows of work
    // (at least MIN_RUN, so the 9-iteration fill of a piece stays small).
    const long total = (long)g.nb * g.ng * a.N;
    const long slots = (long)sms * (per_sm > 0 ? per_sm : 1);
    long run = (total + slots - 1) / slots;
    if (run < MIN_RUN) run = MIN_RUN;
    g.run = run;
    const long blocks = (total + run - 1) / run;
    if (blocks > 0x7fffffffL) return cudaErrorInvalidConfiguration;
    k<<<(unsigned)blocks, threads, smem, st>>>(a, g, y, yout);
    return cudaGetLastError();
}

cudaError_t launch_stream(const LLGArgs &a, const double *y, double *yout, cudaStream_t st) {
    if (a.f0 < 0 || a.nc < 1 || a.f0 + a.nc > a.nfile) return cudaErrorInvalidValue;
    const int sel = (a.use_j2 ? 4 : 0) | (a.use_h ? 2 : 0) | (a.use_damp ? 1 : 0);
    switch (sel) {
        case 0: return launch_stream_t<false, false, false>(a, y, yout, st);
        case 1: return launch_stream_t<false, false, true>(a, y, yout, st);
        case 2: return launch_stream_t<false, true, false>(a, y, yout, st);
        case 3: return launch_stream_t<false, true, true>(a, y, yout, st);
        case 4: return launch_stream_t<true, false, false>(a, y, yout, st);
        case 5: return launch_stream_t<true, false, true>(a, y, yout, st);
        case 6: return launch_stream_t<true, true, false>(a, y, yout, st);
        default: return launch_stream_t<true, true, true>(a, y, yout, st);
    }
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

bool llg_fused_fills(const LLGArgs &a) {
    using namespace stream;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    const long nb = (a.N + WC_MAX - 1) / WC_MAX, ng = (a.nc + SF - 1) / SF;
    const long slots = 2L * sms;  // two CTAs of the streamed step per SM
    return nb * ng * a.N >= 8 * slots;
}

cudaError_t launch_llg_step_fused(const LLGArgs &a, const double *y, double *yout,
                                  cudaStream_t st) {
    return launch_stream(a, y, yout, st);
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
