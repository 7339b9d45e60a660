// batch.cu -- many independent lattices of different sizes and parameters in
// one persistent launch.  The reference runs one lattice per program; this is
// the B200 form of running an ensemble of them (e.g. different temperatures
// and dampings): all lattices' spins stay resident in L2 (FP32, a few MB),
// one cooperative kernel runs every RK4 step of every lattice, and a bounded
// grid barrier separates the four stages of a step.
//
// Arithmetic: the RK4 stages in FP32 with explicitly rounded operations in the
// reference's order (euler / runge_kutta, llg_sqt_baseline.c:29-142), the
// renormalisation in FP64 (norm and division), rounded to FP32 at the end.
// The CPU oracle restates the same FP32 arithmetic, so the comparison is bit
// for bit.
//
// Layout: lattice l occupies planes x, y, z of N_l * N_l floats at offset
// off_l (structure of arrays, one replica per lattice).  Work items are tiles
// of `tile` consecutive sites of one lattice; CTA b processes items b,
// b + grid, ...  The tile width and the CTAs per SM come from the autotuner.
#include <cooperative_groups.h>

#include <algorithm>
#include <type_traits>
#include <chrono>
#include <vector>

#include "asd_internal.h"

namespace asd {

struct BatchLattice {
    int N;
    long off;  // first float of plane x
    float J1, J2, alpha, g, hx, hy, hz, dt;
    double spin_len;
    int use_j2, use_h, use_damp;
};

namespace {

constexpr uint32_t BARRIER_LIMIT = 1u << 22;

__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
// x / d for the constants d = 3 and 6 in FP32, correctly rounded, by
// Markstein's correction step (P. Markstein, IBM J. Res. Dev. 34(1), 1990),
// as the FP64 forms of the LLG kernels: c = RN(1/d), q = RN(x c), the
// remainder q d - x is exact in one FMA, and RN(q - (q d - x) c) = RN(x/d).
// Outside 2^-100 <= |x| <= 2^100 (zeros, tiny and huge values, inf, NaN) the
// division itself.  asd_check_const_division_f32 compares it with __fdiv_rn
// over all 2^32 bit patterns.
__device__ __forceinline__ float fdiv_const(float x, float d, float c) {
    const float ax = fabsf(x);
    if (!(ax >= 0x1p-100f && ax <= 0x1p100f)) return __fdiv_rn(x, d);
    const float q = __fmul_rn(x, c);
    const float t = __fmaf_rn(q, d, -x);
    return __fmaf_rn(-t, c, q);
}
__device__ __forceinline__ float fd3(float x) { return fdiv_const(x, 3.f, 1.f / 3.f); }
__device__ __forceinline__ float fd6(float x) { return fdiv_const(x, 6.f, 1.f / 6.f); }

struct F3 {
    float x, y, z;
};

// Reads that follow a grid barrier must not hit stale L1 lines: L2 only.
__device__ __forceinline__ F3 ld3(const float *p, long M, long i) {
    return F3{__ldcg(p + i), __ldcg(p + M + i), __ldcg(p + 2 * M + i)};
}

// dS/dt from the centre s and the neighbours nb (nearest, in the reference's
// order (row+1), (row-1), (col-1), (col+1)) and n2 (diagonals (+1,+1),
// (+1,-1), (-1,+1), (-1,-1); read only with J2), FP32, explicitly rounded.
// Both batch kernels go through this function: one operation order.
template <bool J2, bool H, bool DAMP>
__device__ __forceinline__ F3 rhs32_vals_t(const F3 &s, const F3 (&nb)[4], const F3 (&n2)[4],
                                           const BatchLattice &L) {
    float ex = 0.f, ey = 0.f, ez = 0.f;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        ex = fa(ex, fm(nb[j].x, L.J1));
        ey = fa(ey, fm(nb[j].y, L.J1));
        ez = fa(ez, fm(nb[j].z, L.J1));
    }
    if (J2) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            ex = fa(ex, fm(n2[j].x, L.J2));
            ey = fa(ey, fm(n2[j].y, L.J2));
            ez = fa(ez, fm(n2[j].z, L.J2));
        }
    }
    if (H) {
        ex = fa(ex, L.hx);
        ey = fa(ey, L.hy);
        ez = fa(ez, L.hz);
    }
    F3 tau{fs(fm(ey, s.z), fm(ez, s.y)), fs(fm(ez, s.x), fm(ex, s.z)), fs(fm(ex, s.y), fm(ey, s.x))};
    if (!DAMP) return tau;
    const float ux = fs(fm(s.y, tau.z), fm(s.z, tau.y));
    const float uy = fs(fm(s.z, tau.x), fm(s.x, tau.z));
    const float uz = fs(fm(s.x, tau.y), fm(s.y, tau.x));
    return F3{fm(L.g, fa(tau.x, fm(L.alpha, ux))), fm(L.g, fa(tau.y, fm(L.alpha, uy))),
              fm(L.g, fa(tau.z, fm(L.alpha, uz)))};
}

__device__ __forceinline__ F3 rhs32_vals(const F3 &s, const F3 (&nb)[4], const F3 (&n2)[4],
                                         const BatchLattice &L) {
    switch ((L.use_j2 ? 4 : 0) | (L.use_h ? 2 : 0) | (L.use_damp ? 1 : 0)) {
        case 0: return rhs32_vals_t<false, false, false>(s, nb, n2, L);
        case 1: return rhs32_vals_t<false, false, true>(s, nb, n2, L);
        case 2: return rhs32_vals_t<false, true, false>(s, nb, n2, L);
        case 3: return rhs32_vals_t<false, true, true>(s, nb, n2, L);
        case 4: return rhs32_vals_t<true, false, false>(s, nb, n2, L);
        case 5: return rhs32_vals_t<true, false, true>(s, nb, n2, L);
        case 6: return rhs32_vals_t<true, true, false>(s, nb, n2, L);
        default: return rhs32_vals_t<true, true, true>(s, nb, n2, L);
    }
}

__device__ __forceinline__ F3 rhs32(const float *ys, const BatchLattice &L, long i) {
    const int N = L.N;
    const long M = (long)N * N;
    const int row = (int)(i / N), col = (int)(i - (long)row * N);
    const int rp = (row + 1 == N) ? 0 : row + 1, rm = (row == 0) ? N - 1 : row - 1;
    const int cp = (col + 1 == N) ? 0 : col + 1, cm = (col == 0) ? N - 1 : col - 1;
    const F3 s = ld3(ys, M, i);
    F3 nb[4], n2[4];
    nb[0] = ld3(ys, M, (long)rp * N + col);
    nb[1] = ld3(ys, M, (long)rm * N + col);
    nb[2] = ld3(ys, M, (long)row * N + cm);
    nb[3] = ld3(ys, M, (long)row * N + cp);
    if (L.use_j2) {
        n2[0] = ld3(ys, M, (long)rp * N + cp);
        n2[1] = ld3(ys, M, (long)rp * N + cm);
        n2[2] = ld3(ys, M, (long)rm * N + cp);
        n2[3] = ld3(ys, M, (long)rm * N + cm);
    }
    return rhs32_vals(s, nb, n2, L);
}

struct BarrierState {
    unsigned count;
    unsigned gen;
};

// Grid-wide barrier for a cooperative launch (all CTAs resident).  Bounded:
// after BARRIER_LIMIT polls the waiting CTA records a timeout in *status and
// every later barrier returns false at once.
__device__ bool grid_barrier(BarrierState *bs, unsigned nblocks, unsigned *status,
                             int *s_fail) {
    __syncthreads();
    if (threadIdx.x == 0 && !*s_fail) {
        volatile unsigned *vgen = &bs->gen;
        const unsigned g = *vgen;
        __threadfence();
        if (atomicAdd(&bs->count, 1u) == nblocks - 1) {
            atomicExch(&bs->count, 0u);
            __threadfence();
            atomicAdd(&bs->gen, 1u);
        } else {
            uint32_t i = 0;
            while (*vgen == g) {
                if (++i > BARRIER_LIMIT || (*(volatile unsigned *)status) != 0u) {
                    atomicOr(status, (unsigned)kStatusTimeout);
                    *s_fail = 1;
                    break;
                }
                if (i > 64) __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return !*s_fail;
}

struct Item {
    int lat;
    int first;  // first site
    int count;
};

// One persistent launch for nsteps steps of every lattice.
__global__ void __launch_bounds__(256, 4) batch_kernel(const BatchLattice *__restrict__ lats,
                                                    const Item *__restrict__ items, int nitems,
                                                    float *y, float *ysa, float *ysb, float *acc,
                                                    int nsteps, BarrierState *bs,
                                                    unsigned *status) {
    __shared__ int s_fail;
    if (threadIdx.x == 0) s_fail = 0;
    __syncthreads();
    for (int step = 0; step < nsteps; ++step) {
        for (int stage = 1; stage <= 4; ++stage) {
            const float *in = (stage == 1) ? y : (stage == 3 ? ysb : ysa);
            float *out = (stage == 2) ? ysb : (stage == 4 ? y : ysa);
            for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
                const Item w = items[it];
                if ((int)threadIdx.x >= w.count) continue;
                const BatchLattice L = lats[w.lat];
                const long M = (long)L.N * L.N;
                const long i = w.first + threadIdx.x;
                float *Y = y + L.off, *A = acc + L.off, *O = out + L.off;
                const float *I = in + L.off;
                const F3 d = rhs32(I, L, i);
                const float k0 = fm(d.x, L.dt), k1 = fm(d.y, L.dt), k2 = fm(d.z, L.dt);
                if (stage == 4) {
                    const double o0 = (double)fa(__ldcg(A + i), fd6(k0));
                    const double o1 = (double)fa(__ldcg(A + M + i), fd6(k1));
                    const double o2 = (double)fa(__ldcg(A + 2 * M + i), fd6(k2));
                    const double nrm = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(o0, o0),
                                                                      __dmul_rn(o1, o1)),
                                                            __dmul_rn(o2, o2)));
                    O[i] = __double2float_rn(__ddiv_rn(__dmul_rn(L.spin_len, o0), nrm));
                    O[M + i] = __double2float_rn(__ddiv_rn(__dmul_rn(L.spin_len, o1), nrm));
                    O[2 * M + i] = __double2float_rn(__ddiv_rn(__dmul_rn(L.spin_len, o2), nrm));
                } else {
                    const F3 yb = ld3(Y, M, i);
                    const F3 kk{k0, k1, k2};
                    F3 o;
                    if (stage == 3) o = F3{fa(yb.x, kk.x), fa(yb.y, kk.y), fa(yb.z, kk.z)};
                    else o = F3{fa(yb.x, fm(kk.x, 0.5f)), fa(yb.y, fm(kk.y, 0.5f)),
                                fa(yb.z, fm(kk.z, 0.5f))};
                    O[i] = o.x;
                    O[M + i] = o.y;
                    O[2 * M + i] = o.z;
                    if (stage == 1) {
                        A[i] = fa(yb.x, fd6(kk.x));
                        A[M + i] = fa(yb.y, fd6(kk.y));
                        A[2 * M + i] = fa(yb.z, fd6(kk.z));
                    } else {
                        A[i] = fa(__ldcg(A + i), fd3(kk.x));
                        A[M + i] = fa(__ldcg(A + M + i), fd3(kk.y));
                        A[2 * M + i] = fa(__ldcg(A + 2 * M + i), fd3(kk.z));
                    }
                }
            }
            if (!grid_barrier(bs, gridDim.x, status, &s_fail)) return;
        }
    }
}

// ------------------------------------------- cluster-resident batch kernel
// The lattices live in shared memory for the whole run.  Each lattice
// belongs to one thread-block cluster; its rows are split over the
// cluster's CTAs (a CTA may hold rows of several lattices, one segment per
// lattice).  A CTA keeps, as float planes (x, y, z), two stage buffers over
// its segments' rows plus one halo row above and below each segment (the
// stencil's inputs, ping-ponged by the four stages: y -> ys1 -> ys2 -> ys3
// -> y_new), and per site the RK4 base value and the running combination.
// After every stage the cluster synchronises (a hardware cluster barrier,
// the same control flow in every CTA) and each CTA copies its segments' two
// halo rows from the owning CTAs' shared memory (distributed shared memory),
// then synchronises its own threads.  Threads walk each segment row by row
// (thread t takes column t % N of rows t / N, t / N + T / N, ...), so a
// lattice's parameters and a site's column and wrap offsets are uniform or
// fixed per segment.  No grid-wide barrier and no global-memory traffic
// between the first load and the final store.
struct CSeg {
    int lat;       // lattice
    int N;         // its side
    int r0, rows;  // lattice rows [r0, r0 + rows)
    int base;      // slot of the top halo row; core row k at base + (k + 1) * N
    int core0;     // first site of the segment in the CTA's site numbering
    int top_rank, top_off, top_buf;  // top halo row (r0 - 1 mod N): owning CTA's
    int bot_rank, bot_off, bot_buf;  //   rank, slot in its planes, its plane length
};
struct CCta {
    int seg0, nseg;  // segments [seg0, seg0 + nseg)
    int nsites;      // core sites
    int buf;         // slots per plane
};
constexpr int CL_THREADS = 896;

__host__ __device__ constexpr size_t cluster_smem_floats(int buf, int sites) {
    return (size_t)6 * buf + (size_t)6 * sites;  // 2 x 3 planes, y base and combination
}

__global__ void __launch_bounds__(CL_THREADS, 1)
    batch_cluster_kernel(const BatchLattice *__restrict__ lats, const CCta *__restrict__ ctas,
                         const CSeg *__restrict__ segs, float *y, int nsteps) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ float cfs[];
    const CCta me = ctas[blockIdx.x];
    const int T = blockDim.x, tid = threadIdx.x, ns = me.nsites;
    // plane c of stage buffer b: cfs + (3 b + c) * buf; y base [3][ns]; combination [3][ns]
    auto plane = [&](int b, int c) { return cfs + (3 * b + c) * me.buf; };
    float *const yb = cfs + 6 * (size_t)me.buf;
    float *const ac = yb + 3 * (size_t)ns;

    for (int k = me.seg0; k < me.seg0 + me.nseg; ++k) {
        const CSeg sg = segs[k];
        const long M = (long)sg.N * sg.N;
        const float *Y = y + lats[sg.lat].off;
        for (int e = tid; e < sg.rows * sg.N; e += T) {
            const int row = e / sg.N, col = e - row * sg.N;
            const long i = (long)(sg.r0 + row) * sg.N + col;
            const int slot = sg.base + (row + 1) * sg.N + col, q = sg.core0 + e;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float v = Y[c * M + i];
                yb[c * ns + q] = v;
                plane(0, c)[slot] = v;
            }
        }
    }
    // halo rows of stage buffer b from the owning CTAs
    auto halo = [&](int b) {
        cluster.sync();
        for (int k = me.seg0; k < me.seg0 + me.nseg; ++k) {
            const CSeg sg = segs[k];
            const float *rt = cluster.map_shared_rank(cfs, sg.top_rank) + sg.top_off;
            const float *rb = cluster.map_shared_rank(cfs, sg.bot_rank) + sg.bot_off;
            for (int col = tid; col < sg.N; col += T) {
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    plane(b, c)[sg.base + col] = rt[(3 * b + c) * sg.top_buf + col];
                    plane(b, c)[sg.base + (sg.rows + 1) * sg.N + col] =
                        rb[(3 * b + c) * sg.bot_buf + col];
                }
            }
        }
        __syncthreads();
    };
    halo(0);

    auto stage = [&](auto sc) {
        constexpr int S = decltype(sc)::value;
        const float *ix = plane((S - 1) & 1, 0), *iy = plane((S - 1) & 1, 1),
                    *iz = plane((S - 1) & 1, 2);
        float *ox = plane(S & 1, 0), *oy = plane(S & 1, 1), *oz = plane(S & 1, 2);
        for (int k = me.seg0; k < me.seg0 + me.nseg; ++k) {
            const CSeg sg = segs[k];
            const BatchLattice L = lats[sg.lat];
            const int N = sg.N, rpp = T / N, r1 = tid / N, col = tid - r1 * N;
            if (r1 >= rpp) continue;  // the last T % N threads
            const int dl = (col == 0) ? N - 1 : -1, dr = (col == N - 1) ? 1 - N : 1;
            // the segment's rows with the lattice's model terms fixed at compile time
            auto rows_t = [&](auto j2c, auto hc, auto dc) {
                constexpr bool J2 = decltype(j2c)::value, H = decltype(hc)::value,
                               DAMP = decltype(dc)::value;
                for (int row = r1; row < sg.rows; row += rpp) {
                    const int c = sg.base + (row + 1) * N + col, q = sg.core0 + row * N + col;
                    auto at = [&](int o) { return F3{ix[o], iy[o], iz[o]}; };
                    F3 nb[4], n2[4];
                    nb[0] = at(c + N);
                    nb[1] = at(c - N);
                    nb[2] = at(c + dl);
                    nb[3] = at(c + dr);
                    if (J2) {
                        n2[0] = at(c + N + dr);
                        n2[1] = at(c + N + dl);
                        n2[2] = at(c - N + dr);
                        n2[3] = at(c - N + dl);
                    }
                    const F3 d = rhs32_vals_t<J2, H, DAMP>(at(c), nb, n2, L);
                    const float k0 = fm(d.x, L.dt), k1 = fm(d.y, L.dt), k2 = fm(d.z, L.dt);
                    if (S == 4) {
                        const double o0 = (double)fa(ac[q], fd6(k0));
                        const double o1 = (double)fa(ac[ns + q], fd6(k1));
                        const double o2 = (double)fa(ac[2 * ns + q], fd6(k2));
                        const double nrm = __dsqrt_rn(__dadd_rn(
                            __dadd_rn(__dmul_rn(o0, o0), __dmul_rn(o1, o1)), __dmul_rn(o2, o2)));
                        const float n0 = __double2float_rn(__ddiv_rn(__dmul_rn(L.spin_len, o0), nrm));
                        const float n1 = __double2float_rn(__ddiv_rn(__dmul_rn(L.spin_len, o1), nrm));
                        const float n2v =
                            __double2float_rn(__ddiv_rn(__dmul_rn(L.spin_len, o2), nrm));
                        yb[q] = ox[c] = n0;
                        yb[ns + q] = oy[c] = n1;
                        yb[2 * ns + q] = oz[c] = n2v;
                    } else {
                        const float bx = yb[q], by = yb[ns + q], bz = yb[2 * ns + q];
                        if (S == 3) {
                            ox[c] = fa(bx, k0);
                            oy[c] = fa(by, k1);
                            oz[c] = fa(bz, k2);
                        } else {
                            ox[c] = fa(bx, fm(k0, 0.5f));
                            oy[c] = fa(by, fm(k1, 0.5f));
                            oz[c] = fa(bz, fm(k2, 0.5f));
                        }
                        if (S == 1) {
                            ac[q] = fa(bx, fd6(k0));
                            ac[ns + q] = fa(by, fd6(k1));
                            ac[2 * ns + q] = fa(bz, fd6(k2));
                        } else {
                            ac[q] = fa(ac[q], fd3(k0));
                            ac[ns + q] = fa(ac[ns + q], fd3(k1));
                            ac[2 * ns + q] = fa(ac[2 * ns + q], fd3(k2));
                        }
                    }
                }
            };
            using TT = std::true_type;
            using FF = std::false_type;
            switch ((L.use_j2 ? 4 : 0) | (L.use_h ? 2 : 0) | (L.use_damp ? 1 : 0)) {
                case 0: rows_t(FF{}, FF{}, FF{}); break;
                case 1: rows_t(FF{}, FF{}, TT{}); break;
                case 2: rows_t(FF{}, TT{}, FF{}); break;
                case 3: rows_t(FF{}, TT{}, TT{}); break;
                case 4: rows_t(TT{}, FF{}, FF{}); break;
                case 5: rows_t(TT{}, FF{}, TT{}); break;
                case 6: rows_t(TT{}, TT{}, FF{}); break;
                default: rows_t(TT{}, TT{}, TT{}); break;
            }
        }
        halo(S & 1);
    };
    for (int step = 0; step < nsteps; ++step) {
        stage(std::integral_constant<int, 1>{});
        stage(std::integral_constant<int, 2>{});
        stage(std::integral_constant<int, 3>{});
        stage(std::integral_constant<int, 4>{});
    }
    // No CTA may exit while another CTA of its cluster can still read its
    // shared memory (the last halo copy).
    cluster.sync();
    for (int k = me.seg0; k < me.seg0 + me.nseg; ++k) {
        const CSeg sg = segs[k];
        const long M = (long)sg.N * sg.N;
        float *Y = y + lats[sg.lat].off;
        for (int e = tid; e < sg.rows * sg.N; e += T) {
            const int row = e / sg.N, col = e - row * sg.N;
            const long i = (long)(sg.r0 + row) * sg.N + col;
            const int q = sg.core0 + e;
            Y[i] = yb[q];
            Y[M + i] = yb[ns + q];
            Y[2 * M + i] = yb[2 * ns + q];
        }
    }
}

// One CTA waits at a grid barrier sized for two: nothing arrives for the
// second, so the bounded barrier must give up and record a timeout.
__global__ void grid_barrier_probe_kernel(BarrierState *bs, unsigned *status) {
    __shared__ int s_fail;
    if (threadIdx.x == 0) s_fail = 0;
    __syncthreads();
    grid_barrier(bs, 2u, status, &s_fail);
}

// Every 32-bit pattern x: counts those for which fd3 / fd6 differ from
// __fdiv_rn in any bit (NaN results count as equal).
__global__ void fdiv_const_check_kernel(unsigned long long *bad) {
    unsigned long long n = 0;
    for (unsigned long long u = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         u < (1ull << 32); u += (unsigned long long)gridDim.x * blockDim.x) {
        const float x = __uint_as_float((unsigned)u);
        const float a3 = fd3(x), b3 = __fdiv_rn(x, 3.f), a6 = fd6(x), b6 = __fdiv_rn(x, 6.f);
        const bool ok3 = __float_as_uint(a3) == __float_as_uint(b3) || (a3 != a3 && b3 != b3);
        const bool ok6 = __float_as_uint(a6) == __float_as_uint(b6) || (a6 != a6 && b6 != b6);
        n += !ok3 + !ok6;
    }
    if (n) atomicAdd(bad, n);
}

}  // namespace

cudaError_t launch_fdiv_const_check(unsigned long long *bad, cudaStream_t st) {
    fdiv_const_check_kernel<<<148 * 8, 256, 0, st>>>(bad);
    return cudaGetLastError();
}

cudaError_t launch_grid_barrier_probe(void *bs, unsigned *status, cudaStream_t st) {
    grid_barrier_probe_kernel<<<1, 32, 0, st>>>(static_cast<BarrierState *>(bs), status);
    return cudaGetLastError();
}

}  // namespace asd

using namespace asd;

struct asd_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<BatchLattice> lat;
    long total = 0;  // floats per buffer
    BatchLattice *d_lat = nullptr;
    float *y = nullptr, *ysa = nullptr, *ysb = nullptr, *acc = nullptr;
    BarrierState *bs = nullptr;
    unsigned *status = nullptr;
    Item *d_items = nullptr;
    int nitems = 0, tile = 0, ctas_per_sm = 0, grid = 0;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = -1;
    // kernel 0: the global-memory kernel (tile, ctas_per_sm); 1: the
    // cluster-resident kernel (cl_size CTAs per cluster, cl_count clusters)
    int kind = 0;
    int cl_size = 0, cl_count = 0, cl_threads = 0;
    size_t cl_smem = 0;
    CCta *d_ctas = nullptr;
    CSeg *d_segs = nullptr;
};

namespace {

int build_items(asd_batch *b, int tile) {
    std::vector<Item> items;
    for (int l = 0; l < (int)b->lat.size(); ++l) {
        const int M = b->lat[l].N * b->lat[l].N;
        for (int f = 0; f < M; f += tile) items.push_back(Item{l, f, std::min(tile, M - f)});
    }
    if (b->d_items) cudaFree(b->d_items);
    b->d_items = nullptr;
    ASD_CUDA_TRY(cudaMalloc(&b->d_items, items.size() * sizeof(Item)));
    ASD_CUDA_TRY(cudaMemcpy(b->d_items, items.data(), items.size() * sizeof(Item),
                            cudaMemcpyHostToDevice));
    b->nitems = (int)items.size();
    b->tile = tile;
    return ASD_OK;
}

int configure(asd_batch *b, int tile, int ctas_per_sm) {
    if (tile < 32 || tile > 256 || tile % 32) return fail(ASD_ERR_INVALID, "tile %d", tile);
    int occ = 0, sms = 0;
    ASD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, 256, 0));
    ASD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    if (ctas_per_sm < 1 || ctas_per_sm > occ)
        return fail(ASD_ERR_INVALID, "ctas_per_sm %d (at most %d resident)", ctas_per_sm, occ);
    int rc = build_items(b, tile);
    if (rc != ASD_OK) return rc;
    b->ctas_per_sm = ctas_per_sm;
    b->grid = std::min(sms * ctas_per_sm, b->nitems);
    b->kind = 0;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = -1;
    return ASD_OK;
}

// Cluster plan: lattices onto C clusters of S CTAs, longest first onto the
// least-loaded cluster; each cluster's rows (lattice after lattice) split
// over its CTAs by site count (a row goes to the CTA whose share holds the
// row's middle site); per CTA its segments laid out one after another, each
// with a halo row above and below.  False if a CTA would need more than
// smem_limit bytes or a lattice row is wider than a CTA's threads.
struct ClusterPlan {
    std::vector<CCta> ctas;
    std::vector<CSeg> segs;
    int max_sites = 0, max_buf = 0;
};

bool plan_clusters(const std::vector<BatchLattice> &lat, int S, int C, int max_sites,
                   size_t smem_limit, ClusterPlan &pl) {
    const int nl = (int)lat.size();
    std::vector<int> order(nl);
    for (int l = 0; l < nl; ++l) order[l] = l;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b2) { return lat[a].N > lat[b2].N; });
    std::vector<long> load(C, 0);
    std::vector<std::vector<int>> members(C);
    for (int l : order) {
        const int c = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        members[c].push_back(l);
        load[c] += (long)lat[l].N * lat[l].N;
    }
    for (const BatchLattice &L : lat)
        if (L.N > CL_THREADS) return false;  // a row per thread pass
    pl.ctas.assign((size_t)C * S, CCta{0, 0, 0, 1});
    pl.segs.clear();
    pl.max_sites = pl.max_buf = 0;
    for (int c = 0; c < C; ++c) {
        std::vector<std::vector<CSeg>> cs(S);
        long acc = 0;
        int r = 0;
        for (int l : members[c]) {
            const int N = lat[l].N;
            for (int row = 0; row < N; ++row) {
                while (r < S - 1 && 2 * (acc + N / 2) >= 2 * (long)(r + 1) * load[c] / S) ++r;
                std::vector<CSeg> &v = cs[r];
                if (!v.empty() && v.back().lat == l && v.back().r0 + v.back().rows == row) {
                    ++v.back().rows;
                } else {
                    CSeg sg{};
                    sg.lat = l;
                    sg.N = N;
                    sg.r0 = row;
                    sg.rows = 1;
                    v.push_back(sg);
                }
                acc += N;
            }
        }
        for (int k = 0; k < S; ++k) {  // layout
            int base = 0, core = 0;
            for (CSeg &sg : cs[k]) {
                sg.base = base;
                sg.core0 = core;
                base += (sg.rows + 2) * sg.N;
                core += sg.rows * sg.N;
            }
            CCta &ct = pl.ctas[(size_t)c * S + k];
            ct.nsites = core;
            ct.buf = base > 0 ? base : 1;
            pl.max_sites = std::max(pl.max_sites, core);
            pl.max_buf = std::max(pl.max_buf, ct.buf);
        }
        // halo sources: the CTA and slot holding row `want` of lattice l
        auto find = [&](int l, int want, int &rank, int &off, int &bufsz) {
            for (int k = 0; k < S; ++k)
                for (const CSeg &sg : cs[k])
                    if (sg.lat == l && want >= sg.r0 && want < sg.r0 + sg.rows) {
                        rank = k;
                        off = sg.base + (want - sg.r0 + 1) * sg.N;
                        bufsz = pl.ctas[(size_t)c * S + k].buf;
                        return;
                    }
        };
        for (int k = 0; k < S; ++k) {
            CCta &ct = pl.ctas[(size_t)c * S + k];
            ct.seg0 = (int)pl.segs.size();
            ct.nseg = (int)cs[k].size();
            for (CSeg sg : cs[k]) {
                find(sg.lat, (sg.r0 - 1 + sg.N) % sg.N, sg.top_rank, sg.top_off, sg.top_buf);
                find(sg.lat, (sg.r0 + sg.rows) % sg.N, sg.bot_rank, sg.bot_off, sg.bot_buf);
                pl.segs.push_back(sg);
            }
        }
    }
    (void)max_sites;
    return cluster_smem_floats(pl.max_buf, pl.max_sites) * sizeof(float) <= smem_limit;
}

cudaError_t launch_cluster(const asd_batch *b, int nsteps, bool query_only = false,
                           int *active = nullptr) {
    auto k = batch_cluster_kernel;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)b->cl_smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(b->cl_count * b->cl_size));
    cfg.blockDim = dim3((unsigned)b->cl_threads);
    cfg.dynamicSmemBytes = b->cl_smem;
    cfg.stream = b->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)b->cl_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (query_only) return cudaOccupancyMaxActiveClusters(active, k, &cfg);
    return cudaLaunchKernelEx(&cfg, k, (const BatchLattice *)b->d_lat, (const CCta *)b->d_ctas,
                              (const CSeg *)b->d_segs, b->y, nsteps);
}

int configure_cluster(asd_batch *b, int S, int threads) {
    if (S < 1 || S > 8) return fail(ASD_ERR_INVALID, "cluster size %d (1..8)", S);
    if (threads == 0) threads = CL_THREADS;
    if (threads < 128 || threads > CL_THREADS || threads % 32)
        return fail(ASD_ERR_INVALID, "threads %d (128..%d, a multiple of 32)", threads, CL_THREADS);
    int sms = 0, smem_optin = 0;
    ASD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    ASD_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                        b->device));
    int C = sms / S;
    ClusterPlan pl;
    for (;;) {
        if (C < 1 || !plan_clusters(b->lat, S, C, 0, (size_t)smem_optin, pl) ||
            [&] { for (const BatchLattice &L : b->lat) if (L.N > threads) return true; return false; }())
            return fail(ASD_ERR_UNSUPPORTED,
                        "the batch does not fit in shared memory with clusters of %d CTAs", S);
        b->cl_size = S;
        b->cl_count = C;
        b->cl_threads = threads;
        b->cl_smem = cluster_smem_floats(pl.max_buf, pl.max_sites) * sizeof(float);
        int active = 0;
        ASD_CUDA_TRY(launch_cluster(b, 0, true, &active));
        if (active >= C) break;
        C = active;  // every cluster resident at once: fewer, larger clusters
    }
    if (b->d_ctas) cudaFree(b->d_ctas);
    if (b->d_segs) cudaFree(b->d_segs);
    b->d_ctas = nullptr;
    b->d_segs = nullptr;
    ASD_CUDA_TRY(cudaMalloc(&b->d_ctas, pl.ctas.size() * sizeof(CCta)));
    ASD_CUDA_TRY(cudaMalloc(&b->d_segs, std::max<size_t>(1, pl.segs.size()) * sizeof(CSeg)));
    ASD_CUDA_TRY(cudaMemcpy(b->d_ctas, pl.ctas.data(), pl.ctas.size() * sizeof(CCta),
                            cudaMemcpyHostToDevice));
    if (!pl.segs.empty())
        ASD_CUDA_TRY(cudaMemcpy(b->d_segs, pl.segs.data(), pl.segs.size() * sizeof(CSeg),
                                cudaMemcpyHostToDevice));
    b->kind = 1;
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
    b->graph_steps = -1;
    return ASD_OK;
}

int launch(asd_batch *b, int nsteps) {
    if (b->kind == 1) {
        ASD_CUDA_TRY(launch_cluster(b, nsteps));
        return ASD_OK;
    }
    // cooperative: every CTA resident, which the grid barrier relies on
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(b->grid);
    cfg.blockDim = dim3(256);
    cfg.stream = b->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ASD_CUDA_TRY(cudaLaunchKernelEx(&cfg, batch_kernel, (const BatchLattice *)b->d_lat,
                                    (const Item *)b->d_items, b->nitems, b->y, b->ysa, b->ysb,
                                    b->acc, nsteps, b->bs, b->status));
    return ASD_OK;
}

int run(asd_batch *b, int nsteps) {
    // one persistent launch, captured once per step count in a CUDA graph
    if (!b->graph || b->graph_steps != nsteps) {
        if (b->graph) cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
        cudaStream_t cap = b->stream;
        bool own = false;
        if (!cap) {  // capture needs a non-default stream
            ASD_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
            own = true;
        }
        cudaGraph_t g = nullptr;
        ASD_CUDA_TRY(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
        cudaStream_t saved = b->stream;
        b->stream = cap;
        const int rc = launch(b, nsteps);
        b->stream = saved;
        const cudaError_t e = cudaStreamEndCapture(cap, &g);
        if (own) cudaStreamDestroy(cap);
        if (rc != ASD_OK) return rc;
        ASD_CUDA_TRY(e);
        const cudaError_t ei = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        ASD_CUDA_TRY(ei);
        b->graph_steps = nsteps;
    }
    ASD_CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
    return ASD_OK;
}

int check_status(asd_batch *b) {
    unsigned st = 0;
    ASD_CUDA_TRY(cudaMemcpyAsync(&st, b->status, sizeof st, cudaMemcpyDeviceToHost, b->stream));
    ASD_CUDA_TRY(cudaMemsetAsync(b->status, 0, sizeof(unsigned), b->stream));
    ASD_CUDA_TRY(cudaMemsetAsync(b->bs, 0, sizeof(BarrierState), b->stream));
    ASD_CUDA_TRY(cudaStreamSynchronize(b->stream));
    if (st) return fail(ASD_ERR_TIMEOUT, "the batch kernel's grid barrier gave up (status %u)", st);
    return ASD_OK;
}

void destroy(asd_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    void *p[] = {b->d_lat, b->y, b->ysa, b->ysb, b->acc, b->bs, b->status, b->d_items,
                 b->d_ctas, b->d_segs};
    for (void *q : p)
        if (q) cudaFree(q);
    delete b;
}

}  // namespace

extern "C" {

int asd_batch_create(const asd_lattice *lats, int count, asd_batch **out) {
    if (!out || !lats || count < 1) return fail(ASD_ERR_INVALID, "bad argument");
    *out = nullptr;
    asd_batch *b = new asd_batch();
    cudaError_t e = cudaGetDevice(&b->device);
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "cudaGetDevice");
    }
    long off = 0;
    for (int l = 0; l < count; ++l) {
        const asd_lattice &p = lats[l];
        if (p.N < 3 || p.N > 4096 || !(p.spin_len > 0)) {
            delete b;
            return fail(ASD_ERR_INVALID, "lattice %d: N=%d spin_len=%g", l, p.N, p.spin_len);
        }
        BatchLattice L;
        L.N = p.N;
        L.off = off;
        L.J1 = (float)p.J1, L.J2 = (float)p.J2, L.alpha = (float)p.alpha;
        L.g = (float)(1.0 / (1.0 + (double)(float)p.alpha * (double)(float)p.alpha));
        L.hx = (float)p.hx, L.hy = (float)p.hy, L.hz = (float)p.hz, L.dt = (float)p.dt;
        L.spin_len = p.spin_len;
        L.use_j2 = p.J2 != 0.0;
        L.use_h = (p.hx != 0.0 || p.hy != 0.0 || p.hz != 0.0);
        L.use_damp = p.alpha != 0.0;
        b->lat.push_back(L);
        off += 3L * p.N * p.N;
    }
    b->total = off;
    const size_t bytes = (size_t)off * sizeof(float);
    int rc = ASD_OK;
    if (cudaMalloc(&b->d_lat, count * sizeof(BatchLattice)) != cudaSuccess ||
        cudaMalloc(&b->y, bytes) != cudaSuccess || cudaMalloc(&b->ysa, bytes) != cudaSuccess ||
        cudaMalloc(&b->ysb, bytes) != cudaSuccess || cudaMalloc(&b->acc, bytes) != cudaSuccess ||
        cudaMalloc(&b->bs, sizeof(BarrierState)) != cudaSuccess ||
        cudaMalloc(&b->status, sizeof(unsigned)) != cudaSuccess) {
        cudaGetLastError();
        destroy(b);
        return fail(ASD_ERR_NOMEM, "cudaMalloc for the batch failed");
    }
    e = cudaMemcpy(b->d_lat, b->lat.data(), count * sizeof(BatchLattice),
                   cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(b->bs, 0, sizeof(BarrierState));
    if (e == cudaSuccess) e = cudaMemset(b->status, 0, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(b->y, 0, bytes);
    if (e != cudaSuccess) {
        destroy(b);
        return cuda_fail(e, "batch set-up copies");
    }
    if ((rc = configure(b, 128, 2)) != ASD_OK) {
        destroy(b);
        return rc;
    }
    *out = b;
    return ASD_OK;
}

int asd_batch_destroy(asd_batch *b) {
    destroy(b);
    return ASD_OK;
}

int asd_batch_set_stream(asd_batch *b, void *stream) {
    if (!b) return fail(ASD_ERR_INVALID, "batch is NULL");
    b->stream = (cudaStream_t)stream;
    return ASD_OK;
}

int asd_batch_set_spins(asd_batch *b, int lattice, const float *spin_aos) {
    if (!b || !spin_aos || lattice < 0 || lattice >= (int)b->lat.size())
        return fail(ASD_ERR_INVALID, "bad argument");
    ASD_CUDA_TRY(cudaSetDevice(b->device));
    const BatchLattice &L = b->lat[lattice];
    const long M = (long)L.N * L.N;
    std::vector<float> soa((size_t)3 * M);
    for (long i = 0; i < M; ++i)
        for (int c = 0; c < 3; ++c) soa[c * M + i] = spin_aos[3 * i + c];
    ASD_CUDA_TRY(cudaMemcpy(b->y + L.off, soa.data(), soa.size() * sizeof(float),
                            cudaMemcpyHostToDevice));
    return ASD_OK;
}

int asd_batch_get_spins(asd_batch *b, int lattice, float *spin_aos) {
    if (!b || !spin_aos || lattice < 0 || lattice >= (int)b->lat.size())
        return fail(ASD_ERR_INVALID, "bad argument");
    ASD_CUDA_TRY(cudaSetDevice(b->device));
    ASD_CUDA_TRY(cudaStreamSynchronize(b->stream));
    const BatchLattice &L = b->lat[lattice];
    const long M = (long)L.N * L.N;
    std::vector<float> soa((size_t)3 * M);
    ASD_CUDA_TRY(cudaMemcpy(soa.data(), b->y + L.off, soa.size() * sizeof(float),
                            cudaMemcpyDeviceToHost));
    for (long i = 0; i < M; ++i)
        for (int c = 0; c < 3; ++c) spin_aos[3 * i + c] = soa[c * M + i];
    return ASD_OK;
}

int asd_batch_run(asd_batch *b, int nsteps) {
    if (!b || nsteps < 0) return fail(ASD_ERR_INVALID, "bad argument");
    if (nsteps == 0) return ASD_OK;
    ASD_CUDA_TRY(cudaSetDevice(b->device));
    int rc = run(b, nsteps);
    if (rc != ASD_OK) return rc;
    return check_status(b);
}

int asd_batch_configure(asd_batch *b, int tile, int ctas_per_sm) {
    if (!b) return fail(ASD_ERR_INVALID, "batch is NULL");
    ASD_CUDA_TRY(cudaSetDevice(b->device));
    return configure(b, tile, ctas_per_sm);
}

int asd_batch_configure_cluster(asd_batch *b, int cluster_size, int threads) {
    if (!b) return fail(ASD_ERR_INVALID, "batch is NULL");
    ASD_CUDA_TRY(cudaSetDevice(b->device));
    return configure_cluster(b, cluster_size, threads);
}

int asd_batch_autotune(asd_batch *b, int trial_steps, int *tile, int *ctas_per_sm,
                       double *ms_per_step) {
    if (!b || trial_steps < 1) return fail(ASD_ERR_INVALID, "bad argument");
    ASD_CUDA_TRY(cudaSetDevice(b->device));
    int occ = 0;
    ASD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, batch_kernel, 256, 0));
    // the trials advance the spins: keep a copy and restore it afterwards
    const size_t bytes = (size_t)b->total * sizeof(float);
    float *save = nullptr;
    ASD_CUDA_TRY(cudaMalloc(&save, bytes));
    cudaMemcpyAsync(save, b->y, bytes, cudaMemcpyDeviceToDevice, b->stream);
    double best = 1e300;
    int bt = 128, bc = 1, bthreads = 0;  // bt = 0: cluster kernel, bc = cluster size
    const int tiles[] = {32, 64, 128, 256};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int rc = ASD_OK;
    // the cluster-resident kernel, where the batch fits in shared memory
    for (int S = 1; S <= 8; ++S) {
        for (int threads : {256, 384, 512, 640, 768, CL_THREADS}) {
            if (configure_cluster(b, S, threads) != ASD_OK) continue;  // does not fit
            if ((rc = asd_batch_run(b, trial_steps)) != ASD_OK) break;  // captures and warms
            cudaEventRecord(e0, b->stream);
            if ((rc = run(b, trial_steps)) != ASD_OK) break;
            cudaEventRecord(e1, b->stream);
            if ((rc = check_status(b)) != ASD_OK) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) best = ms, bt = 0, bc = S, bthreads = threads;
        }
        if (rc != ASD_OK) break;
    }
    for (int t : tiles) {
        if (rc != ASD_OK) break;
        for (int c = 1; c <= std::min(occ, 8); c *= 2) {
            if ((rc = configure(b, t, c)) != ASD_OK) break;
            if ((rc = asd_batch_run(b, trial_steps)) != ASD_OK) break;  // captures and warms
            cudaEventRecord(e0, b->stream);
            if ((rc = run(b, trial_steps)) != ASD_OK) break;
            cudaEventRecord(e1, b->stream);
            if ((rc = check_status(b)) != ASD_OK) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) best = ms, bt = t, bc = c;
        }
        if (rc != ASD_OK) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemcpyAsync(b->y, save, bytes, cudaMemcpyDeviceToDevice, b->stream);
    cudaStreamSynchronize(b->stream);
    cudaFree(save);
    if (rc != ASD_OK) return rc;
    if ((rc = bt == 0 ? configure_cluster(b, bc, bthreads) : configure(b, bt, bc)) != ASD_OK)
        return rc;
    if (tile) *tile = bt;
    if (ctas_per_sm) *ctas_per_sm = bc;
    if (ms_per_step) *ms_per_step = best / trial_steps;
    return ASD_OK;
}

}  // extern "C"

extern "C" int asd_batch_plan_clusters(const int *sizes, int count, int cluster_size,
                                       int clusters, long smem_limit, int *ctas_out,
                                       int *segs_out, int seg_capacity, int *nsegs,
                                       long *smem_bytes) {
    using namespace asd;
    if (!sizes || count < 1 || cluster_size < 1 || cluster_size > 8 || clusters < 1 ||
        smem_limit < 0 || !ctas_out || !nsegs || !smem_bytes || seg_capacity < 0)
        return fail(ASD_ERR_INVALID, "bad argument");
    std::vector<BatchLattice> lat((size_t)count);
    for (int l = 0; l < count; ++l) {
        if (sizes[l] < 1) return fail(ASD_ERR_INVALID, "lattice %d: N=%d", l, sizes[l]);
        lat[l] = BatchLattice{};
        lat[l].N = sizes[l];
    }
    ClusterPlan pl;
    const bool fits = plan_clusters(lat, cluster_size, clusters, 0, (size_t)smem_limit, pl);
    *nsegs = (int)pl.segs.size();
    *smem_bytes = (long)(cluster_smem_floats(pl.max_buf, pl.max_sites) * sizeof(float));
    for (size_t i = 0; i < pl.ctas.size(); ++i) {
        const CCta &c = pl.ctas[i];
        const int v[4] = {c.seg0, c.nseg, c.nsites, c.buf};
        for (int k = 0; k < 4; ++k) ctas_out[4 * i + k] = v[k];
    }
    if (segs_out && (int)pl.segs.size() <= seg_capacity) {
        for (size_t i = 0; i < pl.segs.size(); ++i) {
            const CSeg &g = pl.segs[i];
            const int v[12] = {g.lat, g.N, g.r0, g.rows, g.base, g.core0,
                               g.top_rank, g.top_off, g.top_buf, g.bot_rank, g.bot_off, g.bot_buf};
            for (int k = 0; k < 12; ++k) segs_out[12 * i + k] = v[k];
        }
    }
    if (!fits) return fail(ASD_ERR_UNSUPPORTED, "the plan does not fit the limits");
    return ASD_OK;
}

extern "C" int asd_check_const_division_f32(unsigned long long *bad, void *stream) {
    using namespace asd;
    if (!bad) return fail(ASD_ERR_INVALID, "bad is NULL");
    ASD_CUDA_TRY(launch_fdiv_const_check(bad, (cudaStream_t)stream));
    return ASD_OK;
}

extern "C" int asd_check_bounded_wait(int which, unsigned limit, void *stream) {
    using namespace asd;
    if (which != 0 && which != 1) return fail(ASD_ERR_INVALID, "which must be 0 or 1");
    cudaStream_t st = (cudaStream_t)stream;
    unsigned *d = nullptr;  // status word + a barrier state
    ASD_CUDA_TRY(cudaMalloc(&d, 4 * sizeof(unsigned)));
    cudaError_t e = cudaMemsetAsync(d, 0, 4 * sizeof(unsigned), st);
    if (e == cudaSuccess)
        e = which == 0 ? launch_mbar_timeout_probe(limit, d, st)
                       : launch_grid_barrier_probe(d + 2, d, st);
    unsigned h = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "bounded-wait probe");
    if (h & kStatusTimeout) return fail(ASD_ERR_TIMEOUT, "the probe's wait gave up as designed");
    return ASD_OK;
}
