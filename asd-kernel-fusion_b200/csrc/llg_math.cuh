// llg_math.cuh -- the LLG right-hand side and the explicitly rounded FP64
// helpers shared by the forward kernels (llg_kernels.cu) and the adjoint
// (adjoint.cu).  Included inside an anonymous namespace of each file.
#pragma once

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dq(double a, double b) { return __ddiv_rn(a, b); }
// x / 2: the product by 0.5 is the same correctly rounded value (2 is a power
// of the radix), without a division.
__device__ __forceinline__ double half(double x) { return __dmul_rn(x, 0.5); }

// x / d for the constants d = 3 and 6, correctly rounded, by Markstein's
// correction step (P. Markstein, IBM J. Res. Dev. 34(1), 1990): with
// yinv = RN(1/d), q = RN(x * yinv) is within one ulp of x/d, the remainder
// x - q d is exact in one FMA, and RN(q + (x - q d) * yinv) is RN(x/d).  The
// remainder is formed as -(q d - x): for x != 0 that is the same exact value
// (a zero remainder is absorbed by q != 0), and for x = +-0 it makes the
// result +-0, so zeros keep their sign without a compare.  Valid away from
// overflow and the subnormal range, which the RK4 increments never reach.
// Three FP64 operations instead of a division routine; tests compare it
// with __ddiv_rn bit for bit.
__device__ __forceinline__ double div3(double x) {
    constexpr double yinv = 1.0 / 3.0;  // RN(1/3), folded at compile time
    const double q = __dmul_rn(x, yinv);
    const double t = __fma_rn(q, 3.0, -x);
    return __fma_rn(-t, yinv, q);
}
__device__ __forceinline__ double div6(double x) {
    constexpr double yinv = 1.0 / 6.0;  // RN(1/6)
    const double q = __dmul_rn(x, yinv);
    const double t = __fma_rn(q, 6.0, -x);
    return __fma_rn(-t, yinv, q);
}

struct V3 {
    double x, y, z;
};

// dS/dt from the centre spin s and its neighbours' values nb (nearest, in the
// reference's order) and n2 (diagonal; read only when J2).  The exchange field
// starts at 0 and accumulates t*J1 per neighbour (llg_sqt_baseline.c:52,
// :73-75); tau = H x S (v3d_cross, v3d.h:48-53).  Extensions, each skipped
// when zero: J2 over the diagonal neighbours, the Zeeman field, and Gilbert
// damping g * (tau + alpha * (S x tau)).  Every kernel that evaluates the
// right-hand side goes through this function, so all share one operation order.
template <bool J2, bool H, bool DAMP>
__device__ __forceinline__ V3 llg_rhs_vals(const V3 &s, const V3 (&nb)[4], const V3 (&n2)[4],
                                           const LLGArgs &a) {
    double ex = 0.0, ey = 0.0, ez = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        ex = da(ex, dm(nb[j].x, a.J1));
        ey = da(ey, dm(nb[j].y, a.J1));
        ez = da(ez, dm(nb[j].z, a.J1));
    }
    if (J2) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            ex = da(ex, dm(n2[j].x, a.J2));
            ey = da(ey, dm(n2[j].y, a.J2));
            ez = da(ez, dm(n2[j].z, a.J2));
        }
    }
    if (H) {
        ex = da(ex, a.hx);
        ey = da(ey, a.hy);
        ez = da(ez, a.hz);
    }
    V3 tau;
    tau.x = ds(dm(ey, s.z), dm(ez, s.y));
    tau.y = ds(dm(ez, s.x), dm(ex, s.z));
    tau.z = ds(dm(ex, s.y), dm(ey, s.x));
    if (!DAMP) return tau;
    const double ux = ds(dm(s.y, tau.z), dm(s.z, tau.y));
    const double uy = ds(dm(s.z, tau.x), dm(s.x, tau.z));
    const double uz = ds(dm(s.x, tau.y), dm(s.y, tau.x));
    V3 d;
    d.x = dm(a.g, da(tau.x, dm(a.alpha, ux)));
    d.y = dm(a.g, da(tau.y, dm(a.alpha, uy)));
    d.z = dm(a.g, da(tau.z, dm(a.alpha, uz)));
    return d;
}

// Periodic neighbour sites of (row, col): nearest in the reference's order
// (1,0), (-1,0), (0,-1), (0,1) and diagonal (1,1), (1,-1), (-1,1), (-1,-1).
__device__ __forceinline__ void neighbour_sites(int N, int row, int col, long (&nb)[4],
                                                long (&n2)[4]) {
    const int rp = (row + 1 == N) ? 0 : row + 1;
    const int rm = (row == 0) ? N - 1 : row - 1;
    const int cp = (col + 1 == N) ? 0 : col + 1;
    const int cm = (col == 0) ? N - 1 : col - 1;
    nb[0] = (long)rp * N + col;
    nb[1] = (long)rm * N + col;
    nb[2] = (long)row * N + cm;
    nb[3] = (long)row * N + cp;
    n2[0] = (long)rp * N + cp;
    n2[1] = (long)rp * N + cm;
    n2[2] = (long)rm * N + cp;
    n2[3] = (long)rm * N + cm;
}

// dS/dt at one (site, replica).  y is indexed as y[site*sstride + off + c].
// Neighbour order and periodic wrap follow llg_sqt_baseline.c:59-77 with
// nn = {(1,0), (-1,0), (0,-1), (0,1)} (:175-178).
template <bool J2, bool H, bool DAMP>
__device__ __forceinline__ V3 llg_rhs(const double *__restrict__ y, long sstride, long off,
                                      int N, int row, int col, const LLGArgs &a) {
    long nbs[4], n2s[4];
    neighbour_sites(N, row, col, nbs, n2s);
    const double *c0 = y + ((long)row * N + col) * sstride + off;
    const V3 s{c0[0], c0[1], c0[2]};
    V3 nb[4], n2[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double *t = y + nbs[j] * sstride + off;
        nb[j] = V3{t[0], t[1], t[2]};
    }
    if (J2) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double *t = y + n2s[j] * sstride + off;
            n2[j] = V3{t[0], t[1], t[2]};
        }
    }
    return llg_rhs_vals<J2, H, DAMP>(s, nb, n2, a);
}
