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
// r = x - q d is exact in one FMA, and RN(q + r * yinv) is RN(x/d).  Valid
// away from overflow and the subnormal range, which the RK4 increments never
// reach; zeros keep their sign.  Three FP64 operations instead of a
// division routine; tests compare it with __ddiv_rn bit for bit.
__device__ __forceinline__ double div3(double x) {
    constexpr double yinv = 1.0 / 3.0;  // RN(1/3), folded at compile time
    const double q = __dmul_rn(x, yinv);
    const double r = __fma_rn(-q, 3.0, x);
    return x == 0.0 ? x : __fma_rn(r, yinv, q);
}
__device__ __forceinline__ double div6(double x) {
    constexpr double yinv = 1.0 / 6.0;  // RN(1/6)
    const double q = __dmul_rn(x, yinv);
    const double r = __fma_rn(-q, 6.0, x);
    return x == 0.0 ? x : __fma_rn(r, yinv, q);
}

struct V3 {
    double x, y, z;
};

// dS/dt at one (site, replica).  y is indexed as y[site*sstride + off + c].
// Neighbour order and periodic wrap follow llg_sqt_baseline.c:59-77 with
// nn = {(1,0), (-1,0), (0,-1), (0,1)} (:175-178); the exchange field starts
// at 0 and accumulates t*J1 per neighbour (:52, :73-75); tau = H x S
// (v3d_cross, v3d.h:48-53).  Extensions, each skipped when zero: J2 over the
// diagonal neighbours (1,1), (1,-1), (-1,1), (-1,-1); the Zeeman field; and
// Gilbert damping g * (tau + alpha * (S x tau)).
template <bool J2, bool H, bool DAMP>
__device__ __forceinline__ V3 llg_rhs(const double *__restrict__ y, long sstride, long off,
                                      int N, int row, int col, const LLGArgs &a) {
    const int rp = (row + 1 == N) ? 0 : row + 1;
    const int rm = (row == 0) ? N - 1 : row - 1;
    const int cp = (col + 1 == N) ? 0 : col + 1;
    const int cm = (col == 0) ? N - 1 : col - 1;
    const long site = (long)row * N + col;
    const double *c0 = y + site * sstride + off;
    const double sx = c0[0], sy = c0[1], sz = c0[2];
    const long nb[4] = {(long)rp * N + col, (long)rm * N + col, (long)row * N + cm,
                        (long)row * N + cp};
    double ex = 0.0, ey = 0.0, ez = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double *t = y + nb[j] * sstride + off;
        ex = da(ex, dm(t[0], a.J1));
        ey = da(ey, dm(t[1], a.J1));
        ez = da(ez, dm(t[2], a.J1));
    }
    if (J2) {
        const long nn2[4] = {(long)rp * N + cp, (long)rp * N + cm, (long)rm * N + cp,
                             (long)rm * N + cm};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double *t = y + nn2[j] * sstride + off;
            ex = da(ex, dm(t[0], a.J2));
            ey = da(ey, dm(t[1], a.J2));
            ez = da(ez, dm(t[2], a.J2));
        }
    }
    if (H) {
        ex = da(ex, a.hx);
        ey = da(ey, a.hy);
        ez = da(ez, a.hz);
    }
    V3 tau;
    tau.x = ds(dm(ey, sz), dm(ez, sy));
    tau.y = ds(dm(ez, sx), dm(ex, sz));
    tau.z = ds(dm(ex, sy), dm(ey, sx));
    if (!DAMP) return tau;
    const double ux = ds(dm(sy, tau.z), dm(sz, tau.y));
    const double uy = ds(dm(sz, tau.x), dm(sx, tau.z));
    const double uz = ds(dm(sx, tau.y), dm(sy, tau.x));
    V3 d;
    d.x = dm(a.g, da(tau.x, dm(a.alpha, ux)));
    d.y = dm(a.g, da(tau.y, dm(a.alpha, uy)));
    d.z = dm(a.g, da(tau.z, dm(a.alpha, uz)));
    return d;
}

