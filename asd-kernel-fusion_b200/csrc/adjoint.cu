// adjoint.cu -- kernels of the reverse-mode gradient of an S(q,t)-mismatch
// loss with respect to the model parameters (J1, J2, alpha, hx, hy, hz).
// The reference has no gradient; this is the adjoint of its forward step
// (euler + runge_kutta + renormalisation, llg_sqt_baseline.c:29-142,
// :298-309) extended by damping, Zeeman field and J2.  The schedule
// (checkpoints, recomputation, stage order) is in ctx.cu.
//
// Forward, per (site, replica):  f(S) = g (tau + alpha S x tau),
// tau = H x S, H = J1 sum_nn S + J2 sum_nnn S + h, g = 1/(1+alpha^2).
// For an adjoint mu of f, with nu = g (mu + alpha mu x S):
//   d/dS_i (local)  = g alpha (tau x mu) + nu x H
//   d/dH_i          = P_i = S_i x nu,  flowing to the neighbours as
//                     J1 sum_nn P + J2 sum_nnn P (the lattice is symmetric)
//   d/dJ1 = P . sum_nn S,  d/dJ2 = P . sum_nnn S,  d/dh = P,
//   d/dalpha = mu . (-2 alpha g f + g S x tau).
// Renormalisation y = l v/|v| has the symmetric Jacobian (l/|v|)(I - v^ v^T).
// S(q,t) = (1/(M nfile)) sum_k F_k (G_k - Z_c(k)) with F_k = sum_i u_i A_ik,
// G_k = sum_j w_j B_jk, Z_c = (1/nfile) sum_f G_(f,c) -- the correlation GEMM's
// value in factorised form -- so dS/dA_ik = u_i (G_k - Z_c(k)) / (M nfile).
#include "asd_internal.h"

namespace asd {
namespace {

#include "llg_math.cuh"

__device__ __forceinline__ V3 v3(double x, double y, double z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 vmul(double s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 vcross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 vload(const double *p) { return v3(p[0], p[1], p[2]); }
__device__ __forceinline__ void vstore(double *p, V3 a) {
    p[0] = a.x;
    p[1] = a.y;
    p[2] = a.z;
}

constexpr int NPAR = 6;  // J1, J2, alpha, hx, hy, hz
constexpr int TPB = 256;

struct Site {
    long e;  // element offset of (site, replica)
    long sstride, off;
    int row, col;
};

__device__ __forceinline__ bool site_of(const LLGArgs &a, Site &s) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.M * a.nfile) return false;
    const long site = t / a.nfile;
    const int f = (int)(t - site * a.nfile);
    s.row = (int)(site / a.N);
    s.col = (int)(site - (long)s.row * a.N);
    s.sstride = 3L * a.nfile;
    s.off = 3L * f;
    s.e = site * s.sstride + s.off;
    return true;
}

// Sums of a field over the 4 nearest and the 4 diagonal neighbours.
__device__ __forceinline__ void neighbour_sums(const double *y, const Site &s, int N, V3 &nn,
                                               V3 &nnn) {
    const int rp = (s.row + 1 == N) ? 0 : s.row + 1, rm = (s.row == 0) ? N - 1 : s.row - 1;
    const int cp = (s.col + 1 == N) ? 0 : s.col + 1, cm = (s.col == 0) ? N - 1 : s.col - 1;
    auto at = [&](int r, int c) { return vload(y + ((long)r * N + c) * s.sstride + s.off); };
    nn = vadd(vadd(at(rp, s.col), at(rm, s.col)), vadd(at(s.row, cm), at(s.row, cp)));
    nnn = vadd(vadd(at(rp, cp), at(rp, cm)), vadd(at(rm, cp), at(rm, cm)));
}

__device__ __forceinline__ void block_add(double (&v)[NPAR], double *acc) {
    __shared__ double red[NPAR][TPB];
#pragma unroll
    for (int q = 0; q < NPAR; ++q) red[q][threadIdx.x] = v[q];
    __syncthreads();
    for (int w = TPB / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
#pragma unroll
            for (int q = 0; q < NPAR; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < NPAR) acc[(long)blockIdx.x * NPAR + threadIdx.x] += red[threadIdx.x][0];
}

// The vector-Jacobian product of f at stage state S for the adjoint m of one
// (site, replica): P = S x nu (to be gathered by the neighbours), the local
// part loc, and the parameter derivatives added to part[].
__device__ __forceinline__ void vjp_local(const LLGArgs &a, const Site &s,
                                          const double *__restrict__ S, const V3 &m, double *P,
                                          double *loc, double (&part)[NPAR]) {
    const V3 sv = vload(S + s.e);
    V3 nn, nnn;
    neighbour_sums(S, s, a.N, nn, nnn);
    const V3 H = vadd(vadd(vmul(a.J1, nn), vmul(a.J2, nnn)), v3(a.hx, a.hy, a.hz));
    const V3 tau = vcross(H, sv);
    const V3 nu = vmul(a.g, vadd(m, vmul(a.alpha, vcross(m, sv))));
    const V3 p = vcross(sv, nu);
    const V3 l = vadd(vmul(a.g * a.alpha, vcross(tau, m)), vcross(nu, H));
    vstore(P + s.e, p);
    vstore(loc + s.e, l);
    const V3 sxt = vcross(sv, tau);
    const V3 f = vmul(a.g, vadd(tau, vmul(a.alpha, sxt)));
    part[0] = vdot(p, nn);
    part[1] = vdot(p, nnn);
    part[2] = vdot(m, vadd(vmul(-2.0 * a.alpha * a.g, f), vmul(a.g, sxt)));
    part[3] = p.x;
    part[4] = p.y;
    part[5] = p.z;
}

// Adjoint of the renormalisation, then the vector-Jacobian product at the
// stage-4 state.  v = acc + k4/6 with k4 = dt f(s4) (the forward stage 4),
// lam_v = (l/|v|)(lam - v^ (v^ . lam)), mu4 = dt lam_v / 6 (kept in
// registers: only this element's vector-Jacobian product uses it).  The
// parameter derivatives are added to this block's running slot
// bacc[blockIdx.x][6]; the blocks cover the same sites in every launch, so
// the sums are deterministic.
template <bool J2, bool H, bool DAMP>
__global__ void __launch_bounds__(TPB) adj_renorm_vjp_kernel(
    LLGArgs a, const double *__restrict__ s4, const double *__restrict__ acc,
    const double *__restrict__ lam, double *__restrict__ lam_v, double *__restrict__ P,
    double *__restrict__ loc, double *__restrict__ bacc) {
    double part[NPAR] = {0, 0, 0, 0, 0, 0};
    Site s;
    if (site_of(a, s)) {
        const V3 d = llg_rhs<J2, H, DAMP>(s4, s.sstride, s.off, a.N, s.row, s.col, a);
        const V3 v = v3(da(acc[s.e], div6(dm(d.x, a.dt))), da(acc[s.e + 1], div6(dm(d.y, a.dt))),
                        da(acc[s.e + 2], div6(dm(d.z, a.dt))));
        const double r = sqrt(vdot(v, v));
        const V3 vh = vmul(1.0 / r, v);
        const V3 l = vload(lam + s.e);
        const V3 lv = vmul(a.spin_len / r, vsub(l, vmul(vdot(vh, l), vh)));
        vstore(lam_v + s.e, lv);
        vjp_local(a, s, s4, vmul(a.dt / 6.0, lv), P, loc, part);
    }
    block_add(part, bacc);
}

// lam_s = loc + J1 sum_nn P_in + J2 sum_nnn P_in;  lam_y_out = lam_y_in +
// lam_s.  With a next stage state S: mu = dt (cv lam_v + cs lam_s) and its
// vector-Jacobian product at S, written to P_out (P_in is still being read by
// the neighbours) and loc (read above by this thread only), derivatives to
// bacc.  lam_y_in may equal lam_y_out (each thread reads and writes its own
// element).
__global__ void __launch_bounds__(TPB) vjp_gather_kernel(
    LLGArgs a, const double *__restrict__ P_in, double *loc, const double *__restrict__ lam_v,
    const double *lam_y_in, double *lam_y_out, double cv, double cs,
    const double *__restrict__ S, double *__restrict__ P_out, double *__restrict__ bacc) {
    double part[NPAR] = {0, 0, 0, 0, 0, 0};
    Site s;
    if (site_of(a, s)) {
        V3 nn, nnn;
        neighbour_sums(P_in, s, a.N, nn, nnn);
        const V3 lam_s = vadd(vload(loc + s.e), vadd(vmul(a.J1, nn), vmul(a.J2, nnn)));
        vstore(lam_y_out + s.e, vadd(vload(lam_y_in + s.e), lam_s));
        if (S) {
            const V3 m = vmul(a.dt, vadd(vmul(cv, vload(lam_v + s.e)), vmul(cs, lam_s)));
            vjp_local(a, s, S, m, P_out, loc, part);
        }
    }
    if (S) block_add(part, bacc);  // uniform over the grid
}

// Column sums over sites for each k: Fpart[chunk][k] = sum_i ph_i A[i][k].
__global__ void __launch_bounds__(128) fsum_kernel(const double *__restrict__ A, long M, int K,
                                                   const double2 *__restrict__ ph, long rows,
                                                   double2 *__restrict__ Fpart) {
    const int k = blockIdx.x * 128 + threadIdx.x;
    if (k >= K) return;
    const long i0 = (long)blockIdx.y * rows, i1 = min(M, i0 + rows);
    double re = 0.0, im = 0.0;
    for (long i = i0; i < i1; ++i) {
        const double x = A[i * K + k];
        const double2 p = ph[i];
        re += p.x * x;
        im += p.y * x;
    }
    Fpart[(long)blockIdx.y * K + k] = make_double2(re, im);
}

// G_k = sum over chunks; Z_c = (1/nfile) sum_f G_(f,c).  One block.
__global__ void gz_kernel(const double2 *__restrict__ Fpart, int nchunks, int K, int nfile,
                          double2 *__restrict__ G, double2 *__restrict__ Z) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
        double re = 0.0, im = 0.0;
        for (int c = 0; c < nchunks; ++c) {
            re += Fpart[(long)c * K + k].x;
            im += Fpart[(long)c * K + k].y;
        }
        G[k] = make_double2(re, im);
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double re = 0.0, im = 0.0;
        for (int f = 0; f < nfile; ++f) {
            re += G[3 * f + threadIdx.x].x;
            im += G[3 * f + threadIdx.x].y;
        }
        Z[threadIdx.x] = make_double2(re / nfile, im / nfile);
    }
}

// S = (1/(M nfile)) sum_k F_k (G_k - Z_c(k)), F from the chunk partials.  One
// block of 256 threads, fixed order.
__global__ void __launch_bounds__(256) sqt_value_kernel(const double2 *__restrict__ Fpart,
                                                        int nchunks, int K, int nfile, long M,
                                                        const double2 *__restrict__ G,
                                                        const double2 *__restrict__ Z,
                                                        double2 *__restrict__ out) {
    __shared__ double sre[256], sim[256];
    double re = 0.0, im = 0.0;
    for (int k = threadIdx.x; k < K; k += 256) {
        double fr = 0.0, fi = 0.0;
        for (int c = 0; c < nchunks; ++c) {
            fr += Fpart[(long)c * K + k].x;
            fi += Fpart[(long)c * K + k].y;
        }
        const double gr = G[k].x - Z[k % 3].x, gi = G[k].y - Z[k % 3].y;
        re += fr * gr - fi * gi;
        im += fr * gi + fi * gr;
    }
    sre[threadIdx.x] = re;
    sim[threadIdx.x] = im;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            sre[threadIdx.x] += sre[threadIdx.x + w];
            sim[threadIdx.x] += sim[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double s = 1.0 / ((double)M * nfile);
        *out = make_double2(sre[0] * s, sim[0] * s);
    }
}

// lam[i][k] += Re(coef u_i (G_k - Z_c(k))), coef = dL/dS* in the sense
// dL = Re(coef' dS) with coef' folded with 1/(M nfile) by the caller.
__global__ void __launch_bounds__(256) loss_grad_kernel(double *__restrict__ lam, long M, int K,
                                                        const double2 *__restrict__ u,
                                                        const double2 *__restrict__ G,
                                                        const double2 *__restrict__ Z,
                                                        double cre, double cim) {
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M * K) return;
    const long i = t / K;
    const int k = (int)(t - i * K);
    const double2 ui = u[i];
    const double gr = G[k].x - Z[k % 3].x, gi = G[k].y - Z[k % 3].y;
    const double pr = ui.x * gr - ui.y * gi, pi = ui.x * gi + ui.y * gr;  // u_i (G - Z)
    lam[t] += cre * pr - cim * pi;
}

__global__ void param_reduce_kernel(const double *__restrict__ bacc, int nblocks,
                                    double *__restrict__ grad) {
    __shared__ double red[NPAR][256];
    double v[NPAR] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblocks; b += 256)
#pragma unroll
        for (int q = 0; q < NPAR; ++q) v[q] += bacc[(long)b * NPAR + q];
#pragma unroll
    for (int q = 0; q < NPAR; ++q) red[q][threadIdx.x] = v[q];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w)
#pragma unroll
            for (int q = 0; q < NPAR; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < NPAR) grad[threadIdx.x] = red[threadIdx.x][0];
}

}  // namespace

int adjoint_blocks(const LLGArgs &a) { return (int)((a.M * a.nfile + TPB - 1) / TPB); }

cudaError_t launch_adj_renorm_vjp(const LLGArgs &a, const double *s4, const double *acc,
                                  const double *lam, double *lam_v, double *P, double *loc,
                                  double *bacc, cudaStream_t st) {
    const int sel = (a.use_j2 ? 4 : 0) | (a.use_h ? 2 : 0) | (a.use_damp ? 1 : 0);
    const int nb = adjoint_blocks(a);
#define ASD_ADJ_CASE(S, J, Hh, D)                                                          \
    case S:                                                                                \
        adj_renorm_vjp_kernel<J, Hh, D><<<nb, TPB, 0, st>>>(a, s4, acc, lam, lam_v, P, loc, \
                                                            bacc);                         \
        break;
    switch (sel) {
        ASD_ADJ_CASE(0, false, false, false)
        ASD_ADJ_CASE(1, false, false, true)
        ASD_ADJ_CASE(2, false, true, false)
        ASD_ADJ_CASE(3, false, true, true)
        ASD_ADJ_CASE(4, true, false, false)
        ASD_ADJ_CASE(5, true, false, true)
        ASD_ADJ_CASE(6, true, true, false)
        ASD_ADJ_CASE(7, true, true, true)
    }
#undef ASD_ADJ_CASE
    return cudaGetLastError();
}

cudaError_t launch_vjp_gather(const LLGArgs &a, const double *P_in, double *loc,
                              const double *lam_v, const double *lam_y_in, double *lam_y_out,
                              double cv, double cs, const double *S, double *P_out, double *bacc,
                              cudaStream_t st) {
    vjp_gather_kernel<<<adjoint_blocks(a), TPB, 0, st>>>(a, P_in, loc, lam_v, lam_y_in, lam_y_out,
                                                         cv, cs, S, P_out, bacc);
    return cudaGetLastError();
}

// Rows per chunk of the site sums: 256, halved (down to 16) until the grid
// of (K / 128) x chunks has at least four blocks per SM of a B200, so that
// small lattices (64 x 64 x 100: 48 blocks of 256 rows) still fill the GPU;
// doubled where the chunks would exceed the grid's y extent (N = 4096).
int fsum_rows(long M, int K) {
    constexpr long kMinBlocks = 4 * 148;
    const long kb = (K + 127) / 128;
    int rows = 256;
    while (rows > 16 && kb * ((M + rows - 1) / rows) < kMinBlocks) rows >>= 1;
    while ((M + rows - 1) / rows > 65535) rows <<= 1;  // the grid's y extent
    return rows;
}

int fsum_chunks(long M, int K) { return (int)((M + fsum_rows(M, K) - 1) / fsum_rows(M, K)); }

cudaError_t launch_fsum(const double *A, long M, int K, const double2 *ph, double2 *Fpart,
                        cudaStream_t st) {
    dim3 grid((unsigned)((K + 127) / 128), (unsigned)fsum_chunks(M, K));
    fsum_kernel<<<grid, 128, 0, st>>>(A, M, K, ph, fsum_rows(M, K), Fpart);
    return cudaGetLastError();
}

cudaError_t launch_gz(const double2 *Fpart, long M, int K, int nfile, double2 *G, double2 *Z,
                      cudaStream_t st) {
    gz_kernel<<<1, 256, 0, st>>>(Fpart, fsum_chunks(M, K), K, nfile, G, Z);
    return cudaGetLastError();
}

cudaError_t launch_sqt_value(const double2 *Fpart, long M, int K, int nfile, const double2 *G,
                             const double2 *Z, double2 *out, cudaStream_t st) {
    sqt_value_kernel<<<1, 256, 0, st>>>(Fpart, fsum_chunks(M, K), K, nfile, M, G, Z, out);
    return cudaGetLastError();
}

cudaError_t launch_loss_grad(double *lam, long M, int K, const double2 *u, const double2 *G,
                             const double2 *Z, double cre, double cim, cudaStream_t st) {
    const long n = M * K;
    loss_grad_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(lam, M, K, u, G, Z, cre, cim);
    return cudaGetLastError();
}

cudaError_t launch_param_reduce(const double *bacc, int nblocks, double *grad, cudaStream_t st) {
    param_reduce_kernel<<<1, 256, 0, st>>>(bacc, nblocks, grad);
    return cudaGetLastError();
}

}  // namespace asd
