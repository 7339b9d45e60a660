// asd_internal.h -- declarations shared by the translation units of
// libasd_b200.so (not part of the public ABI; see include/asd_b200.h).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/asd_b200.h"

namespace asd {

// Parameters of the LLG right-hand side, passed by value to the kernels.
struct LLGArgs {
    int N;        // lattice side
    int nfile;    // replicas
    long M;       // N*N
    double J1, J2;
    double hx, hy, hz;
    double alpha;
    double g;     // 1 / (1 + alpha^2), formed once on the host
    double dt;
    double spin_len;
    int use_j2, use_h, use_damp;
    // Replica range the RK4 stage kernels update: [f0, f0 + nc).  The whole
    // ensemble (0, nfile) unless a caller pipelines the step by replica chunk
    // (replicas never interact, so a chunk's step needs no other replica).
    int f0, nc;
};

LLGArgs make_llg_args(const asd_params &p);

// ------------------------------------------------------------ error state
void set_error(const char *fmt, ...);
int fail(int code, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what);
#define ASD_CUDA_TRY(expr)                                   \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) return ::asd::cuda_fail(_e, #expr); \
    } while (0)

// Device status word bits (written by kernels, read by the host).
enum : unsigned { kStatusTimeout = 1u, kStatusBadLaunch = 2u };

// ------------------------------------------------------------ LLG kernels
// Spins live in the "site-major" layout double[M][nfile][3]: for site i the
// 3*nfile values of all replicas are contiguous, which is both the stencil's
// coalescing axis and the K axis of the correlation GEMM (the reference's
// spin_zero layout, llg_sqt_baseline.c:227-236).
// Launches one fused RK4 stage (1..4) over all sites and replicas.
//   stage 1: ys_out = y + k/2,  acc = y + k/6          (k = dt * f(y))
//   stage 2: ys_out = y + k/2,  acc = acc + k/3        (k = dt * f(ys_in))
//   stage 3: ys_out = y + k,    acc = acc + k/3
//   stage 4: y_new  = spin_len * o / |o|, o = acc + k/6 (written to ys_out)
cudaError_t launch_llg_stage(int stage, const LLGArgs &a, const double *y, const double *ys_in,
                             double *acc, double *ys_out, cudaStream_t st);

// One whole RK4 step (all four stages + renormalisation) in one launch,
// streamed down the lattice by column band (llg_kernels.cu): y -> yout
// (distinct buffers), replicas [a.f0, a.f0 + a.nc) only.
cudaError_t launch_llg_step_fused(const LLGArgs &a, const double *y, double *yout,
                                  cudaStream_t st);
// True if the streamed one-launch step has enough work for this lattice and
// replica range to fill the GPU (at least 8 rows per resident CTA).
bool llg_fused_fills(const LLGArgs &a);

// Counts the x[i] for which the constant divisions by 3 and 6 of the LLG
// kernels differ from __ddiv_rn in any bit (diagnostic).
cudaError_t launch_div_check(const double *x, long n, unsigned long long *bad, cudaStream_t st);

// AoS [nfile][M][3] <-> site-major [M][nfile][3]
// Replica-range forms: the AoS side holds replicas [f0, f0 + nc) only
// ([nc][M][3]); the site-major side is the whole [M][nfile][3] array.
cudaError_t launch_aos_to_sitemajor_range(const double *aos, double *sm, long M, int nfile,
                                          int f0, int nc, cudaStream_t st);
cudaError_t launch_sitemajor_to_aos_range(const double *sm, double *aos, long M, int nfile,
                                          int f0, int nc, cudaStream_t st);
cudaError_t launch_aos_to_sitemajor(const double *aos, double *sm, long M, int nfile,
                                    cudaStream_t st);
cudaError_t launch_sitemajor_to_aos(const double *sm, double *aos, long M, int nfile,
                                    cudaStream_t st);

// Drop-in kernels on the reference layout (AoS), reference arithmetic only.
cudaError_t launch_euler_aos(const LLGArgs &a, const double *spin, double *deriv,
                             cudaStream_t st);
// pass 1..4 of runge_kutta's element-wise loops (llg_sqt_baseline.c:104-139)
cudaError_t launch_rk_pass(int pass, long n, double dt, const double *spin, double *cur,
                           double *k, const double *k1, const double *k2, const double *k3,
                           cudaStream_t st);

// --------------------------------------------------------- S(q,t) kernels
// Per-site replica mean (FP64) plus the FP32 epilogue vectors
// vec4[i] = (mx, my, mz, phase.re), vec1[i] = phase.im for i < M.
cudaError_t launch_site_mean(const double *state, long M, int nfile, const double2 *phase,
                             double *mean, float4 *vec4, float *vec1, cudaStream_t st);

// Per-site sums over the context's replicas ([M][3]), and the S(q,t) of a
// replica-sharded ensemble from its all-reduced partial and site sums.
cudaError_t launch_site_sum(const double *state, long M, int nfile, double *sums,
                            cudaStream_t st);
cudaError_t launch_shard_finish(long M, int nfile_total, const double *part, const double *sums,
                                const double *zsums, const double2 *u, const double2 *w,
                                double *out, cudaStream_t st);
// FP64 state [M][K] -> split operands hi/lo [M][Kp] (zero for k >= K):
// kind 1 = TF32 (stored as fp32 bit patterns), 2 = BF16, 3 = FP16 of
// scale * x (scale a power of two; ignored by kinds 1 and 2).
// launch_split_range: columns [kbeg, kend) of every row only (both even,
// kend <= Kp).
cudaError_t launch_split_range(int kind, const double *state, long M, int K, int Kp, int kbeg,
                               int kend, void *hi, void *lo, double scale, cudaStream_t st);
cudaError_t launch_split(int kind, const double *state, long M, int K, int Kp, void *hi,
                         void *lo, double scale, cudaStream_t st);
// Bytes per split operand element and K elements per 128-byte k block.
inline int split_esize(int kind) { return kind == 1 ? 4 : 2; }
// The power of two FP16x3 scales the spins by: spin_len * scale in
// [2^12, 2^13), so components up to 7.9 * spin_len stay below FP16's
// largest finite value (65504) and the lo parts of all components above
// 2^-15 * spin_len are normal numbers.  1 for the other kinds.
double split_scale(int kind, double spin_len);

// ------------------------------------------ FP64 tensor-core GEMM S(q,t)
// (dmma_sqt.cu) C = alpha A B^T over site-major [M][K] FP64 operands, never
// stored: per 128 x 128 tile either the S(q,t) partial (part != nullptr and
// tdiag == nullptr) or the q-grid diagonal partials (tdiag != nullptr).
struct DmmaSqtArgs {
    const double *A, *B;  // [M][K], the state at t and the origin
    long M;
    int K;
    double alpha;
    int outer;            // subtract m_i . z_j (0: a shard's partial GEMM value)
    const double *mrow, *zcol;       // [M][3] replica means at t and 0
    const double2 *uphase, *wphase;  // [M]
    double2 *part;        // one partial per tile, dmma_sqt_tiles(M) of them
    int lat_n = 0;        // q grid: lattice side
    double *tdiag = nullptr;  // q grid: [tiles][dmma_sqt_tile() * 2 - 1][2]
    int abs_sum = 0;      // sum |alpha C_ij - m_i . z_j| instead (no phase)
    // Plain product (the cblas_dgemm drop-in): with C set, B has MB rows and
    // the kernel stores C[i + j ldc] = alpha sum_k A_ik B_jk (+ beta C[..] when
    // beta != 0; C is not read when beta == 0) for i < M, j < MB.
    long MB = 0;
    double *C = nullptr;
    long ldc = 0;
    double beta = 0.0;
};
constexpr int kDmmaTile = 128;  // tile rows = tile columns
long dmma_sqt_tiles(long M);
int launch_dmma_sqt(const DmmaSqtArgs &p, cudaStream_t st);
// Device transpose of a dense [rows][cols] FP64 matrix into [cols][rows].
cudaError_t launch_transpose_f64(const double *in, long rows, long cols, double *out,
                                 cudaStream_t st);
// C[i + j ldc] *= beta for i < m, j < n (beta == 0: set to +0).
cudaError_t launch_scale_f64(double *c, long m, long n, long ldc, double beta, cudaStream_t st);

// q grid (qgrid.cu): from per-tile diagonal partials tdiag[mb][nb][bm+bn-1][2]
// of num_m x num_n tiles of bm x bn sites (bn a multiple of bm) to the N*N
// displacement bins G, in a fixed order; ds holds qgrid_keys() * (bm+bn-1) * 2
// doubles of work space.
long qgrid_keys(int num_m, int num_n, int bm, int bn);
cudaError_t launch_qgrid_bins(const double *tdiag, int num_m, int num_n, int bm, int bn, int lat_n,
                              double *ds, double *G, cudaStream_t st);
// out[2*(a*N+b)+{0,1}] = scale * sum_d G[d] e^{-2 pi i (a dr + b dc)/N}; tmp holds N*N double2.
cudaError_t launch_grid_dft(const double *G, int lat_n, double scale, double2 *tmp, double *out,
                            cudaStream_t st);

// out[0..1] = (sum of nparts partials) * scale, deterministic order.
cudaError_t launch_finalize(const double2 *part, int nparts, double scale, double *out,
                            cudaStream_t st);

// ------------------------------------------------ adjoint (adjoint.cu)
int adjoint_blocks(const LLGArgs &a);
// Adjoint of the renormalisation, then the vector-Jacobian product at s4
// (P, loc, parameter derivatives into bacc).
cudaError_t launch_adj_renorm_vjp(const LLGArgs &a, const double *s4, const double *acc,
                                  const double *lam, double *lam_v, double *P, double *loc,
                                  double *bacc, cudaStream_t st);
// Gather of P_in into lam_y_out = lam_y_in + lam_s; with S != NULL, the
// vector-Jacobian product at S for mu = dt (cv lam_v + cs lam_s) into P_out
// (a buffer other than P_in) and loc.
cudaError_t launch_vjp_gather(const LLGArgs &a, const double *P_in, double *loc,
                              const double *lam_v, const double *lam_y_in, double *lam_y_out,
                              double cv, double cs, const double *S, double *P_out, double *bacc,
                              cudaStream_t st);
int fsum_rows(long M, int K);
int fsum_chunks(long M, int K);
cudaError_t launch_fsum(const double *A, long M, int K, const double2 *ph, double2 *Fpart,
                        cudaStream_t st);
cudaError_t launch_gz(const double2 *Fpart, long M, int K, int nfile, double2 *G, double2 *Z,
                      cudaStream_t st);
cudaError_t launch_sqt_value(const double2 *Fpart, long M, int K, int nfile, const double2 *G,
                             const double2 *Z, double2 *out, cudaStream_t st);
cudaError_t launch_loss_grad(double *lam, long M, int K, const double2 *u, const double2 *G,
                             const double2 *Z, double cre, double cim, cudaStream_t st);
cudaError_t launch_param_reduce(const double *bacc, int nblocks, double *grad, cudaStream_t st);

// ------------------------------------------------ tcgen05 split GEMM S(q,t)
struct UmmaSqtArgs {
    int kind;             // 1 = TF32x3, 2 = BF16x3, 3 = FP16x3
    long M;               // rows (sites at t)   -- also the column count
    int Kp;               // padded K (multiple of the 128-byte k block)
    const void *a_hi, *a_lo;   // [M][Kp]
    const void *b_hi, *b_lo;   // [M][Kp]
    const float4 *row4; const float *row1;   // padded to the tile multiple
    const float4 *col4; const float *col1;
    float alpha;          // 1/nfile (FP16x3: divided by the operands' scale squared)
    double2 *part;        // one partial per CTA
    unsigned *status;     // device status word
    int num_sms;
    int chunk_k = 0;          // K elements per TMEM accumulation chunk (0: all)
    float *dbg_c = nullptr;   // diagnostic: store the accumulator instead
    long dbg_ldc = 0;
    double *tdiag = nullptr;  // q grid: per-tile diagonal partials
                              // [Mp/BM][Mp/BN][BM+BN-1][2] (qgrid.cu)
    int lat_n = 0;            // lattice side (q grid)
    // K sub-range [k_begin, k_end) in elements (multiples of the k block;
    // k_end = 0: to Kp).  The epilogue applies the connected-part term only
    // when outer != 0, so the partial sums of launches over disjoint K
    // ranges, one of them with outer set, add up to S(q,t).
    int k_begin = 0, k_end = 0;
    int outer = 1;
    int max_grid = 0;         // > 0: launch at most this many CTAs (partials)
};
// Returns the number of CTAs launched (partials written) or a negative error.
int launch_umma_sqt(const UmmaSqtArgs &a, cudaStream_t st);
long umma_row_pad(long M);   // rows/cols padded to the tile multiple
int umma_tile_rows();        // BM = 128 (the q grid's tile geometry)
int umma_tile_cols();        // BN = 256
// CTAs launch_umma_sqt launches for M rows on num_sms SMs (max_grid unset).
long umma_max_grid_for(long M, int num_sms);
cudaError_t launch_mbar_timeout_probe(uint32_t limit, unsigned *status, cudaStream_t st);
cudaError_t launch_grid_barrier_probe(void *bs, unsigned *status, cudaStream_t st);

}  // namespace asd
