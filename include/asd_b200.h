/*
 * asd_b200.h -- C ABI of libasd_b200.so, a B200 (sm_100a) implementation of
 * the hot path of hwchen2017/ASD-kernel-fusion: RK4 time stepping of the
 * Landau-Lifshitz(-Gilbert) equation for classical spins on a periodic
 * N x N lattice, and the GEMM-formulated real-space spin-spin correlation
 * that gives the dynamical structure factor S(q,t).
 *
 * Two layers:
 *
 *  1. Drop-in symbols with the reference's names, signatures and semantics
 *     (host pointers, synchronous, parameters taken from the caller's globals
 *     or from asd_set_params):
 *        euler            <- baseline/llg_sqt_baseline.c:29
 *        runge_kutta      <- baseline/llg_sqt_baseline.c:95
 *        fused_dgemm      <- kernel_fusion/gemm_kernel.h:355
 *     and the plain path's BLAS call, cblas_dgemm <- gemm/llg_sqt_mkl.c:378,
 *     as asd_cblas_dgemm (libasd_cblas.so exports it under the BLAS name).
 *     A C program of the reference links libasd_b200.so instead of defining
 *     these functions itself (deleting their bodies and including this
 *     header; the program's globals N, Nfile, J1, dt are read through weak
 *     references).
 *
 *  2. A context API (asd_ctx_*) that keeps the replicas' spins resident in
 *     HBM and runs a whole step on one CUDA stream: the RK4 step with its
 *     renormalisation (one launch, or one kernel per stage), then S(q,t)
 *     through a tcgen05 tensor-core GEMM in split precision (TF32x3,
 *     BF16x3 or FP16x3) whose epilogue applies the phase, the connected-part
 *     subtraction and the reduction, or through the FP64 path.  It replaces
 *     the per-step body of main() (llg_sqt_baseline.c:289-426,
 *     llg_sqt_fusion.c:340-449); host-buffer forms keep the reference's data
 *     flow (spins in host memory between steps).
 *
 * Spin arrays crossing the ABI use the reference's layout, "AoS":
 * double[nfile][N*N][3] (llg_sqt_baseline.c:185, :202), site index
 * i = row*N + col.  All functions returning int return ASD_OK (0) or a
 * negative ASD_ERR_* code; asd_last_error() describes the last failure on the
 * calling thread.  There is no CPU fallback: without a usable sm_100 device
 * every call that computes returns ASD_ERR_CUDA.
 */
#ifndef ASD_B200_H
#define ASD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ASD_OK 0
#define ASD_ERR_INVALID (-1)     /* a parameter is out of range            */
#define ASD_ERR_CUDA (-2)        /* a CUDA runtime or driver call failed     */
#define ASD_ERR_NOMEM (-3)       /* device or host allocation failed         */
#define ASD_ERR_TIMEOUT (-4)     /* a bounded device-side wait gave up       */
#define ASD_ERR_STATE (-5)       /* call order (e.g. no spins set yet)       */
#define ASD_ERR_UNSUPPORTED (-6) /* the device is not sm_100, or a size is
                                    beyond a kernel's stated limits          */

/* Arithmetic of the S(q,t) correlation GEMM. */
typedef enum {
    ASD_SQT_FP64 = 0,   /* the plain path: FP64 tensor-core GEMM (mma.sync .f64) with
                           the phase, connected-part and reduction epilogue fused;
                           one block per 128 x 128 tile, so up to N = 2435
                           (ASD_ERR_UNSUPPORTED beyond) */
    ASD_SQT_TF32X3 = 1, /* tcgen05 kind::tf32, hi*hi + hi*lo + lo*hi, FP32 accumulate   */
    ASD_SQT_BF16X3 = 2, /* tcgen05 kind::f16 (bf16), hi*hi + hi*lo + lo*hi, FP32 accum. */
    ASD_SQT_FP16X3 = 3  /* tcgen05 kind::f16 (fp16), hi*hi + hi*lo + lo*hi, FP32 accum.:
                           the operands are scaled by 2^e (spin_len * 2^e in [2^12, 2^13))
                           before the split, so hi + lo keep 22 bits like TF32's while the
                           products run at the 16-bit rate (measured 1-8 % slower than
                           BF16x3 under the power cap; a third of BF16x3's error at late
                           times, twice its FP32-accumulation error early on at the same
                           chunk_k); components up to
                           7.9 * spin_len always fit, larger ones can overflow FP16
                           and then make S(q,t) non-finite */
} asd_sqt_mode;

/* Model parameters.  The reference hard-wires alpha = J2 = h = 0,
 * spin_len = 1 (1.5 in its fusion program) and vx = vy = N/10
 * (llg_sqt_baseline.c:12-20, :172-173). */
typedef struct {
    int N;           /* lattice side (>= 3); M = N*N sites                        */
    int nfile;       /* independent replicas ("snapshots", Nfile)                */
    double J1;       /* nearest-neighbour exchange (J1, :14)                     */
    double J2;       /* next-nearest (diagonal) exchange                          */
    double alpha;    /* Gilbert damping                                           */
    double hx, hy, hz; /* Zeeman field, added to H_eff.  The reference's commented
                          term exchg.z += -hz (llg_sqt_baseline.c:79) is h=(0,0,-hz). */
    double dt;       /* RK4 step (dt, :16)                                        */
    double spin_len; /* length after renormalisation                              */
    int vx, vy;      /* q = 2*pi*(vx, vy)/N                                       */
} asd_params;

/* ----------------------------------------------------------------- common */
const char *asd_version(void);
const char *asd_last_error(void);
/* Reference defaults for N and nfile: J1=1, dt=0.02, spin_len=1, vx=vy=N/10. */
int asd_params_default(asd_params *p, int N, int nfile);
/* Selects the CUDA device used by later calls on this thread (default 0). */
int asd_set_device(int device);

/* ------------------------------------------------------------ context API */
typedef struct asd_ctx asd_ctx;

/* Allocates the device state for p (about 4 spin arrays in FP64 plus the
 * split GEMM operands).  mode_mask: bit (1<<asd_sqt_mode) for every S(q,t)
 * mode the context must be able to run (0 = all).  Replaces the set-up in
 * main(), llg_sqt_baseline.c:146-287. */
int asd_ctx_create(const asd_params *p, unsigned mode_mask, asd_ctx **out);
int asd_ctx_destroy(asd_ctx *ctx);
/* Runs all later work of ctx on this CUDA stream (a cudaStream_t). */
int asd_ctx_set_stream(asd_ctx *ctx, void *stream);
int asd_ctx_get_params(const asd_ctx *ctx, asd_params *p);

/* Changes the model parameters of an existing context (N and nfile stay). */
int asd_ctx_set_params(asd_ctx *ctx, const asd_params *p);

/* Copies spins (AoS, host) to the device as the current state.  With
 * as_origin != 0 they also become the t = 0 snapshot that S(q,t) correlates
 * against (spin_zero and zerot_avg, llg_sqt_baseline.c:227-259). */
int asd_ctx_set_spins(asd_ctx *ctx, const double *spin_aos, int as_origin);
/* Same from a device buffer in the AoS layout. */
int asd_ctx_set_spins_device(asd_ctx *ctx, const double *d_spin_aos, int as_origin);
/* Copies the current state back (AoS, host). */
int asd_ctx_get_spins(asd_ctx *ctx, double *spin_aos);
int asd_ctx_get_spins_device(asd_ctx *ctx, double *d_spin_aos);

/* nsteps RK4 steps with renormalisation (llg_sqt_baseline.c:296-309),
 * asynchronous on the context's stream. */
int asd_ctx_step(asd_ctx *ctx, int nsteps);

/* S(q,t) between the current state and the origin at q = 2*pi*(vx,vy)/N,
 * into out[0] (real) and out[1] (imaginary); synchronous.  Equals
 * sqt[num] of the reference (llg_sqt_fusion.c:368-442, gemm/llg_sqt_mkl.c:347-423). */
int asd_ctx_sqt(asd_ctx *ctx, asd_sqt_mode mode, double out[2]);
/* Asynchronous form: writes out[0..1] (a device pointer) on the stream. */
int asd_ctx_sqt_async(asd_ctx *ctx, asd_sqt_mode mode, double *d_out);
/* The magnitude of the terms S(q,t) sums, *out = (1/M) sum_ij |C_ij - m_i . z_j|
 * (C the correlation GEMM, m and z the replica means at t and 0), through the
 * FP64 GEMM; synchronous.  S(q,t) is a phase-weighted sum of these terms and
 * can be much smaller than their magnitude, so an error of S relative to this
 * scale measures the arithmetic apart from cancellation.  Needs the FP64 mode.
 * No counterpart in the reference. */
int asd_ctx_sqt_magnitude(asd_ctx *ctx, double *out);

/* S(q,t) for every q = 2*pi*(a, b)/N of the N x N grid, into d_out[2*(a*N+b)]
 * (real) and d_out[2*(a*N+b)+1] (imaginary), a device buffer of 2*N*N
 * doubles; asynchronous.  The same correlation GEMM (any asd_sqt_mode),
 * with an epilogue that sums every connected C_ij - m_i . z_j along the
 * diagonals i - j of each tile; the diagonal sums are binned by displacement
 * r_i - r_j (mod N) and a 2-D DFT of the N*N bins gives S at every q.
 * d_out[2*(vx*N+vy)] equals asd_ctx_sqt's value up to rounding.  Any N; work
 * space on the first call: 8 * (128 + BN - 1) * 2 bytes per GEMM tile (BN =
 * 128 in FP64, 256 in the split modes; 1.1 GB / 0.8 GB at N = 256).  Every
 * sum runs in a fixed order, so results repeat bit for bit.
 * No counterpart in the reference (its programs evaluate one q). */
int asd_ctx_sqt_grid_async(asd_ctx *ctx, asd_sqt_mode mode, double *d_out);
/* Same into host memory (2*N*N doubles); synchronous. */
int asd_ctx_sqt_grid(asd_ctx *ctx, asd_sqt_mode mode, double *out);

/* Loss and gradient for parameter fitting.  Starting from the origin spins,
 * runs nsteps RK4 steps with the context's parameters and evaluates S(q,t) at
 * the steps t_e = e * stride, e = 1..E, E = nsteps / stride (in FP64, through
 * the factorised form of the correlation GEMM); with target (2E doubles,
 * re/im) the loss is L = (1/E) sum_e |S(q,t_e) - target_e|^2 and grad
 * (6 doubles) receives dL/d(J1, J2, alpha, hx, hy, hz), computed by the
 * adjoint of the RK4 step and of the renormalisation, with checkpoints every
 * `checkpoint` steps and recomputation of each segment.  sqt_out (2E
 * doubles) receives the S(q,t_e) values.  Host buffers; synchronous.  The
 * current state is not changed.  Device work space, allocated on the first
 * call and kept by the context: about (nsteps / checkpoint + checkpoint + 13)
 * spin-state arrays; where the RK4 step runs as four stage kernels (small
 * lattices) and half of the free device memory holds them, 4 * checkpoint
 * more, so that the backward pass reads each segment's stage states instead
 * of recomputing them (the results are the same bits either way).  No
 * counterpart in the reference. */
int asd_ctx_loss_grad(asd_ctx *ctx, int nsteps, int stride, int checkpoint, const double *target,
                      double *loss, double *grad, double *sqt_out);
/* asd_ctx_loss_grad in two calls, so that a caller that does not need the
 * gradient (a forward-only evaluation) does not pay for the adjoint.
 * asd_ctx_loss_forward runs the forward pass -- the nsteps RK4 steps with the
 * checkpoints kept on the device, S(q,t_e) into sqt_out (2E doubles, may be
 * NULL) and, with target, the loss into *loss -- and leaves a tape.
 * asd_ctx_loss_backward then runs the adjoint from that tape: grad (6
 * doubles, may be NULL) = dL/d(J1, J2, alpha, hx, hy, hz) and dtarget (2E
 * doubles, may be NULL) = dL/dtarget = -2 (S - target) / E; target (2E
 * doubles) is required.  The tape holds while the parameters and the origin
 * are unchanged (else ASD_ERR_STATE) and until the next forward pass or
 * asd_ctx_loss_grad; backward may run more than once.  Forward + backward
 * give asd_ctx_loss_grad's results bit for bit.  Host buffers; synchronous.
 * No counterpart in the reference. */
int asd_ctx_loss_forward(asd_ctx *ctx, int nsteps, int stride, int checkpoint, const double *target,
                         double *loss, double *sqt_out);
int asd_ctx_loss_backward(asd_ctx *ctx, const double *target, double *grad, double *dtarget);

/* One full step through host buffers, the reference's own contract: spins
 * (AoS) come from host memory, one RK4 step runs, the new spins go back to
 * spin_out and S(q,t) into sqt_out.  spin_in may equal spin_out.  Above 64
 * replicas the step is pipelined by replica chunk (uploads, RK4, downloads
 * and K-range S(q,t) GEMMs overlap); pinned host memory lets the copies run
 * asynchronously.  Synchronous: returns when both buffers are final. */
int asd_ctx_step_host(asd_ctx *ctx, const double *spin_in, double *spin_out,
                      asd_sqt_mode mode, double sqt_out[2]);

/* asd_ctx_step_host without waiting: enqueues the upload of spin_in, one RK4
 * step, the download into spin_out and S(q,t) into sqt_out (2 doubles), and
 * returns.  The buffers must be pinned host memory (cudaMallocHost,
 * cudaHostRegister) or device memory; they are final after
 * asd_ctx_synchronize.  spin_in may equal spin_out, and one call's spin_out
 * may be the next call's spin_in: the upload of each replica chunk waits for
 * the previous call's download of the same chunk, so consecutive calls
 * overlap (the next step's uploads cross PCIe while this step's S(q,t) GEMM
 * runs).  Same results as asd_ctx_step_host; the S(q,t) GEMM runs once over
 * the whole new state, as in asd_ctx_sqt. */
int asd_ctx_step_host_async(asd_ctx *ctx, const double *spin_in, double *spin_out,
                            asd_sqt_mode mode, double *sqt_out);
/* Waits for everything the context enqueued (its stream and its copy
 * streams) and reports a device-side failure, if any. */
int asd_ctx_synchronize(asd_ctx *ctx);

/* Replica sharding of one ensemble over several GPUs, one context per GPU.
 * Replicas never interact, so each context steps its own nfile replicas; the
 * correlation GEMM's K axis is the replica axis, so S(q,t) is the sum over
 * shards of a partial GEMM value plus a connected-part term that needs only
 * the ensemble's site means.  Per evaluation the shards exchange 2 + 3*N*N
 * doubles (an all-reduce the caller runs, e.g. over NCCL); the origin's site
 * sums are exchanged once.  No counterpart in the reference (one process).
 *
 *   asd_ctx_set_ensemble(ctx, nfile_total)            replicas of the whole ensemble
 *   asd_ctx_set_spins(ctx, shard_spins, 1)
 *   asd_ctx_shard_origin_sums(ctx, d_zsums)           [N*N][3] doubles, this shard
 *     (all-reduce d_zsums)
 *   asd_ctx_shard_set_origin_sums(ctx, d_zsums)       the ensemble's
 *   per step:
 *     asd_ctx_step(ctx, 1)
 *     asd_ctx_shard_sqt_async(ctx, mode, d_part, d_sums)   2 + [N*N][3] doubles
 *     (all-reduce d_part and d_sums)
 *     asd_ctx_shard_sqt_finish(ctx, d_part, d_sums, d_out) S(q,t) of the ensemble
 *
 * d_part is this shard's (1/M) sum_ij u_i w_j C_ij with C scaled by
 * 1/nfile_total and no connected-part term; the finish adds that term from
 * the means in FP64.  All pointers are device memory, enqueued on the
 * context's stream.  Setting new origin spins requires a new exchange. */
int asd_ctx_set_ensemble(asd_ctx *ctx, int nfile_total);
int asd_ctx_shard_origin_sums(asd_ctx *ctx, double *d_zsums);
int asd_ctx_shard_set_origin_sums(asd_ctx *ctx, const double *d_zsums);
int asd_ctx_shard_sqt_async(asd_ctx *ctx, asd_sqt_mode mode, double *d_part, double *d_sums);
int asd_ctx_shard_sqt_finish(asd_ctx *ctx, const double *d_part, const double *d_sums,
                             double *d_out);

/* How asd_ctx_step (and asd_ctx_step_host) runs one RK4 step.  Both give
 * bit-identical spins. */
#define ASD_LLG_STAGES 0     /* four launches, one fused kernel per RK4 stage,
                                HBM-bound (384 B of DRAM traffic per
                                site-step; 70-85% of the measured HBM copy
                                bandwidth on B200)                           */
#define ASD_LLG_FUSED_STEP 1 /* one launch per step, the four stages
                                streamed down the lattice through shared
                                memory by column band (48 B of DRAM traffic per
                                site-step; FP64-bound; 1.35x the stages at
                                128x128x500, 1.6x at 256x256x1000 on B200)  */
#define ASD_LLG_AUTO 2       /* default: the one-launch step when the lattice
                                and replicas give it at least 8 rows of work
                                per resident CTA (e.g. 128x128x500, or its
                                64-replica chunks), else the stage kernels
                                (e.g. 64x64x100)                             */
int asd_ctx_set_llg_kernel(asd_ctx *ctx, int kernel);

/* K elements accumulated per TMEM chunk by the split S(q,t) modes (rounded
 * up to the pipeline's k block; 0 = all of K in one accumulator; negative =
 * the default).  The tensor cores' FP32 accumulation loses precision with
 * every accumulation step, so K is cut into chunks whose partial products the
 * epilogue adds in FP64.  Default: 512 for TF32x3 and 1024 for BF16x3 and
 * FP16x3, the same number of accumulation steps (TF32 MMAs take 8 K elements
 * per step, 16-bit ones 16); measured relative error of S(q,t) about 5e-6 and
 * 4e-6 at K = 3000. */
int asd_ctx_set_chunk_k(asd_ctx *ctx, int chunk_k);

/* Number of kernels the last asd_ctx_step / asd_ctx_sqt* call launched. */
int asd_ctx_last_launches(const asd_ctx *ctx);

/* Diagnostic: with on != 0, later calls record CUDA events on the stream each
 * kernel is launched on, around every RK4 step (the one-launch step kernel, or
 * the four stage kernels of one step) and every S(q,t) GEMM kernel (the
 * tcgen05 split GEMM or the FP64 GEMM); nothing is recorded while a stream is
 * being captured.  No counterpart in the reference; the benchmark uses it. */
int asd_ctx_time_kernels(asd_ctx *ctx, int on);
/* Waits for the events recorded since the last read and returns the summed
 * duration in ms and the number of kernel launches of `which` (0 = RK4 step
 * kernels, 1 = S(q,t) GEMM), then forgets them. */
int asd_ctx_kernel_time(asd_ctx *ctx, int which, double *ms, int *launches);

/* Status word set by device code (bounded waits that gave up, etc.);
 * returns ASD_OK or ASD_ERR_TIMEOUT and clears it. */
int asd_ctx_check_device_status(asd_ctx *ctx);

/* Diagnostic, host-side fault injection: the n-th device allocation of the
 * context API from now on (asd_ctx_create and the calls that allocate work
 * space on first use: host-buffer steps, the q grid, the adjoint, the FP64
 * partials) fails as cudaMalloc does on a full device, so the call returns
 * ASD_ERR_NOMEM and frees what it had taken; n = 0 switches it off.  Process
 * wide.  No counterpart in the reference (which never checks an allocation);
 * the failure-path tests use it. */
int asd_debug_fail_alloc(long n);

/* Diagnostic: waits until the context is idle, then fills with NaN bytes
 * (0xFF) every device buffer of the context whose contents do not carry over
 * between calls (stage states, the running RK4 combination, replica means at
 * t, the FP64 band, GEMM partials and result, q-grid bins, host-step staging,
 * the adjoint's state-sized work buffers).  A kernel that read any of them
 * before writing it would show NaN or changed results.  The spins, the
 * origin, the phases, the epilogue vectors and the split operands are kept.
 * No counterpart in the reference; the tests use it. */
int asd_ctx_debug_poison(asd_ctx *ctx);

/* Diagnostic: runs one of the library's bounded waits against a condition
 * that nothing satisfies -- which = 0: the mbarrier wait of the tensor-core
 * GEMM (`limit` polls); which = 1: the grid barrier of the batched kernel --
 * and returns ASD_ERR_TIMEOUT when the wait gave up and reported it, as
 * designed.  No counterpart in the reference; the failure-detection tests use
 * it (no GPU fault is involved). */
int asd_check_bounded_wait(int which, unsigned limit, void *stream);

/* Diagnostic: adds to *bad (device counter) the number of x[i] (device array)
 * for which the LLG kernels' divisions by the constants 3 and 6 (Markstein's
 * correction step) differ in any bit from the correctly rounded division.
 * No counterpart in the reference; tests use it.  Asynchronous on stream. */
int asd_check_const_division(const double *x, long n, unsigned long long *bad, void *stream);
/* Diagnostic: adds to *bad (device counter) the number of float bit patterns,
 * out of all 2^32, for which the batched kernels' FP32 divisions by 3 and 6
 * differ in any bit from the correctly rounded division (NaN = NaN).  No
 * counterpart in the reference; tests use it.  Asynchronous on stream. */
int asd_check_const_division_f32(unsigned long long *bad, void *stream);

/* Diagnostic: the bare tensor-core product of the split S(q,t) GEMM,
 * C[i*ldc + j] = sum_k Ah[i][k]Bh[j][k] + Ah[i][k]Bl[j][k] + Al[i][k]Bh[j][k]
 * in FP32, for device operands [rows][Kp] (kind 1: TF32 bit patterns in
 * float, kind 2: bf16, kind 3: fp16), rows a multiple of 256, Kp a multiple
 * of 32 (TF32) or 64 (16-bit kinds); chunk_k as for asd_ctx_set_chunk_k (the chunk partials are
 * added in FP32 here).  Asynchronous on stream.  It has no counterpart in the
 * reference; tests use it to check the tcgen05 core apart from the epilogue. */
int asd_umma_gemm_f32(int kind, long rows, int Kp, const void *a_hi, const void *a_lo,
                      const void *b_hi, const void *b_lo, float *c, long ldc, int chunk_k,
                      void *stream);

/* Diagnostic: measured FP64 throughput of the current device, the
 * denominators of the FP64 roofline fractions.  which = 0: independent
 * __fma_rn chains on the CUDA cores (an FMA counts 2 flops); which = 1:
 * 16 independent mma.sync m16n8k8 .f64 accumulators per warp (2*16*8*8 flops
 * per product).  32 warps per SM, about a millisecond; *tflops and *ms of the second
 * of two launches.  Synchronous.  No counterpart in the reference. */
int asd_measure_fp64_peak(int which, double *tflops, double *ms, void *stream);
/* Diagnostic: one warp computes D[16][8] = A[16][8] B[8][8] (row-major device
 * arrays) with mma.sync m16n8k8 .f64, loading and storing the fragments in the
 * layout the FP64 GEMM assumes; a test compares D with a host product.
 * Asynchronous on stream.  No counterpart in the reference. */
int asd_check_dmma_layout(const double *A, const double *B, double *D, void *stream);

/* S(q,t) through the split tensor-core GEMM without allocating anything.
 * No counterpart in the reference.  For callers that may not call cudaMalloc
 * or cudaFree while they step a simulation: hosts that give all device memory
 * to their own pool or caching allocator at start-up and run on a fixed
 * budget, and step loops where an allocation call would synchronise the
 * device and stall other streams.  The caller passes every input and output
 * buffer (device pointers, stream-ordered on `stream`):
 *   a_hi, a_lo, b_hi, b_lo  split operands [rows][Kp] (kind 1: TF32 bit
 *                           patterns in float; kind 2: bf16), rows a multiple
 *                           of 256 with zero padding rows, Kp a multiple of 32
 *                           (TF32) or 64 (BF16) with zero padding columns;
 *   row4, row1, col4, col1  epilogue vectors, `rows` entries each, zero past
 *                           the last site: row4[i] = (m_i, Re u_i) as float4,
 *                           row1[i] = Im u_i, col4[j] = (z_j, Re w_j),
 *                           col1[j] = Im w_j, with m, z the replica means at t
 *                           and 0 and u_i w_j = e^{-i q.(r_i - r_j)};
 *   d_out                   2 doubles: S = scale * sum_ij u_i w_j
 *                           (alpha C_ij - m_i . z_j).
 * Its only scratch (one partial per CTA, at most 1024 CTAs = 16 KiB, plus a
 * status word) is a fixed array in the library's device memory that every GPU
 * which loads the library keeps until the process exits.  Limit: at most 1024
 * CTAs, i.e. devices with up to 1024 SMs; larger launches are rejected with
 * ASD_ERR_UNSUPPORTED.  Every call looks up that array's device address in
 * the current device's context (a host-side query that allocates nothing; the
 * first call on a device also loads the library's device code there, so make
 * it before any stream capture); after cudaDeviceReset the next call finds the
 * array again.  `stream` must belong to the current device (else
 * ASD_ERR_INVALID).  All calls share the one array, so calls whose work overlaps on
 * the GPU (different streams, or different host threads) race and must be
 * ordered by the caller.  If a bounded wait in the kernel gives up, d_out
 * receives NaN. */
int asd_sqt_split_noalloc(int kind, long rows, int Kp, const void *a_hi, const void *a_lo,
                          const void *b_hi, const void *b_lo, const void *row4, const float *row1,
                          const void *col4, const float *col1, double alpha, double scale,
                          int chunk_k, double *d_out, void *stream);

/* ------------------------------------------------------ batched lattices */
/* Many independent lattices (one replica each) of different sizes and
 * parameters, stepped together by one persistent, graph-captured launch with
 * all spins resident on the GPU (in shared memory, or in L2 and HBM).  RK4
 * stages in FP32 (explicitly rounded, the reference's operation order),
 * renormalisation in FP64.  No counterpart in the reference, which runs one
 * lattice per program. */
typedef struct {
    int N;
    double J1, J2, alpha, hx, hy, hz, dt, spin_len;
} asd_lattice;
typedef struct asd_batch asd_batch;

int asd_batch_create(const asd_lattice *lattices, int count, asd_batch **out);
int asd_batch_destroy(asd_batch *batch);
int asd_batch_set_stream(asd_batch *batch, void *stream);
/* Spins of one lattice, float[N*N][3] (host). */
int asd_batch_set_spins(asd_batch *batch, int lattice, const float *spin_aos);
int asd_batch_get_spins(asd_batch *batch, int lattice, float *spin_aos);
/* nsteps RK4 steps of every lattice in one persistent launch (a CUDA graph
 * per step count); synchronous; ASD_ERR_TIMEOUT if the kernel's bounded grid
 * barrier gave up. */
int asd_batch_run(asd_batch *batch, int nsteps);
/* Global-memory kernel: spins in L2/HBM, one cooperative launch whose CTAs
 * take work items of `tile` consecutive sites (32..256, a multiple of 32),
 * `ctas_per_sm` resident CTAs per SM, a bounded grid barrier per RK4 stage.
 * Works for any batch. */
int asd_batch_configure(asd_batch *batch, int tile, int ctas_per_sm);
/* Cluster-resident kernel: every lattice lives in the shared memory of one
 * thread-block cluster of `cluster_size` CTAs (1..8; `threads` per CTA 128..896,
 * a multiple of 32, 0 = 896) for the whole run; lattices are packed onto the
 * clusters longest first and each cluster's rows split over its CTAs; halo
 * rows cross between CTAs through distributed shared memory after a cluster
 * barrier per RK4 stage.  As many clusters as the GPU holds at once.  Same
 * arithmetic as the global-memory kernel, bit for bit.  ASD_ERR_UNSUPPORTED
 * if the batch does not fit (48 bytes of shared memory per site plus halo
 * rows; lattice rows no wider than `threads`). */
int asd_batch_configure_cluster(asd_batch *batch, int cluster_size, int threads);
/* Times trial_steps steps for every cluster-resident configuration that fits
 * (cluster sizes 1..8 x 256..896 threads) and every global-memory
 * configuration (tile in {32, 64, 128, 256} x CTAs per SM in {1, 2, 4, 8},
 * as far as they fit), keeps the fastest and reports it: *tile and
 * *ctas_per_sm for the global-memory kernel, or *tile = 0 and *ctas_per_sm =
 * the cluster size for the cluster-resident one.  The spins are restored
 * afterwards. */
int asd_batch_autotune(asd_batch *batch, int trial_steps, int *tile, int *ctas_per_sm,
                       double *ms_per_step);
/* Diagnostic (host only, no GPU): the cluster-resident kernel's plan for
 * lattices of the given sides on `clusters` clusters of `cluster_size` CTAs.
 * ctas_out receives 4 ints per CTA (clusters * cluster_size CTAs, cluster by
 * cluster): first segment, segments, sites, slots per plane; segs_out (if it
 * holds seg_capacity segments) 12 ints per segment: lattice, N, first row,
 * rows, slot of its top halo row, first site, and the top and the bottom halo
 * rows' owning CTA (rank in the cluster), slot there and that CTA's slots per
 * plane; *smem_bytes the dynamic shared memory a CTA needs.  ASD_ERR_UNSUPPORTED
 * (with the outputs filled) if it exceeds smem_limit.  No counterpart in the
 * reference; tests use it. */
int asd_batch_plan_clusters(const int *sizes, int count, int cluster_size, int clusters,
                            long smem_limit, int *ctas_out, int *segs_out, int seg_capacity,
                            int *nsegs, long *smem_bytes);

/* --------------------------------------------------------- spin-state I/O */
/* The reference keeps spins only in memory; these define a file format for
 * checkpoints: a 64-byte header (magic "ASDSPIN1", int32 N, int32 nfile,
 * int64 step, double spin_len, 32 reserved bytes) followed by the spins in
 * the reference's AoS layout, little-endian doubles.  Host only; no GPU. */
int asd_spins_save(const char *path, int N, int nfile, long step, double spin_len,
                   const double *spin_aos);
/* Reads the header into N, nfile (and step, spin_len when not NULL); with
 * spin_aos == NULL only the header is read (size query), else the spins are
 * read into spin_aos, which must hold `capacity` >= nfile*N*N*3 doubles. */
int asd_spins_load(const char *path, int *N, int *nfile, long *step, double *spin_len,
                   double *spin_aos, size_t capacity);

/* ------------------------------------------------------- drop-in symbols */
/* The reference reads N, Nfile, J1, dt, nn and num_neighbor from globals its
 * program defines (llg_sqt_baseline.c:12-20).  The drop-in functions use the
 * values set here; without a call they fall back to those globals when the
 * host program defines them (weak references), else to the reference's
 * initial values (N=100, Nfile=50, J1=1.0, dt=0.02). */
int asd_set_params(int N, int Nfile, double J1, double dt);

/* llg_sqt_baseline.c:29 -- derivative[f][i][:] = H x S for every replica and
 * site, H = J1 * sum of the 4 neighbours; host arrays [Nfile][N*N][3]. */
void euler(double *spin0, double *derivative);

/* llg_sqt_baseline.c:95 -- one RK4 step: cur_input = spin + k1/6 + k2/3 +
 * k3/3 + k4/6 with k_s = dt * f(stage input); k1..k4 receive the scaled
 * increments, as in the reference. */
void runge_kutta(double *spin, double *cur_input, double *k1, double *k2, double *k3,
                 double *k4);

/* kernel_fusion/gemm_kernel.h:355 -- C += fuse_C (x) (alpha * A * B) on the
 * interleaved complex layout (re rows (i/4)*8+i%4, im rows +4, ldc >= 2*m),
 * and sum[0..1] += the sums of the updated real and imaginary parts, once per
 * K block of 240 as the reference does.  Column-major A (m x k, lda) and B
 * (k x n, ldb); all pointers are host memory.  Rows past the last multiple of
 * 4 and a last odd column are left untouched, as in the reference. */
void fused_dgemm(int *m, int *n, int *k, double *alpha, double *a, int *lda, double *b,
                 int *ldb, double *c, int *ldc, double *fuse_C, double *sum);

/* gemm/llg_sqt_mkl.c:378 -- the plain path's cblas_dgemm on the GPU:
 * C = alpha * op(A) * op(B) + beta * C with the CBLAS arguments (order
 * 101 row-major / 102 column-major; trans 111 none, 112 or 113 transpose) and
 * BLAS rules (C is not read when beta == 0; m or n == 0, or k == 0 / alpha
 * == 0 with beta == 1, do nothing).  Host pointers, synchronous; the product
 * runs on the FP64 tensor-core GEMM (mma.sync .f64), so its rounding differs
 * from a CPU BLAS only in the order of the FP64 sums.  libasd_cblas.so
 * (include/asd_cblas.h) exports it under the BLAS name, so that the
 * reference's gemm program links it in place of MKL or OpenBLAS.  Returns
 * ASD_ERR_INVALID for the arguments BLAS rejects. */
int asd_cblas_dgemm(int order, int transa, int transb, int m, int n, int k, double alpha,
                    const double *a, int lda, const double *b, int ldb, double beta, double *c,
                    int ldc);

#ifdef __cplusplus
}
#endif
#endif
