/*
 * asd_oracle.h -- CPU restatement of the reference's hot path, in plain C, FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py may load this library, and only as
 * the checker or the timed CPU arm.  The product (libasd_b200.so) never links
 * or calls it.
 *
 * Every function names the reference file:line it restates (paths relative to
 * the hwchen2017/ASD-kernel-fusion project).  Spin arrays use the reference's
 * own layout, "AoS": double[nfile][N*N][3] (llg_sqt_baseline.c:185, :202).
 *
 * Parity pins (see tests/test_oracle_pins.py): when the reference sources are
 * present, `make -C oracle ref` compiles them into oracle/_ref/ and the tests
 * check this restatement against the reference's own euler/runge_kutta (bit
 * exact, both built with -ffp-contract=off) and fused_dgemm (C bit exact, the
 * running sums to 1e-13), and tests/golden/ holds fixtures produced by the
 * reference's own functions (tests/golden/make_golden.py).
 */
#ifndef ASD_ORACLE_H
#define ASD_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int    N;          /* lattice side; sites M = N*N                          */
    int    nfile;      /* replicas ("snapshots", the K/3 axis of the GEMM)     */
    double J1;         /* nearest-neighbour exchange                           */
    double J2;         /* next-nearest (diagonal) exchange; 0 in the reference */
    double alpha;      /* Gilbert damping; 0 in the reference                  */
    double hx, hy, hz; /* Zeeman field added to H_eff; 0 in the reference      */
    double dt;         /* RK4 step                                             */
    double spin_len;   /* renormalised length: 1.0 (baseline, gemm) / 1.5 (fusion) */
} oracle_params;

/* dS/dt for every replica and site (restates euler, llg_sqt_baseline.c:29-92). */
void oracle_llg_deriv(const oracle_params *p, const double *spin, double *deriv);

/* One RK4 step in the reference's k*dt form; cur receives the un-normalised
 * result, k1..k4 the scaled stage increments (runge_kutta, :95-142).        */
void oracle_rk4(const oracle_params *p, const double *spin, double *cur,
                double *k1, double *k2, double *k3, double *k4);

/* spin_out = spin_len * cur / |cur| (llg_sqt_baseline.c:298-309; the fusion
 * variant uses 1.5, llg_sqt_fusion.c:350-361).                               */
void oracle_renorm(const oracle_params *p, const double *cur, double *spin_out);

/* nsteps of rk4 + renorm in place on spin (the main loop body, :289-309).    */
int oracle_steps(const oracle_params *p, double *spin, int nsteps);

/* S(q,t), OpenBLAS variant (gemm/llg_sqt_mkl.c:349-423): fint_avg, A pack,
 * C = (1/nfile) A B with a naive dot product, outer subtraction, sum C*qmat,
 * divided by N^2.  O(N^4 K).  q = 2*pi*(vx, vy)/N.                          */
void oracle_sqt_gemm(int N, int nfile, int vx, int vy, const double *spin_t,
                     const double *spin_0, double out[2]);

/* S(q,t), baseline variant (llg_sqt_baseline.c:320-418), including the
 * reference's defect: the connected subtraction at :392-394 happens after
 * ssum is formed, so this is the NON-connected correlation.                 */
void oracle_sqt_direct(int N, int nfile, int vx, int vy, const double *spin_t,
                       const double *spin_0, double out[2]);

/* S(q,t), kernel-fusion variant (llg_sqt_fusion.c:370-441): interleaved qmat,
 * C initialised to -(outer)*q, then oracle_fused_dgemm, then sum / N^2.     */
void oracle_sqt_fused(int N, int nfile, int vx, int vy, const double *spin_t,
                      const double *spin_0, double out[2]);

/* S(q,t) through the rank-1 separable phase, O(N^2 K), long double
 * accumulation: an independent check of the GEMM forms at any size.         */
void oracle_sqt_factorized(int N, int nfile, int vx, int vy, const double *spin_t,
                           const double *spin_0, double out[2]);

/* The full q grid: out_re/out_im[qr*N + qc] = S(q = 2 pi (qr, qc)/N, t) in the
 * connected (OpenBLAS variant) convention, via displacement bins.            */
void oracle_sqt_grid(int N, int nfile, const double *spin_t, const double *spin_0,
                     double *out_re, double *out_im);

/* Restatement of fused_dgemm (kernel_fusion/gemm_kernel.h:355-422) with the
 * reference's exact semantics: alpha folded into A (tcopy, :227-249), K in
 * blocks of 240 (:293, :378), a sequential FMA chain per C element (:9-35),
 * C = fma(q, acc, C) in the interleaved re/im layout (:39-46), and the sum of
 * every updated C value added to sum[0..1] once per K block (:59-88).  Rows
 * beyond the last multiple of 4 and a last odd column are left untouched
 * (:199-204, :219-222).  Column-major A (lda), B (ldb); C and q use ldc.     */
void oracle_fused_dgemm(int m, int n, int k, double alpha, const double *a, int lda,
                        const double *b, int ldb, double *c, int ldc,
                        const double *q, double *sum);

/* nsteps of the FP32 RK4 with FP64 renormalisation of the batched-lattice GPU
 * path, one replica, spins float[N*N][3] in place. */
int oracle_steps_f32(const oracle_params *p, float *spin, int nsteps);

/* Interleaved complex layout of the fusion variant (llg_sqt_fusion.c:324-327). */
static inline long oracle_row_re(long i) { return (i / 4) * 8 + (i % 4); }

#ifdef __cplusplus
}
#endif
#endif
