/*
 * ref_glue.c -- a harness around the reference's OWN compiled functions.
 *
 * TEST INFRASTRUCTURE ONLY.  `make -C oracle ref` compiles this file together
 * with one of the reference's programs, taken unmodified from where it lies
 * (main renamed by -Dmain=asd_ref_main), into oracle/_ref/libref_<variant>.so.
 * The reference keeps its state in globals defined by that program
 * (llg_sqt_baseline.c:12-20) and its per-step glue inside main; this harness
 * sets the globals the way main does and repeats main's glue around the
 * reference's euler / runge_kutta / fused_dgemm / cblas_dgemm calls, with
 * seeded spins injected (the reference's own initialisation divides integers
 * and yields NaN, llg_sqt_baseline.c:196-206).
 *
 * Variants (selected by -DREF_VARIANT_*):
 *   BASELINE  llg_sqt_baseline.c  -> runge_kutta, direct S(q,t)
 *   FUSION    llg_sqt_fusion.c    -> runge_kutta, fused_dgemm S(q,t)
 *   GEMM      llg_sqt_mkl.c       -> runge_kutta, cblas_dgemm S(q,t)
 */
#include <complex.h>
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* globals defined by the reference program */
extern int N, num_neighbor, MCsweep, Nfile, vx, vy, trd;
extern double J1, dt;
extern int nn[4][2];
void euler(double *spin0, double *derivative);
void runge_kutta(double *spin, double *cur_input, double *k1, double *k2, double *k3, double *k4);
#if defined(REF_VARIANT_FUSION)
void fused_dgemm(int *m, int *n, int *k, double *alpha, double *a, int *lda, double *b, int *ldb,
                 double *c, int *ldc, double *fuse_C, double *sum);
#endif
#if defined(REF_VARIANT_GEMM)
void cblas_dgemm(int order, int transa, int transb, int m, int n, int k, double alpha,
                 const double *a, int lda, const double *b, int ldb, double beta, double *c, int ldc);
#endif

static int g_threads = 1;

/* main's set-up of the globals (llg_sqt_baseline.c:150-178, :214-216). */
int ref_setup(int n_, int nfile_, double j1_, double dt_, int threads)
{
    N = n_;
    Nfile = nfile_;
    J1 = j1_;
    dt = dt_;
    num_neighbor = 4;
    vx = N / 10;
    vy = N / 10;
    nn[0][0] = 1, nn[0][1] = 0;
    nn[1][0] = -1, nn[1][1] = 0;
    nn[2][0] = 0, nn[2][1] = -1;
    nn[3][0] = 0, nn[3][1] = 1;
    int tot = threads > 0 ? threads : omp_get_max_threads();
    g_threads = tot < 128 ? tot : 128; /* the reference caps at 128 (sum[128*2]) */
    omp_set_num_threads(g_threads);
    return g_threads;
}

int ref_get_vx(void) { return vx; }

void ref_euler(double *spin, double *deriv) { euler(spin, deriv); }

void ref_runge_kutta(double *spin, double *cur, double *k1, double *k2, double *k3, double *k4)
{
    runge_kutta(spin, cur, k1, k2, k3, k4);
}

/* nsteps of runge_kutta + main's renormalisation (llg_sqt_baseline.c:296-309;
 * spin_len 1.5 reproduces llg_sqt_fusion.c:350-361).  With t_last != NULL it
 * receives the wall time of the last step alone (the work buffers, like
 * main's, are allocated and touched before it). */
int ref_steps_timed(double *spin, int nsteps, double spin_len, double *t_last)
{
    const size_t n = (size_t)Nfile * N * N * 3;
    double *buf = (double *)malloc(5 * n * sizeof(double));
    if (!buf) return -1;
    double *cur = buf, *k1 = buf + n, *k2 = buf + 2 * n, *k3 = buf + 3 * n, *k4 = buf + 4 * n;
    for (int s = 0; s < nsteps; s++) {
        const double t0 = omp_get_wtime();
        runge_kutta(spin, cur, k1, k2, k3, k4);
#pragma omp parallel for
        for (long j = 0; j < (long)Nfile * N * N; j++) {
            double tx = cur[j * 3], ty = cur[j * 3 + 1], tz = cur[j * 3 + 2];
            double nrm = sqrt(tx * tx + ty * ty + tz * tz);
            if (spin_len == 1.0) {
                tx = tx / nrm;
                ty = ty / nrm;
                tz = tz / nrm;
            } else {
                tx = spin_len * tx / nrm;
                ty = spin_len * ty / nrm;
                tz = spin_len * tz / nrm;
            }
            spin[j * 3] = tx, spin[j * 3 + 1] = ty, spin[j * 3 + 2] = tz;
        }
        if (t_last) *t_last = omp_get_wtime() - t0;
    }
    free(buf);
    return 0;
}

int ref_steps(double *spin, int nsteps, double spin_len)
{
    return ref_steps_timed(spin, nsteps, spin_len, NULL);
}

static void mean_over_replicas(const double *spin, double *avg)
{
#pragma omp parallel for
    for (int i = 0; i < N * N; i++) {
        double tx = 0.0, ty = 0.0, tz = 0.0;
        for (int id = 0; id < Nfile; id++) {
            tx += spin[id * N * N * 3 + i * 3];
            ty += spin[id * N * N * 3 + i * 3 + 1];
            tz += spin[id * N * N * 3 + i * 3 + 2];
        }
        tx /= (double)Nfile;
        ty /= (double)Nfile;
        tz /= (double)Nfile;
        avg[i * 3] = tx, avg[i * 3 + 1] = ty, avg[i * 3 + 2] = tz;
    }
}

#if defined(REF_VARIANT_FUSION)
/* Persistent state for the fused S(q,t): qmat is formed once, as in main. */
static double *g_qmat, *g_cmat, *g_spint, *g_spin_zero, *g_zerot, *g_fint;
static long g_rows; /* rows of C processed (a band of M for bounded timing) */

void ref_fusion_free(void)
{
    free(g_qmat), free(g_cmat), free(g_spint), free(g_spin_zero), free(g_zerot), free(g_fint);
    g_qmat = g_cmat = g_spint = g_spin_zero = g_zerot = g_fint = NULL;
}

/* llg_sqt_fusion.c:235-268 (spin_zero, zerot_avg) and :298-333 (qmat).  rows
 * limits C to its first `rows` rows (all M when rows <= 0), so that a bounded
 * CPU sample of the same GEMM can be timed at large N. */
int ref_fusion_init(const double *spin_0, long rows)
{
    ref_fusion_free();
    const long M = (long)N * N;
    const int K = Nfile * 3;
    g_rows = (rows <= 0 || rows > M) ? M : rows;
    g_rows -= g_rows % 4;
    if (g_rows <= 0) return -1;
    g_spin_zero = (double *)malloc((size_t)M * K * sizeof(double));
    g_spint = (double *)malloc((size_t)M * K * sizeof(double));
    g_zerot = (double *)malloc((size_t)M * 3 * sizeof(double));
    g_fint = (double *)malloc((size_t)M * 3 * sizeof(double));
    g_qmat = (double *)malloc((size_t)2 * g_rows * M * sizeof(double));
    g_cmat = (double *)malloc((size_t)2 * g_rows * M * sizeof(double));
    if (!g_spin_zero || !g_spint || !g_zerot || !g_fint || !g_qmat || !g_cmat) {
        ref_fusion_free();
        return -2;
    }
#pragma omp parallel for
    for (long i = 0; i < M; i++)
        for (int j = 0; j < Nfile; j++) {
            g_spin_zero[i * Nfile * 3 + j * 3] = spin_0[j * M * 3 + i * 3];
            g_spin_zero[i * Nfile * 3 + j * 3 + 1] = spin_0[j * M * 3 + i * 3 + 1];
            g_spin_zero[i * Nfile * 3 + j * 3 + 2] = spin_0[j * M * 3 + i * 3 + 2];
        }
    mean_over_replicas(spin_0, g_zerot);
    const double qx = 2.0 * M_PI * vx / (double)N;
    const double qy = 2.0 * M_PI * vy / (double)N;
    const long mm = g_rows;
#pragma omp parallel for
    for (long j = 0; j < M; j++)
        for (long i = 0; i < mm; i++) {
            int ri = (int)(i / N), ci = (int)(i % N), rj = (int)(j / N), cj = (int)(j % N);
            double dffr = ri - rj, dffc = ci - cj;
            double complex tmp = cexp(CMPLX(0.0, -1.0) * (qx * dffr + qy * dffc));
            long re = (i / 4) * 8 + (i % 4) + j * 2 * mm;
            g_qmat[re] = creal(tmp);
            g_qmat[re + 4] = cimag(tmp);
        }
    return 0;
}

/* One S(q,t) evaluation, llg_sqt_fusion.c:370-441, over the first g_rows
 * rows.  t_pack (if not NULL) receives the time of the A pack and the replica
 * means (O(M K), the same for any band), t_band the time of the C set-up and
 * fused_dgemm over the band (proportional to its rows). */
int ref_fusion_sqt_timed(const double *spin_all, double out[2], double *t_pack, double *t_band)
{
    const long M = (long)N * N, mm = g_rows;
    if (!g_cmat) return -1;
    const double t0 = omp_get_wtime();
#pragma omp parallel for
    for (long j = 0; j < M; j++)
        for (int i = 0; i < Nfile; i++) {
            g_spint[j + (i * 3) * M] = spin_all[i * M * 3 + j * 3];
            g_spint[j + (i * 3 + 1) * M] = spin_all[i * M * 3 + j * 3 + 1];
            g_spint[j + (i * 3 + 2) * M] = spin_all[i * M * 3 + j * 3 + 2];
        }
    mean_over_replicas(spin_all, g_fint);
    const double t1 = omp_get_wtime();
#pragma omp parallel for
    for (long j = 0; j < M; j++) {
        double zx = g_zerot[j * 3], zy = g_zerot[j * 3 + 1], zz = g_zerot[j * 3 + 2];
        for (long i = 0; i < mm; i++) {
            double tmp = zx * g_fint[i * 3] + zy * g_fint[i * 3 + 1] + zz * g_fint[i * 3 + 2];
            tmp *= -1.0;
            long re = (i / 4) * 8 + (i % 4) + j * 2 * mm;
            g_cmat[re] = tmp * g_qmat[re];
            g_cmat[re + 4] = tmp * g_qmat[re + 4];
        }
    }
    double sum[128 * 2];
    memset(sum, 0, sizeof(sum));
    int m_ = (int)mm, n_ = (int)M, k_ = Nfile * 3, lda = (int)M, ldb = Nfile * 3, ldc = (int)(2 * mm);
    double alpha = 1.0 / (double)Nfile;
    fused_dgemm(&m_, &n_, &k_, &alpha, g_spint, &lda, g_spin_zero, &ldb, g_cmat, &ldc, g_qmat, sum);
    double complex res = CMPLX(0.0, 0.0);
    for (int i = 0; i < 128; i++) res += CMPLX(sum[2 * i], sum[2 * i + 1]);
    res /= (double)(N * N);
    out[0] = creal(res);
    out[1] = cimag(res);
    const double t2 = omp_get_wtime();
    if (t_pack) *t_pack = t1 - t0;
    if (t_band) *t_band = t2 - t1;
    return 0;
}

int ref_fusion_sqt(const double *spin_all, double out[2])
{
    return ref_fusion_sqt_timed(spin_all, out, NULL, NULL);
}

/* Direct access to the reference's fused_dgemm, for element-level pins. */
void ref_fused_dgemm(int m, int n, int k, double alpha, double *a, int lda, double *b, int ldb,
                     double *c, int ldc, double *q, double *sum)
{
    fused_dgemm(&m, &n, &k, &alpha, a, &lda, b, &ldb, c, &ldc, q, sum);
}
#endif

#if defined(REF_VARIANT_GEMM)
/* gemm/llg_sqt_mkl.c:349-423 with the reference's cblas_dgemm call (:378),
 * over the first `rows` rows of C (all M when rows <= 0 or rows > M), so that
 * a bounded CPU sample of the same program can be timed where the whole
 * (M x M) C does not fit in host memory.  t_pack (if not NULL) receives the
 * time of the per-step A pack and replica means (O(M K), the same for any
 * band; the program's one-time B pack is not timed), t_band the time of
 * cblas_dgemm and the subtraction / phase sweep over the band (proportional
 * to its rows). */
int ref_gemm_sqt_band(const double *spin_all, const double *spin_0, long rows, double out[2],
                      double *t_pack, double *t_band)
{
    const long M = (long)N * N;
    const int K = Nfile * 3;
    const long mm = (rows <= 0 || rows > M) ? M : rows;
    double *spin_zero = (double *)malloc((size_t)M * K * sizeof(double));
    double *spint = (double *)malloc((size_t)M * K * sizeof(double));
    double *zerot = (double *)malloc((size_t)M * 3 * sizeof(double));
    double *fint = (double *)malloc((size_t)M * 3 * sizeof(double));
    double *cmat = (double *)malloc((size_t)mm * M * sizeof(double));
    if (!spin_zero || !spint || !zerot || !fint || !cmat) {
        free(spin_zero), free(spint), free(zerot), free(fint), free(cmat);
        return -2;
    }
    /* first touch of the work arrays outside the timing (the reference's
     * program allocates them once and reuses them every step) */
    memset(cmat, 0, (size_t)mm * M * sizeof(double));
    memset(spint, 0, (size_t)M * K * sizeof(double));
    /* the program's one-time set-up (spin_zero and zerot before the time loop) */
#pragma omp parallel for
    for (long i = 0; i < M; i++)
        for (int j = 0; j < Nfile; j++)
            for (int c = 0; c < 3; c++) spin_zero[i * Nfile * 3 + j * 3 + c] = spin_0[j * M * 3 + i * 3 + c];
    mean_over_replicas(spin_0, zerot);
    /* per step: the replica means and the A pack, then the GEMM and the sweep */
    const double t0 = omp_get_wtime();
    mean_over_replicas(spin_all, fint);
#pragma omp parallel for
    for (long j = 0; j < M; j++)
        for (int i = 0; i < Nfile; i++)
            for (int c = 0; c < 3; c++) spint[j + (i * 3 + c) * M] = spin_all[i * M * 3 + j * 3 + c];
    const double t1 = omp_get_wtime();
    const double alpha = 1.0 / (double)Nfile;
    cblas_dgemm(102 /*ColMajor*/, 111 /*NoTrans*/, 111, (int)mm, (int)M, K, alpha, spint, (int)M,
                spin_zero, K, 0.0, cmat, (int)mm);
    const double qx = 2.0 * M_PI * vx / (double)N;
    const double qy = 2.0 * M_PI * vy / (double)N;
    double re = 0.0, im = 0.0;
#pragma omp parallel for reduction(+ : re, im)
    for (long j = 0; j < M; j++) {
        double zx = zerot[j * 3], zy = zerot[j * 3 + 1], zz = zerot[j * 3 + 2];
        for (long i = 0; i < mm; i++) {
            double outer = fint[i * 3] * zx + fint[i * 3 + 1] * zy + fint[i * 3 + 2] * zz;
            double cij = cmat[i + j * mm] - outer;
            int ri = (int)(i / N), ci = (int)(i % N), rj = (int)(j / N), cj = (int)(j % N);
            double dffr = ri - rj, dffc = ci - cj;
            double complex q = cexp(CMPLX(0.0, -1.0) * (qx * dffr + qy * dffc));
            re += cij * creal(q);
            im += cij * cimag(q);
        }
    }
    const double t2 = omp_get_wtime();
    out[0] = re / (double)(N * N);
    out[1] = im / (double)(N * N);
    if (t_pack) *t_pack = t1 - t0;
    if (t_band) *t_band = t2 - t1;
    free(spin_zero), free(spint), free(zerot), free(fint), free(cmat);
    return 0;
}

int ref_gemm_sqt(const double *spin_all, const double *spin_0, double out[2])
{
    return ref_gemm_sqt_band(spin_all, spin_0, 0, out, NULL, NULL);
}
#endif
