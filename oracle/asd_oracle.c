/*
 * asd_oracle.c -- CPU restatement of the reference's hot path (FP64, plain C).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * "port" arm.  The product library never links or calls this file.
 *
 * Build: oracle/Makefile, with -ffp-contract=off so that every a*b+c below is
 * two roundings, exactly as written; fma() is called explicitly where the
 * reference's assembly uses a fused multiply-add.
 *
 * Reference citations are file:line within hwchen2017/ASD-kernel-fusion.
 */
#include "asd_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Neighbour offsets (drow, dcol) in the reference's order (llg_sqt_baseline.c:175-178). */
static const int kNN[4][2] = {{1, 0}, {-1, 0}, {0, -1}, {0, 1}};
/* Next-nearest (diagonal) offsets: an extension, applied after the four
 * nearest neighbours so that J2 = 0 leaves the reference's arithmetic intact. */
static const int kNNN[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

/* euler, llg_sqt_baseline.c:29-92, extended.  H = J1 * sum_nn S (+ J2 * sum_nnn S)
 * (+ h); tau = H x S (v3d_cross, v3d.h:48-53); with damping
 * dS/dt = g * (tau + alpha * (S x tau)), g = 1/(1+alpha^2), which is the
 * Landau-Lifshitz-Gilbert equation -g [S x H + alpha S x (S x H)].  With
 * alpha = J2 = h = 0 the arithmetic is the reference's, operation for operation. */
void oracle_llg_deriv(const oracle_params *p, const double *spin, double *deriv)
{
    const int N = p->N;
    const long M = (long)N * N;
    const int use_j2 = (p->J2 != 0.0);
    const int use_h = (p->hx != 0.0 || p->hy != 0.0 || p->hz != 0.0);
    const int use_damp = (p->alpha != 0.0);
    const double g = 1.0 / (1.0 + p->alpha * p->alpha);

    for (int id = 0; id < p->nfile; id++) {
        const double *s_rep = spin + (long)id * M * 3;
        double *d_rep = deriv + (long)id * M * 3;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < M; i++) {
            const int row = (int)(i / N), col = (int)(i % N);
            const double sx = s_rep[i * 3], sy = s_rep[i * 3 + 1], sz = s_rep[i * 3 + 2];
            double ex = 0.0, ey = 0.0, ez = 0.0;
            for (int j = 0; j < 4; j++) {
                const int nr = (row + kNN[j][0] + N) % N;
                const int nc = (col + kNN[j][1] + N) % N;
                const double *t = s_rep + ((long)nr * N + nc) * 3;
                ex += (t[0] * p->J1);
                ey += (t[1] * p->J1);
                ez += (t[2] * p->J1);
            }
            if (use_j2) {
                for (int j = 0; j < 4; j++) {
                    const int nr = (row + kNNN[j][0] + N) % N;
                    const int nc = (col + kNNN[j][1] + N) % N;
                    const double *t = s_rep + ((long)nr * N + nc) * 3;
                    ex += (t[0] * p->J2);
                    ey += (t[1] * p->J2);
                    ez += (t[2] * p->J2);
                }
            }
            if (use_h) {
                ex += p->hx;
                ey += p->hy;
                ez += p->hz;
            }
            /* tau = H x S */
            const double tx = ey * sz - ez * sy;
            const double ty = ez * sx - ex * sz;
            const double tz = ex * sy - ey * sx;
            if (use_damp) {
                /* S x tau */
                const double ux = sy * tz - sz * ty;
                const double uy = sz * tx - sx * tz;
                const double uz = sx * ty - sy * tx;
                d_rep[i * 3] = g * (tx + p->alpha * ux);
                d_rep[i * 3 + 1] = g * (ty + p->alpha * uy);
                d_rep[i * 3 + 2] = g * (tz + p->alpha * uz);
            } else {
                d_rep[i * 3] = tx;
                d_rep[i * 3 + 1] = ty;
                d_rep[i * 3 + 2] = tz;
            }
        }
    }
}

/* runge_kutta, llg_sqt_baseline.c:95-142: classic RK4 with k = dt * f(y),
 * stage inputs y + k1/2, y + k2/2, y + k3 and the final
 * y + k1/6 + k2/3 + k3/3 + k4/6, summed left to right. */
void oracle_rk4(const oracle_params *p, const double *spin, double *cur,
                double *k1, double *k2, double *k3, double *k4)
{
    const long n = (long)p->nfile * p->N * p->N * 3;
    const double dt = p->dt;
    memcpy(cur, spin, (size_t)n * sizeof(double));
    oracle_llg_deriv(p, cur, k1);
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; j++) {
        k1[j] *= dt;
        cur[j] = spin[j] + k1[j] / 2.0;
    }
    oracle_llg_deriv(p, cur, k2);
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; j++) {
        k2[j] *= dt;
        cur[j] = spin[j] + k2[j] / 2.0;
    }
    oracle_llg_deriv(p, cur, k3);
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; j++) {
        k3[j] *= dt;
        cur[j] = spin[j] + k3[j];
    }
    oracle_llg_deriv(p, cur, k4);
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; j++) {
        k4[j] *= dt;
        cur[j] = spin[j] + k1[j] / 6.0 + k2[j] / 3.0 + k3[j] / 3.0 + k4[j] / 6.0;
    }
}

/* Renormalisation, llg_sqt_baseline.c:298-309 (length 1) and
 * llg_sqt_fusion.c:350-361 (length 1.5): (s * x) / sqrt(x*x + y*y + z*z). */
void oracle_renorm(const oracle_params *p, const double *cur, double *spin_out)
{
    const long n = (long)p->nfile * p->N * p->N;
    const double s = p->spin_len;
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; j++) {
        double tx = cur[j * 3], ty = cur[j * 3 + 1], tz = cur[j * 3 + 2];
        const double nrm = sqrt(tx * tx + ty * ty + tz * tz);
        spin_out[j * 3] = s * tx / nrm;
        spin_out[j * 3 + 1] = s * ty / nrm;
        spin_out[j * 3 + 2] = s * tz / nrm;
    }
}

int oracle_steps(const oracle_params *p, double *spin, int nsteps)
{
    const size_t n = (size_t)p->nfile * p->N * p->N * 3;
    double *buf = (double *)malloc(5 * n * sizeof(double));
    if (!buf) return -1;
    double *cur = buf, *k1 = buf + n, *k2 = buf + 2 * n, *k3 = buf + 3 * n, *k4 = buf + 4 * n;
    for (int s = 0; s < nsteps; s++) {
        oracle_rk4(p, spin, cur, k1, k2, k3, k4);
        oracle_renorm(p, cur, spin);
    }
    free(buf);
    return 0;
}

/* ---------------------------------------------------------------- S(q,t) */

static void q_vector(int N, int vx, int vy, double *qx, double *qy)
{
    /* llg_sqt_baseline.c:267-268 */
    *qx = 2.0 * M_PI * vx / (double)N;
    *qy = 2.0 * M_PI * vy / (double)N;
}

/* Phase e^{-i q.(r_i - r_j)} exactly as the reference forms it
 * (gemm/llg_sqt_mkl.c:294-299, llg_sqt_fusion.c:318-322). */
static double complex phase_ij(int N, double qx, double qy, long i, long j)
{
    const int ri = (int)(i / N), ci = (int)(i % N);
    const int rj = (int)(j / N), cj = (int)(j % N);
    const double dffr = ri - rj;
    const double dffc = ci - cj;
    return cexp(CMPLX(0.0, -1.0) * (qx * dffr + qy * dffc));
}

/* Per-site replica means (llg_sqt_baseline.c:240-259 for t = 0, :320-337 for t). */
static void replica_mean(int N, int nfile, const double *spin, double *avg)
{
    const long M = (long)N * N;
    for (long i = 0; i < M; i++) {
        double tx = 0.0, ty = 0.0, tz = 0.0;
        for (int id = 0; id < nfile; id++) {
            tx += spin[(long)id * M * 3 + i * 3];
            ty += spin[(long)id * M * 3 + i * 3 + 1];
            tz += spin[(long)id * M * 3 + i * 3 + 2];
        }
        tx /= (double)nfile;
        ty /= (double)nfile;
        tz /= (double)nfile;
        avg[i * 3] = tx;
        avg[i * 3 + 1] = ty;
        avg[i * 3 + 2] = tz;
    }
}

void oracle_sqt_gemm(int N, int nfile, int vx, int vy, const double *spin_t,
                     const double *spin_0, double out[2])
{
    const long M = (long)N * N;
    const int K = 3 * nfile;
    const double alpha = 1.0 / (double)nfile; /* gemm/llg_sqt_mkl.c:302 */
    double qx, qy;
    q_vector(N, vx, vy, &qx, &qy);
    double *fint = (double *)malloc((size_t)M * 3 * sizeof(double));
    double *zerot = (double *)malloc((size_t)M * 3 * sizeof(double));
    double *colsum = (double *)malloc((size_t)M * 2 * sizeof(double));
    replica_mean(N, nfile, spin_t, fint);
    replica_mean(N, nfile, spin_0, zerot);

#pragma omp parallel for schedule(static)
    for (long j = 0; j < M; j++) {
        const double zx = zerot[j * 3], zy = zerot[j * 3 + 1], zz = zerot[j * 3 + 2];
        double sre = 0.0, sim = 0.0;
        for (long i = 0; i < M; i++) {
            /* C_ij = alpha * sum_k A(i,k) B(k,j); A(i, 3f+c) = spin_t[f][i][c]
             * (A pack, :369-376), B(3f+c, j) = spin_0[f][j][c] (spin_zero). */
            double acc = 0.0;
            for (int k = 0; k < K; k++) {
                const int f = k / 3, c = k % 3;
                acc += spin_t[(long)f * M * 3 + i * 3 + c] * spin_0[(long)f * M * 3 + j * 3 + c];
            }
            double cij = alpha * acc;
            const double outer = fint[i * 3] * zx + fint[i * 3 + 1] * zy + fint[i * 3 + 2] * zz;
            cij -= outer; /* :395-399 */
            const double complex q = phase_ij(N, qx, qy, i, j);
            sre += cij * creal(q); /* :411 */
            sim += cij * cimag(q);
        }
        colsum[j * 2] = sre;
        colsum[j * 2 + 1] = sim;
    }
    double re = 0.0, im = 0.0;
    for (long j = 0; j < M; j++) {
        re += colsum[j * 2];
        im += colsum[j * 2 + 1];
    }
    out[0] = re / (double)(N * N); /* :422 */
    out[1] = im / (double)(N * N);
    free(fint);
    free(zerot);
    free(colsum);
}

void oracle_sqt_direct(int N, int nfile, int vx, int vy, const double *spin_t,
                       const double *spin_0, double out[2])
{
    const long M = (long)N * N;
    double qx, qy;
    q_vector(N, vx, vy, &qx, &qy);
    double *rowsum = (double *)malloc((size_t)M * 2 * sizeof(double));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; i++) {
        double sre = 0.0, sim = 0.0;
        for (long j = 0; j < M; j++) {
            double t0 = 0.0, t1 = 0.0, t2 = 0.0;
            for (int id = 0; id < nfile; id++) {
                const double *a = spin_t + (long)id * M * 3 + i * 3;
                const double *z = spin_0 + (long)id * M * 3 + j * 3;
                t0 += a[0] * z[0];
                t1 += a[1] * z[1];
                t2 += a[2] * z[2];
            }
            t0 /= (double)nfile;
            t1 /= (double)nfile;
            t2 /= (double)nfile;
            /* :384 -- the subtraction at :392-394 follows and is never used */
            const double ssum = t0 + t1 + t2;
            const double complex q = phase_ij(N, qx, qy, i, j);
            sre += creal(q) * ssum;
            sim += cimag(q) * ssum;
        }
        rowsum[i * 2] = sre;
        rowsum[i * 2 + 1] = sim;
    }
    double re = 0.0, im = 0.0;
    for (long i = 0; i < M; i++) {
        re += rowsum[i * 2];
        im += rowsum[i * 2 + 1];
    }
    out[0] = re / ((double)N * N); /* :418 */
    out[1] = im / ((double)N * N);
    free(rowsum);
}

void oracle_fused_dgemm(int m, int n, int k, double alpha, const double *a, int lda,
                        const double *b, int ldb, double *c, int ldc,
                        const double *q, double *sum)
{
    const int m4 = m - m % 4; /* KERNEL works on m4 blocks only (gemm_kernel.h:199-204) */
    const int n2 = n - n % 2; /* and on 12/8/4/2-wide column strips (:219-222) */
    double *colsum = (double *)malloc((size_t)(n2 > 0 ? n2 : 1) * 2 * sizeof(double));
    for (int k0 = 0; k0 < k; k0 += 240) { /* BLOCKDIM_K (:293, :378-379) */
        const int kinc = (k - k0 > 240) ? 240 : k - k0;
#pragma omp parallel for schedule(static)
        for (int j = 0; j < n2; j++) {
            double sre = 0.0, sim = 0.0;
            for (int i = 0; i < m4; i++) {
                double acc = 0.0;
                for (int kk = k0; kk < k0 + kinc; kk++) {
                    const double as = a[i + (long)kk * lda] * alpha; /* tcopy (:238) */
                    acc = fma(as, b[kk + (long)j * ldb], acc);
                }
                const long ir = oracle_row_re(i) + (long)j * ldc;
                c[ir] = fma(q[ir], acc, c[ir]);
                c[ir + 4] = fma(q[ir + 4], acc, c[ir + 4]);
                sre += c[ir];
                sim += c[ir + 4];
            }
            colsum[j * 2] = sre;
            colsum[j * 2 + 1] = sim;
        }
        double re = 0.0, im = 0.0;
        for (int j = 0; j < n2; j++) {
            re += colsum[j * 2];
            im += colsum[j * 2 + 1];
        }
        sum[0] += re;
        sum[1] += im;
    }
    free(colsum);
}

void oracle_sqt_fused(int N, int nfile, int vx, int vy, const double *spin_t,
                      const double *spin_0, double out[2])
{
    const long M = (long)N * N;
    const int K = 3 * nfile;
    const double alpha = 1.0 / (double)nfile; /* llg_sqt_fusion.c:295 */
    double qx, qy;
    q_vector(N, vx, vy, &qx, &qy);
    double *spint = (double *)malloc((size_t)M * K * sizeof(double));
    double *spin_zero = (double *)malloc((size_t)M * K * sizeof(double));
    double *fint = (double *)malloc((size_t)M * 3 * sizeof(double));
    double *zerot = (double *)malloc((size_t)M * 3 * sizeof(double));
    double *cmat = (double *)malloc((size_t)2 * M * M * sizeof(double));
    double *qmat = (double *)malloc((size_t)2 * M * M * sizeof(double));

    /* spin_zero transpose (:235-245) and A pack (:370-377) */
    for (long i = 0; i < M; i++)
        for (int f = 0; f < nfile; f++)
            for (int c = 0; c < 3; c++) {
                spin_zero[i * K + f * 3 + c] = spin_0[(long)f * M * 3 + i * 3 + c];
                spint[i + (long)(f * 3 + c) * M] = spin_t[(long)f * M * 3 + i * 3 + c];
            }
    replica_mean(N, nfile, spin_0, zerot);
    replica_mean(N, nfile, spin_t, fint);

    /* qmat (:308-333) and C = -(outer) * q (:402-426), interleaved re/im */
#pragma omp parallel for schedule(static)
    for (long j = 0; j < M; j++) {
        const double zx = zerot[j * 3], zy = zerot[j * 3 + 1], zz = zerot[j * 3 + 2];
        for (long i = 0; i < M; i++) {
            const double complex qq = phase_ij(N, qx, qy, i, j);
            const long ir = oracle_row_re(i) + j * 2 * M;
            qmat[ir] = creal(qq);
            qmat[ir + 4] = cimag(qq);
            double tmp = zx * fint[i * 3] + zy * fint[i * 3 + 1] + zz * fint[i * 3 + 2];
            tmp *= -1.0;
            cmat[ir] = tmp * qmat[ir];
            cmat[ir + 4] = tmp * qmat[ir + 4];
        }
    }
    double sum[2] = {0.0, 0.0};
    oracle_fused_dgemm((int)M, (int)M, K, alpha, spint, (int)M, spin_zero, K, cmat,
                       (int)(2 * M), qmat, sum);
    out[0] = sum[0] / (double)(N * N); /* :441 */
    out[1] = sum[1] / (double)(N * N);
    free(spint);
    free(spin_zero);
    free(fint);
    free(zerot);
    free(cmat);
    free(qmat);
}

void oracle_sqt_factorized(int N, int nfile, int vx, int vy, const double *spin_t,
                           const double *spin_0, double out[2])
{
    const long M = (long)N * N;
    const long double qx = 2.0L * 3.14159265358979323846264338327950288L * vx / (long double)N;
    const long double qy = 2.0L * 3.14159265358979323846264338327950288L * vy / (long double)N;
    long double *ure = (long double *)malloc((size_t)M * sizeof(long double));
    long double *uim = (long double *)malloc((size_t)M * sizeof(long double));
    for (long i = 0; i < M; i++) {
        const long double th = qx * (long double)(i / N) + qy * (long double)(i % N);
        ure[i] = cosl(th);
        uim[i] = -sinl(th); /* u_i = e^{-i q.r_i}; the phase is u_i * conj(u_j) */
    }
    /* sum_k F_k conj-side G_k with F_k = sum_i u_i A_ik, G_k = sum_j conj(u_j) B_jk,
     * plus the same contraction of the replica means for the outer term. */
    long double acc_re = 0.0L, acc_im = 0.0L;
    long double fm_re[3] = {0, 0, 0}, fm_im[3] = {0, 0, 0};
    long double zm_re[3] = {0, 0, 0}, zm_im[3] = {0, 0, 0};
    for (int f = 0; f < nfile; f++) {
        for (int c = 0; c < 3; c++) {
            long double fre = 0, fim = 0, gre = 0, gim = 0;
            for (long i = 0; i < M; i++) {
                const long double a = spin_t[(long)f * M * 3 + i * 3 + c];
                const long double b = spin_0[(long)f * M * 3 + i * 3 + c];
                fre += ure[i] * a;
                fim += uim[i] * a;
                gre += ure[i] * b;
                gim -= uim[i] * b;
            }
            acc_re += fre * gre - fim * gim;
            acc_im += fre * gim + fim * gre;
            fm_re[c] += fre;
            fm_im[c] += fim;
            zm_re[c] += gre;
            zm_im[c] += gim;
        }
    }
    const long double inv = 1.0L / (long double)nfile;
    long double o_re = 0, o_im = 0;
    for (int c = 0; c < 3; c++) {
        const long double a_re = fm_re[c] * inv, a_im = fm_im[c] * inv;
        const long double b_re = zm_re[c] * inv, b_im = zm_im[c] * inv;
        o_re += a_re * b_re - a_im * b_im;
        o_im += a_re * b_im + a_im * b_re;
    }
    const long double s_re = (acc_re * inv - o_re) / (long double)M;
    const long double s_im = (acc_im * inv - o_im) / (long double)M;
    out[0] = (double)s_re;
    out[1] = (double)s_im;
    free(ure);
    free(uim);
}

void oracle_sqt_grid(int N, int nfile, const double *spin_t, const double *spin_0,
                     double *out_re, double *out_im)
{
    const long M = (long)N * N;
    const int K = 3 * nfile;
    const double alpha = 1.0 / (double)nfile;
    double *fint = (double *)malloc((size_t)M * 3 * sizeof(double));
    double *zerot = (double *)malloc((size_t)M * 3 * sizeof(double));
    long double *bins = (long double *)calloc((size_t)M, sizeof(long double));
    replica_mean(N, nfile, spin_t, fint);
    replica_mean(N, nfile, spin_0, zerot);
    /* G[d] = sum over pairs with r_i - r_j = d (mod N) of the connected C_ij */
    for (long i = 0; i < M; i++) {
        const int ri = (int)(i / N), ci = (int)(i % N);
        for (long j = 0; j < M; j++) {
            const int rj = (int)(j / N), cj = (int)(j % N);
            double acc = 0.0;
            for (int k = 0; k < K; k++) {
                const int f = k / 3, c = k % 3;
                acc += spin_t[(long)f * M * 3 + i * 3 + c] * spin_0[(long)f * M * 3 + j * 3 + c];
            }
            const double outer = fint[i * 3] * zerot[j * 3] + fint[i * 3 + 1] * zerot[j * 3 + 1] +
                                 fint[i * 3 + 2] * zerot[j * 3 + 2];
            const int dr = ((ri - rj) % N + N) % N, dc = ((ci - cj) % N + N) % N;
            bins[(long)dr * N + dc] += (long double)(alpha * acc - outer);
        }
    }
    const long double two_pi = 2.0L * 3.14159265358979323846264338327950288L;
    for (int a = 0; a < N; a++)
        for (int b = 0; b < N; b++) {
            long double re = 0, im = 0;
            for (int dr = 0; dr < N; dr++)
                for (int dc = 0; dc < N; dc++) {
                    const long double th = two_pi * ((long double)((a * dr) % N) / N +
                                                     (long double)((b * dc) % N) / N);
                    const long double g = bins[(long)dr * N + dc];
                    re += g * cosl(th);
                    im -= g * sinl(th);
                }
            out_re[a * N + b] = (double)(re / (long double)M);
            out_im[a * N + b] = (double)(im / (long double)M);
        }
    free(fint);
    free(zerot);
    free(bins);
}

/* ------------------------------------------------- FP32 RK4 (batched lattices)
 * The arithmetic of the batched-lattice GPU path: the same operations as
 * oracle_llg_deriv / oracle_rk4 (euler / runge_kutta, llg_sqt_baseline.c:29-142)
 * in FP32, each rounded as written (x86-64 SSE float arithmetic with
 * -ffp-contract=off); the renormalisation in FP64 and rounded to FP32 at the
 * end.  One replica; spins float[N*N][3]. */
static void deriv_f32(const oracle_params *p, const float *s, float *d)
{
    const int N = p->N;
    const long M = (long)N * N;
    const float J1 = (float)p->J1, J2 = (float)p->J2, al = (float)p->alpha;
    const float hx = (float)p->hx, hy = (float)p->hy, hz = (float)p->hz;
    const float g = (float)(1.0 / (1.0 + (double)al * (double)al));
    const int use_j2 = p->J2 != 0.0, use_h = (p->hx != 0.0 || p->hy != 0.0 || p->hz != 0.0);
    const int use_damp = p->alpha != 0.0;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < M; i++) {
        const int row = (int)(i / N), col = (int)(i % N);
        const float sx = s[i * 3], sy = s[i * 3 + 1], sz = s[i * 3 + 2];
        float ex = 0.0f, ey = 0.0f, ez = 0.0f;
        for (int j = 0; j < 4; j++) {
            const long nb = (long)((row + kNN[j][0] + N) % N) * N + (col + kNN[j][1] + N) % N;
            ex += s[nb * 3] * J1;
            ey += s[nb * 3 + 1] * J1;
            ez += s[nb * 3 + 2] * J1;
        }
        if (use_j2)
            for (int j = 0; j < 4; j++) {
                const long nb = (long)((row + kNNN[j][0] + N) % N) * N + (col + kNNN[j][1] + N) % N;
                ex += s[nb * 3] * J2;
                ey += s[nb * 3 + 1] * J2;
                ez += s[nb * 3 + 2] * J2;
            }
        if (use_h) {
            ex += hx;
            ey += hy;
            ez += hz;
        }
        const float tx = ey * sz - ez * sy, ty = ez * sx - ex * sz, tz = ex * sy - ey * sx;
        if (use_damp) {
            const float ux = sy * tz - sz * ty, uy = sz * tx - sx * tz, uz = sx * ty - sy * tx;
            d[i * 3] = g * (tx + al * ux);
            d[i * 3 + 1] = g * (ty + al * uy);
            d[i * 3 + 2] = g * (tz + al * uz);
        } else {
            d[i * 3] = tx;
            d[i * 3 + 1] = ty;
            d[i * 3 + 2] = tz;
        }
    }
}

int oracle_steps_f32(const oracle_params *p, float *spin, int nsteps)
{
    const long n = (long)p->N * p->N * 3;
    float *buf = (float *)malloc((size_t)4 * n * sizeof(float));
    if (!buf) return -1;
    float *ys = buf, *acc = buf + n, *d = buf + 2 * n, *ys2 = buf + 3 * n;
    const float dt = (float)p->dt;
    for (int step = 0; step < nsteps; step++) {
        /* stage 1 */
        deriv_f32(p, spin, d);
        for (long j = 0; j < n; j++) {
            const float k = d[j] * dt;
            ys[j] = spin[j] + k * 0.5f;
            acc[j] = spin[j] + k / 6.0f;
        }
        /* stages 2, 3 */
        deriv_f32(p, ys, d);
        for (long j = 0; j < n; j++) {
            const float k = d[j] * dt;
            ys2[j] = spin[j] + k * 0.5f;
            acc[j] = acc[j] + k / 3.0f;
        }
        deriv_f32(p, ys2, d);
        for (long j = 0; j < n; j++) {
            const float k = d[j] * dt;
            ys[j] = spin[j] + k;
            acc[j] = acc[j] + k / 3.0f;
        }
        /* stage 4 + FP64 renormalisation */
        deriv_f32(p, ys, d);
        for (long j = 0; j < n / 3; j++) {
            double o[3];
            for (int c = 0; c < 3; c++) o[c] = (double)(acc[j * 3 + c] + (d[j * 3 + c] * dt) / 6.0f);
            const double nrm = sqrt(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
            for (int c = 0; c < 3; c++) spin[j * 3 + c] = (float)(p->spin_len * o[c] / nrm);
        }
    }
    free(buf);
    return 0;
}
