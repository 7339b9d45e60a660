/*
 * dropin_host.c -- a C program written like the reference's kernel-fusion
 * driver (kernel_fusion/llg_sqt_fusion.c:149-477): the reference's globals,
 * its per-step sequence runge_kutta -> renormalisation -> A pack -> fint_avg
 * -> C = -(outer) q -> fused_dgemm -> sum of the per-thread slots / N^2, but
 * WITHOUT its own euler, runge_kutta and fused_dgemm: those come from
 * libasd_b200.so, which reads N, Nfile, J1 and dt below through weak
 * references (no asd_set_params call).  Test program for the drop-in ABI.
 *
 *   dropin_host in.spins out.spins steps dt J1
 */
#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "asd_b200.h"

int N = 100;
int num_neighbor = 4;
double J1 = 1.0;
int MCsweep = 500;
double dt = 0.02;
int Nfile = 50;
int vx = 5, vy = 5;
int nn[4][2];
int trd = 1;

int main(int argc, char *argv[]) {
    if (argc != 6) {
        fprintf(stderr, "usage: %s in.spins out.spins steps dt J1\n", argv[0]);
        return 2;
    }
    long st0;
    double slen;
    if (asd_spins_load(argv[1], &N, &Nfile, &st0, &slen, NULL, 0) != ASD_OK) {
        fprintf(stderr, "%s\n", asd_last_error());
        return 1;
    }
    const int steps = atoi(argv[3]);
    dt = atof(argv[4]);
    J1 = atof(argv[5]);
    vx = N / 10;
    vy = N / 10;
    nn[0][0] = 1, nn[0][1] = 0;
    nn[1][0] = -1, nn[1][1] = 0;
    nn[2][0] = 0, nn[2][1] = -1;
    nn[3][0] = 0, nn[3][1] = 1;
    const long M = (long)N * N;
    const int K = 3 * Nfile;
    const size_t n = (size_t)Nfile * M * 3;
    double *spin_all = malloc(n * sizeof(double));
    double *cur = malloc(n * sizeof(double)), *k1 = malloc(n * sizeof(double));
    double *k2 = malloc(n * sizeof(double)), *k3 = malloc(n * sizeof(double));
    double *k4 = malloc(n * sizeof(double));
    double *spin_zero = malloc(n * sizeof(double)), *spint = malloc(n * sizeof(double));
    double *zerot = malloc(M * 3 * sizeof(double)), *fint = malloc(M * 3 * sizeof(double));
    double *qmat = malloc((size_t)2 * M * M * sizeof(double));
    double *cmat = malloc((size_t)2 * M * M * sizeof(double));
    if (asd_spins_load(argv[1], &N, &Nfile, &st0, &slen, spin_all, n) != ASD_OK) {
        fprintf(stderr, "%s\n", asd_last_error());
        return 1;
    }
    for (long i = 0; i < M; i++)
        for (int j = 0; j < Nfile; j++)
            for (int c = 0; c < 3; c++) spin_zero[i * K + j * 3 + c] = spin_all[j * M * 3 + i * 3 + c];
    for (long i = 0; i < M; i++) {
        double t[3] = {0, 0, 0};
        for (int j = 0; j < Nfile; j++)
            for (int c = 0; c < 3; c++) t[c] += spin_zero[i * K + j * 3 + c];
        for (int c = 0; c < 3; c++) zerot[i * 3 + c] = t[c] / (double)Nfile;
    }
    const double qx = 2.0 * M_PI * vx / (double)N, qy = 2.0 * M_PI * vy / (double)N;
    for (long j = 0; j < M; j++)
        for (long i = 0; i < M; i++) {
            const double dffr = (double)(i / N - j / N), dffc = (double)(i % N - j % N);
            const double complex q = cexp(CMPLX(0.0, -1.0) * (qx * dffr + qy * dffc));
            const long re = (i / 4) * 8 + (i % 4) + j * 2 * M;
            qmat[re] = creal(q);
            qmat[re + 4] = cimag(q);
        }
    for (int num = 0; num < steps; num++) {
        runge_kutta(spin_all, cur, k1, k2, k3, k4);
        for (long j = 0; j < (long)Nfile * M; j++) {
            double tx = cur[j * 3], ty = cur[j * 3 + 1], tz = cur[j * 3 + 2];
            double nrm = sqrt(tx * tx + ty * ty + tz * tz);
            spin_all[j * 3] = tx / nrm, spin_all[j * 3 + 1] = ty / nrm, spin_all[j * 3 + 2] = tz / nrm;
        }
        for (long j = 0; j < M; j++)
            for (int i = 0; i < Nfile; i++)
                for (int c = 0; c < 3; c++) spint[j + (i * 3 + c) * M] = spin_all[i * M * 3 + j * 3 + c];
        for (long i = 0; i < M; i++) {
            double t[3] = {0, 0, 0};
            for (int id = 0; id < Nfile; id++)
                for (int c = 0; c < 3; c++) t[c] += spin_all[id * M * 3 + i * 3 + c];
            for (int c = 0; c < 3; c++) fint[i * 3 + c] = t[c] / (double)Nfile;
        }
        for (long j = 0; j < M; j++)
            for (long i = 0; i < M; i++) {
                double tmp = zerot[j * 3] * fint[i * 3] + zerot[j * 3 + 1] * fint[i * 3 + 1] +
                             zerot[j * 3 + 2] * fint[i * 3 + 2];
                tmp *= -1.0;
                const long re = (i / 4) * 8 + (i % 4) + j * 2 * M;
                cmat[re] = tmp * qmat[re];
                cmat[re + 4] = tmp * qmat[re + 4];
            }
        double sum[128 * 2];
        memset(sum, 0, sizeof sum);
        int mm = (int)M, ncol = (int)M, kk = K, lda = (int)M, ldb = K, ldc = (int)(2 * M);
        double alpha = 1.0 / (double)Nfile;
        fused_dgemm(&mm, &ncol, &kk, &alpha, spint, &lda, spin_zero, &ldb, cmat, &ldc, qmat, sum);
        double complex res = 0.0;
        for (int i = 0; i < 128; i++) res += CMPLX(sum[2 * i], sum[2 * i + 1]);
        res /= (double)(N * N);
        printf("sqt %d %.17g %.17g\n", num, creal(res), cimag(res));
    }
    if (asd_spins_save(argv[2], N, Nfile, steps, 1.0, spin_all) != ASD_OK) {
        fprintf(stderr, "%s\n", asd_last_error());
        return 1;
    }
    return 0;
}
