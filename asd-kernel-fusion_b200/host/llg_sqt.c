/*
 * llg_sqt.c -- the reference's driver program, on the GPU.
 *
 * Same flags and the same per-step protocol as the reference's main()
 * (baseline/llg_sqt_baseline.c:146-452, kernel_fusion/llg_sqt_fusion.c:149-477):
 * -n N, -f Nfile, -e dt, -m steps (the reference's loop is hard-wired to 60),
 * -t threads (accepted and ignored, as in the reference), -x/-y the q indices
 * (the reference overwrites them with N/10; here N/10 is only the default).
 * Each step runs RK4 + renormalisation and one S(q,t) evaluation; steps from
 * the warm-up count on are timed and "N tlle tsqt" (mean seconds per step) is
 * appended to the timing file, like the reference's amd_gcc_11.2_*_sqt.txt.
 *
 * Extensions: -J J1, -K J2, -a alpha, -H hx,hy,hz, -S spin length, -s seed,
 * -q fp64|tf32x3|bf16x3|fp16x3, -i/-o spin files (asd_spins_load/save
 * format), -w warm-up steps (default 20), -r timing file, -p print S(q,t)
 * every step, -g print S(q,t) on the whole q grid at the end (N*N <= 4096).
 *
 * Initial spins (without -i) are seeded and uniform on the sphere
 * (SplitMix64); the reference's own initialisation yields NaN
 * (llg_sqt_baseline.c:196-206).
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "asd_b200.h"

static double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static uint64_t splitmix64(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static double unit(uint64_t *s) { return (splitmix64(s) >> 11) * 0x1.0p-53; }

static void usage(const char *prog) {
    fprintf(stderr,
            "usage: %s [-n N] [-m steps] [-f Nfile] [-e dt] [-t threads] [-x vx] [-y vy]\n"
            "          [-J J1] [-K J2] [-a alpha] [-H hx,hy,hz] [-S spin_len] [-s seed]\n"
            "          [-q fp64|tf32x3|bf16x3|fp16x3] [-i in.spins] [-o out.spins]\n"
            "          [-w warmup] [-r timing_file] [-p] [-g]\n",
            prog);
}

static int parse_mode(const char *s, asd_sqt_mode *m) {
    if (!strcmp(s, "fp64")) *m = ASD_SQT_FP64;
    else if (!strcmp(s, "tf32x3")) *m = ASD_SQT_TF32X3;
    else if (!strcmp(s, "bf16x3")) *m = ASD_SQT_BF16X3;
    else if (!strcmp(s, "fp16x3")) *m = ASD_SQT_FP16X3;
    else return -1;
    return 0;
}

int main(int argc, char *argv[]) {
    int N = 100, Nfile = 50, steps = 60, warm = 20, vx = -1, vy = -1, print_each = 0, grid = 0;
    double dt = 0.02, J1 = 1.0, J2 = 0.0, alpha = 0.0, hx = 0.0, hy = 0.0, hz = 0.0, slen = 1.0;
    uint64_t seed = 0;
    asd_sqt_mode mode = ASD_SQT_FP64;
    const char *in = NULL, *out = NULL, *timing = "b200_sqt.txt";
    int ch;
    while ((ch = getopt(argc, argv, "n:m:f:e:t:x:y:J:K:a:H:S:s:q:i:o:w:r:pg")) != -1) {
        switch (ch) {
            case 'n': N = atoi(optarg); break;
            case 'm': steps = atoi(optarg); break;
            case 'f': Nfile = atoi(optarg); break;
            case 'e': dt = atof(optarg); break;
            case 't': break; /* parsed and unused, as in the reference */
            case 'x': vx = atoi(optarg); break;
            case 'y': vy = atoi(optarg); break;
            case 'J': J1 = atof(optarg); break;
            case 'K': J2 = atof(optarg); break;
            case 'a': alpha = atof(optarg); break;
            case 'H':
                if (sscanf(optarg, "%lf,%lf,%lf", &hx, &hy, &hz) != 3) {
                    usage(argv[0]);
                    return 2;
                }
                break;
            case 'S': slen = atof(optarg); break;
            case 's': seed = strtoull(optarg, NULL, 10); break;
            case 'q':
                if (parse_mode(optarg, &mode)) {
                    usage(argv[0]);
                    return 2;
                }
                break;
            case 'i': in = optarg; break;
            case 'o': out = optarg; break;
            case 'w': warm = atoi(optarg); break;
            case 'r': timing = optarg; break;
            case 'p': print_each = 1; break;
            case 'g': grid = 1; break;
            default: usage(argv[0]); return 2;
        }
    }
    if (steps < 0 || warm < 0) {
        usage(argv[0]);
        return 2;
    }

    double *spin = NULL;
    if (in) {
        int fn, ff;
        long st;
        double sl;
        if (asd_spins_load(in, &fn, &ff, &st, &sl, NULL, 0) != ASD_OK) {
            fprintf(stderr, "llg_sqt: %s\n", asd_last_error());
            return 1;
        }
        N = fn;
        Nfile = ff;
        size_t n = (size_t)ff * fn * fn * 3;
        spin = (double *)malloc(n * sizeof(double));
        if (!spin || asd_spins_load(in, &fn, &ff, &st, &sl, spin, n) != ASD_OK) {
            fprintf(stderr, "llg_sqt: %s\n", spin ? asd_last_error() : "out of memory");
            return 1;
        }
    }

    asd_params p;
    if (asd_params_default(&p, N, Nfile) != ASD_OK) {
        fprintf(stderr, "llg_sqt: %s\n", asd_last_error());
        return 2;
    }
    p.J1 = J1, p.J2 = J2, p.alpha = alpha, p.hx = hx, p.hy = hy, p.hz = hz;
    p.dt = dt, p.spin_len = slen;
    if (vx >= 0) p.vx = vx;
    if (vy >= 0) p.vy = vy;

    if (!spin) {
        size_t n = (size_t)Nfile * N * N;
        spin = (double *)malloc(n * 3 * sizeof(double));
        if (!spin) {
            fprintf(stderr, "llg_sqt: out of memory\n");
            return 1;
        }
        uint64_t s = seed;
        for (size_t j = 0; j < n; ++j) {
            const double z = 2.0 * unit(&s) - 1.0, phi = 2.0 * M_PI * unit(&s);
            const double r = sqrt(1.0 - z * z);
            spin[3 * j] = slen * r * cos(phi);
            spin[3 * j + 1] = slen * r * sin(phi);
            spin[3 * j + 2] = slen * z;
        }
    }
    printf("N: %d, Nfile: %d, steps: %d, S(q,t) mode: %d, q = 2pi(%d,%d)/N\n", N, Nfile, steps,
           (int)mode, p.vx, p.vy);

    asd_ctx *ctx = NULL;
    if (asd_ctx_create(&p, 0, &ctx) != ASD_OK || asd_ctx_set_spins(ctx, spin, 1) != ASD_OK) {
        fprintf(stderr, "llg_sqt: %s\n", asd_last_error());
        if (ctx) asd_ctx_destroy(ctx);
        return 1;
    }
    double tlle = 0.0, tsqt = 0.0;
    int timed = 0, failed = 0;
    for (int num = 0; num < steps; ++num) {
        if (num % 5 == 0) printf("Step: %d\n", num);
        double t1 = now_s();
        if (asd_ctx_step(ctx, 1) != ASD_OK || asd_ctx_check_device_status(ctx) != ASD_OK) {
            failed = 1;
            break;
        }
        double t2 = now_s();
        double s[2];
        if (asd_ctx_sqt(ctx, mode, s) != ASD_OK) {
            failed = 1;
            break;
        }
        double t3 = now_s();
        if (num >= warm) {
            tlle += t2 - t1;
            tsqt += t3 - t2;
            ++timed;
        }
        if (print_each) printf("sqt %d %.17g %.17g\n", num, s[0], s[1]);
    }
    int rc = 0;
    if (failed) {
        fprintf(stderr, "llg_sqt: %s\n", asd_last_error());
        rc = 1;
    }
    if (rc == 0 && grid) {
        double *g = (double *)malloc((size_t)N * N * 2 * sizeof(double));
        if (!g || asd_ctx_sqt_grid(ctx, mode, g) != ASD_OK) {
            fprintf(stderr, "llg_sqt: %s\n", g ? asd_last_error() : "out of memory");
            rc = 1;
        } else {
            for (int a = 0; a < N; ++a)
                for (int b = 0; b < N; ++b)
                    printf("sqt_grid %d %d %.17g %.17g\n", a, b, g[2 * (a * N + b)],
                           g[2 * (a * N + b) + 1]);
        }
        free(g);
    }
    if (rc == 0 && timed > 0) {
        tlle /= timed;
        tsqt /= timed;
        FILE *fp = fopen(timing, "a");
        if (fp) {
            fprintf(fp, "%d %lf %lf\n", N, tlle, tsqt);
            fclose(fp);
        }
        printf("tlle %.6e s/step (%.3e site-steps/s), tsqt %.6e s/step\n", tlle,
               (double)N * N * Nfile / tlle, tsqt);
    }
    if (rc == 0 && out) {
        if (asd_ctx_get_spins(ctx, spin) != ASD_OK ||
            asd_spins_save(out, N, Nfile, steps, slen, spin) != ASD_OK) {
            fprintf(stderr, "llg_sqt: %s\n", asd_last_error());
            rc = 1;
        }
    }
    asd_ctx_destroy(ctx);
    free(spin);
    return rc;
}
