// dropin.cu -- the reference's own entry points, with its names, signatures
// and semantics, computed on the GPU:
//   euler        baseline/llg_sqt_baseline.c:29
//   runge_kutta  baseline/llg_sqt_baseline.c:95
//   fused_dgemm  kernel_fusion/gemm_kernel.h:355
// and the BLAS product of the reference's plain path, cblas_dgemm
// (gemm/llg_sqt_mkl.c:378), as asd_cblas_dgemm (exported under the BLAS name
// by the separate libasd_cblas.so, csrc/cblas_shim.c).
// They take host pointers and return when the results are back in host
// memory, like the originals.  Device buffers are cached between calls on the
// current device and grow on demand.  The functions return void, as in the
// reference; a failure is reported on stderr and through asd_last_error(),
// and leaves the outputs unchanged.
#include <cstdio>
#include <mutex>
#include <utility>

#include "asd_internal.h"
#include "fp64_gemm.h"

// The reference's globals (llg_sqt_baseline.c:12-19), defined by the host
// program that links this library.  Weak: absent in other processes.
extern "C" {
extern int N __attribute__((weak));
extern int Nfile __attribute__((weak));
extern double J1 __attribute__((weak));
extern double dt __attribute__((weak));
}

namespace asd {
namespace {

struct DropinParams {
    int N = 100, Nfile = 50;
    double J1 = 1.0, dt = 0.02;
    bool set = false;
};

std::mutex g_mu;
DropinParams g_par;

struct Buffers {
    int device = -1;
    size_t cap = 0;  // doubles per array
    double *arr[6] = {};
    size_t gemm_cap[4] = {};
    double *g[4] = {};  // a, b, c, q
    double2 *part = nullptr;
    size_t part_cap = 0;
    size_t blas_cap[4] = {};
    double *blas[4] = {};  // A [m][k], B [n][k], C [n][m], transpose staging
};
Buffers g_buf;

DropinParams current_params() {
    DropinParams p = g_par;
    if (!p.set && &N && &Nfile && &J1 && &dt) {
        p.N = N;
        p.Nfile = Nfile;
        p.J1 = J1;
        p.dt = dt;
    }
    return p;
}

void report(const char *fn) {
    fprintf(stderr, "libasd_b200 %s: %s\n", fn, asd_last_error());
}

// The cached buffers belong to one device.  A call on another device frees
// them there (with that device current, as cudaFree wants) and starts over.
int use_current_device() {
    int dev = 0;
    ASD_CUDA_TRY(cudaGetDevice(&dev));
    if (g_buf.device == dev) return ASD_OK;
    if (g_buf.device >= 0 && cudaSetDevice(g_buf.device) == cudaSuccess) {
        for (double *q : g_buf.arr)
            if (q) cudaFree(q);
        for (double *q : g_buf.g)
            if (q) cudaFree(q);
        for (double *q : g_buf.blas)
            if (q) cudaFree(q);
        if (g_buf.part) cudaFree(g_buf.part);
    }
    cudaGetLastError();
    ASD_CUDA_TRY(cudaSetDevice(dev));
    g_buf = Buffers();
    g_buf.device = dev;
    return ASD_OK;
}

int reserve(double **p, size_t *cap, size_t n) {
    if (n <= *cap && *p) return ASD_OK;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(double));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ASD_ERR_NOMEM, "cudaMalloc(%zu doubles): %s", n, cudaGetErrorString(e));
    }
    *cap = n;
    return ASD_OK;
}

int prepare(int ndouble_arrays, size_t n) {
    int rc0 = use_current_device();
    if (rc0 != ASD_OK) return rc0;
    if (n > g_buf.cap) {
        for (int i = 0; i < 6; ++i) {
            if (g_buf.arr[i]) cudaFree(g_buf.arr[i]);
            g_buf.arr[i] = nullptr;
        }
        g_buf.cap = 0;
        for (int i = 0; i < 6; ++i) {
            cudaError_t e = cudaMalloc((void **)&g_buf.arr[i], n * sizeof(double));
            if (e != cudaSuccess) {
                cudaGetLastError();
                return fail(ASD_ERR_NOMEM, "cudaMalloc: %s", cudaGetErrorString(e));
            }
        }
        g_buf.cap = n;
    }
    (void)ndouble_arrays;
    return ASD_OK;
}

LLGArgs ref_args(const DropinParams &p) {
    asd_params q;
    asd_params_default(&q, p.N, p.Nfile);
    q.J1 = p.J1;
    q.dt = p.dt;
    return make_llg_args(q);
}

int check(const DropinParams &p) {
    if (p.N < 1 || p.Nfile < 1) return fail(ASD_ERR_INVALID, "N=%d Nfile=%d", p.N, p.Nfile);
    return ASD_OK;
}

int do_euler(double *spin0, double *deriv) {
    const DropinParams p = current_params();
    int rc = check(p);
    if (rc != ASD_OK) return rc;
    const size_t n = (size_t)p.Nfile * p.N * p.N * 3;
    if ((rc = prepare(2, n)) != ASD_OK) return rc;
    double *ds = g_buf.arr[0], *dd = g_buf.arr[1];
    ASD_CUDA_TRY(cudaMemcpy(ds, spin0, n * sizeof(double), cudaMemcpyHostToDevice));
    ASD_CUDA_TRY(launch_euler_aos(ref_args(p), ds, dd, 0));
    ASD_CUDA_TRY(cudaMemcpy(deriv, dd, n * sizeof(double), cudaMemcpyDeviceToHost));
    return ASD_OK;
}

int do_rk(double *spin, double *cur, double *k1, double *k2, double *k3, double *k4) {
    const DropinParams p = current_params();
    int rc = check(p);
    if (rc != ASD_OK) return rc;
    const size_t n = (size_t)p.Nfile * p.N * p.N * 3;
    if ((rc = prepare(6, n)) != ASD_OK) return rc;
    double *ds = g_buf.arr[0], *dc = g_buf.arr[1];
    double *dk[4] = {g_buf.arr[2], g_buf.arr[3], g_buf.arr[4], g_buf.arr[5]};
    const LLGArgs a = ref_args(p);
    ASD_CUDA_TRY(cudaMemcpy(ds, spin, n * sizeof(double), cudaMemcpyHostToDevice));
    ASD_CUDA_TRY(cudaMemcpyAsync(dc, ds, n * sizeof(double), cudaMemcpyDeviceToDevice, 0));
    for (int s = 0; s < 4; ++s) {
        ASD_CUDA_TRY(launch_euler_aos(a, dc, dk[s], 0));
        ASD_CUDA_TRY(launch_rk_pass(s + 1, (long)n, p.dt, ds, dc, dk[s], dk[0], dk[1], dk[2], 0));
    }
    ASD_CUDA_TRY(cudaMemcpy(cur, dc, n * sizeof(double), cudaMemcpyDeviceToHost));
    double *outs[4] = {k1, k2, k3, k4};
    for (int s = 0; s < 4; ++s)
        ASD_CUDA_TRY(cudaMemcpy(outs[s], dk[s], n * sizeof(double), cudaMemcpyDeviceToHost));
    return ASD_OK;
}

int do_fused_dgemm(int m, int n, int k, double alpha, const double *a, int lda, const double *b,
                   int ldb, double *c, int ldc, const double *q, double *sum) {
    if (m < 0 || n < 0 || k < 0) return fail(ASD_ERR_INVALID, "negative dimension");
    if (m == 0 || n == 0 || k == 0) return ASD_OK;  // the reference does nothing either
    if (lda < m || ldb < k || ldc < 2 * ((m + 3) / 4) * 4)
        return fail(ASD_ERR_INVALID, "leading dimension too small (lda=%d ldb=%d ldc=%d)", lda,
                    ldb, ldc);
    if (int rc0 = use_current_device()) return rc0;
    const size_t na = (size_t)lda * k, nb = (size_t)ldb * n, nc = (size_t)ldc * n;
    int rc;
    if ((rc = reserve(&g_buf.g[0], &g_buf.gemm_cap[0], na)) != ASD_OK) return rc;
    if ((rc = reserve(&g_buf.g[1], &g_buf.gemm_cap[1], nb)) != ASD_OK) return rc;
    if ((rc = reserve(&g_buf.g[2], &g_buf.gemm_cap[2], nc)) != ASD_OK) return rc;
    if ((rc = reserve(&g_buf.g[3], &g_buf.gemm_cap[3], nc)) != ASD_OK) return rc;
    ASD_CUDA_TRY(cudaMemcpy(g_buf.g[0], a, na * sizeof(double), cudaMemcpyHostToDevice));
    ASD_CUDA_TRY(cudaMemcpy(g_buf.g[1], b, nb * sizeof(double), cudaMemcpyHostToDevice));
    ASD_CUDA_TRY(cudaMemcpy(g_buf.g[2], c, nc * sizeof(double), cudaMemcpyHostToDevice));
    ASD_CUDA_TRY(cudaMemcpy(g_buf.g[3], q, nc * sizeof(double), cudaMemcpyHostToDevice));
    Fp64GemmArgs g{};
    g.m = m;
    g.n = n;
    g.k = k;
    g.a = g_buf.g[0];
    g.sai = 1;
    g.sak = lda;
    g.a_k_fast = 0;
    g.b = g_buf.g[1];
    g.sbk = 1;
    g.sbj = ldb;
    g.b_k_fast = 1;
    g.alpha = alpha;
    g.c = g_buf.g[2];
    g.q = g_buf.g[3];
    g.ldc = ldc;
    g.m4 = m - m % 4;
    g.n2 = n - n % 2;
    const long np = fp64_gemm_num_parts(g);
    if ((size_t)np > g_buf.part_cap) {
        if (g_buf.part) cudaFree(g_buf.part);
        g_buf.part = nullptr;
        g_buf.part_cap = 0;
        cudaError_t e = cudaMalloc((void **)&g_buf.part, (size_t)np * sizeof(double2));
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(ASD_ERR_NOMEM, "cudaMalloc partials: %s", cudaGetErrorString(e));
        }
        g_buf.part_cap = (size_t)np;
    }
    g.part = g_buf.part;
    ASD_CUDA_TRY(launch_fp64_gemm(g, 0));
    double *d_sum = nullptr;
    ASD_CUDA_TRY(cudaMalloc((void **)&d_sum, 2 * sizeof(double)));
    cudaError_t e = launch_finalize(g_buf.part, (int)np, 1.0, d_sum, 0);
    double hs[2] = {0.0, 0.0};
    if (e == cudaSuccess) e = cudaMemcpy(hs, d_sum, sizeof hs, cudaMemcpyDeviceToHost);
    cudaFree(d_sum);
    if (e != cudaSuccess) return cuda_fail(e, "fused_dgemm finalize");
    ASD_CUDA_TRY(cudaMemcpy(c, g_buf.g[2], nc * sizeof(double), cudaMemcpyDeviceToHost));
    // The reference accumulates into per-thread slots sum[2*ithr..]; every
    // caller adds all slots (llg_sqt_fusion.c:432-438), so slot 0 carries the total.
    sum[0] += hs[0];
    sum[1] += hs[1];
    return ASD_OK;
}

// cblas_dgemm with the CBLAS constants (CblasRowMajor 101, CblasColMajor 102,
// CblasNoTrans 111, CblasTrans 112, CblasConjTrans 113 = CblasTrans for real
// data) and the BLAS argument rules.  A row-major product is the column-major
// product of the transposes with the operands swapped.  Column-major
// C (m x n) = alpha op(A) op(B) + beta C runs on the FP64 tensor-core GEMM
// with K-contiguous operands [m][k] and [n][k]: op(A) with transa = T and
// op(B) with transb = N are already K-contiguous in host memory (strided
// copies), the other two are uploaded as they lie and transposed on the
// device.  C is read only when beta != 0, as BLAS specifies.
int do_cblas_dgemm(int order, int transa, int transb, int m, int n, int k, double alpha,
                   const double *a, int lda, const double *b, int ldb, double beta, double *c,
                   int ldc) {
    auto is_trans = [](int t) { return t == 112 || t == 113; };
    if (order != 101 && order != 102) return fail(ASD_ERR_INVALID, "order %d (parameter 1)", order);
    if (transa != 111 && !is_trans(transa))
        return fail(ASD_ERR_INVALID, "transa %d (parameter 2)", transa);
    if (transb != 111 && !is_trans(transb))
        return fail(ASD_ERR_INVALID, "transb %d (parameter 3)", transb);
    if (m < 0 || n < 0 || k < 0) return fail(ASD_ERR_INVALID, "negative dimension");
    if (order == 101) {  // row major: C^T = op(B)^T op(A)^T in column-major terms
        std::swap(transa, transb);
        std::swap(m, n);
        std::swap(a, b);
        std::swap(lda, ldb);
    }
    const bool ta = is_trans(transa), tb = is_trans(transb);
    const int arows = ta ? k : m, brows = tb ? n : k;
    if (lda < (arows > 1 ? arows : 1) || ldb < (brows > 1 ? brows : 1) || ldc < (m > 1 ? m : 1))
        return fail(ASD_ERR_INVALID, "leading dimension too small (lda=%d ldb=%d ldc=%d)", lda, ldb,
                    ldc);
    if (m == 0 || n == 0) return ASD_OK;
    const bool product = (k > 0 && alpha != 0.0);
    if (!product && beta == 1.0) return ASD_OK;
    if (!c || (product && (!a || !b))) return fail(ASD_ERR_INVALID, "NULL matrix");
    if (int rc0 = use_current_device()) return rc0;
    const size_t mk = (size_t)m * k, nk = (size_t)n * k, mn = (size_t)m * n;
    int rc;
    if ((rc = reserve(&g_buf.blas[2], &g_buf.blas_cap[2], mn)) != ASD_OK) return rc;
    double *dC = g_buf.blas[2];  // column-major m x n, leading dimension m
    const size_t D = sizeof(double);
    if (beta != 0.0)
        ASD_CUDA_TRY(cudaMemcpy2D(dC, m * D, c, (size_t)ldc * D, m * D, n, cudaMemcpyHostToDevice));
    if (!product) {
        ASD_CUDA_TRY(launch_scale_f64(dC, m, n, m, beta, 0));
    } else {
        if ((rc = reserve(&g_buf.blas[0], &g_buf.blas_cap[0], mk)) != ASD_OK) return rc;
        if ((rc = reserve(&g_buf.blas[1], &g_buf.blas_cap[1], nk)) != ASD_OK) return rc;
        if ((!ta || tb) &&
            (rc = reserve(&g_buf.blas[3], &g_buf.blas_cap[3], mk > nk ? mk : nk)) != ASD_OK)
            return rc;
        double *dA = g_buf.blas[0], *dB = g_buf.blas[1], *tmp = g_buf.blas[3];
        if (ta) {  // op(A)(i, l) = a[l + i lda]: m rows of k
            ASD_CUDA_TRY(cudaMemcpy2D(dA, k * D, a, (size_t)lda * D, k * D, m, cudaMemcpyHostToDevice));
        } else {  // A(i, l) = a[i + l lda]: k columns of m, transposed on the device
            ASD_CUDA_TRY(cudaMemcpy2D(tmp, m * D, a, (size_t)lda * D, m * D, k, cudaMemcpyHostToDevice));
            ASD_CUDA_TRY(launch_transpose_f64(tmp, k, m, dA, 0));
        }
        if (!tb) {  // op(B)(l, j) = b[l + j ldb]: n rows of k
            ASD_CUDA_TRY(cudaMemcpy2D(dB, k * D, b, (size_t)ldb * D, k * D, n, cudaMemcpyHostToDevice));
        } else {  // op(B)(l, j) = b[j + l ldb]: k rows of n, transposed on the device
            ASD_CUDA_TRY(cudaMemcpy2D(tmp, n * D, b, (size_t)ldb * D, n * D, k, cudaMemcpyHostToDevice));
            ASD_CUDA_TRY(launch_transpose_f64(tmp, k, n, dB, 0));
        }
        DmmaSqtArgs g{};
        g.A = dA;
        g.B = dB;
        g.M = m;
        g.MB = n;
        g.K = k;
        g.alpha = alpha;
        g.C = dC;
        g.ldc = m;
        g.beta = beta;
        if ((rc = launch_dmma_sqt(g, 0)) != ASD_OK) return rc;
    }
    ASD_CUDA_TRY(cudaMemcpy2D(c, (size_t)ldc * D, dC, m * D, m * D, n, cudaMemcpyDeviceToHost));
    return ASD_OK;
}

}  // namespace
}  // namespace asd

using namespace asd;

extern "C" {

int asd_set_params(int n_, int nfile_, double j1_, double dt_) {
    if (n_ < 1 || nfile_ < 1) return fail(ASD_ERR_INVALID, "N=%d Nfile=%d", n_, nfile_);
    std::lock_guard<std::mutex> lk(g_mu);
    g_par.N = n_;
    g_par.Nfile = nfile_;
    g_par.J1 = j1_;
    g_par.dt = dt_;
    g_par.set = true;
    return ASD_OK;
}

void euler(double *spin0, double *derivative) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (do_euler(spin0, derivative) != ASD_OK) report("euler");
}

void runge_kutta(double *spin, double *cur_input, double *k1, double *k2, double *k3, double *k4) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (do_rk(spin, cur_input, k1, k2, k3, k4) != ASD_OK) report("runge_kutta");
}

int asd_cblas_dgemm(int order, int transa, int transb, int m, int n, int k, double alpha,
                    const double *a, int lda, const double *b, int ldb, double beta, double *c,
                    int ldc) {
    std::lock_guard<std::mutex> lk(g_mu);
    return do_cblas_dgemm(order, transa, transb, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc);
}

void fused_dgemm(int *m, int *n, int *k, double *alpha, double *a, int *lda, double *b, int *ldb,
                 double *c, int *ldc, double *fuse_C, double *sum) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!m || !n || !k || !alpha || !lda || !ldb || !ldc) {
        fail(ASD_ERR_INVALID, "NULL scalar argument");
        report("fused_dgemm");
        return;
    }
    if (do_fused_dgemm(*m, *n, *k, *alpha, a, *lda, b, *ldb, c, *ldc, fuse_C, sum) != ASD_OK)
        report("fused_dgemm");
}

}  // extern "C"
