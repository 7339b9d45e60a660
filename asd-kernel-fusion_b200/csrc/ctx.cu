// ctx.cu -- the context API of libasd_b200.so (include/asd_b200.h): device
// state, the per-step schedule and the S(q,t) dispatch.
//
// One context = one lattice with nfile replicas on one device and one CUDA
// stream.  Device memory (site-major FP64 spins, M = N*N sites,
// K = 3*nfile values per site):
//   y, ys_a, ys_b, acc   RK4 state, stage inputs, running combination  4*M*K
//   origin               the t = 0 snapshot (B of the GEMM)               M*K
//   a/b hi/lo            split operands, [Mp][Kp] per enabled split kind
//   q-grid work          per-tile diagonal partials (on the first q grid)
// The AoS <-> site-major transposes stage through ys_b.

#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "asd_internal.h"

namespace asd {

static thread_local char g_err[512] = "";
static thread_local int g_device = 0;

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

int fail(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    snprintf(g_err, sizeof g_err, "%s: %s", what, cudaGetErrorString(e));
    return ASD_ERR_CUDA;
}

int current_device() { return g_device; }

}  // namespace asd

using namespace asd;

struct asd_ctx {
    asd_params p{};
    LLGArgs a{};
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    long M = 0, Mp = 0;
    int K = 0;
    unsigned modes = 0;
    double *y = nullptr, *ys_a = nullptr, *ys_b = nullptr, *acc = nullptr, *origin = nullptr;
    double *mean_t = nullptr, *mean_0 = nullptr;
    double2 *uphase = nullptr, *wphase = nullptr;
    float4 *row4 = nullptr, *col4 = nullptr;
    float *row1 = nullptr, *col1 = nullptr;
    // split operands per kind (index 1 = TF32, 2 = BF16, 3 = FP16), the
    // state / origin version each was split from, and the scale it was split
    // with (FP16: a power of two that follows spin_len)
    void *a_hi[4] = {}, *a_lo[4] = {}, *b_hi[4] = {}, *b_lo[4] = {};
    int Kp[4] = {};
    long a_version[4] = {-1, -1, -1, -1};
    long b_version[4] = {-1, -1, -1, -1};
    double a_scale[4] = {}, b_scale[4] = {};
    double2 *part = nullptr;
    long part_cap = 0;
    double *d_out = nullptr;
    double *h_out = nullptr;  // pinned
    unsigned *status = nullptr;
    long state_version = 0, origin_version = -1;
    bool has_state = false, has_origin = false;
    int last_launches = 0;
    int chunk_k = -1;  // < 0: per mode, 512 for TF32x3, 1024 for BF16x3 and FP16x3
    double *grid_g = nullptr;     // q grid: N*N displacement bins (FP64)
    double2 *grid_t = nullptr;    // q grid: DFT intermediate
    double *grid_out = nullptr;   // q grid: device result for the host-buffer form
    double *grid_tdiag = nullptr; // q grid: per-tile diagonal partials
    size_t grid_tdiag_n = 0;
    double *grid_ds = nullptr;    // q grid: diagonal partials summed by tile key
    size_t grid_ds_n = 0;
    // adjoint work space (allocated on the first asd_ctx_loss_grad)
    std::vector<double *> adj_bufs;
    long adj_states = 0;
    bool adj_keep = false;  // the work space holds every stage state of a segment
    // the tape of the last loss forward pass: its S(q,t) values and sizes,
    // valid while the parameters and the origin stay those it ran with
    bool tape_valid = false;
    bool tape_keep = false;  // the backward pass keeps a segment's stage states
    int tape_nsteps = 0, tape_stride = 0, tape_ckpt = 0;
    long tape_params = -1, tape_origin = -1;
    std::vector<double2> tape_S;
    long params_version = 0;
    // asd_ctx_step_host: copy stream and event for the overlapped read-back
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t spins_ready = nullptr;
    int llg_kernel = ASD_LLG_AUTO;
    // Pipelining of asd_ctx_step behind asd_ctx_sqt_async: once a split-mode
    // S(q,t) has turned y into its GEMM operands, the GEMM reads none of the
    // LLG buffers, so the next RK4 step may run beside it on llg_stream.
    // y_free is recorded on the ctx stream right after the split; armed says
    // that nothing touching y, ys_a, ys_b or acc has been enqueued since.
    // The split-mode GEMM and its finalize run on gemm_stream, created with
    // the greatest priority, so that when the split completes the block
    // scheduler places the persistent GEMM's CTAs before the LLG blocks (the
    // GEMM takes one CTA per SM and leaves room for four 256-thread LLG
    // blocks beside it).  Both side streams are forked from and joined back
    // into the ctx stream with events, so the ctx stream orders everything.
    cudaStream_t llg_stream = nullptr, gemm_stream = nullptr;
    cudaEvent_t y_free = nullptr, llg_done = nullptr, gemm_done = nullptr;
    bool y_free_armed = false;
    // row4.w / row1 (the phase u_i) are written by every site_mean of y;
    // false until the first one and after q changes.
    bool rows_ready = false;
    // asd_ctx_step_host by replica chunk: double-buffered AoS staging for the
    // chunk coming in and the chunk going out, a stream for the uploads
    // (copy_stream carries the downloads) and the events that order them.
    int hp_replicas = 0;  // chunk size the staging was sized for (0: none)
    double *stage_in[2] = {}, *stage_out[2] = {};
    cudaStream_t h2d_stream = nullptr;
    cudaEvent_t in_ready[2] = {}, in_free[2] = {}, out_ready[2] = {}, out_free[2] = {};
    // asd_ctx_step_host_async: whole-state AoS staging in and out (so the
    // copy engines never wait for a staging slot), and per replica chunk the
    // events that order uploads, compute and downloads within a call and
    // across consecutive calls.
    static constexpr int kAsyncChunks = 16;
    double *ast_in = nullptr, *ast_out = nullptr;
    bool ast_events = false;
    cudaEvent_t ast_in_ready[kAsyncChunks] = {}, ast_in_done[kAsyncChunks] = {},
                ast_out_ready[kAsyncChunks] = {}, ast_out_done[kAsyncChunks] = {};
    // Replica sharding: this context holds nfile of the nfile_total replicas
    // of one ensemble (0: not sharded); zsums = the ensemble's origin site
    // sums once exchanged.
    int nfile_total = 0;
    double *zsums = nullptr;
    bool has_zsums = false;
    // asd_ctx_time_kernels: CUDA events recorded on the launching stream
    // around the RK4 step kernels (which = 0) and the S(q,t) GEMM (which = 1),
    // read and recycled by asd_ctx_kernel_time.
    struct Timed {
        int which, launches;
        cudaEvent_t b, e;
    };
    bool timing = false;
    std::vector<Timed> timed;
    std::vector<cudaEvent_t> ev_pool;
};

namespace {

// Host-side allocation-failure injection (asd_debug_fail_alloc): while
// g_fail_in > 0, every device allocation of the context API counts it down,
// and the one that takes it from 1 to 0 fails as cudaMalloc does on a full
// device.  No GPU fault is involved.
std::atomic<long> g_fail_in{0};

bool injected_failure() {
    long n = g_fail_in.load(std::memory_order_relaxed);
    while (n > 0 && !g_fail_in.compare_exchange_weak(n, n - 1, std::memory_order_relaxed)) {
    }
    return n == 1;
}

template <class T>
int dalloc(T **p, size_t bytes) {
    if (injected_failure()) {
        *p = nullptr;
        return fail(ASD_ERR_NOMEM, "cudaMalloc(%zu bytes): injected failure", bytes);
    }
    cudaError_t e = cudaMalloc((void **)p, bytes < 16 ? 16 : bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(ASD_ERR_NOMEM, "cudaMalloc(%zu bytes): %s", bytes, cudaGetErrorString(e));
    }
    return ASD_OK;
}

int check_params(const asd_params *p) {
    if (!p) return fail(ASD_ERR_INVALID, "params is NULL");
    if (p->N < 3 || p->N > 4096) return fail(ASD_ERR_INVALID, "N=%d out of range [3, 4096]", p->N);
    if (p->nfile < 1 || p->nfile > 1000000)
        return fail(ASD_ERR_INVALID, "nfile=%d out of range", p->nfile);
    if (!(p->spin_len > 0.0)) return fail(ASD_ERR_INVALID, "spin_len must be > 0");
    if (!(p->dt == p->dt)) return fail(ASD_ERR_INVALID, "dt is NaN");
    const double lim = 1e300;
    const double v[] = {p->J1, p->J2, p->alpha, p->hx, p->hy, p->hz, p->dt};
    for (double x : v)
        if (!(x > -lim && x < lim)) return fail(ASD_ERR_INVALID, "non-finite parameter");
    const double M = (double)p->N * p->N;
    if (M * 3.0 * p->nfile > 4.0e9) return fail(ASD_ERR_INVALID, "N*N*3*nfile too large");
    return ASD_OK;
}

int ensure_part(asd_ctx *c, long n) {
    if (n <= c->part_cap) return ASD_OK;
    if (c->part) cudaFree(c->part);
    c->part = nullptr;
    c->part_cap = 0;
    int rc = dalloc(&c->part, (size_t)n * sizeof(double2));
    if (rc == ASD_OK) c->part_cap = n;
    return rc;
}

int kp_for(int kind, int K) {
    const int ke = 128 / split_esize(kind);  // K elements per 128-byte k block
    return (K + ke - 1) / ke * ke;
}

// The split kind of an S(q,t) mode (0: the FP64 path).
int mode_kind(int mode) {
    return mode == ASD_SQT_TF32X3 ? 1 : mode == ASD_SQT_BF16X3 ? 2 : mode == ASD_SQT_FP16X3 ? 3 : 0;
}

// K elements per TMEM accumulation chunk: the context's setting, else the
// same number of tensor-core accumulation steps for every kind (TF32 MMAs
// take 8 K elements per step, 16-bit ones 16).
int chunk_for(const asd_ctx *c, int kind) {
    return c->chunk_k >= 0 ? c->chunk_k : (kind == 1 ? 512 : 1024);
}

// Prologue of every entry point that may enqueue work: select the device and
// forget the early y_free point (the caller may touch the LLG buffers next).
cudaError_t enter(asd_ctx *c) {
    c->y_free_armed = false;
    return cudaSetDevice(c->device);
}

bool stream_capturing(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
        cudaGetLastError();
        return true;  // unknown: take the fully ordered path
    }
    return cs != cudaStreamCaptureStatusNone;
}

int ensure_llg_stream(asd_ctx *c) {
    if (c->llg_stream) return ASD_OK;
    int least = 0, greatest = 0;
    ASD_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    ASD_CUDA_TRY(cudaStreamCreateWithPriority(&c->gemm_stream, cudaStreamNonBlocking, greatest));
    ASD_CUDA_TRY(cudaStreamCreateWithPriority(&c->llg_stream, cudaStreamNonBlocking, least));
    ASD_CUDA_TRY(cudaEventCreateWithFlags(&c->y_free, cudaEventDisableTiming));
    ASD_CUDA_TRY(cudaEventCreateWithFlags(&c->llg_done, cudaEventDisableTiming));
    ASD_CUDA_TRY(cudaEventCreateWithFlags(&c->gemm_done, cudaEventDisableTiming));
    return ASD_OK;
}

// Record the point on the ctx stream after which no enqueued work reads or
// writes the LLG buffers (called between the split and the GEMM) and fork
// gemm_stream from it.  Returns the stream the GEMM is to be launched on:
// gemm_stream, or the ctx stream itself while it is being captured.
int arm_y_free(asd_ctx *c, cudaStream_t *gemm) {
    *gemm = c->stream;
    if (stream_capturing(c->stream)) return ASD_OK;
    int rc = ensure_llg_stream(c);
    if (rc != ASD_OK) return rc;
    ASD_CUDA_TRY(cudaEventRecord(c->y_free, c->stream));
    ASD_CUDA_TRY(cudaStreamWaitEvent(c->gemm_stream, c->y_free, 0));
    c->y_free_armed = true;
    *gemm = c->gemm_stream;
    return ASD_OK;
}

// Join gemm_stream back into the ctx stream.
int join_gemm(asd_ctx *c, cudaStream_t gemm) {
    if (gemm == c->stream) return ASD_OK;
    ASD_CUDA_TRY(cudaEventRecord(c->gemm_done, gemm));
    ASD_CUDA_TRY(cudaStreamWaitEvent(c->stream, c->gemm_done, 0));
    return ASD_OK;
}

// Kernel timing: an event recorded on stream s before a timed launch (null
// when timing is off or s is being captured into a graph).
cudaEvent_t time_begin(asd_ctx *c, cudaStream_t s) {
    if (!c->timing || stream_capturing(s)) return nullptr;
    cudaEvent_t ev = nullptr;
    if (!c->ev_pool.empty()) {
        ev = c->ev_pool.back();
        c->ev_pool.pop_back();
    } else if (cudaEventCreate(&ev) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (cudaEventRecord(ev, s) != cudaSuccess) {
        cudaGetLastError();
        c->ev_pool.push_back(ev);
        return nullptr;
    }
    return ev;
}

// ... and after it: the pair is kept for asd_ctx_kernel_time.
void time_end(asd_ctx *c, int which, int launches, cudaStream_t s, cudaEvent_t b) {
    if (!b) return;
    cudaEvent_t ev = nullptr;
    if (!c->ev_pool.empty()) {
        ev = c->ev_pool.back();
        c->ev_pool.pop_back();
    } else if (cudaEventCreate(&ev) != cudaSuccess) {
        cudaGetLastError();
        c->ev_pool.push_back(b);
        return;
    }
    if (cudaEventRecord(ev, s) != cudaSuccess) {
        cudaGetLastError();
        c->ev_pool.push_back(b);
        c->ev_pool.push_back(ev);
        return;
    }
    c->timed.push_back({which, launches, b, ev});
}

int refresh_origin(asd_ctx *c) {
    // origin mean and the column epilogue vectors
    ASD_CUDA_TRY(launch_site_mean(c->origin, c->M, c->p.nfile, c->wphase, c->mean_0, c->col4,
                                  c->col1, c->stream));
    c->last_launches += 1;
    c->origin_version = c->state_version;
    for (int k = 1; k <= 3; ++k) c->b_version[k] = -1;
    return ASD_OK;
}

int set_spins_common(asd_ctx *c, const double *aos, bool host, int as_origin) {
    const size_t bytes = (size_t)c->M * c->K * sizeof(double);
    if (!aos) return fail(ASD_ERR_INVALID, "spins pointer is NULL");
    ASD_CUDA_TRY(cudaMemcpyAsync(c->ys_b, aos, bytes,
                                 host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice,
                                 c->stream));
    ASD_CUDA_TRY(launch_aos_to_sitemajor(c->ys_b, c->y, c->M, c->p.nfile, c->stream));
    c->last_launches += 1;
    c->state_version++;
    c->has_state = true;
    if (as_origin) {
        ASD_CUDA_TRY(cudaMemcpyAsync(c->origin, c->y, bytes, cudaMemcpyDeviceToDevice, c->stream));
        int rc = refresh_origin(c);
        if (rc != ASD_OK) return rc;
        c->has_origin = true;
        c->has_zsums = false;  // the ensemble's origin sums must be exchanged again
    }
    return ASD_OK;
}

// The LLG kernel for replicas [a.f0, a.f0 + a.nc): the one-launch step or
// the four stage kernels (ASD_LLG_AUTO: the former where it fills the GPU).
bool use_fused(const asd_ctx *c, const LLGArgs &a) {
    return c->llg_kernel == ASD_LLG_FUSED_STEP ||
           (c->llg_kernel == ASD_LLG_AUTO && llg_fused_fills(a));
}

int run_steps(asd_ctx *c, int nsteps) {
    if (use_fused(c, c->a)) {
        for (int s = 0; s < nsteps; ++s) {
            cudaEvent_t t0 = time_begin(c, c->stream);
            ASD_CUDA_TRY(launch_llg_step_fused(c->a, c->y, c->ys_a, c->stream));
            time_end(c, 0, 1, c->stream, t0);
            double *t = c->y;  // ping-pong: the new state becomes y
            c->y = c->ys_a;
            c->ys_a = t;
            c->last_launches += 1;
            c->state_version++;
        }
        return ASD_OK;
    }
    for (int s = 0; s < nsteps; ++s) {
        cudaEvent_t t0 = time_begin(c, c->stream);
        ASD_CUDA_TRY(launch_llg_stage(1, c->a, c->y, c->y, c->acc, c->ys_a, c->stream));
        ASD_CUDA_TRY(launch_llg_stage(2, c->a, c->y, c->ys_a, c->acc, c->ys_b, c->stream));
        ASD_CUDA_TRY(launch_llg_stage(3, c->a, c->y, c->ys_b, c->acc, c->ys_a, c->stream));
        ASD_CUDA_TRY(launch_llg_stage(4, c->a, nullptr, c->ys_a, c->acc, c->y, c->stream));
        time_end(c, 0, 4, c->stream, t0);
        c->last_launches += 4;
        c->state_version++;
    }
    return ASD_OK;
}

// The scale of the correlation GEMM: 1 / (replicas of the ensemble).  A
// shard's partial uses the whole ensemble's count and leaves out the
// connected-part term, which only the ensemble's means can give.
double gemm_alpha(const asd_ctx *c, bool shard) {
    return 1.0 / (double)((shard && c->nfile_total > 0) ? c->nfile_total : c->p.nfile);
}

// The plain FP64 path: the FP64 tensor-core GEMM with the fused epilogue,
// one partial per tile, then the fixed-order final sum.
DmmaSqtArgs dmma_args(const asd_ctx *c, bool shard) {
    DmmaSqtArgs g{};
    g.A = c->y;
    g.B = c->origin;
    g.M = c->M;
    g.K = c->K;
    g.alpha = gemm_alpha(c, shard);
    g.outer = shard ? 0 : 1;
    g.mrow = c->mean_t;
    g.zcol = c->mean_0;
    g.uphase = c->uphase;
    g.wphase = c->wphase;
    return g;
}

int sqt_plain(asd_ctx *c, double *d_out, bool shard) {
    const long tiles = dmma_sqt_tiles(c->M);
    if (tiles > 0x7fffffffL) return fail(ASD_ERR_UNSUPPORTED, "lattice too large for the FP64 GEMM");
    int rc = ensure_part(c, tiles);
    if (rc != ASD_OK) return rc;
    DmmaSqtArgs g = dmma_args(c, shard);
    g.part = c->part;
    cudaEvent_t t0 = time_begin(c, c->stream);
    rc = launch_dmma_sqt(g, c->stream);
    time_end(c, 1, 1, c->stream, t0);
    if (rc != ASD_OK) return rc;
    ASD_CUDA_TRY(launch_finalize(c->part, (int)tiles, 1.0 / (double)c->M, d_out, c->stream));
    c->last_launches += 2;
    return ASD_OK;
}

// Splits the origin (B) for `kind` where its operands are out of date: after
// a new origin and, for FP16x3, after a change of spin_len (which changes
// the operands' scale).
int ensure_split_origin(asd_ctx *c, int kind) {
    const double sc = split_scale(kind, c->p.spin_len);
    if (c->b_version[kind] == c->origin_version && c->b_scale[kind] == sc) return ASD_OK;
    ASD_CUDA_TRY(launch_split(kind, c->origin, c->M, c->K, c->Kp[kind], c->b_hi[kind],
                              c->b_lo[kind], sc, c->stream));
    c->b_version[kind] = c->origin_version;
    c->b_scale[kind] = sc;
    c->last_launches += 1;
    return ASD_OK;
}

// Both operands of `kind` up to date: the current state (A) after a step or
// set_spins, and the origin (B).
int ensure_split(asd_ctx *c, int kind) {
    if (!c->a_hi[kind]) return fail(ASD_ERR_STATE, "split mode %d not enabled at create", kind);
    const double sc = split_scale(kind, c->p.spin_len);
    if (c->a_version[kind] != c->state_version || c->a_scale[kind] != sc) {
        ASD_CUDA_TRY(launch_split(kind, c->y, c->M, c->K, c->Kp[kind], c->a_hi[kind],
                                  c->a_lo[kind], sc, c->stream));
        c->a_version[kind] = c->state_version;
        c->a_scale[kind] = sc;
        c->last_launches += 1;
    }
    return ensure_split_origin(c, kind);
}

// The GEMM arguments every split-mode launch shares.  alpha is the product's
// scale; the FP16 operands carry the factor scale^2, which alpha takes out
// (a power of two: the same FP32 roundings as unscaled operands).
UmmaSqtArgs split_args(const asd_ctx *c, int kind, double alpha) {
    const double sc = split_scale(kind, c->p.spin_len);
    UmmaSqtArgs u{};
    u.kind = kind;
    u.M = c->M;
    u.Kp = c->Kp[kind];
    u.a_hi = c->a_hi[kind];
    u.a_lo = c->a_lo[kind];
    u.b_hi = c->b_hi[kind];
    u.b_lo = c->b_lo[kind];
    u.row4 = c->row4;
    u.row1 = c->row1;
    u.col4 = c->col4;
    u.col1 = c->col1;
    u.alpha = (float)(alpha / (sc * sc));
    u.part = c->part;
    u.status = c->status;
    u.num_sms = c->num_sms;
    u.chunk_k = chunk_for(c, kind);
    return u;
}

int sqt_split(asd_ctx *c, int kind, double *d_out, bool shard) {
    int rc = ensure_split(c, kind);
    if (rc != ASD_OK) return rc;
    rc = ensure_part(c, c->num_sms);
    if (rc != ASD_OK) return rc;
    cudaStream_t gemm = c->stream;
    rc = arm_y_free(c, &gemm);
    if (rc != ASD_OK) return rc;
    UmmaSqtArgs u = split_args(c, kind, gemm_alpha(c, shard));
    u.outer = shard ? 0 : 1;
    cudaEvent_t t0 = time_begin(c, gemm);
    const int grid = launch_umma_sqt(u, gemm);
    time_end(c, 1, 1, gemm, t0);
    if (grid >= 0) {
        const cudaError_t e = launch_finalize(c->part, grid, 1.0 / (double)c->M, d_out, gemm);
        if (e != cudaSuccess) rc = cuda_fail(e, "launch_finalize");
        c->last_launches += 2;
    } else {
        rc = grid;
    }
    const int jrc = join_gemm(c, gemm);  // joined on the error paths too
    return rc != ASD_OK ? rc : jrc;
}

int sqt_async(asd_ctx *c, int mode, double *d_out, bool shard = false) {
    if (!c->has_state || !c->has_origin)
        return fail(ASD_ERR_STATE, "set the spins and the origin before S(q,t)");
    if (mode < 0 || mode > 3) return fail(ASD_ERR_INVALID, "unknown S(q,t) mode %d", mode);
    if (!(c->modes & (1u << mode))) return fail(ASD_ERR_STATE, "mode %d not enabled at create", mode);
    ASD_CUDA_TRY(launch_site_mean(c->y, c->M, c->p.nfile, c->uphase, c->mean_t, c->row4, c->row1,
                                  c->stream));
    c->rows_ready = true;
    c->last_launches += 1;
    switch (mode) {
        case ASD_SQT_FP64: return sqt_plain(c, d_out, shard);
        case ASD_SQT_TF32X3: return sqt_split(c, 1, d_out, shard);
        case ASD_SQT_BF16X3: return sqt_split(c, 2, d_out, shard);
        case ASD_SQT_FP16X3: return sqt_split(c, 3, d_out, shard);
    }
    return ASD_ERR_INVALID;
}

// One RK4 step y_in -> y_out on caller-chosen buffers (the four stage kernels;
// s2, s3, s4 and acc receive the stage states and the running combination).
int step_into(asd_ctx *c, const double *y_in, double *s2, double *s3, double *s4, double *acc,
              double *y_out) {
    ASD_CUDA_TRY(launch_llg_stage(1, c->a, y_in, y_in, acc, s2, c->stream));
    ASD_CUDA_TRY(launch_llg_stage(2, c->a, y_in, s2, acc, s3, c->stream));
    ASD_CUDA_TRY(launch_llg_stage(3, c->a, y_in, s3, acc, s4, c->stream));
    if (y_out) ASD_CUDA_TRY(launch_llg_stage(4, c->a, nullptr, s4, acc, y_out, c->stream));
    return ASD_OK;
}

// Work space of the adjoint: state-sized buffers (stage states, adjoint
// variables, checkpoints, one recomputed segment) and small reduction buffers.
// Where the RK4 step runs as four stage kernels and half of the free device
// memory holds them, also the stage states (s2, s3, s4, acc) of every step of
// a segment, so that the backward pass reads them instead of recomputing
// each step's stages a second time (c->adj_keep).
int ensure_adjoint(asd_ctx *c, int nsteps, int stride, int ckpt) {
    const long M = c->M;
    const int K = c->K, E = nsteps / stride;
    const size_t sb = (size_t)M * K * sizeof(double);
    const int nck = (nsteps + ckpt - 1) / ckpt;  // checkpoints at 0, ckpt, 2 ckpt, ...
    long need = 10 + nck + (ckpt + 1);
    const long need_keep = need + 4L * ckpt;
    bool keep = false;
    if (!use_fused(c, c->a)) {
        size_t free_b = 0, total_b = 0;
        if (c->adj_states >= need_keep) {
            keep = true;
        } else if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
            // the buffers held now are freed before the new set is allocated
            const double avail = (double)free_b + (double)c->adj_states * (double)sb;
            keep = (double)need_keep * (double)sb <= 0.5 * avail;
        } else {
            cudaGetLastError();
        }
    }
    if (keep) need = need_keep;
    c->adj_keep = keep;
    int rc;
    if (c->adj_states < need) {
        c->tape_valid = false;
        for (double *q : c->adj_bufs)
            if (q) cudaFree(q);
        c->adj_bufs.assign(need + 2, nullptr);
        c->adj_states = 0;
        for (long i = 0; i < need; ++i)
            if ((rc = dalloc(&c->adj_bufs[i], sb)) != ASD_OK) return rc;
        const int nb = adjoint_blocks(c->a);
        const size_t small = (size_t)nb * 6 * sizeof(double) +
                             ((size_t)fsum_chunks(M, K) * K + 2 * K + 8 + 2) * sizeof(double2);
        if ((rc = dalloc(&c->adj_bufs[need], small)) != ASD_OK) return rc;
        if ((rc = dalloc(&c->adj_bufs[need + 1], (size_t)(E + 8) * sizeof(double2))) != ASD_OK)
            return rc;
        c->adj_states = need;
    } else {
        // the S(q,t) buffer depends on E
        c->tape_valid = false;
        if (c->adj_bufs[c->adj_states + 1]) cudaFree(c->adj_bufs[c->adj_states + 1]);
        c->adj_bufs[c->adj_states + 1] = nullptr;
        if ((rc = dalloc(&c->adj_bufs[c->adj_states + 1], (size_t)(E + 8) * sizeof(double2))) !=
            ASD_OK)
            return rc;
    }
    return ASD_OK;
}

// The adjoint's buffers by role.
struct AdjBufs {
    double *s2, *s3, *s4, *acc, *lam, *lam_v, *lam_y, *P2, *P, *loc;
    double **ck, **seg;
    double **stg;  // with a kept segment: stg[4 (j - 1) + q] = s2, s3, s4, acc of step j
    double *bacc, *dgrad;
    double2 *Fpart, *G, *Z, *Sv;
    int nb;
};

AdjBufs adj_bufs(asd_ctx *c, int nck, int ckpt) {
    double **B = c->adj_bufs.data();
    AdjBufs b;
    b.s2 = B[0], b.s3 = B[1], b.s4 = B[2], b.acc = B[3], b.lam = B[4], b.lam_v = B[5];
    b.lam_y = B[6], b.P2 = B[7], b.P = B[8], b.loc = B[9];
    b.ck = B + 10;        // nck checkpoints
    b.seg = B + 10 + nck; // ckpt + 1 recomputed states
    b.stg = b.seg + ckpt + 1;
    b.nb = adjoint_blocks(c->a);
    b.bacc = B[c->adj_states];
    b.Fpart = reinterpret_cast<double2 *>(b.bacc + (size_t)b.nb * 6);
    b.G = b.Fpart + (size_t)fsum_chunks(c->M, c->K) * c->K;
    b.Z = b.G + c->K;
    b.dgrad = reinterpret_cast<double *>(b.Z + 4);
    b.Sv = reinterpret_cast<double2 *>(B[c->adj_states + 1]);
    return b;
}

// Forward pass of the loss: nsteps RK4 steps from the origin with the
// checkpoints kept for the adjoint, S(q,t) at every stride-th step (host copy
// in c->tape_S), and L against target if given.  Leaves the tape valid for
// loss_backward while the parameters and the origin stay as they are.
int loss_forward(asd_ctx *c, int nsteps, int stride, int ckpt, const double *target, double *loss,
                 double *sqt_out) {
    if (!c->has_origin) return fail(ASD_ERR_STATE, "set the origin (t = 0 spins) first");
    if (nsteps < 1 || stride < 1 || stride > nsteps || ckpt < 1)
        return fail(ASD_ERR_INVALID, "nsteps=%d stride=%d checkpoint=%d", nsteps, stride, ckpt);
    int rc = ensure_adjoint(c, nsteps, stride, ckpt);
    if (rc != ASD_OK) return rc;
    const long M = c->M;
    const int K = c->K, E = nsteps / stride;
    const size_t sb = (size_t)M * K * sizeof(double);
    const int nck = (nsteps + ckpt - 1) / ckpt;
    AdjBufs b = adj_bufs(c, nck, ckpt);
    cudaStream_t st = c->stream;
    c->last_launches = 0;
    c->tape_valid = false;
    // G_k and Z_c of the origin
    ASD_CUDA_TRY(launch_fsum(c->origin, M, K, c->wphase, b.Fpart, st));
    ASD_CUDA_TRY(launch_gz(b.Fpart, M, K, c->p.nfile, b.G, b.Z, st));
    c->last_launches += 2;
    // forward: checkpoints and S(q,t) at every stride-th step
    ASD_CUDA_TRY(cudaMemcpyAsync(b.ck[0], c->origin, sb, cudaMemcpyDeviceToDevice, st));
    double *cur = b.seg[0], *nxt = b.seg[1];
    ASD_CUDA_TRY(cudaMemcpyAsync(cur, c->origin, sb, cudaMemcpyDeviceToDevice, st));
    // Only states are kept on the way forward: one launch per step where
    // that fills the GPU.
    const bool fwd_fused = use_fused(c, c->a);
    for (int n = 1; n <= nsteps; ++n) {
        if (fwd_fused) {
            ASD_CUDA_TRY(launch_llg_step_fused(c->a, cur, nxt, st));
            c->last_launches += 1;
        } else {
            if ((rc = step_into(c, cur, b.s2, b.s3, b.s4, b.acc, nxt)) != ASD_OK) return rc;
            c->last_launches += 4;
        }
        double *t = cur;
        cur = nxt;
        nxt = t;
        if (n % ckpt == 0 && n / ckpt < nck)
            ASD_CUDA_TRY(cudaMemcpyAsync(b.ck[n / ckpt], cur, sb, cudaMemcpyDeviceToDevice, st));
        if (n % stride == 0 && n / stride <= E) {
            ASD_CUDA_TRY(launch_fsum(cur, M, K, c->uphase, b.Fpart, st));
            ASD_CUDA_TRY(launch_sqt_value(b.Fpart, M, K, c->p.nfile, b.G, b.Z, b.Sv + (n / stride - 1), st));
            c->last_launches += 2;
        }
    }
    c->tape_S.assign((size_t)E, make_double2(0.0, 0.0));
    ASD_CUDA_TRY(cudaMemcpyAsync(c->tape_S.data(), b.Sv, (size_t)E * sizeof(double2),
                                 cudaMemcpyDeviceToHost, st));
    ASD_CUDA_TRY(cudaStreamSynchronize(st));
    if (sqt_out)
        for (int e = 0; e < E; ++e) sqt_out[2 * e] = c->tape_S[e].x, sqt_out[2 * e + 1] = c->tape_S[e].y;
    double L = 0.0;
    if (target) {
        for (int e = 0; e < E; ++e) {
            const double dr = c->tape_S[e].x - target[2 * e], di = c->tape_S[e].y - target[2 * e + 1];
            L += dr * dr + di * di;
        }
        L /= E;
    }
    if (loss) *loss = L;
    c->tape_valid = true;
    c->tape_keep = c->adj_keep;
    c->tape_nsteps = nsteps;
    c->tape_stride = stride;
    c->tape_ckpt = ckpt;
    c->tape_params = c->params_version;
    c->tape_origin = c->origin_version;
    return ASD_OK;
}

// Backward pass of the loss from the tape of the last loss_forward:
// dL/d(J1, J2, alpha, hx, hy, hz) by the adjoint of the RK4 step and the
// renormalisation, segment by segment from the checkpoints; and, with
// dtarget, dL/dtarget = -2 (S - target) / E.
int loss_backward(asd_ctx *c, const double *target, double *grad, double *dtarget) {
    if (!target) return fail(ASD_ERR_INVALID, "target is NULL");
    if (!c->tape_valid || c->tape_params != c->params_version || c->tape_origin != c->origin_version)
        return fail(ASD_ERR_STATE, "no forward pass of the loss with the current parameters and origin");
    const long M = c->M;
    const int K = c->K, nsteps = c->tape_nsteps, stride = c->tape_stride, ckpt = c->tape_ckpt;
    const int E = nsteps / stride;
    const size_t sb = (size_t)M * K * sizeof(double);
    const int nck = (nsteps + ckpt - 1) / ckpt;
    AdjBufs b = adj_bufs(c, nck, ckpt);
    cudaStream_t st = c->stream;
    int rc;
    c->last_launches = 0;
    std::vector<double2> coef((size_t)E, make_double2(0.0, 0.0));
    const double scale = 2.0 / ((double)E * (double)M * c->p.nfile);
    for (int e = 0; e < E; ++e) {
        const double dr = c->tape_S[e].x - target[2 * e], di = c->tape_S[e].y - target[2 * e + 1];
        coef[e] = make_double2(scale * dr, -scale * di);  // 2 conj(S - T) / (E M nfile)
        if (dtarget) {
            dtarget[2 * e] = -2.0 * dr / E;
            dtarget[2 * e + 1] = -2.0 * di / E;
        }
    }
    if (!grad) return ASD_OK;
    const bool fwd_fused = use_fused(c, c->a);
    const bool keep = c->tape_keep && !fwd_fused;
    // backward through the segments, last first
    ASD_CUDA_TRY(cudaMemsetAsync(b.lam, 0, sb, st));
    ASD_CUDA_TRY(cudaMemsetAsync(b.bacc, 0, (size_t)b.nb * 6 * sizeof(double), st));
    double **seg = b.seg;
    for (int cidx = nck - 1; cidx >= 0; --cidx) {
        const int base = cidx * ckpt;
        const int len = (nsteps - base < ckpt) ? nsteps - base : ckpt;
        ASD_CUDA_TRY(cudaMemcpyAsync(seg[0], b.ck[cidx], sb, cudaMemcpyDeviceToDevice, st));
        for (int j = 1; j <= len; ++j) {
            double **sj = keep ? b.stg + 4 * (j - 1) : nullptr;
            if (fwd_fused) ASD_CUDA_TRY(launch_llg_step_fused(c->a, seg[j - 1], seg[j], st));
            else if ((rc = keep ? step_into(c, seg[j - 1], sj[0], sj[1], sj[2], sj[3], seg[j])
                                : step_into(c, seg[j - 1], b.s2, b.s3, b.s4, b.acc, seg[j])) != ASD_OK)
                return rc;
            c->last_launches += fwd_fused ? 1 : 4;
        }
        for (int n = base + len; n > base; --n) {
            const int j = n - base;
            if (n % stride == 0 && n / stride <= E) {
                const double2 cf = coef[n / stride - 1];
                ASD_CUDA_TRY(launch_loss_grad(b.lam, M, K, c->uphase, b.G, b.Z, cf.x, cf.y, st));
                c->last_launches += 1;
            }
            // y_{n-1} = seg[j-1]: its stage states (kept from the segment's
            // forward pass, or recomputed), then the adjoint
            double *s2 = b.s2, *s3 = b.s3, *s4 = b.s4, *acc = b.acc;
            if (keep) {
                double **sj = b.stg + 4 * (j - 1);
                s2 = sj[0], s3 = sj[1], s4 = sj[2], acc = sj[3];
            } else {
                if ((rc = step_into(c, seg[j - 1], s2, s3, s4, acc, nullptr)) != ASD_OK) return rc;
                c->last_launches += 4;
            }
            // stage 4 (through the renormalisation), 3, 2, 1: each launch
            // gathers the previous stage's P and forms the next stage's
            // product, so P alternates between two buffers
            const LLGArgs &a = c->a;
            ASD_CUDA_TRY(launch_adj_renorm_vjp(a, s4, acc, b.lam, b.lam_v, b.P, b.loc, b.bacc, st));
            ASD_CUDA_TRY(launch_vjp_gather(a, b.P, b.loc, b.lam_v, b.lam_v, b.lam_y, 1.0 / 3.0, 1.0,
                                           s3, b.P2, b.bacc, st));
            ASD_CUDA_TRY(launch_vjp_gather(a, b.P2, b.loc, b.lam_v, b.lam_y, b.lam_y, 1.0 / 3.0, 0.5,
                                           s2, b.P, b.bacc, st));
            ASD_CUDA_TRY(launch_vjp_gather(a, b.P, b.loc, b.lam_v, b.lam_y, b.lam_y, 1.0 / 6.0, 0.5,
                                           seg[j - 1], b.P2, b.bacc, st));
            ASD_CUDA_TRY(launch_vjp_gather(a, b.P2, b.loc, b.lam_v, b.lam_y, b.lam, 0.0, 0.0, nullptr,
                                           nullptr, b.bacc, st));
            c->last_launches += 5;
        }
    }
    ASD_CUDA_TRY(launch_param_reduce(b.bacc, b.nb, b.dgrad, st));
    c->last_launches += 1;
    ASD_CUDA_TRY(cudaMemcpyAsync(grad, b.dgrad, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
    ASD_CUDA_TRY(cudaStreamSynchronize(st));
    return ASD_OK;
}

int loss_grad(asd_ctx *c, int nsteps, int stride, int ckpt, const double *target, double *loss,
              double *grad, double *sqt_out) {
    int rc = loss_forward(c, nsteps, stride, ckpt, target, loss, sqt_out);
    if (rc != ASD_OK) return rc;
    if (!grad) return ASD_OK;
    for (int q = 0; q < 6; ++q) grad[q] = 0.0;
    if (!target) return ASD_OK;
    return loss_backward(c, target, grad, nullptr);
}

// Work space of the q grid's diagonal partials, grown on demand.
int ensure_grid_work(asd_ctx *c, size_t tdiag_n, size_t ds_n) {
    int rc;
    if (tdiag_n > c->grid_tdiag_n) {
        if (c->grid_tdiag) cudaFree(c->grid_tdiag);
        c->grid_tdiag = nullptr;
        c->grid_tdiag_n = 0;
        if ((rc = dalloc(&c->grid_tdiag, tdiag_n * sizeof(double))) != ASD_OK) return rc;
        c->grid_tdiag_n = tdiag_n;
    }
    if (ds_n > c->grid_ds_n) {
        if (c->grid_ds) cudaFree(c->grid_ds);
        c->grid_ds = nullptr;
        c->grid_ds_n = 0;
        if ((rc = dalloc(&c->grid_ds, ds_n * sizeof(double))) != ASD_OK) return rc;
        c->grid_ds_n = ds_n;
    }
    return ASD_OK;
}

int sqt_grid_async(asd_ctx *c, int mode, double *d_out) {
    if (!c->has_state || !c->has_origin)
        return fail(ASD_ERR_STATE, "set the spins and the origin before S(q,t)");
    const int N = c->p.N;
    const long M = c->M;
    if (mode < 0 || mode > 3)
        return fail(ASD_ERR_UNSUPPORTED, "q-grid S(q,t): mode %d not supported", mode);
    if (!(c->modes & (1u << mode))) return fail(ASD_ERR_STATE, "mode %d not enabled at create", mode);
    int rc;
    // each checked on its own: after a failed allocation of grid_t, grid_g
    // is already there and the next call must still allocate grid_t
    if (!c->grid_g && (rc = dalloc(&c->grid_g, (size_t)M * sizeof(double))) != ASD_OK) return rc;
    if (!c->grid_t && (rc = dalloc(&c->grid_t, (size_t)M * sizeof(double2))) != ASD_OK) return rc;
    ASD_CUDA_TRY(launch_site_mean(c->y, c->M, c->p.nfile, c->uphase, c->mean_t, c->row4, c->row1,
                                  c->stream));
    c->rows_ready = true;
    c->last_launches += 1;
    if (mode == ASD_SQT_FP64) {
        const long nm = (M + kDmmaTile - 1) / kDmmaTile;
        if (nm * nm > 0x7fffffffL) return fail(ASD_ERR_UNSUPPORTED, "lattice too large for the FP64 GEMM");
        const size_t nd2 = 2 * (2 * kDmmaTile - 1);
        rc = ensure_grid_work(c, (size_t)(nm * nm) * nd2,
                              (size_t)qgrid_keys((int)nm, (int)nm, kDmmaTile, kDmmaTile) * nd2);
        if (rc != ASD_OK) return rc;
        DmmaSqtArgs g = dmma_args(c, false);
        g.lat_n = N;
        g.tdiag = c->grid_tdiag;
        if ((rc = launch_dmma_sqt(g, c->stream)) != ASD_OK) return rc;
        ASD_CUDA_TRY(launch_qgrid_bins(c->grid_tdiag, (int)nm, (int)nm, kDmmaTile, kDmmaTile, N,
                                       c->grid_ds, c->grid_g, c->stream));
        ASD_CUDA_TRY(launch_grid_dft(c->grid_g, N, 1.0 / (double)M, c->grid_t, d_out, c->stream));
        c->last_launches += 5;
        return ASD_OK;
    }
    const int kind = mode_kind(mode);
    if ((rc = ensure_split(c, kind)) != ASD_OK) return rc;
    const int bm = umma_tile_rows(), bn = umma_tile_cols();
    const int num_m = (int)(c->Mp / bm), num_n = (int)(c->Mp / bn);
    const size_t nd2 = 2 * (size_t)(bm + bn - 1);
    rc = ensure_grid_work(c, (size_t)num_m * num_n * nd2, (size_t)qgrid_keys(num_m, num_n, bm, bn) * nd2);
    if (rc != ASD_OK) return rc;
    UmmaSqtArgs u = split_args(c, kind, 1.0 / (double)c->p.nfile);
    u.tdiag = c->grid_tdiag;
    u.lat_n = N;
    const int grid = launch_umma_sqt(u, c->stream);
    if (grid < 0) return grid;
    ASD_CUDA_TRY(launch_qgrid_bins(c->grid_tdiag, num_m, num_n, bm, bn, N, c->grid_ds, c->grid_g,
                                   c->stream));
    c->last_launches += 3;
    ASD_CUDA_TRY(launch_grid_dft(c->grid_g, N, 1.0 / (double)M, c->grid_t, d_out, c->stream));
    c->last_launches += 1;
    return ASD_OK;
}

int read_status(asd_ctx *c) {
    unsigned st = 0;
    ASD_CUDA_TRY(cudaMemcpyAsync(&st, c->status, sizeof st, cudaMemcpyDeviceToHost, c->stream));
    ASD_CUDA_TRY(cudaMemsetAsync(c->status, 0, sizeof(unsigned), c->stream));
    ASD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (st & kStatusTimeout) return fail(ASD_ERR_TIMEOUT, "a device-side wait gave up (status %u)", st);
    if (st) return fail(ASD_ERR_CUDA, "device status %u", st);
    return ASD_OK;
}

// Replicas per chunk of the pipelined host step: about an eighth of the
// ensemble, rounded up to a multiple of 64 so that every chunk boundary
// (3 K columns per replica) is a whole k block of both the TF32 (32
// columns) and the BF16 (64 columns) GEMM.
int host_chunk_replicas(int nfile) {
    const int target = (nfile + 7) / 8;
    return (target + 63) / 64 * 64;
}

// The upload and download streams (and the sync pipeline's events).
int ensure_copy_streams(asd_ctx *c) {
    if (!c->copy_stream) {
        ASD_CUDA_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        ASD_CUDA_TRY(cudaEventCreateWithFlags(&c->spins_ready, cudaEventDisableTiming));
    }
    if (!c->h2d_stream) {
        ASD_CUDA_TRY(cudaStreamCreateWithFlags(&c->h2d_stream, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            cudaEvent_t *ev[] = {&c->in_ready[b], &c->in_free[b], &c->out_ready[b],
                                 &c->out_free[b]};
            for (cudaEvent_t *x : ev)
                ASD_CUDA_TRY(cudaEventCreateWithFlags(x, cudaEventDisableTiming));
        }
    }
    return ASD_OK;
}

int ensure_host_pipeline(asd_ctx *c, int cr) {
    int rc0 = ensure_copy_streams(c);
    if (rc0 != ASD_OK) return rc0;
    if (c->hp_replicas == cr) return ASD_OK;
    for (int b = 0; b < 2; ++b) {
        if (c->stage_in[b]) cudaFree(c->stage_in[b]);
        if (c->stage_out[b]) cudaFree(c->stage_out[b]);
        c->stage_in[b] = c->stage_out[b] = nullptr;
    }
    c->hp_replicas = 0;
    const size_t bytes = (size_t)cr * c->M * 3 * sizeof(double);
    for (int b = 0; b < 2; ++b) {
        int rc = dalloc(&c->stage_in[b], bytes);
        if (rc == ASD_OK) rc = dalloc(&c->stage_out[b], bytes);
        if (rc != ASD_OK) return rc;
    }
    c->hp_replicas = cr;
    return ASD_OK;
}

// asd_ctx_step_host in replica chunks.  Replicas never interact, and the
// correlation GEMM's K axis is the replica axis, so each chunk goes through
// upload -> site-major transpose -> the four RK4 stages on its replicas ->
// AoS transpose -> download, and (split modes) the split of its K columns and
// a GEMM over that K range whose partial S(q,t) joins the others in the
// final sum.  Only the last chunk's GEMM carries the connected-part term, after
// the site means of the whole new state.  Uploads, compute and downloads run
// on three streams, so the PCIe traffic of one chunk overlaps the compute of
// its neighbours in both directions.  The spins are bit-identical to the
// one-shot path; S(q,t) differs only in the order of its partial sums.
int step_host_chunked(asd_ctx *c, const double *spin_in, double *spin_out, int mode, int cr) {
    const int nf = c->p.nfile;
    const long M = c->M;
    const int kind = mode_kind(mode);
    if (mode < 0 || mode > 3) return fail(ASD_ERR_INVALID, "unknown S(q,t) mode %d", mode);
    if (!(c->modes & (1u << mode))) return fail(ASD_ERR_STATE, "mode %d not enabled at create", mode);
    int rc = ensure_host_pipeline(c, cr);
    if (rc != ASD_OK) return rc;
    const int nchunks = (nf + cr - 1) / cr;
    if (kind) {
        if (!c->a_hi[kind]) return fail(ASD_ERR_STATE, "split mode %d not enabled at create", kind);
        if ((rc = ensure_split_origin(c, kind)) != ASD_OK) return rc;
        if (!c->rows_ready) {  // the early chunks' epilogues read the phase u_i
            ASD_CUDA_TRY(launch_site_mean(c->y, M, nf, c->uphase, c->mean_t, c->row4, c->row1,
                                          c->stream));
            c->rows_ready = true;
            c->last_launches += 1;
        }
        if ((rc = ensure_part(c, (long)nchunks * c->num_sms)) != ASD_OK) return rc;
    }
    const cudaStream_t comp = c->stream, up = c->h2d_stream, down = c->copy_stream;
    LLGArgs a = c->a;
    long nparts = 0;
    // The one-launch step is out of place: each chunk's new state goes to
    // ys_a (its replicas only), and y and ys_a swap after the last chunk.
    LLGArgs ac = c->a;  // a whole chunk decides the kernel for every chunk
    ac.nc = cr < nf ? cr : nf;
    const bool fused = use_fused(c, ac);
    double *const ynew = fused ? c->ys_a : c->y;
    for (int r = 0; r < nchunks; ++r) {
        const int f0 = r * cr, nc = (nf - f0 < cr) ? nf - f0 : cr, b = r & 1;
        const bool last = (f0 + nc == nf);
        const size_t off = (size_t)f0 * M * 3, bytes = (size_t)nc * M * 3 * sizeof(double);
        ASD_CUDA_TRY(cudaStreamWaitEvent(up, c->in_free[b], 0));
        ASD_CUDA_TRY(cudaMemcpyAsync(c->stage_in[b], spin_in + off, bytes,
                                     cudaMemcpyHostToDevice, up));
        ASD_CUDA_TRY(cudaEventRecord(c->in_ready[b], up));
        ASD_CUDA_TRY(cudaStreamWaitEvent(comp, c->in_ready[b], 0));
        ASD_CUDA_TRY(launch_aos_to_sitemajor_range(c->stage_in[b], c->y, M, nf, f0, nc, comp));
        ASD_CUDA_TRY(cudaEventRecord(c->in_free[b], comp));
        a.f0 = f0;
        a.nc = nc;
        if (fused) {
            ASD_CUDA_TRY(launch_llg_step_fused(a, c->y, ynew, comp));
        } else {
            ASD_CUDA_TRY(launch_llg_stage(1, a, c->y, c->y, c->acc, c->ys_a, comp));
            ASD_CUDA_TRY(launch_llg_stage(2, a, c->y, c->ys_a, c->acc, c->ys_b, comp));
            ASD_CUDA_TRY(launch_llg_stage(3, a, c->y, c->ys_b, c->acc, c->ys_a, comp));
            ASD_CUDA_TRY(launch_llg_stage(4, a, nullptr, c->ys_a, c->acc, c->y, comp));
        }
        ASD_CUDA_TRY(cudaStreamWaitEvent(comp, c->out_free[b], 0));
        ASD_CUDA_TRY(launch_sitemajor_to_aos_range(ynew, c->stage_out[b], M, nf, f0, nc, comp));
        ASD_CUDA_TRY(cudaEventRecord(c->out_ready[b], comp));
        ASD_CUDA_TRY(cudaStreamWaitEvent(down, c->out_ready[b], 0));
        ASD_CUDA_TRY(cudaMemcpyAsync(spin_out + off, c->stage_out[b], bytes,
                                     cudaMemcpyDeviceToHost, down));
        ASD_CUDA_TRY(cudaEventRecord(c->out_free[b], down));
        c->last_launches += fused ? 3 : 6;
        if (!kind) continue;
        const int kbeg = 3 * f0, kend = last ? c->Kp[kind] : 3 * (f0 + nc);
        ASD_CUDA_TRY(launch_split_range(kind, ynew, M, c->K, c->Kp[kind], kbeg, kend,
                                        c->a_hi[kind], c->a_lo[kind],
                                        split_scale(kind, c->p.spin_len), comp));
        c->last_launches += 1;
        if (last) {
            ASD_CUDA_TRY(launch_site_mean(ynew, M, nf, c->uphase, c->mean_t, c->row4, c->row1,
                                          comp));
            c->last_launches += 1;
        }
        UmmaSqtArgs u = split_args(c, kind, 1.0 / (double)nf);
        u.part = c->part + nparts;
        u.k_begin = kbeg;
        u.k_end = kend;
        u.outer = last ? 1 : 0;
        const int grid = launch_umma_sqt(u, comp);
        if (grid < 0) return grid;
        nparts += grid;
        c->last_launches += 1;
    }
    if (fused) {  // ys_a holds the new state of every replica
        c->ys_a = c->y;
        c->y = ynew;
    }
    c->state_version += 2;  // as set_spins + step
    c->has_state = true;
    if (kind) {
        c->a_version[kind] = c->state_version;
        c->a_scale[kind] = split_scale(kind, c->p.spin_len);
        ASD_CUDA_TRY(launch_finalize(c->part, (int)nparts, 1.0 / (double)M, c->d_out, comp));
        c->last_launches += 1;
        return ASD_OK;
    }
    return sqt_async(c, mode, c->d_out);
}

// asd_ctx_step_host_async.  Per replica chunk r: upload (h2d_stream) into
// the chunk's region of the whole-state staging buffer, site-major
// transpose, RK4 on the chunk's replicas, AoS transpose, download
// (copy_stream); then S(q,t) of the new state on the ctx stream.  Nothing
// waits for the host, so consecutive calls overlap: the upload of chunk r
// of the next call waits only for the download of chunk r of this one (the
// caller may pass this call's output as the next call's input) and for the
// transpose that emptied its staging region; the GEMM of one call runs
// while the next call's chunks cross PCIe.
int async_chunk_replicas(int nfile) {
    const int target = (nfile + 7) / 8;
    int cr = (target + 31) / 32 * 32;
    while ((nfile + cr - 1) / cr > asd_ctx::kAsyncChunks) cr += 32;
    return cr;
}

int ensure_async_pipeline(asd_ctx *c) {
    int rc = ensure_copy_streams(c);
    if (rc != ASD_OK) return rc;
    if (!c->ast_events) {
        for (int r = 0; r < asd_ctx::kAsyncChunks; ++r) {
            cudaEvent_t *ev[] = {&c->ast_in_ready[r], &c->ast_in_done[r], &c->ast_out_ready[r],
                                 &c->ast_out_done[r]};
            for (cudaEvent_t *x : ev)
                ASD_CUDA_TRY(cudaEventCreateWithFlags(x, cudaEventDisableTiming));
        }
        c->ast_events = true;
    }
    const size_t bytes = (size_t)c->M * c->K * sizeof(double);
    if (!c->ast_in && (rc = dalloc(&c->ast_in, bytes)) != ASD_OK) return rc;
    if (!c->ast_out && (rc = dalloc(&c->ast_out, bytes)) != ASD_OK) return rc;
    return ASD_OK;
}

bool pinned_or_device(const void *p) {
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost || at.type == cudaMemoryTypeDevice ||
           at.type == cudaMemoryTypeManaged;
}

int step_host_async(asd_ctx *c, const double *spin_in, double *spin_out, int mode,
                    double *sqt_out) {
    const int nf = c->p.nfile;
    const long M = c->M;
    int rc = ensure_async_pipeline(c);
    if (rc != ASD_OK) return rc;
    const int cr = async_chunk_replicas(nf), nchunks = (nf + cr - 1) / cr;
    const cudaStream_t comp = c->stream, up = c->h2d_stream, down = c->copy_stream;
    LLGArgs ac = c->a;  // a whole chunk decides the kernel for every chunk
    ac.nc = cr < nf ? cr : nf;
    const bool fused = use_fused(c, ac);
    double *const ynew = fused ? c->ys_a : c->y;
    LLGArgs a = c->a;
    for (int r = 0; r < nchunks; ++r) {
        const int f0 = r * cr, nc = (nf - f0 < cr) ? nf - f0 : cr;
        const size_t off = (size_t)f0 * M * 3, bytes = (size_t)nc * M * 3 * sizeof(double);
        ASD_CUDA_TRY(cudaStreamWaitEvent(up, c->ast_out_done[r], 0));
        ASD_CUDA_TRY(cudaStreamWaitEvent(up, c->ast_in_done[r], 0));
        ASD_CUDA_TRY(cudaMemcpyAsync(c->ast_in + off, spin_in + off, bytes, cudaMemcpyDefault,
                                     up));  // pinned host or device memory
        ASD_CUDA_TRY(cudaEventRecord(c->ast_in_ready[r], up));
        ASD_CUDA_TRY(cudaStreamWaitEvent(comp, c->ast_in_ready[r], 0));
        ASD_CUDA_TRY(launch_aos_to_sitemajor_range(c->ast_in + off, c->y, M, nf, f0, nc, comp));
        ASD_CUDA_TRY(cudaEventRecord(c->ast_in_done[r], comp));
        a.f0 = f0;
        a.nc = nc;
        if (fused) {
            ASD_CUDA_TRY(launch_llg_step_fused(a, c->y, ynew, comp));
        } else {
            ASD_CUDA_TRY(launch_llg_stage(1, a, c->y, c->y, c->acc, c->ys_a, comp));
            ASD_CUDA_TRY(launch_llg_stage(2, a, c->y, c->ys_a, c->acc, c->ys_b, comp));
            ASD_CUDA_TRY(launch_llg_stage(3, a, c->y, c->ys_b, c->acc, c->ys_a, comp));
            ASD_CUDA_TRY(launch_llg_stage(4, a, nullptr, c->ys_a, c->acc, c->y, comp));
        }
        ASD_CUDA_TRY(cudaStreamWaitEvent(comp, c->ast_out_done[r], 0));
        ASD_CUDA_TRY(launch_sitemajor_to_aos_range(ynew, c->ast_out + off, M, nf, f0, nc, comp));
        ASD_CUDA_TRY(cudaEventRecord(c->ast_out_ready[r], comp));
        ASD_CUDA_TRY(cudaStreamWaitEvent(down, c->ast_out_ready[r], 0));
        ASD_CUDA_TRY(cudaMemcpyAsync(spin_out + off, c->ast_out + off, bytes, cudaMemcpyDefault,
                                     down));
        ASD_CUDA_TRY(cudaEventRecord(c->ast_out_done[r], down));
        c->last_launches += fused ? 3 : 6;
    }
    if (fused) {  // ys_a holds the new state of every replica
        c->ys_a = c->y;
        c->y = ynew;
    }
    c->state_version += 2;  // as set_spins + step
    c->has_state = true;
    if ((rc = sqt_async(c, mode, c->d_out)) != ASD_OK) return rc;
    ASD_CUDA_TRY(cudaMemcpyAsync(sqt_out, c->d_out, 2 * sizeof(double), cudaMemcpyDefault, comp));
    return ASD_OK;
}

void destroy(asd_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    void *ptrs[] = {c->y, c->ys_a, c->ys_b, c->acc, c->origin, c->mean_t, c->mean_0, c->uphase,
                    c->wphase, c->row4, c->col4, c->row1, c->col1, c->grid_tdiag, c->grid_ds, c->part, c->d_out,
                    c->status, c->grid_g, c->grid_t, c->grid_out};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    for (int k = 1; k <= 3; ++k) {
        void *ops[] = {c->a_hi[k], c->a_lo[k], c->b_hi[k], c->b_lo[k]};
        for (void *q : ops)
            if (q) cudaFree(q);
    }
    for (double *q : c->adj_bufs)
        if (q) cudaFree(q);
    if (c->h_out) cudaFreeHost(c->h_out);
    if (c->spins_ready) cudaEventDestroy(c->spins_ready);
    if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
    for (int b = 0; b < 2; ++b) {
        if (c->stage_in[b]) cudaFree(c->stage_in[b]);
        if (c->stage_out[b]) cudaFree(c->stage_out[b]);
        cudaEvent_t ev[] = {c->in_ready[b], c->in_free[b], c->out_ready[b], c->out_free[b]};
        for (cudaEvent_t x : ev)
            if (x) cudaEventDestroy(x);
    }
    if (c->h2d_stream) {
        cudaStreamSynchronize(c->h2d_stream);
        cudaStreamDestroy(c->h2d_stream);
    }
    if (c->ast_in) cudaFree(c->ast_in);
    if (c->ast_out) cudaFree(c->ast_out);
    for (int r = 0; c->ast_events && r < asd_ctx::kAsyncChunks; ++r) {
        cudaEvent_t ev[] = {c->ast_in_ready[r], c->ast_in_done[r], c->ast_out_ready[r],
                            c->ast_out_done[r]};
        for (cudaEvent_t x : ev)
            if (x) cudaEventDestroy(x);
    }
    if (c->llg_stream) {
        cudaStreamSynchronize(c->llg_stream);
        cudaStreamDestroy(c->llg_stream);
    }
    if (c->gemm_stream) {
        cudaStreamSynchronize(c->gemm_stream);
        cudaStreamDestroy(c->gemm_stream);
    }
    if (c->gemm_done) cudaEventDestroy(c->gemm_done);
    if (c->zsums) cudaFree(c->zsums);
    if (c->y_free) cudaEventDestroy(c->y_free);
    if (c->llg_done) cudaEventDestroy(c->llg_done);
    for (auto &t : c->timed) {
        cudaEventDestroy(t.b);
        cudaEventDestroy(t.e);
    }
    for (cudaEvent_t ev : c->ev_pool) cudaEventDestroy(ev);
    delete c;
}

}  // namespace

extern "C" {

const char *asd_version(void) { return "asd_b200 0.1 (sm_100a)"; }

const char *asd_last_error(void) { return g_err; }

int asd_params_default(asd_params *p, int N, int nfile) {
    if (!p) return fail(ASD_ERR_INVALID, "params is NULL");
    std::memset(p, 0, sizeof *p);
    p->N = N;
    p->nfile = nfile;
    p->J1 = 1.0;
    p->dt = 0.02;
    p->spin_len = 1.0;
    p->vx = N / 10;
    p->vy = N / 10;
    return ASD_OK;
}

int asd_set_device(int device) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
    if (device < 0 || device >= n) return fail(ASD_ERR_INVALID, "device %d of %d", device, n);
    g_device = device;
    return ASD_OK;
}

int asd_ctx_create(const asd_params *p, unsigned mode_mask, asd_ctx **out) {
    if (!out) return fail(ASD_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = check_params(p);
    if (rc != ASD_OK) return rc;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        return fail(ASD_ERR_CUDA, "no CUDA device: %s", cudaGetErrorString(e));
    ASD_CUDA_TRY(cudaSetDevice(g_device));
    cudaDeviceProp prop;
    ASD_CUDA_TRY(cudaGetDeviceProperties(&prop, g_device));
    if (prop.major != 10)
        return fail(ASD_ERR_UNSUPPORTED, "device %d is sm_%d%d; this library is built for sm_100a",
                    g_device, prop.major, prop.minor);

    asd_ctx *c = new asd_ctx();
    c->p = *p;
    c->a = make_llg_args(*p);
    c->device = g_device;
    c->num_sms = prop.multiProcessorCount;
    c->M = (long)p->N * p->N;
    c->Mp = umma_row_pad(c->M);
    c->K = 3 * p->nfile;
    if (mode_mask & ~0xFu) {
        delete c;
        return fail(ASD_ERR_INVALID, "mode_mask 0x%x has bits beyond the four S(q,t) modes", mode_mask);
    }
    c->modes = mode_mask ? mode_mask : 0xFu;
    const size_t sbytes = (size_t)c->M * c->K * sizeof(double);
#define ASD_ALLOC(ptr, bytes)                 \
    do {                                      \
        rc = dalloc(&(ptr), (bytes));         \
        if (rc != ASD_OK) { destroy(c); return rc; } \
    } while (0)
    ASD_ALLOC(c->y, sbytes);
    ASD_ALLOC(c->ys_a, sbytes);
    ASD_ALLOC(c->ys_b, sbytes);
    ASD_ALLOC(c->acc, sbytes);
    ASD_ALLOC(c->origin, sbytes);
    ASD_ALLOC(c->mean_t, (size_t)c->M * 3 * sizeof(double));
    ASD_ALLOC(c->mean_0, (size_t)c->M * 3 * sizeof(double));
    ASD_ALLOC(c->uphase, (size_t)c->M * sizeof(double2));
    ASD_ALLOC(c->wphase, (size_t)c->M * sizeof(double2));
    ASD_ALLOC(c->row4, (size_t)c->Mp * sizeof(float4));
    ASD_ALLOC(c->col4, (size_t)c->Mp * sizeof(float4));
    ASD_ALLOC(c->row1, (size_t)c->Mp * sizeof(float));
    ASD_ALLOC(c->col1, (size_t)c->Mp * sizeof(float));
    ASD_ALLOC(c->d_out, 2 * sizeof(double));
    ASD_ALLOC(c->status, sizeof(unsigned));
    for (int mode = ASD_SQT_TF32X3; mode <= ASD_SQT_FP16X3; ++mode) {
        const int kind = mode_kind(mode);
        if (!(c->modes & (1u << mode))) continue;
        c->Kp[kind] = kp_for(kind, c->K);
        const size_t ob = (size_t)c->Mp * c->Kp[kind] * split_esize(kind);
        ASD_ALLOC(c->a_hi[kind], ob);
        ASD_ALLOC(c->a_lo[kind], ob);
        ASD_ALLOC(c->b_hi[kind], ob);
        ASD_ALLOC(c->b_lo[kind], ob);
        // padding rows stay zero for the lifetime of the context
        ASD_CUDA_TRY(cudaMemset(c->a_hi[kind], 0, ob));
        ASD_CUDA_TRY(cudaMemset(c->a_lo[kind], 0, ob));
        ASD_CUDA_TRY(cudaMemset(c->b_hi[kind], 0, ob));
        ASD_CUDA_TRY(cudaMemset(c->b_lo[kind], 0, ob));
    }
#undef ASD_ALLOC
    ASD_CUDA_TRY(cudaMemset(c->row4, 0, (size_t)c->Mp * sizeof(float4)));
    ASD_CUDA_TRY(cudaMemset(c->col4, 0, (size_t)c->Mp * sizeof(float4)));
    ASD_CUDA_TRY(cudaMemset(c->row1, 0, (size_t)c->Mp * sizeof(float)));
    ASD_CUDA_TRY(cudaMemset(c->col1, 0, (size_t)c->Mp * sizeof(float)));
    ASD_CUDA_TRY(cudaMemset(c->status, 0, sizeof(unsigned)));
    e = cudaMallocHost((void **)&c->h_out, 2 * sizeof(double));
    if (e != cudaSuccess) {
        destroy(c);
        return cuda_fail(e, "cudaMallocHost");
    }
    // Phases u_i = e^{-i q.r_i} and w_j = e^{+i q.r_j}, q = 2 pi (vx, vy) / N
    // (llg_sqt_baseline.c:267-268), so that u_i w_j = e^{-i q.(r_i - r_j)}.
    {
        const double qx = 2.0 * M_PI * p->vx / (double)p->N;
        const double qy = 2.0 * M_PI * p->vy / (double)p->N;
        std::vector<double2> u((size_t)c->M), w((size_t)c->M);
        for (long i = 0; i < c->M; ++i) {
            const double th = qx * (double)(i / p->N) + qy * (double)(i % p->N);
            const double cs = std::cos(th), sn = std::sin(th);
            u[i] = make_double2(cs, -sn);
            w[i] = make_double2(cs, sn);
        }
        ASD_CUDA_TRY(cudaMemcpy(c->uphase, u.data(), (size_t)c->M * sizeof(double2),
                                cudaMemcpyHostToDevice));
        ASD_CUDA_TRY(cudaMemcpy(c->wphase, w.data(), (size_t)c->M * sizeof(double2),
                                cudaMemcpyHostToDevice));
    }
    rc = ensure_part(c, c->num_sms);
    if (rc != ASD_OK) {
        destroy(c);
        return rc;
    }
    *out = c;
    return ASD_OK;
}

int asd_ctx_destroy(asd_ctx *ctx) {
    destroy(ctx);
    return ASD_OK;
}

int asd_ctx_set_stream(asd_ctx *c, void *stream) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    c->y_free_armed = false;
    c->stream = (cudaStream_t)stream;
    return ASD_OK;
}

int asd_ctx_get_params(const asd_ctx *c, asd_params *p) {
    if (!c || !p) return fail(ASD_ERR_INVALID, "NULL argument");
    *p = c->p;
    return ASD_OK;
}

int asd_ctx_set_spins(asd_ctx *c, const double *spin_aos, int as_origin) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    int rc = set_spins_common(c, spin_aos, true, as_origin);
    if (rc != ASD_OK) return rc;
    ASD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return ASD_OK;
}

int asd_ctx_set_spins_device(asd_ctx *c, const double *d_spin_aos, int as_origin) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    return set_spins_common(c, d_spin_aos, false, as_origin);
}

int asd_ctx_get_spins(asd_ctx *c, double *spin_aos) {
    if (!c || !spin_aos) return fail(ASD_ERR_INVALID, "NULL argument");
    if (!c->has_state) return fail(ASD_ERR_STATE, "no spins set");
    ASD_CUDA_TRY(enter(c));
    ASD_CUDA_TRY(launch_sitemajor_to_aos(c->y, c->ys_b, c->M, c->p.nfile, c->stream));
    ASD_CUDA_TRY(cudaMemcpyAsync(spin_aos, c->ys_b, (size_t)c->M * c->K * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream));
    ASD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return ASD_OK;
}

int asd_ctx_get_spins_device(asd_ctx *c, double *d_spin_aos) {
    if (!c || !d_spin_aos) return fail(ASD_ERR_INVALID, "NULL argument");
    if (!c->has_state) return fail(ASD_ERR_STATE, "no spins set");
    ASD_CUDA_TRY(enter(c));
    ASD_CUDA_TRY(launch_sitemajor_to_aos(c->y, d_spin_aos, c->M, c->p.nfile, c->stream));
    return ASD_OK;
}

int asd_ctx_step(asd_ctx *c, int nsteps) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    if (nsteps < 0) return fail(ASD_ERR_INVALID, "nsteps < 0");
    if (!c->has_state) return fail(ASD_ERR_STATE, "no spins set");
    const bool overlap = c->y_free_armed && nsteps > 0 && !stream_capturing(c->stream);
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    if (!overlap) return run_steps(c, nsteps);
    // The steps wait only for the split of the last S(q,t), run on llg_stream
    // beside its GEMM, and the ctx stream joins them before its next work.
    const cudaStream_t main = c->stream;
    ASD_CUDA_TRY(cudaStreamWaitEvent(c->llg_stream, c->y_free, 0));
    c->stream = c->llg_stream;
    const int rc = run_steps(c, nsteps);
    c->stream = main;
    ASD_CUDA_TRY(cudaEventRecord(c->llg_done, c->llg_stream));
    ASD_CUDA_TRY(cudaStreamWaitEvent(main, c->llg_done, 0));
    return rc;
}

int asd_ctx_sqt_async(asd_ctx *c, asd_sqt_mode mode, double *d_out) {
    if (!c || !d_out) return fail(ASD_ERR_INVALID, "NULL argument");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    return sqt_async(c, (int)mode, d_out);
}

int asd_ctx_sqt_grid_async(asd_ctx *c, asd_sqt_mode mode, double *d_out) {
    if (!c || !d_out) return fail(ASD_ERR_INVALID, "NULL argument");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    return sqt_grid_async(c, (int)mode, d_out);
}

int asd_ctx_loss_grad(asd_ctx *c, int nsteps, int stride, int checkpoint, const double *target,
                      double *loss, double *grad, double *sqt_out) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    ASD_CUDA_TRY(enter(c));
    return loss_grad(c, nsteps, stride, checkpoint, target, loss, grad, sqt_out);
}

int asd_ctx_loss_forward(asd_ctx *c, int nsteps, int stride, int checkpoint, const double *target,
                         double *loss, double *sqt_out) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    ASD_CUDA_TRY(enter(c));
    return loss_forward(c, nsteps, stride, checkpoint, target, loss, sqt_out);
}

int asd_ctx_loss_backward(asd_ctx *c, const double *target, double *grad, double *dtarget) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    ASD_CUDA_TRY(enter(c));
    return loss_backward(c, target, grad, dtarget);
}

int asd_ctx_set_params(asd_ctx *c, const asd_params *p) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    int rc = check_params(p);
    if (rc != ASD_OK) return rc;
    if (p->N != c->p.N || p->nfile != c->p.nfile)
        return fail(ASD_ERR_INVALID, "N and nfile are fixed at create");
    const bool q_changed = (p->vx != c->p.vx || p->vy != c->p.vy);
    c->p = *p;
    c->params_version++;
    c->a = make_llg_args(*p);
    if (q_changed) {
        const double qx = 2.0 * M_PI * p->vx / (double)p->N, qy = 2.0 * M_PI * p->vy / (double)p->N;
        std::vector<double2> u((size_t)c->M), w((size_t)c->M);
        for (long i = 0; i < c->M; ++i) {
            const double th = qx * (double)(i / p->N) + qy * (double)(i % p->N);
            u[i] = make_double2(std::cos(th), -std::sin(th));
            w[i] = make_double2(std::cos(th), std::sin(th));
        }
        ASD_CUDA_TRY(enter(c));
        c->rows_ready = false;
        ASD_CUDA_TRY(cudaMemcpy(c->uphase, u.data(), (size_t)c->M * sizeof(double2), cudaMemcpyHostToDevice));
        ASD_CUDA_TRY(cudaMemcpy(c->wphase, w.data(), (size_t)c->M * sizeof(double2), cudaMemcpyHostToDevice));
        if (c->has_origin) return refresh_origin(c);
    }
    return ASD_OK;
}

int asd_ctx_sqt_grid(asd_ctx *c, asd_sqt_mode mode, double *out) {
    if (!c || !out) return fail(ASD_ERR_INVALID, "NULL argument");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    const size_t bytes = (size_t)c->M * 2 * sizeof(double);
    int rc;
    if (!c->grid_out && (rc = dalloc(&c->grid_out, bytes)) != ASD_OK) return rc;
    if ((rc = sqt_grid_async(c, (int)mode, c->grid_out)) != ASD_OK) return rc;
    ASD_CUDA_TRY(cudaMemcpyAsync(out, c->grid_out, bytes, cudaMemcpyDeviceToHost, c->stream));
    return read_status(c);  // synchronises
}

int asd_ctx_sqt_magnitude(asd_ctx *c, double *out) {
    if (!c || !out) return fail(ASD_ERR_INVALID, "NULL argument");
    if (!c->has_state || !c->has_origin)
        return fail(ASD_ERR_STATE, "set the spins and the origin before S(q,t)");
    if (!(c->modes & (1u << ASD_SQT_FP64))) return fail(ASD_ERR_STATE, "the FP64 mode is not enabled");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    ASD_CUDA_TRY(launch_site_mean(c->y, c->M, c->p.nfile, c->uphase, c->mean_t, c->row4, c->row1,
                                  c->stream));
    c->rows_ready = true;
    const long tiles = dmma_sqt_tiles(c->M);
    if (tiles > 0x7fffffffL) return fail(ASD_ERR_UNSUPPORTED, "lattice too large for the FP64 GEMM");
    int rc = ensure_part(c, tiles);
    if (rc != ASD_OK) return rc;
    DmmaSqtArgs g = dmma_args(c, false);
    g.part = c->part;
    g.abs_sum = 1;
    if ((rc = launch_dmma_sqt(g, c->stream)) != ASD_OK) return rc;
    ASD_CUDA_TRY(launch_finalize(c->part, (int)tiles, 1.0 / (double)c->M, c->d_out, c->stream));
    c->last_launches = 3;
    ASD_CUDA_TRY(cudaMemcpyAsync(c->h_out, c->d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
    rc = read_status(c);  // synchronises
    if (rc != ASD_OK) return rc;
    *out = c->h_out[0];
    return ASD_OK;
}

int asd_ctx_sqt(asd_ctx *c, asd_sqt_mode mode, double out[2]) {
    if (!c || !out) return fail(ASD_ERR_INVALID, "NULL argument");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    int rc = sqt_async(c, (int)mode, c->d_out);
    if (rc != ASD_OK) return rc;
    ASD_CUDA_TRY(cudaMemcpyAsync(c->h_out, c->d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
    rc = read_status(c);  // synchronises
    if (rc != ASD_OK) return rc;
    out[0] = c->h_out[0];
    out[1] = c->h_out[1];
    return ASD_OK;
}

int asd_ctx_step_host(asd_ctx *c, const double *spin_in, double *spin_out, asd_sqt_mode mode,
                      double sqt_out[2]) {
    if (!c || !spin_in || !spin_out || !sqt_out) return fail(ASD_ERR_INVALID, "NULL argument");
    if (!c->has_origin) return fail(ASD_ERR_STATE, "set the origin (t = 0 spins) first");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    // Downloads of earlier asynchronous calls may still be writing the
    // caller's buffers, which this call may read: let them finish first.
    if (c->ast_events) ASD_CUDA_TRY(cudaStreamSynchronize(c->copy_stream));
    int rc;
    const int cr = host_chunk_replicas(c->p.nfile);
    if (cr < c->p.nfile) {
        rc = step_host_chunked(c, spin_in, spin_out, (int)mode, cr);
        // Never return while a copy may still touch the caller's buffers.
        const cudaError_t e1 = cudaStreamSynchronize(c->h2d_stream);
        const cudaError_t e2 = cudaStreamSynchronize(c->copy_stream);
        if (rc != ASD_OK) {
            cudaStreamSynchronize(c->stream);
            return rc;
        }
        ASD_CUDA_TRY(e1);
        ASD_CUDA_TRY(e2);
    } else {
        rc = set_spins_common(c, spin_in, true, 0);
        if (rc != ASD_OK) return rc;
        rc = run_steps(c, 1);
        if (rc != ASD_OK) return rc;
        // The new spins go back to the host on a second stream while S(q,t)
        // runs: the read-back over PCIe overlaps the correlation GEMM.
        if (!c->copy_stream) {
            ASD_CUDA_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
            ASD_CUDA_TRY(cudaEventCreateWithFlags(&c->spins_ready, cudaEventDisableTiming));
        }
        ASD_CUDA_TRY(launch_sitemajor_to_aos(c->y, c->ys_b, c->M, c->p.nfile, c->stream));
        c->last_launches += 1;
        ASD_CUDA_TRY(cudaEventRecord(c->spins_ready, c->stream));
        ASD_CUDA_TRY(cudaStreamWaitEvent(c->copy_stream, c->spins_ready, 0));
        ASD_CUDA_TRY(cudaMemcpyAsync(spin_out, c->ys_b, (size_t)c->M * c->K * sizeof(double),
                                     cudaMemcpyDeviceToHost, c->copy_stream));
        rc = sqt_async(c, (int)mode, c->d_out);
        const cudaError_t ec = cudaStreamSynchronize(c->copy_stream);
        if (rc != ASD_OK) return rc;
        ASD_CUDA_TRY(ec);
    }
    c->y_free_armed = false;  // the staging buffers were in use on the copy streams
    ASD_CUDA_TRY(cudaMemcpyAsync(c->h_out, c->d_out, 2 * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
    rc = read_status(c);
    if (rc != ASD_OK) return rc;
    sqt_out[0] = c->h_out[0];
    sqt_out[1] = c->h_out[1];
    return ASD_OK;
}

int asd_ctx_step_host_async(asd_ctx *c, const double *spin_in, double *spin_out,
                            asd_sqt_mode mode, double *sqt_out) {
    if (!c || !spin_in || !spin_out || !sqt_out) return fail(ASD_ERR_INVALID, "NULL argument");
    if (!c->has_origin) return fail(ASD_ERR_STATE, "set the origin (t = 0 spins) first");
    if ((int)mode < 0 || (int)mode > 3) return fail(ASD_ERR_INVALID, "unknown S(q,t) mode %d", (int)mode);
    if (!(c->modes & (1u << (int)mode)))
        return fail(ASD_ERR_STATE, "mode %d not enabled at create", (int)mode);
    ASD_CUDA_TRY(enter(c));
    if (!pinned_or_device(spin_in) || !pinned_or_device(spin_out) || !pinned_or_device(sqt_out))
        return fail(ASD_ERR_INVALID, "asd_ctx_step_host_async needs pinned host (cudaMallocHost, "
                                     "cudaHostRegister) or device buffers");
    c->last_launches = 0;
    return step_host_async(c, spin_in, spin_out, (int)mode, sqt_out);
}

int asd_ctx_synchronize(asd_ctx *c) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    ASD_CUDA_TRY(enter(c));
    if (c->h2d_stream) ASD_CUDA_TRY(cudaStreamSynchronize(c->h2d_stream));
    if (c->copy_stream) ASD_CUDA_TRY(cudaStreamSynchronize(c->copy_stream));
    return read_status(c);
}

int asd_ctx_set_ensemble(asd_ctx *c, int nfile_total) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    if (nfile_total < c->p.nfile)
        return fail(ASD_ERR_INVALID, "nfile_total=%d is below this shard's %d replicas", nfile_total,
                    c->p.nfile);
    c->nfile_total = nfile_total;
    c->has_zsums = false;
    return ASD_OK;
}

int asd_ctx_shard_origin_sums(asd_ctx *c, double *d_zsums) {
    if (!c || !d_zsums) return fail(ASD_ERR_INVALID, "NULL argument");
    if (!c->has_origin) return fail(ASD_ERR_STATE, "set the origin (t = 0 spins) first");
    ASD_CUDA_TRY(enter(c));
    ASD_CUDA_TRY(launch_site_sum(c->origin, c->M, c->p.nfile, d_zsums, c->stream));
    c->last_launches = 1;
    return ASD_OK;
}

int asd_ctx_shard_set_origin_sums(asd_ctx *c, const double *d_zsums) {
    if (!c || !d_zsums) return fail(ASD_ERR_INVALID, "NULL argument");
    ASD_CUDA_TRY(enter(c));
    if (!c->zsums) {
        int rc = dalloc(&c->zsums, (size_t)c->M * 3 * sizeof(double));
        if (rc != ASD_OK) return rc;
    }
    ASD_CUDA_TRY(cudaMemcpyAsync(c->zsums, d_zsums, (size_t)c->M * 3 * sizeof(double),
                                 cudaMemcpyDeviceToDevice, c->stream));
    c->has_zsums = true;
    return ASD_OK;
}

int asd_ctx_shard_sqt_async(asd_ctx *c, asd_sqt_mode mode, double *d_part, double *d_sums) {
    if (!c || !d_part || !d_sums) return fail(ASD_ERR_INVALID, "NULL argument");
    if (!c->has_state || !c->has_origin)
        return fail(ASD_ERR_STATE, "set the spins and the origin before S(q,t)");
    ASD_CUDA_TRY(enter(c));
    c->last_launches = 0;
    ASD_CUDA_TRY(launch_site_sum(c->y, c->M, c->p.nfile, d_sums, c->stream));
    c->last_launches += 1;
    return sqt_async(c, (int)mode, d_part, true);
}

int asd_ctx_shard_sqt_finish(asd_ctx *c, const double *d_part, const double *d_sums,
                             double *d_out) {
    if (!c || !d_part || !d_sums || !d_out) return fail(ASD_ERR_INVALID, "NULL argument");
    if (!c->has_zsums)
        return fail(ASD_ERR_STATE, "exchange the ensemble's origin sums first "
                                   "(asd_ctx_shard_set_origin_sums)");
    ASD_CUDA_TRY(enter(c));
    const int nft = c->nfile_total > 0 ? c->nfile_total : c->p.nfile;
    ASD_CUDA_TRY(launch_shard_finish(c->M, nft, d_part, d_sums, c->zsums, c->uphase, c->wphase,
                                     d_out, c->stream));
    c->last_launches = 1;
    return ASD_OK;
}

int asd_ctx_set_llg_kernel(asd_ctx *c, int kernel) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    if (kernel != ASD_LLG_FUSED_STEP && kernel != ASD_LLG_STAGES && kernel != ASD_LLG_AUTO)
        return fail(ASD_ERR_INVALID, "unknown LLG kernel %d", kernel);
    c->llg_kernel = kernel;
    return ASD_OK;
}

int asd_ctx_set_chunk_k(asd_ctx *c, int chunk_k) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    c->chunk_k = chunk_k < 0 ? -1 : chunk_k;
    return ASD_OK;
}

int asd_ctx_last_launches(const asd_ctx *c) { return c ? c->last_launches : 0; }

int asd_ctx_time_kernels(asd_ctx *c, int on) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    c->timing = (on != 0);
    return ASD_OK;
}

int asd_ctx_kernel_time(asd_ctx *c, int which, double *ms, int *launches) {
    if (!c || !ms || !launches) return fail(ASD_ERR_INVALID, "NULL argument");
    if (which != 0 && which != 1) return fail(ASD_ERR_INVALID, "which must be 0 or 1");
    ASD_CUDA_TRY(cudaSetDevice(c->device));
    double total = 0.0;
    int n = 0;
    std::vector<asd_ctx::Timed> keep;
    int rc = ASD_OK;
    for (auto &t : c->timed) {
        if (t.which != which) {
            keep.push_back(t);
            continue;
        }
        float dt = 0.f;
        cudaError_t e = cudaEventSynchronize(t.e);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&dt, t.b, t.e);
        if (e != cudaSuccess && rc == ASD_OK) rc = cuda_fail(e, "cudaEventElapsedTime");
        total += dt;
        n += t.launches;
        c->ev_pool.push_back(t.b);
        c->ev_pool.push_back(t.e);
    }
    c->timed.swap(keep);
    *ms = total;
    *launches = n;
    return rc;
}

int asd_ctx_check_device_status(asd_ctx *c) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    ASD_CUDA_TRY(enter(c));
    return read_status(c);
}

int asd_debug_fail_alloc(long n) {
    if (n < 0) return fail(ASD_ERR_INVALID, "n=%ld is negative", n);
    g_fail_in.store(n);
    return ASD_OK;
}

// Every device buffer of the context whose contents do not carry over from
// one call to the next: RK4 stage states and the running combination, the
// replica means at t, the GEMM partials and result, the q-grid diagonal
// partials, bins and result, the host-step staging and the adjoint's
// state-sized work buffers (checkpoints, recomputed states, adjoint
// variables).  Kept as they are: the spins, the origin and its means, the
// phases, the epilogue vectors and the split operands (their padding rows
// and columns are zeroed once at creation and stay zero).
int asd_ctx_debug_poison(asd_ctx *c) {
    if (!c) return fail(ASD_ERR_INVALID, "ctx is NULL");
    ASD_CUDA_TRY(enter(c));
    c->tape_valid = false;  // the checkpoints are among the poisoned buffers
    const cudaStream_t streams[] = {c->stream, c->llg_stream, c->gemm_stream, c->copy_stream,
                                    c->h2d_stream};
    for (cudaStream_t s : streams)
        if (s) ASD_CUDA_TRY(cudaStreamSynchronize(s));
    const size_t sb = (size_t)c->M * c->K * sizeof(double);
    const size_t chunk = (size_t)c->hp_replicas * c->M * 3 * sizeof(double);
    struct Buf {
        void *p;
        size_t n;
    };
    std::vector<Buf> bufs = {
        {c->ys_a, sb},
        {c->ys_b, sb},
        {c->acc, sb},
        {c->mean_t, (size_t)c->M * 3 * sizeof(double)},
        {c->grid_tdiag, c->grid_tdiag_n * sizeof(double)},
        {c->grid_ds, c->grid_ds_n * sizeof(double)},
        {c->part, (size_t)c->part_cap * sizeof(double2)},
        {c->d_out, 2 * sizeof(double)},
        {c->grid_g, (size_t)c->M * sizeof(double)},
        {c->grid_t, (size_t)c->M * sizeof(double2)},
        {c->grid_out, (size_t)c->M * 2 * sizeof(double)},
        {c->ast_in, sb},
        {c->ast_out, sb},
    };
    for (int b = 0; b < 2; ++b) {
        bufs.push_back({c->stage_in[b], chunk});
        bufs.push_back({c->stage_out[b], chunk});
    }
    for (long i = 0; i < c->adj_states && i < (long)c->adj_bufs.size(); ++i)
        bufs.push_back({c->adj_bufs[i], sb});
    for (const Buf &b : bufs)
        if (b.p && b.n) ASD_CUDA_TRY(cudaMemsetAsync(b.p, 0xFF, b.n, c->stream));
    ASD_CUDA_TRY(cudaStreamSynchronize(c->stream));
    return ASD_OK;
}

}  // extern "C"
