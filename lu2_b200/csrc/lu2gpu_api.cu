// lu2gpu_api.cu -- the C ABI of liblu2gpu.so: lu2's own entry points
// (lu2.c, lu2lib.h, lu2tlib.h, gdrdgemm.h) backed by the sm_100a kernels, and
// the handle-based device-resident API.  Declarations: include/lu2gpu.h.
//
// There is no CPU fallback anywhere: every failure is reported (status code,
// doneflag = 0, lu2gpu_last_error()) and, for the reference's void entry
// points, ends the process like the reference's MP_error (lu2_mp_nompi.c:55-58)
// unless lu2gpu_set_abort_on_error(0) was called.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/lu2gpu.h"
#include "lu2gpu_internal.cuh"

using namespace lu2gpu;

// ---------------------------------------------------------------------------
// errors

static thread_local char g_err[512] = "";
static int g_abort_on_error = 1;
static std::atomic<long> g_launches{0};

void lu2gpu::count_launch(long k) { g_launches += k; }

extern "C" long lu2gpu_kernel_launches(void) { return g_launches.load(); }

// LU2GPU_REPORT=1: print the number of kernel launches when the process exits
static void report_at_exit() { fprintf(stderr, "lu2gpu: %ld kernel launches\n", g_launches.load()); }

static void register_report()
{
    static std::once_flag once;
    std::call_once(once, [] {
        const char *e = getenv("LU2GPU_REPORT");
        if (e && e[0] == '1') atexit(report_at_exit);
    });
}

static void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

// for the reference's void entry points
static void fail_void(const char *where)
{
    fprintf(stderr, "lu2gpu: %s failed: %s\n", where, g_err);
    if (g_abort_on_error) exit(-1);
}

#define CU_TRY(expr)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            set_error("%s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return LU2GPU_ERR_CUDA;                                                         \
        }                                                                                   \
    } while (0)

// ---------------------------------------------------------------------------
// context

// phase 0 is the panel leaves, 5 the updates inside the panel recursion
enum { PH_LEAF = 0, PH_SWAP, PH_TRSM, PH_DGEMM, PH_BACKSOLVE, PH_PANEL, PH_COUNT };
static const char *g_phase_names[PH_COUNT] = {"col dec t",    "swaprows",    "solve tri",
                                              "DGEMMrest",    "backward_sub", "panel update"};

struct lu2gpu_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int *d_status = nullptr;
    double *d_bt = nullptr;
    size_t bt_cap = 0;  // doubles
    // transposed U blocks of the updates inside a panel, apart from d_bt so
    // that a panel can be factored while the previous step's update reads d_bt
    double *d_btp = nullptr;
    size_t btp_cap = 0;
    // lookahead of the FP64 factorization: the next panel on a high-priority stream
    cudaStream_t side = nullptr;
    cudaEvent_t ev_cols = nullptr, ev_panel = nullptr;
    // every buffer comes from fixed scratch (lu2gpu_lusolve_noalloc): nothing is allocated
    bool fixed_scratch = false;
    int *d_ipiv = nullptr;
    double *d_dinv = nullptr;
    size_t piv_cap = 0;
    LeafBuffers leaf{};
    unsigned long long leaf_seq = 0;  // leaf publication stamps issued so far
    int leaf_ctas = 0;
    int leaf_w = 16;
    // staging for the host-pointer entry points
    double *d_stage[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t stage_cap[4] = {0, 0, 0, 0};
    // copies of finished factor blocks to pinned host memory during the factorization
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_ev = nullptr;
    // host-to-device copies of column chunks of a pinned host matrix, one
    // event per chunk, overlapped with the left-looking start of the factorization
    cudaStream_t h2d_stream = nullptr;
    std::vector<cudaEvent_t> h2d_ev;
    std::vector<cudaEvent_t> blk_ev;  // blocks of the overlapped host-pointer DGEMM
    // phase timers
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev[PH_COUNT];
    double acc_ms[PH_COUNT] = {};
    long launches[PH_COUNT] = {};
    // workspaces of the precision form (lu2gpu_mixed_solve), allocated on first use
    struct MixedWork *mx = nullptr;
    // stamped x slots of the persistent back substitution (one per 64-row block)
    unsigned long long *d_bsx = nullptr;
    int bsx_cap = 0;
    unsigned bs_epoch = 0;
    BsBuffers bs{};
};

static void free_mixed(lu2gpu_ctx *c);

// the back substitution's x slots for an order-n system (null when they
// cannot be had: the blocked launches then do it)
static const BsBuffers *bs_buffers(lu2gpu_ctx *c, int n)
{
    if (c->fixed_scratch) return nullptr;
    const int need = (n + 63) / 64;
    if (need > c->bsx_cap) {
        cudaFree(c->d_bsx);
        c->d_bsx = nullptr;
        c->bsx_cap = 0;
        const int cap = need + 256;
        const size_t bytes = (size_t)cap * BS_SLOT_WORDS * sizeof(unsigned long long);
        if (cudaMalloc(&c->d_bsx, bytes) != cudaSuccess || cudaMemsetAsync(c->d_bsx, 0, bytes, c->stream) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(c->d_bsx);
            c->d_bsx = nullptr;
            return nullptr;
        }
        c->bsx_cap = cap;
    }
    c->bs.xslots = c->d_bsx;
    c->bs.cap = c->bsx_cap;
    c->bs.epoch = &c->bs_epoch;
    c->bs.status = c->d_status;
    return &c->bs;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

static int grow(void **p, size_t *cap, size_t bytes)
{
    if (*cap >= bytes && *p) return 0;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMalloc(p, bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc of %zu bytes failed", bytes);
        return LU2GPU_ERR_NOMEM;
    }
    *cap = bytes;
    return 0;
}

static int stage(lu2gpu_ctx *c, int slot, size_t doubles, double **out)
{
    size_t cap = c->stage_cap[slot];
    int rc = grow((void **)&c->d_stage[slot], &cap, doubles * sizeof(double) + 256);
    c->stage_cap[slot] = cap;
    *out = c->d_stage[slot];
    return rc;
}

extern "C" int lu2gpu_create(lu2gpu_ctx **out, int device)
{
    if (!out) {
        set_error("lu2gpu_create: null output pointer");
        return LU2GPU_ERR_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        cudaGetLastError();
        set_error("no CUDA device available");
        return LU2GPU_ERR_NODEV;
    }
    if (device < 0 || device >= ndev) {
        set_error("device %d out of range (%d devices)", device, ndev);
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(device);
    cudaDeviceProp prop;
    CU_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a only", device, prop.major, prop.minor);
        return LU2GPU_ERR_NODEV;
    }
    register_report();
    lu2gpu_ctx *c = new lu2gpu_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete c;
        set_error("cudaStreamCreate failed");
        return LU2GPU_ERR_CUDA;
    }
    c->own_stream = true;
    c->leaf_ctas = leaf_max_ctas(device);
    const int G = c->leaf_ctas;
    // the leaf may use fewer CTAs than fit (fewer participants per column
    // exchange, more rows each): LU2GPU_LEAF_CTAS caps it
    if (const char *e = getenv("LU2GPU_LEAF_CTAS")) {
        const int cap = atoi(e);
        if (cap >= 1 && cap < c->leaf_ctas) c->leaf_ctas = cap;
    }
    size_t leaf_bytes = (size_t)2 * G * sizeof(LeafSlot);
    char *lb = nullptr;
    if (cudaMalloc(&c->d_status, 4 * sizeof(int)) != cudaSuccess || cudaMalloc(&lb, leaf_bytes) != cudaSuccess ||
        cudaMemset(lb, 0, leaf_bytes) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc of the context buffers failed");
        lu2gpu_destroy(c);
        return LU2GPU_ERR_NOMEM;
    }
    c->leaf.slots = (LeafSlot *)lb;
    c->leaf.seq = &c->leaf_seq;
    *out = c;
    return 0;
}

extern "C" int lu2gpu_destroy(lu2gpu_ctx *c)
{
    if (!c) return 0;
    DeviceGuard g(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_status);
    cudaFree(c->leaf.slots);
    cudaFree(c->d_bt);
    cudaFree(c->d_btp);
    if (c->side) {
        cudaStreamSynchronize(c->side);
        cudaStreamDestroy(c->side);
    }
    if (c->ev_cols) cudaEventDestroy(c->ev_cols);
    if (c->ev_panel) cudaEventDestroy(c->ev_panel);
    cudaFree(c->d_ipiv);
    cudaFree(c->d_dinv);
    cudaFree(c->d_bsx);
    for (int i = 0; i < 4; i++) cudaFree(c->d_stage[i]);
    if (c->copy_stream) {
        cudaStreamSynchronize(c->copy_stream);
        cudaStreamDestroy(c->copy_stream);
    }
    if (c->copy_ev) cudaEventDestroy(c->copy_ev);
    if (c->h2d_stream) {
        cudaStreamSynchronize(c->h2d_stream);
        cudaStreamDestroy(c->h2d_stream);
    }
    for (cudaEvent_t e : c->h2d_ev) cudaEventDestroy(e);
    for (cudaEvent_t e : c->blk_ev) cudaEventDestroy(e);
    free_mixed(c);
    for (int p = 0; p < PH_COUNT; p++)
        for (auto &e : c->ev[p]) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return 0;
}

extern "C" int lu2gpu_set_stream(lu2gpu_ctx *c, void *stream)
{
    if (!c) {
        set_error("null context");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    c->stream = (cudaStream_t)stream;
    c->own_stream = false;
    return 0;
}

extern "C" const char *lu2gpu_last_error(void) { return g_err; }

extern "C" int lu2gpu_test_leaf_withhold(lu2gpu_ctx *c, int cta, double wait_ms)
{
    if (!c || !(wait_ms >= 0.0) || wait_ms > 2000.0) {
        set_error("lu2gpu_test_leaf_withhold: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    c->leaf.withhold = cta >= 0 ? cta : -1;
    c->leaf.wait_ns = wait_ms > 0.0 ? (unsigned long long)(wait_ms * 1e6) : WAIT_LIMIT_NS;
    return 0;
}

extern "C" int lu2gpu_set_abort_on_error(int on)
{
    int old = g_abort_on_error;
    g_abort_on_error = on ? 1 : 0;
    return old;
}

// ---------------------------------------------------------------------------
// phase timers (the CUDA-event counterpart of lu2's timerlib accumulators)

struct PhaseTimer {
    lu2gpu_ctx *c;
    int ph;
    cudaEvent_t e1 = nullptr;
    PhaseTimer(lu2gpu_ctx *ctx, int phase) : c(ctx), ph(phase)
    {
        if (!c->timing) return;
        cudaEvent_t e0;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, c->stream);
        c->ev[ph].push_back({e0, e1});
    }
    ~PhaseTimer()
    {
        if (c->timing) cudaEventRecord(e1, c->stream);
    }
};

static void collect_timers(lu2gpu_ctx *c)
{
    for (int p = 0; p < PH_COUNT; p++) {
        for (auto &e : c->ev[p]) {
            float ms = 0;
            cudaEventSynchronize(e.second);
            if (cudaEventElapsedTime(&ms, e.first, e.second) == cudaSuccess) c->acc_ms[p] += ms;
            c->launches[p]++;
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        c->ev[p].clear();
    }
}

extern "C" int lu2gpu_set_timing(lu2gpu_ctx *c, int enable)
{
    if (!c) return LU2GPU_ERR_ARG;
    c->timing = enable != 0;
    return 0;
}

extern "C" int lu2gpu_get_timers(lu2gpu_ctx *c, double *ms, long *counts, int nmax, int reset)
{
    if (!c) return LU2GPU_ERR_ARG;
    DeviceGuard g(c->device);
    collect_timers(c);
    for (int p = 0; p < PH_COUNT && p < nmax; p++) {
        if (ms) ms[p] = c->acc_ms[p];
        if (counts) counts[p] = c->launches[p];
    }
    if (reset)
        for (int p = 0; p < PH_COUNT; p++) {
            c->acc_ms[p] = 0;
            c->launches[p] = 0;
        }
    return PH_COUNT;
}

extern "C" const char *lu2gpu_timer_name(int phase)
{
    return (phase >= 0 && phase < PH_COUNT) ? g_phase_names[phase] : "";
}

// ---------------------------------------------------------------------------
// status

static int begin_status(lu2gpu_ctx *c)
{
    CU_TRY(cudaMemsetAsync(c->d_status, 0x7f, sizeof(int), c->stream));
    CU_TRY(cudaMemsetAsync(c->d_status + 1, 0, 3 * sizeof(int), c->stream));
    return 0;
}

// synchronize and translate the device status; >0 = first zero pivot column + 1
static int end_status(lu2gpu_ctx *c, const char *what)
{
    CU_TRY(cudaStreamSynchronize(c->stream));
    int st[4];
    CU_TRY(cudaMemcpy(st, c->d_status, sizeof(st), cudaMemcpyDeviceToHost));
    if (st[1] != 0) {
        if (st[1] == ERR_BAD_ARG) {
            set_error("%s: a pivot index outside [k, n) was refused on the device (kernel %d)", what, st[2]);
            return LU2GPU_ERR_ARG;
        }
        set_error("%s: a bounded device wait gave up (error bits 0x%x, kernel %d)", what, st[1], st[2]);
        return LU2GPU_ERR_TIMEOUT;
    }
    if (st[0] != INFO_NONE) {
        set_error("%s: zero pivot at column %d", what, st[0] - 1);
        return st[0];
    }
    return 0;
}

// ---------------------------------------------------------------------------
// factorization driver.  A view is the trailing part of a matrix whose element
// (0,0) is global (goff, goff); `n` rows, `ncols` columns (incl. right-hand sides).

struct View {
    double *a;
    long ld;
    int n, ncols, goff;
};

#define K_TRY(expr)                                                                                   \
    do {                                                                                              \
        cudaError_t e_ = (expr);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            set_error("kernel launch %s: %s (%s:%d)", #expr, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return LU2GPU_ERR_CUDA;                                                                   \
        }                                                                                             \
    } while (0)

// Pivots of view columns k0..k1 applied to columns cs..ce, then U rows solved
// and the rows below updated (lu2.c:524-581 / lu2tlib.c:1068-1093).
static int right_part(lu2gpu_ctx *c, const View &v, int k0, int k1, int cs, int ce, bool top)
{
    if (ce <= cs) return 0;
    int *ipiv = c->d_ipiv + v.goff;
    double *dinv = c->d_dinv + v.goff;
    const int K = k1 - k0;
    {
        PhaseTimer t(c, top ? PH_SWAP : PH_PANEL);
        K_TRY(launch_laswp_scale(v.a, v.ld, v.n, k0, k1, ipiv, v.goff, dinv, cs, ce, true, c->d_status, c->stream));
    }
    // inner right parts of a panel (K x (ce - cs) <= nb^2 / 4) use their own
    // buffer, so that a panel factored beside a running update (which reads
    // d_bt) never writes d_bt; wider blocks go to d_bt
    const size_t bt_bytes = (size_t)(ce - cs) * K * sizeof(double);
    double *bt = (!top && c->d_btp && bt_bytes <= c->btp_cap) ? c->d_btp : c->d_bt;
    if (bt == c->d_bt && bt_bytes > c->bt_cap) {
        set_error("right part: transposed U block of %zu bytes exceeds its %zu-byte buffer", bt_bytes, c->bt_cap);
        return LU2GPU_ERR_ARG;
    }
    {
        PhaseTimer t(c, top ? PH_TRSM : PH_PANEL);
        K_TRY(launch_trsm_unit_lower(v.a, v.ld, k0, K, cs, ce, bt, c->stream));
    }
    if (k1 < v.n) {
        PhaseTimer t(c, top ? PH_DGEMM : PH_PANEL);
        K_TRY(launch_dgemm_update(v.a, v.ld, v.n, k1, k0, bt, v.a + (size_t)k1 * v.ld + cs, v.ld, v.n - k1,
                                  ce - cs, K, c->d_status, c->stream));
    }
    return 0;
}

// right_part (top level, no phase timers) with the update's columns split at
// cs + w1: `hook` runs between the update of columns cs..cs+w1-1 and that of
// the rest (the lookahead factors the next panel there)
template <typename Hook>
static int right_part_split(lu2gpu_ctx *c, const View &v, int k0, int k1, int cs, int ce, int w1, Hook hook)
{
    if (ce <= cs) return hook();
    const int K = k1 - k0;
    K_TRY(launch_laswp_scale(v.a, v.ld, v.n, k0, k1, c->d_ipiv + v.goff, v.goff, c->d_dinv + v.goff, cs, ce, true,
                             c->d_status, c->stream));
    K_TRY(launch_trsm_unit_lower(v.a, v.ld, k0, K, cs, ce, c->d_bt, c->stream));
    if (k1 >= v.n) return hook();
    if (w1 > ce - cs) w1 = ce - cs;
    double *C = v.a + (size_t)k1 * v.ld + cs;
    K_TRY(launch_dgemm_update(v.a, v.ld, v.n, k1, k0, c->d_bt, C, v.ld, v.n - k1, w1, K, c->d_status, c->stream));
    const int rc = hook();
    if (rc) return rc;
    if (w1 < ce - cs)
        K_TRY(launch_dgemm_update(v.a, v.ld, v.n, k1, k0, c->d_bt + (size_t)w1 * K, C + w1, v.ld, v.n - k1,
                                  ce - cs - w1, K, c->d_status, c->stream));
    return 0;
}

// Recursive panel (lu2.c:1088-1120): columns c0..c0+m-1, rows c0..n-1.  The
// split keeps every left width a multiple of 16 (the GEMM's K step).
static int panel(lu2gpu_ctx *c, const View &v, int c0, int m, int mode)
{
    if (m <= c->leaf_w) {
        PhaseTimer t(c, PH_LEAF);
        K_TRY(launch_leaf(v.a, v.ld, v.n, c0, m, mode, v.goff, c->d_ipiv + v.goff, c->d_dinv + v.goff, c->leaf,
                          c->d_status, c->leaf_ctas, c->stream));
        return 0;
    }
    int h = ((m / 2) + 15) & ~15;
    if (h >= m) h = m - 16;
    int rc = panel(c, v, c0, h, mode);
    if (rc) return rc;
    rc = right_part(c, v, c0, c0 + h, c0 + h, c0 + m, false);
    if (rc) return rc;
    rc = panel(c, v, c0 + h, m - h, mode);
    if (rc) return rc;
    PhaseTimer t(c, PH_PANEL);
    K_TRY(launch_laswp_scale(v.a, v.ld, v.n, c0 + h, c0 + m, c->d_ipiv + v.goff, v.goff, c->d_dinv + v.goff, c0,
                             c0 + h, true, c->d_status, c->stream));
    return 0;
}

static int ensure_work(lu2gpu_ctx *c, int n, int ncols, int nb)
{
    size_t need_bt = (size_t)ncols * (size_t)nb + 1024;
    if (c->fixed_scratch) {  // lu2gpu_lusolve_noalloc: its buffers are fixed, never grown
        if (need_bt * sizeof(double) > c->bt_cap || (size_t)n > c->piv_cap) {
            set_error("fixed scratch too small for n=%d, %d columns, nb=%d", n, ncols, nb);
            return LU2GPU_ERR_ARG;
        }
        return 0;
    }
    int rc = grow((void **)&c->d_bt, &c->bt_cap, need_bt * sizeof(double));
    if (rc) return rc;
    if ((rc = grow((void **)&c->d_btp, &c->btp_cap, ((size_t)nb * nb + 1024) * sizeof(double)))) return rc;
    if (c->piv_cap < (size_t)n) {
        cudaFree(c->d_ipiv);
        cudaFree(c->d_dinv);
        c->d_ipiv = nullptr;
        c->d_dinv = nullptr;
        c->piv_cap = 0;
        if (cudaMalloc(&c->d_ipiv, (size_t)n * sizeof(int)) != cudaSuccess ||
            cudaMalloc(&c->d_dinv, (size_t)n * sizeof(double)) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc of pivot arrays failed");
            return LU2GPU_ERR_NOMEM;
        }
        c->piv_cap = n;
    }
    return 0;
}

static int check_matrix_args(int n, int nrhs, const double *a, long lda, int nb)
{
    if (n <= 0 || nrhs < 0 || !a || lda < (long)n + nrhs) {
        set_error("bad matrix arguments (n=%d nrhs=%d lda=%ld)", n, nrhs, lda);
        return LU2GPU_ERR_ARG;
    }
    if (nb < 16 || (nb % 16) != 0) {
        set_error("block size nb=%d must be a positive multiple of 16", nb);
        return LU2GPU_ERR_ARG;
    }
    if ((lda & 1) || (reinterpret_cast<uintptr_t>(a) & 15)) {
        set_error("device matrix must be 16-byte aligned with an even row stride (lda=%ld)", lda);
        return LU2GPU_ERR_ARG;
    }
    return 0;
}

// Factor (lumcolumn's panel loop, lu2.c:1126-1141) of the n x (n+nrhs)
// augmented device matrix; the right-hand sides are forward-transformed on the
// way (y).  Pivots go to ctx->d_ipiv (and to ipiv_out if given, device).
// Panels wider than 512 columns are factored as 512-wide panels: the pivot
// sequence does not depend on the panel width, and the in-shared-memory U
// block-row solve holds at most 512 rows.
constexpr int NB_MAX = 512;

// The panel width the GPU uses for a caller's block size m: a multiple of 16
// in [16, NB_MAX] (lu2 callers pass powers of two, e.g. 8 or 2048).
static int gpu_panel_width(int m)
{
    int w = (m / 16) * 16;
    if (w < 16) w = 16;
    if (w > NB_MAX) w = NB_MAX;
    return w;
}

// Lookahead of the FP64 factorization (the reference's lu_mpi_blocked_lookahead
// idea, lu2_mpi.c:3643-3847, on one GPU): step k updates the next panel's
// columns first, then that panel is factored on a high-priority stream while
// the rest of step k's update runs; step k+1's right part waits for it (its
// row exchanges cross the columns the update wrote).  The panel's own updates
// use their own transposed-U buffer (d_btp).  Every element sees the same
// operations in the same order as in the serial schedule: bit-identical.
// Serial when phase timing is on (the phase split stays meaningful), for
// fewer than four panels, on fixed scratch, or with LU2GPU_LOOKAHEAD=0.
//
// A panel factored beside the update holds its leaf to LOOKAHEAD_LEAF_CTAS
// CTAs (more if its slab needs them): each leaf CTA takes the place of one of
// the update's two CTAs on an SM, and the leaf is bound by its per-column
// exchange, not its CTA count.  Measured at N=65536 (TFLOP/s, leaf capped
// everywhere): 148 CTAs 30.36, 96 30.78, 64 31.03, 48 31.02.
constexpr int LOOKAHEAD_LEAF_CTAS = 64;

static bool use_lookahead(const lu2gpu_ctx *c, int rows, int nb)
{
    const char *env = getenv("LU2GPU_LOOKAHEAD");
    return !c->timing && !c->fixed_scratch && c->d_btp && rows >= 4 * nb && !(env && env[0] == '0');
}

template <typename AfterStep>
static int factor_lookahead(lu2gpu_ctx *c, const View &v, int i0, int nb, int mode, AfterStep after_step)
{
    const int n = v.n;
    if (!c->side) {
        int least = 0, greatest = 0;
        CU_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        CU_TRY(cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, greatest));
        CU_TRY(cudaEventCreateWithFlags(&c->ev_cols, cudaEventDisableTiming));
        CU_TRY(cudaEventCreateWithFlags(&c->ev_panel, cudaEventDisableTiming));
    }
    const cudaStream_t main_st = c->stream;
    const int all_ctas = c->leaf_ctas;
    int rc = panel(c, v, i0, std::min(nb, n - i0), mode);  // the first panel, on the main stream
    for (int i = i0; rc == 0 && i < n; i += nb) {
        const int w = std::min(nb, n - i), i1 = i + w, w1 = std::min(nb, n - i1);
        if (i > i0 && cudaStreamWaitEvent(main_st, c->ev_panel, 0) != cudaSuccess) {
            set_error("lookahead: cudaStreamWaitEvent failed");
            rc = LU2GPU_ERR_CUDA;
            break;
        }
        auto next_panel = [&]() -> int {
            if (i1 >= n) return 0;
            CU_TRY(cudaEventRecord(c->ev_cols, main_st));
            CU_TRY(cudaStreamWaitEvent(c->side, c->ev_cols, 0));
            c->stream = c->side;
            c->leaf_ctas = std::min(all_ctas, std::max(LOOKAHEAD_LEAF_CTAS, leaf_min_ctas(n - i1, sizeof(double))));
            const int r = panel(c, v, i1, w1, mode);
            c->stream = main_st;
            c->leaf_ctas = all_ctas;
            if (r) return r;
            CU_TRY(cudaEventRecord(c->ev_panel, c->side));
            return 0;
        };
        rc = right_part_split(c, v, i, i1, i1, v.ncols, w1, next_panel);
        if (!rc) rc = after_step(i, w);
    }
    c->stream = main_st;
    c->leaf_ctas = all_ctas;
    // everything on the panel stream precedes what follows on the main stream
    if (cudaEventRecord(c->ev_panel, c->side) != cudaSuccess ||
        cudaStreamWaitEvent(main_st, c->ev_panel, 0) != cudaSuccess) {
        cudaGetLastError();
        if (!rc) {
            set_error("lookahead: joining the panel stream failed");
            rc = LU2GPU_ERR_CUDA;
        }
    }
    return rc;
}

// `after_step(i, w)`, if given, runs once the enqueue of panel step i..i+w-1
// is complete (rows i..i+w-1 from column i, and columns i..i+w-1 below them,
// hold their final values once that work has executed: later steps touch
// neither, lu2.c:543-553).
//
// `wait_cols(ce)` makes the compute stream wait until columns 0..ce-1 of the
// matrix are on the device.  While they arrive, the first `p0` panels are
// factored left-looking: panel p's columns receive the updates of panels
// 0..p-1 (the same row exchanges, U-block solve and GEMM per element, in the
// same panel order, as the right-looking steps apply to them) and are
// factored; the columns right of panel p0 then catch up in arrival order,
// `group` columns at a time, and the right-looking loop continues from panel
// p0.  Factors and pivots are bit-identical to the right-looking schedule.
template <typename AfterStep, typename WaitCols>
static int factor_enqueue_arriving(lu2gpu_ctx *c, int n, int nrhs, double *a, long lda, int nb, int mode, int p0,
                                   int group, AfterStep after_step, WaitCols wait_cols)
{
    if (nb > NB_MAX) nb = NB_MAX;
    int rc = ensure_work(c, n, n + nrhs, nb);
    if (rc) return rc;
    View v{a, lda, n, n + nrhs, 0};
    const int ncol = n + nrhs;
    int i0 = 0;  // columns 0..i0-1 factored left-looking
    for (int p = 0; p < p0 && i0 < n; ++p) {
        const int w = (n - i0) < nb ? (n - i0) : nb;
        if ((rc = wait_cols(i0 + w))) return rc;
        for (int k = 0; k < i0; k += nb)
            if ((rc = right_part(c, v, k, k + nb, i0, i0 + w, true))) return rc;
        if ((rc = panel(c, v, i0, w, mode))) return rc;
        i0 += w;
    }
    if (i0 > 0) {
        if (group < nb) group = nb;
        for (int cs = i0; cs < ncol; cs += group) {
            const int ce = (ncol - cs) < group ? ncol : cs + group;
            if ((rc = wait_cols(ce))) return rc;
            for (int k = 0; k < i0; k += nb)
                if ((rc = right_part(c, v, k, (i0 - k) < nb ? i0 : k + nb, cs, ce, true))) return rc;
        }
        for (int k = 0; k < i0; k += nb)
            if ((rc = after_step(k, (i0 - k) < nb ? i0 - k : nb))) return rc;
    }
    if ((rc = wait_cols(ncol))) return rc;
    if (i0 < n && use_lookahead(c, n - i0, nb)) return factor_lookahead(c, v, i0, nb, mode, after_step);
    for (int i = i0; i < n; i += nb) {
        const int w = (n - i) < nb ? (n - i) : nb;
        rc = panel(c, v, i, w, mode);
        if (rc) return rc;
        rc = right_part(c, v, i, i + w, i + w, n + nrhs, true);
        if (rc) return rc;
        if ((rc = after_step(i, w))) return rc;
    }
    return 0;
}

template <typename AfterStep>
static int factor_enqueue_with(lu2gpu_ctx *c, int n, int nrhs, double *a, long lda, int nb, int mode,
                               AfterStep after_step)
{
    return factor_enqueue_arriving(c, n, nrhs, a, lda, nb, mode, 0, 0, after_step, [](int) { return 0; });
}

static int factor_enqueue(lu2gpu_ctx *c, int n, int nrhs, double *a, long lda, int nb, int mode)
{
    return factor_enqueue_with(c, n, nrhs, a, lda, nb, mode, [](int, int) { return 0; });
}

extern "C" int lu2gpu_factor(lu2gpu_ctx *c, int n, int nrhs, double *a, long lda, int nb, int pivot_mode, int *ipiv)
{
    if (!c) {
        set_error("null context");
        return LU2GPU_ERR_ARG;
    }
    int rc = check_matrix_args(n, nrhs, a, lda, nb);
    if (rc) return rc;
    if (pivot_mode != LU2GPU_PIVOT_REF && pivot_mode != LU2GPU_PIVOT_PARTIAL) {
        set_error("unknown pivot mode %d", pivot_mode);
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    rc = begin_status(c);
    if (rc) return rc;
    rc = factor_enqueue(c, n, nrhs, a, lda, nb, pivot_mode);
    if (rc) return rc;
    if (ipiv) CU_TRY(cudaMemcpyAsync(ipiv, c->d_ipiv, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    return end_status(c, "lu2gpu_factor");
}

extern "C" int lu2gpu_backsolve(lu2gpu_ctx *c, int n, int nrhs, const double *a, long lda, double *x, long ldx)
{
    if (!c || n <= 0 || nrhs <= 0 || !a || !x || lda < n || ldx < nrhs) {
        set_error("lu2gpu_backsolve: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    int rc = begin_status(c);
    if (rc) return rc;
    {
        PhaseTimer t(c, PH_BACKSOLVE);
        K_TRY(launch_backsolve(a, lda, n, nrhs, x, ldx, bs_buffers(c, n), c->stream));
    }
    return end_status(c, "lu2gpu_backsolve");
}

extern "C" int lu2gpu_lusolve(lu2gpu_ctx *c, int n, int nrhs, double *a, long lda, int nb, int pivot_mode, int *ipiv)
{
    if (!c) {
        set_error("null context");
        return LU2GPU_ERR_ARG;
    }
    if (nrhs < 1) {
        set_error("lu2gpu_lusolve needs at least one right-hand side");
        return LU2GPU_ERR_ARG;
    }
    int rc = check_matrix_args(n, nrhs, a, lda, nb);
    if (rc) return rc;
    if (pivot_mode != LU2GPU_PIVOT_REF && pivot_mode != LU2GPU_PIVOT_PARTIAL) {
        set_error("unknown pivot mode %d", pivot_mode);
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    rc = begin_status(c);
    if (rc) return rc;
    rc = factor_enqueue(c, n, nrhs, a, lda, nb, pivot_mode);
    if (rc) return rc;
    {
        PhaseTimer t(c, PH_BACKSOLVE);
        K_TRY(launch_backsolve(a, lda, n, nrhs, a + n, lda, bs_buffers(c, n), c->stream));
    }
    if (ipiv) CU_TRY(cudaMemcpyAsync(ipiv, c->d_ipiv, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    return end_status(c, "lu2gpu_lusolve");
}

// Solve with the factors of an earlier lu2gpu_factor: per panel of width nb
// (the factorization's, so that the panel's L columns are read in the row
// order they were stored in), the panel's pivots with the 1/pivot scaling, the
// unit-lower solve and the update of the rows below -- what the factorization
// does to its augmented columns (lu2.c:524-581) -- then the back substitution
// (lu2.c:110-116).  b (n x nrhs, row stride ldb) is overwritten by x.
extern "C" int lu2gpu_solve(lu2gpu_ctx *c, int n, const double *a, long lda, int nb, const int *ipiv, double *b,
                            long ldb, int nrhs)
{
    if (!c || n <= 0 || !a || lda < n || !ipiv || !b || nrhs < 1 || ldb < nrhs) {
        set_error("lu2gpu_solve: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    int rc = check_matrix_args(n, 0, a, lda, nb);
    if (rc) return rc;
    if (nb > NB_MAX) nb = NB_MAX;
    DeviceGuard g(c->device);
    if ((rc = ensure_work(c, n, nrhs, nb))) return rc;
    if ((rc = begin_status(c))) return rc;
    K_TRY(launch_diag_inv(a, lda, n, c->d_dinv, c->stream));
    for (int i = 0; i < n; i += nb) {
        const int w = (n - i) < nb ? (n - i) : nb;
        K_TRY(launch_laswp_scale(b, ldb, n, i, i + w, ipiv, 0, c->d_dinv, 0, nrhs, true, c->d_status, c->stream));
        K_TRY(launch_trsm_unit_lower_tx(a + (size_t)i * lda + i, lda, b + (size_t)i * ldb, ldb, w, nrhs, c->d_bt,
                                        c->stream));
        if (i + w < n)
            K_TRY(launch_dgemm_update(a, lda, n, i + w, i, c->d_bt, b + (size_t)(i + w) * ldb, ldb, n - i - w, nrhs,
                                      w, c->d_status, c->stream));
    }
    {
        PhaseTimer t(c, PH_BACKSOLVE);
        K_TRY(launch_backsolve(a, lda, n, nrhs, b, ldb, bs_buffers(c, n), c->stream));
    }
    return end_status(c, "lu2gpu_solve");
}

extern "C" int lu2gpu_generate(lu2gpu_ctx *c, int n, int nrhs, long seed, int kind, double *a, long lda)
{
    if (!c || n <= 0 || nrhs < 0 || !a || lda < (long)n + (nrhs > 0 ? nrhs : 1) || kind < 0 || kind > 1) {
        set_error("lu2gpu_generate: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    K_TRY(launch_generate(a, lda, n, nrhs > 0 ? nrhs : 1, seed, kind, c->stream));
    CU_TRY(cudaStreamSynchronize(c->stream));
    return 0;
}

// C = alpha * A * B + beta * C, row-major device matrices (mydgemm's contract
// on device pointers).  B is transposed into a staging buffer first.
extern "C" int lu2gpu_dgemm_dev(lu2gpu_ctx *c, int m, int n, int k, double alpha, const double *a, long lda,
                                const double *b, long ldb, double beta, double *cm, long ldc)
{
    if (!c || m < 0 || n < 0 || k < 0) {
        set_error("lu2gpu_dgemm_dev: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    if (m == 0 || n == 0) return 0;
    DeviceGuard g(c->device);
    int rc = begin_status(c);
    if (rc) return rc;
    const int kk = k > 0 ? k : 1;
    const long ldy = (kk + 1) & ~1L;
    const long ldx = ldy;
    double *y, *x;
    if ((rc = stage(c, 0, (size_t)n * ldy, &y))) return rc;
    if ((rc = stage(c, 1, (size_t)m * ldx, &x))) return rc;
    if (k == 0) {
        CU_TRY(cudaMemsetAsync(y, 0, (size_t)n * ldy * sizeof(double), c->stream));
        CU_TRY(cudaMemsetAsync(x, 0, (size_t)m * ldx * sizeof(double), c->stream));
    } else {
        K_TRY(launch_transpose(b, ldb, y, ldy, k, n, c->stream));
        CU_TRY(cudaMemcpy2DAsync(x, ldx * sizeof(double), a, lda * sizeof(double), (size_t)k * sizeof(double), m,
                                 cudaMemcpyDeviceToDevice, c->stream));
    }
    K_TRY(launch_dgemm_general(x, ldx, y, ldy, cm, ldc, m, n, kk, alpha, beta, c->d_status, c->stream));
    return end_status(c, "lu2gpu_dgemm_dev");
}

// lu2.c:485-521 on device memory
extern "C" int lu2gpu_solve_triangle_dev(lu2gpu_ctx *c, int K, const double *t, long ldt, double *x, long ldx,
                                         int ncols, double *bt)
{
    if (!c || K <= 0 || K > NB_MAX || !t || ldt < K || !x || ncols < 0 || (ncols > 0 && ldx < ncols)) {
        set_error("lu2gpu_solve_triangle_dev: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    if (ncols == 0) return 0;
    DeviceGuard g(c->device);
    int rc = begin_status(c);
    if (rc) return rc;
    K_TRY(launch_trsm_unit_lower_tx(t, ldt, x, ldx, K, ncols, bt, c->stream));
    return end_status(c, "lu2gpu_solve_triangle_dev");
}

// lu2.c:251-291 over a panel's pivots, as lu2.c:541-554 applies them
extern "C" int lu2gpu_swaprows_dev(lu2gpu_ctx *c, int n, double *a, long lda, int k0, int k1, const int *ipiv,
                                   const double *dinv, int cs, int ce)
{
    if (!c || n <= 0 || !a || !ipiv || k0 < 0 || k1 < k0 || k1 > n || k1 - k0 > 512 || cs < 0 || ce < cs ||
        lda < ce) {
        set_error("lu2gpu_swaprows_dev: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    if (k1 == k0 || ce == cs) return 0;
    DeviceGuard g(c->device);
    int rc = begin_status(c);
    if (rc) return rc;
    K_TRY(launch_laswp_scale(a, lda, n, k0, k1, ipiv, 0, dinv, cs, ce, dinv != nullptr, c->d_status, c->stream));
    return end_status(c, "lu2gpu_swaprows_dev");
}

// ---------------------------------------------------------------------------
// the default context behind the reference-signature entry points

static std::mutex g_mu;
static lu2gpu_ctx *g_ctx = nullptr;
static int g_board = 0;
static int g_pivot_mode = LU2GPU_PIVOT_PARTIAL;
static int g_gdr_ok = 0;

static lu2gpu_ctx *default_ctx()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ctx) {
        const char *pm = getenv("LU2GPU_PIVOT");
        if (pm && (!strcmp(pm, "ref") || !strcmp(pm, "REF"))) g_pivot_mode = LU2GPU_PIVOT_REF;
        if (lu2gpu_create(&g_ctx, g_board) != 0) g_ctx = nullptr;
    }
    return g_ctx;
}

extern "C" int lu2gpu_set_pivot_mode(int mode)
{
    if (mode != LU2GPU_PIVOT_REF && mode != LU2GPU_PIVOT_PARTIAL) {
        set_error("unknown pivot mode %d", mode);
        return LU2GPU_ERR_ARG;
    }
    int old = g_pivot_mode;
    g_pivot_mode = mode;
    return old;
}

extern "C" lu2gpu_ctx *lu2gpu_default_context(void) { return default_ctx(); }

extern "C" int lu2gpu_release(void)
{
    std::lock_guard<std::mutex> lk(g_mu);
    lu2gpu_destroy(g_ctx);
    g_ctx = nullptr;
    g_gdr_ok = 0;
    return 0;
}

// Host-pointer column-major DGEMM, the contract of the board library's
// gdr_dgemm_ (gdrdgemm.c:105-110, 185-186): C = alpha op(A) op(B) + beta C,
// nota/notb = 1 for no transpose.  Computed as the row-major C^T = op(B)^T op(A)^T.
static int host_dgemm_colmajor_overlap(lu2gpu_ctx *c, int nota, int notb, int m, int n, int k, double alpha,
                                       const double *A, int lda, const double *B, int ldb, double beta, double *C,
                                       int ldc, int jb);

static int host_dgemm_colmajor(int nota, int notb, int m, int n, int k, double alpha, const double *A, int lda,
                               const double *B, int ldb, double beta, double *C, int ldc)
{
    lu2gpu_ctx *c = default_ctx();
    if (!c) return LU2GPU_ERR_NODEV;
    if (m < 0 || n < 0 || k < 0 || !C || ldc < (m > 1 ? m : 1)) {
        set_error("gdr_dgemm_: bad sizes m=%d n=%d k=%d ldc=%d", m, n, k, ldc);
        return LU2GPU_ERR_ARG;
    }
    if (m == 0 || n == 0) return 0;
    DeviceGuard g(c->device);
    if (k > 0 && A && B) {
        // C in pinned host memory and at least two blocks of ~16 MB: overlapped
        cudaPointerAttributes pa{};
        const bool pinned = cudaPointerGetAttributes(&pa, C) == cudaSuccess && pa.type == cudaMemoryTypeHost;
        cudaGetLastError();
        const char *ov = getenv("LU2GPU_DGEMM_OVERLAP");
        long jb = (16L << 20) / ((long)m * (long)sizeof(double));
        if (jb < 16) jb = 16;
        if (pinned && !(ov && atoi(ov) == 0) && 2 * jb <= n)
            return host_dgemm_colmajor_overlap(c, nota, notb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, (int)jb);
    }
    int rc = begin_status(c);
    if (rc) return rc;
    const int kk = k > 0 ? k : 1;
    const long ldk = (kk + 1) & ~1L;  // K-contiguous staging rows, even stride
    double *X, *Y, *T, *Cd;
    // X = op(B)^T (n x k), Y = op(A) (m x k), C^T (n x m)
    if ((rc = stage(c, 0, (size_t)n * ldk, &X)) || (rc = stage(c, 1, (size_t)m * ldk, &Y))) return rc;
    const long ldcd = (m + 1) & ~1L;
    if ((rc = stage(c, 2, (size_t)n * ldcd, &Cd))) return rc;
    if (k == 0) {
        CU_TRY(cudaMemsetAsync(X, 0, (size_t)n * ldk * sizeof(double), c->stream));
        CU_TRY(cudaMemsetAsync(Y, 0, (size_t)m * ldk * sizeof(double), c->stream));
    } else {
        if (!A || !B) {
            set_error("gdr_dgemm_: null operand");
            return LU2GPU_ERR_ARG;
        }
        // op(B)^T[j][q]: notb -> B[q + j*ldb] (rows j, contiguous q); else B[j + q*ldb]
        if (notb) {
            CU_TRY(cudaMemcpy2DAsync(X, ldk * sizeof(double), B, (size_t)ldb * sizeof(double),
                                     (size_t)k * sizeof(double), n, cudaMemcpyHostToDevice, c->stream));
        } else {
            const long ldt = (n + 1) & ~1L;
            if ((rc = stage(c, 3, (size_t)k * ldt, &T))) return rc;
            CU_TRY(cudaMemcpy2DAsync(T, ldt * sizeof(double), B, (size_t)ldb * sizeof(double),
                                     (size_t)n * sizeof(double), k, cudaMemcpyHostToDevice, c->stream));
            K_TRY(launch_transpose(T, ldt, X, ldk, k, n, c->stream));
        }
        // op(A)[i][q]: nota -> A[i + q*lda]; else A[q + i*lda] (rows i, contiguous q)
        if (!nota) {
            CU_TRY(cudaMemcpy2DAsync(Y, ldk * sizeof(double), A, (size_t)lda * sizeof(double),
                                     (size_t)k * sizeof(double), m, cudaMemcpyHostToDevice, c->stream));
        } else {
            const long ldt = (m + 1) & ~1L;
            if ((rc = stage(c, 3, (size_t)k * ldt, &T))) return rc;
            CU_TRY(cudaMemcpy2DAsync(T, ldt * sizeof(double), A, (size_t)lda * sizeof(double),
                                     (size_t)m * sizeof(double), k, cudaMemcpyHostToDevice, c->stream));
            K_TRY(launch_transpose(T, ldt, Y, ldk, k, m, c->stream));
        }
    }
    if (beta != 0.0)
        CU_TRY(cudaMemcpy2DAsync(Cd, ldcd * sizeof(double), C, (size_t)ldc * sizeof(double),
                                 (size_t)m * sizeof(double), n, cudaMemcpyHostToDevice, c->stream));
    K_TRY(launch_dgemm_general(X, ldk, Y, ldk, Cd, ldcd, n, m, kk, alpha, beta, c->d_status, c->stream));
    CU_TRY(cudaMemcpy2DAsync(C, (size_t)ldc * sizeof(double), Cd, ldcd * sizeof(double), (size_t)m * sizeof(double),
                             n, cudaMemcpyDeviceToHost, c->stream));
    return end_status(c, "gdr_dgemm_");
}

static int ensure_events(std::vector<cudaEvent_t> &v, size_t count)
{
    while (v.size() < count) {
        cudaEvent_t e;
        CU_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        v.push_back(e);
    }
    return 0;
}

// The same product with C in pinned (or registered) host memory, overlapped
// as the board library's "-ovl" build did (Makefile.mgv:29): op(A) goes to the
// device first; then blocks of jb columns of C (with their columns of op(B))
// go in on one stream, are multiplied on the context's stream and come back on
// a third, so block b+1's copy in, block b's product and block b-1's copy out
// run together (PCIe carries both directions at once).  Each block's product
// is the one-pass product's for those columns: bit-identical results.
static int host_dgemm_colmajor_overlap(lu2gpu_ctx *c, int nota, int notb, int m, int n, int k, double alpha,
                                       const double *A, int lda, const double *B, int ldb, double beta, double *C,
                                       int ldc, int jb)
{
    // nothing of an earlier call (one that may have failed half way) still in flight
    if (c->copy_stream) CU_TRY(cudaStreamSynchronize(c->copy_stream));
    if (c->h2d_stream) CU_TRY(cudaStreamSynchronize(c->h2d_stream));
    int rc = begin_status(c);
    if (rc) return rc;
    const long ldk = (k + 1) & ~1L, ldcd = (m + 1) & ~1L, ldtx = (jb + 1) & ~1L, ldty = (m + 1) & ~1L;
    double *X, *Y, *T, *Cd;
    if ((rc = stage(c, 0, (size_t)n * ldk, &X)) || (rc = stage(c, 1, (size_t)m * ldk, &Y)) ||
        (rc = stage(c, 2, (size_t)n * ldcd, &Cd)) ||
        (rc = stage(c, 3, (size_t)k * (ldtx > ldty ? ldtx : ldty), &T)))
        return rc;
    if (!c->h2d_stream) CU_TRY(cudaStreamCreateWithFlags(&c->h2d_stream, cudaStreamNonBlocking));
    if (!c->copy_stream) {
        CU_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        CU_TRY(cudaEventCreateWithFlags(&c->copy_ev, cudaEventDisableTiming));
    }
    const int nblk = (n + jb - 1) / jb;
    if ((rc = ensure_events(c->h2d_ev, (size_t)nblk + 1)) || (rc = ensure_events(c->blk_ev, (size_t)nblk + 1)))
        return rc;
    // op(A)[i][q] on the context's stream
    if (!nota) {
        CU_TRY(cudaMemcpy2DAsync(Y, ldk * sizeof(double), A, (size_t)lda * sizeof(double), (size_t)k * sizeof(double),
                                 m, cudaMemcpyHostToDevice, c->stream));
    } else {
        CU_TRY(cudaMemcpy2DAsync(T, ldty * sizeof(double), A, (size_t)lda * sizeof(double), (size_t)m * sizeof(double),
                                 k, cudaMemcpyHostToDevice, c->stream));
        K_TRY(launch_transpose(T, ldty, Y, ldk, k, m, c->stream));
    }
    // the block copies start after everything before them on the context's stream
    CU_TRY(cudaEventRecord(c->h2d_ev[nblk], c->stream));
    CU_TRY(cudaStreamWaitEvent(c->h2d_stream, c->h2d_ev[nblk], 0));
    for (int b = 0; b < nblk; b++) {
        const int j0 = b * jb, nj = (n - j0) < jb ? n - j0 : jb;
        // op(B)^T rows j0..j0+nj-1: notb -> B[q + j*ldb]; else B[j + q*ldb] (transposed via T)
        if (notb) {
            CU_TRY(cudaMemcpy2DAsync(X + (size_t)j0 * ldk, ldk * sizeof(double), B + (size_t)j0 * ldb,
                                     (size_t)ldb * sizeof(double), (size_t)k * sizeof(double), nj,
                                     cudaMemcpyHostToDevice, c->h2d_stream));
        } else {
            CU_TRY(cudaMemcpy2DAsync(T, ldtx * sizeof(double), B + j0, (size_t)ldb * sizeof(double),
                                     (size_t)nj * sizeof(double), k, cudaMemcpyHostToDevice, c->h2d_stream));
            K_TRY(launch_transpose(T, ldtx, X + (size_t)j0 * ldk, ldk, k, nj, c->h2d_stream));
        }
        if (beta != 0.0)
            CU_TRY(cudaMemcpy2DAsync(Cd + (size_t)j0 * ldcd, ldcd * sizeof(double), C + (size_t)j0 * ldc,
                                     (size_t)ldc * sizeof(double), (size_t)m * sizeof(double), nj,
                                     cudaMemcpyHostToDevice, c->h2d_stream));
        CU_TRY(cudaEventRecord(c->h2d_ev[b], c->h2d_stream));
        CU_TRY(cudaStreamWaitEvent(c->stream, c->h2d_ev[b], 0));
        K_TRY(launch_dgemm_general(X + (size_t)j0 * ldk, ldk, Y, ldk, Cd + (size_t)j0 * ldcd, ldcd, nj, m, k, alpha,
                                   beta, c->d_status, c->stream));
        CU_TRY(cudaEventRecord(c->blk_ev[b], c->stream));
        CU_TRY(cudaStreamWaitEvent(c->copy_stream, c->blk_ev[b], 0));
        CU_TRY(cudaMemcpy2DAsync(C + (size_t)j0 * ldc, (size_t)ldc * sizeof(double), Cd + (size_t)j0 * ldcd,
                                 ldcd * sizeof(double), (size_t)m * sizeof(double), nj, cudaMemcpyDeviceToHost,
                                 c->copy_stream));
    }
    // the last copy out precedes what follows on the context's stream
    CU_TRY(cudaEventRecord(c->blk_ev[nblk], c->copy_stream));
    CU_TRY(cudaStreamWaitEvent(c->stream, c->blk_ev[nblk], 0));
    return end_status(c, "gdr_dgemm_");
}

// row-major C = alpha A B + beta C (mydgemm, lu2lib.c:2079-2136) as the
// column-major product C^T = B^T A^T, the same swap mygdrdgemm makes
// (gdrdgemm.c:185-186).
static int host_dgemm_rowmajor(int m, int n, int k, double alpha, const double *a, int na, const double *b, int nb,
                               double beta, double *c, int nc)
{
    return host_dgemm_colmajor(1, 1, n, m, k, alpha, b, nb, a, na, beta, c, nc);
}

// ----- lu2lib.h -----

extern "C" void mydgemm(int m, int n, int k, double alpha, double *a, int na, double *b, int nb, double beta,
                        double *c, int nc)
{
    if (host_dgemm_rowmajor(m, n, k, alpha, a, na, b, nb, beta, c, nc) != 0) fail_void("mydgemm");
}

extern "C" void matmul_for_small_nk(int n1, double *a, int n2, double *b, int n3, double *c, int m, int kk, int n)
{
    // C -= A B with A (m x kk, stride n1), B (kk x n, stride n2), C (m x n, stride n3) (lu2lib.c:1984-2077)
    if (host_dgemm_rowmajor(m, n, kk, -1.0, a, n1, b, n2, 1.0, c, n3) != 0) fail_void("matmul_for_small_nk");
}

extern "C" void gdrsetboardid(int boardid)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (boardid != g_board && g_ctx) {
        lu2gpu_destroy(g_ctx);
        g_ctx = nullptr;
        g_gdr_ok = 0;
    }
    g_board = boardid;
}

// one GPU per process: the board count of the multi-board GRAPE-DR host has no meaning here
extern "C" void gdrsetnboards(int nboards) { (void)nboards; }
extern "C" void gdrsetforceswapab(void) {}
extern "C" void gdrresetforceswapab(void) {}
extern "C" void gdrsetskipsendjmat(void) {}
extern "C" void gdrresetskipsendjmat(void) {}
extern "C" void set_matmul_msg_level(int level) { (void)level; }
extern "C" void gdrdgemm_set_stress_factor(int x) { (void)x; }
extern "C" void gdrdgemm_set_procname(int id) { (void)id; }

extern "C" void gdr_init(void)
{
    if (!default_ctx()) fail_void("gdr_init");
}

extern "C" void gdr_free(void) { lu2gpu_release(); }

// ----- gdrdgemm.h -----

extern "C" void gdr_dgemm_(int *nota, int *notb, int *m, int *n, int *k, double *alpha, double *beta, int *lda,
                           int *ldb, int *ldc, const double *a, const double *b, double *c, int *doneflag)
{
    int rc = host_dgemm_colmajor(*nota, *notb, *m, *n, *k, *alpha, a, *lda, b, *ldb, *beta, c, *ldc);
    if (doneflag) *doneflag = (rc == 0) ? 1 : 0;
    if (rc != 0) fprintf(stderr, "lu2gpu: gdr_dgemm_ failed: %s\n", g_err);
}

extern "C" void gdrblas_dgemm(int order, int transa, int transb, int M, int N, int K, double alpha, const double *A,
                              int lda, const double *B, int ldb, double beta, double *C, int ldc)
{
    const int nota = (transa == LU2GPU_CBLAS_NOTRANS) ? 1 : 0;
    const int notb = (transb == LU2GPU_CBLAS_NOTRANS) ? 1 : 0;
    int rc;
    if (order == LU2GPU_CBLAS_COLMAJOR)
        rc = host_dgemm_colmajor(nota, notb, M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
    else
        rc = host_dgemm_colmajor(notb, nota, N, M, K, alpha, B, ldb, A, lda, beta, C, ldc);
    if (rc != 0) fail_void("gdrblas_dgemm");
}

extern "C" void mygdrdgemm(int m, int n, int k, double alpha, double *a, int na, double *b, int nb, double beta,
                           double *c, int nc)
{
    if (host_dgemm_rowmajor(m, n, k, alpha, a, na, b, nb, beta, c, nc) != 0) fail_void("mygdrdgemm");
}

// Self-test of the offload path, as gdr_check_and_restart (gdrdgemm.c:17-58):
// identity(2048) x B must reproduce B exactly.  Bounded: three attempts, the
// context rebuilt between them, then failure.
static int self_test(double *a, double *b, double *cm)
{
    const int N = 2048;
    for (int attempt = 0; attempt < 3; attempt++) {
        for (long i = 0; i < N; i++)
            for (long j = 0; j < N; j++) {
                a[i * N + j] = (i == j) ? 1.0 : 0.0;
                b[i * N + j] = (double)(i * N + j);
                cm[i * N + j] = 0.0;
            }
        int rc = host_dgemm_rowmajor(N, N, N, 1.0, a, N, b, N, 0.0, cm, N);
        long err = 0;
        if (rc == 0)
            for (long i = 0; i < (long)N * N; i++)
                if (b[i] != cm[i]) err++;
        if (rc == 0 && err == 0) {
            fprintf(stderr, "gdr_check_and_restart passed %d\n", attempt);
            return 0;
        }
        fprintf(stderr, "gdr_check_and_restart, err=%ld try=%d rc=%d\n", err, attempt + 1, rc);
        lu2gpu_release();
    }
    set_error("offload self-test failed three times");
    return LU2GPU_ERR_CUDA;
}

extern "C" void gdr_check_and_restart(double *a, double *b, double *c)
{
    if (g_gdr_ok) return;
    if (self_test(a, b, c) != 0) {
        fail_void("gdr_check_and_restart");
        return;
    }
    g_gdr_ok = 1;
}

extern "C" void reset_gdr(int m, double *a, int nb, double *awork, int n)
{
    // lu2lib.c:2138-2168 runs the board self-test on caller buffers; the GPU
    // version uses its own and has no nb >= 2048 restriction (that was the board's).
    (void)m;
    (void)a;
    (void)nb;
    (void)awork;
    (void)n;
    if (g_gdr_ok) return;
    const size_t N2 = (size_t)2048 * 2048;
    double *buf = (double *)malloc(3 * N2 * sizeof(double));
    if (!buf) {
        set_error("reset_gdr: host allocation failed");
        fail_void("reset_gdr");
        return;
    }
    int rc = self_test(buf, buf + N2, buf + 2 * N2);
    free(buf);
    if (rc != 0) {
        fail_void("reset_gdr");
        return;
    }
    g_gdr_ok = 1;
}

// ----- lu2.c: lumcolumn -----

// Panels to factor left-looking while a pinned host matrix streams in: enough
// that the catch-up of each arriving column group (p0 panel updates, 2 n nb
// FLOPs per column each at ~30 TFLOP/s) takes as long as the group's copy
// (8 n bytes per column at ~55 GB/s over PCIe), i.e. p0 = 8 * 30e12 /
// (55e9 * 2 nb), independent of n.  Fewer leaves the compute waiting for the
// copy; more runs a growing start as narrow one-panel-wide updates, whose row
// exchanges and U-block solves cost as much as full-width ones.  Measured at
// n = 65536, nb = 256 (e2e seconds): p0 = 1: 6.76, 4: 6.57, 9: 6.26,
// 16: 6.28, 32: 6.39, 64: 6.75; without the chunked copy 6.82.
static int left_looking_panels(int n, int nb)
{
    const int panels = (n + nb - 1) / nb;
    const int p0 = (int)ceil(8.0 * 30e12 / (55e9 * 2.0 * nb));
    return p0 < panels ? p0 : panels;
}

// lumcolumn (lu2.c:1122-1144) on the caller's host matrix a[n][n+16] (b in
// column n): the matrix goes to the GPU, is factored there (recursive panels,
// nb = m), x = U'^{-1} y is written to b, the factored matrix (with y in
// column n) comes back, and pv[0..m) holds the last panel's pivot rows as in
// the reference.  `recursive` is accepted for signature compatibility; the
// GPU path is always the recursive one.  `awork` is not used.
// Pageable host matrices at least this large are page-locked by lumcolumn
// for the call (the copies then overlap the factorization).
constexpr size_t HOST_REGISTER_MIN_BYTES = (size_t)2 << 30;

// cudaHostRegister for the duration of one call: take() registers a range;
// the destructor waits for the context's streams (copies of the range may
// still be in flight after an error return) and unregisters it.
struct HostRegistration {
    lu2gpu_ctx *c;
    void *ptr = nullptr;
    explicit HostRegistration(lu2gpu_ctx *ctx) : c(ctx) {}
    bool take(void *p, size_t bytes)
    {
        if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        ptr = p;
        return true;
    }
    ~HostRegistration()
    {
        if (!ptr) return;
        cudaStreamSynchronize(c->stream);
        if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
        if (c->h2d_stream) cudaStreamSynchronize(c->h2d_stream);
        cudaHostUnregister(ptr);
        cudaGetLastError();
    }
};

static int lumcolumn_host(int n, double *a, double *b, int m, int *pv)
{
    lu2gpu_ctx *c = default_ctx();
    if (!c) return LU2GPU_ERR_NODEV;
    if (n <= 0 || !a || !b) {
        set_error("lumcolumn: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    const long rdim = (long)n + 16;
    const long ld = ((long)n + 16 + 1) & ~1L;
    double *d, *x;
    int rc;
    if (m <= 0) {
        set_error("lumcolumn: block size %d", m);
        return LU2GPU_ERR_ARG;
    }
    if ((rc = stage(c, 0, (size_t)n * ld, &d))) return rc;
    if ((rc = stage(c, 1, (size_t)n, &x))) return rc;
    const int nbw = gpu_panel_width(m);
    rc = check_matrix_args(n, 1, d, ld, nbw);
    if (rc) return rc;
    // pinned (or registered) host matrix: finished factor blocks go back on a
    // copy stream while the factorization continues; pageable memory would
    // make those copies block the enqueuing thread, so it is copied at the end
    cudaPointerAttributes pa{};
    bool pinned = cudaPointerGetAttributes(&pa, a) == cudaSuccess && pa.type == cudaMemoryTypeHost;
    cudaGetLastError();
    // a large pageable matrix (lu2's main allocates it with malloc or from
    // hugetlbfs, lu2.c:1245-1264) is page-locked for the duration of the call,
    // so that it takes the overlapped path; LU2GPU_HOST_REGISTER=0 never, =1
    // always, default from HOST_REGISTER_MIN_BYTES.  Unregistered on every
    // return, after the streams that copy it are idle.
    HostRegistration reg(c);
    if (!pinned) {
        const char *hr = getenv("LU2GPU_HOST_REGISTER");
        const size_t bytes = (size_t)n * rdim * sizeof(double);
        const bool want = hr ? atoi(hr) != 0 : bytes >= HOST_REGISTER_MIN_BYTES;
        if (want && reg.take(a, bytes)) pinned = true;
    }
    // nothing of an earlier call (one that may have failed half way) still in flight
    if (c->copy_stream) CU_TRY(cudaStreamSynchronize(c->copy_stream));
    if (c->h2d_stream) CU_TRY(cudaStreamSynchronize(c->h2d_stream));
    if (pinned && !c->copy_stream) {
        CU_TRY(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
        CU_TRY(cudaEventCreateWithFlags(&c->copy_ev, cudaEventDisableTiming));
    }
    if ((rc = begin_status(c))) return rc;
    const size_t pitch_h = rdim * sizeof(double), pitch_d = ld * sizeof(double);
    // pinned host matrix: column chunks go to the device on their own stream,
    // one event each, and the factorization starts left-looking on the chunks
    // that have arrived (factor_enqueue_arriving); pageable: one copy first
    const int ncol = n + 1;
    const char *ov = getenv("LU2GPU_H2D_OVERLAP");
    const bool overlap = pinned && !(ov && atoi(ov) == 0);
    int cw = ncol, p0 = 0, group = 0, waited = 0;
    if (overlap) {
        if (!c->h2d_stream) CU_TRY(cudaStreamCreateWithFlags(&c->h2d_stream, cudaStreamNonBlocking));
        cw = (512 / nbw) * nbw;  // >= 4 KB per row segment; nbw <= 512
        const int nchunk = (ncol + cw - 1) / cw;
        while ((int)c->h2d_ev.size() < nchunk) {
            cudaEvent_t e;
            CU_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            c->h2d_ev.push_back(e);
        }
        // the staging matrix is rewritten only after the stream's earlier work on it
        CU_TRY(cudaEventRecord(c->copy_ev, c->stream));
        CU_TRY(cudaStreamWaitEvent(c->h2d_stream, c->copy_ev, 0));
        for (int j = 0; j < nchunk; ++j) {
            const int c0 = j * cw, w = (ncol - c0) < cw ? ncol - c0 : cw;
            CU_TRY(cudaMemcpy2DAsync(d + c0, pitch_d, a + c0, pitch_h, (size_t)w * sizeof(double), n,
                                     cudaMemcpyHostToDevice, c->h2d_stream));
            CU_TRY(cudaEventRecord(c->h2d_ev[j], c->h2d_stream));
        }
        const char *lp = getenv("LU2GPU_LEFT_PANELS");
        p0 = lp ? atoi(lp) : left_looking_panels(n, nbw);
        group = (4096 / cw) * cw;
        if (group < cw) group = cw;
    } else {
        CU_TRY(cudaMemcpy2DAsync(d, pitch_d, a, pitch_h, (size_t)ncol * sizeof(double), n, cudaMemcpyHostToDevice,
                                 c->stream));
    }
    auto wait_cols = [&](int ce) -> int {
        if (!overlap) return 0;
        for (const int need = (ce + cw - 1) / cw; waited < need; ++waited)
            CU_TRY(cudaStreamWaitEvent(c->stream, c->h2d_ev[waited], 0));
        return 0;
    };
    auto copy_back = [&](int i, int w) -> int {
        if (!pinned) return 0;
        CU_TRY(cudaEventRecord(c->copy_ev, c->stream));
        CU_TRY(cudaStreamWaitEvent(c->copy_stream, c->copy_ev, 0));
        // rows i..i+w-1 from column i through column n (y), then columns i..i+w-1 of the rows below
        CU_TRY(cudaMemcpy2DAsync(a + (size_t)i * rdim + i, pitch_h, d + (size_t)i * ld + i, pitch_d,
                                 (size_t)(n + 1 - i) * sizeof(double), w, cudaMemcpyDeviceToHost, c->copy_stream));
        if (i + w < n)
            CU_TRY(cudaMemcpy2DAsync(a + (size_t)(i + w) * rdim + i, pitch_h, d + (size_t)(i + w) * ld + i, pitch_d,
                                     (size_t)w * sizeof(double), n - i - w, cudaMemcpyDeviceToHost, c->copy_stream));
        return 0;
    };
    if ((rc = factor_enqueue_arriving(c, n, 1, d, ld, nbw, g_pivot_mode, p0, group, copy_back, wait_cols)))
        return rc;
    CU_TRY(cudaMemcpy2DAsync(x, sizeof(double), d + n, ld * sizeof(double), sizeof(double), n,
                             cudaMemcpyDeviceToDevice, c->stream));
    {
        PhaseTimer t(c, PH_BACKSOLVE);
        K_TRY(launch_backsolve(d, ld, n, 1, x, 1, bs_buffers(c, n), c->stream));
    }
    if (pinned) {
        CU_TRY(cudaEventRecord(c->copy_ev, c->copy_stream));
        CU_TRY(cudaStreamWaitEvent(c->stream, c->copy_ev, 0));
    } else {
        CU_TRY(cudaMemcpy2DAsync(a, pitch_h, d, pitch_d, (size_t)(n + 1) * sizeof(double), n, cudaMemcpyDeviceToHost,
                                 c->stream));
    }
    CU_TRY(cudaMemcpyAsync(b, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (pv) {
        const int last = ((n - 1) / m) * m;
        CU_TRY(cudaMemcpyAsync(pv, c->d_ipiv + last, (size_t)(n - last) * sizeof(int), cudaMemcpyDeviceToHost,
                               c->stream));
    }
    return end_status(c, "lumcolumn");
}

extern "C" void lumcolumn(int n, double *a, double *b, int m, double *awork, int *pv, int recursive)
{
    (void)awork;
    (void)recursive;
    int rc = lumcolumn_host(n, a, b, m, pv);
    if (rc < 0) fail_void("lumcolumn");
    if (rc > 0) fprintf(stderr, "lu2gpu: lumcolumn: %s\n", g_err);
}

extern "C" int lu2gpu_lumcolumn(int n, double *a, double *b, int m, int *pv, int pivot_mode)
{
    if (pivot_mode != LU2GPU_PIVOT_REF && pivot_mode != LU2GPU_PIVOT_PARTIAL) {
        set_error("unknown pivot mode %d", pivot_mode);
        return LU2GPU_ERR_ARG;
    }
    const int old = g_pivot_mode;
    g_pivot_mode = pivot_mode;
    int rc = lumcolumn_host(n, a, b, m, pv);
    g_pivot_mode = old;
    return rc;
}

// ----- lu2.c per-panel entry points and lu2tlib.h's column-major slab API -----
//
// These take lu2's host arrays like the reference's functions and run the
// same GPU kernels on a device copy of the region each call touches: rows
// i..n-1 of the columns involved, as a view whose element (0,0) is global
// (i, i) so that pivot rows and the reference-mode column parity stay global.

// right part of a view with K = k1 - k0 not a multiple of 16 (the slab API's
// inner blocks): exact-extent tensor maps zero-fill the GEMM's K remainder
static int right_part_anyk(lu2gpu_ctx *c, const View &v, int k0, int k1, int cs, int ce)
{
    if (ce <= cs) return 0;
    if ((k1 - k0) % 16 == 0) return right_part(c, v, k0, k1, cs, ce, false);
    const int K = k1 - k0;
    K_TRY(launch_laswp_scale(v.a, v.ld, v.n, k0, k1, c->d_ipiv + v.goff, v.goff, c->d_dinv + v.goff, cs, ce, true,
                             c->d_status, c->stream));
    K_TRY(launch_trsm_unit_lower(v.a, v.ld, k0, K, cs, ce, c->d_bt, c->stream));
    if (k1 < v.n) {
        const long ldk = (K + 1) & ~1L;
        double *lk;
        int rc = stage(c, 3, (size_t)(v.n - k1) * ldk, &lk);
        if (rc) return rc;
        // L21 (rows k1.., columns k0..k1) into an even-stride buffer, then C -= L21 U12
        CU_TRY(cudaMemcpy2DAsync(lk, ldk * sizeof(double), v.a + (size_t)k1 * v.ld + k0, v.ld * sizeof(double),
                                 (size_t)K * sizeof(double), v.n - k1, cudaMemcpyDeviceToDevice, c->stream));
        // d_bt holds -U12^T
        K_TRY(launch_dgemm_general(lk, ldk, c->d_bt, K, v.a + (size_t)k1 * v.ld + cs, v.ld, v.n - k1, ce - cs, K, 1.0,
                                   1.0, c->d_status, c->stream));
    }
    return 0;
}

// stage rows i..n-1, columns i..i+w-1 of lu2's a[n][rdim] into a device view
static int stage_rows(lu2gpu_ctx *c, const double *a, long rdim, int n, int i, int w, int slot, View *v)
{
    const long ld = ((long)w + 15) & ~15L;
    double *d;
    int rc = stage(c, slot, (size_t)(n - i) * ld, &d);
    if (rc) return rc;
    CU_TRY(cudaMemcpy2DAsync(d, ld * sizeof(double), a + (size_t)i * rdim + i, rdim * sizeof(double),
                             (size_t)w * sizeof(double), n - i, cudaMemcpyHostToDevice, c->stream));
    *v = View{d, ld, n - i, w, i};
    return 0;
}

static int unstage_rows(lu2gpu_ctx *c, double *a, long rdim, int i, int col0, int w, const View &v)
{
    CU_TRY(cudaMemcpy2DAsync(a + (size_t)i * rdim + i + col0, rdim * sizeof(double), v.a + col0, v.ld * sizeof(double),
                             (size_t)w * sizeof(double), v.n, cudaMemcpyDeviceToHost, c->stream));
    return 0;
}

// column_decomposition_recursive (lu2.c:1088-1120): the panel of columns
// i..i+m-1, rows i..n-1, of a[n][n+16]; pv[0..m) = global pivot rows.
static int colrec_host(int n, double *a, int m, int *pv, int i, int mode)
{
    lu2gpu_ctx *c = default_ctx();
    if (!c) return LU2GPU_ERR_NODEV;
    if (n <= 0 || !a || !pv || m <= 0 || i < 0 || i + m > n) {
        set_error("column_decomposition_recursive: bad arguments (n=%d m=%d i=%d)", n, m, i);
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    // the recursion's inner right parts hold a K x (m - K) transposed U block
    int rc = ensure_work(c, n, m + 16, m);
    if (rc) return rc;
    if ((rc = begin_status(c))) return rc;
    View v;
    if ((rc = stage_rows(c, a, (long)n + 16, n, i, m, 0, &v))) return rc;
    if ((rc = panel(c, v, 0, m, mode))) return rc;
    if ((rc = unstage_rows(c, a, (long)n + 16, i, 0, m, v))) return rc;
    CU_TRY(cudaMemcpyAsync(pv, c->d_ipiv + i, (size_t)m * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    return end_status(c, "column_decomposition_recursive");
}

// caller-supplied pivot rows: pv[k] must name a row of the trailing block
// (i + k <= pv[k] < n), as lu2's pivot search produces them
static bool pivots_valid(const int *pv, int m, int i, int n, const char *who)
{
    for (int k = 0; k < m; k++)
        if (pv[k] < i + k || pv[k] >= n) {
            set_error("%s: pivot %d is row %d (must be in [%d, %d))", who, k, pv[k], i + k, n);
            return false;
        }
    return true;
}

// process_right_part (lu2.c:524-581): pivots pv[0..m) of rows i..i+m-1 applied
// to columns i+m..iend-1 with the 1/pivot scaling, U block solved, rows
// i+m..n-1 updated.
static int rightpart_host(int n, double *a, int m, const int *pv, int i, int iend)
{
    lu2gpu_ctx *c = default_ctx();
    if (!c) return LU2GPU_ERR_NODEV;
    if (n <= 0 || !a || !pv || m <= 0 || i < 0 || i + m > n || iend < i + m || iend > n + 16) {
        set_error("process_right_part: bad arguments (n=%d m=%d i=%d iend=%d)", n, m, i, iend);
        return LU2GPU_ERR_ARG;
    }
    if (!pivots_valid(pv, m, i, n, "process_right_part")) return LU2GPU_ERR_ARG;
    DeviceGuard g(c->device);
    int rc = ensure_work(c, n, iend - i + 16, m);
    if (rc) return rc;
    if ((rc = begin_status(c))) return rc;
    View v;
    if ((rc = stage_rows(c, a, (long)n + 16, n, i, iend - i, 0, &v))) return rc;
    CU_TRY(cudaMemcpyAsync(c->d_ipiv + i, pv, (size_t)m * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    K_TRY(launch_diag_inv(v.a, v.ld, m, c->d_dinv + i, c->stream));
    if ((rc = right_part_anyk(c, v, 0, m, m, iend - i))) return rc;
    if ((rc = unstage_rows(c, a, (long)n + 16, i, m, iend - i - m, v))) return rc;
    return end_status(c, "process_right_part");
}

// backward_sub (lu2.c:110-116): b = U'^{-1} (column n) with a's unit upper factor
static int backsub_host(int n, const double *a, double *b)
{
    lu2gpu_ctx *c = default_ctx();
    if (!c) return LU2GPU_ERR_NODEV;
    if (n <= 0 || !a || !b) {
        set_error("backward_sub: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    const long rdim = (long)n + 16, ld = ((long)n + 16 + 1) & ~1L;
    double *d, *x;
    int rc;
    if ((rc = stage(c, 0, (size_t)n * ld, &d)) || (rc = stage(c, 1, (size_t)n, &x))) return rc;
    if ((rc = begin_status(c))) return rc;
    CU_TRY(cudaMemcpy2DAsync(d, ld * sizeof(double), a, rdim * sizeof(double), (size_t)(n + 1) * sizeof(double), n,
                             cudaMemcpyHostToDevice, c->stream));
    CU_TRY(cudaMemcpy2DAsync(x, sizeof(double), d + n, ld * sizeof(double), sizeof(double), n,
                             cudaMemcpyDeviceToDevice, c->stream));
    K_TRY(launch_backsolve(d, ld, n, 1, x, 1, bs_buffers(c, n), c->stream));
    CU_TRY(cudaMemcpyAsync(b, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    return end_status(c, "backward_sub");
}

extern "C" void column_decomposition_recursive(int n, double *a, int m, double *awork, int *pv, int i)
{
    (void)awork;
    if (colrec_host(n, a, m, pv, i, g_pivot_mode) < 0) fail_void("column_decomposition_recursive");
}

extern "C" void process_right_part(int n, double *a, int m, double *awork, int *pv, int i, int iend)
{
    (void)awork;
    if (rightpart_host(n, a, m, pv, i, iend) < 0) fail_void("process_right_part");
}

extern "C" void backward_sub(int n, double *a, double *b)
{
    if (backsub_host(n, a, b) < 0) fail_void("backward_sub");
}

// The column-major slab of lu2tlib.c: a[j][r] at a + j*n + r (column stride
// n), columns 0..m-1 relative to a (or 0..iend-i-1), rows i..n-1.  Staged
// transposed into a row-major device view.
static int stage_slab(lu2gpu_ctx *c, const double *a, int n, int i, int cols, View *v)
{
    const int rows = n - i;
    const long ld = ((long)cols + 15) & ~15L, ldt = ((long)rows + 1) & ~1L;
    double *d, *t;
    int rc;
    if ((rc = stage(c, 0, (size_t)rows * ld, &d)) || (rc = stage(c, 2, (size_t)cols * ldt, &t))) return rc;
    CU_TRY(cudaMemcpy2DAsync(t, ldt * sizeof(double), a + i, (size_t)n * sizeof(double), (size_t)rows * sizeof(double),
                             cols, cudaMemcpyHostToDevice, c->stream));
    K_TRY(launch_transpose(t, ldt, d, ld, cols, rows, c->stream));
    *v = View{d, ld, rows, cols, i};
    return 0;
}

static int unstage_slab(lu2gpu_ctx *c, double *a, int n, int i, int col0, int cols, const View &v)
{
    const int rows = n - i;
    const long ldt = ((long)rows + 1) & ~1L;
    double *t;
    int rc = stage(c, 2, (size_t)(col0 + cols) * ldt, &t);
    if (rc) return rc;
    K_TRY(launch_transpose(v.a + col0, v.ld, t, ldt, rows, cols, c->stream));
    CU_TRY(cudaMemcpy2DAsync(a + (size_t)col0 * n + i, (size_t)n * sizeof(double), t, ldt * sizeof(double),
                             (size_t)rows * sizeof(double), cols, cudaMemcpyDeviceToHost, c->stream));
    return 0;
}

static int cm_decomp_host(int n, double *a, int m, int *pv, int i, bool recursive)
{
    lu2gpu_ctx *c = default_ctx();
    if (!c) return LU2GPU_ERR_NODEV;
    if (n <= 0 || !a || !pv || m <= 0 || i < 0 || i + m > n) {
        set_error("cm_column_decomposition: bad arguments (n=%d m=%d i=%d)", n, m, i);
        return LU2GPU_ERR_ARG;
    }
    int mode = g_pivot_mode;
    if (!recursive) {
        // column_decomposition (lu2tlib.c:1041-1066) called on the whole slab:
        // in the reference's pivot search every column searches column 0
        if (m > 16) {
            set_error("cm_column_decomposition: slab of %d columns (at most 16)", m);
            return LU2GPU_ERR_ARG;
        }
        if (mode == LU2GPU_PIVOT_REF) mode = PIVOT_REF_FIRST;
    }
    DeviceGuard g(c->device);
    int rc = ensure_work(c, n, m + 16, m < 16 ? 16 : m);
    if (rc) return rc;
    if ((rc = begin_status(c))) return rc;
    View v;
    if ((rc = stage_slab(c, a, n, i, m, &v))) return rc;
    if (recursive) {
        if ((rc = panel(c, v, 0, m, mode))) return rc;
    } else {
        K_TRY(launch_leaf(v.a, v.ld, v.n, 0, m, mode, v.goff, c->d_ipiv + v.goff, c->d_dinv + v.goff, c->leaf,
                          c->d_status, c->leaf_ctas, c->stream));
    }
    if ((rc = unstage_slab(c, a, n, i, 0, m, v))) return rc;
    CU_TRY(cudaMemcpyAsync(pv, c->d_ipiv + i, (size_t)m * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    return end_status(c, "cm_column_decomposition");
}

extern "C" void cm_column_decomposition_recursive(int n, double *a, int m, int *pv, int i)
{
    if (cm_decomp_host(n, a, m, pv, i, true) < 0) fail_void("cm_column_decomposition_recursive");
}

extern "C" void cm_column_decomposition(int n, double *a, int m, int *pv, int i)
{
    if (cm_decomp_host(n, a, m, pv, i, false) < 0) fail_void("cm_column_decomposition");
}

// process_right_part of the slab (lu2tlib.c:1068-1093): columns m..iend-i-1
static int cm_right_host(int n, double *a, int m, const int *pv, int i, int iend)
{
    lu2gpu_ctx *c = default_ctx();
    if (!c) return LU2GPU_ERR_NODEV;
    if (n <= 0 || !a || !pv || m <= 0 || i < 0 || i + m > n || iend < i + m || iend - i > n + 1) {
        set_error("cm_process_right_part: bad arguments (n=%d m=%d i=%d iend=%d)", n, m, i, iend);
        return LU2GPU_ERR_ARG;
    }
    if (!pivots_valid(pv, m, i, n, "cm_process_right_part")) return LU2GPU_ERR_ARG;
    DeviceGuard g(c->device);
    const int cols = iend - i;
    int rc = ensure_work(c, n, cols + 16, ((m + 15) / 16) * 16);
    if (rc) return rc;
    if ((rc = begin_status(c))) return rc;
    View v;
    if ((rc = stage_slab(c, a, n, i, cols, &v))) return rc;
    CU_TRY(cudaMemcpyAsync(c->d_ipiv + i, pv, (size_t)m * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    K_TRY(launch_diag_inv(v.a, v.ld, m, c->d_dinv + i, c->stream));
    if ((rc = right_part_anyk(c, v, 0, m, m, cols))) return rc;
    if ((rc = unstage_slab(c, a, n, i, m, cols - m, v))) return rc;
    return end_status(c, "cm_process_right_part");
}

extern "C" void cm_process_right_part(int n, double *a, int m, int *pv, int i, int iend)
{
    if (cm_right_host(n, a, m, pv, i, iend) < 0) fail_void("cm_process_right_part");
}

extern "C" int lu2gpu_copy_pivots(lu2gpu_ctx *c, int *ipiv_host, int n)
{
    if (!c || !ipiv_host || n <= 0 || (size_t)n > c->piv_cap) {
        set_error("lu2gpu_copy_pivots: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    CU_TRY(cudaStreamSynchronize(c->stream));
    CU_TRY(cudaMemcpy(ipiv_host, c->d_ipiv, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost));
    return 0;
}

// ---------------------------------------------------------------------------
// Allocation-free solve for small systems.
//
// Some callers cannot allocate device memory when they need a solve: the
// device memory may already be owned by another allocator (a framework's
// caching allocator that has reserved most of HBM, or an application with a
// fixed memory budget), or the caller cannot afford cudaMalloc/cudaFree, which
// synchronize the whole device and stall every other stream.  For them this
// entry point takes all of its scratch (pivot arrays, the transposed U block
// row, the panel-exchange buffers, the status words) from one file-scope
// device array of fixed size.  Every GPU that loads this library holds that
// array until the process exits.

constexpr int NOALLOC_MAX_N = 2048;
constexpr int NOALLOC_MAX_NB = 128;
constexpr int NOALLOC_MAX_NRHS = 16;
constexpr int NOALLOC_LEAF_CTAS = (NOALLOC_MAX_N + 127) / 128;  // leaf grid at n <= 2048

constexpr size_t na_round(size_t b) { return (b + 255) & ~size_t(255); }
constexpr size_t NA_STATUS = 0;
constexpr size_t NA_LEAF = NA_STATUS + na_round(4 * sizeof(int));
constexpr size_t NA_LEAF_BYTES = na_round((size_t)2 * NOALLOC_LEAF_CTAS * sizeof(LeafSlot));
constexpr size_t NA_DINV = NA_LEAF + NA_LEAF_BYTES;
constexpr size_t NA_IPIV = NA_DINV + na_round(NOALLOC_MAX_N * sizeof(double));
constexpr size_t NA_BT = NA_IPIV + na_round(NOALLOC_MAX_N * sizeof(int));
constexpr size_t NA_BT_BYTES =
    ((size_t)(NOALLOC_MAX_N + NOALLOC_MAX_NRHS) * NOALLOC_MAX_NB + 1024) * sizeof(double);
constexpr size_t NOALLOC_SCRATCH_BYTES = NA_BT + na_round(NA_BT_BYTES);  // about 2.1 MB

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Device address of g_noalloc_scratch per device, looked up once per device
// with that device current.  In host code the symbol itself is only a host-side
// stand-in and must never be passed to a kernel.
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[128];
static int g_noalloc_ctas[128];
static int g_noalloc_major[128];  // compute capability major of each device, 0 until looked up
// leaf publication stamps per device; the slots start zeroed (static storage)
// and every stamp is used once, so leftovers of earlier calls never match
static unsigned long long g_noalloc_seq[128];

static int noalloc_setup(int device, unsigned char **base, int *leaf_ctas)
{
    if (device < 0 || device >= 128) {
        set_error("lu2gpu_lusolve_noalloc: device ordinal %d out of range", device);
        return LU2GPU_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_major[device]) {
        int major = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess) {
            cudaGetLastError();
            set_error("lu2gpu_lusolve_noalloc: no usable CUDA device %d", device);
            return LU2GPU_ERR_NODEV;
        }
        g_noalloc_major[device] = major;
    }
    if (g_noalloc_major[device] != 10) {
        set_error("lu2gpu_lusolve_noalloc: device %d is sm_%d*; this library is built for sm_100a only", device,
                  g_noalloc_major[device]);
        return LU2GPU_ERR_NODEV;
    }
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error("lu2gpu_lusolve_noalloc: cudaGetSymbolAddress failed on device %d: %s", device,
                      cudaGetErrorString(e));
            return LU2GPU_ERR_CUDA;
        }
        int ctas = leaf_max_ctas(device);
        g_noalloc_ctas[device] = ctas < NOALLOC_LEAF_CTAS ? ctas : NOALLOC_LEAF_CTAS;
        g_noalloc_ptr[device] = p;
    }
    *base = (unsigned char *)g_noalloc_ptr[device];
    *leaf_ctas = g_noalloc_ctas[device];
    return 0;
}

extern "C" int lu2gpu_lusolve_noalloc(int n, int nrhs, double *a, long lda, int nb, int pivot_mode, int *ipiv,
                                      void *stream)
{
    if (n <= 0 || n > NOALLOC_MAX_N || nrhs < 1 || nrhs > NOALLOC_MAX_NRHS || nb > NOALLOC_MAX_NB) {
        set_error("lu2gpu_lusolve_noalloc: n=%d nrhs=%d nb=%d outside the fixed scratch limits "
                  "(n <= %d, 1 <= nrhs <= %d, nb <= %d)",
                  n, nrhs, nb, NOALLOC_MAX_N, NOALLOC_MAX_NRHS, NOALLOC_MAX_NB);
        return LU2GPU_ERR_ARG;
    }
    int rc = check_matrix_args(n, nrhs, a, lda, nb);
    if (rc) return rc;
    if (pivot_mode != LU2GPU_PIVOT_REF && pivot_mode != LU2GPU_PIVOT_PARTIAL) {
        set_error("unknown pivot mode %d", pivot_mode);
        return LU2GPU_ERR_ARG;
    }
    int device = 0;
    CU_TRY(cudaGetDevice(&device));
    unsigned char *base = nullptr;
    int leaf_ctas = 0;
    if ((rc = noalloc_setup(device, &base, &leaf_ctas))) return rc;

    // A context on the host stack whose buffers all point into the scratch
    // array; its capacities cover the limits above, so nothing is allocated.
    lu2gpu_ctx c;
    c.device = device;
    c.stream = (cudaStream_t)stream;
    c.own_stream = false;
    c.d_status = (int *)(base + NA_STATUS);
    c.leaf.slots = (LeafSlot *)(base + NA_LEAF);
    c.leaf.seq = &g_noalloc_seq[device];
    c.leaf_ctas = leaf_ctas;
    c.d_dinv = (double *)(base + NA_DINV);
    c.d_ipiv = ipiv ? ipiv : (int *)(base + NA_IPIV);
    c.piv_cap = NOALLOC_MAX_N;
    c.d_bt = (double *)(base + NA_BT);
    c.bt_cap = NA_BT_BYTES;
    c.fixed_scratch = true;

    // The status words must start cleared (begin_status); the leaf barrier
    // counter is cleared before every leaf launch.  Pivots, 1/pivot and the U
    // block row are written before they are read in every call.
    if ((rc = begin_status(&c))) return rc;
    if ((rc = factor_enqueue(&c, n, nrhs, a, lda, nb, pivot_mode))) return rc;
    K_TRY(launch_backsolve(a, lda, n, nrhs, a + n, lda, nullptr, c.stream));
    return end_status(&c, "lu2gpu_lusolve_noalloc");
}

// ---------------------------------------------------------------------------
// Precision form: lu2's factorization (same recursion, pivoting and storage)
// on an FP32 copy of A, the panel in exact FP32, the trailing updates as BF16
// products on the tensor cores with FP32 accumulation and per-panel
// power-of-two operand scales; then classical iterative refinement with the
// residual r = b - A x and the update of x in FP64 until the HPL scaled
// residual is below 16.

struct MixedWork {
    float *a32 = nullptr;
    size_t a32_cap = 0;
    void *l16 = nullptr;  // L21 of the current panel, BF16, M x nb
    size_t l16_cap = 0;
    void *u16 = nullptr;  // U12 transposed, BF16, N x nb
    size_t u16_cap = 0;
    float *bt32 = nullptr;  // transposed U blocks of the panel recursion (FP32)
    size_t bt32_cap = 0;
    float *dinv = nullptr;
    size_t dinv_cap = 0;
    double *vec = nullptr;  // x, r, rowabs (n doubles each) + v32 (n floats)
    size_t vec_cap = 0;
    void *small = nullptr;  // amax[2] (float bits), scales[3], norms[4] (double bits)
    size_t small_cap = 0;
    unsigned *amax() { return (unsigned *)small; }
    float *scales() { return (float *)((char *)small + 16); }
    unsigned long long *norms() { return (unsigned long long *)((char *)small + 64); }
    // trailing-update precision of the factorization: BF16 (per-panel scales)
    // or FP8 E4M3 (per-128x128-tile scales)
    int update = LU2GPU_UPDATE_BF16;
    uint8_t *l8 = nullptr, *b8 = nullptr;  // L21 (M x nb) and U12^T (N x nb), E4M3
    size_t l8_cap = 0, b8_cap = 0;
    float *dq = nullptr;  // tile dequantization factors of L21 then of U12^T
    size_t dq_cap = 0;
    float *bt32top = nullptr;  // U12^T (N x nb) in FP32 from the top-level TRSM
    size_t bt32top_cap = 0;
    double *gm = nullptr;  // GMRES: basis (restart+1 vectors), w, z, d, t, partial sums, dots
    size_t gm_cap = 0;
    // lookahead: panel k+1 on `side` while the rest of update k runs on the context's stream
    cudaStream_t side = nullptr;
    cudaEvent_t ev_cols = nullptr, ev_panel = nullptr;
};

static void free_mixed(lu2gpu_ctx *c)
{
    if (!c->mx) return;
    MixedWork *m = c->mx;
    cudaFree(m->a32);
    cudaFree(m->l16);
    cudaFree(m->u16);
    cudaFree(m->bt32);
    cudaFree(m->dinv);
    cudaFree(m->vec);
    cudaFree(m->small);
    cudaFree(m->l8);
    cudaFree(m->b8);
    cudaFree(m->dq);
    cudaFree(m->bt32top);
    cudaFree(m->gm);
    if (m->side) {
        cudaStreamSynchronize(m->side);
        cudaStreamDestroy(m->side);
    }
    if (m->ev_cols) cudaEventDestroy(m->ev_cols);
    if (m->ev_panel) cudaEventDestroy(m->ev_panel);
    delete m;
    c->mx = nullptr;
}

// FP8 form buffers for an n x n matrix with nb-wide panels
static int fp8_work(lu2gpu_ctx *c, int n, int nb)
{
    MixedWork *m = c->mx;
    int rc;
    const size_t tiles = ((size_t)n + 127) / 128 + 1;
    if ((rc = grow((void **)&m->l8, &m->l8_cap, (size_t)n * nb + 1024))) return rc;
    if ((rc = grow((void **)&m->b8, &m->b8_cap, (size_t)(n + 16) * nb + 1024))) return rc;
    if ((rc = grow((void **)&m->dq, &m->dq_cap, 2 * tiles * (nb / 128) * sizeof(float) + 256))) return rc;
    return grow((void **)&m->bt32top, &m->bt32top_cap, (size_t)(n + 16) * nb * sizeof(float) + 1024);
}

static int mixed_work(lu2gpu_ctx *c, int n, long ld32, int nb)
{
    if (!c->mx) c->mx = new MixedWork();
    MixedWork *m = c->mx;
    int rc;
    if ((rc = grow((void **)&m->a32, &m->a32_cap, (size_t)n * ld32 * sizeof(float)))) return rc;
    if ((rc = grow(&m->l16, &m->l16_cap, (size_t)n * nb * 2 + 1024))) return rc;
    if ((rc = grow(&m->u16, &m->u16_cap, (size_t)n * nb * 2 + 1024))) return rc;
    if ((rc = grow((void **)&m->bt32, &m->bt32_cap, (size_t)nb * nb * sizeof(float) + 1024))) return rc;
    if ((rc = grow((void **)&m->dinv, &m->dinv_cap, (size_t)n * sizeof(float) + 256))) return rc;
    if ((rc = grow((void **)&m->vec, &m->vec_cap, (size_t)n * (3 * sizeof(double) + sizeof(float)) + 1024))) return rc;
    if ((rc = grow(&m->small, &m->small_cap, 256))) return rc;
    return ensure_work(c, n, 16, nb);  // pivot sequence in c->d_ipiv
}

struct View32 {
    float *a;
    long ld;
    int n, ncols, goff;
};

// Top-level right part of the precision forms with the trailing update in two
// launches: columns cs..cs+w1-1 first (the next panel's), then `after_first()`
// (the lookahead hook), then the rest; update kernels capped at max_ctas CTAs.
template <typename Hook>
static int right_part32_split(lu2gpu_ctx *c, const View32 &v, int k0, int k1, int cs, int ce, int w1, int max_ctas,
                              Hook after_first);

static int right_part32(lu2gpu_ctx *c, const View32 &v, int k0, int k1, int cs, int ce, bool top)
{
    if (ce <= cs) return 0;
    if (top) return right_part32_split(c, v, k0, k1, cs, ce, 0, 0, []() { return 0; });
    MixedWork *m = c->mx;
    int *ipiv = c->d_ipiv + v.goff;
    float *dinv = m->dinv + v.goff;
    const int K = k1 - k0;
    {
        PhaseTimer t(c, top ? PH_SWAP : PH_PANEL);
        K_TRY(launch_laswp_scale(v.a, v.ld, v.n, k0, k1, ipiv, v.goff, dinv, cs, ce, true, c->d_status, c->stream));
    }
    const float *T = v.a + (size_t)k0 * v.ld + k0;
    float *X = v.a + (size_t)k0 * v.ld + cs;
    if (!top) {
        PhaseTimer t(c, PH_PANEL);
        K_TRY(launch_trsm_unit_lower_f32(T, v.ld, X, v.ld, K, ce - cs, m->bt32, c->stream));
        if (k1 < v.n)
            K_TRY(launch_sgemm_update(v.a + (size_t)k1 * v.ld + k0, v.ld, m->bt32, v.a + (size_t)k1 * v.ld + cs, v.ld,
                                      v.n - k1, ce - cs, K, c->stream));
    }
    return 0;
}

template <typename Hook>
static int right_part32_split(lu2gpu_ctx *c, const View32 &v, int k0, int k1, int cs, int ce, int w1, int max_ctas,
                              Hook after_first)
{
    if (ce <= cs) return after_first();
    MixedWork *m = c->mx;
    int *ipiv = c->d_ipiv + v.goff;
    float *dinv = m->dinv + v.goff;
    const int K = k1 - k0, M = v.n - k1, N = ce - cs;
    // the second launch starts at a quantization tile boundary of U12^T
    if (w1 <= 0 || w1 >= N || (w1 % 128)) w1 = N;
    {
        PhaseTimer t(c, PH_SWAP);
        K_TRY(launch_laswp_scale(v.a, v.ld, v.n, k0, k1, ipiv, v.goff, dinv, cs, ce, true, c->d_status, c->stream));
    }
    const float *T = v.a + (size_t)k0 * v.ld + k0;
    float *X = v.a + (size_t)k0 * v.ld + cs;
    const float *L = v.a + (size_t)k1 * v.ld + k0;
    float *C = v.a + (size_t)k1 * v.ld + cs;
    int rc;
    if (m->update == LU2GPU_UPDATE_FP8) {
        {
            PhaseTimer t(c, PH_TRSM);
            // U12 solved in place; its transpose (N x K, FP32) feeds the quantizer
            K_TRY(launch_trsm_unit_lower_f32(T, v.ld, X, v.ld, K, N, k1 < v.n ? m->bt32top : nullptr, c->stream));
        }
        if (k1 >= v.n) return after_first();
        const int KB = K / 128;
        float *dqa = m->dq, *dqb = m->dq + (((size_t)M + 127) / 128) * KB;
        {
            PhaseTimer t(c, PH_DGEMM);
            K_TRY(launch_quant_fp8_tiles(L, v.ld, M, K, m->l8, K, dqa, c->stream));
            K_TRY(launch_quant_fp8_tiles(m->bt32top, K, N, K, m->b8, K, dqb, c->stream));
            K_TRY(launch_lowp_update_fp8(m->l8, K, dqa, m->b8, K, dqb, C, v.ld, M, w1, K, c->d_status, max_ctas,
                                         c->stream));
        }
        rc = after_first();
    if (rc) return rc;
        if (w1 < N) {
            PhaseTimer t(c, PH_DGEMM);
            K_TRY(launch_lowp_update_fp8(m->l8, K, dqa, m->b8 + (size_t)w1 * K, K, dqb + (size_t)(w1 / 128) * KB,
                                         C + w1, v.ld, M, N - w1, K, c->d_status, max_ctas, c->stream));
        }
        return 0;
    }
    {
        PhaseTimer t(c, PH_TRSM);
        K_TRY(launch_trsm_unit_lower_f32(T, v.ld, X, v.ld, K, N, nullptr, c->stream));
    }
    if (k1 >= v.n) return after_first();
    const char *u16 = static_cast<const char *>(m->u16);
    {
        PhaseTimer t(c, PH_DGEMM);
        CU_TRY(cudaMemsetAsync(m->amax(), 0, 2 * sizeof(unsigned), c->stream));
        K_TRY(launch_absmax(L, v.ld, M, K, m->amax(), c->stream));
        K_TRY(launch_absmax(X, v.ld, K, N, m->amax() + 1, c->stream));
        K_TRY(launch_panel_scales(m->amax(), m->scales(), c->stream));
        K_TRY(launch_f32_to_bf16(L, v.ld, m->l16, K, M, K, m->scales(), c->stream));
        K_TRY(launch_f32_transpose_bf16(X, v.ld, K, N, m->u16, m->scales() + 1, c->stream));
        K_TRY(launch_lowp_update_bf16(m->l16, K, u16, K, C, v.ld, M, w1, K, m->scales() + 2, c->d_status, max_ctas,
                                      c->stream));
    }
    rc = after_first();
    if (rc) return rc;
    if (w1 < N) {
        PhaseTimer t(c, PH_DGEMM);
        K_TRY(launch_lowp_update_bf16(m->l16, K, u16 + (size_t)w1 * K * 2, K, C + w1, v.ld, M, N - w1, K,
                                      m->scales() + 2, c->d_status, max_ctas, c->stream));
    }
    return 0;
}

static int panel32(lu2gpu_ctx *c, const View32 &v, int c0, int m, int mode)
{
    if (m <= c->leaf_w) {
        PhaseTimer t(c, PH_LEAF);
        K_TRY(launch_leaf(v.a, v.ld, v.n, c0, m, mode, v.goff, c->d_ipiv + v.goff, c->mx->dinv + v.goff, c->leaf,
                          c->d_status, c->leaf_ctas, c->stream));
        return 0;
    }
    int h = ((m / 2) + 15) & ~15;
    if (h >= m) h = m - 16;
    int rc = panel32(c, v, c0, h, mode);
    if (rc) return rc;
    if ((rc = right_part32(c, v, c0, c0 + h, c0 + h, c0 + m, false))) return rc;
    if ((rc = panel32(c, v, c0 + h, m - h, mode))) return rc;
    PhaseTimer t(c, PH_PANEL);
    K_TRY(launch_laswp_scale(v.a, v.ld, v.n, c0 + h, c0 + m, c->d_ipiv + v.goff, v.goff, c->mx->dinv + v.goff, c0,
                             c0 + h, true, c->d_status, c->stream));
    return 0;
}

// FP32 forward solve with the stored factors (what the factorization applies
// to an augmented column, panel by panel), then the back substitution.
static int solve32_enqueue(lu2gpu_ctx *c, int n, const float *a, long ld, int nb, float *v)
{
    MixedWork *m = c->mx;
    for (int i = 0; i < n; i += nb) {
        const int w = (n - i) < nb ? (n - i) : nb;
        K_TRY(launch_laswp_scale(v, 1, n, i, i + w, c->d_ipiv, 0, m->dinv, 0, 1, true, c->d_status, c->stream));
        K_TRY(launch_trsm_unit_lower_f32(a + (size_t)i * ld + i, ld, v + i, 1, w, 1, nullptr, c->stream));
        if (i + w < n)
            K_TRY(launch_gemv_sub(a + (size_t)(i + w) * ld + i, ld, n - i - w, w, v + i, v + i + w, c->stream));
    }
    K_TRY(launch_backsolve(a, ld, n, 1, v, 1, bs_buffers(c, n), c->stream));
    return 0;
}

extern "C" int lu2gpu_bf16_update_dev(lu2gpu_ctx *c, int M, int N, int K, const void *a16, long lda, const void *bt16,
                                      long ldb, float *c32, long ldc, float scale)
{
    if (!c || M < 0 || N < 0 || K < 64 || K > 256 || (K % 64) || !a16 || !bt16 || !c32) {
        set_error("lu2gpu_bf16_update_dev: bad arguments (K must be 64, 128, 192 or 256)");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    int rc = ensure_work(c, 16, 16, 16);
    if (rc) return rc;
    if ((rc = begin_status(c))) return rc;
    // the scale travels as a device scalar (the factorization computes it on the device)
    float *dscale = reinterpret_cast<float *>(c->d_bt);
    CU_TRY(cudaMemcpyAsync(dscale, &scale, sizeof(float), cudaMemcpyHostToDevice, c->stream));
    K_TRY(launch_lowp_update_bf16(a16, lda, bt16, ldb, c32, ldc, M, N, K, dscale, c->d_status, 0, c->stream));
    return end_status(c, "lu2gpu_bf16_update_dev");
}

// ---------------------------------------------------------------------------
// Batching form: many independent systems of uneven order in one persistent
// launch (kernels_batch.cu), replayed from a CUDA graph.

constexpr int BATCH_BUCKETS = 4;

struct lu2gpu_batch {
    lu2gpu_ctx *ctx = nullptr;
    int count = 0, max_n = 0;
    std::vector<BatchSys> sys;
    BatchSys *d_sys = nullptr;
    int *d_order = nullptr, *d_counter = nullptr, *d_info = nullptr;
    double *d_data = nullptr, *d_orig = nullptr, *d_resid = nullptr;
    size_t total = 0;  // doubles
    int threads = 256, pw = 32, ctas_per_sm = 1;
    long smem_doubles = 0;
    int grid = 0;
    // FP32-LU + FP64 refinement variant
    int mode = LU2GPU_BATCH_FP64, max_iter = 10;
    long long *d_woff = nullptr;
    uint8_t *d_arena = nullptr;
    int *d_iters = nullptr;
    long smem_floats = 0;
    cudaStream_t capture = nullptr;  // private stream the graph is captured on
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int bucket_pw[BATCH_BUCKETS] = {0, 0, 0, 0};  // autotuned panel width per size bucket (0: the launch's)
};

static int batch_clear_bucket_pw(lu2gpu_batch *b);

static void batch_drop_graph(lu2gpu_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

// adopt a launch shape if every system of the batch fits it; 0 or an error status
static int batch_configure(lu2gpu_batch *b, int threads, int pw, int ctas_per_sm)
{
    if (b->mode == LU2GPU_BATCH_FP32_IR) {
        // the FP32 variant keeps as many systems as fit entirely in shared memory;
        // for two CTAs per SM each keeps 8 KB clear for the kernel's static shared memory
        const long floor_floats =
            (long)((ctas_per_sm > 1 ? BATCH_SMEM_MAX / 2 - 8192 : BATCH_SMEM_MAX) / sizeof(float));
        const long sf = batch_ir_smem_floats(b->sys.data(), b->count, pw, floor_floats);
        if ((size_t)sf * sizeof(float) > BATCH_SMEM_MAX) {
            set_error("batch: panel width %d needs %ld bytes of shared memory for n=%d (limit %zu)", pw,
                      sf * (long)sizeof(float), b->max_n, BATCH_SMEM_MAX);
            return LU2GPU_ERR_ARG;
        }
        int grid = 0;
        cudaError_t e = batch_ir_grid(threads, sf, ctas_per_sm, b->count, &grid);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("batch: launch shape threads=%d pw=%d ctas=%d not launchable: %s", threads, pw, ctas_per_sm,
                      cudaGetErrorString(e));
            return LU2GPU_ERR_ARG;
        }
        b->threads = threads;
        b->pw = pw;
        b->ctas_per_sm = ctas_per_sm;
        b->smem_floats = sf;
        b->grid = grid;
        batch_drop_graph(b);
        return 0;
    }
    const long sd = batch_smem_doubles(b->sys.data(), b->count, pw);
    if ((size_t)sd * sizeof(double) > BATCH_SMEM_MAX) {
        set_error("batch: panel width %d needs %ld bytes of shared memory for n=%d (limit %zu)", pw,
                  sd * (long)sizeof(double), b->max_n, BATCH_SMEM_MAX);
        return LU2GPU_ERR_ARG;
    }
    int grid = 0;
    cudaError_t e = batch_lu_grid(threads, sd, ctas_per_sm, b->count, &grid);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("batch: launch shape threads=%d pw=%d ctas=%d not launchable: %s", threads, pw, ctas_per_sm,
                  cudaGetErrorString(e));
        return LU2GPU_ERR_ARG;
    }
    b->threads = threads;
    b->pw = pw;
    b->ctas_per_sm = ctas_per_sm;
    b->smem_doubles = sd;
    b->grid = grid;
    batch_drop_graph(b);
    return 0;
}

extern "C" int lu2gpu_batch_destroy(lu2gpu_batch *b)
{
    if (!b) return 0;
    DeviceGuard g(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    batch_drop_graph(b);
    cudaFree(b->d_sys);
    cudaFree(b->d_order);
    cudaFree(b->d_counter);
    cudaFree(b->d_info);
    cudaFree(b->d_data);
    cudaFree(b->d_orig);
    cudaFree(b->d_resid);
    cudaFree(b->d_woff);
    cudaFree(b->d_arena);
    cudaFree(b->d_iters);
    if (b->capture) cudaStreamDestroy(b->capture);
    delete b;
    return 0;
}

extern "C" int lu2gpu_batch_create(lu2gpu_ctx *c, int count, const int *n, const int *nrhs, lu2gpu_batch **out)
{
    if (!c || count <= 0 || !n || !out) {
        set_error("lu2gpu_batch_create: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    *out = nullptr;
    lu2gpu_batch *b = new lu2gpu_batch();
    b->ctx = c;
    b->count = count;
    b->sys.resize(count);
    size_t off = 0;
    for (int i = 0; i < count; i++) {
        const int ni = n[i], ri = nrhs ? nrhs[i] : 1;
        if (ni < 1 || ni > 4096 || ri < 1 || ri > 64) {
            delete b;
            set_error("lu2gpu_batch_create: system %d has n=%d nrhs=%d (1 <= n <= 4096, 1 <= nrhs <= 64)", i, ni, ri);
            return LU2GPU_ERR_ARG;
        }
        const int ld = (ni + ri + 1) & ~1;
        b->sys[i] = BatchSys{(long long)off, ni, ri, ld, 0};
        off += ((size_t)ni * ld + 1) & ~(size_t)1;  // every system starts 16-byte aligned
        if (ni > b->max_n) b->max_n = ni;
    }
    b->total = off;
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return b->sys[x].n > b->sys[y].n; });
    DeviceGuard g(c->device);
    if (cudaMalloc(&b->d_sys, sizeof(BatchSys) * count) != cudaSuccess ||
        cudaMalloc(&b->d_order, sizeof(int) * count) != cudaSuccess ||
        cudaMalloc(&b->d_counter, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->d_info, sizeof(int) * count) != cudaSuccess ||
        cudaMalloc(&b->d_resid, sizeof(double) * count) != cudaSuccess ||
        cudaMalloc(&b->d_data, sizeof(double) * b->total) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        lu2gpu_batch_destroy(b);
        set_error("lu2gpu_batch_create: device allocation of %zu bytes failed", sizeof(double) * off);
        return LU2GPU_ERR_NOMEM;
    }
    int rc = 0;
    if (cudaMemcpy(b->d_sys, b->sys.data(), sizeof(BatchSys) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->d_order, order.data(), sizeof(int) * count, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(b->d_data, 0, sizeof(double) * b->total) != cudaSuccess) {
        cudaGetLastError();
        set_error("lu2gpu_batch_create: device copy failed");
        rc = LU2GPU_ERR_CUDA;
    } else if (batch_configure(b, 256, 32, 1) != 0) {
        rc = batch_configure(b, 256, 16, 1);  // default panel width 32, 16 for larger systems
    }
    if (rc) {
        lu2gpu_batch_destroy(b);
        return rc;
    }
    *out = b;
    return 0;
}

extern "C" int lu2gpu_batch_system(lu2gpu_batch *b, int i, double **a, long *ld)
{
    if (!b || i < 0 || i >= b->count) {
        set_error("lu2gpu_batch_system: bad index");
        return LU2GPU_ERR_ARG;
    }
    if (a) *a = b->d_data + b->sys[i].off;
    if (ld) *ld = b->sys[i].ld;
    return 0;
}

extern "C" int lu2gpu_batch_generate(lu2gpu_batch *b, long seed)
{
    if (!b) return LU2GPU_ERR_ARG;
    DeviceGuard g(b->ctx->device);
    K_TRY(launch_batch_generate(b->d_data, b->d_sys, b->count, (unsigned long long)seed, nullptr, b->ctx->stream));
    CU_TRY(cudaStreamSynchronize(b->ctx->stream));
    return 0;
}

// System i := lu2's stream with seed seeds[i] (host list of count seeds): a
// shard of a larger batch generates the same systems as the whole batch would.
extern "C" int lu2gpu_batch_generate_seeds(lu2gpu_batch *b, const long long *seeds)
{
    if (!b || !seeds) {
        set_error("lu2gpu_batch_generate_seeds: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(b->ctx->device);
    long long *d = nullptr;
    if (cudaMalloc(&d, sizeof(long long) * b->count) != cudaSuccess) {
        cudaGetLastError();
        set_error("lu2gpu_batch_generate_seeds: allocation failed");
        return LU2GPU_ERR_NOMEM;
    }
    int rc = 0;
    if (cudaMemcpy(d, seeds, sizeof(long long) * b->count, cudaMemcpyHostToDevice) != cudaSuccess ||
        launch_batch_generate(b->d_data, b->d_sys, b->count, 0, d, b->ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->ctx->stream) != cudaSuccess) {
        set_error("lu2gpu_batch_generate_seeds: %s", cudaGetErrorString(cudaGetLastError()));
        rc = LU2GPU_ERR_CUDA;
    }
    cudaFree(d);
    return rc;
}

extern "C" int lu2gpu_batch_snapshot(lu2gpu_batch *b)
{
    if (!b) return LU2GPU_ERR_ARG;
    DeviceGuard g(b->ctx->device);
    if (!b->d_orig && cudaMalloc(&b->d_orig, sizeof(double) * b->total) != cudaSuccess) {
        cudaGetLastError();
        set_error("lu2gpu_batch_snapshot: allocation failed");
        return LU2GPU_ERR_NOMEM;
    }
    CU_TRY(cudaMemcpyAsync(b->d_orig, b->d_data, sizeof(double) * b->total, cudaMemcpyDeviceToDevice,
                           b->ctx->stream));
    CU_TRY(cudaStreamSynchronize(b->ctx->stream));
    return 0;
}

extern "C" int lu2gpu_batch_restore(lu2gpu_batch *b)
{
    if (!b || !b->d_orig) {
        set_error("lu2gpu_batch_restore: no snapshot");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(b->ctx->device);
    CU_TRY(cudaMemcpyAsync(b->d_data, b->d_orig, sizeof(double) * b->total, cudaMemcpyDeviceToDevice,
                           b->ctx->stream));
    return 0;
}

static int batch_enqueue(lu2gpu_batch *b, cudaStream_t st)
{
    if (b->mode == LU2GPU_BATCH_FP32_IR) {
        K_TRY(launch_batch_ir(b->d_data, b->d_sys, b->d_woff, b->d_arena, b->d_order, b->count, b->d_counter,
                              b->d_info, b->d_iters, b->smem_floats, b->pw, b->threads, b->grid, b->max_iter, st));
        return 0;
    }
    K_TRY(launch_batch_lu(b->d_data, b->d_sys, b->d_order, b->count, b->d_counter, b->d_info, b->smem_doubles, b->pw,
                          b->threads, b->grid, st));
    return 0;
}

// Select the arithmetic of lu2gpu_batch_solve: plain FP64, or FP32 factors
// with FP64 refinement (nrhs <= 8 per system) of at most max_iter corrections.
extern "C" int lu2gpu_batch_set_mode(lu2gpu_batch *b, int mode, int max_iter)
{
    if (!b || (mode != LU2GPU_BATCH_FP64 && mode != LU2GPU_BATCH_FP32_IR) || max_iter < 1) {
        set_error("lu2gpu_batch_set_mode: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(b->ctx->device);
    if (mode == LU2GPU_BATCH_FP32_IR && !b->d_arena) {
        std::vector<long long> woff(b->count);
        size_t off = 0;
        for (int i = 0; i < b->count; i++) {
            if (b->sys[i].nrhs > IR_MAX_RHS) {
                set_error("lu2gpu_batch_set_mode: system %d has %d right-hand sides (at most %d with refinement)", i,
                          b->sys[i].nrhs, IR_MAX_RHS);
                return LU2GPU_ERR_ARG;
            }
            woff[i] = (long long)off;
            off += ir_slot_bytes(b->sys[i].n, b->sys[i].nrhs);
        }
        if (cudaMalloc(&b->d_woff, sizeof(long long) * b->count) != cudaSuccess ||
            cudaMalloc(&b->d_arena, off + 256) != cudaSuccess ||
            cudaMalloc(&b->d_iters, sizeof(int) * b->count) != cudaSuccess) {
            cudaGetLastError();
            cudaFree(b->d_woff);
            cudaFree(b->d_arena);
            cudaFree(b->d_iters);
            b->d_woff = nullptr;
            b->d_arena = nullptr;
            b->d_iters = nullptr;
            set_error("lu2gpu_batch_set_mode: device allocation of %zu bytes failed", off);
            return LU2GPU_ERR_NOMEM;
        }
        CU_TRY(cudaMemcpy(b->d_woff, woff.data(), sizeof(long long) * b->count, cudaMemcpyHostToDevice));
        CU_TRY(cudaMemset(b->d_iters, 0, sizeof(int) * b->count));
    }
    const int old = b->mode;
    b->mode = mode;
    b->max_iter = max_iter;
    int rc = batch_clear_bucket_pw(b);
    if (rc) return rc;
    rc = batch_configure(b, 256, 32, 1);
    if (rc) rc = batch_configure(b, 256, 16, 1);
    if (rc) b->mode = old;
    return rc;
}

// Refinement corrections each system took in the last FP32-IR solve.
extern "C" int lu2gpu_batch_iterations(lu2gpu_batch *b, int *iters_host)
{
    if (!b || !iters_host || !b->d_iters) {
        set_error("lu2gpu_batch_iterations: no FP32-IR solve on this batch");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(b->ctx->device);
    CU_TRY(cudaMemcpy(iters_host, b->d_iters, sizeof(int) * b->count, cudaMemcpyDeviceToHost));
    return 0;
}

extern "C" int lu2gpu_batch_set_config(lu2gpu_batch *b, int threads, int pw, int ctas_per_sm)
{
    if (!b || threads < 64 || threads > 512 || (threads & 31) || pw < 16 || pw > 64 || ctas_per_sm < 1) {
        set_error("lu2gpu_batch_set_config: threads in [64,512] (multiple of 32), pw in [16,64], ctas >= 1");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(b->ctx->device);
    int rc = batch_clear_bucket_pw(b);  // one panel width for every system
    return rc ? rc : batch_configure(b, threads, pw, ctas_per_sm);
}

// Factor and solve every system in place; the launch is captured into a CUDA
// graph on the first call with the current configuration and replayed after.
extern "C" int lu2gpu_batch_solve(lu2gpu_batch *b, int *info_host)
{
    if (!b) return LU2GPU_ERR_ARG;
    DeviceGuard g(b->ctx->device);
    cudaStream_t st = b->ctx->stream;
    if (!b->exec) {
        // captured on the batch's own stream (the context's may be the legacy
        // default stream, which cannot be captured), launched on the context's
        CU_TRY(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
        int rc = batch_enqueue(b, b->capture);
        cudaGraph_t gr = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->capture, &gr);
        if (rc) {
            if (gr) cudaGraphDestroy(gr);
            return rc;
        }
        CU_TRY(e);
        b->graph = gr;
        CU_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
    }
    CU_TRY(cudaGraphLaunch(b->exec, st));
    CU_TRY(cudaStreamSynchronize(st));
    if (info_host) CU_TRY(cudaMemcpy(info_host, b->d_info, sizeof(int) * b->count, cudaMemcpyDeviceToHost));
    return 0;
}

// Size buckets of the autotuner's per-bucket panel width: n in [lo_k, lo_{k+1}).
static const int BATCH_BUCKET_LO[BATCH_BUCKETS + 1] = {1, 64, 128, 256, 1 << 30};

// Panel width pw (0: the launch's) for the blocked path of every system in
// bucket k; re-uploads the system table.
static int batch_set_bucket_pw(lu2gpu_batch *b, int k, int pw)
{
    bool changed = false;
    for (auto &S : b->sys)
        if (S.n >= BATCH_BUCKET_LO[k] && S.n < BATCH_BUCKET_LO[k + 1] && S.pw != pw) {
            S.pw = pw;
            changed = true;
        }
    b->bucket_pw[k] = pw;
    if (!changed) return 0;
    batch_drop_graph(b);
    CU_TRY(cudaMemcpy(b->d_sys, b->sys.data(), sizeof(BatchSys) * b->count, cudaMemcpyHostToDevice));
    return 0;
}

static int batch_clear_bucket_pw(lu2gpu_batch *b)
{
    for (int k = 0; k < BATCH_BUCKETS; k++) {
        int rc = batch_set_bucket_pw(b, k, 0);
        if (rc) return rc;
    }
    return 0;
}

// Median of three timed launches of the current configuration, each on the
// batch restored from its snapshot; *ms = 1e30 if a launch failed.
static int batch_time3(lu2gpu_batch *b, cudaStream_t st, cudaEvent_t e0, cudaEvent_t e1, float *ms)
{
    float t[3];
    for (int r = 0; r < 3; r++) {
        int rc = lu2gpu_batch_restore(b);
        if (rc) return rc;
        CU_TRY(cudaEventRecord(e0, st));
        if ((rc = batch_enqueue(b, st))) return rc;
        CU_TRY(cudaEventRecord(e1, st));
        CU_TRY(cudaEventSynchronize(e1));
        t[r] = 0.f;
        cudaEventElapsedTime(&t[r], e0, e1);
    }
    std::sort(t, t + 3);
    *ms = t[1];
    return 0;
}

// Time the persistent launch over launch shapes (threads per CTA, panel width,
// CTAs per SM) on this batch's own data (restored from a snapshot before every
// trial; the median of three trials per candidate) and keep the fastest; then,
// in the FP64 mode, choose the panel width of each size bucket the same way
// with the shape fixed.  params_out = {threads, pw, ctas_per_sm, best us}.
extern "C" int lu2gpu_batch_autotune(lu2gpu_batch *b, int *params_out)
{
    if (!b) return LU2GPU_ERR_ARG;
    DeviceGuard g(b->ctx->device);
    int rc = lu2gpu_batch_snapshot(b);
    if (rc) return rc;
    if ((rc = batch_clear_bucket_pw(b))) return rc;
    cudaStream_t st = b->ctx->stream;
    const int cand_threads[3] = {128, 256, 512}, cand_pw[3] = {16, 32, 64}, cand_ctas[2] = {1, 2};
    float best = 1e30f;
    int bt = b->threads, bp = b->pw, bc = b->ctas_per_sm;
    cudaEvent_t e0, e1;
    CU_TRY(cudaEventCreate(&e0));
    CU_TRY(cudaEventCreate(&e1));
    for (int ti = 0; ti < 3 && !rc; ti++)
        for (int pi = 0; pi < 3 && !rc; pi++)
            for (int ci = 0; ci < 2 && !rc; ci++) {
                if (batch_configure(b, cand_threads[ti], cand_pw[pi], cand_ctas[ci])) continue;  // does not fit
                float ms = 0.f;
                if ((rc = batch_time3(b, st, e0, e1, &ms))) break;
                if (ms < best) {
                    best = ms;
                    bt = b->threads;
                    bp = b->pw;
                    bc = b->ctas_per_sm;
                }
            }
    if (!rc) rc = batch_configure(b, bt, bp, bc);
    if (!rc && b->mode == LU2GPU_BATCH_FP64) {
        // per size bucket (largest first), the launch's panel width or another
        for (int k = BATCH_BUCKETS - 1; k >= 0 && !rc; k--) {
            bool any = false;
            for (const auto &S : b->sys) any |= (S.n >= BATCH_BUCKET_LO[k] && S.n < BATCH_BUCKET_LO[k + 1]);
            if (!any) continue;
            int keep = 0;
            for (int pi = 0; pi < 3 && !rc; pi++) {
                if (cand_pw[pi] == bp) continue;  // the launch's width is the time already measured
                if ((rc = batch_set_bucket_pw(b, k, cand_pw[pi]))) break;
                if (batch_configure(b, bt, bp, bc)) continue;  // does not fit
                float ms = 0.f;
                if ((rc = batch_time3(b, st, e0, e1, &ms))) break;
                if (ms < 0.99f * best) {  // a bucket leaves the launch's width only for a clear gain
                    best = ms;
                    keep = cand_pw[pi];
                }
            }
            if (!rc) rc = batch_set_bucket_pw(b, k, keep);
            if (!rc) rc = batch_configure(b, bt, bp, bc);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if ((rc = lu2gpu_batch_restore(b))) return rc;
    CU_TRY(cudaStreamSynchronize(st));
    if (params_out) {
        params_out[0] = bt;
        params_out[1] = bp;
        params_out[2] = bc;
        params_out[3] = (int)(best * 1000.f);
    }
    return 0;
}

// The panel width the autotuner chose for each size bucket: out[2k] = the
// smallest n of bucket k, out[2k+1] = its panel width (0: the launch's).
extern "C" int lu2gpu_batch_bucket_pw(lu2gpu_batch *b, int *out)
{
    if (!b || !out) {
        set_error("lu2gpu_batch_bucket_pw: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    for (int k = 0; k < BATCH_BUCKETS; k++) {
        out[2 * k] = BATCH_BUCKET_LO[k];
        out[2 * k + 1] = b->bucket_pw[k];
    }
    return 0;
}

extern "C" int lu2gpu_batch_residuals(lu2gpu_batch *b, double *out_host)
{
    if (!b || !b->d_orig || !out_host) {
        set_error("lu2gpu_batch_residuals: needs a snapshot of the original systems");
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(b->ctx->device);
    K_TRY(launch_batch_residual(b->d_orig, b->d_data, b->d_sys, b->count, b->d_resid, b->ctx->stream));
    CU_TRY(cudaStreamSynchronize(b->ctx->stream));
    CU_TRY(cudaMemcpy(out_host, b->d_resid, sizeof(double) * b->count, cudaMemcpyDeviceToHost));
    return 0;
}

// The batch of the benchmark: n_i log-uniform in [nmin, nmax] and, for a
// fraction frac_multi of the systems, nrhs_multi right-hand sides (else one),
// from the 48-bit drand48 stream seeded with `seed`.
extern "C" int lu2gpu_batch_sizes(int count, long seed, int nmin, int nmax, double frac_multi, int nrhs_multi,
                                  int *n_out, int *nrhs_out)
{
    if (count <= 0 || nmin < 1 || nmax < nmin || !n_out || !nrhs_out) {
        set_error("lu2gpu_batch_sizes: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    unsigned long long x = ((((unsigned long long)seed) & 0xffffffffull) << 16) | 0x330Eull;
    auto next = [&]() {
        x = (0x5DEECE66Dull * x + 0xBull) & ((1ull << 48) - 1);
        return (double)x * (1.0 / 281474976710656.0);
    };
    const double l0 = log((double)nmin), l1 = log((double)nmax + 1.0);
    for (int i = 0; i < count; i++) {
        int ni = (int)floor(exp(l0 + next() * (l1 - l0)));
        if (ni < nmin) ni = nmin;
        if (ni > nmax) ni = nmax;
        n_out[i] = ni;
        nrhs_out[i] = (next() < frac_multi) ? nrhs_multi : 1;
    }
    return 0;
}

// lumcolumn's panel loop (lu2.c:1126-1141) on the FP32 working matrix
static int factor32_serial(lu2gpu_ctx *c, const View32 &v, int n, int nb, int mode)
{
    for (int i = 0; i < n; i += nb) {
        const int w = (n - i) < nb ? (n - i) : nb;
        int rc = panel32(c, v, i, w, mode);
        if (rc) return rc;
        if ((rc = right_part32(c, v, i, i + w, i + w, n, true))) return rc;
    }
    return 0;
}

// Lookahead (the reference's lu_mpi_blocked_lookahead idea, lu2_mpi.c:3643-
// 3847, on one GPU): step k updates the next panel's columns first, then the
// next panel is factored on a second stream while the rest of the update runs.
// The persistent update kernel is held to sms - R CTAs (one per SM, by its
// shared memory), which leaves R SMs for the panel's leaf CTAs (R = the
// fewest CTAs whose FP32 slab fits, at least 32).  Step k+1's right part waits
// for that panel: its row exchanges cross the columns the update wrote.
// Serial when phase timing is on (so the phase split stays meaningful), for
// small n, or with LU2GPU_LOOKAHEAD=0.
static int factor32_or_fail(lu2gpu_ctx *c, int n, float *a, long ld, int nb, int mode)
{
    View32 v{a, ld, n, n, 0};
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
    // SMs held for the panel beside the update (LU2GPU_PANEL_SMS, read per
    // call; N=65536 BF16 factor: 24 SMs 1.002 s, 32 0.996 s, 48 1.018 s)
    const char *ps = getenv("LU2GPU_PANEL_SMS");
    const int R = std::max(ps ? atoi(ps) : 32, leaf_min_ctas(n, sizeof(float)));
    const char *env = getenv("LU2GPU_LOOKAHEAD");
    const bool lookahead = !c->timing && n >= 4 * nb && 2 * R < sms && !(env && env[0] == '0');
    if (!lookahead) return factor32_serial(c, v, n, nb, mode);
    MixedWork *m = c->mx;
    if (!m->side) {
        CU_TRY(cudaStreamCreateWithFlags(&m->side, cudaStreamNonBlocking));
        CU_TRY(cudaEventCreateWithFlags(&m->ev_cols, cudaEventDisableTiming));
        CU_TRY(cudaEventCreateWithFlags(&m->ev_panel, cudaEventDisableTiming));
    }
    const cudaStream_t main_st = c->stream;
    const int all_ctas = c->leaf_ctas;
    int rc = panel32(c, v, 0, std::min(nb, n), mode);  // the first panel, on the main stream
    for (int i = 0; rc == 0 && i < n; i += nb) {
        const int w = std::min(nb, n - i), i1 = i + w, w1 = std::min(nb, n - i1);
        if (i > 0 && cudaStreamWaitEvent(main_st, m->ev_panel, 0) != cudaSuccess) {
            set_error("lookahead: cudaStreamWaitEvent failed");
            rc = LU2GPU_ERR_CUDA;
            break;
        }
        auto next_panel = [&]() -> int {
            if (i1 >= n) return 0;
            CU_TRY(cudaEventRecord(m->ev_cols, main_st));
            CU_TRY(cudaStreamWaitEvent(m->side, m->ev_cols, 0));
            c->stream = m->side;
            c->leaf_ctas = std::min(all_ctas, R);
            const int r = panel32(c, v, i1, w1, mode);
            c->stream = main_st;
            c->leaf_ctas = all_ctas;
            if (r) return r;
            CU_TRY(cudaEventRecord(m->ev_panel, m->side));
            return 0;
        };
        rc = right_part32_split(c, v, i, i1, i1, n, w1, sms - R, next_panel);
    }
    c->stream = main_st;
    c->leaf_ctas = all_ctas;
    // everything on the side stream precedes what follows on the main stream
    if (cudaEventRecord(m->ev_panel, m->side) != cudaSuccess ||
        cudaStreamWaitEvent(main_st, m->ev_panel, 0) != cudaSuccess) {
        cudaGetLastError();
        if (!rc) {
            set_error("lookahead: joining the panel stream failed");
            rc = LU2GPU_ERR_CUDA;
        }
    }
    return rc;
}

extern "C" int lu2gpu_mixed_solve(lu2gpu_ctx *c, int n, const double *a, long lda, const double *b, double *x, int nb,
                                  int pivot_mode, int max_iter, double *out)
{
    if (!c || n <= 0 || !a || !b || !x || lda < n || max_iter < 1) {
        set_error("lu2gpu_mixed_solve: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    if ((lda & 1) || (reinterpret_cast<uintptr_t>(a) & 15)) {
        set_error("lu2gpu_mixed_solve: A must be 16-byte aligned with an even row stride");
        return LU2GPU_ERR_ARG;
    }
    if (nb < 64 || nb > 256 || (nb % 64)) {
        set_error("lu2gpu_mixed_solve: nb=%d must be 64, 128, 192 or 256 (the BF16 update's K)", nb);
        return LU2GPU_ERR_ARG;
    }
    if (pivot_mode != LU2GPU_PIVOT_REF && pivot_mode != LU2GPU_PIVOT_PARTIAL) {
        set_error("unknown pivot mode %d", pivot_mode);
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    const long ld32 = ((long)n + 31) & ~31L;
    int rc = mixed_work(c, n, ld32, nb);
    if (rc) return rc;
    MixedWork *m = c->mx;
    m->update = LU2GPU_UPDATE_BF16;
    double *r = m->vec + n, *rowabs = m->vec + 2 * (size_t)n;
    float *v32 = reinterpret_cast<float *>(m->vec + 3 * (size_t)n);
    cudaEvent_t ev[3];
    for (int i = 0; i < 3; i++) CU_TRY(cudaEventCreate(&ev[i]));
    if ((rc = begin_status(c))) return rc;
    CU_TRY(cudaEventRecord(ev[0], c->stream));
    K_TRY(launch_f64_to_f32(a, lda, m->a32, ld32, n, n, c->stream));
    if ((rc = factor32_or_fail(c, n, m->a32, ld32, nb, pivot_mode))) return rc;
    CU_TRY(cudaEventRecord(ev[1], c->stream));

    // refinement: x_0 = 0, r_0 = b; d = LU^{-1} r (FP32), x += d, r = b - A x (FP64)
    CU_TRY(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), c->stream));
    CU_TRY(cudaMemcpyAsync(r, b, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    const double eps = 1.1102230246251565e-16;  // 2^-53
    double hpl = 0, norms_h[4] = {0, 0, 0, 0};
    int it = 0;
    for (it = 1; it <= max_iter; it++) {
        K_TRY(launch_f64_to_f32(r, 1, v32, 1, n, 1, c->stream));
        if ((rc = solve32_enqueue(c, n, m->a32, ld32, nb, v32))) return rc;
        K_TRY(launch_add_f32_to_f64(v32, x, n, c->stream));
        K_TRY(launch_residual(a, lda, n, b, x, r, it == 1 ? rowabs : nullptr, c->stream));
        CU_TRY(cudaMemsetAsync(m->norms(), 0, (it == 1 ? 4 : 2) * sizeof(unsigned long long), c->stream));
        K_TRY(launch_vec_absmax(r, n, m->norms(), c->stream));
        K_TRY(launch_vec_absmax(x, n, m->norms() + 1, c->stream));
        if (it == 1) {
            K_TRY(launch_vec_absmax(b, n, m->norms() + 2, c->stream));
            K_TRY(launch_vec_absmax(rowabs, n, m->norms() + 3, c->stream));
        }
        unsigned long long nb_h[4];
        CU_TRY(cudaMemcpyAsync(nb_h, m->norms(), (it == 1 ? 4 : 2) * sizeof(unsigned long long),
                               cudaMemcpyDeviceToHost, c->stream));
        CU_TRY(cudaStreamSynchronize(c->stream));
        for (int q = 0; q < (it == 1 ? 4 : 2); q++) memcpy(&norms_h[q], &nb_h[q], sizeof(double));
        hpl = norms_h[0] / (eps * (norms_h[3] * norms_h[1] + norms_h[2]) * n);
        if (hpl < 16.0) break;
    }
    if (it > max_iter) it = max_iter;
    CU_TRY(cudaEventRecord(ev[2], c->stream));
    rc = end_status(c, "lu2gpu_mixed_solve");
    float t_fac = 0, t_ir = 0;
    cudaEventElapsedTime(&t_fac, ev[0], ev[1]);
    cudaEventElapsedTime(&t_ir, ev[1], ev[2]);
    for (int i = 0; i < 3; i++) cudaEventDestroy(ev[i]);
    if (out) {
        out[0] = it;
        out[1] = hpl;
        out[2] = t_fac * 1e-3;
        out[3] = t_ir * 1e-3;
    }
    if (rc) return rc;
    if (hpl >= 16.0) {
        set_error("lu2gpu_mixed_solve: refinement did not reach a scaled residual < 16 in %d iterations (%.3g)",
                  max_iter, hpl);
        return LU2GPU_ERR_NOCONV;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// GMRES-IR

// z = U^{-1} L^{-1} P w with the FP32 factors (FP64 vectors in and out)
static int precond_apply(lu2gpu_ctx *c, int n, long ld32, int nb, const double *w, double *z)
{
    MixedWork *m = c->mx;
    float *v32 = reinterpret_cast<float *>(m->vec + 3 * (size_t)n);
    K_TRY(launch_f64_to_f32(w, 1, v32, 1, n, 1, c->stream));
    int rc = solve32_enqueue(c, n, m->a32, ld32, nb, v32);
    if (rc) return rc;
    K_TRY(launch_f32_to_f64(v32, 1, z, 1, n, 1, c->stream));
    return 0;
}

// The precision forms' factorization on its own (what lu2gpu_mixed_solve and
// lu2gpu_gmres_solve precondition with): lu2's LU of an FP32 copy of a, the
// panels in FP32, the top-level trailing updates with BF16 or E4M3 operands.
extern "C" int lu2gpu_lowp_factor(lu2gpu_ctx *c, int n, const double *a, long lda, int nb, int update,
                                  float *f, long ldf, int *ipiv)
{
    if (!c || n <= 0 || !a || lda < n || !f || ldf < n) {
        set_error("lu2gpu_lowp_factor: bad arguments");
        return LU2GPU_ERR_ARG;
    }
    if ((lda & 1) || (reinterpret_cast<uintptr_t>(a) & 15)) {
        set_error("lu2gpu_lowp_factor: A must be 16-byte aligned with an even row stride");
        return LU2GPU_ERR_ARG;
    }
    if (!((update == LU2GPU_UPDATE_BF16 && nb >= 64 && nb <= 256 && nb % 64 == 0) ||
          (update == LU2GPU_UPDATE_FP8 && (nb == 128 || nb == 256)))) {
        set_error("lu2gpu_lowp_factor: update %d with nb=%d (BF16: 64..256 step 64; FP8: 128 or 256)", update, nb);
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    const long ld32 = ((long)n + 31) & ~31L;
    int rc = mixed_work(c, n, ld32, nb);
    if (rc) return rc;
    MixedWork *m = c->mx;
    m->update = update;
    if (update == LU2GPU_UPDATE_FP8 && (rc = fp8_work(c, n, nb))) return rc;
    if ((rc = begin_status(c))) return rc;
    K_TRY(launch_f64_to_f32(a, lda, m->a32, ld32, n, n, c->stream));
    if ((rc = factor32_or_fail(c, n, m->a32, ld32, nb, LU2GPU_PIVOT_PARTIAL))) return rc;
    CU_TRY(cudaMemcpy2DAsync(f, (size_t)ldf * sizeof(float), m->a32, (size_t)ld32 * sizeof(float),
                             (size_t)n * sizeof(float), n, cudaMemcpyDeviceToDevice, c->stream));
    if (ipiv) CU_TRY(cudaMemcpyAsync(ipiv, c->d_ipiv, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, c->stream));
    return end_status(c, "lu2gpu_lowp_factor");
}

extern "C" int lu2gpu_gmres_solve(lu2gpu_ctx *c, int n, const double *a, long lda, const double *b, double *x, int nb,
                                  int update, int restart, double inner_tol, int max_iter, double *out)
{
    if (!c || n <= 0 || !a || !b || !x || lda < n || restart < 1 || restart > 32 || max_iter < 1 ||
        !(inner_tol > 0.0 && inner_tol < 1.0)) {
        set_error("lu2gpu_gmres_solve: bad arguments (restart in [1, 32], max_iter >= 1, 0 < inner_tol < 1)");
        return LU2GPU_ERR_ARG;
    }
    if ((lda & 1) || (reinterpret_cast<uintptr_t>(a) & 15)) {
        set_error("lu2gpu_gmres_solve: A must be 16-byte aligned with an even row stride");
        return LU2GPU_ERR_ARG;
    }
    if (update == LU2GPU_UPDATE_BF16) {
        if (nb < 64 || nb > 256 || (nb % 64)) {
            set_error("lu2gpu_gmres_solve: nb=%d must be 64, 128, 192 or 256 for the BF16 update", nb);
            return LU2GPU_ERR_ARG;
        }
    } else if (update == LU2GPU_UPDATE_FP8) {
        if (nb != 128 && nb != 256) {
            set_error("lu2gpu_gmres_solve: nb=%d must be 128 or 256 for the FP8 update", nb);
            return LU2GPU_ERR_ARG;
        }
    } else {
        set_error("lu2gpu_gmres_solve: unknown update precision %d", update);
        return LU2GPU_ERR_ARG;
    }
    DeviceGuard g(c->device);
    const long ld32 = ((long)n + 31) & ~31L;
    int rc = mixed_work(c, n, ld32, nb);
    if (rc) return rc;
    MixedWork *m = c->mx;
    m->update = update;
    if (update == LU2GPU_UPDATE_FP8 && (rc = fp8_work(c, n, nb))) return rc;
    const long ldv = ((long)n + 31) & ~31L;
    const size_t gm_doubles = (size_t)(restart + 1 + 4) * ldv + 64 * MULTI_DOT_BLOCKS + 256;
    if ((rc = grow((void **)&m->gm, &m->gm_cap, gm_doubles * sizeof(double)))) return rc;
    double *V = m->gm, *w = V + (size_t)(restart + 1) * ldv, *z = w + ldv, *d = z + ldv, *t = d + ldv;
    double *partial = t + ldv, *dots = partial + 64 * MULTI_DOT_BLOCKS;  // dots: h[32] h2[32] |z|^2 . y[32] one
    double *r = m->vec + n, *rowabs = m->vec + 2 * (size_t)n;
    cudaEvent_t ev[3];
    for (int i = 0; i < 3; i++) CU_TRY(cudaEventCreate(&ev[i]));
    if ((rc = begin_status(c))) return rc;
    CU_TRY(cudaEventRecord(ev[0], c->stream));
    K_TRY(launch_f64_to_f32(a, lda, m->a32, ld32, n, n, c->stream));
    if ((rc = factor32_or_fail(c, n, m->a32, ld32, nb, LU2GPU_PIVOT_PARTIAL))) return rc;
    CU_TRY(cudaEventRecord(ev[1], c->stream));

    const double one = 1.0;
    CU_TRY(cudaMemcpyAsync(dots + 128, &one, sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CU_TRY(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), c->stream));
    K_TRY(launch_residual(a, lda, n, b, x, r, rowabs, c->stream));  // r = b, row sums of |A|
    CU_TRY(cudaMemsetAsync(m->norms(), 0, 4 * sizeof(unsigned long long), c->stream));
    K_TRY(launch_vec_absmax(b, n, m->norms() + 2, c->stream));
    K_TRY(launch_vec_absmax(rowabs, n, m->norms() + 3, c->stream));
    const double eps = 1.1102230246251565e-16;  // 2^-53
    double bnorm = 0, anorm = 0;
    auto hpl_now = [&](double *h) -> int {
        CU_TRY(cudaMemsetAsync(m->norms(), 0, 2 * sizeof(unsigned long long), c->stream));
        K_TRY(launch_vec_absmax(r, n, m->norms(), c->stream));
        K_TRY(launch_vec_absmax(x, n, m->norms() + 1, c->stream));
        unsigned long long nb_h[4];
        CU_TRY(cudaMemcpyAsync(nb_h, m->norms(), 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
        CU_TRY(cudaStreamSynchronize(c->stream));
        double v[4];
        memcpy(v, nb_h, sizeof(v));
        bnorm = v[2];
        anorm = v[3];
        *h = v[0] / (eps * (anorm * v[1] + bnorm) * n);
        return 0;
    };
    // |z| on the host (one dot product)
    auto norm_of = [&](const double *vec, double *nrm) -> int {
        K_TRY(launch_multi_dot(vec, ldv, 1, vec, n, partial, dots + 64, c->stream));
        double s = 0;
        CU_TRY(cudaMemcpyAsync(&s, dots + 64, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CU_TRY(cudaStreamSynchronize(c->stream));
        *nrm = sqrt(s);
        return 0;
    };

    double H[33][32], cs[32], sn[32], gvec[33], hpl = 0;
    int total = 0, outer = 0;
    bool finite = true;  // the preconditioner maps finite vectors to finite vectors
    for (;;) {
        if ((rc = hpl_now(&hpl))) return rc;
        if (hpl < 16.0 || total >= max_iter) break;
        outer++;
        // correction equation A d = r, left-preconditioned: M^{-1} A d = M^{-1} r
        CU_TRY(cudaMemsetAsync(d, 0, (size_t)n * sizeof(double), c->stream));
        if ((rc = precond_apply(c, n, ld32, nb, r, z))) return rc;
        double beta0 = 0;
        if ((rc = norm_of(z, &beta0))) return rc;
        if (!std::isfinite(beta0)) {  // the FP32 solve with the low-precision factors overflowed
            finite = false;
            break;
        }
        if (!(beta0 > 0.0)) break;  // r = 0
        double beta = beta0;
        bool conv = false;
        while (!conv && total < max_iter) {
            K_TRY(launch_vec_scale(z, 1.0 / beta, V, n, c->stream));
            for (int i = 0; i <= restart; i++) gvec[i] = 0.0;
            gvec[0] = beta;
            int k = 0;
            while (k < restart && total < max_iter) {
                double *vk = V + (size_t)k * ldv;
                K_TRY(launch_residual(a, lda, n, nullptr, vk, w, nullptr, c->stream));  // w = A v_k
                if ((rc = precond_apply(c, n, ld32, nb, w, z))) return rc;
                // classical Gram-Schmidt, twice
                K_TRY(launch_multi_dot(V, ldv, k + 1, z, n, partial, dots, c->stream));
                K_TRY(launch_multi_axpy(V, ldv, k + 1, dots, -1.0, z, n, c->stream));
                K_TRY(launch_multi_dot(V, ldv, k + 1, z, n, partial, dots + 32, c->stream));
                K_TRY(launch_multi_axpy(V, ldv, k + 1, dots + 32, -1.0, z, n, c->stream));
                K_TRY(launch_multi_dot(z, ldv, 1, z, n, partial, dots + 64, c->stream));
                double hd[65];
                CU_TRY(cudaMemcpyAsync(hd, dots, 65 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
                CU_TRY(cudaStreamSynchronize(c->stream));
                total++;
                for (int j = 0; j <= k; j++) H[j][k] = hd[j] + hd[32 + j];
                const double hk1 = sqrt(hd[64] > 0 ? hd[64] : 0.0);
                // previous rotations, then the one that zeroes H[k+1][k]
                for (int j = 0; j < k; j++) {
                    const double t0 = cs[j] * H[j][k] + sn[j] * H[j + 1][k];
                    H[j + 1][k] = -sn[j] * H[j][k] + cs[j] * H[j + 1][k];
                    H[j][k] = t0;
                }
                const double den = hypot(H[k][k], hk1);
                cs[k] = den > 0 ? H[k][k] / den : 1.0;
                sn[k] = den > 0 ? hk1 / den : 0.0;
                H[k][k] = den;
                gvec[k + 1] = -sn[k] * gvec[k];
                gvec[k] = cs[k] * gvec[k];
                k++;
                if (fabs(gvec[k]) <= inner_tol * beta0 || !(hk1 > 0.0)) {
                    conv = true;
                    break;
                }
                if (k < restart) K_TRY(launch_vec_scale(z, 1.0 / hk1, V + (size_t)k * ldv, n, c->stream));
            }
            // y = H(0:k, 0:k)^{-1} g(0:k); d += V y
            double y[32];
            for (int i = k - 1; i >= 0; i--) {
                double s = gvec[i];
                for (int j = i + 1; j < k; j++) s -= H[i][j] * y[j];
                y[i] = H[i][i] != 0.0 ? s / H[i][i] : 0.0;
            }
            if (k > 0) {
                CU_TRY(cudaMemcpy(dots + 96, y, (size_t)k * sizeof(double), cudaMemcpyHostToDevice));
                K_TRY(launch_multi_axpy(V, ldv, k, dots + 96, 1.0, d, n, c->stream));
            }
            if (!conv && total < max_iter) {
                // restart from the true correction residual r - A d
                K_TRY(launch_residual(a, lda, n, r, d, t, nullptr, c->stream));
                if ((rc = precond_apply(c, n, ld32, nb, t, z))) return rc;
                if ((rc = norm_of(z, &beta))) return rc;
                if (!(beta > inner_tol * beta0)) conv = true;
            }
        }
        K_TRY(launch_multi_axpy(d, ldv, 1, dots + 128, 1.0, x, n, c->stream));  // x += d
        K_TRY(launch_residual(a, lda, n, b, x, r, nullptr, c->stream));         // r = b - A x
    }
    CU_TRY(cudaEventRecord(ev[2], c->stream));
    rc = end_status(c, "lu2gpu_gmres_solve");
    float t_fac = 0, t_ir = 0;
    cudaEventElapsedTime(&t_fac, ev[0], ev[1]);
    cudaEventElapsedTime(&t_ir, ev[1], ev[2]);
    for (int i = 0; i < 3; i++) cudaEventDestroy(ev[i]);
    if (out) {
        out[0] = outer;
        out[1] = total;
        out[2] = hpl;
        out[3] = t_fac * 1e-3;
        out[4] = t_ir * 1e-3;
        out[5] = finite ? 1.0 : 0.0;
    }
    if (rc) return rc;
    if (!finite) {
        set_error("lu2gpu_gmres_solve: applying the low-precision factors overflowed FP32 (their pivots grew "
                  "geometrically: the low-precision updates are too coarse for this matrix); no refinement possible");
        return LU2GPU_ERR_NOCONV;
    }
    if (!(hpl < 16.0)) {
        set_error("lu2gpu_gmres_solve: scaled residual %.3g after %d GMRES iterations (%d refinement steps)", hpl,
                  total, outer);
        return LU2GPU_ERR_NOCONV;
    }
    return 0;
}

extern "C" int lu2gpu_fp8_update_dev(lu2gpu_ctx *c, int M, int N, int K, const float *a, long lda, const float *bt,
                                     long ldb, float *c32, long ldc, float *a_deq, float *bt_deq)
{
    if (!c || M < 0 || N < 0 || (K != 128 && K != 256) || !a || !bt || !c32 || lda < K || ldb < K || (lda & 3) ||
        (ldb & 3) || (reinterpret_cast<uintptr_t>(a) & 15) || (reinterpret_cast<uintptr_t>(bt) & 15)) {
        set_error("lu2gpu_fp8_update_dev: bad arguments (K must be 128 or 256, strides multiples of 4, "
                  "16-byte aligned operands)");
        return LU2GPU_ERR_ARG;
    }
    if (M == 0 || N == 0) return 0;
    DeviceGuard g(c->device);
    int rc = ensure_work(c, 16, 16, 16);
    if (rc) return rc;
    double *s0, *s1, *s2;
    const size_t tm = ((size_t)M + 127) / 128, tn = ((size_t)N + 127) / 128;
    if ((rc = stage(c, 0, ((size_t)M * K + 7) / 8, &s0)) || (rc = stage(c, 1, ((size_t)N * K + 7) / 8, &s1)) ||
        (rc = stage(c, 2, (tm + tn) * (K / 128), &s2)))
        return rc;
    uint8_t *a8 = reinterpret_cast<uint8_t *>(s0), *b8 = reinterpret_cast<uint8_t *>(s1);
    float *dqa = reinterpret_cast<float *>(s2), *dqb = dqa + tm * (K / 128);
    if ((rc = begin_status(c))) return rc;
    K_TRY(launch_quant_fp8_tiles(a, lda, M, K, a8, K, dqa, c->stream));
    K_TRY(launch_quant_fp8_tiles(bt, ldb, N, K, b8, K, dqb, c->stream));
    if (a_deq) K_TRY(launch_dequant_fp8_tiles(a8, K, dqa, M, K, a_deq, K, c->stream));
    if (bt_deq) K_TRY(launch_dequant_fp8_tiles(b8, K, dqb, N, K, bt_deq, K, c->stream));
    K_TRY(launch_lowp_update_fp8(a8, K, dqa, b8, K, dqb, c32, ldc, M, N, K, c->d_status, 0, c->stream));
    return end_status(c, "lu2gpu_fp8_update_dev");
}
