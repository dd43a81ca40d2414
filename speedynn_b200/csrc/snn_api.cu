// snn_api.cu -- host driver and C ABI of libspeedynn_b200.so.
//
// The greedy loop of speedynn/lib/nearest_neighbors_feature_selection.c:76-233
// (backward) and :243-394 (forward) runs here as a fixed sequence of kernel
// launches per step on one CUDA stream: score -> reduce -> select -> commit.
// The winner never travels to the host between steps (the select kernel
// writes it to device state that the commit and the next scoring read), so a
// whole selection is issued without synchronisation and waited for once.
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/speedynn_b200.h"
#include "snn_internal.h"

using snn::Bufs;
using snn::State;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define SNN_CUDA(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(SNN_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                                           __FILE__, __LINE__);                                         \
    } while (0)

inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

struct EventPair {
    cudaEvent_t a = nullptr, b = nullptr;
};

}  // namespace

namespace snn {
// Record a failure for snn_last_error() from another translation unit.
int record_error(int code, const char *msg)
{
    g_err = msg;
    return code;
}
void clear_error() { g_err.clear(); }
}  // namespace snn

struct snn_handle {
    snn_desc desc{};
    std::vector<int> kvals;
    int n_rows = 0, n_cols = 0, p = 0, cv = 0, npf = 1, kmax = 0, nk = 0;
    int ldc = 0, ldr = 0;
    int total_steps = 0;
    snn::ScorePlan plan{0, 0, 0};
    int device = 0;
    cudaStream_t stream = nullptr;
    // device buffers
    float *XT = nullptr, *XV = nullptr, *yc = nullptr, *yr = nullptr, *D = nullptr, *pred = nullptr;
    float *rmse32 = nullptr, *err = nullptr, *stage = nullptr;
    double *rmse64 = nullptr, *err64 = nullptr;
    int *kv = nullptr, *cands = nullptr, *prev_cands = nullptr, *mask = nullptr, *order = nullptr, *stepk = nullptr;
    int *perm = nullptr;           // candidate slot order: ascending training variance
    float *fvar = nullptr;         // per-feature training variance
    // model: regression (kNN mean) or classification (mode), and the losses
    int model = 0;
    std::vector<int> loss_ids{0};  // reference loss ids; [0] decides
    int *d_loss_ids = nullptr;
    float *lossval = nullptr, *err_all = nullptr;
    float *kth_prev = nullptr;     // backward: last step's k-th distances [p][n_rows]
    float *dmax = nullptr;         // backward: per row, the largest finite entry of the full D
    bool prev_ok = false;          // kth_prev holds the previous step's values
    int inject_stall = -1;         // fault injection (see dev_alloc): stage to withhold once
    int inject_launch = -1;        // fault injection: greedy step whose launch fails once
    bool extra_losses() const { return !(loss_ids.size() == 1 && loss_ids[0] == 0); }
    State *st = nullptr;
    // forward: seed columns of each row under the committed D (written by the
    // commit before a seeded step) and their distances, [n_rows][kSeeds]
    int *seeds = nullptr;
    float *seed_d = nullptr;
    float *sbound = nullptr;      // [p][n_rows] starting bounds of a seeded step
    // forward holdout: training values of each feature sorted ([p][ldc], with
    // their column indices) for the first step, and the sort's work buffers
    float *sval = nullptr, *skey = nullptr;
    int *sidx = nullptr, *sord = nullptr, *soff = nullptr;
    char *stemp = nullptr;
    size_t stemp_bytes = 0;
    unsigned long long *walked = nullptr;  // columns walked by the sorted second step
    bool sorted_start = true;     // SNN_OPT_SORTED_START
    bool seeds_ok = false;        // seeds hold the current D's seed columns
    int seed_step = 2;            // SNN_OPT_SEED_STEP: first forward step scored from seed bounds (set at create)
    unsigned long long *fcount = nullptr;  // filter counters of the TMA-fed scorer (3)
    bool count_filter = false;             // SNN_OPT_COUNTERS
    int kernel = 0;               // scoring kernel: 0 auto, 1 rows per lane, 3 TMA-fed row tiles
    int max_smem = 0;
    int *nn_idx = nullptr;
    float *nn_dist = nullptr;
    bool keep_nn = false;
    int nn_ncand = 0;
    int last_ncand = 0;  // candidates of the most recent scored step (prediction slots)
    bool loaded = false;
    int host_step = 0;  // steps issued since the last reset
    // timing
    bool step_events = true;  // per-step CUDA events (off for batch problems: only total_ev is read)
    bool arena = false;       // device buffers are sub-allocations of a batch arena (never freed one by one)
    std::vector<EventPair> score_ev, commit_ev;
    EventPair total_ev;
    EventPair setup_ev;  // the last reset's initial distance matrix (full distance or empty)
    bool setup_timed = false;
    int n_score = 0, n_commit = 0, n_launch = 0;

    Bufs bufs() const
    {
        Bufs b;
        b.XT = XT;
        b.XV = XV;
        b.ldc = ldc;
        b.ldr = ldr;
        b.yc = yc;
        b.yr = yr;
        b.D = D;
        b.n_rows = n_rows;
        b.n_cols = n_cols;
        b.p = p;
        b.kvals = kv;
        b.nk = nk;
        b.kmax = kmax;
        b.pred = pred;
        b.rmse32 = rmse32;
        b.rmse64 = rmse64;
        b.cands = cands;
        b.prev_cands = prev_cands;
        b.perm = perm;
        b.mask = mask;
        b.order = order;
        b.err = err;
        b.err64 = err64;
        b.stepk = stepk;
        b.st = st;
        // classification predicts from the neighbour lists, so it always keeps them
        b.nn_idx = keep_nn || model == 1 ? nn_idx : nullptr;
        b.nn_dist = keep_nn || model == 1 ? nn_dist : nullptr;
        b.nloss = extra_losses() ? (int)loss_ids.size() : 0;
        b.loss_ids = d_loss_ids;
        b.lossval = lossval;
        b.err_all = err_all;
        b.kth_prev = kth_prev;
        b.use_prev = 0;
        b.dmax = dmax;
        b.inject_stall = 0;
        b.fcount = count_filter ? fcount : nullptr;
        b.seeds = seeds;
        b.seed_d = seed_d;
        b.bound = sbound;
        b.use_seeds = 0;
        b.only_if_full = 0;
        return b;
    }
};

namespace {

// Fault injection for tests (environment, read by snn_create; each fires once):
//   SNN_INJECT_FAIL=alloc:N   the N-th device allocation of that snn_create fails (SNN_ERR_NOMEM)
//   SNN_INJECT_FAIL=launch:N  the scoring launch of greedy step N fails (SNN_ERR_CUDA)
//   SNN_INJECT_STALL=N        block 0 of the next TMA-fed scoring launch never issues the copies
//                             of stage N, so its bounded waits run out (SNN_ERR_TIMEOUT)
thread_local int t_fail_alloc = 0;  // countdown to the injected allocation failure, 0 = off

// Bump allocator over one device allocation: while a batch creates and loads
// the problems of a wave on this thread, their buffers are carved from it
// (one cudaMalloc per batch run instead of a score per problem; cudaFree
// also waits for the whole device).  256-byte aligned sub-allocations.
struct Arena {
    char *base = nullptr;
    size_t cap = 0, used = 0;
};
thread_local Arena *t_arena = nullptr;

template <typename T>
int dev_alloc(T **p, size_t n, const char *what)
{
    *p = nullptr;
    if (t_fail_alloc > 0 && --t_fail_alloc == 0) return fail(SNN_ERR_NOMEM, "injected failure of the allocation of %s", what);
    if (n == 0) n = 1;
    if (t_arena) {
        const size_t off = (t_arena->used + 255) & ~(size_t)255;
        const size_t bytes = n * sizeof(T);
        if (off > t_arena->cap || bytes > t_arena->cap - off)
            return fail(SNN_ERR_NOMEM, "batch arena full at %s (%zu bytes)", what, bytes);
        *p = reinterpret_cast<T *>(t_arena->base + off);
        t_arena->used = off + bytes;
        return SNN_OK;
    }
    cudaError_t e = cudaMalloc((void **)p, n * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? SNN_ERR_NOMEM : SNN_ERR_CUDA,
                    "cudaMalloc of %s (%zu bytes) failed: %s", what, n * sizeof(T), cudaGetErrorString(e));
    }
    return SNN_OK;
}

void free_all(snn_handle *h)
{
    cudaSetDevice(h->device);
    if (!h->arena) {  // an arena's buffers are freed by its owner
        void *ptrs[] = {h->XT, h->cv ? nullptr : h->XV, h->yc, h->cv ? nullptr : h->yr, h->D, h->pred, h->rmse32,
                        h->err, h->stage, h->rmse64, h->err64, h->kv, h->cands, h->prev_cands, h->mask, h->order,
                        h->stepk, h->st, h->nn_idx, h->nn_dist, h->seeds, h->seed_d, h->sbound, h->sval, h->skey, h->sidx,
                        h->sord, h->soff, h->stemp, h->walked, h->perm, h->fvar,
                        h->d_loss_ids, h->lossval, h->err_all, h->kth_prev, h->dmax, h->fcount};
        for (void *q : ptrs)
            if (q) cudaFree(q);
    }
    for (auto &e : h->score_ev) {
        if (e.a) cudaEventDestroy(e.a);
        if (e.b) cudaEventDestroy(e.b);
    }
    for (auto &e : h->commit_ev) {
        if (e.a) cudaEventDestroy(e.a);
        if (e.b) cudaEventDestroy(e.b);
    }
    if (h->total_ev.a) cudaEventDestroy(h->total_ev.a);
    if (h->total_ev.b) cudaEventDestroy(h->total_ev.b);
    if (h->setup_ev.a) cudaEventDestroy(h->setup_ev.a);
    if (h->setup_ev.b) cudaEventDestroy(h->setup_ev.b);
    if (h->stream) cudaStreamDestroy(h->stream);
}

int make_pair(EventPair &e)
{
    if (!e.a) SNN_CUDA(cudaEventCreate(&e.a));
    if (!e.b) SNN_CUDA(cudaEventCreate(&e.b));
    return SNN_OK;
}

int check_device(int device)
{
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(SNN_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    }
    if (device < 0 || device >= n) return fail(SNN_ERR_ARG, "device %d out of range (%d devices)", device, n);
    cudaDeviceProp prop;
    SNN_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return fail(SNN_ERR_CUDA, "device %d is sm_%d%d; this library is built for sm_100a", device,
                                      prop.major, prop.minor);
    return SNN_OK;
}

// The TMA-fed scorer (k_max <= 64) is the automatic choice; option 1 forces
// the rows-per-lane scorer (any k_max <= 256).
bool use_tma(const snn_handle *h) { return h->kernel == 3 || (h->kernel == 0 && snn::score_tma_supported(h->kmax)); }

// Forward step t (t features committed) is scored from seed bounds once
// t >= seed_step: after two commits the columns nearest under D are mostly
// near under D + one more feature too, and the bound over 256 of them beats a
// first pass over a quarter of the columns (on the fwd-64k data, rows whose
// filter fires: 17.9 % against 21.5 % at step 2, 6.9 % against 12.1 % at
// step 14; at step 1, with one feature committed, the first pass is better).
// With k above 16 the seeds start a step later: a k-th distance over the
// seeds needs them to be near in more features (fwd-200k, k = 50: step 2
// took 913 ms seeded against 845 ms with the first pass, step 3 767 against
// 825).  The commit before such a step writes the seeds.
bool seeds_for_step(const snn_handle *h, int t)
{
    return !h->desc.backward && h->seeds && use_tma(h) && t >= h->seed_step;
}

// The first two forward steps of a holdout problem run from sorted feature
// columns (D is zero, then one-dimensional there); CV mode excludes same-fold
// pairs and takes the scan.
bool sorted_step(const snn_handle *h, int t)
{
    if (!h->sorted_start || !h->sval || h->desc.backward || h->cv) return false;
    return t == 0 || (t == 1 && h->kmax <= 64);  // the second step's walk keeps at most 64 entries
}

// Issue one greedy step (no synchronisation).
int issue_step(snn_handle *h, int t)
{
    Bufs b = h->bufs();
    const int n_cand = h->p - t;  // forward: p - t unselected; backward: p - t still selected
    const int backward = h->desc.backward;
    const int it = backward ? h->p - 1 - t : t;
    EventPair *se = nullptr;
    if (h->step_events) {
        if ((int)h->score_ev.size() <= h->n_score) h->score_ev.resize(h->n_score + 1);
        se = &h->score_ev[h->n_score];
        if (int rc = make_pair(*se)) return rc;
        SNN_CUDA(cudaEventRecord(se->a, h->stream));
    }
    if (t == h->inject_launch) {
        h->inject_launch = -1;
        return fail(SNN_ERR_CUDA, "injected launch failure at step %d", t);
    }
    bool tma_step = false;
    if (sorted_step(h, t)) {
        if (t == 0) SNN_CUDA(snn::launch_first_step(b, h->sval, h->sidx, n_cand, h->stream));
        else SNN_CUDA(snn::launch_second_step(b, h->sval, h->sidx, h->skey, n_cand, h->walked, h->stream));
        b.only_if_full = 1;  // the scan below runs only if some tie group was too large
        h->n_launch += t == 0 ? 1 : 2;  // the second step gathers the candidates in sorted order first
    }
    if (use_tma(h)) {
        b.use_prev = backward && h->prev_ok ? 1 : 0;
        b.use_seeds = seeds_for_step(h, t) && h->seeds_ok ? 1 : 0;
        if (!b.only_if_full) {  // the injected stall goes to a launch that scans
            b.inject_stall = h->inject_stall + 1;  // 0: off
            h->inject_stall = -1;
        }
        if (b.use_seeds) {
            // the sort's value buffer (p x ldc, unused after load) holds the row-major candidates
            SNN_CUDA(snn::launch_seed_bounds(b, n_cand, reinterpret_cast<float *>(h->sord), h->stream));
            h->n_launch += h->kmax <= 16 && h->sord ? 2 : 1;
        }
        SNN_CUDA(snn::launch_score_tma(b, n_cand, backward, h->stream));
        h->n_launch += snn::score_tma_launches(h->kmax, n_cand, backward) - 1;  // counted once below
        h->prev_ok = backward && h->kth_prev;  // this step wrote every candidate's k-th distances
        tma_step = true;
    } else {
        SNN_CUDA(snn::launch_score(b, n_cand, h->plan, backward, h->stream));
    }
    if (se) {
        SNN_CUDA(cudaEventRecord(se->b, h->stream));
        h->n_score++;
    }
    if (!tma_step) h->prev_ok = false;
    if (h->model == 1) {
        SNN_CUDA(snn::launch_mode_predict(b, n_cand, h->stream));
        h->n_launch += 1;
    }
    SNN_CUDA(snn::launch_reduce(b, n_cand, h->stream));
    if (b.nloss) {
        SNN_CUDA(snn::launch_losses(b, n_cand, h->stream));
        h->n_launch += 1;
    }
    SNN_CUDA(snn::launch_select(b, n_cand, it, t, h->total_steps, backward, h->desc.auto_feature, h->stream));
    h->n_launch += 3;
    if (h->keep_nn) h->nn_ncand = n_cand;
    h->last_ncand = n_cand;
    if (t + 1 < h->total_steps) {
        EventPair *ce = nullptr;
        if (h->step_events) {
            if ((int)h->commit_ev.size() <= h->n_commit) h->commit_ev.resize(h->n_commit + 1);
            ce = &h->commit_ev[h->n_commit];
            if (int rc = make_pair(*ce)) return rc;
            SNN_CUDA(cudaEventRecord(ce->a, h->stream));
        }
        const bool sd = seeds_for_step(h, t + 1);
        SNN_CUDA(snn::launch_commit(b, backward, sd ? h->seeds : nullptr, sd ? h->seed_d : nullptr, h->stream));
        h->seeds_ok = sd;
        if (ce) {
            SNN_CUDA(cudaEventRecord(ce->b, h->stream));
            h->n_commit++;
        }
        h->n_launch += 1;
    }
    return SNN_OK;
}

int issue_reset(snn_handle *h)
{
    h->prev_ok = false;
    h->seeds_ok = false;
    h->last_ncand = 0;
    const Bufs b = h->bufs();
    SNN_CUDA(snn::launch_reset_state(b, h->desc.backward, h->total_steps, h->stream));
    h->setup_timed = h->step_events;
    if (h->setup_timed) {
        if (int rc = make_pair(h->setup_ev)) return rc;
        SNN_CUDA(cudaEventRecord(h->setup_ev.a, h->stream));
    }
    if (h->desc.backward) {
        SNN_CUDA(snn::launch_full_distance(b, h->cv, h->npf, h->stream));
        SNN_CUDA(snn::launch_row_dmax(b, h->dmax, h->stream));
        h->n_launch += 1;
    } else {
        SNN_CUDA(snn::launch_init_forward(b, h->cv, h->npf, h->stream));
    }
    if (h->setup_timed) SNN_CUDA(cudaEventRecord(h->setup_ev.b, h->stream));
    h->n_launch += 2;
    h->host_step = 0;
    return SNN_OK;
}

int read_state(snn_handle *h, State *s)
{
    SNN_CUDA(cudaMemcpyAsync(s, h->st, sizeof(State), cudaMemcpyDeviceToHost, h->stream));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    return SNN_OK;
}

void reset_timing(snn_handle *h)
{
    h->n_score = h->n_commit = h->n_launch = 0;
    if (h->fcount) cudaMemsetAsync(h->fcount, 0, 3 * sizeof(unsigned long long), h->stream);
}

}  // namespace

// ===========================================================================
// Handle API
// ===========================================================================
extern "C" {

SNN_API const char *snn_last_error(void) { return g_err.c_str(); }

SNN_API const char *snn_version(void) { return "speedynn_b200 0.1.0 (sm_100a)"; }

// Descriptor checks shared by snn_create and snn_batch_create (no CUDA calls).
static int validate_desc(const snn_desc *d, int *kmax_out)
{
    if (d->n_train <= 0 || d->p <= 0 || d->n_val < 0) return fail(SNN_ERR_ARG, "bad shape n_train=%d n_val=%d p=%d",
                                                                 d->n_train, d->n_val, d->p);
    if (!d->k_vals || d->num_k_vals <= 0) return fail(SNN_ERR_ARG, "k_vals must be a non-empty array");
    int kmax = 0;
    for (int m = 0; m < d->num_k_vals; ++m) {
        if (d->k_vals[m] <= 0) return fail(SNN_ERR_ARG, "k_vals[%d]=%d must be >= 1", m, d->k_vals[m]);
        kmax = std::max(kmax, d->k_vals[m]);
    }
    if (d->num_features < 0 || d->num_features > d->p)
        return fail(SNN_ERR_ARG, "num_features=%d must lie in [0, p=%d]", d->num_features, d->p);
    if (d->n_val == 0 && (d->k_fold <= 0 || d->k_fold > d->n_train))
        return fail(SNN_ERR_ARG, "k_fold=%d must lie in [1, n=%d]", d->k_fold, d->n_train);
    if (kmax > snn::kScoreMaxK)
        return fail(SNN_ERR_UNSUPPORTED, "k_max=%d is above the supported maximum of %d", kmax, snn::kScoreMaxK);
    *kmax_out = kmax;
    return SNN_OK;
}

// Device bytes a handle for this descriptor allocates (buffers of snn_create
// plus the load staging buffer), for the batch's memory waves.
static size_t handle_bytes(const snn_desc *d, int kmax)
{
    const size_t p = (size_t)d->p, n_cols = (size_t)d->n_train;
    const bool cv = d->n_val == 0;
    const size_t n_rows = cv ? n_cols : (size_t)d->n_val;
    const size_t ldc = (size_t)round_up(d->n_train, snn::kPadCols);
    const size_t ldr = cv ? ldc : (size_t)round_up((int)n_rows, snn::kPadCols);
    const size_t M = d->backward ? 0 : 2 * (size_t)snn::kSeeds + p;  // seed columns, distances, bounds
    (void)kmax;
    size_t f = p * ldc + n_rows * ldc + p * (size_t)d->num_k_vals * n_rows + std::max(n_rows, n_cols) * p +
               n_rows * M + n_cols + n_rows;
    // sorted feature columns of the first forward step and the sort's buffers
    if (!d->backward && !cv) f += 4 * p * ldc + 2 * p + snn::sort_temp_bytes(d->p, (int)ldc) / sizeof(float) + 1;
    if (d->backward) f += p * n_rows + n_rows;  // kth_prev, dmax
    if (!cv) f += p * ldr;
    return sizeof(float) * f + ((size_t)1 << 20);
}

SNN_API int snn_create(const snn_desc *d, snn_handle **out)
{
    g_err.clear();
    if (!d || !out) return fail(SNN_ERR_ARG, "null descriptor or output pointer");
    *out = nullptr;
    int kmax = 0;
    if (int rc = validate_desc(d, &kmax)) return rc;
    const int cv = d->n_val == 0;
    if (int rc = check_device(d->device)) return rc;

    snn_handle *h = new snn_handle();
    h->arena = t_arena != nullptr;  // a batch creating this handle from its arena
    if (const char *f = getenv("SNN_INJECT_FAIL")) {
        if (!strncmp(f, "alloc:", 6)) t_fail_alloc = atoi(f + 6);
        if (!strncmp(f, "launch:", 7)) h->inject_launch = atoi(f + 7);
    }
    if (const char *f = getenv("SNN_INJECT_STALL")) h->inject_stall = atoi(f);
    h->desc = *d;
    h->kvals.assign(d->k_vals, d->k_vals + d->num_k_vals);
    h->desc.k_vals = nullptr;
    h->device = d->device;
    h->p = d->p;
    h->cv = cv;
    h->n_cols = d->n_train;
    h->n_rows = cv ? d->n_train : d->n_val;
    h->npf = cv ? d->n_train / d->k_fold : 1;
    h->kmax = kmax;
    h->seed_step = kmax <= 16 ? 2 : 3;
    h->nk = d->num_k_vals;
    h->ldc = round_up(h->n_cols, snn::kPadCols);
    h->ldr = cv ? h->ldc : round_up(h->n_rows, snn::kPadCols);
    if (d->auto_feature)
        h->total_steps = d->p;
    else
        h->total_steps = d->backward ? d->p - d->num_features : d->num_features;

    int rc = SNN_OK;
    auto bail = [&](int code) {
        t_fail_alloc = 0;
        free_all(h);
        delete h;
        return code;
    };
    if (cudaSetDevice(h->device) != cudaSuccess) return bail(fail(SNN_ERR_CUDA, "cudaSetDevice(%d) failed", h->device));
    int max_smem = 0;
    cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    h->max_smem = max_smem;
    h->plan = snn::plan_score(kmax, d->p, max_smem);
    if (h->plan.cc == 0)
        return bail(fail(SNN_ERR_UNSUPPORTED, "k_max=%d is above the supported maximum of %d", kmax, snn::kScoreMaxK));
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(fail(SNN_ERR_CUDA, "cudaStreamCreate failed"));

    const size_t p = (size_t)h->p;
    if ((rc = dev_alloc(&h->XT, p * h->ldc, "X_train"))) return bail(rc);
    if ((rc = dev_alloc(&h->yc, (size_t)h->n_cols, "y_train"))) return bail(rc);
    if (cv) {
        h->XV = h->XT;
        h->yr = h->yc;
    } else {
        if ((rc = dev_alloc(&h->XV, p * h->ldr, "X_val"))) return bail(rc);
        if ((rc = dev_alloc(&h->yr, (size_t)h->n_rows, "y_val"))) return bail(rc);
    }
    if ((rc = dev_alloc(&h->D, (size_t)h->n_rows * h->ldc, "distance matrix"))) return bail(rc);
    if ((rc = dev_alloc(&h->pred, p * h->nk * h->n_rows, "predictions"))) return bail(rc);
    if ((rc = dev_alloc(&h->rmse32, p * h->nk, "errors"))) return bail(rc);
    if ((rc = dev_alloc(&h->rmse64, p * h->nk, "errors64"))) return bail(rc);
    if ((rc = dev_alloc(&h->err, p, "step errors"))) return bail(rc);
    if ((rc = dev_alloc(&h->err64, p, "step errors64"))) return bail(rc);
    if ((rc = dev_alloc(&h->kv, (size_t)h->nk, "k_vals"))) return bail(rc);
    if ((rc = dev_alloc(&h->cands, p, "candidates"))) return bail(rc);
    if ((rc = dev_alloc(&h->prev_cands, p, "candidates"))) return bail(rc);
    if ((rc = dev_alloc(&h->perm, p, "feature order"))) return bail(rc);
    if (d->backward && (rc = dev_alloc(&h->kth_prev, p * (size_t)h->n_rows, "k-th distances"))) return bail(rc);
    if (d->backward && (rc = dev_alloc(&h->dmax, (size_t)h->n_rows, "row maxima"))) return bail(rc);
    if ((rc = dev_alloc(&h->fvar, p, "feature variances"))) return bail(rc);
    if ((rc = dev_alloc(&h->mask, p, "mask"))) return bail(rc);
    if ((rc = dev_alloc(&h->order, p, "ordering"))) return bail(rc);
    if ((rc = dev_alloc(&h->stepk, p, "best k"))) return bail(rc);
    if ((rc = dev_alloc(&h->st, 1, "state"))) return bail(rc);
    if ((rc = dev_alloc(&h->fcount, 3, "filter counters"))) return bail(rc);
    if (!d->backward) {
        if ((rc = dev_alloc(&h->seeds, (size_t)h->n_rows * snn::kSeeds, "seed columns"))) return bail(rc);
        if ((rc = dev_alloc(&h->seed_d, (size_t)h->n_rows * snn::kSeeds, "seed distances"))) return bail(rc);
        if ((rc = dev_alloc(&h->sbound, p * h->n_rows, "seed bounds"))) return bail(rc);
    }
    if (!d->backward && !cv) {
        const size_t pl = p * h->ldc;
        if ((rc = dev_alloc(&h->sval, pl, "sorted values"))) return bail(rc);
        // the sort's keys at load, then the second step's candidate values in sorted order
        if ((rc = dev_alloc(&h->skey, pl, "sort keys"))) return bail(rc);
        if ((rc = dev_alloc(&h->sidx, pl, "sorted indices"))) return bail(rc);
        if ((rc = dev_alloc(&h->sord, pl, "sort values"))) return bail(rc);
        if ((rc = dev_alloc(&h->soff, 2 * p, "sort offsets"))) return bail(rc);
        h->stemp_bytes = snn::sort_temp_bytes(h->p, h->ldc);
        if ((rc = dev_alloc(&h->stemp, h->stemp_bytes, "sort workspace"))) return bail(rc);
        if ((rc = dev_alloc(&h->walked, 1, "walk counter"))) return bail(rc);
    }
    // On the handle's stream, so every kernel that reads k_vals comes after it
    // (the source lives as long as the handle).  A cudaMemcpy here would run on
    // the legacy stream, which does not order the handle's non-blocking stream,
    // and from pageable memory it may return before its DMA lands.
    if (cudaMemcpyAsync(h->kv, h->kvals.data(), sizeof(int) * h->nk, cudaMemcpyHostToDevice, h->stream) != cudaSuccess)
        return bail(fail(SNN_ERR_CUDA, "copy of k_vals failed"));
    if (make_pair(h->total_ev)) return bail(SNN_ERR_CUDA);
    t_fail_alloc = 0;
    *out = h;
    return SNN_OK;
}

static int load_matrix(snn_handle *h, const float *X, int n, float *XT, int ld, bool device_src)
{
    const size_t bytes = sizeof(float) * (size_t)n * h->p;
    const float *src = X;
    if (!device_src) {
        if (!h->stage) {
            size_t n_stage = (size_t)std::max(h->n_rows, h->n_cols) * h->p;
            if (int rc = dev_alloc(&h->stage, n_stage, "staging")) return rc;
        }
        SNN_CUDA(cudaMemcpyAsync(h->stage, X, bytes, cudaMemcpyHostToDevice, h->stream));
        src = h->stage;
    }
    SNN_CUDA(snn::launch_transpose(src, n, h->p, XT, ld, h->stream));
    return SNN_OK;
}

static int load_impl(snn_handle *h, const float *X_train, const float *y_train, const float *X_val,
                     const float *y_val, bool device_src, bool wait = true)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (!X_train || !y_train) return fail(SNN_ERR_ARG, "X_train and y_train are required");
    if (!h->cv && (!X_val || !y_val)) return fail(SNN_ERR_ARG, "holdout mode needs X_val and y_val");
    SNN_CUDA(cudaSetDevice(h->device));
    const cudaMemcpyKind kind = device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    if (int rc = load_matrix(h, X_train, h->n_cols, h->XT, h->ldc, device_src)) return rc;
    SNN_CUDA(cudaMemcpyAsync(h->yc, y_train, sizeof(float) * h->n_cols, kind, h->stream));
    if (!h->cv) {
        // the staging buffer is reused: order the second upload after the first transpose
        if (int rc = load_matrix(h, X_val, h->n_rows, h->XV, h->ldr, device_src)) return rc;
        SNN_CUDA(cudaMemcpyAsync(h->yr, y_val, sizeof(float) * h->n_rows, kind, h->stream));
    }
    // candidate slot order: ascending training variance, so that the four
    // candidates a scoring warp shares a filter bound with have distances of
    // similar scale (any order gives the same results)
    SNN_CUDA(snn::launch_feature_variance(h->bufs(), h->fvar, h->stream));
    SNN_CUDA(snn::launch_feature_order(h->fvar, h->p, h->perm, h->stream));
    if (h->sval)
        SNN_CUDA(snn::launch_sort_features(h->bufs(), h->skey, h->sord, h->soff, h->sval, h->sidx, h->stemp,
                                           h->stemp_bytes, h->stream));
    h->loaded = true;
    reset_timing(h);
    if (int rc = issue_reset(h)) return rc;
    // A batch issues the selection on the same stream right away (its inputs
    // stay valid until the batch run returns); a single load waits, so the
    // caller may reuse pinned source buffers at once.
    if (wait) SNN_CUDA(cudaStreamSynchronize(h->stream));
    return SNN_OK;
}

SNN_API int snn_load(snn_handle *h, const float *X_train, const float *y_train, const float *X_val, const float *y_val)
{
    return load_impl(h, X_train, y_train, X_val, y_val, false);
}

SNN_API int snn_reset(snn_handle *h)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (!h->loaded) return fail(SNN_ERR_STATE, "snn_reset before snn_load");
    SNN_CUDA(cudaSetDevice(h->device));
    reset_timing(h);
    if (int rc = issue_reset(h)) return rc;
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    return SNN_OK;
}

SNN_API int snn_run(snn_handle *h)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (!h->loaded) return fail(SNN_ERR_STATE, "snn_run before snn_load");
    SNN_CUDA(cudaSetDevice(h->device));
    reset_timing(h);
    SNN_CUDA(cudaEventRecord(h->total_ev.a, h->stream));
    // every run is a complete selection from the initial distance matrix
    if (int rc = issue_reset(h)) return rc;
    for (int t = 0; t < h->total_steps; ++t)
        if (int rc = issue_step(h, t)) return rc;
    h->host_step = h->total_steps;
    SNN_CUDA(cudaEventRecord(h->total_ev.b, h->stream));
    State s;
    if (int rc = read_state(h, &s)) return rc;
    if (s.error == snn::kErrTimeout) return fail(SNN_ERR_TIMEOUT, "a device pipeline wait timed out at step %d", s.step);
    if (s.error) return fail(s.error, "no candidate had an error below FLT_MAX at step %d (non-finite labels?)", s.step);
    return SNN_OK;
}

SNN_API int snn_step(snn_handle *h)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (!h->loaded) return fail(SNN_ERR_STATE, "snn_step before snn_load");
    SNN_CUDA(cudaSetDevice(h->device));
    State s;
    if (int rc = read_state(h, &s)) return rc;
    if (s.error) return fail(s.error, "selection stopped with an error at step %d", s.step);
    if (s.done || h->host_step >= h->total_steps) return 0;
    reset_timing(h);
    SNN_CUDA(cudaEventRecord(h->total_ev.a, h->stream));
    if (int rc = issue_step(h, h->host_step)) return rc;
    SNN_CUDA(cudaEventRecord(h->total_ev.b, h->stream));
    h->host_step++;
    if (int rc = read_state(h, &s)) return rc;
    if (s.error == snn::kErrTimeout) return fail(SNN_ERR_TIMEOUT, "a device pipeline wait timed out at step %d", s.step);
    if (s.error) return fail(s.error, "no candidate had an error below FLT_MAX at step %d", s.step);
    return 1;
}

SNN_API int snn_commit_sequence(snn_handle *h, const int *seq, int n)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (!h->loaded) return fail(SNN_ERR_STATE, "snn_commit_sequence before snn_load");
    if (n < 0 || n > h->total_steps || (n > 0 && !seq))
        return fail(SNN_ERR_ARG, "sequence length %d outside [0, %d]", n, h->total_steps);
    std::vector<char> used(h->p, 0);
    for (int i = 0; i < n; ++i) {
        if (seq[i] < 0 || seq[i] >= h->p || used[seq[i]])
            return fail(SNN_ERR_ARG, "sequence entry %d (=%d) is out of range or repeated", i, seq[i]);
        used[seq[i]] = 1;
    }
    SNN_CUDA(cudaSetDevice(h->device));
    reset_timing(h);
    if (int rc = issue_reset(h)) return rc;
    const Bufs b = h->bufs();
    for (int t = 0; t < n; ++t) {
        const int it = h->desc.backward ? h->p - 1 - t : t;
        SNN_CUDA(snn::launch_force(b, seq[t], it, t, h->total_steps, h->desc.backward, h->stream));
        const bool sd = t + 1 == n && seeds_for_step(h, n);  // the step after the sequence may use seeds
        SNN_CUDA(snn::launch_commit(b, h->desc.backward, sd ? h->seeds : nullptr, sd ? h->seed_d : nullptr, h->stream));
        h->seeds_ok = sd;
    }
    h->host_step = n;
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    return SNN_OK;
}

SNN_API int snn_get_results(snn_handle *h, int *ordering, int *mask, float *errors, double *errors64, int *step_best_k,
                            int *best_k, int *num_final)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    SNN_CUDA(cudaSetDevice(h->device));
    const size_t p = (size_t)h->p;
    if (ordering) SNN_CUDA(cudaMemcpyAsync(ordering, h->order, p * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (mask) SNN_CUDA(cudaMemcpyAsync(mask, h->mask, p * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    if (errors) SNN_CUDA(cudaMemcpyAsync(errors, h->err, p * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    if (errors64) SNN_CUDA(cudaMemcpyAsync(errors64, h->err64, p * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (step_best_k) SNN_CUDA(cudaMemcpyAsync(step_best_k, h->stepk, p * sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    State s;
    if (int rc = read_state(h, &s)) return rc;
    if (best_k) *best_k = s.best_k_last;
    if (num_final) *num_final = s.num_final;
    return SNN_OK;
}

SNN_API int snn_set_model(snn_handle *h, const int *loss_ids, int n_losses, int model_type)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (!loss_ids || n_losses <= 0) return fail(SNN_ERR_ARG, "at least one loss id is required");
    for (int l = 0; l < n_losses; ++l)
        if (loss_ids[l] < 0 || loss_ids[l] > 8) return fail(SNN_ERR_ARG, "loss id %d is not one of 0..8", loss_ids[l]);
    if (model_type != 0 && model_type != 1) return fail(SNN_ERR_ARG, "model_type %d is not 0 or 1", model_type);
    SNN_CUDA(cudaSetDevice(h->device));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    if (!h->arena) {  // an arena's sub-allocations are freed with the arena
        cudaFree(h->d_loss_ids);
        cudaFree(h->lossval);
        cudaFree(h->err_all);
    }
    h->d_loss_ids = nullptr;
    h->lossval = h->err_all = nullptr;
    h->loss_ids.assign(loss_ids, loss_ids + n_losses);
    h->model = model_type;
    const size_t nl = (size_t)n_losses, p = (size_t)h->p;
    if (h->extra_losses()) {
        if (int rc = dev_alloc(&h->d_loss_ids, nl, "loss ids")) return rc;
        if (int rc = dev_alloc(&h->lossval, nl * p * h->nk, "losses")) return rc;
        if (int rc = dev_alloc(&h->err_all, nl * p, "losses per step")) return rc;
        // on the handle's stream (see the k_vals copy in snn_create); the wait lets
        // the caller reuse loss_ids at once
        SNN_CUDA(cudaMemcpyAsync(h->d_loss_ids, h->loss_ids.data(), sizeof(int) * nl, cudaMemcpyHostToDevice, h->stream));
        SNN_CUDA(cudaStreamSynchronize(h->stream));
    }
    if (model_type == 1 && !h->nn_idx) {
        const size_t n = p * h->n_rows * h->kmax;
        if (int rc = dev_alloc(&h->nn_idx, n, "neighbour indices")) return rc;
        if (int rc = dev_alloc(&h->nn_dist, n, "neighbour distances")) return rc;
    }
    if (h->loaded) {
        if (int rc = issue_reset(h)) return rc;
        SNN_CUDA(cudaStreamSynchronize(h->stream));
    }
    return SNN_OK;
}

SNN_API int snn_get_errors_all(snn_handle *h, float *errors, int n)
{
    g_err.clear();
    if (!h || !errors) return fail(SNN_ERR_ARG, "null handle or output");
    const size_t want = h->loss_ids.size() * (size_t)h->p;
    if (n < (int)want) return fail(SNN_ERR_ARG, "errors needs %zu entries (losses x p)", want);
    SNN_CUDA(cudaSetDevice(h->device));
    if (h->extra_losses()) {
        SNN_CUDA(cudaMemcpyAsync(errors, h->err_all, sizeof(float) * want, cudaMemcpyDeviceToHost, h->stream));
    } else {
        SNN_CUDA(cudaMemcpyAsync(errors, h->err, sizeof(float) * want, cudaMemcpyDeviceToHost, h->stream));
    }
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    return SNN_OK;
}

SNN_API int snn_keep_neighbours(snn_handle *h, int enable)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    SNN_CUDA(cudaSetDevice(h->device));
    if (enable && !h->nn_idx) {
        const size_t n = (size_t)h->p * h->n_rows * h->kmax;
        if (int rc = dev_alloc(&h->nn_idx, n, "neighbour indices")) return rc;
        if (int rc = dev_alloc(&h->nn_dist, n, "neighbour distances")) return rc;
    }
    h->keep_nn = enable != 0;
    h->nn_ncand = 0;
    return SNN_OK;
}

SNN_API int snn_get_neighbours(snn_handle *h, int *cands, int *n_cand, int *k_max, int *idx, float *dist)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (!h->keep_nn || h->nn_ncand == 0) return fail(SNN_ERR_STATE, "no neighbour lists kept (snn_keep_neighbours)");
    SNN_CUDA(cudaSetDevice(h->device));
    if (n_cand) *n_cand = h->nn_ncand;
    if (k_max) *k_max = h->kmax;
    const size_t n = (size_t)h->nn_ncand * h->n_rows * h->kmax;
    if (cands) SNN_CUDA(cudaMemcpyAsync(cands, h->prev_cands, sizeof(int) * h->nn_ncand, cudaMemcpyDeviceToHost, h->stream));
    if (idx) SNN_CUDA(cudaMemcpyAsync(idx, h->nn_idx, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
    if (dist) SNN_CUDA(cudaMemcpyAsync(dist, h->nn_dist, sizeof(float) * n, cudaMemcpyDeviceToHost, h->stream));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    return SNN_OK;
}

}  // extern "C"

namespace {

// Copy the rows rows[0..n_sel) of a [n_cand][n_rows][w] device array into
// out[n_cand][n_sel][w], one candidate slab at a time through a host buffer.
template <typename T>
int gather_rows(snn_handle *h, const T *dev, int n_cand, int w, const int *rows, int n_sel, T *out)
{
    std::vector<T> slab((size_t)h->n_rows * w);
    for (int c = 0; c < n_cand; ++c) {
        SNN_CUDA(cudaMemcpyAsync(slab.data(), dev + (size_t)c * h->n_rows * w, sizeof(T) * slab.size(),
                                 cudaMemcpyDeviceToHost, h->stream));
        SNN_CUDA(cudaStreamSynchronize(h->stream));
        for (int i = 0; i < n_sel; ++i)
            memcpy(out + ((size_t)c * n_sel + i) * w, slab.data() + (size_t)rows[i] * w, sizeof(T) * w);
    }
    return SNN_OK;
}

int check_rows(const snn_handle *h, const int *rows, int n_sel)
{
    if (n_sel < 0 || (n_sel > 0 && !rows)) return fail(SNN_ERR_ARG, "rows must list n_sel >= 0 row indices");
    for (int i = 0; i < n_sel; ++i)
        if (rows[i] < 0 || rows[i] >= h->n_rows)
            return fail(SNN_ERR_ARG, "row %d (=%d) outside [0, %d)", i, rows[i], h->n_rows);
    return SNN_OK;
}

}  // namespace

extern "C" {

SNN_API int snn_get_neighbours_rows(snn_handle *h, const int *rows, int n_sel, int *idx, float *dist)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (!h->keep_nn || h->nn_ncand == 0) return fail(SNN_ERR_STATE, "no neighbour lists kept (snn_keep_neighbours)");
    if (int rc = check_rows(h, rows, n_sel)) return rc;
    SNN_CUDA(cudaSetDevice(h->device));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    if (idx) {
        if (int rc = gather_rows(h, h->nn_idx, h->nn_ncand, h->kmax, rows, n_sel, idx)) return rc;
    }
    if (dist) {
        if (int rc = gather_rows(h, h->nn_dist, h->nn_ncand, h->kmax, rows, n_sel, dist)) return rc;
    }
    return SNN_OK;
}

SNN_API int snn_get_predictions(snn_handle *h, const int *rows, int n_sel, int *cands, int *n_cand, float *pred)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    if (h->last_ncand == 0) return fail(SNN_ERR_STATE, "no step has been scored since the last reset");
    if (int rc = check_rows(h, rows, n_sel)) return rc;
    SNN_CUDA(cudaSetDevice(h->device));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    if (n_cand) *n_cand = h->last_ncand;
    if (cands)
        SNN_CUDA(cudaMemcpyAsync(cands, h->prev_cands, sizeof(int) * h->last_ncand, cudaMemcpyDeviceToHost, h->stream));
    if (pred) {
        // pred is [slot][k][n_rows]: gather as [slot * nk + m] slabs of n_rows values
        if (int rc = gather_rows(h, h->pred, h->last_ncand * h->nk, 1, rows, n_sel, pred)) return rc;
    }
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    return SNN_OK;
}

SNN_API int snn_get_timing(snn_handle *h, double *score_ms, int *score_launches, double *commit_ms, int *commit_launches,
                           double *total_ms, int *total_launches)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    SNN_CUDA(cudaSetDevice(h->device));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    double s = 0.0, c = 0.0;
    for (int i = 0; i < h->n_score; ++i) {
        float ms = 0.f;
        SNN_CUDA(cudaEventElapsedTime(&ms, h->score_ev[i].a, h->score_ev[i].b));
        s += ms;
    }
    for (int i = 0; i < h->n_commit; ++i) {
        float ms = 0.f;
        SNN_CUDA(cudaEventElapsedTime(&ms, h->commit_ev[i].a, h->commit_ev[i].b));
        c += ms;
    }
    float tot = 0.f;
    if (h->n_launch > 0) {
        cudaError_t e = cudaEventElapsedTime(&tot, h->total_ev.a, h->total_ev.b);
        if (e != cudaSuccess) {
            cudaGetLastError();
            tot = 0.f;
        }
    }
    if (score_ms) *score_ms = s;
    if (score_launches) *score_launches = h->n_score;
    if (commit_ms) *commit_ms = c;
    if (commit_launches) *commit_launches = h->n_commit;
    if (total_ms) *total_ms = tot;
    if (total_launches) *total_launches = h->n_launch;
    return SNN_OK;
}

SNN_API int snn_set_option(snn_handle *h, int option, int value)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    switch (option) {
    case SNN_OPT_KERNEL:
        if (value != 0 && value != 1 && value != 3) return fail(SNN_ERR_ARG, "kernel choice %d is not 0, 1 or 3", value);
        if (value == 3 && !snn::score_tma_supported(h->kmax))
            return fail(SNN_ERR_UNSUPPORTED, "the TMA-fed kernel handles k_max <= 64");
        h->kernel = value;
        h->seeds_ok = false;
        return SNN_OK;
    case SNN_OPT_SORTED_START: h->sorted_start = value != 0; return SNN_OK;
    case SNN_OPT_SEED_STEP:
        if (value < 1) return fail(SNN_ERR_ARG, "seed step %d must be >= 1", value);
        h->seed_step = value;
        h->seeds_ok = false;
        return SNN_OK;
    case SNN_OPT_COUNTERS: h->count_filter = value != 0; return SNN_OK;
    default: return fail(SNN_ERR_ARG, "unknown option %d", option);
    }
}

SNN_API int snn_get_filter_counters(snn_handle *h, unsigned long long *row_chunks, unsigned long long *flagged,
                                    unsigned long long *passed)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    SNN_CUDA(cudaSetDevice(h->device));
    unsigned long long c[3] = {0, 0, 0};
    SNN_CUDA(cudaMemcpyAsync(c, h->fcount, sizeof c, cudaMemcpyDeviceToHost, h->stream));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    if (row_chunks) *row_chunks = c[0];
    if (flagged) *flagged = c[1];
    if (passed) *passed = c[2];
    return SNN_OK;
}

SNN_API int snn_get_step_timing(snn_handle *h, float *score_ms, float *commit_ms, int n)
{
    g_err.clear();
    if (!h) return fail(SNN_ERR_ARG, "null handle");
    SNN_CUDA(cudaSetDevice(h->device));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    for (int i = 0; i < n; ++i) {
        float ms = 0.f;
        if (score_ms) {
            if (i < h->n_score) SNN_CUDA(cudaEventElapsedTime(&ms, h->score_ev[i].a, h->score_ev[i].b));
            score_ms[i] = i < h->n_score ? ms : 0.f;
        }
        if (commit_ms) {
            ms = 0.f;
            if (i < h->n_commit) SNN_CUDA(cudaEventElapsedTime(&ms, h->commit_ev[i].a, h->commit_ev[i].b));
            commit_ms[i] = i < h->n_commit ? ms : 0.f;
        }
    }
    return h->n_score;
}

SNN_API int snn_get_setup_timing(snn_handle *h, float *ms)
{
    g_err.clear();
    if (!h || !ms) return fail(SNN_ERR_ARG, "null handle or output");
    if (!h->setup_timed) return fail(SNN_ERR_STATE, "no timed reset (the handle was never loaded or reset)");
    SNN_CUDA(cudaSetDevice(h->device));
    SNN_CUDA(cudaStreamSynchronize(h->stream));
    SNN_CUDA(cudaEventElapsedTime(ms, h->setup_ev.a, h->setup_ev.b));
    return SNN_OK;
}

SNN_API int snn_destroy(snn_handle *h)
{
    if (!h) return SNN_OK;
    free_all(h);
    delete h;
    return SNN_OK;
}

}  // extern "C"

// ===========================================================================
// Batches of independent problems
// ===========================================================================
struct snn_batch {
    struct Problem {
        snn_desc desc;
        std::vector<int> kvals;
        const float *Xt = nullptr, *yt = nullptr, *Xv = nullptr, *yv = nullptr;
        int status = SNN_ERR_STATE;  // until run
        std::vector<int> loss_ids{0};  // snn_batch_set_model: losses (the first decides) and model type
        int model = 0;
        std::vector<int> ordering, mask, stepk;
        std::vector<float> err, err_all;
        std::vector<double> err64;
        int best_k = 0, num_final = 0;
    };
    std::vector<Problem> prob;
    unsigned long long max_bytes = 0;  // 0: free device memory less a reserve
    double run_ms = 0.0;
    int waves = 0;
};

namespace {

// Device bytes snn_set_model adds to a batch problem's handle: the loss ids,
// every (loss, candidate, k) value and the winners' losses when a loss list
// other than {RMSE} is set; the neighbour lists for classification.  Each
// buffer may take up to 256 bytes more for its alignment in the arena.
size_t model_bytes(const snn_batch::Problem &P, int kmax)
{
    const size_t nl = P.loss_ids.size(), p = (size_t)P.desc.p, nk = (size_t)P.desc.num_k_vals;
    const size_t n_rows = P.desc.n_val > 0 ? (size_t)P.desc.n_val : (size_t)P.desc.n_train;
    size_t f = 0;
    if (P.loss_ids != std::vector<int>{0}) f += nl + nl * p * nk + nl * p;
    if (P.model == 1) f += 2 * p * n_rows * (size_t)kmax;
    return sizeof(float) * f + 5 * 256;
}

// Issue a loaded batch problem's whole selection on its own stream, between
// its total_ev events (snn_load has just reset it), without waiting.
int issue_batch_problem(snn_handle *h)
{
    reset_timing(h);
    SNN_CUDA(cudaEventRecord(h->total_ev.a, h->stream));
    for (int t = 0; t < h->total_steps; ++t)
        if (int rc = issue_step(h, t)) return rc;
    h->host_step = h->total_steps;
    SNN_CUDA(cudaEventRecord(h->total_ev.b, h->stream));
    return SNN_OK;
}

// Collect the results of problems [i0, i0 + hs.size()) of the batch, all
// issued, and add the wave's device time: the union of the problems' event
// intervals (the GPU ran some selection of the wave throughout it).
int finish_wave(snn_batch *B, std::vector<snn_handle *> &hs, int i0)
{
    std::vector<std::pair<float, float>> iv;
    for (size_t j = 0; j < hs.size(); ++j) {
        snn_handle *h = hs[j];
        snn_batch::Problem &P = B->prob[i0 + j];
        State st;
        cudaSetDevice(h->device);
        if (int rc = read_state(h, &st)) return rc;
        const size_t p = (size_t)h->p;
        P.ordering.assign(p, 0);
        P.mask.assign(p, 0);
        P.stepk.assign(p, 0);
        P.err.assign(p, 0.0f);
        P.err64.assign(p, 0.0);
        P.status = st.error == snn::kErrTimeout ? SNN_ERR_TIMEOUT : st.error;
        if (int rc = snn_get_results(h, P.ordering.data(), P.mask.data(), P.err.data(), P.err64.data(), P.stepk.data(),
                                     &P.best_k, &P.num_final))
            P.status = rc;
        P.err_all.assign(P.loss_ids.size() * p, 0.0f);
        if (int rc = snn_get_errors_all(h, P.err_all.data(), (int)P.err_all.size())) P.status = rc;
        float a = 0.0f, b = 0.0f;  // relative to the first problem's start event
        SNN_CUDA(cudaEventElapsedTime(&a, hs[0]->total_ev.a, h->total_ev.a));
        SNN_CUDA(cudaEventElapsedTime(&b, hs[0]->total_ev.a, h->total_ev.b));
        iv.emplace_back(a, b);
    }
    std::sort(iv.begin(), iv.end());
    double busy = 0.0, lo = 0.0, hi = 0.0;
    for (size_t j = 0; j < iv.size(); ++j) {
        if (j == 0 || iv[j].first > hi) {
            busy += hi - lo;
            lo = iv[j].first;
            hi = iv[j].second;
        } else {
            hi = std::max<double>(hi, iv[j].second);
        }
    }
    busy += hi - lo;
    B->run_ms += busy;
    B->waves++;
    return SNN_OK;
}

}  // namespace

extern "C" {

SNN_API int snn_batch_create(const snn_desc *descs, int n, unsigned long long max_device_bytes, snn_batch **out)
{
    g_err.clear();
    if (!descs || !out || n <= 0) return fail(SNN_ERR_ARG, "snn_batch_create needs n >= 1 descriptors and an output");
    *out = nullptr;
    snn_batch *B = new snn_batch();
    B->prob.resize(n);
    for (int i = 0; i < n; ++i) {
        int kmax = 0;
        if (int rc = validate_desc(descs + i, &kmax)) {
            delete B;
            return fail(rc, "problem %d: %s", i, std::string(g_err).c_str());
        }
        B->prob[i].desc = descs[i];
        B->prob[i].kvals.assign(descs[i].k_vals, descs[i].k_vals + descs[i].num_k_vals);
        B->prob[i].desc.k_vals = B->prob[i].kvals.data();
    }
    B->max_bytes = max_device_bytes;
    *out = B;
    return SNN_OK;
}

SNN_API int snn_batch_load(snn_batch *B, int i, const float *X_train, const float *y_train, const float *X_val,
                           const float *y_val)
{
    g_err.clear();
    if (!B || i < 0 || i >= (int)B->prob.size()) return fail(SNN_ERR_ARG, "snn_batch_load: no problem %d", i);
    snn_batch::Problem &P = B->prob[i];
    if (!X_train || !y_train) return fail(SNN_ERR_ARG, "X_train and y_train are required");
    if (P.desc.n_val > 0 && (!X_val || !y_val)) return fail(SNN_ERR_ARG, "holdout mode needs X_val and y_val");
    P.Xt = X_train;
    P.yt = y_train;
    P.Xv = X_val;
    P.yv = y_val;
    return SNN_OK;
}

SNN_API int snn_batch_set_model(snn_batch *B, int i, const int *loss_ids, int n_losses, int model_type)
{
    g_err.clear();
    if (!B || i < 0 || i >= (int)B->prob.size()) return fail(SNN_ERR_ARG, "snn_batch_set_model: no problem %d", i);
    if (!loss_ids || n_losses <= 0) return fail(SNN_ERR_ARG, "at least one loss id is required");
    for (int l = 0; l < n_losses; ++l)
        if (loss_ids[l] < 0 || loss_ids[l] > 8) return fail(SNN_ERR_ARG, "loss id %d is not one of 0..8", loss_ids[l]);
    if (model_type != 0 && model_type != 1) return fail(SNN_ERR_ARG, "model_type %d is not 0 or 1", model_type);
    snn_batch::Problem &P = B->prob[i];
    P.loss_ids.assign(loss_ids, loss_ids + n_losses);
    P.model = model_type;
    return SNN_OK;
}

SNN_API int snn_batch_run(snn_batch *B)
{
    g_err.clear();
    if (!B) return fail(SNN_ERR_ARG, "null batch");
    for (size_t i = 0; i < B->prob.size(); ++i)
        if (!B->prob[i].Xt) return fail(SNN_ERR_STATE, "snn_batch_run: problem %zu has no inputs", i);
    B->run_ms = 0.0;
    B->waves = 0;
    const int n = (int)B->prob.size();
    int i = 0;
    while (i < n) {
        // one wave: consecutive problems on one device within the memory budget
        const int dev = B->prob[i].desc.device;
        if (int rc = check_device(dev)) return rc;
        SNN_CUDA(cudaSetDevice(dev));
        size_t budget = (size_t)B->max_bytes;
        if (!budget) {
            size_t fr = 0, tot = 0;
            SNN_CUDA(cudaMemGetInfo(&fr, &tot));
            const size_t reserve = std::max<size_t>((size_t)1 << 30, tot / 50);
            budget = fr > reserve ? fr - reserve : 0;
        }
        // the wave's buffers come from one device allocation of the budget
        // (without it, from cudaMalloc per buffer)
        // (a wave always admits its first problem, whatever the budget)
        int kmax0 = 0;
        validate_desc(&B->prob[i].desc, &kmax0);
        const size_t cap = std::max(budget, handle_bytes(&B->prob[i].desc, kmax0) + model_bytes(B->prob[i], kmax0));
        Arena arena;
        void *abase = nullptr;
        if (cudaMalloc(&abase, cap) == cudaSuccess) {
            arena.base = static_cast<char *>(abase);
            arena.cap = cap;
        } else {
            cudaGetLastError();
        }
        std::vector<snn_handle *> hs;
        size_t used = 0;
        const int i0 = i;
        int rc = SNN_OK;
        while (i < n && B->prob[i].desc.device == dev) {
            int kmax = 0;
            validate_desc(&B->prob[i].desc, &kmax);
            const snn_batch::Problem &P = B->prob[i];
            const size_t need = handle_bytes(&P.desc, kmax) + model_bytes(P, kmax);
            if (!hs.empty() && used + need > budget) break;
            snn_handle *h = nullptr;
            t_arena = arena.base ? &arena : nullptr;
            rc = snn_create(&P.desc, &h);
            if (rc == SNN_OK && (P.loss_ids != std::vector<int>{0} || P.model != 0))
                rc = snn_set_model(h, P.loss_ids.data(), (int)P.loss_ids.size(), P.model);
            if (rc == SNN_OK) {
                h->step_events = false;  // only the selection's total events are read (finish_wave)
                rc = load_impl(h, P.Xt, P.yt, P.Xv, P.yv, false, false);
            }
            t_arena = nullptr;
            if (rc) {
                snn_destroy(h);
                if (rc == SNN_ERR_NOMEM && !hs.empty()) {
                    rc = SNN_OK;  // run what fits, retry this problem in the next wave
                    break;
                }
                break;
            }
            hs.push_back(h);
            used += need;
            ++i;
            // start this problem now: later creates and uploads overlap its steps
            if ((rc = issue_batch_problem(h))) break;
        }
        if (rc == SNN_OK && !hs.empty()) rc = finish_wave(B, hs, i0);
        for (snn_handle *h : hs) snn_destroy(h);
        if (abase) cudaFree(abase);
        if (rc) return fail(rc, "snn_batch_run, problem %d: %s", i, std::string(g_err).c_str());
    }
    return SNN_OK;
}

SNN_API int snn_batch_get_results(snn_batch *B, int i, int *ordering, int *mask, float *errors, double *errors64,
                                  int *step_best_k, int *best_k, int *num_final)
{
    g_err.clear();
    if (!B || i < 0 || i >= (int)B->prob.size()) return fail(SNN_ERR_ARG, "snn_batch_get_results: no problem %d", i);
    const snn_batch::Problem &P = B->prob[i];
    if (P.status == SNN_ERR_STATE && P.ordering.empty()) return fail(SNN_ERR_STATE, "problem %d has not run", i);
    const size_t p = (size_t)P.desc.p;
    if (ordering) memcpy(ordering, P.ordering.data(), sizeof(int) * p);
    if (mask) memcpy(mask, P.mask.data(), sizeof(int) * p);
    if (errors) memcpy(errors, P.err.data(), sizeof(float) * p);
    if (errors64) memcpy(errors64, P.err64.data(), sizeof(double) * p);
    if (step_best_k) memcpy(step_best_k, P.stepk.data(), sizeof(int) * p);
    if (best_k) *best_k = P.best_k;
    if (num_final) *num_final = P.num_final;
    if (P.status) return fail(P.status, "problem %d ended with status %d", i, P.status);
    return SNN_OK;
}

SNN_API int snn_batch_get_errors_all(snn_batch *B, int i, float *errors, int n)
{
    g_err.clear();
    if (!B || i < 0 || i >= (int)B->prob.size()) return fail(SNN_ERR_ARG, "snn_batch_get_errors_all: no problem %d", i);
    if (!errors) return fail(SNN_ERR_ARG, "null output");
    const snn_batch::Problem &P = B->prob[i];
    if (P.status == SNN_ERR_STATE && P.err_all.empty()) return fail(SNN_ERR_STATE, "problem %d has not run", i);
    if (n < (int)P.err_all.size()) return fail(SNN_ERR_ARG, "errors needs %zu entries (losses x p)", P.err_all.size());
    memcpy(errors, P.err_all.data(), sizeof(float) * P.err_all.size());
    if (P.status) return fail(P.status, "problem %d ended with status %d", i, P.status);
    return SNN_OK;
}

SNN_API int snn_batch_get_timing(snn_batch *B, double *run_ms, int *waves)
{
    g_err.clear();
    if (!B) return fail(SNN_ERR_ARG, "null batch");
    if (run_ms) *run_ms = B->run_ms;
    if (waves) *waves = B->waves;
    return SNN_OK;
}

SNN_API int snn_batch_destroy(snn_batch *B)
{
    delete B;
    return SNN_OK;
}

}  // extern "C"
