// Internal declarations shared by the kernels (snn_kernels.cu) and the host
// driver (snn_api.cu).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace snn {

// Selection state kept on the device so that a whole greedy step (score ->
// reduce -> select -> commit) runs without a host round trip.
struct State {
    int step;         // greedy steps completed
    int done;         // 1: selection finished (last step, auto stop or error)
    int error;        // SNN_ERR_NO_WINNER when no candidate had a finite error
    int winner;       // feature chosen by the last completed step
    int n_cand;       // candidates of the next step
    int best_k_last;  // best k of the last winner
    int num_final;    // features in the model after the last step
    int full_scan;    // 1: the sorted first step left problems to the full scan (snn_sorted.cu)
};

// Everything a kernel needs, passed by value.
//
// Layout in HBM:
//   XT  [p][ldc]  neighbour (training) points, feature-major, zero padded
//   XV  [p][ldr]  scored points, feature-major (aliases XT in CV mode)
//   D   [n_rows][ldc]  committed FP32 distance matrix, row = scored point;
//                 +inf on excluded pairs (same CV fold) and on pad columns
//   pred [p][nk][n_rows]  kNN-mean prediction per (candidate slot, k, row)
struct Bufs {
    const float *XT;
    const float *XV;
    int ldc, ldr;
    const float *yc;
    const float *yr;
    float *D;
    int n_rows, n_cols, p;
    const int *kvals;
    int nk, kmax;
    float *pred;
    float *rmse32;
    double *rmse64;
    int *cands;       // current candidate list, in the order of perm
    int *prev_cands;  // candidate list of the last scored step
    const int *perm;  // all features, ascending training variance (ties: ascending id)
    int *mask;
    int *order;
    float *err;
    double *err64;
    int *stepk;
    State *st;
    int *nn_idx;      // optional [n_cand][n_rows][kmax]
    float *nn_dist;
    // losses beyond the default RMSE (nloss 0: RMSE only, nothing recorded)
    int nloss;
    const int *loss_ids;  // [nloss] reference loss ids; index 0 decides
    float *lossval;       // [nloss][n_cand][nk] this step's losses
    float *err_all;       // [nloss][p] the winners' losses, reference order l * p + i
    // backward: each (feature, row)'s k-th distance of the last step, [p][n_rows];
    // removing a feature only lowers distances, so it bounds the next step's k-th
    float *kth_prev;
    int use_prev;         // 1: this step may take its bounds from kth_prev
    const float *dmax;    // backward: per row, >= every finite committed distance (filter margin)
    int inject_stall;     // test hook, 0 off: block 0 never issues the copies of stage inject_stall - 1
    // optional filter counters of the TMA-fed scorer: [0] (row, chunk) pairs of
    // the full pass, [1] of them flagged by the filter, [2] holding an exact pass
    unsigned long long *fcount;
    // forward: kSeeds columns per row near it under the committed D, and their
    // distances [n_rows][kSeeds] (written by the previous step's commit); when
    // use_seeds is set the TMA-fed scorer takes its starting bounds from them
    const int *seeds;
    const float *seed_d;
    float *bound;  // forward: [p][n_rows] starting bounds of a seeded step (k_seed_bounds)
    int use_seeds;
    int only_if_full;  // scoring kernels return at once unless st->full_scan is set (sorted first step)
};

constexpr int kPadCols = 64;     // row stride multiple of the feature-major arrays / D
constexpr int kScoreMaxK = 256;  // largest k_max of the scoring kernel

// Launch shape of the scoring kernel: cc candidates per thread, `warps`
// warps per block (32 scored rows per block), dynamic shared memory bytes.
struct ScorePlan {
    int cc;
    int warps;
    int smem;
};
ScorePlan plan_score(int kmax, int p, int max_smem);

constexpr int kErrTimeout = -7;  // SNN_ERR_TIMEOUT: a bounded device wait gave up

// snn_last_error() plumbing shared by the C-ABI translation units.
int record_error(int code, const char *msg);
void clear_error();

// Warp-specialised TMA scoring (snn_score_tma.cu), k_max <= 64.
bool score_tma_supported(int kmax);  // kernel option 3: k_max <= 64
cudaError_t launch_score_tma(const Bufs &b, int n_cand, int backward, cudaStream_t s);
int score_tma_launches(int kmax, int n_cand, int backward);  // kernels one launch_score_tma issues
// Seeded forward steps: each candidate's starting bound from the seed columns, into b.bound.
// xrm: n_cols x n_cand floats of scratch (the candidates' columns row-major),
// or null to take the bounds from part of the seeds (k_seed_bounds).
cudaError_t launch_seed_bounds(const Bufs &b, int n_cand, float *xrm, cudaStream_t s);

// Commit the winner into D (snn_commit.cu); forward commits given seed
// buffers also keep kSeeds near columns per row for the next step's bounds.
constexpr int kSeedsPerLane = 8;        // seed columns each lane of the commit keeps
constexpr int kSeeds = 32 * kSeedsPerLane;  // seed columns per row
cudaError_t launch_commit(const Bufs &b, int backward, int *seeds, float *seed_d, cudaStream_t s);

// First forward step of a holdout problem from per-feature sorted training
// values (snn_sorted.cu): sort at load, then one thread per problem.
size_t sort_temp_bytes(int p, int ldc);
cudaError_t launch_sort_features(const Bufs &b, float *keys, int *vals, int *offsets, float *sv, int *si, void *temp,
                                 size_t temp_bytes, cudaStream_t s);
cudaError_t launch_first_step(const Bufs &b, const float *sv, const int *si, int n_cand, cudaStream_t s);
// The second step: walks of the first winner's sorted values (xs: n_cand x ldc
// floats of scratch for the candidates' values in that order; walked: a device
// counter).
cudaError_t launch_second_step(const Bufs &b, const float *sv, const int *si, float *xs, int n_cand,
                               unsigned long long *walked, cudaStream_t s);

cudaError_t launch_transpose(const float *X, int n, int p, float *XT, int ld, cudaStream_t s);
cudaError_t launch_init_forward(const Bufs &b, int cv, int npf, cudaStream_t s);
cudaError_t launch_full_distance(const Bufs &b, int cv, int npf, cudaStream_t s);
cudaError_t launch_score(const Bufs &b, int n_cand, const ScorePlan &plan, int backward, cudaStream_t s);
cudaError_t launch_reduce(const Bufs &b, int n_cand, cudaStream_t s);
cudaError_t launch_select(const Bufs &b, int n_cand, int it, int t, int total_steps, int backward,
                          int auto_feature, cudaStream_t s);
cudaError_t launch_reset_state(const Bufs &b, int backward, int total_steps, cudaStream_t s);
// Classification predictions from the kept neighbour lists (mode of the k labels).
cudaError_t launch_mode_predict(const Bufs &b, int n_cand, cudaStream_t s);
// Requested losses of every (candidate, k) prediction vector (b.nloss > 0).
cudaError_t launch_losses(const Bufs &b, int n_cand, cudaStream_t s);
// Per row of D: the largest finite entry (backward; D only shrinks afterwards).
cudaError_t launch_row_dmax(const Bufs &b, float *dmax, cudaStream_t s);
// Per-feature training variance (FP64 sums) into var[p], NaN for non-finite columns.
cudaError_t launch_feature_variance(const Bufs &b, float *var, cudaStream_t s);
// perm[0..p) = features by ascending var (NaN last, ties by id): the candidate slot order.
cudaError_t launch_feature_order(const float *var, int p, int *perm, cudaStream_t s);
cudaError_t launch_force(const Bufs &b, int w, int it, int t, int total_steps, int backward, cudaStream_t s);

}  // namespace snn
