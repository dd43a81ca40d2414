/*
 * speedynn_b200.h -- C ABI of libspeedynn_b200.so: greedy nearest-neighbour
 * wrapper feature selection (forward selection / backward elimination scored
 * by kNN-regression RMSE) on one NVIDIA B200 (sm_100a).
 *
 * Two layers:
 *
 *  1. Drop-in entry points with the names and argument lists of speedynn's
 *     SWIG-wrapped C API (speedynn/lib/nearest_neighbors_feature_selection.h:59-80,
 *     typemaps speedynn/lib/nearest_neighbors_feature_selection_float_gpu.i:14-22).
 *     Like the reference they keep the last result in library state that the
 *     get_* functions read; unlike it they never exit the process: failures
 *     return a negative status and set snn_last_error().
 *
 *  2. A handle API (snn_*) that adds a train/validation holdout mode, device
 *     selection, step-wise execution, FP64 errors beside the reference's FP32
 *     errors, neighbour-list introspection and kernel timing.
 *
 * All arrays are plain host pointers owned by the caller, float32 row-major
 * for matrices ([n][p]), int32 for indices.  No call retains a caller pointer
 * after it returns.  Calls on one handle must come from one thread at a time;
 * different handles are independent.  The drop-in layer shares one library
 * state and is not re-entrant (as in the reference).
 */
#ifndef SPEEDYNN_B200_H
#define SPEEDYNN_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SNN_API __attribute__((visibility("default")))
#else
#define SNN_API
#endif

/* status codes (>= 0 success) */
#define SNN_OK 0
#define SNN_ERR_ARG (-1)          /* invalid argument or shape */
#define SNN_ERR_CUDA (-2)         /* CUDA runtime error, or no usable sm_100 device */
#define SNN_ERR_NOMEM (-3)        /* device or host allocation failed */
#define SNN_ERR_UNSUPPORTED (-4)  /* a reference option outside this library's path */
#define SNN_ERR_NO_WINNER (-5)    /* no candidate had an error below FLT_MAX (e.g. NaN labels) */
#define SNN_ERR_STATE (-6)        /* call out of order (e.g. run before load) */
#define SNN_ERR_TIMEOUT (-7)      /* a bounded wait inside a kernel gave up (pipeline stalled) */

/* loss ids, speedynn/base.py:13-23 */
#define SNN_LOSS_RMSE 0
#define SNN_LOSS_RMSE_NORM 1
#define SNN_LOSS_MAD 2
#define SNN_LOSS_MAD_NORM 3
#define SNN_LOSS_ZERO_ONE 4
#define SNN_LOSS_STD 5
#define SNN_LOSS_RMSE_NORM_MAD_NORM_STD 6
#define SNN_LOSS_RMSE_NORM_MAD_NORM_GALAXIES 7
#define SNN_LOSS_RMSE_STD 8

/* ---------------------------------------------------------------------------
 * 1. Reference-compatible entry points
 * ------------------------------------------------------------------------- */

/* Replaces train_forward_selection
 * (speedynn/lib/nearest_neighbors_feature_selection.h:65, .c:60-65).
 * CV mode over Xtrain [nXtrain][dXtrain]: folds are contiguous row blocks of
 * nXtrain / kfold rows (a remainder forms an extra fold).  Returns the final
 * number of features, or a negative status.  loss_functions: reference
 * loss ids, the first decides; model_type 0 regression, 1 classification. */
SNN_API int train_forward_selection(float *Xtrain, int nXtrain, int dXtrain, float *Ytrain, int nYtrain,
                                    int *kvals, int num_kvals, int num_features, int kfold,
                                    int *loss_functions, int num_loss_functions, int auto_feature,
                                    int model_type);

/* Replaces train_backward_selection
 * (speedynn/lib/nearest_neighbors_feature_selection.h:59, .c:49-54). */
SNN_API int train_backward_selection(float *Xtrain, int nXtrain, int dXtrain, float *Ytrain, int nYtrain,
                                     int *kvals, int num_kvals, int num_features, int kfold,
                                     int *loss_functions, int num_loss_functions, int auto_feature,
                                     int model_type);

/* Replace the getters of speedynn/lib/nearest_neighbors_feature_selection.h:73-77
 * (.c:401-432): copy min(n, p) entries (errors: min(n, num_losses*p)) of the
 * last run's 0/1 mask, ordering and per-step errors (index l*p + i). */
SNN_API void get_selected_dimensions(int *selected_dimensions_extern, int num_selected_dimensions_extern);
SNN_API void get_selected_ordering(int *selected_ordering_extern, int num_selected_ordering_extern);
SNN_API void get_selected_errors(float *selected_errors_extern, int num_selected_errors_extern);
/* best k of the last winner (nearest_neighbors_feature_selection.c:170, :332) */
SNN_API int get_final_optimal_model_k(void);

/* Replaces get_loss_all (speedynn/lib/nearest_neighbors_feature_selection.h:78,
 * loss_functions.c:6-38): a host-side utility over two label vectors, all nine
 * reference loss ids.  Returns NaN for an unknown id or a length mismatch. */
SNN_API float get_loss_all(float *labels, int num_labels, float *predictions, int num_predictions,
                           int loss_function);

/* ---------------------------------------------------------------------------
 * 2. Handle API
 * ------------------------------------------------------------------------- */

typedef struct snn_handle snn_handle;

typedef struct snn_desc {
    int n_train;          /* neighbour (training) points                               */
    int n_val;            /* scored (validation) points; 0 selects CV mode over n_train */
    int p;                /* features                                                  */
    const int *k_vals;    /* candidate k values (copied at create)                     */
    int num_k_vals;
    int backward;         /* 0 forward selection, 1 backward elimination               */
    int num_features;     /* forward: features to add; backward: features to keep     */
    int k_fold;           /* CV mode: number of folds (reference fold rule)            */
    int auto_feature;     /* stop when the error rises (nearest_neighbors_feature_selection.c:446-465) */
    int device;           /* CUDA device ordinal                                       */
} snn_desc;

/* Validate the descriptor, pick the device and allocate its buffers
 * (the committed distance matrix is n_rows x round_up(n_train, 32) floats). */
SNN_API int snn_create(const snn_desc *desc, snn_handle **out);

/* Copy host inputs to the device (row-major float32).  X_val/y_val are
 * ignored (may be NULL) in CV mode.  Resets the selection to step 0. */
SNN_API int snn_load(snn_handle *h, const float *X_train, const float *y_train, const float *X_val,
                     const float *y_val);

/* Run the whole selection (all greedy steps) on the handle's stream; blocks
 * until done. */
SNN_API int snn_run(snn_handle *h);

/* Restart from step 0 with the loaded data (no copies). */
SNN_API int snn_reset(snn_handle *h);

/* Run one greedy step.  Returns 1 if a step ran, 0 if the selection had
 * already finished, or a negative status.  Blocks until the step is done. */
SNN_API int snn_step(snn_handle *h);

/* Warm start / resume: restart from step 0 and commit seq[0..n) in order
 * (forward: features added; backward: features removed) without scoring
 * them, as the reference's distance update would have (the counterpart of
 * compute_distance_matrix_selected, speedynn/lib/cpu.c:185-215 with
 * selected_only, but in commit order so later steps stay bit-identical).
 * Their ordering slots are filled, their errors and best k stay 0.
 * Subsequent snn_step calls continue from step n. */
SNN_API int snn_commit_sequence(snn_handle *h, const int *seq, int n);

/* Results so far, all optional (NULL skips), arrays of length p, indexed like
 * the reference outputs: ordering/errors slot i is the step's loop index
 * (forward: step number; backward: p-1 down to num_features).
 * errors: FP32 RMSE bit-identical to the reference; errors64: the same
 * residuals summed in FP64; step_best_k: best k of each step's winner. */
SNN_API int snn_get_results(snn_handle *h, int *ordering, int *mask, float *errors, double *errors64,
                            int *step_best_k, int *best_k, int *num_final);

/* Model and losses (speedynn/lib/cpu.c:21-126, loss_functions.c:6-183).
 * model_type 0 predicts the mean of the k nearest labels, 1 (classification)
 * their mode with the reference's rule (first position of the strictly
 * largest count, each label counted at its first occurrence in rank order,
 * util.c:165-188).  Every loss of loss_ids (reference ids 0..8, the
 * SNN_LOSS_* values) is evaluated for every candidate and k with the
 * reference's float/double operation order; loss_ids[0] picks each
 * candidate's best k and the winner, and snn_get_errors_all returns all of
 * them for each step's winner.  When loss_ids[0] is not RMSE, errors64 of
 * snn_get_results holds that loss's FP32 value.  Default: {RMSE},
 * regression.  Resets a loaded handle to step 0. */
SNN_API int snn_set_model(snn_handle *h, const int *loss_ids, int n_losses, int model_type);

/* Every loss of every step, in the reference's selected_errors layout
 * errors[l * p + i] (n >= n_losses * p). */
SNN_API int snn_get_errors_all(snn_handle *h, float *errors, int n);

/* Neighbour lists of the most recent step, for inspection: when enabled
 * before a step, that step keeps idx/dist[n_cand][n_rows][k_max] (candidates
 * in the handle's slot order -- ascending training variance -- listed in
 * cands[n_cand]).  Pass NULL to query sizes through n_cand/k_max. */
SNN_API int snn_keep_neighbours(snn_handle *h, int enable);
SNN_API int snn_get_neighbours(snn_handle *h, int *cands, int *n_cand, int *k_max, int *idx, float *dist);

/* The kept lists of selected scored rows only (for problems whose full
 * lists are too large to copy): idx/dist[n_cand][n_sel][k_max] for
 * rows[0..n_sel), candidates as snn_get_neighbours lists them. */
SNN_API int snn_get_neighbours_rows(snn_handle *h, const int *rows, int n_sel, int *idx, float *dist);

/* Predictions of the most recent scored step for selected scored rows:
 * pred[n_cand][num_k_vals][n_sel] (kNN mean, or the mode for
 * classification), candidates in the order written to cands[n_cand]
 * (optional; n_cand receives the count).  Available until the next step or
 * reset, without snn_keep_neighbours. */
SNN_API int snn_get_predictions(snn_handle *h, const int *rows, int n_sel, int *cands, int *n_cand, float *pred);

/* Kernel time of the last snn_run/snn_step calls (CUDA events on the handle's
 * stream): total milliseconds and launches of the candidate-scoring kernel,
 * of the commit kernel and of everything the selection launched. */
SNN_API int snn_get_timing(snn_handle *h, double *score_ms, int *score_launches, double *commit_ms,
                           int *commit_launches, double *total_ms, int *total_launches);

/* Options:
 *   SNN_OPT_KERNEL scoring kernel: 0 automatic (3 for k_max <= 64, else 1),
 *                  1 rows per lane (any k_max <= 256), 3 row tiles fed by a
 *                  TMA/mbarrier ring (k_max <= 64).  Results are identical;
 *                  this exists for cross-checks and measurement. */
#define SNN_OPT_KERNEL 2
/*   SNN_OPT_COUNTERS 1: the TMA-fed scorer keeps the filter counters read by
 *                  snn_get_filter_counters (a little slower).  Default 0. */
#define SNN_OPT_COUNTERS 3
/*   SNN_OPT_SEED_STEP forward step (= features already committed) from which
 *                  the TMA-fed scorer takes each candidate's starting bound on
 *                  its k-th neighbour distance from 256 "seed" columns near
 *                  the row (kept by the previous commit) instead of a first
 *                  pass over a quarter of the columns.  Results are identical;
 *                  only the work differs.  Default 2 (3 when k_max > 16); a
 *                  large value turns it off. */
#define SNN_OPT_SEED_STEP 4
/*   SNN_OPT_SORTED_START 1 (default): the first two forward steps of a
 *                  holdout problem take their lists from training values
 *                  sorted at load instead of a scan.  Step 1 (nothing
 *                  committed, every candidate's distances one-dimensional): a
 *                  binary search and a short outward walk per (row,
 *                  candidate).  Step 2 (one feature committed): a walk of that
 *                  feature's sorted values in increasing committed distance,
 *                  ended once it exceeds the candidate's k-th distance.  Data
 *                  with too many tied distances fall back to the scan.  0:
 *                  scan these steps too.  Results are identical. */
#define SNN_OPT_SORTED_START 5
SNN_API int snn_set_option(snn_handle *h, int option, int value);

/* Tracing of the TMA-fed scorer since the last run/step/reset: (row, chunk)
 * pairs of its full passes (a chunk = 64 training columns), how many the
 * sign-bit filter flagged for exact re-scoring, and how many of those held a
 * passing column.  Kept by that scorer only (k_max <= 64) and only while
 * SNN_OPT_COUNTERS is set. */
SNN_API int snn_get_filter_counters(snn_handle *h, unsigned long long *row_chunks, unsigned long long *flagged,
                                    unsigned long long *passed);

/* CUDA-event milliseconds of each greedy step of the last run/step calls:
 * score_ms[i] and commit_ms[i] for i < n (0 past the steps run).  Returns the
 * number of steps timed. */
SNN_API int snn_get_step_timing(snn_handle *h, float *score_ms, float *commit_ms, int n);

/* CUDA-event milliseconds of the last reset's initial distance matrix: the
 * full distance over all features for backward elimination
 * (compute_distance_matrix_cpu, speedynn/lib/cpu.c:185-215, plus the per-row
 * maxima of the backward filter), the empty matrix for forward selection
 * (empty_distance_matrix_cpu, cpu.c:171-183).  Every run starts with a reset. */
SNN_API int snn_get_setup_timing(snn_handle *h, float *ms);

SNN_API int snn_destroy(snn_handle *h);

/* ---------------------------------------------------------------------------
 * 2b. Batches of independent problems
 *
 * No single reference function: the reference runs one problem per process
 * (global state, speedynn/lib/nearest_neighbors_feature_selection.c:6-35).
 * A batch runs many selections -- different shapes, k values, directions --
 * with each problem on its own CUDA stream so small problems overlap on the
 * GPU.  Problems are grouped into waves that fit the device memory budget
 * (max_device_bytes, or 0 for the free memory less a reserve); each wave's
 * handles are created, loaded, run and freed in turn.  Results are those of
 * snn_create/snn_load/snn_run on each problem alone.
 * ------------------------------------------------------------------------- */

typedef struct snn_batch snn_batch;

/* Copy and validate n descriptors (k_vals are copied); no device memory yet. */
SNN_API int snn_batch_create(const snn_desc *descs, int n, unsigned long long max_device_bytes, snn_batch **out);

/* Attach problem i's host inputs (row-major float32, as snn_load).  The
 * arrays are read during snn_batch_run and must stay valid until it returns. */
SNN_API int snn_batch_load(snn_batch *b, int i, const float *X_train, const float *y_train, const float *X_val,
                           const float *y_val);

/* Problem i's losses and model, as snn_set_model on a handle (loss ids 0..8,
 * the first decides; model_type 0 regression, 1 classification).  Call
 * before snn_batch_run; default {RMSE}, regression.  Counterpart:
 * train_*_selection's loss_functions and model_type
 * (speedynn/lib/nearest_neighbors_feature_selection.h:59-80). */
SNN_API int snn_batch_set_model(snn_batch *b, int i, const int *loss_ids, int n_losses, int model_type);

/* Run every problem's whole selection; blocks until all are done.  A failing
 * problem keeps its status for snn_batch_get_results; device or argument
 * errors stop the batch with a negative status. */
SNN_API int snn_batch_run(snn_batch *b);

/* Problem i's results, as snn_get_results; returns that problem's status. */
SNN_API int snn_batch_get_results(snn_batch *b, int i, int *ordering, int *mask, float *errors, double *errors64,
                                  int *step_best_k, int *best_k, int *num_final);

/* Problem i's errors of every loss for each step's winner, as
 * snn_get_errors_all ([loss][step slot], n >= n_losses * p). */
SNN_API int snn_batch_get_errors_all(snn_batch *b, int i, float *errors, int n);

/* Device time of the last snn_batch_run's selections, and the number of
 * waves.  Each problem's selection is issued on its stream as soon as the
 * problem is created and loaded, so later creates and uploads overlap earlier
 * selections; run_ms is the union, over waves, of the intervals in which some
 * selection of the wave was running (CUDA events around each problem's greedy
 * steps; creating, loading and reading results are outside them). */
SNN_API int snn_batch_get_timing(snn_batch *b, double *run_ms, int *waves);

SNN_API int snn_batch_destroy(snn_batch *b);

/* ---------------------------------------------------------------------------
 * 3. One greedy step without device allocation
 * ------------------------------------------------------------------------- */

/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- code running under another runtime's allocator or a fixed
 * memory budget, hosts that forbid allocation after start-up, paths that
 * must not let cudaMalloc/cudaFree synchronise the device -- this scores one
 * greedy step from caller-owned DEVICE buffers and writes every candidate's
 * RMSE for every k: errors[c * num_k_vals + m] (FP32, the reference's value)
 * and errors64 (same residuals summed in FP64).  It never allocates: its
 * scratch (kNN predictions, step state, copies of cands and k_vals) is a
 * fixed 16 MB static device array, so n_cand * num_k_vals * n_rows must not
 * exceed 4,194,304 (else SNN_ERR_ARG), num_k_vals <= 256, n_cand <= 1024.
 *
 * Layouts (the handle API's): D [n_rows][ld] committed distances with
 * ld % 64 == 0, ld >= n_train and +inf in columns >= n_train (and on
 * excluded pairs); XT [p][ld] training points feature-major; XV [p][ldr]
 * scored points feature-major; y_train [n_train], y_val [n_rows].  cands
 * and k_vals are HOST arrays (feature ids to score, k values).  backward=1
 * scores removals (D - square) instead of additions.  D and XT must be
 * 16-byte aligned (they are read with TMA copies).  For a forward step
 * (backward=0) every entry of D must be >= 0 or +inf, as sums of squares
 * are: the scorer's exact filter relies on it.  stream: a cudaStream_t
 * (NULL = legacy default stream); the call waits for it.
 *
 * The scratch is placed on a GPU when the CUDA runtime loads this library's
 * kernels there (lazily: at the first call of any library entry point on
 * that GPU), so a caller with a strict no-allocation window makes one call
 * per GPU before the window opens.  Every call looks up the scratch's device
 * address with the device current (it can move after a device reset); make
 * the first call on a device before any stream capture.  All calls share the
 * scratch and it keeps the last call's contents: calls whose GPU work
 * overlaps race on it. */
SNN_API int snn_score_step_noalloc(const float *D, int ld, const float *XT, const float *XV, int ldr,
                                   const float *y_train, const float *y_val, int n_rows, int n_train, int p,
                                   const int *cands, int n_cand, const int *k_vals, int num_k_vals, int backward,
                                   float *errors, double *errors64, void *stream);

/* Message of the last failure on the calling thread ("" if none). */
SNN_API const char *snn_last_error(void);

/* Library version string. */
SNN_API const char *snn_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SPEEDYNN_B200_H */
