/*
 * snn_oracle.c -- CPU restatement of speedynn's greedy kNN wrapper feature
 * selection (forward selection / backward elimination, each candidate scored
 * by kNN-regression RMSE).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: tests/, the smoke
 * check and the bench's CPU-baseline leg call it through ctypes to compare
 * against the CUDA product path.  It is never linked into, or called by, the
 * product library.
 *
 * Parity pin: tests/test_oracle_golden.py checks this restatement against
 * golden vectors produced by speedynn's own CPU backend (compiled from the
 * reference sources by oracle/Makefile, generator tests/golden/make_golden.py):
 * selected ordering, mask, per-step errors, best k and the neighbour indices
 * of get_k_nearest_neighbors_cpu.
 *
 * What it restates (reference file:line, paths inside the speedynn project):
 *   - fold rule: num_per_fold = n / k_fold, fold(i) = i / num_per_fold
 *     (speedynn/lib/cpu.c:38,48,139); an n % k_fold remainder forms an extra
 *     partial fold.
 *   - candidate distance d = D[r,i] + mult*((x_r,c - x_i,c)*(x_r,c - x_i,c)),
 *     product and sum rounded separately (cpu.c:142-144, util.c:19-21).
 *   - top-k_max insertion: slots start at (FLT_MAX, index 0); an item enters
 *     only if strictly below the last slot and bubbles while strictly smaller
 *     (cpu.c:128-168) -> a stable sort by (distance, index) of the items
 *     with distance < FLT_MAX, padded with (FLT_MAX, 0).
 *   - prediction: FP32 sum of labels in neighbour-rank order, then / k
 *     (cpu.c:56-66).
 *   - RMSE: FP32 sequential sum of squared residuals, / n, sqrt in double,
 *     stored as float (loss_functions.c:41-50).
 *   - best k: first strict minimum in k_vals order (cpu.c:111-120).
 *   - best candidate: first strict minimum in ascending dimension order
 *     (nearest_neighbors_feature_selection.c:155-167, :318-329).
 *   - committed distance: forward D = ((0 + s_w0) + s_w1) + ... in selection
 *     order (cpu.c:171-183, :217-231); backward D = sum over all dims taken
 *     in DESCENDING order (util.c:10-17), then minus each removed dim in
 *     removal order.
 *   - output indexing, auto_feature stop rule, return value
 *     (nearest_neighbors_feature_selection.c:76-233, :243-394, :446-465).
 *
 * Additions the reference does not have: a holdout mode (rows = validation
 * points, columns = training points, no folds), an FP64 accumulation of the
 * same FP32-model residuals, and an all-FP64 pipeline used to state the FP32
 * error of each reported RMSE.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef struct {
    const float *Xr;  /* scored rows, row-major [nr][p]   */
    const float *yr;
    int nr;
    const float *Xc;  /* neighbour columns, row-major [nc][p] */
    const float *yc;
    int nc;
    int p;
    int cv;           /* 1: rows and columns are the same points, same-fold excluded */
    int num_per_fold;
} problem_t;

static int kmax_of(const int *kvals, int nk)
{
    int m = kvals[0];
    for (int i = 1; i < nk; ++i)
        if (kvals[i] > m) m = kvals[i];
    return m;
}

/* Committed FP32 distance row D[r, :] for the committed sequence `seq`
 * (forward: added dims in order; backward: removed dims in order). */
static void d_row32(const problem_t *P, int r, const int *seq, int nseq, int backward, float *D)
{
    const int p = P->p;
    const float *a = P->Xr + (size_t)r * p;
    for (int i = 0; i < P->nc; ++i) {
        const float *b = P->Xc + (size_t)i * p;
        float d = 0.0f;
        if (backward) {
            for (int k = p; k--;) {
                float t = a[k] - b[k];
                d += t * t;
            }
            for (int s = 0; s < nseq; ++s) {
                float t = a[seq[s]] - b[seq[s]];
                float q = t * t;
                d = d - q;
            }
        } else {
            for (int s = 0; s < nseq; ++s) {
                float t = a[seq[s]] - b[seq[s]];
                float q = t * t;
                d = d + q;
            }
        }
        D[i] = d;
    }
}

static void d_row64(const problem_t *P, int r, const int *seq, int nseq, int backward, double *D)
{
    const int p = P->p;
    const float *a = P->Xr + (size_t)r * p;
    for (int i = 0; i < P->nc; ++i) {
        const float *b = P->Xc + (size_t)i * p;
        double d = 0.0;
        if (backward) {
            for (int k = p; k--;) {
                double t = (double)a[k] - (double)b[k];
                d += t * t;
            }
            for (int s = 0; s < nseq; ++s) {
                double t = (double)a[seq[s]] - (double)b[seq[s]];
                d -= t * t;
            }
        } else {
            for (int s = 0; s < nseq; ++s) {
                double t = (double)a[seq[s]] - (double)b[seq[s]];
                d += t * t;
            }
        }
        D[i] = d;
    }
}

static int excluded(const problem_t *P, int r, int i)
{
    return P->cv && (i / P->num_per_fold == r / P->num_per_fold);
}

/* top-k_max of candidate c for row r, reference insertion rule. */
static void topk32(const problem_t *P, int r, const float *D, int c, int backward,
                   int kmax, int *idx, float *dist)
{
    for (int j = 0; j < kmax; ++j) {
        idx[j] = 0;
        dist[j] = FLT_MAX;
    }
    const float ac = P->Xr[(size_t)r * P->p + c];
    for (int i = 0; i < P->nc; ++i) {
        if (excluded(P, r, i)) continue;
        float t = ac - P->Xc[(size_t)i * P->p + c];
        float q = t * t;
        float d = backward ? D[i] - q : D[i] + q;
        int j = kmax - 1;
        if (dist[j] > d) {
            dist[j] = d;
            idx[j] = i;
            for (; j > 0; --j) {
                if (dist[j] < dist[j - 1]) {
                    float tf = dist[j]; dist[j] = dist[j - 1]; dist[j - 1] = tf;
                    int ti = idx[j]; idx[j] = idx[j - 1]; idx[j - 1] = ti;
                } else {
                    break;
                }
            }
        }
    }
}

static void topk64(const problem_t *P, int r, const double *D, int c, int backward,
                   int kmax, int *idx, double *dist)
{
    for (int j = 0; j < kmax; ++j) {
        idx[j] = 0;
        dist[j] = DBL_MAX;
    }
    const double ac = P->Xr[(size_t)r * P->p + c];
    for (int i = 0; i < P->nc; ++i) {
        if (excluded(P, r, i)) continue;
        double t = ac - (double)P->Xc[(size_t)i * P->p + c];
        double d = backward ? D[i] - t * t : D[i] + t * t;
        int j = kmax - 1;
        if (dist[j] > d) {
            dist[j] = d;
            idx[j] = i;
            for (; j > 0; --j) {
                if (dist[j] < dist[j - 1]) {
                    double tf = dist[j]; dist[j] = dist[j - 1]; dist[j - 1] = tf;
                    int ti = idx[j]; idx[j] = idx[j - 1]; idx[j - 1] = ti;
                } else {
                    break;
                }
            }
        }
    }
}

static int init_problem(problem_t *P, const float *Xr, const float *yr, int nr,
                        const float *Xc, const float *yc, int nc, int p, int cv, int k_fold)
{
    if (nr <= 0 || nc <= 0 || p <= 0) return -1;
    P->Xr = Xr; P->yr = yr; P->nr = nr;
    P->Xc = Xc; P->yc = yc; P->nc = nc;
    P->p = p;
    P->cv = cv;
    P->num_per_fold = 1;
    if (cv) {
        if (k_fold <= 0 || k_fold > nr || nr != nc) return -1;
        P->num_per_fold = nr / k_fold;
    }
    return 0;
}

/*
 * One greedy step for a subset of rows.
 *
 * precision 0: reference FP32 path.  sq32[c][m][rr] = (y_r - pred)^2 in FP32,
 *              sq64[c][m][rr] = the same residual squared in FP64.
 * precision 1: all-FP64 pipeline (distances, neighbour order, predictions);
 *              only sq64 is written.
 * nn_idx / nn_dist (optional): [ncand][nrows_sel][kmax] neighbour lists.
 */
int snn_oracle_step(const float *Xr, const float *yr, int nr,
                    const float *Xc, const float *yc, int nc, int p,
                    int cv, int k_fold, const int *kvals, int nk,
                    int backward, const int *seq, int nseq,
                    const int *cands, int ncand,
                    const int *rows, int nrows_sel,
                    int precision, int nthreads,
                    int *nn_idx, float *nn_dist, float *sq32, double *sq64)
{
    problem_t P;
    if (init_problem(&P, Xr, yr, nr, Xc, yc, nc, p, cv, k_fold)) return -1;
    if (nk <= 0 || ncand < 0) return -1;
    for (int m = 0; m < nk; ++m)
        if (kvals[m] <= 0) return -1;
    const int kmax = kmax_of(kvals, nk);
    const int nsel = rows ? nrows_sel : nr;
    if (nthreads > 0) omp_set_num_threads(nthreads);

    int status = 0;
#pragma omp parallel
    {
        float *D32 = NULL;
        double *D64 = NULL;
        int *idx = (int *)malloc(sizeof(int) * (size_t)kmax);
        float *dist32 = (float *)malloc(sizeof(float) * (size_t)kmax);
        double *dist64 = (double *)malloc(sizeof(double) * (size_t)kmax);
        if (precision == 0) D32 = (float *)malloc(sizeof(float) * (size_t)nc);
        else D64 = (double *)malloc(sizeof(double) * (size_t)nc);
        if (!idx || !dist32 || !dist64 || (!D32 && !D64)) {
#pragma omp atomic write
            status = -2;
        } else {
#pragma omp for schedule(dynamic, 1)
            for (int rr = 0; rr < nsel; ++rr) {
                const int r = rows ? rows[rr] : rr;
                if (precision == 0) d_row32(&P, r, seq, nseq, backward, D32);
                else d_row64(&P, r, seq, nseq, backward, D64);
                for (int ci = 0; ci < ncand; ++ci) {
                    const int c = cands[ci];
                    if (precision == 0) topk32(&P, r, D32, c, backward, kmax, idx, dist32);
                    else topk64(&P, r, D64, c, backward, kmax, idx, dist64);
                    if (nn_idx) {
                        size_t o = ((size_t)ci * nsel + rr) * kmax;
                        for (int j = 0; j < kmax; ++j) {
                            nn_idx[o + j] = idx[j];
                            if (nn_dist) nn_dist[o + j] = precision == 0 ? dist32[j] : (float)dist64[j];
                        }
                    }
                    for (int m = 0; m < nk; ++m) {
                        const int k = kvals[m];
                        size_t o = ((size_t)ci * nk + m) * nsel + rr;
                        if (precision == 0) {
                            float pred = 0.0f;
                            for (int j = 0; j < k; ++j) pred += P.yc[idx[j]];
                            pred /= (float)k;
                            float e = P.yr[r] - pred;
                            if (sq32) sq32[o] = e * e;
                            double e64 = (double)P.yr[r] - (double)pred;
                            if (sq64) sq64[o] = e64 * e64;
                        } else {
                            double pred = 0.0;
                            for (int j = 0; j < k; ++j) pred += (double)P.yc[idx[j]];
                            pred /= (double)k;
                            double e64 = (double)P.yr[r] - pred;
                            if (sq64) sq64[o] = e64 * e64;
                        }
                    }
                }
            }
        }
        free(D32); free(D64); free(idx); free(dist32); free(dist64);
    }
    return status;
}

/* RMSE exactly as speedynn/lib/loss_functions.c:41-50 (sequential FP32 sum). */
static float rmse32_seq(const float *sq, int n)
{
    float sum = 0.0f;
    for (int i = 0; i < n; ++i) sum += sq[i];
    sum /= (float)n;
    return (float)sqrt((double)sum);
}

static double rmse64_seq(const double *sq, int n)
{
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += sq[i];
    return sqrt(sum / (double)n);
}

/*
 * Full greedy selection (forward or backward), reference semantics.
 *
 * Outputs (all length p): ordering, mask, errors (FP32, reference-exact),
 * errors64 (FP64 sum of the same residuals), step_best_k; scalar
 * final_best_k and num_final.  Indexing follows
 * nearest_neighbors_feature_selection.c:175-180 (backward) and :336-342
 * (forward).  Returns 0, or a negative status (-1 bad arguments, -2 out of
 * memory, -3 no candidate had a finite error).
 */
int snn_oracle_select(const float *Xr, const float *yr, int nr,
                      const float *Xc, const float *yc, int nc, int p,
                      int cv, int k_fold, const int *kvals, int nk,
                      int backward, int num_features, int auto_feature, int nthreads,
                      int *ordering, int *mask, float *errors, double *errors64,
                      int *step_best_k, int *final_best_k, int *num_final)
{
    problem_t P;
    if (init_problem(&P, Xr, yr, nr, Xc, yc, nc, p, cv, k_fold)) return -1;
    if (nk <= 0 || num_features < 0 || num_features > p) return -1;

    int *cands = (int *)malloc(sizeof(int) * (size_t)p);
    int *seq = (int *)malloc(sizeof(int) * (size_t)p);
    float *sq32 = (float *)malloc(sizeof(float) * (size_t)p * nk * nr);
    double *sq64 = (double *)malloc(sizeof(double) * (size_t)p * nk * nr);
    if (!cands || !seq || !sq32 || !sq64) {
        free(cands); free(seq); free(sq32); free(sq64);
        return -2;
    }
    for (int j = 0; j < p; ++j) {
        ordering[j] = 0;
        mask[j] = backward ? 1 : 0;
        errors[j] = 0.0f;
        errors64[j] = 0.0;
        step_best_k[j] = 0;
    }
    int desired = num_features;
    if (auto_feature) desired = backward ? 0 : p;
    int nfinal = backward ? p : 0;
    int nseq = 0;
    int best_k_last = 0;
    int status = 0;

    const int first = backward ? p - 1 : 0;
    for (int it = first; backward ? it >= desired : it < desired; it += backward ? -1 : 1) {
        nfinal += backward ? -1 : 1;
        int ncand = 0;
        for (int j = 0; j < p; ++j)
            if (mask[j] == (backward ? 1 : 0)) cands[ncand++] = j;
        status = snn_oracle_step(Xr, yr, nr, Xc, yc, nc, p, cv, k_fold, kvals, nk, backward,
                                 seq, nseq, cands, ncand, NULL, 0, 0, nthreads,
                                 NULL, NULL, sq32, sq64);
        if (status) break;
        float min_err = FLT_MAX;
        double min_err64 = 0.0;
        int min_dim = -1, min_k = 0;
        for (int ci = 0; ci < ncand; ++ci) {
            float best = FLT_MAX;
            double best64 = 0.0;
            int bestk = -1;
            for (int m = 0; m < nk; ++m) {
                float e = rmse32_seq(sq32 + ((size_t)ci * nk + m) * nr, nr);
                if (e < best) {
                    best = e;
                    bestk = kvals[m];
                    best64 = rmse64_seq(sq64 + ((size_t)ci * nk + m) * nr, nr);
                }
            }
            if (bestk < 0) continue; /* no finite error: never a winner */
            if (best < min_err) {
                min_err = best;
                min_err64 = best64;
                min_dim = cands[ci];
                min_k = bestk;
            }
        }
        if (min_dim < 0) {
            status = -3;
            break;
        }
        best_k_last = min_k;
        mask[min_dim] = backward ? 0 : 1;
        ordering[it] = min_dim;
        errors[it] = min_err;
        errors64[it] = min_err64;
        step_best_k[it] = min_k;
        seq[nseq++] = min_dim;
        if (auto_feature) {
            /* nearest_neighbors_feature_selection.c:446-465 */
            if (!backward) {
                if (it > 0 && errors[it - 1] < errors[it]) break;
            } else {
                if (it > 0 && it < p - 1 && errors[it + 1] < errors[it]) break;
            }
        }
    }
    *final_best_k = best_k_last;
    *num_final = nfinal;
    free(cands); free(seq); free(sq32); free(sq64);
    return status;
}
