// snn_sorted.cu -- the first forward step of a holdout problem from sorted
// feature columns.
//
// Before anything is committed, D is zero on every (scored row, training
// column) pair, so candidate c's distances are one-dimensional:
// d_i = fl(fl(x_r,c - x_i,c)^2) (speedynn/lib/cpu.c:142-144 with D = 0).  With
// the training values of c sorted, t = fl(x_r - x_i) is monotone in x_i and d
// is non-increasing up to x_r's insertion point and non-decreasing after it,
// so the k smallest distances are a window around that point.  One thread per
// (candidate, row) finds the point by binary search and walks outwards, taking
// the smaller frontier distance each time; all columns with the same distance
// (a tie group: a contiguous run on each side) are taken together and ordered
// by column index, which reproduces the reference's stable (distance, index)
// order (cpu.c:128-168).  The walk ends at k entries or at the first distance
// >= FLT_MAX (such items never enter a list); the rest is padding (FLT_MAX, 0).
// Then the kNN-mean predictions as the scoring kernels form them (cpu.c:56-66).
// The second step walks the first winner's sorted values the same way
// (k_second_step below).
//
// A tie group larger than kTieCap (e.g. integer-valued features with
// thousands of equal values) is not resolved here: the thread raises
// State::full_scan and the step's regular scoring launch, which otherwise
// returns at once, scores every problem by the full scan.
#include <cub/device/device_segmented_radix_sort.cuh>
#include <float.h>
#include <math.h>

#include "snn_internal.h"

namespace snn {

namespace {

constexpr int kTieCap = 64;  // columns of one tie group a thread orders itself

// Sort keys: the training values, NaN as +inf (its distance is NaN or inf, so
// it never enters a list wherever it sorts); pad columns are outside the segments.
__global__ void k_sort_keys(const float *XT, int ldc, int n_cols, int p, float *keys, int *vals, int *offsets)
{
    const size_t total = (size_t)p * ldc;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(e % ldc);
        const float x = XT[e];
        keys[e] = isnan(x) ? INFINITY : x;
        vals[e] = i;
    }
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < p) {
        offsets[j] = j * ldc;
        offsets[p + j] = j * ldc + n_cols;
    }
}

__device__ __forceinline__ float dist1(float a, float b)
{
    const float t = __fsub_rn(a, b);
    const float d = __fmul_rn(t, t);
    return d < FLT_MAX ? d : INFINITY;  // NaN and values at or above FLT_MAX never enter
}

// Sorted insertion of column index v into ix[0..n) (ascending).
__device__ __forceinline__ void insert_idx(int *ix, int n, int v)
{
    int j = n;
    while (j > 0 && ix[j - 1] > v) {
        ix[j] = ix[j - 1];
        --j;
    }
    ix[j] = v;
}

template <int KL>
__global__ void __launch_bounds__(256) k_first_step(Bufs b, const float *sv, const int *si, int n_cand)
{
    if (b.st->done) return;
    const int slot = blockIdx.y;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= n_cand || r >= b.n_rows) return;
    const int c = b.cands[slot];
    const int K = b.kmax;
    const int n = b.n_cols;
    const float *bv = sv + (size_t)c * b.ldc;
    const int *bi = si + (size_t)c * b.ldc;
    const float a = b.XV[(size_t)c * b.ldr + r];

    float ld[KL];
    int li[KL];
    int cnt = 0;
    if (isfinite(a)) {
        int lo = 0, hi = n;  // first position with value >= a
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (bv[mid] < a) lo = mid + 1;
            else hi = mid;
        }
        int L = lo - 1, R = lo;
        float dl = L >= 0 ? dist1(a, bv[L]) : INFINITY;
        float dr = R < n ? dist1(a, bv[R]) : INFINITY;
        int tie[kTieCap];
        while (cnt < K) {
            const float dm = fminf(dl, dr);
            if (!(dm < FLT_MAX)) break;
            int g = 0;
            bool over = false;
            while (L >= 0 && dl == dm) {  // the group's run on the left
                if (g < kTieCap) insert_idx(tie, g, bi[L]);
                else over = true;
                ++g;
                --L;
                dl = L >= 0 ? dist1(a, bv[L]) : INFINITY;
            }
            while (R < n && dr == dm) {  // and on the right
                if (g < kTieCap) insert_idx(tie, g, bi[R]);
                else over = true;
                ++g;
                ++R;
                dr = R < n ? dist1(a, bv[R]) : INFINITY;
            }
            if (over) {  // more equal distances than this thread orders: full scan
                atomicExch(&b.st->full_scan, 1);
                return;
            }
            for (int j = 0; j < g && cnt < K; ++j) {
                ld[cnt] = dm;
                li[cnt] = tie[j];
                ++cnt;
            }
        }
    }
    for (int j = cnt; j < K; ++j) {
        ld[j] = FLT_MAX;
        li[j] = 0;
    }
    if (b.nn_idx) {
        const size_t o = ((size_t)slot * b.n_rows + r) * K;
        for (int j = 0; j < K; ++j) {
            b.nn_idx[o + j] = li[j];
            b.nn_dist[o + j] = ld[j];
        }
    }
    // labels summed in rank order (sequential FP32), as the scoring kernels
    float acc = 0.0f;
    for (int j = 0; j < K; ++j) {
        acc = __fadd_rn(acc, __ldg(b.yc + li[j]));
        for (int m = 0; m < b.nk; ++m) {
            const int k = __ldg(b.kvals + m);
            if (k == j + 1) b.pred[((size_t)slot * b.nk + m) * b.n_rows + r] = __fdiv_rn(acc, (float)k);
        }
    }
}

// k_second_step: the second forward step of a holdout problem.  With one
// feature w committed, D[r][i] = fl(fl(x_r,w - x_i,w)^2) is one-dimensional
// again, so walking w's sorted values outwards from x_r,w (the smaller
// frontier D first) visits the columns in increasing D.  Candidate c's
// distance d = fl(D + fl((x_r,c - x_i,c)^2)) is at least D, so once the
// frontier D exceeds the k-th distance of the list held so far no further
// column can enter and the walk ends.  Columns arrive out of index order, so
// the list is kept sorted by (distance, index), the reference's stable order.
// D is recomputed from the sorted values (the same rounding the commit used),
// not read from memory.
//
// Walks are usually short (on the fwd-64k data a median of ~1,000 columns of
// 65,536) but not bounded: every warp adds its lanes' walked columns to a
// global count every 256 steps, and once the count passes `budget` (an
// eighth of a full scan) the kernel raises State::full_scan and every warp
// leaves; the step's regular scoring launch then scans everything.
template <int KL>
__global__ void __launch_bounds__(256) k_second_step(Bufs b, const float *sv, const int *si, int n_cand,
                                                     unsigned long long *walked, unsigned long long budget)
{
    if (b.st->done) return;
    const unsigned kFull = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int slot = blockIdx.y;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = slot < n_cand && r < b.n_rows;
    const int K = b.kmax;
    const int n = b.n_cols;
    const int w = b.st->winner;
    const int c = valid ? b.cands[slot] : 0;
    const float aw = valid ? b.XV[(size_t)w * b.ldr + r] : 0.0f;
    const float ac = valid ? b.XV[(size_t)c * b.ldr + r] : 0.0f;
    const float *bv = sv + (size_t)w * b.ldc;
    const int *bi = si + (size_t)w * b.ldc;
    const float *xc = b.XT + (size_t)c * b.ldc;

    float ld[KL];
    int li[KL];
    int cnt = 0;
    // non-finite x_r,w or x_r,c: no distance below FLT_MAX, the list stays padding
    bool active = valid && isfinite(aw) && isfinite(ac);
    int L = -1, R = 0;
    float dl = INFINITY, dr = INFINITY;
    if (active) {
        int lo = 0, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (bv[mid] < aw) lo = mid + 1;
            else hi = mid;
        }
        L = lo - 1;
        R = lo;
        dl = L >= 0 ? dist1(aw, bv[L]) : INFINITY;
        dr = R < n ? dist1(aw, bv[R]) : INFINITY;
    }
    for (unsigned it = 1;; ++it) {
        if ((it & 255u) == 0u) {  // account for the walk; leave when the budget is spent
            const unsigned act = __popc(__ballot_sync(kFull, active));
            int stop = 0;
            if (lane == 0) {
                const unsigned long long tot = atomicAdd(walked, 256ull * act) + 256ull * act;
                if (tot > budget) atomicExch(&b.st->full_scan, 1);
                stop = tot > budget || *(volatile int *)&b.st->full_scan;
            }
            if (__shfl_sync(kFull, stop, 0)) return;
        }
        if (!__any_sync(kFull, active)) break;
        if (!active) continue;
        const float dm = fminf(dl, dr);
        if (!(dm < FLT_MAX) || (cnt == K && dm > ld[K - 1])) {
            active = false;
            continue;
        }
        int j;
        if (dl <= dr) {
            j = L--;
            dl = L >= 0 ? dist1(aw, bv[L]) : INFINITY;
        } else {
            j = R++;
            dr = R < n ? dist1(aw, bv[R]) : INFINITY;
        }
        const int i = bi[j];
        const float t = __fsub_rn(ac, __ldg(xc + i));
        const float d = __fadd_rn(dm, __fmul_rn(t, t));
        if (d < FLT_MAX && (cnt < K || d < ld[K - 1] || (d == ld[K - 1] && i < li[K - 1]))) {
            int q = cnt < K ? cnt++ : K - 1;  // the last entry drops out of a full list
            while (q > 0 && (ld[q - 1] > d || (ld[q - 1] == d && li[q - 1] > i))) {
                ld[q] = ld[q - 1];
                li[q] = li[q - 1];
                --q;
            }
            ld[q] = d;
            li[q] = i;
        }
    }
    if (!valid) return;
    for (int j = cnt; j < K; ++j) {
        ld[j] = FLT_MAX;
        li[j] = 0;
    }
    if (b.nn_idx) {
        const size_t o = ((size_t)slot * b.n_rows + r) * K;
        for (int j = 0; j < K; ++j) {
            b.nn_idx[o + j] = li[j];
            b.nn_dist[o + j] = ld[j];
        }
    }
    float acc = 0.0f;
    for (int j = 0; j < K; ++j) {
        acc = __fadd_rn(acc, __ldg(b.yc + li[j]));
        for (int m = 0; m < b.nk; ++m) {
            const int k = __ldg(b.kvals + m);
            if (k == j + 1) b.pred[((size_t)slot * b.nk + m) * b.n_rows + r] = __fdiv_rn(acc, (float)k);
        }
    }
}

}  // namespace

size_t sort_temp_bytes(int p, int ldc)
{
    size_t bytes = 0;
    cub::DeviceSegmentedRadixSort::SortPairs(nullptr, bytes, (const float *)nullptr, (float *)nullptr,
                                             (const int *)nullptr, (int *)nullptr, p * ldc, p, (const int *)nullptr,
                                             (const int *)nullptr, 0, 32, (cudaStream_t)0);
    return bytes;
}

cudaError_t launch_sort_features(const Bufs &b, float *keys, int *vals, int *offsets, float *sv, int *si, void *temp,
                                 size_t temp_bytes, cudaStream_t s)
{
    const long long total = (long long)b.p * b.ldc;
    int grid = (int)std::min<long long>((total + 255) / 256, 4096);
    if (grid < (b.p + 255) / 256) grid = (b.p + 255) / 256;
    k_sort_keys<<<grid, 256, 0, s>>>(b.XT, b.ldc, b.n_cols, b.p, keys, vals, offsets);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return cub::DeviceSegmentedRadixSort::SortPairs(temp, temp_bytes, keys, sv, vals, si, b.p * b.ldc, b.p, offsets,
                                                    offsets + b.p, 0, 32, s);
}

cudaError_t launch_second_step(const Bufs &b, const float *sv, const int *si, int n_cand,
                               unsigned long long *walked, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(walked, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    const unsigned long long budget = (unsigned long long)b.n_rows * (unsigned long long)n_cand * b.n_cols / 8;
    const dim3 grid((b.n_rows + 255) / 256, n_cand);
    if (b.kmax <= 16) k_second_step<16><<<grid, 256, 0, s>>>(b, sv, si, n_cand, walked, budget);
    else if (b.kmax <= 64) k_second_step<64><<<grid, 256, 0, s>>>(b, sv, si, n_cand, walked, budget);
    else k_second_step<kScoreMaxK><<<grid, 256, 0, s>>>(b, sv, si, n_cand, walked, budget);
    return cudaGetLastError();
}

cudaError_t launch_first_step(const Bufs &b, const float *sv, const int *si, int n_cand, cudaStream_t s)
{
    const dim3 grid((b.n_rows + 255) / 256, n_cand);
    if (b.kmax <= 16) k_first_step<16><<<grid, 256, 0, s>>>(b, sv, si, n_cand);
    else if (b.kmax <= 64) k_first_step<64><<<grid, 256, 0, s>>>(b, sv, si, n_cand);
    else k_first_step<kScoreMaxK><<<grid, 256, 0, s>>>(b, sv, si, n_cand);
    return cudaGetLastError();
}

}  // namespace snn
