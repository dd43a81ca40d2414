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

cudaError_t launch_first_step(const Bufs &b, const float *sv, const int *si, int n_cand, cudaStream_t s)
{
    const dim3 grid((b.n_rows + 255) / 256, n_cand);
    if (b.kmax <= 16) k_first_step<16><<<grid, 256, 0, s>>>(b, sv, si, n_cand);
    else if (b.kmax <= 64) k_first_step<64><<<grid, 256, 0, s>>>(b, sv, si, n_cand);
    else k_first_step<kScoreMaxK><<<grid, 256, 0, s>>>(b, sv, si, n_cand);
    return cudaGetLastError();
}

}  // namespace snn
