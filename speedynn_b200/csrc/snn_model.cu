// snn_model.cu -- classification predictions and the reference's loss
// functions over every (candidate, k) prediction vector.
//
// Regression predictions (kNN means) come from the scoring kernels.  For the
// classification model (speedynn/lib/cpu.c:70-95) k_mode_predict replaces
// them with the mode of the k nearest labels, using the reference's rule
// (speedynn/lib/util.c:165-188): every label counts towards its first
// occurrence in rank order, and the first position with the strictly largest
// count wins.  k_losses evaluates the requested losses of
// speedynn/lib/loss_functions.c:6-183 with the reference's float/double
// operation order; loss 0 of the list decides best k and winner, as in
// cpu.c:104-120 and nearest_neighbors_feature_selection.c:316-330.
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "snn_internal.h"

namespace snn {

namespace {

// One thread per (candidate slot, scored row).  idx holds the row's k_max
// nearest training points in rank order.
__global__ void k_mode_predict(Bufs b, int n_cand)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n_cand * b.n_rows) return;
    const int slot = (int)(t / b.n_rows), r = (int)(t % b.n_rows);
    const int *idx = b.nn_idx + ((size_t)slot * b.n_rows + r) * b.kmax;
    for (int m = 0; m < b.nk; ++m) {
        const int k = b.kvals[m];
        int best = 0, best_cnt = -1;
        // count of position i = number of j in [i, k) whose label first occurs at i
        for (int i = 0; i < k; ++i) {
            const float yi = __ldg(b.yc + idx[i]);
            bool first = true;
            for (int j = 0; j < i && first; ++j) first = __ldg(b.yc + idx[j]) != yi;
            if (!first) continue;  // counted at its first occurrence
            int cnt = 0;
            for (int j = i; j < k; ++j) cnt += __ldg(b.yc + idx[j]) == yi;
            if (cnt > best_cnt) {  // the first strict maximum in position order
                best_cnt = cnt;
                best = i;
            }
        }
        b.pred[((size_t)slot * b.nk + m) * b.n_rows + r] = __ldg(b.yc + idx[best]);
    }
}

// Order-preserving key of a float (NaN above +inf).
__device__ __forceinline__ uint32_t fkey(float v)
{
    const uint32_t u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float fkey_inv(uint32_t k) { return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k); }

// Element of rank `rank` (0-based, ascending) of the n values val(i), by a
// most-significant-digit radix select over the keys; the whole block calls it.
template <class F>
__device__ float block_select(int n, int rank, F val, uint32_t *hist, uint32_t *shared_word)
{
    uint32_t prefix = 0u, mask = 0u;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[d] = 0u;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const uint32_t key = fkey(val(i));
            if ((key & mask) == prefix) atomicAdd(hist + ((key >> shift) & 255u), 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int d = 0;
            while (d < 255 && (int)hist[d] <= rank) rank -= (int)hist[d++];
            shared_word[0] = (uint32_t)d;
            shared_word[1] = (uint32_t)rank;
        }
        __syncthreads();
        prefix |= shared_word[0] << shift;
        mask |= 255u << shift;
        rank = (int)shared_word[1];
        __syncthreads();
    }
    return fkey_inv(prefix);
}

// speedynn/lib/loss_functions.c:88-111 (norm) and :66-86: median of the
// errors, then median of their distances to it (find_median = element n/2 of
// the sorted array, :173-183).
__device__ float mad_value(const float *pred, const float *y, int n, bool norm, uint32_t *hist, uint32_t *sw)
{
    auto err = [&](int i) {
        const float t = y[i];
        const float d = __fsub_rn(t, pred[i]);
        return norm ? (float)__ddiv_rn((double)d, __dadd_rn(1.0, (double)t)) : d;
    };
    const float m1 = block_select(n, n / 2, err, hist, sw);
    auto dev = [&](int i) { return fabsf(__fsub_rn(err(i), m1)); };
    return block_select(n, n / 2, dev, hist, sw);
}

// Sequential single-thread losses (thread 0 of the block).
__device__ float rmse_norm_value(const float *pred, const float *y, int n)
{
    float sum = 0.0f;
    for (int i = n; i--;) {  // loss_functions.c:55, descending
        const float t = y[i];
        const float tmp = (float)__ddiv_rn((double)__fsub_rn(t, pred[i]), __dadd_rn(1.0, (double)t));
        sum = __fadd_rn(sum, __fmul_rn(tmp, tmp));
    }
    sum = __fdiv_rn(sum, (float)n);
    return (float)sqrt((double)sum);
}

__device__ float std_value(const float *pred, const float *y, int n)
{
    float mean = 0.0f;
    for (int i = 0; i < n; ++i) mean = __fadd_rn(mean, __fsub_rn(y[i], pred[i]));
    mean = __fdiv_rn(mean, (float)n);
    // loss_functions.c:141 assigns instead of accumulating: only the last row counts
    const float a = __fsub_rn(__fsub_rn(y[n - 1], pred[n - 1]), mean);
    const float sum = __fdiv_rn(__fmul_rn(a, a), (float)(n - 1));
    return (float)sqrt((double)sum);
}

__device__ float rmse_value(const float *pred, const float *y, int n)
{
    float sum = 0.0f;
    for (int i = 0; i < n; ++i) {
        const float tmp = __fsub_rn(y[i], pred[i]);
        sum = __fadd_rn(sum, __fmul_rn(tmp, tmp));
    }
    sum = __fdiv_rn(sum, (float)n);
    return (float)sqrt((double)sum);
}

// loss_functions.c:113-127 passes the float difference to int abs(): on the
// host this truncates towards zero (x86 cvttss2si), and a difference that
// does not fit an int (or NaN) becomes INT_MIN, whose abs() stays negative.
// So a row counts as a miss iff 1 <= |t - p| < 2^31.
__device__ __forceinline__ unsigned zero_one_miss(float t, float p)
{
    const float a = fabsf(__fsub_rn(t, p));
    return (a >= 1.0f && a < 2147483648.0f) ? 1u : 0u;
}

// One block per (candidate slot, k index): every requested loss of that
// prediction vector into lossval[(l * n_cand + slot) * nk + m].  A non-RMSE
// deciding loss (index 0) also replaces rmse32/rmse64, which best k and the
// winner are chosen from.
__global__ void k_losses(Bufs b, int n_cand)
{
    __shared__ uint32_t hist[256];
    __shared__ uint32_t sw[2];
    __shared__ float comp[4];
    __shared__ unsigned miss_total;
    const int slot = blockIdx.x / b.nk, m = blockIdx.x % b.nk;
    const int n = b.n_rows;
    const float *pred = b.pred + ((size_t)slot * b.nk + m) * n;
    const float *y = b.yr;
    for (int l = 0; l < b.nloss; ++l) {
        const int id = b.loss_ids[l];
        float v = 0.0f;
        if (id == 2 || id == 3 || id == 6 || id == 7) {
            const float md = mad_value(pred, y, n, id != 2, hist, sw);
            if (threadIdx.x == 0) {
                if (id == 2 || id == 3) {
                    comp[0] = md;
                } else {
                    const float rn = rmse_norm_value(pred, y, n);
                    if (id == 6) {
                        const float sd = std_value(pred, y, n);
                        comp[0] = (float)__dadd_rn(__dadd_rn(__ddiv_rn((double)rn, 0.19), __ddiv_rn((double)md, 0.041)),
                                                   __ddiv_rn((double)sd, 0.16));
                    } else {
                        comp[0] = (float)__dadd_rn(__ddiv_rn((double)rn, 0.019), __ddiv_rn((double)md, 0.009));
                    }
                }
            }
        } else if (id == 4) {
            if (threadIdx.x == 0) miss_total = 0u;
            __syncthreads();
            unsigned c = 0u;
            for (int i = threadIdx.x; i < n; i += blockDim.x) c += zero_one_miss(y[i], pred[i]);
            atomicAdd(&miss_total, c);
            __syncthreads();
            // adding 1.0f once per miss in row order is exact below 2^24 misses
            if (threadIdx.x == 0) comp[0] = __fdiv_rn((float)miss_total, (float)n);
        } else if (threadIdx.x == 0) {
            // rmse32 holds the RMSE unless a non-RMSE loss 0 has replaced it
            if (id == 0) comp[0] = b.loss_ids[0] == 0 ? b.rmse32[slot * b.nk + m] : rmse_value(pred, y, n);
            else if (id == 1) comp[0] = rmse_norm_value(pred, y, n);
            else if (id == 5) comp[0] = std_value(pred, y, n);
            else if (id == 8) comp[0] = __fadd_rn(rmse_value(pred, y, n), std_value(pred, y, n));
            else comp[0] = NAN;
        }
        __syncthreads();
        v = comp[0];
        if (threadIdx.x == 0) {
            b.lossval[((size_t)l * n_cand + slot) * b.nk + m] = v;
            if (l == 0 && id != 0) {
                b.rmse32[slot * b.nk + m] = v;
                b.rmse64[slot * b.nk + m] = (double)v;
            }
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_mode_predict(const Bufs &b, int n_cand, cudaStream_t s)
{
    const long long n = (long long)n_cand * b.n_rows;
    if (n <= 0) return cudaSuccess;
    k_mode_predict<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(b, n_cand);
    return cudaGetLastError();
}

cudaError_t launch_losses(const Bufs &b, int n_cand, cudaStream_t s)
{
    if (n_cand <= 0) return cudaSuccess;
    k_losses<<<n_cand * b.nk, 256, 0, s>>>(b, n_cand);
    return cudaGetLastError();
}

}  // namespace snn
