// snn_kernels.cu -- sm_100a kernels of one greedy feature-selection step.
//
// Arithmetic contract (bit parity with speedynn's CPU path):
//   candidate distance  d = D[r,i] +/- fl(fl(x_r,c - x_i,c)^2)
//                       (speedynn/lib/cpu.c:142-144, util.c:19-21), every op
//                       rounded separately: __fsub_rn/__fmul_rn/__fadd_rn keep
//                       the compiler from contracting into FMA;
//   neighbour list      stable (distance, index) order of the items with
//                       distance < FLT_MAX, padded with (FLT_MAX, 0)
//                       (cpu.c:128-168);
//   prediction          FP32 label sum in rank order, then / k (cpu.c:56-66);
//   RMSE                FP32 sequential sum over rows, / n, sqrt in double,
//                       rounded to float (loss_functions.c:41-50);
//   committed distance  forward fl(D + s_w) in selection order
//                       (cpu.c:217-231); backward: full distance summed over
//                       dims in descending order (util.c:10-17), then
//                       fl(D - s_w) in removal order.
#include <float.h>
#include <math.h>

#include "snn_internal.h"

namespace snn {

namespace {

__device__ __forceinline__ float sqdiff(float a, float b)
{
    const float t = __fsub_rn(a, b);
    return __fmul_rn(t, t);
}

// ---------------------------------------------------------------------------
// Row-major [n][p] -> feature-major [p][ld], zero padded up to ld.
// ---------------------------------------------------------------------------
__global__ void k_transpose(const float *__restrict__ X, int n, int p, float *__restrict__ XT, int ld)
{
    __shared__ float tile[32][33];
    const int i0 = blockIdx.x * 32;  // points
    const int f0 = blockIdx.y * 32;  // features
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int i = i0 + k, f = f0 + threadIdx.x;
        tile[k][threadIdx.x] = (i < n && f < p) ? X[(size_t)i * p + f] : 0.0f;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int f = f0 + k, i = i0 + threadIdx.x;
        if (f < p && i < ld) XT[(size_t)f * ld + i] = tile[threadIdx.x][k];
    }
}

// ---------------------------------------------------------------------------
// Forward start: D = 0 on scored pairs, +inf on excluded / pad columns
// (speedynn/lib/cpu.c:171-183 zero-fills; exclusion is the fold rule of
// cpu.c:139 folded into the matrix so the scoring loop needs no test).
// ---------------------------------------------------------------------------
__global__ void k_init_forward(Bufs b, int cv, int npf)
{
    const int ld4 = b.ldc >> 2;
    for (int r = blockIdx.x; r < b.n_rows; r += gridDim.x) {
        const int lo = cv ? (r / npf) * npf : 0;
        float4 *row = reinterpret_cast<float4 *>(b.D + (size_t)r * b.ldc);
        for (int q = threadIdx.x; q < ld4; q += blockDim.x) {
            float v[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int i = q * 4 + e;
                const bool ex = (i >= b.n_cols) || (cv && (unsigned)(i - lo) < (unsigned)npf);
                v[e] = ex ? INFINITY : 0.0f;
            }
            row[q] = make_float4(v[0], v[1], v[2], v[3]);
        }
    }
}

// ---------------------------------------------------------------------------
// Backward start: full distance over all p dims, summed in DESCENDING
// dimension order (speedynn/lib/util.c:10-17).  64x64 output tile per block,
// 4x4 per thread, features streamed through shared memory in chunks.
// ---------------------------------------------------------------------------
constexpr int kFdTile = 64;
constexpr int kFdChunk = 16;

__global__ void __launch_bounds__(256) k_full_distance(Bufs b, int cv, int npf)
{
    __shared__ __align__(16) float sv[kFdChunk][kFdTile];
    __shared__ __align__(16) float sc[kFdChunk][kFdTile];
    const int r0 = blockIdx.y * kFdTile;
    const int i0 = blockIdx.x * kFdTile;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = 0.0f;

    for (int kk = b.p; kk > 0; kk -= kFdChunk) {
        const int kb = kk > kFdChunk ? kk - kFdChunk : 0;
        const int cnt = kk - kb;
        __syncthreads();
        for (int e = threadIdx.x; e < kFdChunk * kFdTile; e += blockDim.x) {
            const int q = e / kFdTile, x = e % kFdTile;
            float a = 0.0f, c = 0.0f;
            if (q < cnt) {
                a = b.XV[(size_t)(kb + q) * b.ldr + r0 + x];  // ldr, ldc are multiples of 64
                c = b.XT[(size_t)(kb + q) * b.ldc + i0 + x];
            }
            sv[q][x] = a;
            sc[q][x] = c;
        }
        __syncthreads();
        for (int q = cnt - 1; q >= 0; --q) {
            const float4 a4 = *reinterpret_cast<const float4 *>(&sv[q][ty * 4]);
            const float4 c4 = *reinterpret_cast<const float4 *>(&sc[q][tx * 4]);
            const float a[4] = {a4.x, a4.y, a4.z, a4.w};
            const float c[4] = {c4.x, c4.y, c4.z, c4.w};
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = __fadd_rn(acc[u][v], sqdiff(a[u], c[v]));
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int r = r0 + ty * 4 + u;
        if (r >= b.n_rows) continue;
        const int lo = cv ? (r / npf) * npf : 0;
        float v4[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int i = i0 + tx * 4 + v;
            const bool ex = (i >= b.n_cols) || (cv && (unsigned)(i - lo) < (unsigned)npf);
            v4[v] = ex ? INFINITY : acc[u][v];
        }
        *reinterpret_cast<float4 *>(b.D + (size_t)r * b.ldc + i0 + tx * 4) = make_float4(v4[0], v4[1], v4[2], v4[3]);
    }
}

// ---------------------------------------------------------------------------
// Per (candidate, k) error: one warp per pair.  Lanes form the squared
// residuals in parallel; lane 0 adds them in row order in FP32 (the
// reference's sequential sum); every lane also accumulates its residuals in
// FP64, combined by a fixed shuffle tree (deterministic).
// ---------------------------------------------------------------------------
constexpr int kReduceWarps = 4;
constexpr int kReduceChunk = 256;

__global__ void __launch_bounds__(kReduceWarps * 32) k_reduce(Bufs b, int n_cand)
{
    __shared__ float sq[kReduceWarps][kReduceChunk];
    if (b.st->done) return;
    const int wl = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int w = blockIdx.x * kReduceWarps + wl;
    if (w >= n_cand * b.nk) return;
    const float *pr = b.pred + (size_t)w * b.n_rows;
    float s32 = 0.0f;
    double s64 = 0.0;
    constexpr int Q = kReduceChunk / 32;
    // the next chunk's values are loaded while lane 0 sums the current one
    float pv[Q], yv[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int rr = q * 32 + lane;
        pv[q] = rr < b.n_rows ? pr[rr] : 0.0f;
        yv[q] = rr < b.n_rows ? b.yr[rr] : 0.0f;
    }
    for (int base = 0; base < b.n_rows; base += kReduceChunk) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int rr = base + q * 32 + lane;
            if (rr < b.n_rows) {
                const float e = __fsub_rn(yv[q], pv[q]);
                sq[wl][q * 32 + lane] = __fmul_rn(e, e);
                const double e64 = (double)yv[q] - (double)pv[q];
                s64 += e64 * e64;
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int rr = base + kReduceChunk + q * 32 + lane;
            pv[q] = rr < b.n_rows ? pr[rr] : 0.0f;
            yv[q] = rr < b.n_rows ? b.yr[rr] : 0.0f;
        }
        if (lane == 0) {
            const int cnt = min(kReduceChunk, b.n_rows - base);
            for (int t = 0; t < cnt; ++t) s32 = __fadd_rn(s32, sq[wl][t]);
        }
        __syncwarp();
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s64 += __shfl_down_sync(0xffffffffu, s64, off);
    if (lane == 0) {
        const float mean = __fdiv_rn(s32, (float)b.n_rows);
        b.rmse32[w] = __double2float_rn(sqrt((double)mean));
        b.rmse64[w] = sqrt(s64 / (double)b.n_rows);
    }
}

// ---------------------------------------------------------------------------
// Best k per candidate (first strict minimum in k_vals order, cpu.c:111-120),
// best candidate (first strict minimum in ascending feature order,
// nearest_neighbors_feature_selection.c:155-167 / :318-329), bookkeeping as in
// :169-181 / :331-342, next candidate list, auto stop (:446-465).
// ---------------------------------------------------------------------------
__global__ void k_select(Bufs b, int n_cand, int it, int t, int total_steps, int backward, int auto_feature)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    State *st = b.st;
    if (st->done) return;
    float minv = FLT_MAX;
    double min64 = 0.0;
    int wi = -1, wk = 0, wm = 0;
    for (int ci = 0; ci < n_cand; ++ci) {
        float best = FLT_MAX;
        int bm = -1;
        for (int m = 0; m < b.nk; ++m) {
            const float e = b.rmse32[ci * b.nk + m];
            if (e < best) {
                best = e;
                bm = m;
            }
        }
        if (bm < 0) continue;
        // first strict minimum in ascending feature order (slots follow perm)
        if (best < minv || (best == minv && wi >= 0 && b.cands[ci] < b.cands[wi])) {
            minv = best;
            wi = ci;
            wm = bm;
            wk = b.kvals[bm];
            min64 = b.rmse64[ci * b.nk + bm];
        }
    }
    for (int ci = 0; ci < n_cand; ++ci) b.prev_cands[ci] = b.cands[ci];
    if (wi < 0) {
        st->error = -5;  // SNN_ERR_NO_WINNER
        st->done = 1;
        return;
    }
    const int wdim = b.cands[wi];
    st->winner = wdim;
    b.order[it] = wdim;
    b.err[it] = minv;
    b.err64[it] = min64;
    b.stepk[it] = wk;
    for (int l = 0; l < b.nloss; ++l) b.err_all[l * b.p + it] = b.lossval[((size_t)l * n_cand + wi) * b.nk + wm];
    st->best_k_last = wk;
    b.mask[wdim] = backward ? 0 : 1;
    st->num_final = backward ? b.p - (t + 1) : t + 1;
    st->step = t + 1;
    int nc = 0;
    for (int jj = 0; jj < b.p; ++jj) {
        const int j = b.perm[jj];
        if (b.mask[j] == (backward ? 1 : 0)) b.cands[nc++] = j;
    }
    st->n_cand = nc;
    if (auto_feature) {
        if (!backward) {
            if (it > 0 && b.err[it - 1] < b.err[it]) st->done = 1;
        } else {
            if (it > 0 && it < b.p - 1 && b.err[it + 1] < b.err[it]) st->done = 1;
        }
    }
    if (t + 1 >= total_steps) st->done = 1;
}

// Warm start: record a given winner without scoring (same bookkeeping as
// k_select), so the commit kernel and later steps see it.
__global__ void k_force(Bufs b, int w, int it, int t, int total_steps, int backward)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    State *st = b.st;
    st->winner = w;
    b.order[it] = w;
    b.err[it] = 0.0f;
    b.err64[it] = 0.0;
    b.stepk[it] = 0;
    b.mask[w] = backward ? 0 : 1;
    st->num_final = backward ? b.p - (t + 1) : t + 1;
    st->step = t + 1;
    int nc = 0;
    for (int jj = 0; jj < b.p; ++jj) {
        const int j = b.perm[jj];
        if (b.mask[j] == (backward ? 1 : 0)) b.cands[nc++] = j;
    }
    st->n_cand = nc;
    if (t + 1 >= total_steps) st->done = 1;
}

__global__ void k_reset_state(Bufs b, int backward, int total_steps)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < b.p) {
        b.mask[j] = backward ? 1 : 0;
        b.order[j] = 0;
        b.err[j] = 0.0f;
        b.err64[j] = 0.0;
        b.stepk[j] = 0;
        b.cands[j] = b.perm[j];
        b.prev_cands[j] = b.perm[j];
        for (int l = 0; l < b.nloss; ++l) b.err_all[l * b.p + j] = 0.0f;
    }
    if (j == 0) {
        State s;
        s.step = 0;
        s.done = total_steps <= 0 ? 1 : 0;
        s.error = 0;
        s.winner = -1;
        s.n_cand = b.p;
        s.best_k_last = 0;
        s.num_final = backward ? b.p : 0;
        s.full_scan = 0;
        *b.st = s;
    }
}

// One block per row: the largest finite committed distance (non-negative
// finite floats order like their bit patterns).  Backward elimination only
// lowers D afterwards, so the value bounds the row for the whole run.
__global__ void k_row_dmax(Bufs b, float *dmax)
{
    const int r = blockIdx.x;
    const float *d = b.D + (size_t)r * b.ldc;
    float m = 0.0f;
    for (int i = threadIdx.x; i < b.n_cols; i += blockDim.x) {
        const float v = d[i];
        if (v < INFINITY && v > m) m = v;  // skips +inf (excluded pairs) and NaN
    }
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float red[32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmaxf(m, red[w]);
        dmax[r] = fmaxf(m, red[0]);
    }
}

// One block per feature: variance of the training column (FP64 sums).  Used
// only to order candidate slots so that a scoring warp's candidates have
// distances of similar scale; never part of a result.
__global__ void k_feature_variance(Bufs b, float *var)
{
    const int j = blockIdx.x;
    const float *x = b.XT + (size_t)j * b.ldc;
    double s1 = 0.0, s2 = 0.0;
    for (int i = threadIdx.x; i < b.n_cols; i += blockDim.x) {
        const double v = x[i];
        s1 += v;
        s2 += v * v;
    }
    __shared__ double r1[8], r2[8];
    for (int o = 16; o > 0; o >>= 1) {
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
        s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if ((threadIdx.x & 31) == 0) {
        r1[threadIdx.x >> 5] = s1;
        r2[threadIdx.x >> 5] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t1 = 0.0, t2 = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            t1 += r1[w];
            t2 += r2[w];
        }
        const double m = t1 / b.n_cols;
        const double v = t2 / b.n_cols - m * m;
        var[j] = isfinite(v) ? (float)fmax(v, 0.0) : NAN;
    }
}

// Stable ascending order of the feature variances, NaN last: each thread
// ranks one feature by counting the features that precede it (O(p^2), p is
// the number of features).
__global__ void k_feature_order(const float *var, int p, int *perm)
{
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < p; j += gridDim.x * blockDim.x) {
        const float vj = var[j];
        const bool nj = isnan(vj);
        int rank = 0;
        for (int i = 0; i < p; ++i) {
            const float vi = var[i];
            const bool ni = isnan(vi);
            bool before;
            if (ni != nj) before = nj;    // finite before NaN
            else if (ni) before = i < j;  // both NaN: by id
            else before = vi < vj || (vi == vj && i < j);
            rank += before ? 1 : 0;
        }
        perm[rank] = j;
    }
}

int sm_count()
{
    // initialised once, thread-safely (handles may be created from several threads)
    static const int n = [] {
        int dev = 0, c = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
        return c > 0 ? c : 148;
    }();
    return n;
}

}  // namespace

cudaError_t launch_transpose(const float *X, int n, int p, float *XT, int ld, cudaStream_t s)
{
    dim3 grid((ld + 31) / 32, (p + 31) / 32);
    k_transpose<<<grid, dim3(32, 8), 0, s>>>(X, n, p, XT, ld);
    return cudaGetLastError();
}

cudaError_t launch_init_forward(const Bufs &b, int cv, int npf, cudaStream_t s)
{
    int grid = b.n_rows < sm_count() * 8 ? b.n_rows : sm_count() * 8;
    k_init_forward<<<grid, 256, 0, s>>>(b, cv, npf);
    return cudaGetLastError();
}

cudaError_t launch_full_distance(const Bufs &b, int cv, int npf, cudaStream_t s)
{
    dim3 grid(b.ldc / kFdTile, (b.n_rows + kFdTile - 1) / kFdTile);
    k_full_distance<<<grid, 256, 0, s>>>(b, cv, npf);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const Bufs &b, int n_cand, cudaStream_t s)
{
    const int pairs = n_cand * b.nk;
    k_reduce<<<(pairs + kReduceWarps - 1) / kReduceWarps, kReduceWarps * 32, 0, s>>>(b, n_cand);
    return cudaGetLastError();
}

cudaError_t launch_select(const Bufs &b, int n_cand, int it, int t, int total_steps, int backward, int auto_feature,
                          cudaStream_t s)
{
    k_select<<<1, 32, 0, s>>>(b, n_cand, it, t, total_steps, backward, auto_feature);
    return cudaGetLastError();
}

cudaError_t launch_force(const Bufs &b, int w, int it, int t, int total_steps, int backward, cudaStream_t s)
{
    k_force<<<1, 32, 0, s>>>(b, w, it, t, total_steps, backward);
    return cudaGetLastError();
}

cudaError_t launch_feature_variance(const Bufs &b, float *var, cudaStream_t s)
{
    k_feature_variance<<<b.p, 256, 0, s>>>(b, var);
    return cudaGetLastError();
}

cudaError_t launch_feature_order(const float *var, int p, int *perm, cudaStream_t s)
{
    k_feature_order<<<(p + 127) / 128, 128, 0, s>>>(var, p, perm);
    return cudaGetLastError();
}

cudaError_t launch_row_dmax(const Bufs &b, float *dmax, cudaStream_t s)
{
    k_row_dmax<<<b.n_rows, 256, 0, s>>>(b, dmax);
    return cudaGetLastError();
}

cudaError_t launch_reset_state(const Bufs &b, int backward, int total_steps, cudaStream_t s)
{
    k_reset_state<<<(b.p + 127) / 128, 128, 0, s>>>(b, backward, total_steps);
    return cudaGetLastError();
}

}  // namespace snn
