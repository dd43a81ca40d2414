// snn_commit.cu -- commit the winning feature into the distance matrix.
//
// k_commit: D <- fl(D +/- fl((x_r,w - x_i,w)^2)) in place for the winner w of
// the step that just ran (read from the device state, so the host never waits
// for it): speedynn/lib/cpu.c:217-231 and
// kernels/update_current_distance_matrix_float.cl:5-32, with the product and
// the sum rounded separately.  A warp streams one row with 16-byte loads and
// stores (HBM-bound: 8 bytes per entry).
//
// Seeds (forward steps only).  While it streams a row, each lane also keeps
// the kSeedsPerLane (8) smallest new distances among the columns it visits
// (lane l sees the float4 groups l, l+32, l+64, ...), so every row leaves 256
// distinct real columns that lie near it under the committed features:
// seeds[r][j*32+l] and their distances seed_d[r][j*32+l] (lane l's j-th
// smallest; index -1 and +inf where a lane saw fewer finite distances).  The
// next forward scoring step takes, for each candidate, the k-th smallest
// exact distance over these columns as its starting bound on the candidate's
// k-th neighbour distance (any k distinct columns bound it; near ones bound it
// tightly), in place of a first pass over the columns (k_seed_bounds).
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

// Insert (v, col) into the lane's ascending N-entry list if v is below its
// last entry (strict: +inf and NaN never enter).  Fully unrolled, so the list
// stays in registers.
template <int N>
__device__ __forceinline__ void keep_n(float (&s)[N], int (&i)[N], float v, int col)
{
    if (!(v < s[N - 1])) return;
    bool placed = false;
#pragma unroll
    for (int j = N - 1; j > 0; --j) {
        if (!placed) {
            if (v < s[j - 1]) {
                s[j] = s[j - 1];
                i[j] = i[j - 1];
            } else {
                s[j] = v;
                i[j] = col;
                placed = true;
            }
        }
    }
    if (!placed) {
        s[0] = v;
        i[0] = col;
    }
}

// Three blocks of 256 threads per SM, each lane with four float4 loads of D in
// flight: the stream needs that many bytes in flight to stay HBM-bound (four
// blocks with two loads per lane while the seed lists take registers: 44.0
// against 43.0 ms of commits per fwd-64k selection).
template <bool BWD, bool SEEDS>
__global__ void __launch_bounds__(256, 3) k_commit(Bufs b, int *seeds, float *seed_d)
{
    if (b.st->done) return;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int w = b.st->winner;
    const float *xt = b.XT + (size_t)w * b.ldc;
    const float *xv = b.XV + (size_t)w * b.ldr;
    const float4 *xt4 = reinterpret_cast<const float4 *>(xt);
    const int n4 = b.ldc >> 2;
    for (int r = blockIdx.x * wpb + (threadIdx.x >> 5); r < b.n_rows; r += gridDim.x * wpb) {
        const float a = __ldg(xv + r);
        float4 *row = reinterpret_cast<float4 *>(b.D + (size_t)r * b.ldc);
        float sv[kSeedsPerLane];
        int si[kSeedsPerLane];
#pragma unroll
        for (int j = 0; j < kSeedsPerLane; ++j) {
            sv[j] = INFINITY;
            si[j] = -1;
        }
        constexpr int U = 4;  // float4 loads per lane in flight
        for (int q0 = 0; q0 < n4; q0 += 32 * U) {
            float4 d[U], c[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int q = q0 + u * 32 + lane;
                if (q < n4) {
                    d[u] = __ldcs(row + q);
                    c[u] = __ldg(xt4 + q);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int q = q0 + u * 32 + lane;
                if (q < n4) {
                    if (BWD) {
                        d[u].x = __fsub_rn(d[u].x, sqdiff(a, c[u].x));
                        d[u].y = __fsub_rn(d[u].y, sqdiff(a, c[u].y));
                        d[u].z = __fsub_rn(d[u].z, sqdiff(a, c[u].z));
                        d[u].w = __fsub_rn(d[u].w, sqdiff(a, c[u].w));
                    } else {
                        d[u].x = __fadd_rn(d[u].x, sqdiff(a, c[u].x));
                        d[u].y = __fadd_rn(d[u].y, sqdiff(a, c[u].y));
                        d[u].z = __fadd_rn(d[u].z, sqdiff(a, c[u].z));
                        d[u].w = __fadd_rn(d[u].w, sqdiff(a, c[u].w));
                    }
                    __stcs(row + q, d[u]);
                    if (SEEDS) {
                        // entries are rare once the list holds near columns: one
                        // test per float4 keeps the insertion code off the common path
                        const float lim = sv[kSeedsPerLane - 1];
                        if (fminf(fminf(d[u].x, d[u].y), fminf(d[u].z, d[u].w)) < lim) {
                            keep_n(sv, si, d[u].x, 4 * q);
                            keep_n(sv, si, d[u].y, 4 * q + 1);
                            keep_n(sv, si, d[u].z, 4 * q + 2);
                            keep_n(sv, si, d[u].w, 4 * q + 3);
                        }
                    }
                }
            }
        }
        if (SEEDS) {
#pragma unroll
            for (int j = 0; j < kSeedsPerLane; ++j) {
                seeds[(size_t)r * kSeeds + j * 32 + lane] = si[j];
                seed_d[(size_t)r * kSeeds + j * 32 + lane] = sv[j];
            }
        }
    }
}

int sm_count_commit()
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

cudaError_t launch_commit(const Bufs &b, int backward, int *seeds, float *seed_d, cudaStream_t s)
{
    int grid = (b.n_rows + 7) / 8;
    const int cap = sm_count_commit() * 6;
    if (grid > cap) grid = cap;
    if (backward) k_commit<true, false><<<grid, 256, 0, s>>>(b, nullptr, nullptr);
    else if (seeds && seed_d) k_commit<false, true><<<grid, 256, 0, s>>>(b, seeds, seed_d);
    else k_commit<false, false><<<grid, 256, 0, s>>>(b, nullptr, nullptr);
    return cudaGetLastError();
}

}  // namespace snn
