// snn_sparse.cu -- exact pruned scoring for forward steps after the first.
//
// Forward selection only ever adds a non-negative term: for every candidate c
//     d(r,i,c) = fl(D[r,i] + fl((x_r,c - x_i,c)^2)) >= D[r,i]      (fl is monotone)
// so once candidate c has an upper bound T_c on its k-th neighbour distance,
// a training column i with D[r,i] > max_c T_c cannot enter any candidate's
// list.  The bound comes from M "seed" columns per row -- the columns nearest
// to r under the committed D, found by the commit kernel while it streams D --
// as the k-th smallest exact distance over those M columns (any M real
// columns give a valid bound; near ones give a tight one).  Results stay
// bit-identical to the full scan:
//   * an item enters while the list still holds padding only if d <= T_c,
//     afterwards only if d < current k-th (strict: columns are visited in
//     ascending order) -- one inclusive register threshold covers both
//     (d < x  <=>  d <= nextafter(x, -inf));
//   * every member of the true top-k has d <= true k-th <= T_c, so it passes.
//
// k_commit_seeds: D <- fl(D +/- s_w) in place (speedynn/lib/cpu.c:217-231),
//   plus, per row, the M smallest new distances (warp per row, list spread
//   over lanes in registers, cooperative insertion).  HBM-bound.
// k_score_sparse: warp per row; D streamed once (float4, coalesced); columns
//   with D <= max_c T_c are queued in ascending order and scored with lanes
//   over candidates (x of a survivor read from a row-major copy, one
//   coalesced segment per survivor); per-lane neighbour lists in shared memory.
#include <float.h>
#include <math.h>

#include "snn_internal.h"

namespace snn {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kSeedG = kMaxSeeds / 32;  // seed-list elements per lane (max)
constexpr int kQueue = 160;             // survivor queue per warp (flushed at >= 32)
constexpr int kPrefetch = 8;            // survivors whose x values are fetched together

__device__ __forceinline__ float sqdiff(float a, float b)
{
    const float t = __fsub_rn(a, b);
    return __fmul_rn(t, t);
}

__device__ __forceinline__ float below(float x) { return nextafterf(x, -INFINITY); }

// Cooperative insertion into a register-resident sorted list: lane j of
// group g holds element g*32+j; G groups (G*32 = M elements).
template <int GM>
__device__ __forceinline__ void reg_insert(float (&ev)[GM], int (&iv)[GM], int G, float v, int col, int lane)
{
    int pos = 0;
#pragma unroll
    for (int g = 0; g < GM; ++g)
        if (g < G) pos += __popc(__ballot_sync(kFull, ev[g] <= v));
    float carry_e = 0.0f;
    int carry_i = 0;
#pragma unroll
    for (int g = 0; g < GM; ++g) {
        if (g < G) {
            const int x = g * 32 + lane;
            float up = __shfl_up_sync(kFull, ev[g], 1);
            int upi = __shfl_up_sync(kFull, iv[g], 1);
            if (lane == 0) {
                up = carry_e;
                upi = carry_i;
            }
            carry_e = __shfl_sync(kFull, ev[g], 31);
            carry_i = __shfl_sync(kFull, iv[g], 31);
            if (x == pos) {
                ev[g] = v;
                iv[g] = col;
            } else if (x > pos) {
                ev[g] = up;
                iv[g] = upi;
            }
        }
    }
}

template <bool BWD, bool SEEDS>
__global__ void __launch_bounds__(256) k_commit_seeds(Bufs b, int *seeds, int M)
{
    if (b.st->done) return;
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int G = M >> 5;
    const int w = b.st->winner;
    const float *xt = b.XT + (size_t)w * b.ldc;
    const float *xv = b.XV + (size_t)w * b.ldr;
    for (int r = blockIdx.x * wpb + (threadIdx.x >> 5); r < b.n_rows; r += gridDim.x * wpb) {
        const float a = __ldg(xv + r);
        float4 *row = reinterpret_cast<float4 *>(b.D + (size_t)r * b.ldc);
        const float4 *xt4 = reinterpret_cast<const float4 *>(xt);
        float ev[kSeedG];
        int iv[kSeedG];
#pragma unroll
        for (int g = 0; g < kSeedG; ++g) {
            ev[g] = INFINITY;
            iv[g] = -1;  // padding: never a seed (a repeated column would understate the bound)
        }
        float thr = INFINITY;
        const int n4 = b.ldc >> 2;
        for (int q0 = 0; q0 < n4; q0 += 128) {  // 4 float4 per lane in flight
            float4 d[4], c[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int q = q0 + u * 32 + lane;
                if (q < n4) {
                    d[u] = __ldcs(row + q);
                    c[u] = __ldg(xt4 + q);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
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
                }
            }
            if (SEEDS) {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int q = q0 + u * 32 + lane;
                    const float vv[4] = {d[u].x, d[u].y, d[u].z, d[u].w};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float v = q < n4 ? vv[e] : INFINITY;
                        unsigned m = __ballot_sync(kFull, v < thr);
                        while (m) {
                            const int L = __ffs(m) - 1;
                            m &= m - 1;
                            const float vl = __shfl_sync(kFull, v, L);
                            if (!(vl < thr)) continue;
                            reg_insert<kSeedG>(ev, iv, G, vl, (q0 + u * 32 + L) * 4 + e, lane);
                            float last = ev[0];
#pragma unroll
                            for (int g = 1; g < kSeedG; ++g)
                                if (g == G - 1) last = ev[g];
                            thr = __shfl_sync(kFull, last, 31);
                        }
                    }
                }
            }
        }
        if (SEEDS) {
#pragma unroll
            for (int g = 0; g < kSeedG; ++g)
                if (g < G) seeds[(size_t)r * M + g * 32 + lane] = iv[g];
        }
    }
}

// Thread-local sorted insertion (value + index) into a list in shared memory
// with element stride 1; returns the new last value.
__device__ __forceinline__ float lane_insert(float *Ld, int *Li, int K, float d, int i)
{
    int pos = K - 1;
    while (pos > 0) {
        const float prev = Ld[pos - 1];
        if (!(prev > d)) break;
        Ld[pos] = prev;
        Li[pos] = Li[pos - 1];
        --pos;
    }
    Ld[pos] = d;
    Li[pos] = i;
    return Ld[K - 1];
}

template <int CG>
__global__ void __launch_bounds__(256) k_score_sparse(Bufs b, SparseBufs sp, int n_cand, int M)
{
    extern __shared__ __align__(16) float smem[];
    const int K = b.kmax;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, wpb = blockDim.x >> 5;
    // per warp: lists [n_cand][K] distances + indices, queue columns + D values
    const int per_warp = 2 * n_cand * K + 2 * kQueue;
    float *Ld = smem + (size_t)wib * per_warp;
    int *Li = reinterpret_cast<int *>(Ld + n_cand * K);
    int *qcol = Li + n_cand * K;
    float *qd = reinterpret_cast<float *>(qcol + kQueue);
    if (b.st->done) return;

    unsigned long long surv_total = 0;
    for (int r = blockIdx.x * wpb + wib; r < b.n_rows; r += gridDim.x * wpb) {
        int cid[CG];
        float xv[CG], thr[CG];
#pragma unroll
        for (int g = 0; g < CG; ++g) {
            const int c = g * 32 + lane;
            cid[g] = c < n_cand ? b.cands[c] : -1;
            xv[g] = cid[g] >= 0 ? __ldg(b.XV + (size_t)cid[g] * b.ldr + r) : NAN;
            if (cid[g] >= 0)
                for (int j = 0; j < K; ++j) {
                    Ld[c * K + j] = FLT_MAX;
                    Li[c * K + j] = 0;
                }
        }
        const float *Drow = b.D + (size_t)r * b.ldc;
        // -- per-candidate bound from the seed columns
        for (int s0 = 0; s0 < M; s0 += 32) {
            const int sc = sp.seeds[(size_t)r * M + s0 + lane];
            const float sd = sc >= 0 ? __ldg(Drow + sc) : INFINITY;
            for (int j = 0; j < 32; ++j) {
                const int col = __shfl_sync(kFull, sc, j);
                const float dcol = __shfl_sync(kFull, sd, j);
                if (col < 0) continue;
#pragma unroll
                for (int g = 0; g < CG; ++g) {
                    if (cid[g] < 0) continue;
                    const float d = __fadd_rn(dcol, sqdiff(xv[g], __ldg(sp.Xrow + (size_t)col * sp.ldp + cid[g])));
                    const int c = g * 32 + lane;
                    if (d < Ld[c * K + K - 1]) lane_insert(Ld + c * K, Li + c * K, K, d, col);
                }
            }
        }
        float Tr = -INFINITY;
#pragma unroll
        for (int g = 0; g < CG; ++g) {
            const int c = g * 32 + lane;
            thr[g] = -INFINITY;
            if (cid[g] >= 0) {
                const float T = Ld[c * K + K - 1];
                thr[g] = T < FLT_MAX ? T : below(FLT_MAX);  // inclusive bound; FLT_MAX itself never enters
                Tr = fmaxf(Tr, thr[g]);
                for (int j = 0; j < K; ++j) {
                    Ld[c * K + j] = FLT_MAX;
                    Li[c * K + j] = 0;
                }
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) Tr = fmaxf(Tr, __shfl_xor_sync(kFull, Tr, off));

        // -- scan the row; queue survivors in ascending column order
        auto flush = [&](int qn) {
            for (int q0 = 0; q0 < qn; q0 += kPrefetch) {
                float xs[kPrefetch][CG];
#pragma unroll
                for (int u = 0; u < kPrefetch; ++u) {
                    const int col = q0 + u < qn ? qcol[q0 + u] : qcol[q0];
#pragma unroll
                    for (int g = 0; g < CG; ++g)
                        xs[u][g] = cid[g] >= 0 ? __ldg(sp.Xrow + (size_t)col * sp.ldp + cid[g]) : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < kPrefetch; ++u) {
                    if (q0 + u >= qn) break;
                    const int col = qcol[q0 + u];
                    const float dcol = qd[q0 + u];
#pragma unroll
                    for (int g = 0; g < CG; ++g) {
                        const float d = __fadd_rn(dcol, sqdiff(xv[g], xs[u][g]));
                        if (d <= thr[g]) {
                            const int c = g * 32 + lane;
                            const float last = lane_insert(Ld + c * K, Li + c * K, K, d, col);
                            if (last < FLT_MAX) thr[g] = below(last);
                        }
                    }
                }
            }
            __syncwarp();
        };

        int qn = 0;
        const int n4 = b.ldc >> 2;
        const float4 *row4 = reinterpret_cast<const float4 *>(Drow);
        const unsigned lt = (1u << lane) - 1u;
        for (int q0 = 0; q0 < n4; q0 += 64) {
            float4 dv[2];
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const int q = q0 + u * 32 + lane;
                dv[u] = q < n4 ? __ldcs(row4 + q) : make_float4(INFINITY, INFINITY, INFINITY, INFINITY);
            }
#pragma unroll
            for (int u = 0; u < 2; ++u) {
                const float v[4] = {dv[u].x, dv[u].y, dv[u].z, dv[u].w};
                unsigned bal[4];
                int tot = 0;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    bal[e] = __ballot_sync(kFull, v[e] <= Tr);
                    tot += __popc(bal[e]);
                }
                if (tot) {
                    // position of (lane, e) = survivors in lower lanes (all e) + own lower e
                    int before = 0;
#pragma unroll
                    for (int e = 0; e < 4; ++e) before += __popc(bal[e] & lt);
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        if (v[e] <= Tr) {
                            qcol[qn + before] = (q0 + u * 32 + lane) * 4 + e;
                            qd[qn + before] = v[e];
                            ++before;
                        }
                    }
                    qn += tot;
                    surv_total += tot;
                    __syncwarp();
                    if (qn >= kQueue - 128) {
                        flush(qn);
                        qn = 0;
                    }
                }
            }
        }
        if (qn) flush(qn);

        // -- epilogue: predictions (and optional lists)
#pragma unroll
        for (int g = 0; g < CG; ++g) {
            if (cid[g] < 0) continue;
            const int c = g * 32 + lane;
            float *L = Ld + c * K;
            const int *I = Li + c * K;
            if (b.nn_idx) {
                const size_t o = ((size_t)c * b.n_rows + r) * K;
                for (int j = 0; j < K; ++j) {
                    b.nn_idx[o + j] = I[j];
                    b.nn_dist[o + j] = L[j];
                }
            }
            float acc = 0.0f;
            for (int j = 0; j < K; ++j) {
                acc = __fadd_rn(acc, __ldg(b.yc + I[j]));
                L[j] = acc;
            }
            for (int m = 0; m < b.nk; ++m) {
                const int k = __ldg(b.kvals + m);
                b.pred[((size_t)c * b.nk + m) * b.n_rows + r] = __fdiv_rn(L[k - 1], (float)k);
            }
        }
        __syncwarp();
    }
    if (lane == 0 && sp.survivors) atomicAdd(sp.survivors, surv_total);
}

int sm_count_sp()
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

template <int CG>
cudaError_t launch_sparse_cg(const Bufs &b, const SparseBufs &sp, int n_cand, int M, int warps, cudaStream_t s)
{
    const size_t smem = sparse_smem_per_warp(n_cand, b.kmax) * warps;
    cudaError_t e = cudaFuncSetAttribute(k_score_sparse<CG>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_score_sparse<CG>, warps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    long long grid = (long long)sm_count_sp() * per_sm;
    const long long need = (b.n_rows + warps - 1) / warps;
    if (grid > need) grid = need;
    k_score_sparse<CG><<<(unsigned)grid, warps * 32, smem, s>>>(b, sp, n_cand, M);
    return cudaGetLastError();
}

}  // namespace

size_t sparse_smem_per_warp(int n_cand, int kmax)
{
    return sizeof(float) * (2 * (size_t)n_cand * kmax + 2 * kQueue);
}

int seeds_for_k(int kmax)
{
    int m = ((2 * kmax + 31) / 32) * 32;
    if (m < 32) m = 32;
    return m <= kMaxSeeds ? m : 0;
}

cudaError_t launch_commit_seeds(const Bufs &b, int backward, int *seeds, int M, cudaStream_t s)
{
    int grid = (b.n_rows + 7) / 8;
    const int cap = sm_count_sp() * 8;
    if (grid > cap) grid = cap;
    if (seeds) {
        if (backward) k_commit_seeds<true, true><<<grid, 256, 0, s>>>(b, seeds, M);
        else k_commit_seeds<false, true><<<grid, 256, 0, s>>>(b, seeds, M);
    } else {
        if (backward) k_commit_seeds<true, false><<<grid, 256, 0, s>>>(b, seeds, M);
        else k_commit_seeds<false, false><<<grid, 256, 0, s>>>(b, seeds, M);
    }
    return cudaGetLastError();
}

cudaError_t launch_score_sparse(const Bufs &b, const SparseBufs &sp, int n_cand, int M, int max_smem, cudaStream_t s)
{
    const size_t pw = sparse_smem_per_warp(n_cand, b.kmax);
    int warps = 8;
    while (warps > 1 && pw * warps > (size_t)max_smem) --warps;
    if (pw * warps > (size_t)max_smem) return cudaErrorInvalidConfiguration;
    const int cg = (n_cand + 31) / 32;
    switch (cg) {
    case 1: return launch_sparse_cg<1>(b, sp, n_cand, M, warps, s);
    case 2: return launch_sparse_cg<2>(b, sp, n_cand, M, warps, s);
    case 3: return launch_sparse_cg<3>(b, sp, n_cand, M, warps, s);
    case 4: return launch_sparse_cg<4>(b, sp, n_cand, M, warps, s);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace snn
