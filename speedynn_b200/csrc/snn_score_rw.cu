// snn_score_rw.cu -- candidate scoring with one scored row per warp.
//
// Same contract as snn_score.cu (exact top-k_max lists in the reference's
// stable (distance, index) order, kNN-mean predictions), different mapping:
//
//   * a warp owns ONE scored row r and CB candidates; its lanes walk the
//     training columns, two adjacent columns per lane (packed f32x2), so a
//     64-column chunk is one step of the warp;
//   * each (r, c) list lives in registers spread over the lanes (lane j
//     holds element j, j+32, ...), its k-th distance is warp-uniform, and an
//     insertion is a ballot/popc for the position plus one shuffle-up -- about
//     ten instructions, with no shared-memory traffic;
//   * a block is NW warps = NW consecutive rows sharing the same CB
//     candidates: the candidates' 256-column slices of X are staged once per
//     block in shared memory (cp.async ring) together with the NW rows of D.
//
// The pass test is strict d < k-th distance because each problem's columns
// are visited in ascending order (chunk by chunk, lanes ascending, and the
// two columns of a lane in order), exactly the reference's insertion order.
#include <float.h>
#include <math.h>

#include "snn_internal.h"

namespace snn {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kChunk = 64;              // columns per warp step (2 per lane)
constexpr int kStageCols = 256;         // columns per pipeline stage
constexpr int kStagesRW = 3;

__device__ __forceinline__ unsigned long long as_u64(float2 v) { return *reinterpret_cast<unsigned long long *>(&v); }
__device__ __forceinline__ float2 as_f2(unsigned long long v) { return *reinterpret_cast<float2 *>(&v); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)));
    return as_f2(d);
}
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    unsigned long long d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)));
    return as_f2(d);
}
// fl(t*t) via fma(t, t, +0): a packed mul.rn feeding an add.rn is contracted
// into one FMA by ptxas; the fma form keeps the reference's two roundings.
__device__ __forceinline__ float2 sq2(float2 t)
{
    unsigned long long d;
    const unsigned long long z = 0ull;
    asm("fma.rn.f32x2 %0, %1, %1, %2;" : "=l"(d) : "l"(as_u64(t)), "l"(z));
    return as_f2(d);
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Insert (v, col) into the register list (ld, li) of GK elements per lane;
// returns the new k-th distance (warp-uniform).
template <int GK>
__device__ __forceinline__ float reg_list_insert(float (&ld)[GK], int (&li)[GK], int K, float v, int col, int lane)
{
    int pos = 0;
#pragma unroll
    for (int g = 0; g < GK; ++g) pos += __popc(__ballot_sync(kFull, ld[g] <= v));
    float carry = 0.0f;
    int carryi = 0;
#pragma unroll
    for (int g = 0; g < GK; ++g) {
        const int x = g * 32 + lane;
        float up = __shfl_up_sync(kFull, ld[g], 1);
        int upi = __shfl_up_sync(kFull, li[g], 1);
        if (lane == 0) {
            up = carry;
            upi = carryi;
        }
        if (GK > 1) {
            carry = __shfl_sync(kFull, ld[g], 31);
            carryi = __shfl_sync(kFull, li[g], 31);
        }
        if (x < K) {
            if (x == pos) {
                ld[g] = v;
                li[g] = col;
            } else if (x > pos) {
                ld[g] = up;
                li[g] = upi;
            }
        }
    }
    const int gl = (K - 1) >> 5;
    float last = ld[0];
#pragma unroll
    for (int g = 1; g < GK; ++g)
        if (g == gl) last = ld[g];
    return __shfl_sync(kFull, last, (K - 1) & 31);
}

template <int CB, int GK, bool BWD>
__global__ void __launch_bounds__(512) k_score_rw(Bufs b, int n_cand, int n_cg)
{
    extern __shared__ __align__(16) float sm[];
    const int NW = blockDim.x >> 5;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float *Ds = sm;                                   // [stages][NW][kStageCols]
    float *Xs = Ds + kStagesRW * NW * kStageCols;     // [stages][CB][kStageCols]
    int *srcand = reinterpret_cast<int *>(Xs + kStagesRW * CB * kStageCols);  // [CB]

    if (b.st->done) return;
    const int K = b.kmax;
    const int cg = blockIdx.x % n_cg;
    const int r0 = (blockIdx.x / n_cg) * NW;
    const int r = r0 + w;
    const bool rvalid = r < b.n_rows;
    const int c0 = cg * CB;

    if (threadIdx.x < CB) {
        const int s = c0 + threadIdx.x;
        srcand[threadIdx.x] = b.cands[s < n_cand ? s : 0];
    }
    __syncthreads();

    float2 xv2[CB];
    float thr[CB];
    float ld[CB][GK];
    int li[CB][GK];
#pragma unroll
    for (int c = 0; c < CB; ++c) {
        const bool cv = c0 + c < n_cand && rvalid;
        const float x = cv ? __ldg(b.XV + (size_t)srcand[c] * b.ldr + r) : NAN;  // NaN never passes
        xv2[c] = make_float2(x, x);
        thr[c] = FLT_MAX;
#pragma unroll
        for (int g = 0; g < GK; ++g) {
            ld[c][g] = (g * 32 + lane < K) ? FLT_MAX : INFINITY;  // elements >= K never count
            li[c][g] = 0;
        }
    }

    const int nstages = b.ldc / kStageCols + (b.ldc % kStageCols ? 1 : 0);
    const int rlast = b.n_rows - 1;
    auto issue = [&](int st, int slot) {
        const int i0 = st * kStageCols;
        float *D_s = Ds + slot * NW * kStageCols;
        float *X_s = Xs + slot * CB * kStageCols;
        const int per_row = kStageCols / 4;  // 16-byte pieces per row
        for (int q = threadIdx.x; q < (NW + CB) * per_row; q += blockDim.x) {
            const int row = q / per_row, p4 = (q % per_row) * 4;
            const int col = min(i0 + p4, b.ldc - 4);  // the last stage may overrun ldc: clamp (never used)
            if (row < NW) {
                const int rr = min(r0 + row, rlast);
                cp_async16(D_s + row * kStageCols + p4, b.D + (size_t)rr * b.ldc + col);
            } else {
                const int c = row - NW;
                cp_async16(X_s + c * kStageCols + p4, b.XT + (size_t)srcand[c] * b.ldc + col);
            }
        }
    };

    issue(0, 0);
    cp_async_commit();
    if (nstages > 1) issue(1, 1);
    cp_async_commit();

    for (int st = 0; st < nstages; ++st) {
        const int slot = st % kStagesRW;
        cp_async_wait<1>();
        __syncthreads();
        if (st + 2 < nstages) issue(st + 2, (st + 2) % kStagesRW);
        cp_async_commit();
        if (!rvalid) continue;
        const float *D_s = Ds + slot * NW * kStageCols + w * kStageCols;
        const float *X_s = Xs + slot * CB * kStageCols;
        const int i0 = st * kStageCols;
        const int cols = min(kStageCols, b.ldc - i0);
        for (int q0 = 0; q0 < cols; q0 += kChunk) {
            const float2 dv = *reinterpret_cast<const float2 *>(D_s + q0 + 2 * lane);
            bool any = false;
#pragma unroll
            for (int c = 0; c < CB; ++c) {
                const float2 xt = *reinterpret_cast<const float2 *>(X_s + c * kStageCols + q0 + 2 * lane);
                const float2 s = sq2(sub2(xv2[c], xt));
                const float2 e = BWD ? sub2(dv, s) : add2(dv, s);
                any |= (e.x < thr[c]) | (e.y < thr[c]);
            }
            if (__any_sync(kFull, any)) {
                // rare path: recompute the chunk's distances candidate by candidate
                const int colbase = i0 + q0;
#pragma unroll
                for (int c = 0; c < CB; ++c) {
                    const float2 xt = *reinterpret_cast<const float2 *>(X_s + c * kStageCols + q0 + 2 * lane);
                    const float2 s = sq2(sub2(xv2[c], xt));
                    float2 ec = BWD ? sub2(dv, s) : add2(dv, s);
                    const float2 e[1] = {ec};
                    unsigned m = __ballot_sync(kFull, (e[0].x < thr[c]) | (e[0].y < thr[c]));
                    while (m) {
                        const int L = __ffs(m) - 1;
                        m &= m - 1;
                        const float ex = __shfl_sync(kFull, e[0].x, L);
                        const float ey = __shfl_sync(kFull, e[0].y, L);
                        if (ex < thr[c]) thr[c] = reg_list_insert<GK>(ld[c], li[c], K, ex, colbase + 2 * L, lane);
                        if (ey < thr[c]) thr[c] = reg_list_insert<GK>(ld[c], li[c], K, ey, colbase + 2 * L + 1, lane);
                    }
                }
            }
        }
    }
    cp_async_wait<0>();
    if (!rvalid) return;

#pragma unroll
    for (int c = 0; c < CB; ++c) {
        const int slot = c0 + c;
        if (slot >= n_cand) continue;
        if (b.nn_idx) {
            const size_t o = ((size_t)slot * b.n_rows + r) * K;
#pragma unroll
            for (int g = 0; g < GK; ++g) {
                const int x = g * 32 + lane;
                if (x < K) {
                    b.nn_idx[o + x] = li[c][g];
                    b.nn_dist[o + x] = ld[c][g];
                }
            }
        }
        // label sum in rank order (sequential FP32, as the reference), all lanes in step
        float acc = 0.0f;
        int m = 0;
        const int nk = b.nk;
        for (int j = 0; j < K; ++j) {
            int idx = li[c][0];
#pragma unroll
            for (int g = 1; g < GK; ++g)
                if (g == (j >> 5)) idx = li[c][g];
            idx = __shfl_sync(kFull, idx, j & 31);
            acc = __fadd_rn(acc, __ldg(b.yc + idx));
            // k_vals may repeat or be unsorted: test every entry
            for (m = 0; m < nk; ++m) {
                const int k = __ldg(b.kvals + m);
                if (k == j + 1 && lane == 0) b.pred[((size_t)slot * nk + m) * b.n_rows + r] = __fdiv_rn(acc, (float)k);
            }
        }
    }
}

template <int CB, int GK>
size_t rw_smem(int NW)
{
    return sizeof(float) * (size_t)kStagesRW * (NW + CB) * kStageCols + sizeof(int) * CB;
}

template <int CB, int GK, bool BWD>
cudaError_t launch_rw3(const Bufs &b, int n_cand, cudaStream_t s)
{
    const int NW = 16;
    const int n_cg = (n_cand + CB - 1) / CB;
    const long long blocks = (long long)((b.n_rows + NW - 1) / NW) * n_cg;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    const size_t smem = rw_smem<CB, GK>(NW);
    cudaError_t e = cudaFuncSetAttribute(k_score_rw<CB, GK, BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_score_rw<CB, GK, BWD><<<(unsigned)blocks, NW * 32, smem, s>>>(b, n_cand, n_cg);
    return cudaGetLastError();
}

template <int CB, int GK>
cudaError_t launch_rw2(const Bufs &b, int n_cand, int backward, cudaStream_t s)
{
    return backward ? launch_rw3<CB, GK, true>(b, n_cand, s) : launch_rw3<CB, GK, false>(b, n_cand, s);
}

}  // namespace

bool score_rw_supported(int kmax) { return kmax >= 1 && kmax <= 64; }

cudaError_t launch_score_rw(const Bufs &b, int n_cand, int backward, cudaStream_t s)
{
    if (b.kmax <= 32) return launch_rw2<16, 1>(b, n_cand, backward, s);
    if (b.kmax <= 64) return launch_rw2<8, 2>(b, n_cand, backward, s);
    return cudaErrorInvalidValue;
}

}  // namespace snn
