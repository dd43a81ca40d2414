// snn_score.cu -- the candidate-scoring kernel (one launch per greedy step).
//
// For every scored row r and candidate feature c it computes the exact
// top-k_max neighbour list of
//     d_i = fl(D[r,i] +/- fl(fl(x_r,c - x_i,c)^2))       (speedynn/lib/cpu.c:142-144)
// over all training columns i, in the reference's stable (distance, index)
// order with (FLT_MAX, 0) padding (cpu.c:128-168), then the kNN-mean
// prediction for every k of k_vals (cpu.c:56-66).
//
// Mapping (B200, 148 SMs, 227 KB shared memory per block):
//   * a block owns 32 scored rows (lane = row) and W*CC candidates
//     (warp w owns CC of them); the 32-row x 32-column tile of D and the
//     candidates' 32-column slices of X stream through a 3-stage cp.async
//     ring, so each D element leaves L2 once per block and every warp reuses it;
//   * arithmetic pairs two adjacent columns of one candidate in packed FP32
//     (sub/fma/add.rn.f32x2), so a pair of evaluations costs three issue
//     slots plus two compares.  The square is formed as fma.rn.f32x2(t, t, +0)
//     rather than mul.rn.f32x2: ptxas contracts a single-use packed
//     mul.rn + add.rn pair into one FMA despite the rounding modifiers (about
//     17 % of results then differ by one ulp from the reference's two
//     roundings), while fl(t*t + 0) = fl(t*t) for t*t >= 0 and cannot be
//     folded into the following add;
//   * each (row, candidate) keeps its current k-th distance in a register;
//     four columns are tested against it and one warp vote decides whether
//     anything must be inserted;
//   * insertions are warp-cooperative: for each pending (row, candidate) the
//     32 lanes hold the k_max-element list (k_max <= 256, ceil(k_max/32) per
//     lane), find the stable position by ballot/popc, shift by shuffle and
//     write back -- no lane-divergent loops.
#include <float.h>
#include <math.h>

#include "snn_internal.h"

namespace snn {

namespace {

constexpr int kRows = 32;           // scored rows per block (one per lane)
constexpr int kCols = 32;           // columns per tile
constexpr int kDsLd = kCols + 4;    // padded row stride of the D tile (conflict-free 128-bit reads)
constexpr int kStages = 3;          // cp.async ring depth
constexpr unsigned kFull = 0xffffffffu;

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
// fl(t*t), exactly as a rounded multiply, but immune to contraction with the
// next add (see the file comment).
__device__ __forceinline__ float2 sq2(float2 t)
{
    unsigned long long d;
    const unsigned long long z = 0ull;  // (+0.0f, +0.0f)
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

// Insert (dv, col) into the sorted list at Ld/Li[base .. base+K) with all 32
// lanes (lane j holds elements j, j+32, ...); the item goes after every
// element <= dv (stable: the scan visits columns in ascending order).
// Returns the new K-th distance.  Kept out of line: it has many call sites
// on the rare path and must not bloat the hot loop's instruction footprint.
__device__ __noinline__ float coop_insert(float *Ld, int *Li, int base, int K, float dv, int col)
{
    const int lane = threadIdx.x & 31;
    int pos = 0;
    for (int g0 = 0; g0 < K; g0 += 32) {
        const int x = g0 + lane;
        const bool ok = x < K;
        const float e = ok ? Ld[base + x] : FLT_MAX;
        pos += __popc(__ballot_sync(kFull, ok && e <= dv));
    }
    float carry_e = 0.0f;
    int carry_i = 0;
    for (int g0 = 0; g0 < K; g0 += 32) {
        const int x = g0 + lane;
        const bool ok = x < K;
        const float e = ok ? Ld[base + x] : FLT_MAX;
        const int ix = ok ? Li[base + x] : 0;
        float up = __shfl_up_sync(kFull, e, 1);
        int upi = __shfl_up_sync(kFull, ix, 1);
        if (lane == 0) {
            up = carry_e;
            upi = carry_i;
        }
        carry_e = __shfl_sync(kFull, e, 31);
        carry_i = __shfl_sync(kFull, ix, 31);
        if (ok && x >= pos) {
            Ld[base + x] = (x == pos) ? dv : up;
            Li[base + x] = (x == pos) ? col : upi;
        }
    }
    __syncwarp();
    return Ld[base + K - 1];
}

struct Layout {
    int WCC;
    float *Ds, *Xs, *Ld;
    int *Li, *scand, *srcand;
};

__device__ __forceinline__ Layout carve(float *sm, int WCC, int K)
{
    Layout L;
    L.WCC = WCC;
    L.Ds = sm;
    L.Xs = L.Ds + kStages * kRows * kDsLd;
    L.Ld = L.Xs + kStages * WCC * kCols;
    L.Li = reinterpret_cast<int *>(L.Ld + (size_t)kRows * WCC * K);
    L.scand = L.Li + (size_t)kRows * WCC * K;
    L.srcand = L.scand + WCC;
    return L;
}

template <int CC, bool BWD>
__global__ void __launch_bounds__(512) k_score(Bufs b, int n_cand, int W, int n_chunks)
{
    extern __shared__ __align__(16) float sm[];
    const int K = b.kmax;
    const int WCC = W * CC;
    const Layout S = carve(sm, WCC, K);

    if (b.st->done) return;
    if (b.only_if_full && !b.st->full_scan) return;  // the sorted first step scored every problem

    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int nthr = blockDim.x;
    const int chunk = blockIdx.x % n_chunks;
    const int r0 = (blockIdx.x / n_chunks) * kRows;
    const int r = r0 + lane;
    const int s0 = chunk * WCC;

    for (int i = tid; i < WCC; i += nthr) {
        const int s = s0 + i;
        const int cid = s < n_cand ? b.cands[s] : -1;
        S.scand[i] = cid;
        S.srcand[i] = cid >= 0 ? cid : b.cands[0];
    }
    // each warp owns the lists of its CC candidates for all 32 rows
    for (int e = lane; e < kRows * CC * K; e += 32) {
        const int row = e / (CC * K), rem = e % (CC * K);
        const int o = (row * WCC + w * CC) * K + rem;
        S.Ld[o] = FLT_MAX;
        S.Li[o] = 0;
    }
    __syncthreads();

    float2 xv2[CC];
    float thr[CC];
#pragma unroll
    for (int c = 0; c < CC; ++c) {
        const int cid = S.scand[w * CC + c];
        const float x = (cid >= 0 && r < b.n_rows) ? b.XV[(size_t)cid * b.ldr + r] : NAN;  // NaN never passes
        xv2[c] = make_float2(x, x);
        thr[c] = FLT_MAX;
    }

    const int ntiles = b.ldc / kCols;
    const int rlast = b.n_rows - 1;
    auto issue = [&](int tile, int stage) {
        const int i0 = tile * kCols;
        float *Ds = S.Ds + stage * kRows * kDsLd;
        float *Xs = S.Xs + stage * WCC * kCols;
        for (int q = tid; q < kRows * 8; q += nthr) {
            const int row = q >> 3, c4 = q & 7;
            const int rr = min(r0 + row, rlast);
            cp_async16(Ds + row * kDsLd + c4 * 4, b.D + (size_t)rr * b.ldc + i0 + c4 * 4);
        }
        for (int q = tid; q < WCC * 8; q += nthr) {
            const int s = q >> 3, c4 = q & 7;
            cp_async16(Xs + s * kCols + c4 * 4, b.XT + (size_t)S.srcand[s] * b.ldc + i0 + c4 * 4);
        }
    };

    issue(0, 0);
    cp_async_commit();
    if (ntiles > 1) issue(1, 1);
    cp_async_commit();

    for (int tile = 0; tile < ntiles; ++tile) {
        const int stage = tile % kStages;
        cp_async_wait<1>();
        __syncthreads();
        if (tile + 2 < ntiles) issue(tile + 2, (tile + 2) % kStages);
        cp_async_commit();

        const float *Dr = S.Ds + stage * kRows * kDsLd + lane * kDsLd;
        const float *Xw = S.Xs + stage * WCC * kCols + (w * CC) * kCols;
        const int i0 = tile * kCols;
#pragma unroll 2
        for (int q0 = 0; q0 < kCols; q0 += 4) {
            const float4 dv = *reinterpret_cast<const float4 *>(Dr + q0);
            const float2 d01 = make_float2(dv.x, dv.y), d23 = make_float2(dv.z, dv.w);
            float2 e01[CC], e23[CC];
            bool pass = false;
#pragma unroll
            for (int c = 0; c < CC; ++c) {
                const float4 xt = *reinterpret_cast<const float4 *>(Xw + c * kCols + q0);
                const float2 t01 = sub2(xv2[c], make_float2(xt.x, xt.y));
                const float2 t23 = sub2(xv2[c], make_float2(xt.z, xt.w));
                const float2 s01 = sq2(t01), s23 = sq2(t23);
                e01[c] = BWD ? sub2(d01, s01) : add2(d01, s01);
                e23[c] = BWD ? sub2(d23, s23) : add2(d23, s23);
                pass |= (e01[c].x < thr[c]) | (e01[c].y < thr[c]) | (e23[c].x < thr[c]) | (e23[c].y < thr[c]);
            }
            if (__any_sync(kFull, pass)) {
#pragma unroll
                for (int qq = 0; qq < 4; ++qq) {
#pragma unroll
                    for (int c = 0; c < CC; ++c) {
                        const float dq = qq == 0 ? e01[c].x : qq == 1 ? e01[c].y : qq == 2 ? e23[c].x : e23[c].y;
                        unsigned m = __ballot_sync(kFull, dq < thr[c]);
                        while (m) {
                            const int L = __ffs(m) - 1;
                            m &= m - 1;
                            const float dl = __shfl_sync(kFull, dq, L);
                            const int base = (L * WCC + w * CC + c) * K;
                            const float nt = coop_insert(S.Ld, S.Li, base, K, dl, i0 + q0 + qq);
                            if (lane == L) thr[c] = nt;
                        }
                    }
                }
            }
        }
    }
    cp_async_wait<0>();

    if (r >= b.n_rows) return;
#pragma unroll
    for (int c = 0; c < CC; ++c) {
        const int slot = s0 + w * CC + c;
        if (slot >= n_cand) continue;
        const int base = (lane * WCC + w * CC + c) * K;
        if (b.nn_idx) {
            const size_t o = ((size_t)slot * b.n_rows + r) * K;
            for (int j = 0; j < K; ++j) {
                b.nn_idx[o + j] = S.Li[base + j];
                b.nn_dist[o + j] = S.Ld[base + j];
            }
        }
        float acc = 0.0f;
        for (int j = 0; j < K; ++j) {
            acc = __fadd_rn(acc, __ldg(b.yc + S.Li[base + j]));
            S.Ld[base + j] = acc;  // label prefix sums replace the distances
        }
        for (int m = 0; m < b.nk; ++m) {
            const int k = __ldg(b.kvals + m);
            b.pred[((size_t)slot * b.nk + m) * b.n_rows + r] = __fdiv_rn(S.Ld[base + k - 1], (float)k);
        }
    }
}

size_t plan_smem(int CC, int W, int K)
{
    const size_t WCC = (size_t)W * CC;
    return sizeof(float) * (kStages * kRows * kDsLd + kStages * WCC * kCols) + (sizeof(float) + sizeof(int)) * kRows * WCC * K +
           sizeof(int) * 2 * WCC;
}

template <int CC, bool BWD>
cudaError_t launch_cc(const Bufs &b, int n_cand, const ScorePlan &pl, cudaStream_t s)
{
    const int WCC = pl.warps * CC;
    const int n_chunks = (n_cand + WCC - 1) / WCC;
    const long long blocks = (long long)((b.n_rows + kRows - 1) / kRows) * n_chunks;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    const size_t smem = plan_smem(CC, pl.warps, b.kmax);
    cudaError_t e = cudaFuncSetAttribute(k_score<CC, BWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k_score<CC, BWD><<<(unsigned)blocks, 32 * pl.warps, smem, s>>>(b, n_cand, pl.warps, n_chunks);
    return cudaGetLastError();
}

}  // namespace

ScorePlan plan_score(int kmax, int p, int max_smem)
{
    ScorePlan pl{0, 0, 0};
    if (kmax < 1 || kmax > kScoreMaxK) return pl;
    // prefer 4 candidates per thread (more reuse of each D value); fall back to 2
    const int ccs[2] = {kmax <= 32 ? 4 : 2, 2};
    for (int t = 0; t < 2; ++t) {
        const int CC = ccs[t];
        int W = (p + CC - 1) / CC;
        if (W > 16) W = 16;
        while (W > 0 && plan_smem(CC, W, kmax) > (size_t)max_smem) --W;
        if (W > 0) {
            pl.cc = CC;
            pl.warps = W;
            pl.smem = (int)plan_smem(CC, W, kmax);
            return pl;
        }
    }
    return pl;
}

cudaError_t launch_score(const Bufs &b, int n_cand, const ScorePlan &pl, int backward, cudaStream_t s)
{
    if (pl.cc == 4) return backward ? launch_cc<4, true>(b, n_cand, pl, s) : launch_cc<4, false>(b, n_cand, pl, s);
    if (pl.cc == 2) return backward ? launch_cc<2, true>(b, n_cand, pl, s) : launch_cc<2, false>(b, n_cand, pl, s);
    return cudaErrorInvalidValue;
}

}  // namespace snn
