// snn_score_tma.cu -- candidate scoring, warp-specialised TMA pipeline.
//
// Same contract and warp tiling as snn_score_rw.cu (exact top-k_max lists in
// the reference's stable (distance, index) order, kNN-mean predictions; a
// consumer warp owns 4 scored rows x 4 candidates and walks the columns two
// per lane with packed f32x2), different feeding:
//
//   * one producer warp streams each 128-column stage with bulk TMA copies
//     (cp.async.bulk ... mbarrier::complete_tx): 16 rows of D and the 16
//     candidates' slices of X, 512 bytes each, into an 8-stage ring;
//   * each stage has a "full" mbarrier (producer arrive + expected bytes) and
//     an "empty" mbarrier (one arrive per consumer warp); consumers never meet
//     at a block barrier, so a warp busy inserting falls behind by up to eight
//     stages without stalling the other fifteen;
//   * every wait is bounded: on timeout the warp records SNN_ERR_TIMEOUT in
//     the device state and leaves (the producer first drains its copies).
//
// Exactness notes are those of snn_score_rw.cu: the first pass over a quarter
// of the columns gives an inclusive bound T (k-th smallest of per-lane
// minima = the distance of k distinct columns), the full pass inserts d <= T
// until the list is full and then d < k-th, columns in ascending order.
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "snn_internal.h"

namespace snn {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kChunk = 64;        // columns per warp step (2 per lane)
constexpr int kSC = 128;          // columns per stage
constexpr int kRing = 8;          // stages in the ring
constexpr int kRowsB = 16;        // scored rows per block
constexpr int kCandB = 16;        // candidates per block
constexpr int kConsumers = 16;    // consumer warps (4 row groups x 4 candidate groups)
constexpr int kRW = 4, kCW = 4, kP = kRW * kCW;
constexpr long long kSpinLimit = 1ll << 22;  // try_wait polls before giving up
constexpr unsigned long long kWaitNs = 1000000000ull;  // one second

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
__device__ __forceinline__ unsigned le_mask(float a, float b)
{
    unsigned r;
    asm("set.le.u32.f32 %0, %1, %2;" : "=r"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float sqdiff1(float a, float b)
{
    const float t = __fsub_rn(a, b);
    return __fmul_rn(t, t);
}

// ---- mbarrier / bulk-copy primitives ---------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
    unsigned ok;
    asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                 : "=r"(ok)
                 : "r"(smem_addr(bar)), "r"(parity)
                 : "memory");
    return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Bounded wait: gives up after kSpinLimit polls or one second of wall time,
// whichever comes first (a stage normally completes within microseconds).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (long long i = 0; i < kSpinLimit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255) == 255 && global_ns() - t0 > kWaitNs) return false;
    }
    return false;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Insert (v, col) into the sorted list Ld/Li[0..K) with all 32 lanes; the
// item goes after every element <= v.  Returns the new k-th distance.
__device__ __forceinline__ float smem_list_insert(float *Ld, int *Li, int K, float v, int col, int lane)
{
    int pos = 0;
    for (int g0 = 0; g0 < K; g0 += 32) {
        const int x = g0 + lane;
        const bool ok = x < K;
        const float e = ok ? Ld[x] : INFINITY;
        pos += __popc(__ballot_sync(kFull, ok && e <= v));
    }
    float carry = 0.0f;
    int carryi = 0;
    for (int g0 = 0; g0 < K; g0 += 32) {
        const int x = g0 + lane;
        const bool ok = x < K;
        const float e = ok ? Ld[x] : INFINITY;
        const int ix = ok ? Li[x] : 0;
        float up = __shfl_up_sync(kFull, e, 1);
        int upi = __shfl_up_sync(kFull, ix, 1);
        if (lane == 0) {
            up = carry;
            upi = carryi;
        }
        carry = __shfl_sync(kFull, e, 31);
        carryi = __shfl_sync(kFull, ix, 31);
        if (ok && x >= pos) {
            Ld[x] = (x == pos) ? v : up;
            Li[x] = (x == pos) ? col : upi;
        }
    }
    __syncwarp();
    return Ld[K - 1];
}

// Rare path (out of line): insert the chunk's passing distances of the
// warp's problems, problem by problem, lanes and columns in ascending order.
template <bool BWD>
__device__ __noinline__ void rare_path(unsigned pm, float *myL, int *myI, float *myT, const float *myX,
                                       const float *D_w, const float *X_w, int q0, int colbase, int K, int KL)
{
    const int lane = threadIdx.x & 31;
    unsigned wm = __reduce_or_sync(kFull, pm);
    while (wm) {
        const int p = __ffs(wm) - 1;
        wm &= wm - 1;
        unsigned m = __ballot_sync(kFull, (pm >> p) & 1u);
        const float *drow = D_w + (p / kCW) * kSC + q0;
        const float *xrow = X_w + (p % kCW) * kSC + q0;
        const float xv = myX[p];
        float th = myT[p];
        float *L = myL + p * KL;
        int *LI = myI + p * KL;
        while (m) {
            const int Lh = __ffs(m) - 1;
            m &= m - 1;
#pragma unroll 1
            for (int h = 0; h < 2; ++h) {
                const int c = 2 * Lh + h;
                const float s1 = sqdiff1(xv, xrow[c]);
                const float d = BWD ? __fsub_rn(drow[c], s1) : __fadd_rn(drow[c], s1);
                if (d <= th) {
                    const float kth = smem_list_insert(L, LI, K, d, colbase + c, lane);
                    if (kth < FLT_MAX) th = nextafterf(kth, -INFINITY);
                }
            }
        }
        if (lane == 0) myT[p] = th;
        __syncwarp();
    }
}

// Ascending bitonic sort of 32 values over the warp.
__device__ __forceinline__ float warp_sort32(float v, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const float o = __shfl_xor_sync(kFull, v, j);
            const bool up = (lane & k) == 0;
            const bool lower = (lane & j) == 0;
            const float mn = fminf(v, o), mx = fmaxf(v, o);
            v = (lower == up) ? mn : mx;
        }
    }
    return v;
}

struct TmaSmem {
    float *Ds, *Xs, *Lds, *thr_s, *xv_s;
    int *Lis, *srcand;
    uint64_t *full, *empty;
    int *flag;
};

__device__ __forceinline__ TmaSmem carve_tma(unsigned char *base, int KL)
{
    TmaSmem S;
    uint64_t *bars = reinterpret_cast<uint64_t *>(base);
    S.full = bars;
    S.empty = bars + kRing;
    float *f = reinterpret_cast<float *>(bars + 2 * kRing);
    S.Ds = f;                                        // [kRing][kRowsB][kSC]
    S.Xs = S.Ds + kRing * kRowsB * kSC;               // [kRing][kCandB][kSC]
    S.Lds = S.Xs + kRing * kCandB * kSC;              // [kConsumers][kP][KL]
    S.Lis = reinterpret_cast<int *>(S.Lds + kConsumers * kP * KL);
    S.thr_s = reinterpret_cast<float *>(S.Lis + kConsumers * kP * KL);  // [kConsumers][kP]
    S.xv_s = S.thr_s + kConsumers * kP;
    S.srcand = reinterpret_cast<int *>(S.xv_s + kConsumers * kP);      // [kCandB]
    S.flag = S.srcand + kCandB;
    return S;
}

template <bool BWD>
__global__ void __launch_bounds__((kConsumers + 1) * 32, 1) k_score_tma(Bufs b, int n_cand, int n_cg)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    const int K = b.kmax;
    const int KL = K <= 32 ? 32 : 64;
    const TmaSmem S = carve_tma(smraw, KL);
    if (b.st->done) return;

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int cgb = blockIdx.x % n_cg;
    const int r0 = (blockIdx.x / n_cg) * kRowsB;
    const int c0 = cgb * kCandB;

    if (threadIdx.x < kCandB) {
        const int s = c0 + threadIdx.x;
        S.srcand[threadIdx.x] = b.cands[s < n_cand ? s : 0];
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kRing; ++s) {
            mbar_init(S.full + s, 1);
            mbar_init(S.empty + s, kConsumers);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int nstages = (b.ldc + kSC - 1) / kSC;
    const int nA = nstages >= 4 ? nstages / 4 : 1;
    const int nvirt = nA + nstages;

    if (w == kConsumers) {
        // ---------------- producer warp ----------------
        const int rlast = b.n_rows - 1;
        int issued = 0;
        bool ok = true;
        for (int v = 0; v < nvirt; ++v) {
            const int s = v % kRing;
            if (!mbar_wait(S.empty + s, ((v / kRing) & 1) ^ 1)) {
                ok = false;
                break;
            }
            const int st = v < nA ? v : v - nA;
            const int i0 = st * kSC;
            const int ncols = min(kSC, b.ldc - i0);
            const unsigned bytes = (unsigned)ncols * 4u;
            if (lane == 0) mbar_arrive_expect_tx(S.full + s, bytes * (kRowsB + kCandB));
            __syncwarp();
            if (lane < kRowsB) {
                const int rr = min(r0 + lane, rlast);
                bulk_g2s(S.Ds + (s * kRowsB + lane) * kSC, b.D + (size_t)rr * b.ldc + i0, bytes, S.full + s);
            } else {
                const int c = lane - kRowsB;
                bulk_g2s(S.Xs + (s * kCandB + c) * kSC, b.XT + (size_t)S.srcand[c] * b.ldc + i0, bytes, S.full + s);
            }
            issued = v + 1;
        }
        if (!ok) {
            if (lane == 0) {
                atomicExch(&b.st->error, kErrTimeout);
                atomicExch(&b.st->done, 1);
            }
            // drain: wait (bounded) for the copies of the stages still in flight
            for (int v = issued > kRing ? issued - kRing : 0; v < issued; ++v) mbar_wait(S.full + v % kRing, (v / kRing) & 1);
        }
        return;
    }

    // ---------------- consumer warps ----------------
    const int rg = w / (kCandB / kCW), cw = w % (kCandB / kCW);
    const int wr0 = r0 + rg * kRW;
    const int wc = cw * kCW;
    const bool wvalid = wr0 < b.n_rows;
    float *myL = S.Lds + w * kP * KL;
    int *myI = S.Lis + w * kP * KL;
    float *myT = S.thr_s + w * kP;
    float *myX = S.xv_s + w * kP;
    for (int e = lane; e < kP * KL; e += 32) {
        myL[e] = (e % KL) < K ? FLT_MAX : INFINITY;
        myI[e] = 0;
    }
    float2 xv2[kP];
    float thr[kP];
#pragma unroll
    for (int ri = 0; ri < kRW; ++ri)
#pragma unroll
        for (int ci = 0; ci < kCW; ++ci) {
            const int p = ri * kCW + ci;
            const int r = wr0 + ri;
            const bool okp = r < b.n_rows && c0 + wc + ci < n_cand;
            const float x = okp ? __ldg(b.XV + (size_t)S.srcand[wc + ci] * b.ldr + r) : NAN;  // NaN never passes
            xv2[p] = make_float2(x, x);
            if (lane == 0) myX[p] = x;
        }
    __syncwarp();

    bool alive = true;
    // first pass: per-lane minimum per problem over nA stages
    {
        float mn[kP];
#pragma unroll
        for (int p = 0; p < kP; ++p) mn[p] = INFINITY;
        for (int v = 0; v < nA && alive; ++v) {
            const int s = v % kRing;
            if (!mbar_wait(S.full + s, (v / kRing) & 1)) {
                alive = false;
                break;
            }
            const int i0 = v * kSC;
            const int cols = min(kSC, b.ldc - i0);
            const float *D_w = S.Ds + (s * kRowsB + rg * kRW) * kSC + 2 * lane;
            const float *X_w = S.Xs + (s * kCandB + wc) * kSC + 2 * lane;
            if (wvalid) {
#pragma unroll 2
                for (int q0 = 0; q0 < cols; q0 += kChunk) {
                    float2 dp[kRW], xp[kCW];
#pragma unroll
                    for (int ri = 0; ri < kRW; ++ri) dp[ri] = *reinterpret_cast<const float2 *>(D_w + ri * kSC + q0);
#pragma unroll
                    for (int ci = 0; ci < kCW; ++ci) xp[ci] = *reinterpret_cast<const float2 *>(X_w + ci * kSC + q0);
#pragma unroll
                    for (int ri = 0; ri < kRW; ++ri)
#pragma unroll
                        for (int ci = 0; ci < kCW; ++ci) {
                            const int p = ri * kCW + ci;
                            const float2 s2 = sq2(sub2(xv2[p], xp[ci]));
                            const float2 e = BWD ? sub2(dp[ri], s2) : add2(dp[ri], s2);
                            mn[p] = fminf(mn[p], fminf(e.x, e.y));
                        }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(S.empty + s);
        }
        // T = k-th smallest of the 32 lane minima (k <= 32): the distance of k distinct columns
#pragma unroll
        for (int p = 0; p < kP; ++p) {
            const float srt = warp_sort32(mn[p], lane);
            const float T = __shfl_sync(kFull, srt, (K - 1) & 31);
            thr[p] = T < FLT_MAX ? T : nextafterf(FLT_MAX, 0.0f);  // inclusive bound
            if (lane == 0) myT[p] = thr[p];
        }
        __syncwarp();
    }

    // full pass
    for (int v = nA; v < nvirt && alive; ++v) {
        const int s = v % kRing;
        if (!mbar_wait(S.full + s, (v / kRing) & 1)) {
            alive = false;
            break;
        }
        const int i0 = (v - nA) * kSC;
        const int cols = min(kSC, b.ldc - i0);
        const float *D_w = S.Ds + (s * kRowsB + rg * kRW) * kSC;
        const float *X_w = S.Xs + (s * kCandB + wc) * kSC;
        if (wvalid) {
#pragma unroll 2
            for (int q0 = 0; q0 < cols; q0 += kChunk) {
                float2 dp[kRW], xp[kCW];
#pragma unroll
                for (int ri = 0; ri < kRW; ++ri) dp[ri] = *reinterpret_cast<const float2 *>(D_w + ri * kSC + q0 + 2 * lane);
#pragma unroll
                for (int ci = 0; ci < kCW; ++ci) xp[ci] = *reinterpret_cast<const float2 *>(X_w + ci * kSC + q0 + 2 * lane);
                unsigned pm = 0u;
#pragma unroll
                for (int ri = 0; ri < kRW; ++ri)
#pragma unroll
                    for (int ci = 0; ci < kCW; ++ci) {
                        const int p = ri * kCW + ci;
                        const float2 s2 = sq2(sub2(xv2[p], xp[ci]));
                        const float2 e = BWD ? sub2(dp[ri], s2) : add2(dp[ri], s2);
                        pm |= (le_mask(e.x, thr[p]) | le_mask(e.y, thr[p])) & (1u << p);
                    }
                if (__any_sync(kFull, pm != 0u)) {
                    rare_path<BWD>(pm, myL, myI, myT, myX, D_w, X_w, q0, i0 + q0, K, KL);
#pragma unroll
                    for (int p = 0; p < kP; ++p) thr[p] = myT[p];
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(S.empty + s);
    }
    if (!alive) {
        if (lane == 0) {
            atomicExch(&b.st->error, kErrTimeout);
            atomicExch(&b.st->done, 1);
        }
        return;
    }
    if (!wvalid) return;

    const int nk = b.nk;
    for (int p = 0; p < kP; ++p) {
        const int r = wr0 + p / kCW;
        const int slot = c0 + wc + p % kCW;
        if (r >= b.n_rows || slot >= n_cand) continue;
        const float *L = myL + p * KL;
        const int *LI = myI + p * KL;
        if (b.nn_idx) {
            const size_t o = ((size_t)slot * b.n_rows + r) * K;
            for (int x = lane; x < K; x += 32) {
                b.nn_idx[o + x] = LI[x];
                b.nn_dist[o + x] = L[x];
            }
        }
        // label sum in rank order (sequential FP32, as the reference), lane 0
        if (lane == 0) {
            float acc = 0.0f;
            for (int j = 0; j < K; ++j) {
                acc = __fadd_rn(acc, __ldg(b.yc + LI[j]));
                for (int m = 0; m < nk; ++m) {
                    const int k = __ldg(b.kvals + m);
                    if (k == j + 1) b.pred[((size_t)slot * nk + m) * b.n_rows + r] = __fdiv_rn(acc, (float)k);
                }
            }
        }
    }
}

size_t tma_smem_bytes(int K)
{
    const int KL = K <= 32 ? 32 : 64;
    return sizeof(uint64_t) * 2 * kRing + sizeof(float) * (size_t)kRing * (kRowsB + kCandB) * kSC +
           (sizeof(float) + sizeof(int)) * (size_t)kConsumers * kP * KL + 2 * sizeof(float) * kConsumers * kP +
           sizeof(int) * (kCandB + 1);
}

}  // namespace

bool score_tma_supported(int kmax) { return kmax >= 1 && kmax <= 32; }

cudaError_t launch_score_tma(const Bufs &b, int n_cand, int backward, cudaStream_t s)
{
    const int n_cg = (n_cand + kCandB - 1) / kCandB;
    const long long blocks = (long long)((b.n_rows + kRowsB - 1) / kRowsB) * n_cg;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    const size_t smem = tma_smem_bytes(b.kmax);
    auto kern = backward ? k_score_tma<true> : k_score_tma<false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)blocks, (kConsumers + 1) * 32, smem, s>>>(b, n_cand, n_cg);
    return cudaGetLastError();
}

}  // namespace snn
