// snn_score_rw.cu -- candidate scoring with one scored row per warp.
//
// Same contract as snn_score.cu (exact top-k_max lists in the reference's
// stable (distance, index) order, kNN-mean predictions), different mapping:
//
//   * a warp owns a tile of RW scored rows x CW candidates; its lanes walk
//     the training columns, two adjacent columns per lane (packed f32x2), so
//     a 64-column chunk is one step of the warp;
//   * each (r, c) list lives in registers spread over the lanes (lane j
//     holds element j, j+32, ...), its k-th distance is warp-uniform, and an
//     insertion is a ballot/popc for the position plus one shuffle-up -- about
//     ten instructions, with no shared-memory traffic;
//   * a block of 16 warps covers 16 rows x (16 or 8) candidates: the rows'
//     256-column slices of D and the candidates' slices of X are staged once
//     per block in shared memory (cp.async ring) and each value is reused by
//     every warp tile that needs it.
//
// Two passes.  A scan that starts from an empty list inserts about
// k*(1 + ln(n/k)) items per (row, candidate) -- the k-th distance only
// tightens as the scan proceeds -- and each insertion costs a warp step.  So a
// first pass over the first quarter of the columns keeps, per lane and
// candidate, only the minimum distance of the lane's own columns (one fminf
// per evaluation, no branches); the k-th smallest of the 32 lane minima (64
// for k <= 64: an even-chunk and an odd-chunk minimum per lane) is the
// distance of k distinct real columns, hence an upper bound T on the true
// k-th distance, typically near rank 4(k+1) of all n.  The full pass then
// admits an item while the list holds padding only if d <= T, afterwards if
// d < the list's k-th (strict: each problem's columns are visited in
// ascending order -- chunk by chunk, lanes ascending, a lane's two columns
// in order -- the reference's insertion order), so only ~k(1 + ln 4.6)
// items are inserted and the results are those of the plain scan.
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

// Ascending bitonic sort of G*32 values spread over the warp (element
// g*32 + lane in v[g]).
template <int G>
__device__ __forceinline__ void warp_sort(float (&v)[G], int lane)
{
    constexpr int N = 32 * G;
#pragma unroll
    for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            float o[G];
#pragma unroll
            for (int g = 0; g < G; ++g) o[g] = (j >= 32) ? v[g ^ (j >> 5)] : __shfl_xor_sync(kFull, v[g], j);
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int i = g * 32 + lane;
                const bool up = (i & k) == 0;
                const bool lower = (i & j) == 0;
                // the lower index of an ascending pair keeps the min
                const float mn = fminf(v[g], o[g]), mx = fmaxf(v[g], o[g]);
                v[g] = (lower == up) ? mn : mx;
            }
        }
    }
}

// Insert (v, col) into the sorted list Ld/Li[0..K) in shared memory with all
// 32 lanes (lane j handles elements j, j+32, ...); the item goes after every
// element <= v.  Returns the new k-th distance (warp-uniform).
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

// All-ones if a <= b (false for NaN), else 0: a predicate-free compare, so a
// sequence of them never turns into per-problem branches in the hot loop.
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

// The rare path of the scoring loop, out of line so that the hot loop stays
// small enough for the compiler to unroll and pipeline (its mere presence
// inline cost 2.4x).  Everything it needs is in shared memory: the warp's
// lists, thresholds and x values, and the staged D and X tiles; it recomputes
// the passing distances with scalar .rn operations (bit-identical to the
// packed ones) and inserts them problem by problem, lanes and columns in
// ascending order.  `pm` is the lane's mask of problems with a passing column.
template <int CW, bool BWD>
__device__ __noinline__ void rare_path(unsigned pm, float *myL, int *myI, float *myT, const float *myX,
                                       const float *D_w, const float *X_w, int q0, int colbase, int K, int KL)
{
    const int lane = threadIdx.x & 31;
    unsigned wm = __reduce_or_sync(kFull, pm);
    while (wm) {
        const int p = __ffs(wm) - 1;
        wm &= wm - 1;
        unsigned m = __ballot_sync(kFull, (pm >> p) & 1u);
        const float *drow = D_w + (p / CW) * kStageCols + q0;
        const float *xrow = X_w + (p % CW) * kStageCols + q0;
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
                // inclusive threshold: T until the list is full, then just below its k-th
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

// Warp tile: RW scored rows x CW candidates (P = RW*CW problems, all lanes
// walking the same columns).  Block: NRG x NCG warps = BR rows x BC
// candidates sharing one D tile and one X tile per pipeline stage; per warp
// step a lane loads RW + CW float2 (two columns) and evaluates 2P distances.
//
// The hot loop keeps per problem only the inclusive threshold (register) and
// builds a per-lane bit mask of problems with a passing column; one warp
// vote per step.  The rare taken path is a single compact loop over the set
// bits: lists, thresholds and x values of the warp's problems are mirrored in
// shared memory so the problem index can be dynamic, and the passing
// distances are recomputed with scalar .rn operations from the staged tiles
// (bit-identical to the packed ones).  Keeping that path small matters: 16
// unrolled copies of it thrashed the instruction cache on every taken step.
template <int RW, int CW, int NRG, int NCG, int GK, bool BWD>
__global__ void __launch_bounds__(NRG *NCG * 32, 1) k_score_rw(Bufs b, int n_cand, int n_cg)
{
    constexpr int P = RW * CW;
    constexpr int BR = NRG * RW;
    constexpr int BC = NCG * CW;
    constexpr int NWB = NRG * NCG;
    constexpr int KL = 32 * GK;  // padded list length
    extern __shared__ __align__(16) float sm[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int rg = w / NCG, cw = w % NCG;
    float *Ds = sm;                                               // [stages][BR][kStageCols]
    float *Xs = Ds + kStagesRW * BR * kStageCols;                 // [stages][BC][kStageCols]
    float *Lds = Xs + kStagesRW * BC * kStageCols;                // [NWB][P][KL]
    int *Lis = reinterpret_cast<int *>(Lds + NWB * P * KL);       // [NWB][P][KL]
    float *thr_s = reinterpret_cast<float *>(Lis + NWB * P * KL);  // [NWB][P]
    float *xv_s = thr_s + NWB * P;                                // [NWB][P]
    int *srcand = reinterpret_cast<int *>(xv_s + NWB * P);        // [BC]

    if (b.st->done) return;
    const int K = b.kmax;
    const int cgb = blockIdx.x % n_cg;
    const int r0 = (blockIdx.x / n_cg) * BR;
    const int c0 = cgb * BC;
    const int wr0 = r0 + rg * RW;   // warp's first row
    const int wc = cw * CW;         // warp's first candidate within the block
    const bool wvalid = wr0 < b.n_rows;
    float *myL = Lds + w * P * KL;
    int *myI = Lis + w * P * KL;
    float *myT = thr_s + w * P;
    float *myX = xv_s + w * P;

    if (threadIdx.x < BC) {
        const int s = c0 + threadIdx.x;
        srcand[threadIdx.x] = b.cands[s < n_cand ? s : 0];
    }
    for (int e = lane; e < P * KL; e += 32) {
        myL[e] = (e % KL) < K ? FLT_MAX : INFINITY;
        myI[e] = 0;
    }
    __syncthreads();

    float2 xv2[P];
    float thr[P];
    float mn[P][GK];
#pragma unroll
    for (int ri = 0; ri < RW; ++ri)
#pragma unroll
        for (int ci = 0; ci < CW; ++ci) {
            const int p = ri * CW + ci;
            const int r = wr0 + ri;
            const bool ok = r < b.n_rows && c0 + wc + ci < n_cand;
            const float x = ok ? __ldg(b.XV + (size_t)srcand[wc + ci] * b.ldr + r) : NAN;  // NaN never passes
            xv2[p] = make_float2(x, x);
            thr[p] = FLT_MAX;
            if (lane == 0) myX[p] = x;
#pragma unroll
            for (int g = 0; g < GK; ++g) mn[p][g] = INFINITY;
        }

    const int nstages = b.ldc / kStageCols + (b.ldc % kStageCols ? 1 : 0);
    const int rlast = b.n_rows - 1;
    auto issue = [&](int st, int slot) {
        const int i0 = st * kStageCols;
        float *D_s = Ds + slot * BR * kStageCols;
        float *X_s = Xs + slot * BC * kStageCols;
        constexpr int per_row = kStageCols / 4;  // 16-byte pieces per row
        for (int q = threadIdx.x; q < (BR + BC) * per_row; q += blockDim.x) {
            const int row = q / per_row, p4 = (q % per_row) * 4;
            const int col = min(i0 + p4, b.ldc - 4);  // the last stage may overrun ldc: clamp (never used)
            if (row < BR) {
                const int rr = min(r0 + row, rlast);
                cp_async16(D_s + row * kStageCols + p4, b.D + (size_t)rr * b.ldc + col);
            } else {
                const int c = row - BR;
                cp_async16(X_s + c * kStageCols + p4, b.XT + (size_t)srcand[c] * b.ldc + col);
            }
        }
    };

    // virtual stage sequence: [0, nA) first pass (lane minima), then all stages
    const int nA = nstages >= 4 ? nstages / 4 : 1;
    const int nvirt = nA + nstages;
    auto phys = [&](int v) { return v < nA ? v : v - nA; };

    issue(phys(0), 0);
    cp_async_commit();
    if (nvirt > 1) issue(phys(1), 1);
    cp_async_commit();

    for (int v = 0; v < nvirt; ++v) {
        const int slot = v % kStagesRW;
        cp_async_wait<1>();
        __syncthreads();
        if (v + 2 < nvirt) issue(phys(v + 2), (v + 2) % kStagesRW);
        cp_async_commit();
        if (!wvalid) continue;
        const int st = phys(v);
        const float *D_w = Ds + slot * BR * kStageCols + (rg * RW) * kStageCols;  // warp's rows
        const float *X_w = Xs + slot * BC * kStageCols + wc * kStageCols;         // warp's candidates
        const int i0 = st * kStageCols;
        const int cols = min(kStageCols, b.ldc - i0);
        if (v < nA) {
            // first pass: per-lane minimum per problem (even / odd chunks for GK = 2)
            for (int q0 = 0; q0 < cols; q0 += kChunk) {
                float2 dp[RW], xp[CW];
#pragma unroll
                for (int ri = 0; ri < RW; ++ri) dp[ri] = *reinterpret_cast<const float2 *>(D_w + ri * kStageCols + q0 + 2 * lane);
#pragma unroll
                for (int ci = 0; ci < CW; ++ci) xp[ci] = *reinterpret_cast<const float2 *>(X_w + ci * kStageCols + q0 + 2 * lane);
                const int gsel = (q0 / kChunk) & 1;
#pragma unroll
                for (int ri = 0; ri < RW; ++ri)
#pragma unroll
                    for (int ci = 0; ci < CW; ++ci) {
                        const int p = ri * CW + ci;
                        const float2 s2 = sq2(sub2(xv2[p], xp[ci]));
                        const float2 e = BWD ? sub2(dp[ri], s2) : add2(dp[ri], s2);
                        const float m2 = fminf(e.x, e.y);
                        if (GK == 1 || gsel == 0) mn[p][0] = fminf(mn[p][0], m2);
                        else mn[p][GK - 1] = fminf(mn[p][GK - 1], m2);
                    }
            }
            if (v == nA - 1) {
                // T = k-th smallest of the lane minima: the distance of k distinct columns
#pragma unroll
                for (int p = 0; p < P; ++p) {
                    warp_sort<GK>(mn[p], lane);
                    float pick = mn[p][0];
#pragma unroll
                    for (int g = 1; g < GK; ++g)
                        if (g == ((K - 1) >> 5)) pick = mn[p][g];
                    const float T = __shfl_sync(kFull, pick, (K - 1) & 31);
                    thr[p] = T < FLT_MAX ? T : nextafterf(FLT_MAX, 0.0f);  // inclusive bound
                    if (lane == 0) myT[p] = thr[p];
                }
                __syncwarp();
            }
            continue;
        }
#pragma unroll 2
        for (int q0 = 0; q0 < cols; q0 += kChunk) {
            float2 dp[RW], xp[CW];
#pragma unroll
            for (int ri = 0; ri < RW; ++ri) dp[ri] = *reinterpret_cast<const float2 *>(D_w + ri * kStageCols + q0 + 2 * lane);
#pragma unroll
            for (int ci = 0; ci < CW; ++ci) xp[ci] = *reinterpret_cast<const float2 *>(X_w + ci * kStageCols + q0 + 2 * lane);
            unsigned pm = 0u;
#pragma unroll
            for (int ri = 0; ri < RW; ++ri)
#pragma unroll
                for (int ci = 0; ci < CW; ++ci) {
                    const int p = ri * CW + ci;
                    const float2 s2 = sq2(sub2(xv2[p], xp[ci]));
                    const float2 e = BWD ? sub2(dp[ri], s2) : add2(dp[ri], s2);
                    pm |= (le_mask(e.x, thr[p]) | le_mask(e.y, thr[p])) & (1u << p);
                }
            if (__any_sync(kFull, pm != 0u)) {
                rare_path<CW, BWD>(pm, myL, myI, myT, myX, D_w, X_w, q0, i0 + q0, K, KL);
#pragma unroll
                for (int p = 0; p < P; ++p) thr[p] = myT[p];
            }
        }
    }
    cp_async_wait<0>();
    if (!wvalid) return;

    const int nk = b.nk;
    for (int p = 0; p < P; ++p) {
        const int r = wr0 + p / CW;
        const int slot = c0 + wc + p % CW;
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
                // k_vals may repeat or be unsorted: test every entry
                for (int m = 0; m < nk; ++m) {
                    const int k = __ldg(b.kvals + m);
                    if (k == j + 1) b.pred[((size_t)slot * nk + m) * b.n_rows + r] = __fdiv_rn(acc, (float)k);
                }
            }
        }
    }
}

template <int RW, int CW, int NRG, int NCG, int GK, bool BWD>
cudaError_t launch_rw(const Bufs &b, int n_cand, cudaStream_t s)
{
    constexpr int BR = NRG * RW, BC = NCG * CW;
    const int n_cg = (n_cand + BC - 1) / BC;
    const long long blocks = (long long)((b.n_rows + BR - 1) / BR) * n_cg;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    constexpr int P = RW * CW, NWB = NRG * NCG, KL = 32 * GK;
    const size_t smem = sizeof(float) * (size_t)kStagesRW * (BR + BC) * kStageCols +
                        (sizeof(float) + sizeof(int)) * (size_t)NWB * P * KL + 2 * sizeof(float) * NWB * P +
                        sizeof(int) * BC;
    auto kern = k_score_rw<RW, CW, NRG, NCG, GK, BWD>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)blocks, NRG * NCG * 32, smem, s>>>(b, n_cand, n_cg);
    return cudaGetLastError();
}

}  // namespace

bool score_rw_supported(int kmax) { return kmax >= 1 && kmax <= 64; }

cudaError_t launch_score_rw(const Bufs &b, int n_cand, int backward, cudaStream_t s)
{
    if (b.kmax <= 32)
        return backward ? launch_rw<4, 4, 4, 4, 1, true>(b, n_cand, s) : launch_rw<4, 4, 4, 4, 1, false>(b, n_cand, s);
    if (b.kmax <= 64)
        return backward ? launch_rw<2, 4, 8, 2, 2, true>(b, n_cand, s) : launch_rw<2, 4, 8, 2, 2, false>(b, n_cand, s);
    return cudaErrorInvalidValue;
}

}  // namespace snn
