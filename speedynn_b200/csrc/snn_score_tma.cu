// snn_score_tma.cu -- candidate scoring, warp-specialised TMA pipeline.
//
// For every (scored row, candidate): the exact top-k_max list (k <= 64) of
// d_i = fl(D[r,i] +/- fl((x_r,c - x_i,c)^2)) over the training columns i in
// the reference's stable (distance, index) order
// (speedynn/lib/cpu.c:128-168) and the kNN-mean predictions (cpu.c:56-66).
// A block scores 24 (forward with k <= 16: 12) rows x 12 candidates; each of
// its 18 (9) consumer warps owns 4 rows x 4 candidates and walks the columns
// two per lane with packed f32x2 (19 warps per block, or two blocks of 10
// warps per SM: at most 5 warps per SM sub-partition at 96 registers;
// 12-candidate groups leave no padded slot for 60 candidates).  For
// 32 < k <= 64 the 64-slot lists (two entries per lane) take more shared
// memory, which leaves room for a 2-slot ring.
//
//   * Feed: one producer lane streams 256-column stages into a ring of
//     shared-memory slots (as deep as fits beside the lists): a 2-D
//     tensor-map TMA copy of the block's D rows and three tile::gather4
//     copies of the 12 candidate rows of X, all completing on the stage's "full"
//     mbarrier; consumers release a slot through its "empty" mbarrier, so a
//     warp busy inserting falls behind by up to a ring of stages without
//     stalling the others.
//   * Starting bound on each problem's k-th distance (k distinct columns lie
//     at or below it): a first pass over a quarter of the columns (per-lane
//     minima, their k-th smallest); or, on seeded forward steps, the k-th
//     smallest exact distance over the row's 256 seed columns (the columns
//     nearest the row under the committed D, kept by the last commit),
//     computed beforehand by k_seed_bounds; or, on
//     backward steps after the first, the previous step's k-th distances
//     (kth_prev), which removal only lowers.
//   * Full pass: forward, 64-column chunks whose committed distances all
//     exceed the warp's row bounds are skipped (d >= D); in the rest a
//     conservative sign-bit filter (one sub and one FMA per evaluation;
//     filter_bound / filter_bound_bwd) flags rows that may hold a passing
//     column; flagged rows are re-scored with the reference's
//     rounding and passes are inserted in column order (d <= T until the list
//     is full, then d < k-th).
//   * Every wait is bounded: on timeout the warp records SNN_ERR_TIMEOUT in
//     the device state and leaves (the producer first drains its copies).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <float.h>
#include <math.h>
#include <stdint.h>

#include <mutex>

#include "snn_internal.h"

namespace snn {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kChunk = 64;        // columns per warp step (2 per lane)
constexpr int kSC = 256;          // columns per stage
constexpr int kMaxRing = 8;       // most stages in the ring (the depth is a template argument)
constexpr int kBarBytes = 128;    // full + empty mbarriers, padded so the tiles stay 128-byte aligned
static_assert(2 * kMaxRing * sizeof(uint64_t) <= kBarBytes, "mbarriers must fit their area");
// A block has RG x CG consumer warps (template arguments), each owning kRW
// rows x kCW candidates: kRowsB = RG * kRW scored rows, kCandB = CG * kCW
// candidates, kConsumers = RG * CG.
constexpr int kRingDeep = 5;      // ring slots beside 16-slot lists (k <= 16, backward)
constexpr int kRingShallow = 4;   // ring slots beside 32- and 64-slot lists
constexpr int kRW = 4, kCW = 4, kP = kRW * kCW;
constexpr long long kSpinLimit = 1ll << 22;  // try_wait polls before giving up
constexpr unsigned long long kWaitNs = 1000000000ull;  // one second

// Shared-memory slots per neighbour list (k <= 64).
__host__ __device__ constexpr int list_slots(int K) { return K <= 16 ? 16 : K <= 32 ? 32 : 64; }

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
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(as_u64(a)), "l"(as_u64(b)), "l"(as_u64(c)));
    return as_f2(d);
}
__device__ __forceinline__ float min3f(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ unsigned f2u(float v) { return __float_as_uint(v); }

// Inclusive bound on the exact forward distance from a first-pass value
// a = fl(t*t + D), D >= 0: d = fl(D + fl(t*t)) <= a (1 + 3.01 * 2^-24) + 2^-147,
// and fma(a, 1 + 2^-20, 2^-140) exceeds that after its own rounding.  Capped
// at the largest float below FLT_MAX (items at FLT_MAX never enter a list).
__device__ __forceinline__ float fwd_bound(float a)
{
    return fminf(fmaf(a, 1.0f + 0x1p-20f, 0x1p-140f), 0x1.fffffcp+127f);
}

// Filter bound H for an inclusive threshold T (forward, D >= 0).  If
// d = fl(D + fl(t*t)) <= T then the exact value t*t + fl(D - H) is negative:
// D + t*t <= T+ (1 + 2^-23) + 2^-149 with T+ = max(T, 0), fl(D - H) is off by
// at most H * 2^-24 + 2^-150 because 0 <= D <= H, and H >= T+ (1 + 2^-19) +
// 2^-126 after rounding.  A negative exact value keeps its sign bit through
// the FMA's rounding (an underflow gives -0), so testing the sign bit of
// u = fma(t, t, fl(D - H)) never misses a passing column.
__device__ __forceinline__ float filter_bound(float T) { return fmaf(fmaxf(T, 0.0f), 1.0f + 0x1p-18f, 0x1p-125f); }

// Backward filter bound: d = fl(D - fl(t*t)) <= T implies that the exact value
// t*t + fl(H - D) is positive when H >= T+ (1 + 2^-19) + Dm 2^-21 + 2^-126,
// Dm >= every finite D of the row (t*t <= D + T+ there, and fl(H - D) is off
// by at most max(D, H) 2^-24).  A positive exact value keeps a clear sign bit
// through the FMA's rounding, so u = fma(t, t, fl(H - D)) >= 0 (sign bit
// clear) for every passing column.
__device__ __forceinline__ float filter_bound_bwd(float T, float Dm)
{
    return fmaf(fmaxf(T, 0.0f), 1.0f + 0x1p-18f, fmaf(Dm, 0x1p-20f, 0x1p-125f));
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
// One 2-D tile (box of the tensor map) into shared memory, completing on bar.
__device__ __forceinline__ void tma_tile_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}
// Four rows y0..y3 of a 2-D tensor (box one row high), columns x.., stacked in
// shared memory in that order, completing on bar.
__device__ __forceinline__ void tma_gather4(void *dst, const CUtensorMap *map, int x, int y0, int y1, int y2, int y3,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cta.global.tile::gather4.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
        "%6}], [%7];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3), "r"(smem_addr(bar))
        : "memory");
}

// Largest float below x for 0 <= x < FLT_MAX (forward distances): turns the
// strict test d < kth into the inclusive d <= below(kth).
__device__ __forceinline__ float below(float x) { return x > 0.0f ? __int_as_float(__float_as_int(x) - 1) : -0x1p-149f; }

// Insert a chunk's passing distances into the warp's lists (K <= KL <= 64).  pm holds this lane's passes, bit 2*p + h for problem p and chunk
// column 2*lane + h; D_s / X_s are the warp's D rows and candidate X rows of
// the stage (kSC columns each).  Items go in column order with the reference
// rule (after every element <= d, entry below the k-th once the list is
// full); every lane recomputes each item's exact distance from shared
// memory, and the list being filled sits in registers, lane j holding entry j
// (entries 2j and 2j+1 for k_max > 32).
// Returns a mask of the warp's rows (bit p / kCW) whose thresholds may have
// changed.
template <bool BWD, int KL>
__device__ __forceinline__ unsigned insert_chunk(unsigned pm, const float *D_s, const float *X_s, const float *myX, float *myL,
                                          int *myI, float *myT, int q0, int colbase, int K)
{
    constexpr bool LONG = KL > 32;
    const int lane = threadIdx.x & 31;
    unsigned rows = 0u;
    unsigned any = __reduce_or_sync(kFull, pm);
    while (any) {
        const int p = (__ffs(any) - 1) >> 1;
        any &= ~(3u << (2 * p));
        float *L = myL + p * KL;
        int *LI = myI + p * KL;
        float th = myT[p];
        const float xv = myX[p];
        const float *xrow = X_s + (p % kCW) * kSC + q0;
        const float *dr = D_s + (p / kCW) * kSC + q0;
        const unsigned mine = (pm >> (2 * p)) & 3u;
        unsigned m = __ballot_sync(kFull, mine != 0u);
        if constexpr (LONG) {
            // k_max > 32: lane j holds the adjacent entries 2j and 2j+1 (one
            // 64-bit shared-memory access each for distances and columns), so
            // an insertion shifts the list with one shuffle per array
            const int e0 = 2 * lane;
            float2 Lv = make_float2(INFINITY, INFINITY);
            int2 Iv = make_int2(0, 0);
            if (e0 < K) {
                Lv = *reinterpret_cast<const float2 *>(L + e0);
                Iv = *reinterpret_cast<const int2 *>(LI + e0);
                if (e0 + 1 >= K) {
                    Lv.y = INFINITY;
                    Iv.y = 0;
                }
            }
            while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                const unsigned hb = __shfl_sync(kFull, mine, l);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (!((hb >> h) & 1u)) continue;
                    const int c = 2 * l + h;
                    const float s1 = sqdiff1(xv, xrow[c]);
                    const float d = BWD ? __fsub_rn(dr[c], s1) : __fadd_rn(dr[c], s1);
                    if (d <= th) {
                        // d < FLT_MAX and, for a full list, d < k-th: the slot is < K
                        const int pos = __popc(__ballot_sync(kFull, e0 < K && Lv.x <= d)) +
                                        __popc(__ballot_sync(kFull, e0 + 1 < K && Lv.y <= d));
                        const float pL = __shfl_up_sync(kFull, Lv.y, 1);  // entry 2j - 1
                        const int pI = __shfl_up_sync(kFull, Iv.y, 1);
                        // entry 2j + 1 first: it may take the old entry 2j
                        if (e0 + 1 == pos) {
                            Lv.y = d;
                            Iv.y = colbase + c;
                        } else if (e0 + 1 > pos) {
                            Lv.y = Lv.x;
                            Iv.y = Iv.x;
                        }
                        if (e0 == pos) {
                            Lv.x = d;
                            Iv.x = colbase + c;
                        } else if (e0 > pos) {
                            Lv.x = pL;
                            Iv.x = pI;
                        }
                        const float kth = __shfl_sync(kFull, ((K - 1) & 1) ? Lv.y : Lv.x, (K - 1) >> 1);
                        if (kth < FLT_MAX) th = BWD ? nextafterf(kth, -INFINITY) : below(kth);
                    }
                }
            }
            // with K odd, lane (K-1)/2 also writes slot K, which lies past the list and is never read
            if (e0 < K) {
                *reinterpret_cast<float2 *>(L + e0) = Lv;
                *reinterpret_cast<int2 *>(LI + e0) = Iv;
            }
        } else {
            // lane j holds entry j
            float L0 = lane < K ? L[lane] : INFINITY;
            int I0 = lane < K ? LI[lane] : 0;
            while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                const unsigned hb = __shfl_sync(kFull, mine, l);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (!((hb >> h) & 1u)) continue;
                    const int c = 2 * l + h;
                    const float s1 = sqdiff1(xv, xrow[c]);
                    const float d = BWD ? __fsub_rn(dr[c], s1) : __fadd_rn(dr[c], s1);
                    if (d <= th) {
                        // d < FLT_MAX and, for a full list, d < k-th: the slot is < K
                        const int pos = __popc(__ballot_sync(kFull, lane < K && L0 <= d));
                        const float up0 = __shfl_up_sync(kFull, L0, 1);
                        const int upi0 = __shfl_up_sync(kFull, I0, 1);
                        if (lane == pos) {
                            L0 = d;
                            I0 = colbase + c;
                        } else if (lane > pos) {
                            L0 = up0;
                            I0 = upi0;
                        }
                        const float kth = __shfl_sync(kFull, L0, K - 1);
                        if (kth < FLT_MAX) th = BWD ? nextafterf(kth, -INFINITY) : below(kth);
                    }
                }
            }
            if (lane < K) {
                L[lane] = L0;
                LI[lane] = I0;
            }
        }
        if (lane == 0) myT[p] = th;
        rows |= 1u << (p / kCW);
    }
    __syncwarp();
    return rows;
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

// Ascending bitonic sort of 32*V values over the warp, V per lane: lane l
// holds elements V*l .. V*l+V-1 (NaN must not occur: fminf/fmaxf would drop it).
template <int V>
__device__ __forceinline__ void warp_sort_v(float (&v)[V], int lane)
{
#pragma unroll
    for (int k = 2; k <= 32 * V; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= V) {  // partner in lane ^ (j / V), same slot
#pragma unroll
                for (int h = 0; h < V; ++h) {
                    const float o = __shfl_xor_sync(kFull, v[h], j / V);
                    const int i = V * lane + h;
                    v[h] = (((i & j) == 0) == ((i & k) == 0)) ? fminf(v[h], o) : fmaxf(v[h], o);
                }
            } else {  // partner in the same lane
#pragma unroll
                for (int h = 0; h < V; ++h) {
                    if ((h & j) == 0) {
                        const bool up = ((V * lane + h) & k) == 0;
                        const float a = v[h], c = v[h + j];
                        v[h] = up ? fminf(a, c) : fmaxf(a, c);
                        v[h + j] = up ? fmaxf(a, c) : fminf(a, c);
                    }
                }
            }
        }
    }
}

// K-th smallest (1-based, K <= 32*V) of the 32*V values v[] over the warp.
template <int V>
__device__ __forceinline__ float warp_kth(float (&v)[V], int K, int lane)
{
    warp_sort_v<V>(v, lane);
    float sel = v[0];
#pragma unroll
    for (int h = 1; h < V; ++h)
        if (h == (K - 1) % V) sel = v[h];
    return __shfl_sync(kFull, sel, (K - 1) / V);
}

// xrm[i][slot] = X[cands[slot]][i]: the step's candidate columns, row-major
// (n_cols x n_cand), through 32 x 32 shared-memory tiles.
__global__ void __launch_bounds__(256) k_candidates_rowmajor(Bufs b, int n_cand, float *xrm)
{
    __shared__ float tile[32][33];
    if (b.st->done) return;
    const int i0 = blockIdx.x * 32, s0 = blockIdx.y * 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int k = ty; k < 32; k += 8) {
        const int slot = s0 + k, i = i0 + tx;
        tile[k][tx] = slot < n_cand && i < b.n_cols ? __ldg(b.XT + (size_t)__ldg(b.cands + slot) * b.ldc + i) : 0.0f;
    }
    __syncthreads();
    for (int k = ty; k < 32; k += 8) {
        const int i = i0 + k, slot = s0 + tx;
        if (i < b.n_cols && slot < n_cand) xrm[(size_t)i * n_cand + slot] = tile[tx][k];
    }
}

// k_seed_bounds_exact (K <= L <= 16): the bound of each (candidate, scored row)
// problem is the K-th smallest exact distance d = fl(D + fl((x_r,c - x_i,c)^2))
// over ALL kSeeds seed columns of the row (see k_seed_bounds for why any K
// distinct columns bound the final K-th distance).  One warp per row, lane l
// taking candidate slot l (then l + 32, ...): the L smallest distances seen
// sit sorted in registers (L the list length rounded up to 4, 8, 12 or 16), and each seed column's values for 32 candidates
// are one contiguous read of xrm.  Seeds are taken in the commit's order;
// a seed whose committed distance already reaches every lane's L-th smallest
// is skipped (d >= D).
template <int L>
__global__ void __launch_bounds__(256) k_seed_bounds_exact(Bufs b, int n_cand, const float *xrm, float *bound)
{
    if (b.st->done) return;
    const int lane = threadIdx.x & 31;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (r >= b.n_rows) return;  // warp-uniform
    const int K = b.kmax;
    for (int c0 = 0; c0 < n_cand; c0 += 32) {
        const int slot = c0 + lane;
        const bool live = slot < n_cand;
        const int c = live ? __ldg(b.cands + slot) : 0;  // the candidate feature
        const float xv = live ? __ldg(b.XV + (size_t)c * b.ldr + r) : 0.0f;
        float l[L];
#pragma unroll
        for (int j = 0; j < L; ++j) l[j] = INFINITY;
        for (int j0 = 0; j0 < kSeeds; j0 += 32) {
            const int myi = __ldg(b.seeds + (size_t)r * kSeeds + j0 + lane);
            const float myd = __ldg(b.seed_d + (size_t)r * kSeeds + j0 + lane);
            // eight seeds at a time: their loads are issued together, then inserted in order
            for (int j8 = 0; j8 < 32; j8 += 8) {
                int ii[8];
                float DD[8], xx[8];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    ii[u] = __shfl_sync(kFull, myi, j8 + u);
                    DD[u] = __shfl_sync(kFull, myd, j8 + u);
                    xx[u] = live && ii[u] >= 0 ? __ldg(xrm + (size_t)ii[u] * n_cand + slot) : 0.0f;
                }
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const float t = __fsub_rn(xv, xx[u]);
                    float d = __fadd_rn(DD[u], __fmul_rn(t, t));
                    // padding seed, NaN or overflow: never a neighbour
                    if (!(d < FLT_MAX) || !live || ii[u] < 0) d = INFINITY;
                    if (__any_sync(kFull, d < l[L - 1])) {
                        // keep the L smallest sorted: l[j] = min(l[j], max(l[j-1], d))
#pragma unroll
                        for (int j = L - 1; j > 0; --j) l[j] = fminf(l[j], fmaxf(l[j - 1], d));
                        l[0] = fminf(l[0], d);
                    }
                }
            }
        }
        float kth = l[0];
#pragma unroll
        for (int j = 1; j < L; ++j)
            if (j == K - 1) kth = l[j];
        if (live) bound[(size_t)c * b.n_rows + r] = kth;  // indexed by feature, as k_seed_bounds
    }
}

// k_seed_bounds: the starting bound of every (candidate, scored row) problem
// of a seeded forward step, bound[c][r] = the K-th smallest exact distance
// d = fl(D + fl((x_r,c - x_i,c)^2)) over columns of the row's kSeeds seed
// columns (kept by the last commit, snn_commit.cu).  Any K distinct columns
// have their K-th smallest distance at or above the final K-th neighbour
// distance, so it is an inclusive bound; padding seeds (index -1) and NaN
// distances count as +inf.  One warp per row, lane l holding seeds
// l + 32 j (j < kSeedsPerLane); the gathers of two candidates are issued
// together, and many warps per SM hide their latency.  Each lane keeps its
// V smallest values (V = 2 for K <= 16, 4 above), and the K-th smallest of
// those 32 V values is the bound: a subset of the seeds, so still K distinct
// columns, and as tight as all of them unless a lane holds more than V of
// the K nearest.
template <int V>
__global__ void __launch_bounds__(256) k_seed_bounds(Bufs b, int n_cand, float *bound)
{
    constexpr int S = kSeedsPerLane;
    if (b.st->done) return;
    const int lane = threadIdx.x & 31;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (r >= b.n_rows) return;
    const int K = b.kmax;
    int si[S];
    float sd[S];
#pragma unroll
    for (int j = 0; j < S; ++j) {
        si[j] = __ldg(b.seeds + (size_t)r * kSeeds + j * 32 + lane);
        sd[j] = __ldg(b.seed_d + (size_t)r * kSeeds + j * 32 + lane);
    }
    constexpr int Q = 2;  // candidates whose gathers are in flight together (4: 96 registers, no faster)
    for (int c0 = 0; c0 < n_cand; c0 += Q) {
        int cid[Q];
        float xr[Q], g[Q][S];
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            cid[q] = c0 + q < n_cand ? __ldg(b.cands + c0 + q) : -1;
            xr[q] = cid[q] >= 0 ? __ldg(b.XV + (size_t)cid[q] * b.ldr + r) : 0.0f;
#pragma unroll
            for (int j = 0; j < S; ++j)
                g[q][j] = cid[q] >= 0 && si[j] >= 0 ? __ldg(b.XT + (size_t)cid[q] * b.ldc + si[j]) : 0.0f;
        }
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (cid[q] < 0) break;  // warp-uniform
            // the lane's V smallest of its S distances, by insertion into a sorted list
            float best[V];
#pragma unroll
            for (int h = 0; h < V; ++h) best[h] = INFINITY;
#pragma unroll
            for (int j = 0; j < S; ++j) {
                float d = si[j] >= 0 ? __fadd_rn(sd[j], sqdiff1(xr[q], g[q][j])) : INFINITY;
                d = d <= FLT_MAX ? d : INFINITY;
#pragma unroll
                for (int h = 0; h < V; ++h) {  // compare-exchange down the list
                    const float lo = fminf(best[h], d);
                    d = fmaxf(best[h], d);
                    best[h] = lo;
                }
            }
            const float T = warp_kth<V>(best, K, lane);
            if (lane == 0) bound[(size_t)cid[q] * b.n_rows + r] = T;
        }
    }
}

struct TmaSmem {
    float *Ds, *Xs, *Lds, *thr_s, *xv_s;
    int *Lis, *srcand, *wcnt;
    uint64_t *full, *empty;
    int *flag;
};

template <int RG, int CG>
__device__ __forceinline__ TmaSmem carve_tma(unsigned char *base, int KL, int ring)
{
    constexpr int kRowsB = RG * kRW, kCandB = CG * kCW, kConsumers = RG * CG;
    TmaSmem S;
    uint64_t *bars = reinterpret_cast<uint64_t *>(base);
    S.full = bars;
    S.empty = bars + ring;
    float *f = reinterpret_cast<float *>(base + kBarBytes);  // tiles start 128-byte aligned
    S.Ds = f;                                        // [ring][kRowsB][kSC]
    S.Xs = S.Ds + ring * kRowsB * kSC;                // [ring][kCandB][kSC]
    S.Lds = S.Xs + ring * kCandB * kSC;               // [kConsumers][kP][KL]
    S.Lis = reinterpret_cast<int *>(S.Lds + kConsumers * kP * KL);
    S.thr_s = reinterpret_cast<float *>(S.Lis + kConsumers * kP * KL);  // [kConsumers][kP]
    S.xv_s = S.thr_s + kConsumers * kP;
    S.srcand = reinterpret_cast<int *>(S.xv_s + kConsumers * kP);      // [kCandB]
    S.flag = S.srcand + kCandB;
    S.wcnt = S.flag + 1;  // [kConsumers][2] flagged / passing (row, chunk) pairs
    return S;
}

// RG x CG consumer warps (row groups x candidate groups of 4); KL list slots
// per row (16, 32 or 64).  KL = 64 (k_max in (32, 64]) keeps two list entries
// and two first-pass minima per lane.
// (32, 64] -- two list entries per lane and two first-pass minima per lane.
template <bool BWD, int ring, bool COUNT, int RG, int CG, int KL>
__global__ void __launch_bounds__((RG * CG + 1) * 32, RG * CG <= 9 ? 2 : 1) k_score_tma(Bufs b, int n_cand, int n_cg, int slot0,
                                                                     const __grid_constant__ CUtensorMap tmD,
                                                                     const __grid_constant__ CUtensorMap tmX)
{
    constexpr int kRowsB = RG * kRW, kCandB = CG * kCW, kConsumers = RG * CG;
    extern __shared__ __align__(128) unsigned char smraw[];
    const int K = b.kmax;
    constexpr bool LONG = KL > 32;
    const TmaSmem S = carve_tma<RG, CG>(smraw, KL, ring);
    if (b.st->done) return;
    if (b.only_if_full && !b.st->full_scan) return;  // the sorted first step scored every problem

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int cgb = blockIdx.x % n_cg;
    const int r0 = (blockIdx.x / n_cg) * kRowsB;
    const int c0 = slot0 + cgb * kCandB;  // the block's first candidate slot

    if (threadIdx.x < kCandB) {
        const int s = c0 + threadIdx.x;
        S.srcand[threadIdx.x] = b.cands[s < n_cand ? s : 0];
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < ring; ++s) {
            mbar_init(S.full + s, 1);
            mbar_init(S.empty + s, kConsumers);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int nstages = (b.ldc + kSC - 1) / kSC;
    // Backward steps after the first reuse the last step's k-th distances as
    // bounds (D only shrinks when a feature is removed) and skip the first pass.
    const bool reuse = BWD && b.use_prev && b.kth_prev != nullptr;
    // Seeded forward steps take their bounds from the previous commit's seed
    // columns and skip the first pass as well.
    const bool seeded = !BWD && b.use_seeds && b.bound != nullptr;
    const int nA = reuse || seeded ? 0 : (nstages >= 4 ? nstages / 4 : 1);
    const int nvirt = nA + nstages;

    if (w == kConsumers) {
        // ---------------- producer warp (one lane) ----------------
        // Per stage: the D tile (kRowsB rows x kSC columns, rows past n_rows
        // read as 0 and belong to padded problems) and the block's kCandB
        // candidate rows of X, gathered four at a time.  Columns past ldc in the
        // last stage also read as 0; consumers never look past ldc.
        if (lane == 0) {
            constexpr unsigned kStageBytes = sizeof(float) * kSC * (kRowsB + kCandB);
            int issued = 0;
            bool ok = true;
            for (int v = 0; v < nvirt; ++v) {
                const int s = v % ring;
                if (!mbar_wait(S.empty + s, ((v / ring) & 1) ^ 1)) {
                    ok = false;
                    break;
                }
                const int i0 = (v < nA ? v : v - nA) * kSC;
                if (blockIdx.x == 0 && v + 1 == b.inject_stall) {  // test hook: the consumers' waits run out
                    issued = v + 1;
                    continue;
                }
                mbar_arrive_expect_tx(S.full + s, kStageBytes);
                tma_tile_2d(S.Ds + s * kRowsB * kSC, &tmD, i0, r0, S.full + s);
#pragma unroll
                for (int g = 0; g < kCandB / 4; ++g)
                    tma_gather4(S.Xs + (s * kCandB + 4 * g) * kSC, &tmX, i0, S.srcand[4 * g], S.srcand[4 * g + 1],
                                S.srcand[4 * g + 2], S.srcand[4 * g + 3], S.full + s);
                issued = v + 1;
            }
            if (!ok) {
                atomicExch(&b.st->error, kErrTimeout);
                atomicExch(&b.st->done, 1);
                // drain: wait (bounded) for the copies of the stages still in flight
                for (int v = issued > ring ? issued - ring : 0; v < issued; ++v)
                    mbar_wait(S.full + v % ring, (v / ring) & 1);
            }
        }
        return;
    }

    // ---------------- consumer warps ----------------
    const int rg = w / (kCandB / kCW), cw = w % (kCandB / kCW);
    const int wr0 = r0 + rg * kRW;
    const int wc = cw * kCW;
    // a warp whose rows or candidate slots are all padding only releases stages
    const bool wvalid = wr0 < b.n_rows && c0 + wc < n_cand;
    float *myL = S.Lds + w * kP * KL;
    int *myI = S.Lis + w * kP * KL;
    float *myT = S.thr_s + w * kP;
    float *myX = S.xv_s + w * kP;
    int *myCnt = S.wcnt + 2 * w;
    if (COUNT && lane == 0) myCnt[0] = myCnt[1] = 0;
    for (int e = lane; e < kP * KL; e += 32) {
        myL[e] = (e % KL) < K ? FLT_MAX : INFINITY;
        myI[e] = 0;
    }
    // A padded problem (row past n_rows or candidate slot past n_cand) gets a
    // scored value that can never pass: NaN for backward (d = NaN), +inf for
    // forward (d = D + inf = inf, and the forward filter value stays >= 0);
    // backward padded candidate slots on real rows are shadows (below).
    float2 xv2[kP];
    unsigned okmask = 0u;
#pragma unroll
    for (int ri = 0; ri < kRW; ++ri)
#pragma unroll
        for (int ci = 0; ci < kCW; ++ci) {
            const int p = ri * kCW + ci;
            const int r = wr0 + ri;
            const bool okp = r < b.n_rows && c0 + wc + ci < n_cand;
            // Backward scores a padded candidate slot as a shadow copy of a real
            // candidate (srcand repeats cands[0]; nothing of it is written), so its
            // filter flags no more often than a real problem's.
            const bool live = BWD ? r < b.n_rows : okp;
            const float x = live ? __ldg(b.XV + (size_t)S.srcand[wc + ci] * b.ldr + r) : (BWD ? NAN : INFINITY);
            xv2[p] = make_float2(x, x);
            okmask |= okp ? (1u << p) : 0u;
            if (lane == 0) myX[p] = x;
        }
    __syncwarp();

    // backward: per-row bound on the finite committed distances (filter margin)
    float myDm[kRW];
#pragma unroll
    for (int ri = 0; ri < kRW; ++ri)
        myDm[ri] = !BWD || wr0 + ri >= b.n_rows ? 0.0f : b.dmax ? b.dmax[wr0 + ri] : FLT_MAX;  // no bound: flag all
    bool alive = true;
    // First pass over nA stages: per-lane minimum per problem.  Backward takes
    // the exact distance; forward takes a = fl(t*t + D) (one FMA), which is at
    // most 3 ulp below the exact d = fl(D + fl(t*t)) for D >= 0, so the bound
    // derived from it is widened by 2^-20 relative (see fwd_bound).
    // For k_max > 32 each lane keeps two minima (its even and its odd columns),
    // 64 values from distinct columns.
    if (seeded) {
        // bounds from the seed columns, computed by k_seed_bounds
        if (lane < kP) {
            const int p = lane;
            float th = -1.0f;  // padded problem: never passes
            if ((okmask >> p) & 1u) {
                const float T = b.bound[(size_t)S.srcand[wc + p % kCW] * b.n_rows + wr0 + p / kCW];
                th = T < FLT_MAX ? T : 0x1.fffffcp+127f;  // inclusive; FLT_MAX itself never enters
            }
            myT[p] = th;
        }
        __syncwarp();
    } else {
        float mn[kP], mn2[kP];  // mn2: LONG only
#pragma unroll
        for (int p = 0; p < kP; ++p) mn[p] = mn2[p] = INFINITY;
        for (int v = 0; v < nA && alive; ++v) {
            const int s = v % ring;
            if (!__all_sync(kFull, mbar_wait(S.full + s, (v / ring) & 1))) {  // warp-uniform: collectives follow
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
                            const float2 t = sub2(xv2[p], xp[ci]);
                            float2 e;
                            if constexpr (BWD) e = sub2(dp[ri], sq2(t));
                            else e = fma2(t, t, dp[ri]);
                            if constexpr (LONG) {
                                mn[p] = fminf(mn[p], e.x);
                                mn2[p] = fminf(mn2[p], e.y);
                            } else {
                                mn[p] = min3f(mn[p], e.x, e.y);
                            }
                        }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(S.empty + s);
        }
        // T = k-th smallest of the 32 (64) lane minima: k distinct columns lie at or below it
#pragma unroll
        for (int p = 0; p < kP; ++p) {
            float T;
            if constexpr (LONG) {
                // both halves sorted, the second reversed: element-wise min / max split
                // the 64 values into the 32 smallest and the 32 largest
                const float a = warp_sort32(mn[p], lane);
                const float bz = __shfl_sync(kFull, warp_sort32(mn2[p], lane), 31 - lane);
                const float lo = warp_sort32(fminf(a, bz), lane), hi = warp_sort32(fmaxf(a, bz), lane);
                T = K <= 32 ? __shfl_sync(kFull, lo, (K - 1) & 31) : __shfl_sync(kFull, hi, (K - 33) & 31);
            } else {
                const float srt = warp_sort32(mn[p], lane);
                T = __shfl_sync(kFull, srt, K - 1);
            }
            float th;
            if constexpr (BWD) {
                float Tb = T;
                if (reuse) {  // k distinct columns were at or below it last step and have not grown
                    const int r = wr0 + p / kCW;
                    Tb = r < b.n_rows ? b.kth_prev[(size_t)S.srcand[wc + p % kCW] * b.n_rows + r] : T;
                }
                th = Tb < FLT_MAX ? Tb : nextafterf(FLT_MAX, 0.0f);  // inclusive bound
            }
            else th = (okmask >> p) & 1u ? fwd_bound(T) : -1.0f;                // padded: never passes
            if (lane == 0) myT[p] = th;
        }
        __syncwarp();
    }

    {
        // Full pass through a conservative filter.  Per scored row the warp
        // keeps H = the largest filter bound of its four problems.  Forward: a
        // column can pass (d <= threshold) only if u = fl(t*t + fl(D - H)) < 0,
        // so the sign bits are ORed.  Backward (d = D - t*t): only if
        // u = fl(t*t + fl(H - D)) >= 0, so the sign bits are ANDed and a clear
        // bit flags the row.  The hot loop costs one sub and one FMA per
        // evaluation; a flagged row is re-scored with the reference's rounding.
        float2 H2[kRW];
        auto row_H = [&](int ri) {
            float h = -INFINITY;
#pragma unroll
            for (int ci = 0; ci < kCW; ++ci) {
                const float T = myT[ri * kCW + ci];
                h = fmaxf(h, BWD ? filter_bound_bwd(T, myDm[ri]) : filter_bound(T));
            }
            return make_float2(h, h);
        };
#pragma unroll
        for (int ri = 0; ri < kRW; ++ri) H2[ri] = row_H(ri);
        for (int v = nA; v < nvirt && alive; ++v) {
            const int s = v % ring;
            if (!__all_sync(kFull, mbar_wait(S.full + s, (v / ring) & 1))) {  // warp-uniform: collectives follow
                alive = false;
                break;
            }
            const int i0 = (v - nA) * kSC;
            const float *D_s = S.Ds + (s * kRowsB + rg * kRW) * kSC;
            const float *X_s = S.Xs + (s * kCandB + wc) * kSC;
            const float *D_w = D_s + 2 * lane;
            const float *X_w = X_s + 2 * lane;
            if (wvalid) {
                const int nch = min(kSC, b.ldc - i0) / kChunk;  // ldc is a multiple of kChunk
#pragma unroll 1
                for (int q = 0; q < kSC / kChunk; ++q) {
                    if (q >= nch) break;
                    const int q0 = q * kChunk;
                    float2 dp[kRW], E[kRW], xp[kCW];
#pragma unroll
                    for (int ri = 0; ri < kRW; ++ri) {
                        dp[ri] = *reinterpret_cast<const float2 *>(D_w + ri * kSC + q0);
                        E[ri] = BWD ? sub2(H2[ri], dp[ri]) : sub2(dp[ri], H2[ri]);
                    }
                    if constexpr (!BWD) {
                        // Forward, d = fl(D + fl(t*t)) >= D: a column passes only if
                        // D <= T < H, i.e. fl(D - H) < 0 for one of the warp's rows.
                        unsigned a = 0u;
#pragma unroll
                        for (int ri = 0; ri < kRW; ++ri) a |= f2u(E[ri].x) | f2u(E[ri].y);
                        if (!__any_sync(kFull, (int)a < 0)) continue;
                    }
#pragma unroll
                    for (int ci = 0; ci < kCW; ++ci) xp[ci] = *reinterpret_cast<const float2 *>(X_w + ci * kSC + q0);
                    unsigned acc[kRW];
#pragma unroll
                    for (int ri = 0; ri < kRW; ++ri) {
                        float2 u[kCW];
#pragma unroll
                        for (int ci = 0; ci < kCW; ++ci) {
                            const float2 t = sub2(xv2[ri * kCW + ci], xp[ci]);
                            u[ci] = fma2(t, t, E[ri]);
                        }
                        if constexpr (BWD)
                            acc[ri] = (f2u(u[0].x) & f2u(u[0].y) & f2u(u[1].x)) & (f2u(u[1].y) & f2u(u[2].x) & f2u(u[2].y)) &
                                      (f2u(u[3].x) & f2u(u[3].y));
                        else
                            acc[ri] = (f2u(u[0].x) | f2u(u[0].y) | f2u(u[1].x)) | (f2u(u[1].y) | f2u(u[2].x) | f2u(u[2].y)) |
                                      (f2u(u[3].x) | f2u(u[3].y));
                    }
                    const unsigned all = BWD ? ((acc[0] & acc[1]) & (acc[2] & acc[3])) : ((acc[0] | acc[1]) | (acc[2] | acc[3]));
                    if (__any_sync(kFull, BWD ? (int)all >= 0 : (int)all < 0)) {
                        unsigned pm = 0u;  // bit 2p+h: column 2*lane+h passes problem p exactly
                        int nfl = 0;
#pragma unroll
                        for (int ri = 0; ri < kRW; ++ri) {
                            if (__any_sync(kFull, BWD ? (int)acc[ri] >= 0 : (int)acc[ri] < 0)) {
                                if constexpr (COUNT) ++nfl;
#pragma unroll
                                for (int ci = 0; ci < kCW; ++ci) {
                                    const int p = ri * kCW + ci;
                                    const float th = myT[p];
                                    const float2 s2 = sq2(sub2(xv2[p], xp[ci]));
                                    const float2 e = BWD ? sub2(dp[ri], s2) : add2(dp[ri], s2);
                                    pm |= (le_mask(e.x, th) & (1u << (2 * p))) | (le_mask(e.y, th) & (2u << (2 * p)));
                                }
                            }
                        }
                        if constexpr (COUNT) {
                            const unsigned pmw = __reduce_or_sync(kFull, pm);
                            if (lane == 0) {
                                unsigned rp = 0u;  // rows holding a pass
#pragma unroll
                                for (int ri = 0; ri < kRW; ++ri) rp |= ((pmw >> (8 * ri)) & 0xffu) ? (1u << ri) : 0u;
                                myCnt[0] += nfl;
                                myCnt[1] += __popc(rp);
                            }
                        }
                        if (__any_sync(kFull, pm != 0u)) {
                            const unsigned rows =
                                insert_chunk<BWD, KL>(pm, D_s, X_s, myX, myL, myI, myT, q0, i0 + q0, K);
#pragma unroll
                            for (int ri = 0; ri < kRW; ++ri)
                                if ((rows >> ri) & 1u) H2[ri] = row_H(ri);
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(S.empty + s);
        }
    }
    if (COUNT && wvalid && lane == 0) {
        atomicAdd(b.fcount + 0, (unsigned long long)kRW * (unsigned long long)(b.ldc / kChunk));
        atomicAdd(b.fcount + 1, (unsigned long long)myCnt[0]);
        atomicAdd(b.fcount + 2, (unsigned long long)myCnt[1]);
    }
    if (!alive) {
        if (lane == 0) {
            atomicExch(&b.st->error, kErrTimeout);
            atomicExch(&b.st->done, 1);
        }
        return;
    }
    if (!wvalid) return;

    // Epilogue: the k-th distances for the next backward step, the optional
    // neighbour dump, then labels gathered by all lanes and summed in rank
    // order (sequential FP32, as the reference) by lane p.
    if (BWD && b.kth_prev && lane < kP && ((okmask >> lane) & 1u)) {
        const int p = lane;
        b.kth_prev[(size_t)S.srcand[wc + p % kCW] * b.n_rows + wr0 + p / kCW] = myL[p * KL + K - 1];
    }
    if (b.nn_idx) {
        for (int p = 0; p < kP; ++p) {
            const int r = wr0 + p / kCW;
            const int slot = c0 + wc + p % kCW;
            if (!((okmask >> p) & 1u)) continue;
            const size_t o = ((size_t)slot * b.n_rows + r) * K;
            for (int x = lane; x < K; x += 32) {
                b.nn_idx[o + x] = myI[p * KL + x];
                b.nn_dist[o + x] = myL[p * KL + x];
            }
        }
        __syncwarp();
    }
    for (int e = lane; e < kP * K; e += 32) {
        const int p = e / K, j = e - p * K;
        if ((okmask >> p) & 1u) myL[p * KL + j] = __ldg(b.yc + myI[p * KL + j]);
    }
    __syncwarp();
    if (lane < kP && ((okmask >> lane) & 1u)) {
        const int p = lane;
        const int r = wr0 + p / kCW;
        const int slot = c0 + wc + p % kCW;
        const int nk = b.nk;
        float acc = 0.0f;
        for (int j = 0; j < K; ++j) {
            acc = __fadd_rn(acc, myL[p * KL + j]);
            for (int m = 0; m < nk; ++m) {
                const int k = __ldg(b.kvals + m);
                if (k == j + 1) b.pred[((size_t)slot * nk + m) * b.n_rows + r] = __fdiv_rn(acc, (float)k);
            }
        }
    }
}

size_t tma_smem_bytes(int K, int ring, int RG, int CG)
{
    const int KL = list_slots(K);
    const int kRowsB = RG * kRW, kCandB = CG * kCW, kConsumers = RG * CG;
    return kBarBytes + sizeof(float) * (size_t)ring * (kRowsB + kCandB) * kSC +
           (sizeof(float) + sizeof(int)) * (size_t)kConsumers * kP * KL + 2 * sizeof(float) * kConsumers * kP +
           sizeof(int) * (kCandB + 1 + 2 * kConsumers);
}

}  // namespace

bool score_tma_supported(int kmax) { return kmax >= 1 && kmax <= 64; }

namespace {

PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        cudaGetLastError();
    });
    return fn;
}

// Row-major FP32 matrix [rows][ld] (ld a multiple of 4, base 16-byte aligned)
// as a 2-D tensor map with a box of box_rows x kSC; out-of-range reads give 0.
bool encode_rows(CUtensorMap *m, const float *base, int ld, long long rows, int box_rows)
{
    const PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || (reinterpret_cast<uintptr_t>(base) & 15u) || ld % 4) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)ld, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
    const cuuint32_t box[2] = {(cuuint32_t)kSC, (cuuint32_t)box_rows};
    const cuuint32_t estr[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

namespace {

// One launch over candidate slots [slot0, slot0 + n_slots) of the step's n_cand.
template <bool BWD, bool COUNT, int RING, int RG, int CG, int KL>
cudaError_t launch_shape(const Bufs &b, int n_cand, int slot0, int n_slots, int max_smem, cudaStream_t s)
{
    constexpr int kRowsB = RG * kRW, kCandB = CG * kCW;
    const int n_cg = (n_slots + kCandB - 1) / kCandB;
    const long long blocks = (long long)((b.n_rows + kRowsB - 1) / kRowsB) * n_cg;
    if (blocks > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    CUtensorMap tmD, tmX;
    if (!encode_rows(&tmD, b.D, b.ldc, b.n_rows, kRowsB) || !encode_rows(&tmX, b.XT, b.ldc, b.p, 1))
        return cudaErrorInvalidValue;
    const size_t smem = tma_smem_bytes(b.kmax, RING, RG, CG);
    if (smem > (size_t)max_smem) return cudaErrorInvalidConfiguration;
    if (list_slots(b.kmax) != KL) return cudaErrorInvalidValue;
    auto kern = k_score_tma<BWD, RING, COUNT, RG, CG, KL>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<(unsigned)blocks, (RG * CG + 1) * 32, smem, s>>>(b, n_cand, n_cg, slot0, tmD, tmX);
    return cudaGetLastError();
}

// With 16-slot lists the remainder of n_cand over 12-candidate groups (1 to 8
// candidates) gets its own launch with fewer candidates and more rows per
// block, so that no block holds idle candidate warps (a block takes as long as
// its busiest warp, so a block with one of three candidate warps busy costs
// about as much as a full one).  Returns 0 (one launch) or the remainder
// blocks' candidate warps, 1 or 2.
int remainder_shape(int kmax, int n_cand, int)
{
    if (list_slots(kmax) != 16) return 0;
    const int rem = n_cand % 12;
    if (n_cand < 12 || rem == 0 || rem > 8) return 0;
    return rem <= 4 ? 1 : 2;  // candidate warps per block of the remainder launch
}

template <bool BWD, bool COUNT>
cudaError_t launch_k(const Bufs &b, int n_cand, int max_smem, cudaStream_t s)
{
    // 12-candidate blocks.  Forward with 16-slot lists: 12-row blocks with a
    // 3-slot ring, two blocks per SM (a block waits for its slowest warp, and
    // the other block's warps fill the gap; fwd-64k 376.8 -> 367.1 ms per
    // selection against one 24-row block); the remainder candidates in
    // 36-row x 4-candidate or 16-row x 8-candidate blocks.  Backward keeps one
    // 24-row block per SM with a 5-slot ring (bwd-50k 1710 against 1754 ms);
    // its remainder in 72-row x 4-candidate or 36-row x 8-candidate blocks.  32-slot
    // lists leave room for 4 slots, 64-slot lists (k <= 64) for 2 (measured on
    // k = 50: 19 warps with 2 slots beat 16 warps with 3 and 13 warps with 4).
    switch (list_slots(b.kmax)) {
    case 16:
        if constexpr (BWD) {
            const int rs = remainder_shape(b.kmax, n_cand, 1);
            if (rs == 0) return launch_shape<BWD, COUNT, kRingDeep, 6, 3, 16>(b, n_cand, 0, n_cand, max_smem, s);
            const int n_full = n_cand - n_cand % 12;
            cudaError_t e = launch_shape<BWD, COUNT, kRingDeep, 6, 3, 16>(b, n_cand, 0, n_full, max_smem, s);
            if (e != cudaSuccess) return e;
            if (rs == 1) return launch_shape<BWD, COUNT, 2, 18, 1, 16>(b, n_cand, n_full, n_cand - n_full, max_smem, s);
            return launch_shape<BWD, COUNT, 4, 9, 2, 16>(b, n_cand, n_full, n_cand - n_full, max_smem, s);
        } else {
            const int rs = remainder_shape(b.kmax, n_cand, 0);
            if (rs == 0) return launch_shape<BWD, COUNT, 3, 3, 3, 16>(b, n_cand, 0, n_cand, max_smem, s);
            const int n_full = n_cand - n_cand % 12;
            cudaError_t e = launch_shape<BWD, COUNT, 3, 3, 3, 16>(b, n_cand, 0, n_full, max_smem, s);
            if (e != cudaSuccess) return e;
            if (rs == 1) return launch_shape<BWD, COUNT, 2, 9, 1, 16>(b, n_cand, n_full, n_cand - n_full, max_smem, s);
            return launch_shape<BWD, COUNT, 3, 4, 2, 16>(b, n_cand, n_full, n_cand - n_full, max_smem, s);
        }
    case 32: return launch_shape<BWD, COUNT, kRingShallow, 6, 3, 32>(b, n_cand, 0, n_cand, max_smem, s);
    default: return launch_shape<BWD, COUNT, 2, 6, 3, 64>(b, n_cand, 0, n_cand, max_smem, s);
    }
}

}  // namespace

cudaError_t launch_seed_bounds(const Bufs &b, int n_cand, float *xrm, cudaStream_t s)
{
    const int grid = (b.n_rows + 7) / 8;
    if (b.kmax <= 16 && xrm) {
        k_candidates_rowmajor<<<dim3((b.n_cols + 31) / 32, (n_cand + 31) / 32), 256, 0, s>>>(b, n_cand, xrm);
        if (b.kmax <= 4) k_seed_bounds_exact<4><<<grid, 256, 0, s>>>(b, n_cand, xrm, b.bound);
        else if (b.kmax <= 8) k_seed_bounds_exact<8><<<grid, 256, 0, s>>>(b, n_cand, xrm, b.bound);
        else if (b.kmax <= 12) k_seed_bounds_exact<12><<<grid, 256, 0, s>>>(b, n_cand, xrm, b.bound);
        else k_seed_bounds_exact<16><<<grid, 256, 0, s>>>(b, n_cand, xrm, b.bound);
        return cudaGetLastError();
    }
    if (b.kmax > 16) k_seed_bounds<4><<<grid, 256, 0, s>>>(b, n_cand, b.bound);
    else k_seed_bounds<2><<<grid, 256, 0, s>>>(b, n_cand, b.bound);
    return cudaGetLastError();
}

int score_tma_launches(int kmax, int n_cand, int backward) { return remainder_shape(kmax, n_cand, backward) ? 2 : 1; }

cudaError_t launch_score_tma(const Bufs &b, int n_cand, int backward, cudaStream_t s)
{
    int dev = 0, max_smem = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&max_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    // the counting variants are separate instantiations: the default code has no counting at all
    const bool cnt = b.fcount != nullptr;
    if (backward) return cnt ? launch_k<true, true>(b, n_cand, max_smem, s) : launch_k<true, false>(b, n_cand, max_smem, s);
    return cnt ? launch_k<false, true>(b, n_cand, max_smem, s) : launch_k<false, false>(b, n_cand, max_smem, s);
}

}  // namespace snn
