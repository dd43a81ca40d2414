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
// The second step walks the first winner's sorted values the same way
// (k_second_step below).
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
// Ascending bitonic sort of one 64-bit key per lane over the warp.
__device__ __forceinline__ unsigned long long warp_sort64(unsigned long long key, int lane)
{
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, j);
            const bool keep_min = ((lane & j) == 0) == ((lane & k) == 0);
            key = keep_min ? (o < key ? o : key) : (o > key ? o : key);
        }
    }
    return key;
}

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

// k_second_step: the second forward step of a holdout problem.  With one
// feature w committed, D[r][i] = fl(fl(x_r,w - x_i,w)^2) is one-dimensional
// again: walking w's sorted values outwards from x_r,w visits each side's
// columns in increasing D.  Candidate c's distance
// d = fl(D + fl((x_r,c - x_i,c)^2)) is at least D, so a side is finished once
// its next D exceeds the k-th distance of the list held so far.  One warp per
// (candidate, row): each iteration lanes 0-15 take the next 16 columns on the
// left, lanes 16-31 the next 16 on the right (all 32 lanes the open side once
// the other is finished); columns whose D already exceeds
// the k-th distance are skipped, and the few that pass are inserted into
// a register-held list (lane j holds entry j; k_second_step_long below keeps
// k in (32, 64]) sorted
// by (distance, index) -- columns arrive out of index order, and that order
// is the reference's stable one.  D is recomputed from the sorted values (the
// commit's rounding), not read from memory, and the candidates' values come
// from xs, X's candidate rows put in w's sorted column order beforehand
// (k_gather_sorted), so every load of the walk is contiguous and none waits
// for another.
//
// Walks are usually short (on the fwd-64k data a median of ~1,000 columns of
// 65,536, ~32 iterations) but not bounded: a warp adds its columns to a
// global count every 64 iterations, and once the count passes `budget` (an
// eighth of a full scan) the kernel raises State::full_scan and every warp
// leaves; the step's regular scoring launch then scans everything.
// xs[slot][j] = X[c][i_j] for the step's candidates c = cands[slot] and w's
// sorted columns i_j (w = the first step's winner).
__global__ void __launch_bounds__(256) k_gather_sorted(Bufs b, const int *si, float *xs, int n_cand)
{
    if (b.st->done) return;
    const int slot = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= n_cand || j >= b.n_cols) return;
    const int w = b.st->winner;
    const int c = b.cands[slot];
    xs[(size_t)slot * b.ldc + j] = __ldg(b.XT + (size_t)c * b.ldc + __ldg(si + (size_t)w * b.ldc + j));
}

__global__ void __launch_bounds__(256, 8) k_second_step(Bufs b, const float *sv, const int *si, const float *xs,
                                                     int n_cand, unsigned long long *walked,
                                                     unsigned long long budget)
{
    constexpr unsigned kFull = 0xffffffffu;
    if (b.st->done) return;
    const int lane = threadIdx.x & 31;
    const int slot = blockIdx.y;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (slot >= n_cand || r >= b.n_rows) return;  // warp-uniform
    const int K = b.kmax;
    const int n = b.n_cols;
    const int w = b.st->winner;
    const int c = b.cands[slot];
    const float aw = b.XV[(size_t)w * b.ldr + r];
    const float ac = b.XV[(size_t)c * b.ldr + r];
    const float *bv = sv + (size_t)w * b.ldc;
    const int *bi = si + (size_t)w * b.ldc;
    const float *xsc = xs + (size_t)slot * b.ldc;

    // the list: entry e (e < cnt) at lane e
    float L0 = INFINITY;
    int I0 = 0x7fffffff;
    int cnt = 0;
    float th = INFINITY;  // the k-th entry once the list is full
    int thi = 0x7fffffff;
    // non-finite x_r,w or x_r,c: no distance below FLT_MAX, the list stays padding
    if (isfinite(aw) && isfinite(ac)) {
        int lo = 0, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (bv[mid] < aw) lo = mid + 1;
            else hi = mid;
        }
        int ln = lo - 1, rn = lo;  // next unvisited position on each side
        bool ldone = ln < 0, rdone = rn >= n;
        for (int it = 1; !(ldone && rdone); ++it) {
            if ((it & 63) == 0) {  // account for the walk; leave when the budget is spent
                int stop = 0;
                if (lane == 0) {
                    const unsigned long long tot = atomicAdd(walked, 64ull * 32ull) + 64ull * 32ull;
                    if (tot > budget) atomicExch(&b.st->full_scan, 1);
                    stop = tot > budget || *(volatile int *)&b.st->full_scan;
                }
                if (__shfl_sync(kFull, stop, 0)) return;
            }
            // 16 columns per side, or all 32 lanes on the side still open
            const int nl = ldone ? 0 : (rdone ? 32 : 16);
            const bool left = lane < nl;
            const int j = left ? ln - lane : rn + (lane - nl);
            const bool in = left ? j >= 0 : (!rdone && j < n);
            // the three loads are independent (and contiguous across the lanes)
            const float vj = in ? bv[j] : 0.0f, xj = in ? xsc[j] : 0.0f;
            const int ij = in ? bi[j] : 0x7fffffff;
            const float D = in ? dist1(aw, vj) : INFINITY;
            float d = INFINITY;
            int i = 0x7fffffff;
            if (in && D <= th) {  // d >= D: beyond the k-th distance nothing enters
                i = ij;
                const float t = __fsub_rn(ac, xj);
                d = __fadd_rn(D, __fmul_rn(t, t));
            }
            const bool fill = cnt == 0;
            if (fill) {
                // the first batch fills the empty list at once: its finite distances
                // sorted by (distance, index) (distances are >= +0, so their bits
                // order like the values), the first K kept
                const unsigned long long key =
                    d < FLT_MAX ? ((unsigned long long)__float_as_uint(d) << 32) | (unsigned)i : ~0ull;
                const unsigned long long srt = warp_sort64(key, lane);
                cnt = min(__popc(__ballot_sync(kFull, d < FLT_MAX)), K);
                if (lane < cnt) {
                    L0 = __uint_as_float((unsigned)(srt >> 32));
                    I0 = (int)(unsigned)(srt & 0xffffffffu);
                }
                if (cnt == K) {  // K <= 32 here
                    th = __shfl_sync(kFull, L0, (K - 1) & 31);
                    thi = __shfl_sync(kFull, I0, (K - 1) & 31);
                }
            }
            unsigned m = fill ? 0u : __ballot_sync(kFull, d < FLT_MAX && (d < th || (d == th && i < thi)));
            while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                const float dv = __shfl_sync(kFull, d, l);
                const int iv = __shfl_sync(kFull, i, l);
                if (!(dv < th || (dv == th && iv < thi))) continue;  // the list tightened meanwhile
                // position: entries ordered before (dv, iv)
                const int pos = __popc(__ballot_sync(kFull, lane < cnt && (L0 < dv || (L0 == dv && I0 < iv))));
                const float up0 = __shfl_up_sync(kFull, L0, 1);
                const int upi0 = __shfl_up_sync(kFull, I0, 1);
                if (lane == pos) {
                    L0 = dv;
                    I0 = iv;
                } else if (lane > pos && lane < K) {
                    L0 = up0;
                    I0 = upi0;
                }
                if (cnt < K) ++cnt;
                if (cnt == K) {
                    th = __shfl_sync(kFull, L0, K - 1);
                    thi = __shfl_sync(kFull, I0, K - 1);
                }
            }
            // a side is finished past its end or once its farthest D of this batch exceeds the k-th
            const float dl_far = __shfl_sync(kFull, D, nl > 0 ? nl - 1 : 0), dr_far = __shfl_sync(kFull, D, 31);
            ln -= nl;
            rn += 32 - nl;
            ldone = ldone || ln < 0 || (nl > 0 && dl_far > th);
            rdone = rdone || rn >= n || (nl < 32 && dr_far > th);
        }
    }
    // entries past cnt are padding (FLT_MAX, 0)
    if (lane >= cnt) {
        L0 = FLT_MAX;
        I0 = 0;
    }
    if (b.nn_idx) {
        const size_t o = ((size_t)slot * b.n_rows + r) * K;
        if (lane < K) {
            b.nn_idx[o + lane] = I0;
            b.nn_dist[o + lane] = L0;
        }
    }
    // labels summed in rank order (sequential FP32) by lane 0, as the scoring kernels
    const float y0 = lane < K ? __ldg(b.yc + I0) : 0.0f;
    float acc = 0.0f;
    for (int e = 0; e < K; ++e) {
        const float ye = __shfl_sync(kFull, y0, e);
        acc = __fadd_rn(acc, ye);
        if (lane == 0)
            for (int m = 0; m < b.nk; ++m) {
                const int k = __ldg(b.kvals + m);
                if (k == e + 1) b.pred[((size_t)slot * b.nk + m) * b.n_rows + r] = __fdiv_rn(acc, (float)k);
            }
    }
}


// Ascending bitonic sort of 64 keys over the warp, two per lane: lane l ends
// with elements 2l and 2l+1.
__device__ __forceinline__ void warp_sort64x2(unsigned long long (&v)[2], int lane)
{
#pragma unroll
    for (int k = 2; k <= 64; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 2) {  // partner in lane ^ (j / 2), same slot
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const unsigned long long o = __shfl_xor_sync(0xffffffffu, v[h], j >> 1);
                    const int i = 2 * lane + h;
                    v[h] = (((i & j) == 0) == ((i & k) == 0)) ? min(v[h], o) : max(v[h], o);
                }
            } else {  // partner in the same lane
                const bool up = ((2 * lane) & k) == 0;
                const unsigned long long a = v[0], c = v[1];
                v[0] = up ? min(a, c) : max(a, c);
                v[1] = up ? max(a, c) : min(a, c);
            }
        }
    }
}

// k_second_step_long: the walk of k_second_step for 32 < k <= 64.  The list
// sits as adjacent pairs (lane j holds entries 2j and 2j+1), so an insertion
// shifts it with one shuffle per array; and the first 64 columns (32 per side,
// or 64 on the side still open) are read together and sorted into the list at
// once, so with k finite distances among them the list is full -- and the
// walk's sides can finish -- from the first batch on.
__global__ void __launch_bounds__(256, 8) k_second_step_long(Bufs b, const float *sv, const int *si, const float *xs,
                                                          int n_cand, unsigned long long *walked,
                                                          unsigned long long budget)
{
    constexpr unsigned kFull = 0xffffffffu;
    if (b.st->done) return;
    const int lane = threadIdx.x & 31;
    const int slot = blockIdx.y;
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (slot >= n_cand || r >= b.n_rows) return;  // warp-uniform
    const int K = b.kmax;
    const int n = b.n_cols;
    const int w = b.st->winner;
    const int c = b.cands[slot];
    const float aw = b.XV[(size_t)w * b.ldr + r];
    const float ac = b.XV[(size_t)c * b.ldr + r];
    const float *bv = sv + (size_t)w * b.ldc;
    const int *bi = si + (size_t)w * b.ldc;
    const float *xsc = xs + (size_t)slot * b.ldc;
    // the list: entries e0 = 2 * lane and e0 + 1 (valid below cnt)
    const int e0 = 2 * lane;
    float2 Lv = make_float2(INFINITY, INFINITY);
    int2 Iv = make_int2(0x7fffffff, 0x7fffffff);
    int cnt = 0;
    float th = INFINITY;  // the k-th entry once the list is full
    int thi = 0x7fffffff;
    // non-finite x_r,w or x_r,c: no distance below FLT_MAX, the list stays padding
    if (isfinite(aw) && isfinite(ac)) {
        int lo = 0, hi = n;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (bv[mid] < aw) lo = mid + 1;
            else hi = mid;
        }
        int ln = lo - 1, rn = lo;  // next unvisited position on each side
        bool ldone = ln < 0, rdone = rn >= n;
        // batch position q: the left side's (q+1)-th next column for q < nl, else the right side's
        auto visit = [&](int q, int nl, float &D, float &d, int &i) {
            const bool left = q < nl;
            const int j = left ? ln - q : rn + (q - nl);
            const bool in = left ? j >= 0 : (!rdone && j < n);
            // the three loads are independent (and contiguous across the lanes)
            const float vj = in ? bv[j] : 0.0f, xj = in ? xsc[j] : 0.0f;
            const int ij = in ? bi[j] : 0x7fffffff;
            D = in ? dist1(aw, vj) : INFINITY;
            d = INFINITY;
            i = 0x7fffffff;
            if (in && D <= th) {  // d >= D: beyond the k-th distance nothing enters
                i = ij;
                const float t = __fsub_rn(ac, xj);
                d = __fadd_rn(D, __fmul_rn(t, t));
            }
        };
        if (!(ldone && rdone)) {
            // first batch, 64 columns: their finite distances sorted by (distance, index)
            // (distances are >= +0, so their bits order like the values), the first K kept
            const int nl = ldone ? 0 : (rdone ? 64 : 32);
            float Da, da, Db, db;
            int ia, ib;
            visit(lane, nl, Da, da, ia);
            visit(lane + 32, nl, Db, db, ib);
            unsigned long long kk[2] = {
                da < FLT_MAX ? ((unsigned long long)__float_as_uint(da) << 32) | (unsigned)ia : ~0ull,
                db < FLT_MAX ? ((unsigned long long)__float_as_uint(db) << 32) | (unsigned)ib : ~0ull};
            cnt = min(__popc(__ballot_sync(kFull, da < FLT_MAX)) + __popc(__ballot_sync(kFull, db < FLT_MAX)), K);
            warp_sort64x2(kk, lane);
            if (e0 < cnt) {
                Lv.x = __uint_as_float((unsigned)(kk[0] >> 32));
                Iv.x = (int)(unsigned)(kk[0] & 0xffffffffu);
            }
            if (e0 + 1 < cnt) {
                Lv.y = __uint_as_float((unsigned)(kk[1] >> 32));
                Iv.y = (int)(unsigned)(kk[1] & 0xffffffffu);
            }
            if (cnt == K) {
                th = __shfl_sync(kFull, ((K - 1) & 1) ? Lv.y : Lv.x, (K - 1) >> 1);
                thi = __shfl_sync(kFull, ((K - 1) & 1) ? Iv.y : Iv.x, (K - 1) >> 1);
            }
            // a side is finished past its end or once its farthest D of the batch exceeds the k-th
            const int ql = nl > 0 ? nl - 1 : 0;
            const float dl_far = __shfl_sync(kFull, ql < 32 ? Da : Db, ql & 31);
            const float dr_far = __shfl_sync(kFull, Db, 31);
            ln -= nl;
            rn += 64 - nl;
            ldone = ldone || ln < 0 || (nl > 0 && dl_far > th);
            rdone = rdone || rn >= n || (nl < 64 && dr_far > th);
        }
        for (int it = 1; !(ldone && rdone); ++it) {
            if ((it & 63) == 0) {  // account for the walk; leave when the budget is spent
                int stop = 0;
                if (lane == 0) {
                    const unsigned long long tot = atomicAdd(walked, 64ull * 32ull) + 64ull * 32ull;
                    if (tot > budget) atomicExch(&b.st->full_scan, 1);
                    stop = tot > budget || *(volatile int *)&b.st->full_scan;
                }
                if (__shfl_sync(kFull, stop, 0)) return;
            }
            // 16 columns per side, or all 32 lanes on the side still open
            const int nl = ldone ? 0 : (rdone ? 32 : 16);
            float D, d;
            int i;
            visit(lane, nl, D, d, i);
            unsigned m = __ballot_sync(kFull, d < FLT_MAX && (d < th || (d == th && i < thi)));
            while (m) {
                const int l = __ffs(m) - 1;
                m &= m - 1;
                const float dv = __shfl_sync(kFull, d, l);
                const int iv = __shfl_sync(kFull, i, l);
                if (!(dv < th || (dv == th && iv < thi))) continue;  // the list tightened meanwhile
                // position: entries ordered before (dv, iv)
                const int pos = __popc(__ballot_sync(kFull, e0 < cnt && (Lv.x < dv || (Lv.x == dv && Iv.x < iv)))) +
                                __popc(__ballot_sync(kFull, e0 + 1 < cnt && (Lv.y < dv || (Lv.y == dv && Iv.y < iv))));
                const float pL = __shfl_up_sync(kFull, Lv.y, 1);  // entry 2j - 1
                const int pI = __shfl_up_sync(kFull, Iv.y, 1);
                // entry 2j + 1 first: it may take the old entry 2j
                if (e0 + 1 == pos) {
                    Lv.y = dv;
                    Iv.y = iv;
                } else if (e0 + 1 > pos && e0 + 1 < K) {
                    Lv.y = Lv.x;
                    Iv.y = Iv.x;
                }
                if (e0 == pos) {
                    Lv.x = dv;
                    Iv.x = iv;
                } else if (e0 > pos && e0 < K) {
                    Lv.x = pL;
                    Iv.x = pI;
                }
                if (cnt < K) ++cnt;
                if (cnt == K) {
                    th = __shfl_sync(kFull, ((K - 1) & 1) ? Lv.y : Lv.x, (K - 1) >> 1);
                    thi = __shfl_sync(kFull, ((K - 1) & 1) ? Iv.y : Iv.x, (K - 1) >> 1);
                }
            }
            // a side is finished past its end or once its farthest D of this batch exceeds the k-th
            const float dl_far = __shfl_sync(kFull, D, nl > 0 ? nl - 1 : 0), dr_far = __shfl_sync(kFull, D, 31);
            ln -= nl;
            rn += 32 - nl;
            ldone = ldone || ln < 0 || (nl > 0 && dl_far > th);
            rdone = rdone || rn >= n || (nl < 32 && dr_far > th);
        }
    }
    // entries past cnt are padding (FLT_MAX, 0)
    if (e0 >= cnt) {
        Lv.x = FLT_MAX;
        Iv.x = 0;
    }
    if (e0 + 1 >= cnt) {
        Lv.y = FLT_MAX;
        Iv.y = 0;
    }
    if (b.nn_idx) {
        const size_t o = ((size_t)slot * b.n_rows + r) * K;
        if (e0 < K) {
            b.nn_idx[o + e0] = Iv.x;
            b.nn_dist[o + e0] = Lv.x;
        }
        if (e0 + 1 < K) {
            b.nn_idx[o + e0 + 1] = Iv.y;
            b.nn_dist[o + e0 + 1] = Lv.y;
        }
    }
    // labels summed in rank order (sequential FP32) by lane 0, as the scoring kernels
    const float y0 = e0 < K ? __ldg(b.yc + Iv.x) : 0.0f;
    const float y1 = e0 + 1 < K ? __ldg(b.yc + Iv.y) : 0.0f;
    float acc = 0.0f;
    for (int e = 0; e < K; ++e) {
        const float ye = __shfl_sync(kFull, (e & 1) ? y1 : y0, e >> 1);
        acc = __fadd_rn(acc, ye);
        if (lane == 0)
            for (int m = 0; m < b.nk; ++m) {
                const int k = __ldg(b.kvals + m);
                if (k == e + 1) b.pred[((size_t)slot * b.nk + m) * b.n_rows + r] = __fdiv_rn(acc, (float)k);
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

cudaError_t launch_second_step(const Bufs &b, const float *sv, const int *si, float *xs, int n_cand,
                               unsigned long long *walked, cudaStream_t s)
{
    cudaError_t e = cudaMemsetAsync(walked, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    k_gather_sorted<<<dim3((b.n_cols + 255) / 256, n_cand), 256, 0, s>>>(b, si, xs, n_cand);
    const unsigned long long budget = (unsigned long long)b.n_rows * (unsigned long long)n_cand * b.n_cols / 8;
    const dim3 grid((b.n_rows + 7) / 8, n_cand);  // a warp per (candidate, row)
    if (b.kmax <= 32) k_second_step<<<grid, 256, 0, s>>>(b, sv, si, xs, n_cand, walked, budget);
    else if (b.kmax <= 64) k_second_step_long<<<grid, 256, 0, s>>>(b, sv, si, xs, n_cand, walked, budget);
    else return cudaErrorInvalidValue;  // k above 64 scans
    return cudaGetLastError();
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
