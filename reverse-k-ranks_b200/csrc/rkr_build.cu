// rkr_build.cu -- index build on the device: score rows, sampled thresholds, query-rank distribution.
//
// The reference sorts every user's full score row and then reads a few positions
// (ComputeScoreTableBatch + SampleSearch::LoopPreprocess, bsibc; QueryRankCPU + lower_bound, qdibc).
// Here a batch of users' rows is computed exactly (binary32, reference order) into device memory,
// and one CTA per row finds only what is asked for: it bins the row by value (bins are a
// monotone function of the score, so they keep the order), scatters it into bin order, and sorts
// only the bins that contain a requested position.  The row is never sorted as a whole unless a
// full sort is what the caller wants (rkr_score_sort_batch).
#include <algorithm>
#include <vector>

#include "rkr_internal.cuh"

namespace rkr {

constexpr int kBins = 4096;
constexpr int kSelThreads = 512;

// Score rows of users [u0, u0 + nu) against all items: rows[u - u0][i] = InnerProduct(user, item)
// (CPUScoreTable.hpp:372-386), stored with row stride ld.
__global__ void __launch_bounds__(kTileThreads) score_rows_kernel(const float *__restrict__ item, int64_t n_item,
                                                                 const float *__restrict__ user, int64_t u0, int64_t nu,
                                                                 int dim, float *__restrict__ rows, int64_t ld) {
    __shared__ TileSmem sm;
    const int64_t a0 = (int64_t) blockIdx.x * kTile;  // items
    const int64_t b0 = (int64_t) blockIdx.y * kTile;  // users (relative to u0)
    float lo[4][4], hi[4][4];
    exact_tile(sm, item, nullptr, n_item, dim, a0, user + u0 * dim, nu, dim, b0, 0, dim, dim, lo, hi);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int64_t u = b0 + 4 * ty + j;
        if (u >= nu) continue;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int64_t it = a0 + 4 * tx + i;
            if (it < n_item) rows[u * ld + it] = lo[i][j];
        }
    }
}

// score_rows on 128 x 128 tiles (items x users): rows[u - u0][i] = InnerProduct(user, item).
struct ScoreRowsEpi {
    static constexpr size_t kExtra = 0;
    float *rows;
    int64_t ld, n_item, n_rows;
    __device__ void prologue(char *, int64_t, int64_t) const {}
    __device__ bool active(char *, int64_t, int64_t) const { return true; }
    __device__ void finish(char *, const BigResult &res, int64_t a0, int64_t b0, bool) const {
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7;
        const int64_t it = a0 + ra;
        if (it >= n_item) return;
#pragma unroll 8
        for (int i = 0; i < kBig / 2; i++) {
            const int rb = half + 2 * i;
            if (b0 + rb >= n_rows) break;
            rows[(b0 + rb) * ld + it] = res.v[rb][ra];
        }
    }
};

// Ascending sort of up to 32 keys held one per lane (missing lanes hold +inf).
__device__ __forceinline__ float warp_sort32(float v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            const float o = __shfl_xor_sync(0xffffffffu, v, j);
            const bool up = (lane & k) == 0;
            const bool lower = (lane & j) == 0;
            v = (lower == up) ? fminf(v, o) : fmaxf(v, o);
        }
    return v;
}

// The l-th smallest value (0-based) of seg[0..n) for one warp; every lane returns it.
// Values are compared as floats (the reference sorts floats with std::greater; NaNs do not occur).
__device__ float warp_select(const float *seg, int n, int l) {
    const int lane = threadIdx.x & 31;
    if (n <= 32) {
        float v = lane < n ? seg[lane] : __int_as_float(0x7f800000);
        v = warp_sort32(v);
        return __shfl_sync(0xffffffffu, v, l);
    }
    float ans = 0.0f;
    bool found = false;
    for (int i0 = 0; i0 < n && !__any_sync(0xffffffffu, found); i0 += 32) {
        const int i = i0 + lane;
        if (i < n) {
            const float x = seg[i];
            int lt = 0, eq = 0;
            for (int t = 0; t < n; t++) {
                const float y = seg[t];
                lt += y < x;
                eq += y == x;
            }
            if (lt <= l && l < lt + eq) { ans = x; found = true; }
        }
    }
    const unsigned m = __ballot_sync(0xffffffffu, found);
    return __shfl_sync(0xffffffffu, ans, __ffs(m) - 1);
}

struct SelectArgs {
    const float *rows;       // [n_rows][ld]
    int64_t ld;
    int n_rows;
    int n_item;
    // thresholds
    const int32_t *sample_rank;  // [S] or nullptr
    int S;
    float *thr_out;          // [n_rows][S]
    // query-rank distribution
    const int32_t *sample_item;  // [n_si] or nullptr
    int n_si;
    int32_t *rank_hist;      // [n_si][n_item + 1], atomically incremented
    // full sort (descending) into sorted_out [n_rows][n_item] (or nullptr)
    float *sorted_out;
    // global scratch when the row does not fit in shared memory ([gridDim.x][2][n_item])
    float *gscratch;
    // rows to process (indices into rows), or nullptr for all n_rows
    const int32_t *row_list;
    int n_list;
};

__device__ __forceinline__ int value_bin(float x, float mn, float scale) {
    const int b = (int) __fmul_rn(__fsub_rn(x, mn), scale);
    return min(max(b, 0), kBins - 1);
}

// One CTA per row: bins, scatter, and the requested order statistics.
__global__ void __launch_bounds__(kSelThreads) row_select_kernel(SelectArgs a, int use_smem) {
    extern __shared__ float dyn[];
    __shared__ int hist[kBins];
    __shared__ int start[kBins + 1];
    __shared__ float red_mn[32], red_mx[32];
    __shared__ int warp_tot[32];
    const int n = a.n_item;
    float *vals, *buf;
    if (use_smem) {
        vals = dyn;
        buf = dyn + n;
    } else {
        vals = a.gscratch + (int64_t) blockIdx.x * 2 * n;
        buf = vals + n;
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int n_iter = a.row_list ? a.n_list : a.n_rows;
    for (int ri = blockIdx.x; ri < n_iter; ri += gridDim.x) {
        const int row = a.row_list ? a.row_list[ri] : ri;
        const float *src = a.rows + (int64_t) row * a.ld;
        float mn = __int_as_float(0x7f800000), mx = -mn;
        // the row in 16-byte loads, four per thread in flight before their values are stored (rows
        // start 16-byte aligned: ld is a multiple of 4)
        const float4 *src4 = reinterpret_cast<const float4 *>(src);
        const int n4 = n >> 2;
        for (int i0 = threadIdx.x; i0 < n4; i0 += 4 * blockDim.x) {
            float4 x[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int i = i0 + k * blockDim.x;
                if (i < n4) x[k] = __ldcs(src4 + i);
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int i = i0 + k * blockDim.x;
                if (i < n4) {
                    vals[4 * i] = x[k].x;
                    vals[4 * i + 1] = x[k].y;
                    vals[4 * i + 2] = x[k].z;
                    vals[4 * i + 3] = x[k].w;
                    mn = fminf(fminf(mn, x[k].x), fminf(fminf(x[k].y, x[k].z), x[k].w));
                    mx = fmaxf(fmaxf(mx, x[k].x), fmaxf(fmaxf(x[k].y, x[k].z), x[k].w));
                }
            }
        }
        for (int i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) {
            const float x = src[i];
            vals[i] = x;
            mn = fminf(mn, x);
            mx = fmaxf(mx, x);
        }
        for (int o = 16; o > 0; o >>= 1) {
            mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if (lane == 0) { red_mn[w] = mn; red_mx[w] = mx; }
        for (int b = threadIdx.x; b < kBins; b += blockDim.x) hist[b] = 0;
        __syncthreads();
        if (w == 0) {
            mn = lane < nw ? red_mn[lane] : __int_as_float(0x7f800000);
            mx = lane < nw ? red_mx[lane] : -__int_as_float(0x7f800000);
            for (int o = 16; o > 0; o >>= 1) {
                mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
            }
            if (lane == 0) { red_mn[0] = mn; red_mx[0] = mx; }
        }
        __syncthreads();
        mn = red_mn[0];
        mx = red_mx[0];
        const float range = __fsub_rn(mx, mn);
        const float scale = range > 0.0f ? __fdiv_rn((float) kBins, range) : 0.0f;
        for (int i = threadIdx.x; i < n; i += blockDim.x) atomicAdd(&hist[value_bin(vals[i], mn, scale)], 1);
        __syncthreads();
        // exclusive scan of hist into start (kBins / blockDim per thread)
        {
            const int per = kBins / kSelThreads;
            int loc[kBins / kSelThreads];
            int s = 0;
            for (int t = 0; t < per; t++) { loc[t] = s; s += hist[threadIdx.x * per + t]; }
            int incl = s;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (lane == 31) warp_tot[w] = incl;
            __syncthreads();
            if (w == 0) {
                const int v = lane < nw ? warp_tot[lane] : 0;
                int iv = v;
                for (int o = 1; o < 32; o <<= 1) {
                    const int x = __shfl_up_sync(0xffffffffu, iv, o);
                    if (lane >= o) iv += x;
                }
                if (lane < nw) warp_tot[lane] = iv - v;
            }
            __syncthreads();
            const int base = warp_tot[w] + incl - s;
            for (int t = 0; t < per; t++) {
                start[threadIdx.x * per + t] = base + loc[t];
                hist[threadIdx.x * per + t] = base + loc[t];  // scatter cursor
            }
            if (threadIdx.x == 0) start[kBins] = n;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const float x = vals[i];
            buf[atomicAdd(&hist[value_bin(x, mn, scale)], 1)] = x;
        }
        __syncthreads();
        // thresholds: position r (descending) is ascending position n - 1 - r
        if (a.thr_out) {
            for (int j = w; j < a.S; j += nw) {
                const int p = n - 1 - a.sample_rank[j];
                int lo = 0, len = kBins;  // last bin with start <= p
                while (len > 0) {
                    const int h = len >> 1, m = lo + h;
                    if (start[m + 1] <= p) { lo = m + 1; len -= h + 1; } else len = h;
                }
                const int b = lo;
                const float v = warp_select(buf + start[b], start[b + 1] - start[b], p - start[b]);
                if (lane == 0) a.thr_out[(int64_t) row * a.S + j] = v;
            }
        }
        // query ranks: number of items scoring strictly above each sampled item's score
        if (a.rank_hist) {
            for (int s = threadIdx.x; s < a.n_si; s += blockDim.x) {
                const float sv = vals[a.sample_item[s]];
                const int b = value_bin(sv, mn, scale);
                int cnt = n - start[b + 1];
                for (int t = start[b]; t < start[b + 1]; t++) cnt += buf[t] > sv;
                atomicAdd(&a.rank_hist[(int64_t) s * (n + 1) + cnt], 1);
            }
        }
        // full descending sort
        if (a.sorted_out) {
            float *dst = a.sorted_out + (int64_t) row * n;
            for (int b = w; b < kBins; b += nw) {
                const int s0 = start[b], nb = start[b + 1] - s0;
                if (nb == 0) continue;
                if (nb <= 32) {
                    float v = lane < nb ? buf[s0 + lane] : __int_as_float(0x7f800000);
                    v = warp_sort32(v);
                    if (lane < nb) dst[n - 1 - (s0 + lane)] = v;
                } else {
                    for (int i = lane; i < nb; i += 32) {
                        const float x = buf[s0 + i];
                        int lt = 0, eq_before = 0;
                        for (int t = 0; t < nb; t++) {
                            const float y = buf[s0 + t];
                            lt += y < x;
                            eq_before += (y == x) & (t < i);
                        }
                        dst[n - 1 - (s0 + lt + eq_before)] = x;
                    }
                }
            }
        }
        __syncthreads();
    }
}

// ---- the query-rank distribution's counting ------------------------------------------------------------
//
// ComputeQueryRankByComputation (QueryRankByComputation.hpp:122-242) needs, per user and sampled
// item, the number of items scoring strictly above the sampled item's score.  Per row: the sampled
// items' scores sorted descending (w), then one stream of the row in which every score x goes to
// bucket b(x) = #{k : w_k >= x} (a binary search in shared memory), counted per warp.  A score beats
// w_p exactly when b(x) <= p, so the rank of the sampled item at sorted position p is the number of
// scores in buckets 0 .. p.  No copy of the row, no value bins, one pass.
constexpr int kRankMaxSample = 1024;  // sampled items per row this kernel holds
inline size_t row_rank_smem(int n_si) {
    return sizeof(float) * 2 * (size_t) n_si + sizeof(int) * (size_t) n_si +
           sizeof(int) * (size_t) (kSelThreads / 32) * (size_t) (n_si + 1);
}

__global__ void __launch_bounds__(kSelThreads) row_rank_kernel(SelectArgs a) {
    extern __shared__ __align__(16) int rk_smem[];
    const int ns = a.n_si, n = a.n_item;
    const int nw = blockDim.x >> 5, w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *sval = reinterpret_cast<float *>(rk_smem);  // [ns] the sampled items' scores
    float *wsort = sval + ns;                          // [ns] the same, descending
    int *pos_of = reinterpret_cast<int *>(wsort + ns);  // [ns] sorted position of sampled item s
    int *cnt = pos_of + ns;                            // [nw][ns + 1] bucket counts per warp
    const int n_iter = a.row_list ? a.n_list : a.n_rows;
    for (int ri = blockIdx.x; ri < n_iter; ri += gridDim.x) {
        const int row = a.row_list ? a.row_list[ri] : ri;
        const float *src = a.rows + (int64_t) row * a.ld;
        for (int t = threadIdx.x; t < ns; t += blockDim.x) sval[t] = src[a.sample_item[t]];
        for (int t = threadIdx.x; t < nw * (ns + 1); t += blockDim.x) cnt[t] = 0;
        __syncthreads();
        // sorted position: the scores above it, then the equal ones listed before it
        for (int t = threadIdx.x; t < ns; t += blockDim.x) {
            const float v = sval[t];
            int p = 0;
            for (int k = 0; k < ns; k++) {
                const float y = sval[k];
                p += (y > v) | ((y == v) & (k < t));
            }
            wsort[p] = v;
            pos_of[t] = p;
        }
        __syncthreads();
        int *cw = cnt + w * (ns + 1);
        auto bucket = [&](float x) {  // first k with wsort[k] < x
            int lo = 0, len = ns;
            while (len > 0) {
                const int half = len >> 1, mid = lo + half;
                if (wsort[mid] >= x) { lo = mid + 1; len -= half + 1; } else len = half;
            }
            return lo;
        };
        // the row in 16-byte loads, four in flight per thread (rows start 16-byte aligned)
        const float4 *src4 = reinterpret_cast<const float4 *>(src);
        const int n4 = n >> 2;
        for (int i0 = threadIdx.x; i0 < n4; i0 += 4 * blockDim.x) {
            float4 x[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int i = i0 + k * blockDim.x;
                if (i < n4) x[k] = __ldcs(src4 + i);
            }
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int i = i0 + k * blockDim.x;
                if (i < n4) {
                    atomicAdd(&cw[bucket(x[k].x)], 1);
                    atomicAdd(&cw[bucket(x[k].y)], 1);
                    atomicAdd(&cw[bucket(x[k].z)], 1);
                    atomicAdd(&cw[bucket(x[k].w)], 1);
                }
            }
        }
        for (int i = 4 * n4 + threadIdx.x; i < n; i += blockDim.x) atomicAdd(&cw[bucket(src[i])], 1);
        __syncthreads();
        // the warps' counts summed into warp 0's row, then its inclusive prefix (warp 0, 32 at a time)
        for (int b = threadIdx.x; b <= ns; b += blockDim.x) {
            int t = 0;
            for (int k = 0; k < nw; k++) t += cnt[k * (ns + 1) + b];
            cnt[b] = t;
        }
        __syncthreads();
        if (w == 0) {
            int base = 0;
            for (int b0 = 0; b0 <= ns; b0 += 32) {
                const int b = b0 + lane;
                int v = b <= ns ? cnt[b] : 0;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, v, o);
                    if (lane >= o) v += y;
                }
                if (b <= ns) cnt[b] = base + v;
                base += __shfl_sync(0xffffffffu, v, 31);
            }
        }
        __syncthreads();
        for (int t = threadIdx.x; t < ns; t += blockDim.x)
            atomicAdd(&a.rank_hist[(int64_t) t * (n + 1) + cnt[pos_of[t]]], 1);
        __syncthreads();
    }
}

// ---- rows longer than shared memory ------------------------------------------------------------------
//
// A row of config-4 size (624,961 items) does not fit in shared memory.  Instead of copying it to a
// global scratch row and scattering it there in bin order (a scattered 4-byte store per item), the
// CTA streams the row from where the score pass wrote it: its range, a histogram of kGBins value
// bins, and then -- for the bins holding a requested position or a sampled item's score only -- a
// copy of those values into shared memory, where the order statistics are taken.  Requested bins
// that do not fit the staging buffer together are staged in several rounds (one more stream each).
// A row whose scores are all equal needs no bins; a row with a requested bin larger than the whole
// buffer (an extreme concentration of scores) is listed, untouched, for the scatter form
// (row_select_kernel on global scratch).
constexpr int kGBins = 16384;
constexpr int kGStage = 23552;  // staged values (92 KB)
constexpr size_t kGSmem = sizeof(int) * (2 * kGBins + 1) + sizeof(uint32_t) * (kGBins / 32) + sizeof(float) * kGStage;

__device__ __forceinline__ int value_bin_g(float x, float mn, float scale) {
    const int b = (int) __fmul_rn(__fsub_rn(x, mn), scale);
    return min(max(b, 0), kGBins - 1);
}

// Calls f on every value of a row (16-byte aligned, as the score rows are): four float4 loads in
// flight per thread, so that one CTA per SM keeps enough of the row in flight.
template <class F>
__device__ __forceinline__ void stream_row(const float *__restrict__ src, int n, F f) {
    // 16-byte loads, four in flight per thread before their values are visited
    const float4 *s4 = reinterpret_cast<const float4 *>(src);
    const int n4 = n >> 2;
    for (int i0 = threadIdx.x; i0 < n4; i0 += 4 * blockDim.x) {
        float4 v[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int i = i0 + k * blockDim.x;
            if (i < n4) v[k] = __ldg(s4 + i);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            if (i0 + k * blockDim.x < n4) {
                f(v[k].x);
                f(v[k].y);
                f(v[k].z);
                f(v[k].w);
            }
        }
    }
    for (int i = (n4 << 2) + threadIdx.x; i < n; i += blockDim.x) f(__ldg(src + i));
}

// Exclusive scan of v(b) over the kGBins bins, kGBins / blockDim.x consecutive bins per thread:
// out(b, offset) for every bin; returns the total in every thread.  Called by the whole block.
template <class V, class O>
__device__ __forceinline__ int bins_excl_scan(V v, O out, int *warp_tot) {
    constexpr int per = kGBins / kSelThreads;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int loc[per];
    int s = 0;
#pragma unroll
    for (int t = 0; t < per; t++) { loc[t] = s; s += v(threadIdx.x * per + t); }
    int incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += x;
    }
    __syncthreads();  // warp_tot free
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    int total = 0;
    for (int i = 0; i < nw; i++) total += warp_tot[i];
    int before = 0;
    for (int i = 0; i < w; i++) before += warp_tot[i];
    const int base = before + incl - s;
#pragma unroll
    for (int t = 0; t < per; t++) out(threadIdx.x * per + t, base + loc[t]);
    return total;
}

// The bin holding ascending position p: the last bin whose start is <= p.
__device__ __forceinline__ int bin_of_pos(const int *start, int p) {
    int lo = 0, len = kGBins;
    while (len > 0) {
        const int h = len >> 1, m = lo + h;
        if (start[m + 1] <= p) { lo = m + 1; len -= h + 1; } else len = h;
    }
    return lo;
}

__global__ void __launch_bounds__(kSelThreads) row_select_global_kernel(SelectArgs a, int32_t *__restrict__ defer,
                                                                        int *__restrict__ n_defer) {
    extern __shared__ int gdyn[];
    int *hist = gdyn;                                                   // counts, then staging cursors
    int *start = hist + kGBins;                                         // [kGBins + 1] bin starts
    uint32_t *want = reinterpret_cast<uint32_t *>(start + kGBins + 1);  // requested bins, one bit each
    float *stage = reinterpret_cast<float *>(want + kGBins / 32);       // [kGStage]
    __shared__ float red_mn[32], red_mx[32];
    __shared__ int warp_tot[32];
    __shared__ int round_lo, round_hi, too_big;
    const int n = a.n_item;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    constexpr int per = kGBins / kSelThreads;
    auto requested = [&](int b) { return (want[b >> 5] >> (b & 31)) & 1u; };
    for (int row = blockIdx.x; row < a.n_rows; row += gridDim.x) {
        const float *src = a.rows + (int64_t) row * a.ld;
        // stream 1: the row's range
        float mn = __int_as_float(0x7f800000), mx = -mn;
        stream_row(src, n, [&](float x) {
            mn = fminf(mn, x);
            mx = fmaxf(mx, x);
        });
        for (int o = 16; o > 0; o >>= 1) {
            mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
            mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        }
        if (lane == 0) { red_mn[w] = mn; red_mx[w] = mx; }
        for (int b = threadIdx.x; b < kGBins; b += blockDim.x) hist[b] = 0;
        for (int b = threadIdx.x; b < kGBins / 32; b += blockDim.x) want[b] = 0u;
        if (threadIdx.x == 0) too_big = 0;
        __syncthreads();
        mn = red_mn[0];
        mx = red_mx[0];
        for (int i = 1; i < nw; i++) { mn = fminf(mn, red_mn[i]); mx = fmaxf(mx, red_mx[i]); }
        const float range = __fsub_rn(mx, mn);
        if (!(range > 0.0f)) {
            // every score equal: every threshold is that score, and no item scores above any other
            if (a.thr_out)
                for (int j = threadIdx.x; j < a.S; j += blockDim.x) a.thr_out[(int64_t) row * a.S + j] = mn;
            if (a.rank_hist)
                for (int s2 = threadIdx.x; s2 < a.n_si; s2 += blockDim.x) atomicAdd(&a.rank_hist[(int64_t) s2 * (n + 1)], 1);
            __syncthreads();
            continue;
        }
        const float scale = __fdiv_rn((float) kGBins, range);
        // stream 2: the histogram
        stream_row(src, n, [&](float x) { atomicAdd(&hist[value_bin_g(x, mn, scale)], 1); });
        __syncthreads();
        {  // exclusive scan of the counts into start
            int loc[per];
            int s = 0;
#pragma unroll
            for (int t = 0; t < per; t++) { loc[t] = s; s += hist[threadIdx.x * per + t]; }
            int incl = s;
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (lane == 31) warp_tot[w] = incl;
            __syncthreads();
            if (w == 0) {
                const int v = lane < nw ? warp_tot[lane] : 0;
                int iv = v;
                for (int o = 1; o < 32; o <<= 1) {
                    const int x = __shfl_up_sync(0xffffffffu, iv, o);
                    if (lane >= o) iv += x;
                }
                if (lane < nw) warp_tot[lane] = iv - v;
            }
            __syncthreads();
            const int base = warp_tot[w] + incl - s;
#pragma unroll
            for (int t = 0; t < per; t++) start[threadIdx.x * per + t] = base + loc[t];
            if (threadIdx.x == 0) start[kGBins] = n;
        }
        __syncthreads();
        // the requested bins: each threshold's position (descending rank r is ascending n - 1 - r)
        // and each sampled item's score
        if (a.thr_out)
            for (int j = threadIdx.x; j < a.S; j += blockDim.x) {
                const int b = bin_of_pos(start, n - 1 - a.sample_rank[j]);
                atomicOr(&want[b >> 5], 1u << (b & 31));
                if (start[b + 1] - start[b] > kGStage) too_big = 1;
            }
        if (a.rank_hist)
            for (int s2 = threadIdx.x; s2 < a.n_si; s2 += blockDim.x) {
                const int b = value_bin_g(__ldg(src + a.sample_item[s2]), mn, scale);
                atomicOr(&want[b >> 5], 1u << (b & 31));
                if (start[b + 1] - start[b] > kGStage) too_big = 1;
            }
        __syncthreads();
        if (too_big) {  // left whole to the scatter form
            if (threadIdx.x == 0) defer[atomicAdd(n_defer, 1)] = row;
            __syncthreads();
            continue;
        }
        // The requested bins' staging cursors from a block-wide scan of their sizes: when they fit the
        // buffer together (nearly always) that is the only round; otherwise rounds over the requested
        // bins in bin order, each staging what fits, planned bin by bin.
        const int req_total = bins_excl_scan(
            [&](int b) { return requested(b) ? start[b + 1] - start[b] : 0; },
            [&](int b, int off) { if (requested(b)) hist[b] = off; }, warp_tot);
        const bool one_round = req_total <= kGStage;
        if (threadIdx.x == 0) round_hi = 0;
        __syncthreads();
        while (true) {
            if (one_round) {
                if (threadIdx.x == 0) {
                    round_lo = round_hi == 0 ? 0 : kGBins;
                    round_hi = kGBins;
                }
            } else if (threadIdx.x == 0) {
                int b = round_hi;
                while (b < kGBins && !requested(b)) b++;
                round_lo = b;
                int off = 0, e = b;
                for (; e < kGBins; e++) {
                    if (!requested(e)) continue;
                    const int sz = start[e + 1] - start[e];
                    if (off + sz > kGStage) break;
                    hist[e] = off;  // the bin's staging cursor
                    off += sz;
                }
                round_hi = e;
            }
            __syncthreads();
            const int lo_b = round_lo, hi_b = round_hi;
            if (lo_b >= kGBins) break;
            // stream 3: this round's values into the staging buffer
            stream_row(src, n, [&](float x) {
                const int b = value_bin_g(x, mn, scale);
                if (b >= lo_b && b < hi_b && requested(b)) stage[atomicAdd(&hist[b], 1)] = x;
            });
            __syncthreads();
            // thresholds whose position lies in this round's bins (a bin's values end at its cursor)
            if (a.thr_out)
                for (int j = w; j < a.S; j += nw) {
                    const int p = n - 1 - a.sample_rank[j];
                    const int b = bin_of_pos(start, p);
                    if (b < lo_b || b >= hi_b) continue;
                    const int sz = start[b + 1] - start[b];
                    const float v = warp_select(stage + hist[b] - sz, sz, p - start[b]);
                    if (lane == 0) a.thr_out[(int64_t) row * a.S + j] = v;
                }
            // query ranks: items scoring strictly above each sampled item's score
            if (a.rank_hist)
                for (int s2 = threadIdx.x; s2 < a.n_si; s2 += blockDim.x) {
                    const float sv = __ldg(src + a.sample_item[s2]);
                    const int b = value_bin_g(sv, mn, scale);
                    if (b < lo_b || b >= hi_b) continue;
                    const int sz = start[b + 1] - start[b];
                    const float *seg = stage + hist[b] - sz;
                    int cnt = n - start[b + 1];
                    for (int t = 0; t < sz; t++) cnt += seg[t] > sv;
                    atomicAdd(&a.rank_hist[(int64_t) s2 * (n + 1) + cnt], 1);
                }
            __syncthreads();
        }
        __syncthreads();
    }
}

// Inclusive prefix sums of each row of h ([rows][len]), one block per row: each thread sums its own
// contiguous segment, the block scans the segment sums, and each thread rewrites its segment from its
// starting offset.
constexpr int kPrefixThreads = 1024;
__global__ void __launch_bounds__(kPrefixThreads) prefix_rows_kernel(int32_t *__restrict__ h, int rows, int64_t len) {
    __shared__ int32_t warp_tot[kPrefixThreads / 32];
    const int r = blockIdx.x;
    if (r >= rows) return;
    int32_t *p = h + (int64_t) r * len;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int64_t per = (len + blockDim.x - 1) / blockDim.x;
    const int64_t b = (int64_t) threadIdx.x * per, e = min(len, b + per);
    int32_t s = 0;
    for (int64_t i = b; i < e; i++) s += p[i];
    int32_t incl = s;
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int32_t v = lane < nw ? warp_tot[lane] : 0;
        int32_t iv = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t x = __shfl_up_sync(0xffffffffu, iv, o);
            if (lane >= o) iv += x;
        }
        if (lane < nw) warp_tot[lane] = iv - v;
    }
    __syncthreads();
    int32_t run = warp_tot[w] + incl - s;  // the sum of every segment before this thread's
    for (int64_t i = b; i < e; i++) {
        run += p[i];
        p[i] = run;
    }
}

// ---- host side --------------------------------------------------------------------------------------

namespace {

// Raises row_select_kernel's dynamic shared-memory limit on the current device to the largest the
// device allows.  Every caller sets the same value, so callers on other host threads never lower
// the limit under each other's launches; it is set on every call (cheap) rather than cached, so a
// device reset, which restores the default, needs no special handling.
int row_select_allow_max_smem() {
    int dev = 0, optin = 0;
    RKR_CUDA(cudaGetDevice(&dev));
    RKR_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    RKR_CUDA(cudaFuncGetAttributes(&fa, row_select_kernel));
    RKR_CUDA(cudaFuncSetAttribute(row_select_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  optin - (int) fa.sharedSizeBytes));
    RKR_CUDA(cudaFuncGetAttributes(&fa, row_select_global_kernel));
    RKR_CUDA(cudaFuncSetAttribute(row_select_global_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  optin - (int) fa.sharedSizeBytes));
    return RKR_OK;
}

struct RowPipeline {
    rkr_index *ix;
    int64_t batch = 0;
    int64_t ld = 0;
    int grid = 0;
    size_t smem = 0;
    int use_smem = 1;
    int sms = 0;
};

int setup_pipeline(rkr_index *ix, RowPipeline &P) {
    P.ix = ix;
    const int64_t n = ix->n_item;
    P.ld = (n + 3) / 4 * 4;
    P.batch = std::max<int64_t>(64, std::min<int64_t>(ix->n_user, (int64_t(3) << 30) / (P.ld * 4)));
    P.batch = (P.batch + kTile - 1) / kTile * kTile;
    int dev_smem = 0;
    RKR_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ix->device));
    const size_t static_smem = sizeof(int) * (2 * kBins + 1) + 64 * sizeof(float) * 2 + 32 * sizeof(int);
    P.smem = (size_t) 2 * n * sizeof(float);
    P.use_smem = P.smem + static_smem + 1024 <= (size_t) dev_smem;
    if (!P.use_smem) P.smem = 0;
    RKR_TRY(row_select_allow_max_smem());
    RKR_CUDA(cudaDeviceGetAttribute(&P.sms, cudaDevAttrMultiProcessorCount, ix->device));
    P.grid = P.sms;
    RKR_TRY(ix->ws_bucket.ensure((size_t) P.batch * P.ld * sizeof(float)));
    // long rows: the deferred-row list of the streaming selection (the scatter form's global
    // scratch is allocated only if a row is deferred to it)
    if (!P.use_smem) RKR_TRY(ix->ws_defer.ensure(sizeof(int32_t) * (size_t) (P.batch + 1)));
    return RKR_OK;
}

int run_rows(RowPipeline &P, int64_t u0, int64_t nu, SelectArgs sa) {
    rkr_index *ix = P.ix;
    cudaStream_t st = ix->stream;
    float *rows = ix->ws_bucket.as<float>();
    ScoreRowsEpi epi;
    epi.rows = rows;
    epi.ld = P.ld;
    epi.n_item = ix->n_item;
    epi.n_rows = nu;
    cudaError_t ce = cudaSuccess;
    timed(ix, st, "score_rows", [&] {
        ce = launch_big(ix->item.as<float>(), nullptr, ix->n_item, ix->dim, ix->user.as<float>() + u0 * ix->dim, nu,
                        ix->dim, 0, ix->dim, epi, st);
    });
    RKR_CUDA(ce);
    sa.rows = rows;
    sa.ld = P.ld;
    sa.n_rows = (int) nu;
    sa.n_item = (int) ix->n_item;
    if (sa.rank_hist && !sa.thr_out && !sa.sorted_out && sa.n_si <= kRankMaxSample) {
        // the query-rank distribution alone: one counting stream per row, any row length
        const size_t smem = row_rank_smem(sa.n_si);
        RKR_CUDA(cudaFuncSetAttribute(row_rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
        timed(ix, st, "row_rank", [&] {
            row_rank_kernel<<<(unsigned) std::min<int64_t>(4 * P.sms, nu), kSelThreads, smem, st>>>(sa);
        });
        RKR_CUDA(cudaGetLastError());
        return RKR_OK;
    }
    if (P.use_smem || sa.sorted_out) {
        // rows in shared memory; or a full sort (rkr_score_sort_batch), which scatters long rows
        // on global scratch
        const int grid = P.use_smem ? P.grid : 2 * P.sms;
        if (!P.use_smem) {
            RKR_TRY(ix->ws_misc.ensure((size_t) grid * 2 * ix->n_item * sizeof(float)));
            sa.gscratch = ix->ws_misc.as<float>();
        }
        timed(ix, st, "row_select", [&] {
            row_select_kernel<<<(unsigned) std::min<int64_t>(grid, nu), kSelThreads, P.smem, st>>>(sa, P.use_smem);
        });
        RKR_CUDA(cudaGetLastError());
        return RKR_OK;
    }
    // long rows: the streaming selection; rows it defers (a requested bin larger than its staging
    // buffer) take the scatter form afterwards
    int32_t *defer = ix->ws_defer.as<int32_t>();
    RKR_CUDA(cudaMemsetAsync(defer + P.batch, 0, sizeof(int32_t), st));
    timed(ix, st, "row_select_stream", [&] {
        row_select_global_kernel<<<(unsigned) std::min<int64_t>(2 * P.sms, nu), kSelThreads, kGSmem, st>>>(
            sa, defer, defer + P.batch);
    });
    RKR_CUDA(cudaGetLastError());
    int n_defer = 0;
    RKR_CUDA(cudaMemcpyAsync(&n_defer, defer + P.batch, sizeof(int), cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    if (n_defer > 0) {
        const int grid = std::min(n_defer, P.sms);
        RKR_TRY(ix->ws_misc.ensure((size_t) grid * 2 * ix->n_item * sizeof(float)));
        sa.gscratch = ix->ws_misc.as<float>();
        sa.row_list = defer;
        sa.n_list = n_defer;
        timed(ix, st, "row_select", [&] { row_select_kernel<<<(unsigned) grid, kSelThreads, 0, st>>>(sa, 0); });
        RKR_CUDA(cudaGetLastError());
        if (ix->prof.on) ix->prof.add_count("row_select_deferred_rows", n_defer);
    }
    return RKR_OK;
}

}  // namespace

int build_sample_search(rkr_index *ix, const int32_t *sample_rank, int n_sample) {
    RKR_TRY(ensure_device(ix));
    RowPipeline P;
    RKR_TRY(setup_pipeline(ix, P));
    RKR_TRY(ix->sample_rank.ensure(sizeof(int32_t) * n_sample));
    RKR_TRY(ix->thr.ensure(sizeof(float) * (size_t) ix->n_user * n_sample));
    RKR_CUDA(cudaMemcpyAsync(ix->sample_rank.p, sample_rank, sizeof(int32_t) * n_sample, cudaMemcpyHostToDevice, ix->stream));
    ix->n_sample = n_sample;
    ix->h_sample_rank.assign(sample_rank, sample_rank + n_sample);
    for (int64_t u0 = 0; u0 < ix->n_user; u0 += P.batch) {
        const int64_t nu = std::min(P.batch, ix->n_user - u0);
        SelectArgs sa = {};
        sa.sample_rank = ix->sample_rank.as<int32_t>();
        sa.S = n_sample;
        sa.thr_out = ix->thr.as<float>() + u0 * n_sample;
        RKR_TRY(run_rows(P, u0, nu, sa));
    }
    RKR_TRY(thr_summary_build(ix));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}

int build_thresholds_range(rkr_index *ix, int64_t u_begin, int64_t u_end) {
    RowPipeline P;
    RKR_TRY(setup_pipeline(ix, P));
    const int S = ix->n_sample;
    for (int64_t u0 = u_begin; u0 < u_end; u0 += P.batch) {
        const int64_t nu = std::min(P.batch, u_end - u0);
        SelectArgs sa = {};
        sa.sample_rank = ix->sample_rank.as<int32_t>();
        sa.S = S;
        sa.thr_out = ix->thr.as<float>() + u0 * S;
        RKR_TRY(run_rows(P, u0, nu, sa));
    }
    return RKR_OK;
}

int score_sort_rows(rkr_index *ix, int64_t start, int64_t n_rows, float *h_rows) {
    RKR_TRY(ensure_device(ix));
    RowPipeline P;
    RKR_TRY(setup_pipeline(ix, P));
    const int64_t n = ix->n_item;
    const int64_t per = std::max<int64_t>(1, std::min<int64_t>(P.batch, (int64_t(1) << 30) / (n * 4)));
    RKR_TRY(ix->ws_out.ensure((size_t) per * n * sizeof(float)));
    for (int64_t r0 = 0; r0 < n_rows; r0 += per) {
        const int64_t nr = std::min(per, n_rows - r0);
        SelectArgs sa = {};
        sa.sorted_out = ix->ws_out.as<float>();
        RKR_TRY(run_rows(P, start + r0, nr, sa));
        RKR_CUDA(cudaMemcpyAsync(h_rows + r0 * n, ix->ws_out.p, (size_t) nr * n * sizeof(float), cudaMemcpyDeviceToHost,
                                 ix->stream));
        RKR_CUDA(cudaStreamSynchronize(ix->stream));
    }
    return RKR_OK;
}

int query_rank_distribution(rkr_index *ix, const int32_t *sample_item, int n_sample_item, int32_t *h_accu) {
    RKR_TRY(ensure_device(ix));
    RowPipeline P;
    RKR_TRY(setup_pipeline(ix, P));
    const int64_t n = ix->n_item;
    RKR_TRY(ix->ws_hist.ensure(sizeof(int32_t) * (size_t) n_sample_item * (n + 1)));
    RKR_TRY(ix->ws_res.ensure(sizeof(int32_t) * n_sample_item));
    RKR_CUDA(cudaMemsetAsync(ix->ws_hist.p, 0, sizeof(int32_t) * (size_t) n_sample_item * (n + 1), ix->stream));
    RKR_CUDA(cudaMemcpyAsync(ix->ws_res.p, sample_item, sizeof(int32_t) * n_sample_item, cudaMemcpyHostToDevice, ix->stream));
    for (int64_t u0 = 0; u0 < ix->n_user; u0 += P.batch) {
        const int64_t nu = std::min(P.batch, ix->n_user - u0);
        SelectArgs sa = {};
        sa.sample_item = ix->ws_res.as<int32_t>();
        sa.n_si = n_sample_item;
        sa.rank_hist = ix->ws_hist.as<int32_t>();
        RKR_TRY(run_rows(P, u0, nu, sa));
    }
    // user shards: every shard's counts
    RKR_TRY(shard_sum(ix, ix->ws_hist.as<int32_t>(), (int64_t) n_sample_item * (n + 1), ix->stream));
    timed(ix, ix->stream, "prefix_rows", [&] {
        prefix_rows_kernel<<<n_sample_item, kPrefixThreads, 0, ix->stream>>>(ix->ws_hist.as<int32_t>(), n_sample_item, n + 1);
    });
    RKR_CUDA(cudaGetLastError());
    RKR_CUDA(cudaMemcpyAsync(h_accu, ix->ws_hist.p, sizeof(int32_t) * (size_t) n_sample_item * (n + 1),
                             cudaMemcpyDeviceToHost, ix->stream));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}

// ---- threshold build without device allocation ------------------------------------------------------
//
// rkr_build_thresholds_static serves callers that must not allocate device memory themselves or
// through the library: code running where cudaMalloc is not allowed or not wanted (inside a
// memory pool that has already been carved up, an allocator hook, a real-time service that fixes
// its footprint at start-up).  Its only scratch is this fixed array, which every GPU that loads the
// library holds until the process exits: the sampled ranks (first 64 KiB) and one batch of score
// rows (the rest).  In host code g_static_scratch names a host-side stand-in, not device memory,
// so the kernels receive the address cudaGetSymbolAddress returns for the current device.

constexpr size_t kStaticScratchBytes = size_t(32) << 20;
constexpr size_t kStaticRankBytes = size_t(64) << 10;
constexpr int kStaticMaxSample = (int) (kStaticRankBytes / sizeof(int32_t));
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

// The array's device address in the current device's context.  It is looked up on every call
// (cudaGetSymbolAddress is cheap once the module is loaded) instead of being cached, so that the
// address is right after a device reset, which reloads the module in a new context.
static int static_scratch_address(unsigned char **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) {
        set_error("rkr_build_thresholds_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return RKR_ERR_CUDA;
    }
    *out = static_cast<unsigned char *>(p);
    return RKR_OK;
}

}  // namespace rkr

extern "C" int rkr_build_thresholds_static(const float *d_user, int64_t n_user, const float *d_item, int64_t n_item,
                                           int32_t dim, const int32_t *sample_rank, int32_t n_sample,
                                           float *d_thresholds, void *stream) {
    using namespace rkr;
    RKR_REQUIRE(d_user && d_item && sample_rank && d_thresholds, "rkr_build_thresholds_static: null argument");
    RKR_REQUIRE(n_user > 0 && n_item > 1 && dim > 0 && dim <= 4096, "rkr_build_thresholds_static: bad sizes");
    RKR_REQUIRE(n_sample > 0 && n_sample < n_item, "rkr_build_thresholds_static: n_sample %d must be in (0, n_item)",
                n_sample);
    RKR_REQUIRE(n_sample <= kStaticMaxSample, "rkr_build_thresholds_static: n_sample %d above the maximum %d",
                n_sample, kStaticMaxSample);
    for (int j = 0; j < n_sample; j++) {
        RKR_REQUIRE(sample_rank[j] >= 0 && sample_rank[j] < n_item, "sample rank %d out of range", sample_rank[j]);
        RKR_REQUIRE(j == 0 || sample_rank[j] >= sample_rank[j - 1], "sample ranks must be ascending");
    }
    const int64_t ld = (n_item + 3) / 4 * 4;
    const int64_t row_bytes = ld * (int64_t) sizeof(float);
    const int64_t batch = (int64_t) (kStaticScratchBytes - kStaticRankBytes) / row_bytes;
    RKR_REQUIRE(batch >= 1, "rkr_build_thresholds_static: n_item %lld exceeds the %zu-byte scratch",
                (long long) n_item, kStaticScratchBytes - kStaticRankBytes);
    int dev = 0;
    RKR_CUDA(cudaGetDevice(&dev));
    int dev_smem = 0;
    RKR_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t smem = (size_t) 2 * n_item * sizeof(float);
    const size_t static_smem = sizeof(int) * (2 * kBins + 1) + 64 * sizeof(float) * 2 + 32 * sizeof(int);
    RKR_REQUIRE(smem + static_smem + 1024 <= (size_t) dev_smem,
                "rkr_build_thresholds_static: n_item %lld too large for the shared-memory row selection",
                (long long) n_item);
    unsigned char *scratch = nullptr;
    RKR_TRY(static_scratch_address(&scratch));
    int32_t *d_rank = reinterpret_cast<int32_t *>(scratch);
    float *rows = reinterpret_cast<float *>(scratch + kStaticRankBytes);
    cudaStream_t st = (cudaStream_t) stream;
    RKR_CUDA(cudaMemcpyAsync(d_rank, sample_rank, sizeof(int32_t) * n_sample, cudaMemcpyHostToDevice, st));
    RKR_TRY(row_select_allow_max_smem());
    int sms = 0;
    RKR_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    for (int64_t u0 = 0; u0 < n_user; u0 += batch) {
        const int64_t nu = std::min(batch, n_user - u0);
        ScoreRowsEpi epi;
        epi.rows = rows;
        epi.ld = ld;
        epi.n_item = n_item;
        epi.n_rows = nu;
        RKR_CUDA(launch_big(d_item, nullptr, n_item, dim, d_user + u0 * dim, nu, dim, 0, dim, epi, st));
        SelectArgs sa = {};
        sa.rows = rows;
        sa.ld = ld;
        sa.n_rows = (int) nu;
        sa.n_item = (int) n_item;
        sa.sample_rank = d_rank;
        sa.S = n_sample;
        sa.thr_out = d_thresholds + u0 * n_sample;
        row_select_kernel<<<(unsigned) std::min<int64_t>(sms, nu), kSelThreads, smem, st>>>(sa, 1);
        RKR_CUDA(cudaGetLastError());
    }
    RKR_CUDA(cudaStreamSynchronize(st));
    return RKR_OK;
}
