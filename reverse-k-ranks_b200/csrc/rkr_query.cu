// rkr_query.cu -- batched reverse k-ranks retrieval on the device (QS, QSRPNormalLP, US).
//
// A batch of queries runs as a short pipeline of kernels; every (query, user) decision the
// reference makes one query at a time (src/impl/QS.hpp:127-224, src/impl/QSRPNormalLP.hpp:137-253,
// src/impl/US.hpp:117-201) is made for the whole batch at once:
//
//   score_bucket      exact query score of every (user, query) pair + binary search over the
//                     user's sampled thresholds -> one 16-bit bucket per pair      [SIMT, FP32 exact]
//   select_bucket     per query: histogram of buckets -> k-th smallest lower/upper rank bound ->
//                     class (result / prune / refine) of every bucket value
//   compact           per query, in user-id order: first top-k result users, all candidates
//   refine_prep       candidates: exact score, norm cut-off, rank when the bounds already agree
//   refine_tile       candidates x norm-ordered items: exact split-sum scores, bound tests,
//                     count of items scoring >= the query (or > for US)      [SIMT, FP32 exact]
//   assemble          per query: results in user-id order, then candidates by (rank, user id)
//
// QSRPNormalLP adds the regression stage before it (qsrp_* kernels below).
#include <algorithm>
#include <cstring>
#include <numeric>

#include "rkr_internal.cuh"

namespace rkr {

// ============================================================================================
// shared pieces
// ============================================================================================

// ============================================================================================
// QS / US: bucket per pair
// ============================================================================================

// queryIP = InnerProduct(query, user) over all dims (QS.hpp:137-143, US.hpp:125-131), then
// SampleSearch::CoarseBinarySearch's bucket (SampleSearch.hpp:91-107).
__global__ void __launch_bounds__(kTileThreads) score_bucket_kernel(const float *__restrict__ user, int64_t n_user,
                                                                   int dim, const float *__restrict__ query,
                                                                   int n_query, const float *__restrict__ thr, int S,
                                                                   uint16_t *__restrict__ bucket) {
    __shared__ TileSmem sm;
    __shared__ ThrSummary ts;
    const int64_t b0 = (int64_t) blockIdx.x * kTile;  // queries
    const int64_t a0 = (int64_t) blockIdx.y * kTile;  // users
    load_thr_summary(ts, thr, n_user, a0, S);
    float lo[4][4], hi[4][4];
    exact_tile(sm, user, nullptr, n_user, dim, a0, query, n_query, dim, b0, 0, dim, dim, lo, hi);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int64_t u = a0 + 4 * tx + i;
        if (u >= n_user) continue;
        const float *row = thr + u * S;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t q = b0 + 4 * ty + j;
            if (q >= n_query) continue;
            bucket[q * n_user + u] = (uint16_t) bucket_of_2level(ts.v[4 * tx + i], row, S, lo[i][j]);
        }
    }
}

// score_bucket on 128 x 128 tiles: the exact score of each (user, query) pair and its bucket.
struct QsBucketEpi {
    static constexpr size_t kExtra = sizeof(float) * kBig * ThrSummary::kMaxGroups;
    const float *thr;
    int64_t n_user, n_query;
    int S;
    uint16_t *bucket;
    __device__ void prologue(char *extra, int64_t a0, int64_t) const {
        load_thr_summary_rows(reinterpret_cast<float *>(extra), kBig, thr, n_user, a0, S);
    }
    __device__ bool active(char *, int64_t, int64_t) const { return true; }
    __device__ void finish(char *extra, const BigResult &res, int64_t a0, int64_t b0, bool) const {
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7;
        const int64_t u = a0 + ra;
        if (u >= n_user) return;
        const float *summ = reinterpret_cast<const float *>(extra) + ra * ThrSummary::kMaxGroups;
        const float *row = thr + u * S;
#pragma unroll 4
        for (int i = 0; i < kBig / 2; i++) {
            const int rb = half + 2 * i;
            const int64_t q = b0 + rb;
            if (q >= n_query) break;
            bucket[q * n_user + u] = (uint16_t) bucket_of_2level(summ, row, S, res.v[rb][ra]);
        }
    }
};

__global__ void select_bucket_kernel(const int *__restrict__ hist_all, int S, const int32_t *__restrict__ rank,
                                     int n_item, int topk, int n_user, uint8_t *__restrict__ cls,
                                     QueryCounts *__restrict__ counts) {
    const int q = blockIdx.x;
    const int *hist = hist_all + (int64_t) q * (S + 1);
    if (threadIdx.x == 0) {
        int bk = S;
        int64_t cum = 0;
        for (int b = 0; b <= S; b++) {
            cum += hist[b];
            if (cum >= topk) { bk = b; break; }
        }
        int L, U;
        bucket_bounds(bk, S, rank, n_item, L, U);
        QueryCounts c = {};
        c.bk = bk; c.lstar = L; c.ustar = U;
        c.ip_base = n_user;
        uint8_t *cq = cls + (int64_t) q * (S + 1);
        if (L == U) {
            int64_t nres = 0;
            for (int b = 0; b <= S; b++) {
                int lb, ub;
                bucket_bounds(b, S, rank, n_item, lb, ub);
                const bool r = ub <= L && lb <= L;
                cq[b] = r ? kClsResult : kClsIdle;
                if (r) nres += hist[b];
            }
            c.mode = 1; c.n_result = topk; c.n_prune = 0; c.n_cand = 0;
            c.n_res_emit = (int) (nres < topk ? nres : (int64_t) topk);
        } else {
            int64_t nres = 0, npr = 0, nref = 0;
            for (int b = 0; b <= S; b++) {
                int lb, ub;
                bucket_bounds(b, S, rank, n_item, lb, ub);
                uint8_t k;
                if (lb <= U) { k = kClsResult; nres += hist[b]; }
                else if (L <= ub) { k = kClsPrune; npr += hist[b]; }
                else { k = kClsRefine; nref += hist[b]; }
                cq[b] = k;
            }
            c.mode = 0;
            if (nres + nref == topk) {  // PruneCandidateByBound.hpp:139-150
                for (int b = 0; b <= S; b++) if (cq[b] == kClsRefine) cq[b] = kClsResult;
                nres = topk; nref = 0;
            }
            c.n_result = (int) nres; c.n_prune = (int) npr;
            c.n_cand = nres >= topk ? 0 : (int) nref;
            c.n_res_emit = (int) (nres < topk ? nres : (int64_t) topk);
        }
        counts[q] = c;
    }
}

// QS / US classification of a pair for the ordered compaction: the class of its bucket.
struct QsCompactPolicy {
    struct Aux { uint16_t b; };
    const uint16_t *bucket;
    int64_t n_user;
    const uint8_t *cls;
    int S;
    const QueryCounts *counts;
    const int64_t *cand_off;
    int topk;
    int32_t *res_user, *cand_user, *cand_query;
    uint16_t *cand_bucket;
    __device__ bool query_active(int q) const { return true; }
    __device__ uint32_t need_mask(int, int64_t, int n) const { return (1u << n) - 1; }
    __device__ int classify(int q, int64_t u, Aux &aux, bool) const {
        const uint16_t b = bucket[(int64_t) q * n_user + u];
        aux.b = b;
        const uint8_t k = __ldg(cls + (int64_t) q * (S + 1) + b);
        if (k == kClsResult) return 1;
        return (k == kClsRefine && counts[q].n_cand > 0) ? 2 : 0;
    }
    __device__ void emit_result(int q, int pos, int64_t u, const Aux &) const {
        res_user[(int64_t) q * topk + pos] = (int32_t) u;
    }
    __device__ void emit_cand(int q, int pos, int64_t u, const Aux &aux) const {
        if (pos >= counts[q].n_cand) return;  // the count pass disagrees; reported by compact_scan
        const int64_t e = cand_off[q] + pos;
        cand_user[e] = (int32_t) u;
        cand_query[e] = q;
        cand_bucket[e] = aux.b;
    }
};

// ============================================================================================
// refinement
// ============================================================================================


// Score of each candidate and its rank when the bounds agree (ComputeAllIPBound.hpp:319-341;
// ComputeAll.hpp:84-100); the rest are queued for refine_tile with their item cut-off
// (RefineCPUIPBound.hpp:475-484: items whose norm exceeds queryIP - 8e-3).
__global__ void refine_prep_kernel(RefineArgs a) {
    const int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= a.n_cand) return;
    const int u = a.cand_user[e];
    float qip;
    if (a.cand_qip) qip = a.cand_qip[e];
    else qip = exact_dot(a.query + (int64_t) a.cand_query[e] * a.dim, a.user + (int64_t) u * a.dim, a.dim);
    a.qip[e] = qip;
    const int lb = a.cand_lb[e], ub = a.cand_ub[e];
    if (lb == ub) {
        a.rank[e] = lb;
        a.nproc[e] = 0;
        a.undecided[e] = 0;
        return;
    }
    int np = (int) a.n_item;
    if (a.ipbound) {
        const float lowq = __fsub_rn(qip, 8e-3f);
        int lo = 0, len = (int) a.n_item;
        while (len > 0) {
            const int h = len >> 1, m = lo + h;
            if (__ldg(a.item_norm + m) > lowq) { lo = m + 1; len -= h + 1; } else len = h;
        }
        np = lo;
    }
    a.rank[e] = 0;
    a.nproc[e] = np;
    a.undecided[e] = 0;
    const int slot = atomicAdd(a.n_ref, 1);
    a.ref_idx[slot] = (int32_t) e;
    a.ref_user[slot] = u;
}

// Candidates x items on 128 x 128 tiles: the reference's per-item test, summed per candidate
// (RefineCPUIPBound::RefineRank, RefineCPUIPBound.hpp:93-150, with the split sums of
// RefineCPUPartDimPartNorm.hpp:83-152; RefineCPU::RefineRank, RefineCPU.hpp:33-55).  The partial
// score over the first check_dim coordinates +- the product of the remaining norms settles most
// items; the undecided ones are tested on partial + remainder.  Rows are the refined candidates
// (users gathered through ref_user, whose entries past n_ref are 0), columns the items in the
// order the bound assumes; a candidate's items past its cut-off nproc are not counted.
struct RefineEpi {
    static constexpr size_t kExtra = sizeof(int) * kBig * 2 + sizeof(float) * kBig * 3 + sizeof(uint32_t) * kBigThreads * 2;
    RefineArgs a;
    const float *item_rnorm, *user_rnorm;
    int64_t row0;  // candidate offset of this launch
    __device__ int *rows_e(char *x) const { return reinterpret_cast<int *>(x); }
    __device__ int *rows_np(char *x) const { return reinterpret_cast<int *>(x) + kBig; }
    __device__ float *rows_qv(char *x) const { return reinterpret_cast<float *>(x) + 2 * kBig; }
    __device__ float *rows_un(char *x) const { return reinterpret_cast<float *>(x) + 3 * kBig; }
    __device__ float *cols_rn(char *x) const { return reinterpret_cast<float *>(x) + 4 * kBig; }
    __device__ uint32_t *und_bits(char *x) const { return reinterpret_cast<uint32_t *>(x) + 5 * kBig; }
    __device__ bool prologue(char *x, int64_t a0, int64_t b0) const {
        const int n_ref = *a.n_ref;
        bool live = false;
        if (threadIdx.x < kBig) {
            const int64_t r = row0 + a0 + threadIdx.x;
            int e = -1, np = 0;
            float qv = 0.0f, un = 0.0f;
            if (r < n_ref) {
                e = a.ref_idx[r];
                np = a.nproc[e];
                qv = a.qip[e];
                if (a.ipbound) un = user_rnorm[a.ref_user[r]];
            }
            rows_e(x)[threadIdx.x] = e;
            rows_np(x)[threadIdx.x] = np;
            rows_qv(x)[threadIdx.x] = qv;
            rows_un(x)[threadIdx.x] = un;
            const int64_t it = b0 + threadIdx.x;
            cols_rn(x)[threadIdx.x] = a.ipbound && it < a.n_item ? __ldg(item_rnorm + it) : 0.0f;
            live = b0 < np;
        }
        return __syncthreads_or(live);
    }
    __device__ void finish_lo(char *x, const BigResult &res, int64_t, int64_t b0) const {
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7;
        const int e = rows_e(x)[ra];
        uint32_t bits[2] = {0u, 0u};
        if (e >= 0) {
            const int np = rows_np(x)[ra];
            const float qv = rows_qv(x)[ra], un = rows_un(x)[ra];
            const float lowq = __fsub_rn(qv, 8e-3f), highq = __fadd_rn(qv, 8e-3f);
            const float *rn = cols_rn(x);
            int c = 0, und = 0;
            for (int i = 0; i < kBig / 2; i++) {
                const int rb = half + 2 * i;
                if (b0 + rb >= np) break;
                const float lo = res.v[rb][ra];
                if (a.ipbound) {
                    const float right = __fmul_rn(rn[rb], un);
                    const float lbv = __fsub_rn(lo, right), ubv = __fadd_rn(lo, right);
                    if (lowq > ubv) continue;
                    if (highq < lbv) { c++; continue; }
                    und++;
                    bits[i >> 5] |= 1u << (i & 31);
                } else {
                    c += lo > qv;
                }
            }
            if (c) atomicAdd(a.rank + e, c);
            if (und) atomicAdd(a.undecided + e, und);
        }
        und_bits(x)[2 * threadIdx.x] = bits[0];
        und_bits(x)[2 * threadIdx.x + 1] = bits[1];
    }
    __device__ void finish_hi(char *x, const BigResult &res, int64_t, int64_t, char *) const {
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7;
        const int e = rows_e(x)[ra];
        if (e < 0) return;
        const float qv = rows_qv(x)[ra];
        int c = 0;
        for (int w = 0; w < 2; w++)
            for (uint32_t m = und_bits(x)[2 * threadIdx.x + w]; m; m &= m - 1) {
                const int i = 32 * w + __ffs(m) - 1;
                c += res.v[half + 2 * i][ra] >= qv;
            }
        if (c) atomicAdd(a.rank + e, c);
    }
};

// ============================================================================================
// assembly
// ============================================================================================

constexpr int kSortCap = 4096;

struct AssembleArgs {
    const QueryCounts *counts;
    const int64_t *cand_off;
    const int32_t *res_user;     // [n_query][topk]
    const int32_t *res_rank;     // [n_query][topk]
    const float *res_qip;        // [n_query][topk]
    const int32_t *cand_user;
    const int32_t *cand_rank;
    const float *cand_qip;
    const int32_t *cand_nproc;
    const int32_t *cand_undecided;
    const int32_t *cand_lb, *cand_ub;
    int topk;
    int ipbound, dim, check_dim;
    rkr_user_rank *out;          // [n_query][topk]
    rkr_query_stats *stats;      // [n_query] or nullptr
    uint64_t *scratch;           // keys for candidates beyond kSortCap (indexed by candidate)
};

__device__ __forceinline__ uint64_t cand_key(int rank, int user) {
    return ((uint64_t) (uint32_t) rank << 32) | (uint32_t) user;
}

// Results in user-id order with rank = lower bound, then the candidates sorted by
// (rank, user id) (ComputeAllIPBound.hpp:366-367 and UserRankElement::operator<), until top-k
// entries are filled (QS.hpp:185-198).
__global__ void assemble_kernel(AssembleArgs a) {
    __shared__ uint64_t keys[kSortCap];
    __shared__ int n_refined, warp_tot[9];
    __shared__ int64_t n_items, ip_refine;
    __shared__ uint64_t thresh;
    const int q = blockIdx.x;
    const QueryCounts c = a.counts[q];
    const int topk = a.topk;
    rkr_user_rank *out = a.out + (int64_t) q * topk;
    const int nres = c.n_res_emit;
    for (int k = threadIdx.x; k < nres; k += blockDim.x) {
        const int64_t i = (int64_t) q * topk + k;
        out[k].user_id = a.res_user[i];
        out[k].rank = a.res_rank[i];
        out[k].query_ip = a.res_qip[i];
    }
    const int64_t off = a.cand_off[q];
    const int nc = c.n_cand;
    const int m = min(topk - nres, nc);
    if (threadIdx.x == 0) { n_refined = 0; n_items = 0; ip_refine = 0; }
    __syncthreads();
    for (int e = threadIdx.x; e < nc; e += blockDim.x) {
        if (a.cand_lb[off + e] != a.cand_ub[off + e]) {
            const int np = a.cand_nproc[off + e];
            atomicAdd(&n_refined, 1);
            atomicAdd((unsigned long long *) &n_items, (unsigned long long) np);
            // RefineCPUIPBound.hpp:491,518 (bound pass plus items scored in full); ComputeAll.hpp:112-116
            const int64_t cost = a.ipbound ? (int64_t) (int) (np * 1.0 * (a.check_dim + 1) / a.dim) + a.cand_undecided[off + e]
                                           : (int64_t) np;
            atomicAdd((unsigned long long *) &ip_refine, (unsigned long long) cost);
        }
    }
    if (m > 0) {
        if (nc <= kSortCap) {
            int n2 = 1;
            while (n2 < nc) n2 <<= 1;
            for (int e = threadIdx.x; e < n2; e += blockDim.x)
                keys[e] = e < nc ? cand_key(a.cand_rank[off + e], a.cand_user[off + e]) : ~0ull;
            __syncthreads();
            for (int k = 2; k <= n2; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = threadIdx.x; i < n2; i += blockDim.x) {
                        const int p = i ^ j;
                        if (p > i) {
                            const bool up = (i & k) == 0;
                            const uint64_t x = keys[i], y = keys[p];
                            if ((x > y) == up) { keys[i] = y; keys[p] = x; }
                        }
                    }
                    __syncthreads();
                }
        } else {
            // m-th smallest key by an 8-pass radix select over the candidates, then sort the <= m keys.
            int *hist = reinterpret_cast<int *>(keys);  // 256 ints
            uint64_t prefix = 0;
            int want = m;  // rank (1-based) of the target among keys matching prefix
            for (int pass = 7; pass >= 0; pass--) {
                const int shift = 8 * pass;
                const uint64_t hmask = pass == 7 ? 0ull : (~0ull << (shift + 8));
                for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
                __syncthreads();
                for (int e = threadIdx.x; e < nc; e += blockDim.x) {
                    const uint64_t kk = cand_key(a.cand_rank[off + e], a.cand_user[off + e]);
                    if ((kk & hmask) == prefix) atomicAdd(&hist[(kk >> shift) & 255], 1);
                }
                __syncthreads();
                if (threadIdx.x == 0) {
                    int cum = 0, b = 0;
                    for (; b < 256; b++) {
                        if (cum + hist[b] >= want) break;
                        cum += hist[b];
                    }
                    want -= cum;
                    thresh = prefix | ((uint64_t) b << shift);
                }
                __syncthreads();
                prefix = thresh;
                __syncthreads();
            }
            // collect the keys <= the m-th smallest (exactly m of them: keys are unique)
            __shared__ int n_sel;
            if (threadIdx.x == 0) n_sel = 0;
            __syncthreads();
            for (int e = threadIdx.x; e < nc; e += blockDim.x) {
                const uint64_t kk = cand_key(a.cand_rank[off + e], a.cand_user[off + e]);
                if (kk <= prefix) {
                    const int s = atomicAdd(&n_sel, 1);
                    keys[s] = kk;
                }
            }
            __syncthreads();
            int n2 = 1;
            while (n2 < m) n2 <<= 1;
            for (int e = m + threadIdx.x; e < n2; e += blockDim.x) keys[e] = ~0ull;
            __syncthreads();
            for (int k = 2; k <= n2; k <<= 1)
                for (int j = k >> 1; j > 0; j >>= 1) {
                    for (int i = threadIdx.x; i < n2; i += blockDim.x) {
                        const int p = i ^ j;
                        if (p > i) {
                            const bool up = (i & k) == 0;
                            const uint64_t x = keys[i], y = keys[p];
                            if ((x > y) == up) { keys[i] = y; keys[p] = x; }
                        }
                    }
                    __syncthreads();
                }
        }
        __syncthreads();
        // Map each selected key back to its candidate for the score.
        for (int e = threadIdx.x; e < nc; e += blockDim.x) {
            const uint64_t kk = cand_key(a.cand_rank[off + e], a.cand_user[off + e]);
            int lo = 0, len = m;  // position of kk among the m smallest (sorted)
            while (len > 0) {
                const int h = len >> 1, mid = lo + h;
                if (keys[mid] < kk) { lo = mid + 1; len -= h + 1; } else len = h;
            }
            if (lo < m && keys[lo] == kk) {
                out[nres + lo].user_id = a.cand_user[off + e];
                out[nres + lo].rank = a.cand_rank[off + e];
                out[nres + lo].query_ip = a.cand_qip[off + e];
            }
        }
    }
    for (int k = nres + max(m, 0) + threadIdx.x; k < topk; k += blockDim.x) {
        out[k].user_id = -1;
        out[k].rank = -1;
        out[k].query_ip = -1.0f;
    }
    __syncthreads();
    if (a.stats && threadIdx.x == 0) {
        rkr_query_stats s;
        s.n_prune = c.n_prune;
        s.n_result = c.n_result;
        s.n_refine = n_refined;
        s.n_candidate = nc;
        s.n_compute_item = n_items;
        s.ip_cost = (int64_t) c.ip_base + ip_refine;
        a.stats[q] = s;
    }
}

// Ranks and exact scores of the emitted result users (QS/US): rank = lower bound of the bucket,
// score = InnerProduct(query, user).
__global__ void result_fill_kernel(const QueryCounts *__restrict__ counts, const int32_t *__restrict__ res_user,
                                   const uint16_t *__restrict__ bucket, int64_t n_user, const float *__restrict__ user,
                                   const float *__restrict__ query, int dim, int S, const int32_t *__restrict__ rank,
                                   int n_item, int topk, int32_t *__restrict__ res_rank, float *__restrict__ res_qip) {
    const int q = blockIdx.x;
    const int n = counts[q].n_res_emit;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int64_t i = (int64_t) q * topk + k;
        const int u = res_user[i];
        int lb, ub;
        bucket_bounds(bucket[(int64_t) q * n_user + u], S, rank, n_item, lb, ub);
        res_rank[i] = lb;
        res_qip[i] = exact_dot(query + (int64_t) q * dim, user + (int64_t) u * dim, dim);
    }
}

// Bounds of each candidate from its bucket.
__global__ void cand_bounds_kernel(const uint16_t *__restrict__ cand_bucket, int64_t n, int S,
                                   const int32_t *__restrict__ rank, int n_item, int32_t *__restrict__ lb_out,
                                   int32_t *__restrict__ ub_out) {
    const int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    int lb, ub;
    bucket_bounds(cand_bucket[e], S, rank, n_item, lb, ub);
    lb_out[e] = lb;
    ub_out[e] = ub;
}

// ============================================================================================
// host orchestration
// ============================================================================================

namespace {

template <typename T> T *carve(uint8_t *&p, size_t n) {
    uintptr_t v = reinterpret_cast<uintptr_t>(p);
    v = (v + 255) & ~uintptr_t(255);
    T *r = reinterpret_cast<T *>(v);
    p = reinterpret_cast<uint8_t *>(v + n * sizeof(T));
    return r;
}

inline size_t carve_size(size_t n, size_t elem) { return ((n * elem + 255) & ~size_t(255)) + 256; }

}  // namespace

// Runs candidate refinement and assembly for one chunk whose candidates are listed in the pool.
static int refine_and_assemble(rkr_index *ix, int method, const float *d_query, int nq, int topk,
                               const QueryCounts *d_counts, const std::vector<QueryCounts> &h_counts,
                               const int32_t *d_res_user, const int32_t *d_res_rank, const float *d_res_qip,
                               int64_t n_cand, int32_t *d_cand_user, int32_t *d_cand_query, int32_t *d_cand_lb,
                               int32_t *d_cand_ub, const float *d_cand_qip_given, const int64_t *d_cand_off,
                               rkr_user_rank *d_out, rkr_query_stats *d_stats, cudaStream_t st) {
    const bool ipbound = method != RKR_METHOD_US;
    size_t need = carve_size(n_cand, 4) * 7 + carve_size(1, 4) + carve_size((size_t) ix->dim * kmajor_ld(n_cand), 4);
    RKR_TRY(ix->ws_refine.ensure(need));
    uint8_t *p = ix->ws_refine.as<uint8_t>();
    float *qip = carve<float>(p, n_cand);
    int32_t *rank = carve<int32_t>(p, n_cand);
    int32_t *nproc = carve<int32_t>(p, n_cand);
    int32_t *ref_idx = carve<int32_t>(p, n_cand);
    int32_t *ref_user = carve<int32_t>(p, n_cand);
    int32_t *undecided = carve<int32_t>(p, n_cand);
    int32_t *n_ref = carve<int32_t>(p, 1);
    float *cand_km = carve<float>(p, (size_t) ix->dim * kmajor_ld(n_cand));
    RKR_CUDA(cudaMemsetAsync(n_ref, 0, sizeof(int32_t), st));
    RKR_CUDA(cudaMemsetAsync(ref_user, 0, sizeof(int32_t) * n_cand, st));
    if (n_cand > 0) {
        RefineArgs ra;
        ra.user = ix->user.as<float>();
        ra.query = d_query;
        ra.cand_qip = d_cand_qip_given;
        ra.cand_user = d_cand_user;
        ra.cand_query = d_cand_query;
        ra.cand_lb = d_cand_lb;
        ra.cand_ub = d_cand_ub;
        ra.n_cand = n_cand;
        ra.dim = ix->dim;
        ra.ipbound = ipbound ? 1 : 0;
        ra.item_norm = ix->item_norm.as<float>();
        ra.n_item = ix->n_item;
        ra.qip = qip;
        ra.rank = rank;
        ra.nproc = nproc;
        ra.ref_idx = ref_idx;
        ra.ref_user = ref_user;
        ra.n_ref = n_ref;
        ra.undecided = undecided;
        timed(ix, st, "refine_prep", [&] { refine_prep_kernel<<<(unsigned) ((n_cand + 255) / 256), 256, 0, st>>>(ra); });
        RKR_CUDA(cudaGetLastError());
        bool tc_done = false;
        if (ix->refine_tc_on) RKR_TRY(refine_tc(ix, ra, st, &tc_done));
        if (!tc_done) {
        // the refined candidates' user vectors, gathered k-major (rows past n_ref gather user 0)
        timed(ix, st, "refine_gather", [&] { to_kmajor(ix->user.as<float>(), ref_user, n_cand, ix->dim, cand_km, st); });
        RKR_CUDA(cudaGetLastError());
        const KMajor items = {ipbound ? ix->item_sorted_km.as<float>() : ix->item_km.as<float>(), ix->n_item,
                              kmajor_ld(ix->n_item), kmajor_ld(ix->n_item)};
        RefineEpi re;
        re.a = ra;
        re.item_rnorm = ix->item_rnorm.as<float>();
        re.user_rnorm = ix->user_rnorm.as<float>();
        const int k_split = ipbound ? ix->check_dim : ix->dim;
        const int64_t per = (int64_t) 65535 * kBig;
        const int64_t ldc = kmajor_ld(n_cand);
        for (int64_t r0 = 0; r0 < n_cand; r0 += per) {
            re.row0 = r0;
            const KMajor cands = {cand_km + r0, std::min(per, n_cand - r0), ldc, ldc - r0};
            cudaError_t ce = cudaSuccess;
            timed(ix, st, "refine_tile", [&] { ce = launch_big_split(cands, items, k_split, ix->dim, re, st); });
            RKR_CUDA(ce);
        }
        }
    }
    AssembleArgs aa;
    aa.counts = d_counts;
    aa.cand_off = d_cand_off;
    aa.res_user = d_res_user;
    aa.res_rank = d_res_rank;
    aa.res_qip = d_res_qip;
    aa.cand_user = d_cand_user;
    aa.cand_rank = rank;
    aa.cand_qip = qip;
    aa.cand_nproc = nproc;
    aa.cand_undecided = undecided;
    aa.ipbound = ipbound ? 1 : 0;
    aa.dim = ix->dim;
    aa.check_dim = ix->check_dim;
    aa.cand_lb = d_cand_lb;
    aa.cand_ub = d_cand_ub;
    aa.topk = topk;
    aa.out = d_out;
    aa.stats = d_stats;
    aa.scratch = nullptr;
    timed(ix, st, "assemble", [&] { assemble_kernel<<<nq, 256, 0, st>>>(aa); });
    RKR_CUDA(cudaGetLastError());
    (void) h_counts;
    return RKR_OK;
}

// QS and US: one chunk of queries.
static int qs_chunk(rkr_index *ix, int method, const float *d_query, int nq, int topk, rkr_user_rank *d_out,
                    rkr_query_stats *d_stats, cudaStream_t st) {
    const int64_t U = ix->n_user;
    const int S = ix->n_sample;
    const int dim = ix->dim;
    RKR_TRY(ix->ws_bucket.ensure((size_t) nq * (size_t) U * sizeof(uint16_t)));
    uint16_t *bucket = ix->ws_bucket.as<uint16_t>();
    RKR_TRY(ix->ws_cls.ensure((size_t) nq * (S + 1)));
    RKR_TRY(ix->ws_counts.ensure(sizeof(QueryCounts) * (size_t) nq));
    RKR_TRY(ix->ws_hist.ensure(sizeof(int) * (size_t) nq * (S + 1)));
    QueryCounts *counts = ix->ws_counts.as<QueryCounts>();
    int *hist = ix->ws_hist.as<int>();
    {
        QsBucketEpi epi;
        epi.thr = ix->thr.as<float>();
        epi.n_user = U;
        epi.n_query = nq;
        epi.S = S;
        epi.bucket = bucket;
        cudaError_t e = cudaSuccess;
        timed(ix, st, "score_bucket", [&] {
            e = launch_big(ix->user.as<float>(), nullptr, U, dim, d_query, nq, dim, 0, dim, epi, st);
        });
        RKR_CUDA(e);
        RKR_CUDA(cudaMemsetAsync(hist, 0, sizeof(int) * (size_t) nq * (S + 1), st));
        const int64_t chunk = 16384;
        dim3 hg((unsigned) ((U + chunk - 1) / chunk), (unsigned) nq);
        timed(ix, st, "bucket_hist", [&] {
            bucket_hist_kernel<<<hg, kHistThreads, hist_copies(S + 1) * (S + 1) * sizeof(int), st>>>(bucket, U, S + 1,
                                                                                                  chunk, hist);
        });
        RKR_CUDA(cudaGetLastError());
        timed(ix, st, "select_bucket", [&] {
            select_bucket_kernel<<<nq, 32, 0, st>>>(hist, S, ix->sample_rank.as<int32_t>(), (int) ix->n_item, topk,
                                                   (int) U, ix->ws_cls.as<uint8_t>(), counts);
        });
        RKR_CUDA(cudaGetLastError());
    }
    std::vector<QueryCounts> hc(nq);
    RKR_CUDA(cudaMemcpyAsync(hc.data(), counts, sizeof(QueryCounts) * nq, cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    std::vector<int64_t> off(nq + 1, 0);
    for (int q = 0; q < nq; q++) off[q + 1] = off[q] + hc[q].n_cand;
    const int64_t n_cand = off[nq];
    size_t need = carve_size(nq + 1, 8) + carve_size((size_t) nq * topk, 4) * 3 + carve_size(n_cand, 4) * 4 +
                  carve_size(n_cand, 2);
    RKR_TRY(ix->ws_cand.ensure(need));
    uint8_t *p = ix->ws_cand.as<uint8_t>();
    int64_t *d_off = carve<int64_t>(p, nq + 1);
    int32_t *res_user = carve<int32_t>(p, (size_t) nq * topk);
    int32_t *res_rank = carve<int32_t>(p, (size_t) nq * topk);
    float *res_qip = carve<float>(p, (size_t) nq * topk);
    int32_t *cand_user = carve<int32_t>(p, n_cand);
    int32_t *cand_query = carve<int32_t>(p, n_cand);
    int32_t *cand_lb = carve<int32_t>(p, n_cand);
    int32_t *cand_ub = carve<int32_t>(p, n_cand);
    uint16_t *cand_bucket = carve<uint16_t>(p, n_cand);
    RKR_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(int64_t) * (nq + 1), cudaMemcpyHostToDevice, st));
    QsCompactPolicy pol;
    pol.bucket = bucket;
    pol.n_user = U;
    pol.cls = ix->ws_cls.as<uint8_t>();
    pol.S = S;
    pol.counts = counts;
    pol.cand_off = d_off;
    pol.topk = topk;
    pol.res_user = res_user;
    pol.cand_user = cand_user;
    pol.cand_query = cand_query;
    pol.cand_bucket = cand_bucket;
    RKR_TRY(run_compaction(ix, pol, nq, topk, counts, st));
    timed(ix, st, "result_fill", [&] {
        result_fill_kernel<<<nq, 128, 0, st>>>(counts, res_user, bucket, U, ix->user.as<float>(), d_query, dim, S,
                                               ix->sample_rank.as<int32_t>(), (int) ix->n_item, topk, res_rank, res_qip);
    });
    RKR_CUDA(cudaGetLastError());
    if (n_cand > 0) {
        timed(ix, st, "cand_bounds", [&] {
            cand_bounds_kernel<<<(unsigned) ((n_cand + 255) / 256), 256, 0, st>>>(
                cand_bucket, n_cand, S, ix->sample_rank.as<int32_t>(), (int) ix->n_item, cand_lb, cand_ub);
        });
        RKR_CUDA(cudaGetLastError());
    }
    RKR_TRY(refine_and_assemble(ix, method, d_query, nq, topk, counts, hc, res_user, res_rank, res_qip, n_cand,
                                cand_user, cand_query, cand_lb, cand_ub, nullptr, d_off, d_out, d_stats, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    return RKR_OK;
}

int qsrp_chunk(rkr_index *ix, const float *d_query, int nq, int topk, rkr_user_rank *d_out, rkr_query_stats *d_stats,
               cudaStream_t st);

int refine_and_assemble_qsrp(rkr_index *ix, const float *d_query, int nq, int topk, const QueryCounts *d_counts,
                             const int32_t *d_res_user, const int32_t *d_res_rank, const float *d_res_qip, int64_t n_cand,
                             int32_t *d_cand_user, int32_t *d_cand_query, int32_t *d_cand_lb, int32_t *d_cand_ub,
                             const float *d_cand_qip, const int64_t *d_cand_off, rkr_user_rank *d_out,
                             rkr_query_stats *d_stats, cudaStream_t st) {
    std::vector<QueryCounts> unused;
    return refine_and_assemble(ix, RKR_METHOD_QSRP_NORMAL_LP, d_query, nq, topk, d_counts, unused, d_res_user, d_res_rank,
                               d_res_qip, n_cand, d_cand_user, d_cand_query, d_cand_lb, d_cand_ub, d_cand_qip, d_cand_off,
                               d_out, d_stats, st);
}

int query_batch(rkr_index *ix, int method, const float *d_query, int n_query, int topk, rkr_user_rank *d_out,
                rkr_query_stats *d_stats, cudaStream_t st) {
    // Chunk so the per-pair bucket array stays within a bounded slice of device memory.
    const int64_t budget = int64_t(6) << 30;
    int64_t per_q = ix->n_user * 4 + 4096;
    int chunk = (int) std::max<int64_t>(1, std::min<int64_t>(n_query, budget / per_q));
    chunk = std::min(chunk, 4096);
    for (int q0 = 0; q0 < n_query; q0 += chunk) {
        const int nq = std::min(chunk, n_query - q0);
        const float *dq = d_query + (int64_t) q0 * ix->dim;
        rkr_user_rank *dout = d_out + (int64_t) q0 * topk;
        rkr_query_stats *dst = d_stats ? d_stats + q0 : nullptr;
        if (method == RKR_METHOD_QSRP_NORMAL_LP) {
            RKR_TRY(qsrp_chunk(ix, dq, nq, topk, dout, dst, st));
        } else {
            RKR_TRY(qs_chunk(ix, method, dq, nq, topk, dout, dst, st));
        }
    }
    return RKR_OK;
}

}  // namespace rkr
