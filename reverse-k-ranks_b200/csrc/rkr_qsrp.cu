// rkr_qsrp.cu -- QSRPNormalLP retrieval on the device (src/impl/QSRPNormalLP.hpp:116-260).
//
// Per query the reference runs two bound/prune rounds before refinement:
//   1. SVD-space partial score on the first check_dim coordinates +- the product of the remaining
//      norms (PartDimPartNorm::IPBound, PartDimPartNorm.hpp:52-74) -> regression rank bounds
//      (NormalLinearRegressionLP::ComputeRankBound, NormalLinearRegressionLP.hpp:326-398) -> prune.
//   2. full SVD-space score for the survivors (ComputeRemainDim, :76-95) -> sampled-threshold
//      bounds (SampleSearch::RankBound) -> prune again.
// Here a batch of queries runs as passes over all (query, user) pairs:
//   * one kernel scores every pair and decides its round-1 levels and the coarse group of its
//     sampled-threshold bucket (a per-user summary of every 16th threshold): on the tensor cores
//     (rkr_scores_tc.cu: int8 digit products, a rigorous bound against the reference's sums, exact
//     resolution of the pairs the bound leaves undecided), or, where that path does not fit, as
//     exact SIMT tiles (Round1Epi below: exact scores, a fast binary32 screen of the regression
//     arithmetic, undecided pairs fixed by the reference's own arithmetic);
//   * round 2 is a streaming pass that marks the pairs that did not survive round 1 and counts the
//     survivors by group;
//   * the exact bucket is resolved only where the k-th bound and the class counts need it: for the
//     pairs in the critical group(s) of each query, and for the users that end up reported, from
//     recomputed scores.
// The reference keeps its per-user score vector across queries; users accepted in round 1 are
// reported with whatever that vector holds for them.  The batch reproduces it: the score a user had
// at its latest earlier query in which it reached round 2, or the index's carried state when there
// is none.
#include <algorithm>
#include <vector>

#include "rkr_internal.cuh"
#include "rkr_regression.cuh"

namespace rkr {

// in rkr_query.cu
int refine_and_assemble_pairs(rkr_index *ix, int method, const float *d_query, int nq, int topk,
                              const QueryCounts *d_counts, const int32_t *d_res_user, const int32_t *d_res_rank,
                              const float *d_res_qip, int64_t n_cand, int32_t *d_cand_user, int32_t *d_cand_query,
                              int32_t *d_cand_lb, int32_t *d_cand_ub, const float *d_cand_qip,
                              const int64_t *d_cand_off, rkr_user_rank *d_out, rkr_query_stats *d_stats,
                              cudaStream_t st);

// ---- per-query state ---------------------------------------------------------------------------------

// Round-2 codes per pair: 0..nb a coarse threshold group (nb: bucket S); otherwise the round-1 state.
constexpr uint8_t kCodeResult1 = 0xfe, kCodePruned1 = 0xff;
constexpr uint8_t kClsMixed = 0xff;  // a group whose buckets fall in more than one class

struct QsrpParams {
    int32_t mode1, all1, L1, U1;           // round 1: equal-bounds mode, "all survivors accepted", k-th bounds
    int32_t n_res1, n_pr1, n_ref1, skip2;  // round-1 counts; skip2: round 1 already produced top-k results
    int32_t mode2, L2, U2, n_elig2;        // round 2
    int32_t exact1, lv_res, lv_pr, lv_m1;  // exact1: count round-1 classes pair by pair; level thresholds
    int32_t crit, cum_before, mask1, mask2;  // critical coarse group, users below it, groups to resolve
    int32_t gneed_lo, gneed_hi, pad0, pad1;  // groups 0..31 / 32 whose pairs the compaction must classify
};

// Round-1 class in level space: rank(level) is non-decreasing in the level, so lb <= U1 is
// lvl_lb <= lv_res, L1 <= ub is lvl_ub >= lv_pr and the equal-bounds test is a test against lv_m1.
__device__ __forceinline__ int class1_lv(const QsrpParams &p, int l, int h) {
    if (p.mode1) return (h <= p.lv_m1 && l <= p.lv_m1) ? kClsResult : kClsIdle;
    if (l <= p.lv_res) return kClsResult;
    if (h >= p.lv_pr) return kClsPrune;
    return p.all1 ? kClsResult : kClsRefine;
}

__device__ __forceinline__ int class1_of(const QsrpParams &p, int lb, int ub) {
    if (p.mode1) return (ub <= p.L1 && lb <= p.L1) ? kClsResult : kClsIdle;
    if (lb <= p.U1) return kClsResult;
    if (p.L1 <= ub) return kClsPrune;
    return p.all1 ? kClsResult : kClsRefine;
}

// ---- round 1 + full scores -------------------------------------------------------------------------

// SVD::TransferQuery (SVD.hpp:156-164) and the query's remaining-dims norm (PartDimPartNorm.hpp:56-57).
__global__ void transfer_query_kernel(const float *__restrict__ query, const float *__restrict__ transfer, int dim,
                                      int check_dim, float *__restrict__ qtr, float *__restrict__ qnorm) {
    const int q = blockIdx.x;
    const float *qv = query + (int64_t) q * dim;
    float *out = qtr + (int64_t) q * dim;
    for (int t = threadIdx.x; t < dim; t += blockDim.x) out[t] = exact_dot(transfer + (int64_t) t * dim, qv, dim);
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int j = check_dim; j < dim; j++) s = __fadd_rn(s, __fmul_rn(out[j], out[j]));
        qnorm[q] = __fsqrt_rn(s);
    }
}

// Exact SVD-space partial score of (query, user) over the first check_dim coordinates
// (PartDimPartNorm.hpp:62).
struct ScoreSrc {
    const float *svd_user, *qtr;
    int dim, c;
    __device__ float left(int64_t u, int64_t q) const { return exact_dot(svd_user + u * dim, qtr + q * dim, c); }
};

// The batch's full scores as the tile kernel stored them ([query][user]).
struct QipView {
    float *qip;
    int64_t n_user;
    // the reference's score of a pair: a sum over [0, c) and one over [c, dim), added once (c == dim:
    // one sum); the user rows are SVD-space for QSRP
    const float *urow, *qrow;
    int dim, c;
    PairScreen scr;  // scr.umeta null: the stored scores are the reference's
    // stored values are read through L2: passes write recomputed scores back
    __device__ float stored(int64_t u, int64_t q) const { return __ldcg(qip + q * n_user + u); }
    __device__ bool is_exact(int64_t u, int64_t q) const {
        if (!scr.umeta) return true;
        const int64_t words = (n_user + 31) >> 5;
        return (__ldcg(scr.xbits + q * words + (u >> 5)) >> (u & 31)) & 1u;
    }
    // The reference's score; a recomputed one is stored back and marked, so that later passes
    // over the same pair read it.
    __device__ float exact(int64_t u, int64_t q) const {
        const int64_t o = q * n_user + u;
        if (is_exact(u, q)) return __ldcg(qip + o);
        const float *ur = urow + u * dim, *qr = qrow + q * dim;
        const float left = exact_dot(ur, qr, c);
        const float v = c < dim ? __fadd_rn(left, exact_dot(ur + c, qr + c, dim - c)) : left;
        qip[o] = v;
        __threadfence();
        atomicOr(scr.xbits + q * ((n_user + 31) >> 5) + (u >> 5), 1u << (u & 31));
        if (scr.n_exact) atomicAdd(scr.n_exact, 1);
        return v;
    }
    // distance bound between a stored score s and the reference's
    __device__ float delta(int64_t u, int64_t q, float s) const {
        const float4 um = __ldg(scr.umeta + u), qm = __ldg(scr.qmeta + q);
        const float ee = um.x * qm.x;
        // per part: the weighted-norm term, the digits' term and the combination's leading term
        // 3.002 u |part| <= 2.2 u Wa Wb (|part| <= Wa Wb / sqrt 2: every weight is at least 2)
        const float nl = um.y * qm.y, nr = um.z * qm.z;
        const float d = fmaf(scr.cl + 1.32e-7f, nl, ee * scr.kl) + fmaf(scr.cr + 1.32e-7f, nr, ee * scr.kr);
        return fmaf(fabsf(s), 2.4e-7f, d * 1.0001f);
    }
};

// The bucket of s inside coarse group g (< nb): g * gs + the group's thresholds >= s.
__device__ __forceinline__ int fine_bucket(const float *__restrict__ row, int S, int gs, int g, float s) {
    const int base = g * gs, end = min(base + gs, S);
    int c = 0;
    if ((gs & 15) == 0 && end - base == gs && (S & 3) == 0) {
        const float4 *p = reinterpret_cast<const float4 *>(row + base);
        for (int t = 0; t < gs / 16; t++, p += 4) {
            const float4 x0 = __ldg(p), x1 = __ldg(p + 1), x2 = __ldg(p + 2), x3 = __ldg(p + 3);
            c += (x0.x >= s) + (x0.y >= s) + (x0.z >= s) + (x0.w >= s) + (x1.x >= s) + (x1.y >= s) + (x1.z >= s) +
                 (x1.w >= s) + (x2.x >= s) + (x2.y >= s) + (x2.z >= s) + (x2.w >= s) + (x3.x >= s) + (x3.y >= s) +
                 (x3.z >= s) + (x3.w >= s);
        }
    } else {
        for (int i = base; i < end; i++) c += __ldg(row + i) >= s;
    }
    return base + c;
}

// Thresholds of group g (< nb) >= hi and >= lo, in one pass.
__device__ __forceinline__ void fine_bucket2(const float *__restrict__ row, int S, int gs, int g, float hi, float lo,
                                             int &b_hi, int &b_lo) {
    const int base = g * gs, end = min(base + gs, S);
    int ch = 0, cl = 0;
    if ((gs & 3) == 0 && end - base == gs && (S & 3) == 0) {
        const float4 *p = reinterpret_cast<const float4 *>(row + base);
        for (int t = 0; t < gs / 4; t++) {
            const float4 x = __ldg(p + t);
            ch += (x.x >= hi) + (x.y >= hi) + (x.z >= hi) + (x.w >= hi);
            cl += (x.x >= lo) + (x.y >= lo) + (x.z >= lo) + (x.w >= lo);
        }
    } else {
        for (int i = base; i < end; i++) {
            const float x = __ldg(row + i);
            ch += x >= hi;
            cl += x >= lo;
        }
    }
    b_hi = base + ch;
    b_lo = base + cl;
}

// The bucket (inside its coarse group g) of a pair's reference score: from the stored score when it
// is exact or no threshold lies within its bound, else from the recomputed score.
__device__ __forceinline__ int pair_bucket(const QipView &sc, const float *__restrict__ thr, int S, int gs, int g,
                                           int64_t u, int64_t q) {
    const float *row = thr + u * S;
    if (sc.is_exact(u, q)) return fine_bucket(row, S, gs, g, sc.stored(u, q));  // the bit first, then the value
    const float s = sc.stored(u, q);
    const float d = sc.delta(u, q, s);
    int b_hi, b_lo;
    fine_bucket2(row, S, gs, g, s + d, s - d, b_hi, b_lo);
    if (b_hi == b_lo) return b_hi;
    return fine_bucket(row, S, gs, g, sc.exact(u, q));
}

// Pairs the screen left undecided, resolved by qsrp_fix1_kernel: (query, user, partial score).
// Past the list's capacity the pair's levels are written as kLvUndecided and count keeps growing,
// which sends qsrp_fix1_scan_kernel over the whole batch.
struct FixList {
    int4 *e;
    int *count;
    int cap;
};
constexpr uint32_t kLvUndecided = 0xffffffffu;

// Tiles of 128 users x 128 queries: the partial score over the first check_dim coordinates, the
// bounds partial -+ norms and their regression levels (lb | ub << 16); then the full score and the
// coarse group of its sampled-threshold bucket (the round-2 code of the pair if it reaches round 2).
struct Round1Epi {
    static constexpr size_t kExtra = sizeof(float) * kBig;
    static constexpr int kSummStride = ThrSummary::kMaxGroups + 1;
    const float *unorm, *qnorm, *thr_summ;
    RegModel m;
    uint32_t *lv;
    uint8_t *code;
    float *qip;
    int nb;
    int64_t n_user, n_query;
    FixList fix;
    __device__ bool prologue(char *x, int64_t, int64_t b0) const {
        float *qn = reinterpret_cast<float *>(x);
        if (threadIdx.x < kBig) qn[threadIdx.x] = b0 + threadIdx.x < n_query ? __ldg(qnorm + b0 + threadIdx.x) : 0.0f;
        return true;
    }
    __device__ void finish_lo(char *x, const BigResult &res, int64_t a0, int64_t b0) const {
        if (!lv) return;  // no round 1 (QS, US)
        const float *qn = reinterpret_cast<const float *>(x);
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7, lane = threadIdx.x & 31;
        const int64_t u = a0 + ra;
        const unsigned alive = __ballot_sync(0xffffffffu, u < n_user);
        if (u >= n_user) return;
        const RegUser r = reg_user(m, u);
        const float un = __ldg(unorm + u);
        uint32_t *out = lv + (b0 + half) * n_user + u;
        const int64_t step = 2 * n_user;
        const int64_t left_rows = (n_query - b0 - half + 1) / 2;
        const int nrow = left_rows < kBig / 2 ? (int) left_rows : kBig / 2;
        // two queries per iteration: their screens are independent chains
        for (int i = 0; i < nrow; i += 2, out += 2 * step) {
            float left[2];
            uint32_t packed[2];
            bool ok[2];
#pragma unroll
            for (int g = 0; g < 2; g++) {
                const int rb = half + 2 * min(i + g, nrow - 1);
                left[g] = res.v[rb][ra];
                const float right = __fmul_rn(un, qn[rb]);
                int l, h;
                ok[g] = regression_levels_fast(r, m.S, __fsub_rn(left[g], right), __fadd_rn(left[g], right), l, h);
                packed[g] = (uint32_t) l | ((uint32_t) h << 16);
            }
            ok[1] = ok[1] || i + 1 >= nrow;
#pragma unroll
            for (int g = 0; g < 2; g++) {
                const unsigned need = __ballot_sync(alive, !ok[g]);
                if (need) {
                    const int leader = __ffs(need) - 1;
                    int base = 0;
                    if (lane == leader) base = atomicAdd(fix.count, __popc(need));
                    base = __shfl_sync(alive, base, leader);
                    if (!ok[g]) {
                        const int idx = base + __popc(need & ((1u << lane) - 1));
                        if (idx < fix.cap)
                            fix.e[idx] = make_int4((int) (b0 + half + 2 * (i + g)), (int) u, __float_as_int(left[g]), 0);
                        else packed[g] = kLvUndecided;
                    }
                }
            }
            out[0] = packed[0];
            if (i + 1 < nrow) out[step] = packed[1];
        }
    }
    __device__ void finish_hi(char *, const BigResult &res, int64_t a0, int64_t b0, char *spare) const {
        float *summ = reinterpret_cast<float *>(spare);  // [128][kSummStride]
        for (int idx = threadIdx.x; idx < kBig * ThrSummary::kMaxGroups; idx += kBigThreads) {
            const int rr = idx / ThrSummary::kMaxGroups, j = idx % ThrSummary::kMaxGroups;
            summ[rr * kSummStride + j] =
                a0 + rr < n_user ? __ldg(thr_summ + (a0 + rr) * ThrSummary::kMaxGroups + j) : 0.0f;
        }
        __syncthreads();
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7;
        const int64_t u = a0 + ra;
        if (u >= n_user) return;
        const float *sm = summ + ra * kSummStride;
        const int64_t base = (b0 + half) * n_user + u, step = 2 * n_user;
        const int64_t left_rows = (n_query - b0 - half + 1) / 2;
        const int nrow = left_rows < kBig / 2 ? (int) left_rows : kBig / 2;
        // Groups are the summary entries >= s (the summary descends; unused entries are -inf):
        // a fixed five-step search plus one compare, four queries at a time.
        constexpr int G = 4;
        for (int i0 = 0; i0 < nrow; i0 += G) {
            float sv[G];
            int lo[G];
#pragma unroll
            for (int g = 0; g < G; g++) {
                sv[g] = res.v[half + 2 * min(i0 + g, nrow - 1)][ra];
                lo[g] = 0;
            }
#pragma unroll
            for (int st = 16; st >= 1; st >>= 1)
#pragma unroll
                for (int g = 0; g < G; g++) lo[g] += sm[lo[g] + st - 1] >= sv[g] ? st : 0;
#pragma unroll
            for (int g = 0; g < G; g++) {
                lo[g] = min(lo[g] + (sm[lo[g]] >= sv[g]), nb);  // a score of -inf passes the padding too
                if (i0 + g < nrow) {
                    code[base + (i0 + g) * step] = (uint8_t) lo[g];
                    qip[base + (i0 + g) * step] = sv[g];
                }
            }
        }
    }
};

// The reference's arithmetic for the pairs the screen left undecided (the listed ones).
__global__ void qsrp_fix1_kernel(FixList fix, RegModel m, const float *__restrict__ unorm,
                                 const float *__restrict__ qnorm, int64_t n_user, uint32_t *__restrict__ lv) {
    const int n = min(*fix.count, fix.cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 e = fix.e[i];
        const float left = __int_as_float(e.z);
        const float right = __fmul_rn(__ldg(unorm + e.y), __ldg(qnorm + e.x));
        lv[(int64_t) e.x * n_user + e.y] =
            regression_levels_exact(m.rec, m.S, m.err_cap, e.y, __fsub_rn(left, right), __fadd_rn(left, right));
    }
}

// Undecided pairs beyond the list's capacity: a scan of the batch's levels for kLvUndecided, with the
// partial score recomputed.  Returns at once when the list held them all.
__global__ void qsrp_fix1_scan_kernel(const int *__restrict__ count, int cap, RegModel m, ScoreSrc sc,
                                      const float *__restrict__ unorm, const float *__restrict__ qnorm, int64_t n_user,
                                      int nq, uint32_t *__restrict__ lv) {
    if (*count <= cap) return;
    const int64_t n = n_user * nq;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        if (lv[i] != kLvUndecided) continue;
        const int64_t q = i / n_user, u = i % n_user;
        const float left = sc.left(u, q);
        const float right = __fmul_rn(__ldg(unorm + u), __ldg(qnorm + q));
        lv[i] = regression_levels_exact(m.rec, m.S, m.err_cap, u, __fsub_rn(left, right), __fadd_rn(left, right));
    }
}

// Histograms of the round-1 lower- and upper-bound levels per query, one CTA per (user chunk,
// query), counted in per-warp shared-memory copies; also counts pairs whose upper bound exceeds
// their lower bound (never expected, but it would void the shortcut qsrp_select1 takes for the
// class counts).
__global__ void __launch_bounds__(kHistThreads) level_hist_kernel(const uint32_t *__restrict__ lv, int64_t n_user,
                                                                 const int32_t *__restrict__ rank, int S, int n_item,
                                                                 int64_t chunk, int *__restrict__ hist,
                                                                 int *__restrict__ anomaly) {
    extern __shared__ int h[];
    __shared__ int anom;
    const int nl = S + 2, nb = 2 * nl;
    const int copies = hist_copies(nb);
    const int q = blockIdx.y;
    for (int b = threadIdx.x; b < copies * nb; b += blockDim.x) h[b] = 0;
    if (threadIdx.x == 0) anom = 0;
    __syncthreads();
    int *mine = h + ((threadIdx.x >> 5) % copies) * nb;
    const uint32_t *row = lv + (int64_t) q * n_user;
    const int64_t u0 = (int64_t) blockIdx.x * chunk, u1 = min(u0 + chunk, n_user);
    int my_anom = 0;
    constexpr int G = 8;  // loads in flight per thread
    for (int64_t ub = u0 + threadIdx.x; ub < u1; ub += G * kHistThreads) {
        uint32_t v[G];
#pragma unroll
        for (int g = 0; g < G; g++) v[g] = ub + g * kHistThreads < u1 ? __ldg(row + ub + g * kHistThreads) : 0xffffffffu;
#pragma unroll
        for (int g = 0; g < G; g++) {
            if (v[g] == 0xffffffffu) continue;
            const int l = v[g] & 0xffff, hh = v[g] >> 16;
            atomicAdd(mine + l, 1);
            atomicAdd(mine + nl + hh, 1);
            my_anom += hh > l && level_rank(hh, rank, S, n_item) > level_rank(l, rank, S, n_item);
        }
    }
    if (my_anom) atomicAdd(&anom, my_anom);
    __syncthreads();
    int *g = hist + (int64_t) q * nb;
    for (int b = threadIdx.x; b < nb; b += blockDim.x) {
        int sum = 0;
        for (int c = 0; c < copies; c++) sum += h[c * nb + b];
        if (sum) atomicAdd(g + b, sum);
    }
    if (threadIdx.x == 0 && anom) atomicAdd(anomaly + q, anom);
}

// ---- one warp per query -------------------------------------------------------------------------

__device__ __forceinline__ int64_t warp_sum64(int64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// First index b in [0, n) at which the running sum of h reaches need (n - 1 if it never does).
__device__ __forceinline__ int warp_first_reaching(const int *__restrict__ h, int n, int64_t need) {
    const int lane = threadIdx.x & 31;
    int64_t base = 0;
    for (int c0 = 0; c0 < n; c0 += 32) {
        const int b = c0 + lane;
        const int v = b < n ? h[b] : 0;
        const int incl = warp_incl_scan(v);
        const unsigned hit = __ballot_sync(0xffffffffu, b < n && base + incl >= need);
        if (hit) return c0 + __ffs(hit) - 1;
        base += __shfl_sync(0xffffffffu, incl, 31);
    }
    return n - 1;
}

// Round-1 k-th smallest bounds per query (PruneCandidateByBound.hpp:36-77 with nothing excluded)
// and the class counts, one warp per query.  While every pair has ub <= lb, a result (lb <= U*)
// and a prune (ub >= L*) cannot coincide unless L* == U*, so the counts follow from the two
// histograms; otherwise qsrp_count1 counts pair by pair.  rank(level) is non-decreasing, so the
// levels with rank <= X form a prefix and the thresholds are counts.
__global__ void qsrp_select1_kernel(const int *__restrict__ hist_all, const int *__restrict__ anomaly, int64_t n_user,
                                    const int32_t *__restrict__ rank, int S, int n_item, int topk, int nq,
                                    QsrpParams *__restrict__ par) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= nq) return;
    const int nl = S + 2;
    const int *h = hist_all + (int64_t) q * 2 * nl;
    const int kl = warp_first_reaching(h, nl, topk), kh = warp_first_reaching(h + nl, nl, topk);
    QsrpParams p = {};
    p.L1 = level_rank(kl, rank, S, n_item);
    p.U1 = level_rank(kh, rank, S, n_item);
    p.mode1 = p.L1 == p.U1;
    int64_t c_res = 0, c_m1 = 0, c_lt = 0;
    for (int l = lane; l < nl; l += 32) {
        const int rl = level_rank(l, rank, S, n_item);
        c_res += rl <= p.U1;
        c_m1 += rl <= p.L1;
        c_lt += rl < p.L1;
    }
    p.lv_res = (int) warp_sum64(c_res) - 1;
    p.lv_m1 = (int) warp_sum64(c_m1) - 1;
    p.lv_pr = (int) warp_sum64(c_lt);
    if (!p.mode1) {
        if (anomaly[q]) {
            p.exact1 = 1;
        } else {
            int64_t nres = 0, npr = 0;
            for (int b = lane; b < nl; b += 32) {
                if (b <= p.lv_res) nres += h[b];
                if (b >= p.lv_pr) npr += h[nl + b];
            }
            nres = warp_sum64(nres);
            npr = warp_sum64(npr);
            p.n_res1 = (int) nres;
            p.n_pr1 = (int) npr;
            p.n_ref1 = (int) (n_user - nres - npr);
        }
    }
    if (lane == 0) par[q] = p;
}

// Round-1 class counts pair by pair (the reduction at PruneCandidateByBound.hpp:115-136), for
// queries where the histogram shortcut does not apply.
__global__ void qsrp_count1_kernel(const uint32_t *__restrict__ lv, int64_t n_user, QsrpParams *__restrict__ par) {
    const int q = blockIdx.y;
    const QsrpParams p = par[q];
    if (p.mode1 || !p.exact1) return;
    __shared__ int cnt[3];
    if (threadIdx.x < 3) cnt[threadIdx.x] = 0;
    __syncthreads();
    int c[3] = {0, 0, 0};
    const uint32_t *row = lv + (int64_t) q * n_user;
    for (int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; u < n_user; u += (int64_t) gridDim.x * blockDim.x) {
        const uint32_t v = row[u];
        const int k = class1_lv(p, v & 0xffff, v >> 16);
        c[k == kClsResult ? 0 : (k == kClsPrune ? 1 : 2)]++;
    }
    for (int i = 0; i < 3; i++) {
        int v = c[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&cnt[i], v);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&par[q].n_res1, cnt[0]);
        atomicAdd(&par[q].n_pr1, cnt[1]);
        atomicAdd(&par[q].n_ref1, cnt[2]);
    }
}

// Round-1 closing rules (PruneCandidateByBound.hpp:93-94, 139-150).
__global__ void qsrp_final1_kernel(QsrpParams *__restrict__ par, int nq, int topk) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    QsrpParams p = par[q];
    if (p.mode1) {
        p.n_res1 = topk;
        p.n_pr1 = 0;
        p.n_ref1 = 0;
    } else if (p.n_res1 + p.n_ref1 == topk) {
        p.all1 = 1;
        p.n_res1 = topk;
        p.n_ref1 = 0;
    }
    p.skip2 = p.n_res1 >= topk;
    par[q] = p;
}

// QS and US have no round 1: every user reaches the sampled-threshold bounds, and the reference's
// ip_cost starts at n_user (QS.hpp:143, US.hpp:131).
__global__ void qs_params_kernel(QsrpParams *__restrict__ par, int nq, int64_t n_user) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    QsrpParams p = {};
    p.lv_res = -1;
    p.lv_pr = 1 << 30;
    p.lv_m1 = -1;
    p.n_ref1 = (int) n_user;
    par[q] = p;
}

// ---- round 2 -------------------------------------------------------------------------------------

// Round 2 per (user chunk, query): pairs that did not reach round 2 get their round-1 state code in
// place of the group code; the others are counted by group (per-warp shared-memory copies).
__global__ void __launch_bounds__(kHistThreads) qsrp_round2_kernel(const uint32_t *__restrict__ lv,
                                                                  uint8_t *__restrict__ code, int64_t n_user,
                                                                  const QsrpParams *__restrict__ par, int nb,
                                                                  int64_t chunk, int *__restrict__ hist_c) {
    extern __shared__ int h[];
    const int nbin = nb + 1, copies = hist_copies(nbin);
    const int q = blockIdx.y;
    QsrpParams p;
    {
        const QsrpParams &g = par[q];
        p.mode1 = g.mode1; p.all1 = g.all1; p.lv_res = g.lv_res; p.lv_pr = g.lv_pr; p.lv_m1 = g.lv_m1;
    }
    const bool all_survive = lv == nullptr;  // QS and US: no round 1
    for (int b = threadIdx.x; b < copies * nbin; b += blockDim.x) h[b] = 0;
    __syncthreads();
    int *mine = h + ((threadIdx.x >> 5) % copies) * nbin;
    const uint32_t *lrow = lv ? lv + (int64_t) q * n_user : nullptr;
    uint8_t *crow = code + (int64_t) q * n_user;
    const int64_t u0 = (int64_t) blockIdx.x * chunk, u1 = min(u0 + chunk, n_user);
    constexpr int G = 4;  // pairs in flight per thread; the group code is loaded with the levels
    for (int64_t ub = u0 + threadIdx.x; ub < u1; ub += G * kHistThreads) {
        uint32_t v[G];
        unsigned cc[G];
#pragma unroll
        for (int g = 0; g < G; g++) {
            const bool in = ub + g * kHistThreads < u1;
            v[g] = in && !all_survive ? __ldg(lrow + ub + g * kHistThreads) : 0u;
            cc[g] = in ? crow[ub + g * kHistThreads] : 0u;
        }
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int64_t u = ub + g * kHistThreads;
            if (u >= u1) break;
            const int k = all_survive ? kClsRefine : class1_lv(p, v[g] & 0xffff, v[g] >> 16);
            if (k == kClsRefine || k == kClsIdle) atomicAdd(mine + cc[g], 1);
            else crow[u] = k == kClsResult ? kCodeResult1 : kCodePruned1;
        }
    }
    __syncthreads();
    int *gh = hist_c + (int64_t) q * nbin;
    for (int b = threadIdx.x; b < nbin; b += blockDim.x) {
        int sum = 0;
        for (int c = 0; c < copies; c++) sum += h[c * nbin + b];
        if (sum) atomicAdd(gh + b, sum);
    }
}

// Round-2 selection, coarse step (second PruneCandidateByBound call, QSRPNormalLP.hpp:187-190):
// the coarse group holding the kp-th smallest bucket among the users that reached round 2
// (kp = topk - round-1 results), or, with fewer such users than kp, the highest occupied group.
__global__ void qsrp_select2c_kernel(const int *__restrict__ hist_c, int nb, int topk, int nq,
                                     QsrpParams *__restrict__ par, QueryCounts *__restrict__ counts) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    QsrpParams p = par[q];
    p.crit = -1; p.cum_before = -1; p.mask1 = 0; p.mask2 = 0; p.gneed_lo = 0; p.gneed_hi = 0;
    if (p.skip2) {
        QueryCounts c = {};
        c.n_result = p.n_res1;
        c.n_prune = p.n_pr1;
        c.n_cand = 0;
        c.mode = 2;
        c.ip_base = p.n_ref1;
        counts[q] = c;
        par[q] = p;
        return;
    }
    const int *h = hist_c + (int64_t) q * (nb + 1);
    const int kp = topk - p.n_res1;
    int64_t n_el = 0;
    for (int g = 0; g <= nb; g++) n_el += h[g];
    p.n_elig2 = (int) n_el;
    if (n_el < kp) {
        for (int g = nb; g >= 0; g--) if (h[g]) { p.crit = g; break; }
    } else {
        int64_t cum = 0;
        for (int g = 0; g <= nb; g++) {
            if (cum + h[g] >= kp) { p.crit = g; p.cum_before = (int) cum; break; }
            cum += h[g];
        }
    }
    if (p.crit >= 0 && p.crit < nb) p.mask1 = (int32_t) (1u << p.crit);
    par[q] = p;
}

// Pairs whose exact bucket a fine pass needs: (query << 40 | user << 8 | group), resolved by
// qsrp_fine2_list_kernel; past the capacity the scan resolves them itself.
struct HitList {
    uint64_t *e;
    int *count;
    int cap;
};

__device__ __forceinline__ void fine2_hit(const HitList &hl, bool hit, int64_t q, int64_t u, unsigned c, QipView sc,
                                          const float *__restrict__ thr, int S, int gs, int *__restrict__ hist_f) {
    const unsigned want = __ballot_sync(0xffffffffu, hit);  // called by whole warps
    if (!want) return;
    const int lane = threadIdx.x & 31, leader = __ffs(want) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(hl.count, __popc(want));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (!hit) return;
    const int idx = base + __popc(want & ((1u << lane) - 1));
    if (idx < hl.cap) hl.e[idx] = ((uint64_t) q << 40) | ((uint64_t) u << 8) | c;
    else atomicAdd(hist_f + q * (S + 1) + pair_bucket(sc, thr, S, gs, (int) c, u, q), 1);
}

// Scan for the pairs whose coarse group is flagged for their query (mask1, or mask2 when any
// query has one): a grid-stride pass over the batch's codes as one flat [query][user] array, 16
// codes per thread and 512 per warp and step.
__global__ void __launch_bounds__(256) qsrp_fine2_kernel(const uint8_t *__restrict__ code, QipView sc, int64_t n_user,
                                                        int nq, double inv_user, const float *__restrict__ thr, int S,
                                                        int gs, const QsrpParams *__restrict__ par, int second,
                                                        const int *__restrict__ any2, HitList hl,
                                                        int *__restrict__ hist_f) {
    if (second && !*any2) return;
    const int64_t total = n_user * nq;
    // whole warps step together over 512-code segments (the hit appends are warp-wide)
    const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = (int64_t) gridDim.x * blockDim.x * 16;
    for (int64_t seg = warp * 512; seg < total; seg += stride) {
        const int64_t base = seg + (threadIdx.x & 31) * 16;
        uint32_t w[4];
        if (base >= total) {
            w[0] = w[1] = w[2] = w[3] = 0xffffffffu;
        } else if (base + 16 <= total) {
            const uint4 x = *reinterpret_cast<const uint4 *>(code + base);
            w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                w[i] = 0xffffffffu;
                for (int j = 0; j < 4; j++)
                    if (base + 4 * i + j < total) w[i] = (w[i] & ~(0xffu << (8 * j))) | ((uint32_t) code[base + 4 * i + j] << (8 * j));
            }
        }
        if (n_user < 512) {  // a segment may span several queries
            for (int e = 0; e < 16; e++) {
                const unsigned c = (w[e >> 2] >> (8 * (e & 3))) & 0xff;
                const int64_t pos = base + e;
                if (pos >= total || c >= 32) continue;
                const int64_t q = pos / n_user, u = pos % n_user;
                if ((uint32_t) (second ? par[q].mask2 : par[q].mask1) >> c & 1u)
                    atomicAdd(hist_f + q * (S + 1) + pair_bucket(sc, thr, S, gs, (int) c, u, q), 1);
            }
            continue;
        }
        // with at least 512 users a 512-code segment meets at most one query boundary: the
        // segment's first query, found once per warp, and the next
        int64_t qs = 0;
        if ((threadIdx.x & 31) == 0) {
            qs = (int64_t) ((double) seg * inv_user);
            if (qs * n_user > seg) qs--;
            else if ((qs + 1) * n_user <= seg) qs++;
        }
        qs = __shfl_sync(0xffffffffu, qs, 0);
        int64_t q0 = 0, edge = 0;
        uint32_t m0 = 0, m1 = 0;
        if (base < total) {
            q0 = base >= (qs + 1) * n_user ? qs + 1 : qs;
            edge = (q0 + 1) * n_user;
            m0 = (uint32_t) (second ? par[q0].mask2 : par[q0].mask1);
            m1 = edge < base + 16 && q0 + 1 < nq ? (uint32_t) (second ? par[q0 + 1].mask2 : par[q0 + 1].mask1) : 0u;
        }
        uint32_t hits = 0;
        const bool one_query = edge >= base + 16 && base + 16 <= total;
        if (one_query && !m0) {
            // nothing flagged for this query
        } else if (one_query && (m0 & (m0 - 1)) == 0) {
            // one flagged group and one query: a bytewise compare per word
            const uint32_t pat = (uint32_t) (__ffs(m0) - 1) * 0x01010101u;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t eq = __vcmpeq4(w[i], pat) & 0x01010101u;
                hits |= ((eq * 0x01020408u) >> 24) << (4 * i);
            }
        } else if (m0 | m1) {
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const unsigned c = (w[e >> 2] >> (8 * (e & 3))) & 0xff;
                const uint32_t m = base + e >= edge ? m1 : m0;
                hits |= (uint32_t) (base + e < total && c < 32 && (m >> c & 1u)) << e;
            }
        }
        // one hit per lane and round, so that the list append stays warp-aggregated
        while (__any_sync(0xffffffffu, hits != 0)) {
            const int e = hits ? __ffs(hits) - 1 : 0;
            const int64_t pos = base + e;
            const int64_t q = pos >= edge ? q0 + 1 : q0;
            fine2_hit(hl, hits != 0, q, pos - q * n_user, (w[e >> 2] >> (8 * (e & 3))) & 0xff, sc, thr, S, gs, hist_f);
            hits &= hits - 1;
        }
    }
}

// Exact buckets of the listed pairs.
__global__ void __launch_bounds__(256, 4) qsrp_fine2_list_kernel(HitList hl, QipView sc, int64_t n_user, const float *__restrict__ thr, int S,
                                       int gs, int *__restrict__ hist_f) {
    const int n = min(*hl.count, hl.cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t x = hl.e[i];
        const int64_t q = (int64_t) (x >> 40), u = (int64_t) ((x >> 8) & 0xffffffffu);
        const int c = (int) (x & 0xff);
        atomicAdd(hist_f + q * (S + 1) + pair_bucket(sc, thr, S, gs, c, u, q), 1);
    }
}

// Class of bucket b for the round-2 bounds (L, U): mode2 (L == U) marks results only.
__device__ __forceinline__ uint8_t class2_of(int b, int S, const int32_t *rank, int n_item, int L, int U, bool mode2) {
    int lb, ub;
    bucket_bounds(b, S, rank, n_item, lb, ub);
    if (mode2) return (ub <= L && lb <= L) ? kClsResult : kClsIdle;
    if (lb <= U) return kClsResult;
    if (L <= ub) return kClsPrune;
    return kClsRefine;
}

// Round-2 selection, exact step, one warp per query: the k-th bucket from the critical group's
// exact histogram, the bounds (L2, U2), each bucket's and each group's class, and the mixed groups
// still without an exact histogram (mask2).
__global__ void qsrp_select2f_kernel(const int *__restrict__ hist_f, int nb, int gs, int S,
                                     const int32_t *__restrict__ rank, int n_item, int topk, int nq,
                                     QsrpParams *__restrict__ par, uint8_t *__restrict__ cls2,
                                     uint8_t *__restrict__ clsg, int *__restrict__ any2) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= nq) return;
    QsrpParams p = par[q];
    if (p.skip2) return;
    const int *hf = hist_f + (int64_t) q * (S + 1);
    int L = 0, U = 0;
    if (p.cum_before < 0) {  // the reference's zero-filled heap: max(bounds of the highest bucket, 0)
        int bmax = -1;
        if (p.crit == nb) bmax = S;
        else if (p.crit >= 0)
            for (int b = min(p.crit * gs + gs, S) - 1; b >= p.crit * gs; b--) if (hf[b]) { bmax = b; break; }
        if (bmax >= 0) {
            int lb, ub;
            bucket_bounds(bmax, S, rank, n_item, lb, ub);
            L = max(lb, 0); U = max(ub, 0);
        }
    } else {
        int bk = S;
        if (p.crit < nb) {
            const int need = topk - p.n_res1 - p.cum_before;
            const int end = min(p.crit * gs + gs, S);
            int c = 0;
            bk = end - 1;
            for (int b = p.crit * gs; b < end; b++) { c += hf[b]; if (c >= need) { bk = b; break; } }
        }
        bucket_bounds(bk, S, rank, n_item, L, U);
    }
    p.L2 = L; p.U2 = U; p.mode2 = L == U;
    uint8_t *cq = cls2 + (int64_t) q * (S + 1);
    uint8_t *cg = clsg + (int64_t) q * (nb + 1);
    for (int b = lane; b <= S; b += 32) cq[b] = class2_of(b, S, rank, n_item, L, U, p.mode2);
    uint32_t mask2 = 0;
    for (int g = lane; g < nb; g += 32) {
        const int b0 = g * gs, b1 = min(b0 + gs, S);
        uint8_t k = class2_of(b0, S, rank, n_item, L, U, p.mode2);
        for (int b = b0 + 1; b < b1; b++) if (class2_of(b, S, rank, n_item, L, U, p.mode2) != k) { k = kClsMixed; break; }
        cg[g] = k;
        if (k == kClsMixed && !p.mode2 && !(p.mask1 >> g & 1)) mask2 |= 1u << g;
    }
    mask2 = __reduce_or_sync(0xffffffffu, mask2);
    if (lane == 0) {
        cg[nb] = class2_of(S, S, rank, n_item, L, U, p.mode2);
        p.mask2 = (int32_t) mask2;
        par[q] = p;
        if (mask2) *any2 = 1;
    }
}

// Round-2 class counts (PruneCandidateByBound.hpp:83-150), one warp per query: pure groups count
// whole from the coarse histogram, mixed groups bucket by bucket; then the "all survivors are
// results" rule and the groups the compaction must classify.
__global__ void qsrp_final2_kernel(const int *__restrict__ hist_c, const int *__restrict__ hist_f, int nb, int gs, int S,
                                   int topk, int nq, QsrpParams *__restrict__ par, uint8_t *__restrict__ cls2,
                                   uint8_t *__restrict__ clsg, QueryCounts *__restrict__ counts) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= nq) return;
    QsrpParams p = par[q];
    if (p.skip2) return;
    QueryCounts c = {};
    c.lstar = p.L2;
    c.ustar = p.U2;
    c.ip_base = p.n_ref1;  // QSRPNormalLP.hpp:177: refine_user_size after the first prune
    uint8_t *cq = cls2 + (int64_t) q * (S + 1);
    uint8_t *cg = clsg + (int64_t) q * (nb + 1);
    bool all2 = false;
    if (p.mode2) {
        c.mode = 1;
        c.n_result = topk;
        c.n_prune = p.n_pr1;
        c.n_cand = 0;
    } else {
        const int *hc = hist_c + (int64_t) q * (nb + 1);
        const int *hf = hist_f + (int64_t) q * (S + 1);
        int64_t n[4] = {0, 0, 0, 0};
        for (int g = lane; g <= nb; g += 32) {
            const uint8_t k = cg[g];
            if (k != kClsMixed) {
                n[k] += hc[g];
            } else {
                for (int b = g * gs; b < min(g * gs + gs, S); b++) n[cq[b]] += hf[b];
            }
        }
        int64_t nres = p.n_res1 + warp_sum64(n[kClsResult]), npr = p.n_pr1 + warp_sum64(n[kClsPrune]);
        int64_t nref = warp_sum64(n[kClsRefine]);
        if (nres + nref == topk) {
            all2 = true;
            for (int b = lane; b <= S; b += 32) if (cq[b] == kClsRefine) cq[b] = kClsResult;
            nres = topk;
            nref = 0;
        }
        c.mode = 0;
        c.n_result = (int) nres;
        c.n_prune = (int) npr;
        c.n_cand = nres >= topk ? 0 : (int) nref;
    }
    uint32_t need_lo = 0, need_hi = 0;
    for (int g = lane; g <= nb; g += 32) {
        uint8_t k = cg[g];
        if (all2 && k == kClsRefine) cg[g] = k = kClsResult;
        const bool need = k == kClsResult || k == kClsMixed || (k == kClsRefine && c.n_cand > 0);
        if (need) { if (g < 32) need_lo |= 1u << g; else need_hi |= 1u << (g - 32); }
    }
    need_lo = __reduce_or_sync(0xffffffffu, need_lo);
    need_hi = __reduce_or_sync(0xffffffffu, need_hi);
    if (lane == 0) {
        p.gneed_lo = (int32_t) need_lo;
        p.gneed_hi = (int32_t) need_hi;
        par[q] = p;
        counts[q] = c;
    }
}

// Classification of a pair after both rounds for the ordered compaction: result users carry their
// reported rank (the lower bound in force) and whether their score is this query's; candidates
// carry their round-2 bounds.  Exact buckets are resolved only where the group does not settle the
// class or the entry's fields are asked for.
struct QsrpCompactPolicy {
    struct Aux { int rank, fresh, lb, ub; };
    const uint32_t *lv;
    const uint8_t *code;
    const float *thr;
    QipView sc;
    int64_t n_user;
    const int32_t *reg_rank, *rank;
    int S_reg, S, n_item, nb, gs;
    const QsrpParams *par;
    const uint8_t *cls2, *clsg;
    const QueryCounts *counts;
    const int64_t *cand_off;
    int topk;
    int32_t *res_user, *res_rank;
    uint8_t *res_fresh;
    int32_t *cand_user, *cand_query, *cand_lb, *cand_ub;
    __device__ bool query_active(int q) const { return true; }
    // Users whose code can make them a result or a candidate: a group the compaction must
    // classify, a round-1 result, or any non-survivor under the equal-bounds rule.
    __device__ uint32_t need_mask(int q, int64_t u, int n) const {
        const QsrpParams &p = par[q];
        const uint64_t gneed = (uint64_t) (uint32_t) p.gneed_lo | ((uint64_t) (uint32_t) p.gneed_hi << 32);
        const bool state_any = !p.skip2 && p.mode2;
        uint32_t w[4];
        load16_bytes(code + (int64_t) q * n_user + u, w);
        uint32_t m = 0;
#pragma unroll
        for (int e = 0; e < kCompactPer; e++) {
            const unsigned c = (w[e >> 2] >> (8 * (e & 3))) & 0xff;
            const bool nd = c <= (unsigned) nb ? (bool) (gneed >> c & 1) : (c == kCodeResult1 || state_any);
            m |= (uint32_t) nd << e;
        }
        return n >= 32 ? m : m & ((1u << n) - 1);
    }
    __device__ int classify(int q, int64_t u, Aux &aux, bool with_aux) const {
        const int64_t at = (int64_t) q * n_user + u;
        const unsigned c = code[at];
        if (c <= (unsigned) nb) {  // reached round 2
            if (par[q].skip2) return 0;
            const uint8_t kg = clsg[(int64_t) q * (nb + 1) + c];
            if (kg == kClsPrune || kg == kClsIdle) return 0;
            const bool cand_ok = counts[q].n_cand > 0;
            if (kg == kClsRefine && !cand_ok) return 0;
            if (!with_aux && kg != kClsMixed) return kg == kClsResult ? 1 : 2;
            const int b = c == (unsigned) nb ? S : pair_bucket(sc, thr, S, gs, (int) c, u, q);
            const uint8_t k2 = cls2[(int64_t) q * (S + 1) + b];
            int lb, ub;
            bucket_bounds(b, S, rank, n_item, lb, ub);
            aux.rank = lb; aux.fresh = 1; aux.lb = lb; aux.ub = ub;
            if (k2 == kClsResult) return 1;
            return (k2 == kClsRefine && cand_ok) ? 2 : 0;
        }
        aux.fresh = 0;
        const QsrpParams &p = par[q];
        if (c == kCodeResult1 || (!p.skip2 && p.mode2)) {
            const uint32_t v = lv[at];
            const int lb1 = level_rank(v & 0xffff, reg_rank, S_reg, n_item);
            const int ub1 = level_rank(v >> 16, reg_rank, S_reg, n_item);
            aux.rank = lb1; aux.lb = lb1; aux.ub = ub1;
            if (c == kCodeResult1) return 1;
            return (ub1 <= p.L2 && lb1 <= p.L2) ? 1 : 0;  // the equal-bounds rule scans every user
        }
        return 0;
    }
    __device__ void emit_result(int q, int pos, int64_t u, const Aux &aux) const {
        const int64_t i = (int64_t) q * topk + pos;
        res_user[i] = (int32_t) u;
        res_rank[i] = aux.rank;
        res_fresh[i] = (uint8_t) aux.fresh;
    }
    __device__ void emit_cand(int q, int pos, int64_t u, const Aux &aux) const {
        if (pos >= counts[q].n_cand) return;  // the count pass disagrees; reported by compact_scan
        const int64_t e = cand_off[q] + pos;
        cand_user[e] = (int32_t) u;
        cand_query[e] = q;
        cand_lb[e] = aux.lb;
        cand_ub[e] = aux.ub;
    }
};

// Scores of the emitted result users: this query's score when the user reached round 2, else the
// score from its latest earlier round-2 query in the batch, else the carried state.
__global__ void __launch_bounds__(128, 8) qsrp_result_fill_kernel(const QueryCounts *__restrict__ counts, const int32_t *__restrict__ res_user,
                                        const uint8_t *__restrict__ res_fresh, const uint8_t *__restrict__ code,
                                        QipView sc, int64_t n_user, const float *__restrict__ state, int topk,
                                        float *__restrict__ res_qip) {
    const int q = blockIdx.x;
    const int n = counts[q].n_res_emit;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int64_t i = (int64_t) q * topk + k;
        const int u = res_user[i];
        int src = res_fresh[i] ? q : -1;
        for (int qq = q - 1; src < 0 && qq >= 0; qq--)
            if (code[(int64_t) qq * n_user + u] < kCodeResult1) src = qq;
        res_qip[i] = src >= 0 ? sc.exact(u, src) : state[u];
    }
}

__global__ void __launch_bounds__(256, 4) qsrp_cand_fill_kernel(const int32_t *__restrict__ cand_user, const int32_t *__restrict__ cand_query,
                                      int64_t n, QipView sc, float *__restrict__ cand_qip) {
    const int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    cand_qip[e] = sc.exact(cand_user[e], cand_query[e]);
}

// Carried state after the batch: each user's score at its last round-2 query of the batch.
__global__ void __launch_bounds__(256, 4) qsrp_state_kernel(const uint8_t *__restrict__ code, QipView sc, int64_t n_user, int nq,
                                  float *__restrict__ state) {
    const int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_user) return;
    for (int q = nq - 1; q >= 0; q--)
        if (code[(int64_t) q * n_user + u] < kCodeResult1) {
            state[u] = sc.exact(u, q);
            return;
        }
}

// ---- host orchestration ----------------------------------------------------------------------------

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

// One chunk of queries.  QSRPNormalLP runs both rounds; QS and US (no regression round, scores
// in the original space) run the scores tile without levels and start at round 2.
int pair_chunk(rkr_index *ix, int method, const float *d_query, int nq, int topk, rkr_user_rank *d_out,
               rkr_query_stats *d_stats, cudaStream_t st) {
    const bool qsrp = method == RKR_METHOD_QSRP_NORMAL_LP;
    const int64_t U = ix->n_user;
    const int dim = ix->dim, c = ix->check_dim, S = ix->n_sample, Sr = ix->n_sample_reg;
    const int n_item = (int) ix->n_item;
    const int nl = Sr + 2;
    const int gs = thr_group(S), nb = (S + gs - 1) / gs;
    RKR_TRY(ix->ws_qtr.ensure(carve_size((size_t) nq * dim, 4) + carve_size(nq, 4) + carve_size(nq, sizeof(QsrpParams)) +
                              carve_size(nq, 4) + carve_size(1, 4) * 2 + carve_size(2, 4)));
    uint8_t *p0 = ix->ws_qtr.as<uint8_t>();
    float *qtr = carve<float>(p0, (size_t) nq * dim);
    float *qnorm = carve<float>(p0, nq);
    QsrpParams *par = carve<QsrpParams>(p0, nq);
    int *anomaly = carve<int>(p0, nq);
    int *fix_count = carve<int>(p0, 1);
    int *any2 = carve<int>(p0, 1);
    int *hit_count = carve<int>(p0, 2);
    RKR_TRY(ix->ws_levels.ensure((size_t) nq * U * 8));
    RKR_TRY(ix->ws_bucket2.ensure((size_t) nq * U));
    RKR_TRY(ix->ws_cls.ensure(carve_size((size_t) nq * (S + 1), 1) + carve_size((size_t) nq * (nb + 1), 1)));
    RKR_TRY(ix->ws_counts.ensure(sizeof(QueryCounts) * (size_t) nq));
    const size_t n_hist_l = (size_t) nq * 2 * nl, n_hist_c = (size_t) nq * (nb + 1), n_hist_f = (size_t) nq * (S + 1);
    RKR_TRY(ix->ws_hist.ensure(carve_size(n_hist_l, 4) + carve_size(n_hist_c, 4) + carve_size(n_hist_f, 4)));
    const int fix_cap = (int) std::min<int64_t>(int64_t(1) << 26, std::max<int64_t>(int64_t(1) << 20, U * nq / 64));
    const int hit_cap = 1 << 22;
    RKR_TRY(ix->ws_fix.ensure(carve_size(fix_cap, sizeof(int4)) + carve_size(hit_cap, 8)));
    uint32_t *lv = ix->ws_levels.as<uint32_t>();
    float *qip = reinterpret_cast<float *>(lv + (size_t) nq * U);
    uint8_t *code = ix->ws_bucket2.as<uint8_t>();
    uint8_t *pc = ix->ws_cls.as<uint8_t>();
    uint8_t *cls2 = carve<uint8_t>(pc, (size_t) nq * (S + 1));
    uint8_t *clsg = carve<uint8_t>(pc, (size_t) nq * (nb + 1));
    QueryCounts *counts = ix->ws_counts.as<QueryCounts>();
    uint8_t *ph = ix->ws_hist.as<uint8_t>();
    int *hist_l = carve<int>(ph, n_hist_l);
    int *hist_c = carve<int>(ph, n_hist_c);
    int *hist_f = carve<int>(ph, n_hist_f);
    uint8_t *pm = ix->ws_fix.as<uint8_t>();
    FixList fix;
    fix.e = carve<int4>(pm, fix_cap);
    fix.count = fix_count;
    fix.cap = fix_cap;
    HitList hl;
    hl.e = carve<uint64_t>(pm, hit_cap);
    hl.cap = hit_cap;
    RKR_CUDA(cudaMemsetAsync(anomaly, 0, sizeof(int) * nq, st));
    RKR_CUDA(cudaMemsetAsync(fix_count, 0, sizeof(int), st));
    RKR_CUDA(cudaMemsetAsync(any2, 0, sizeof(int), st));
    RKR_CUDA(cudaMemsetAsync(hit_count, 0, 2 * sizeof(int), st));
    RKR_CUDA(cudaMemsetAsync(ix->ws_hist.p, 0, (size_t) (ph - ix->ws_hist.as<uint8_t>()), st));

    if (qsrp) {
        timed(ix, st, "transfer_query", [&] {
            transfer_query_kernel<<<nq, 128, 0, st>>>(d_query, ix->transfer_item.as<float>(), dim, c, qtr, qnorm);
        });
        RKR_CUDA(cudaGetLastError());
    } else {
        RKR_CUDA(cudaMemsetAsync(qnorm, 0, sizeof(float) * nq, st));
    }
    ScoreSrc sc;
    sc.svd_user = ix->svd_user.as<float>();
    sc.qtr = qtr;
    sc.dim = dim;
    sc.c = c;
    RegModel m;
    m.rec = ix->reg.as<float>();
    m.rank = ix->reg_rank.as<int32_t>();
    m.S = Sr;
    m.err_cap = (double) Sr - 1e-3;
    m.n_item = n_item;
    QipView qv;
    qv.qip = qip;
    qv.n_user = U;
    qv.urow = (qsrp ? ix->svd_user : ix->user).as<float>();
    qv.qrow = qsrp ? qtr : d_query;
    qv.dim = dim;
    qv.c = qsrp ? c : dim;
    Round1Epi e1;
    e1.unorm = ix->svd_unorm.as<float>();
    e1.qnorm = qnorm;
    e1.thr_summ = ix->thr_summ.as<float>();
    e1.m = m;
    e1.lv = qsrp ? lv : nullptr;
    e1.code = code;
    e1.qip = qip;
    e1.nb = nb;
    e1.n_user = U;
    e1.n_query = nq;
    e1.fix = fix;
    // pair scores, levels and coarse groups: on the tensor cores with exact resolution of undecided
    // pairs where the shape allows, else on the exact tiles
    bool tc_done = false;
    {
        ScoresTcCall call;
        call.qsrp = qsrp;
        call.qrows = qv.qrow;
        call.qnorm = qnorm;
        call.unorm = e1.unorm;
        call.nq = nq;
        call.m = m;
        call.nb = nb;
        call.lv = e1.lv;
        call.code = code;
        call.qip = qip;
        RKR_TRY(scores_tc(ix, call, st, &qv.scr, &tc_done));
    }
    if (!tc_done) {
        qv.scr = PairScreen();
        RKR_TRY(ix->ws_km.ensure(sizeof(float) * (size_t) dim * (size_t) kmajor_ld(nq)));
        RKR_TRY(to_kmajor(qsrp ? qtr : d_query, nullptr, nq, dim, ix->ws_km.as<float>(), st));
        cudaError_t ce = cudaSuccess;
        const KMajor ka = {(qsrp ? ix->svd_user_km : ix->user_km).as<float>(), U, kmajor_ld(U), kmajor_ld(U)};
        const KMajor kb = {ix->ws_km.as<float>(), nq, kmajor_ld(nq), kmajor_ld(nq)};
        // QS / US: one sequential sum over all coordinates (QS.hpp:137-143), seen by finish_hi
        timed(ix, st, "qsrp_scores", [&] { ce = launch_big_split(ka, kb, qsrp ? c : dim, dim, e1, st); });
        RKR_CUDA(ce);
    }
    const int64_t chunk = 16384;
    dim3 hg((unsigned) ((U + chunk - 1) / chunk), (unsigned) nq);
    if (qsrp) {
    if (!tc_done) {
        timed(ix, st, "qsrp_fix1", [&] { qsrp_fix1_kernel<<<148 * 4, 256, 0, st>>>(fix, m, e1.unorm, qnorm, U, lv); });
        RKR_CUDA(cudaGetLastError());
        timed(ix, st, "qsrp_fix1_scan", [&] {
            qsrp_fix1_scan_kernel<<<148 * 8, 256, 0, st>>>(fix_count, fix_cap, m, sc, e1.unorm, qnorm, U, nq, lv);
        });
        RKR_CUDA(cudaGetLastError());
    }
    timed(ix, st, "level_hist", [&] {
        level_hist_kernel<<<hg, kHistThreads, hist_copies(2 * nl) * 2 * nl * sizeof(int), st>>>(lv, U, m.rank, Sr, n_item,
                                                                                               chunk, hist_l, anomaly);
    });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_select1", [&] {
        qsrp_select1_kernel<<<(nq + 3) / 4, 128, 0, st>>>(hist_l, anomaly, U, m.rank, Sr, n_item, topk, nq, par);
    });
    RKR_CUDA(cudaGetLastError());
    {
        dim3 g((unsigned) std::min<int64_t>((U + 1023) / 1024, 64), (unsigned) nq);
        timed(ix, st, "qsrp_count1", [&] { qsrp_count1_kernel<<<g, 256, 0, st>>>(lv, U, par); });
        RKR_CUDA(cudaGetLastError());
    }
    timed(ix, st, "qsrp_final1", [&] { qsrp_final1_kernel<<<(nq + 127) / 128, 128, 0, st>>>(par, nq, topk); });
    RKR_CUDA(cudaGetLastError());
    } else {
        qs_params_kernel<<<(nq + 127) / 128, 128, 0, st>>>(par, nq, U);
        RKR_CUDA(cudaGetLastError());
    }
    timed(ix, st, "qsrp_round2", [&] {
        qsrp_round2_kernel<<<hg, kHistThreads, hist_copies(nb + 1) * (nb + 1) * sizeof(int), st>>>(
            qsrp ? lv : nullptr, code, U, par, nb, chunk, hist_c);
    });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_select2c", [&] {
        qsrp_select2c_kernel<<<(nq + 127) / 128, 128, 0, st>>>(hist_c, nb, topk, nq, par, counts);
    });
    RKR_CUDA(cudaGetLastError());
    const float *thr = ix->thr.as<float>();
    const int32_t *srank = ix->sample_rank.as<int32_t>();
    const unsigned fg = 148 * 16;
    const double inv_user = 1.0 / (double) U;
    hl.count = hit_count;
    timed(ix, st, "qsrp_fine2", [&] {
        qsrp_fine2_kernel<<<fg, 256, 0, st>>>(code, qv, U, nq, inv_user, thr, S, gs, par, 0, any2, hl, hist_f);
    });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_fine2_list", [&] { qsrp_fine2_list_kernel<<<148 * 8, 256, 0, st>>>(hl, qv, U, thr, S, gs, hist_f); });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_select2f", [&] {
        qsrp_select2f_kernel<<<(nq + 3) / 4, 128, 0, st>>>(hist_f, nb, gs, S, srank, n_item, topk, nq, par, cls2, clsg, any2);
    });
    RKR_CUDA(cudaGetLastError());
    hl.count = hit_count + 1;
    timed(ix, st, "qsrp_fine2", [&] {
        qsrp_fine2_kernel<<<fg, 256, 0, st>>>(code, qv, U, nq, inv_user, thr, S, gs, par, 1, any2, hl, hist_f);
    });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_fine2_list", [&] { qsrp_fine2_list_kernel<<<148 * 8, 256, 0, st>>>(hl, qv, U, thr, S, gs, hist_f); });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_final2", [&] {
        qsrp_final2_kernel<<<(nq + 3) / 4, 128, 0, st>>>(hist_c, hist_f, nb, gs, S, topk, nq, par, cls2, clsg, counts);
    });
    RKR_CUDA(cudaGetLastError());

    std::vector<QueryCounts> hc(nq);
    int h_fix = 0;
    RKR_CUDA(cudaMemcpyAsync(hc.data(), counts, sizeof(QueryCounts) * nq, cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaMemcpyAsync(&h_fix, fix_count, sizeof(int), cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    if (ix->prof.on) ix->prof.add_count("screen_undecided_pairs", h_fix);
    std::vector<int64_t> off(nq + 1, 0);
    for (int q = 0; q < nq; q++) off[q + 1] = off[q] + hc[q].n_cand;
    const int64_t n_cand = off[nq];
    size_t need = carve_size(nq + 1, 8) + carve_size((size_t) nq * topk, 4) * 3 + carve_size((size_t) nq * topk, 1) +
                  carve_size(n_cand, 4) * 5;
    RKR_TRY(ix->ws_cand.ensure(need));
    uint8_t *p = ix->ws_cand.as<uint8_t>();
    int64_t *d_off = carve<int64_t>(p, nq + 1);
    int32_t *res_user = carve<int32_t>(p, (size_t) nq * topk);
    int32_t *res_rank = carve<int32_t>(p, (size_t) nq * topk);
    float *res_qip = carve<float>(p, (size_t) nq * topk);
    uint8_t *res_fresh = carve<uint8_t>(p, (size_t) nq * topk);
    int32_t *cand_user = carve<int32_t>(p, n_cand);
    int32_t *cand_query = carve<int32_t>(p, n_cand);
    int32_t *cand_lb = carve<int32_t>(p, n_cand);
    int32_t *cand_ub = carve<int32_t>(p, n_cand);
    float *cand_qip = carve<float>(p, n_cand);
    RKR_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(int64_t) * (nq + 1), cudaMemcpyHostToDevice, st));
    QsrpCompactPolicy pol;
    pol.lv = lv;
    pol.code = code;
    pol.thr = thr;
    pol.sc = qv;
    pol.n_user = U;
    pol.reg_rank = m.rank;
    pol.rank = srank;
    pol.S_reg = Sr;
    pol.S = S;
    pol.n_item = n_item;
    pol.nb = nb;
    pol.gs = gs;
    pol.par = par;
    pol.cls2 = cls2;
    pol.clsg = clsg;
    pol.counts = counts;
    pol.cand_off = d_off;
    pol.topk = topk;
    pol.res_user = res_user;
    pol.res_rank = res_rank;
    pol.res_fresh = res_fresh;
    pol.cand_user = cand_user;
    pol.cand_query = cand_query;
    pol.cand_lb = cand_lb;
    pol.cand_ub = cand_ub;
    RKR_TRY(run_compaction(ix, pol, nq, topk, counts, st));
    timed(ix, st, "qsrp_result_fill", [&] {
        qsrp_result_fill_kernel<<<nq, 128, 0, st>>>(counts, res_user, res_fresh, code, qv, U, ix->qip_state.as<float>(),
                                                    topk, res_qip);
    });
    RKR_CUDA(cudaGetLastError());
    if (n_cand > 0) {
        timed(ix, st, "qsrp_cand_fill", [&] {
            qsrp_cand_fill_kernel<<<(unsigned) ((n_cand + 255) / 256), 256, 0, st>>>(cand_user, cand_query, n_cand, qv,
                                                                                    cand_qip);
        });
        RKR_CUDA(cudaGetLastError());
    }
    RKR_TRY(refine_and_assemble_pairs(ix, method, d_query, nq, topk, counts, res_user, res_rank, res_qip, n_cand,
                                      cand_user, cand_query, cand_lb, cand_ub, cand_qip, d_off, d_out, d_stats, st));
    if (qsrp) timed(ix, st, "qsrp_state", [&] {
        qsrp_state_kernel<<<(unsigned) ((U + 255) / 256), 256, 0, st>>>(code, qv, U, nq, ix->qip_state.as<float>());
    });
    RKR_CUDA(cudaGetLastError());
    RKR_CUDA(cudaStreamSynchronize(st));
    if (ix->prof.on && qv.scr.n_exact) {
        int h = 0;
        RKR_CUDA(cudaMemcpy(&h, qv.scr.n_exact, sizeof(int), cudaMemcpyDeviceToHost));
        ix->prof.add_count("rescored_pairs", h);
    }
    return RKR_OK;
}

}  // namespace rkr
