// rkr_qsrp.cu -- QSRPNormalLP retrieval on the device (src/impl/QSRPNormalLP.hpp:116-260).
//
// Per query the reference runs two bound/prune rounds before refinement:
//   1. SVD-space partial score on the first check_dim coordinates +- the product of the remaining
//      norms (PartDimPartNorm::IPBound, PartDimPartNorm.hpp:52-74) -> regression rank bounds
//      (NormalLinearRegressionLP::ComputeRankBound, NormalLinearRegressionLP.hpp:326-398) -> prune.
//   2. full SVD-space score for the survivors (ComputeRemainDim, :76-95) -> sampled-threshold
//      bounds (SampleSearch::RankBound) -> prune again.
// Here a batch of queries runs as passes over all (query, user) pairs:
//   * one kernel scores every pair and stores two bytes: the coarse levels (lvt_coarse) of its
//     two round-1 bounds (the per-user level-boundary tables, rkr_levels.cu) and the coarse group of
//     its sampled-threshold bucket (a per-user summary of every 16th threshold), and counts the
//     coarse levels per query; on the tensor cores (rkr_scores_tc.cu: int8 digit products, a
//     rigorous bound against the reference's sums, exact resolution of the pairs the bound leaves
//     undecided), or, where that path does not fit, as exact SIMT tiles (Round1Epi below);
//   * the round-1 selection (PruneCandidateByBound) runs on the coarse histograms; only the pairs in
//     a query's critical coarse levels get their exact levels (fine passes: the reference's own
//     arithmetic, recomputed), first to find the k-th bounds, then to classify the pairs whose
//     coarse level straddles a class threshold;
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
int refine_and_assemble_pairs(rkr_index *ix, int method, const float *d_query, int nq, KSpec ks,
                              const int64_t *d_out_off, const QueryCounts *d_counts, const int32_t *d_res_user, const int32_t *d_res_rank,
                              const float *d_res_qip, int64_t n_cand, int32_t *d_cand_user, int32_t *d_cand_query,
                              int32_t *d_cand_lb, int32_t *d_cand_ub, const float *d_cand_qip,
                              const int64_t *d_cand_off, rkr_user_rank *d_out, rkr_query_stats *d_stats,
                              cudaStream_t st);

// ---- per-query state ---------------------------------------------------------------------------------

// Round-2 codes per pair: 0..nb a coarse threshold group (nb: bucket S); otherwise the round-1 state.
constexpr uint8_t kCodeResult1 = 0xfe, kCodePruned1 = 0xff;
// Round 2 counts the codes below this group exactly in its first pass (qsrp_round2_kernel).
constexpr int kRound2Cap = 12;
constexpr uint8_t kClsMixed = 0xff;  // a group whose buckets fall in more than one class
// Coarse-level bytes per pair: lower-bound coarse level (1 .. 15) | upper-bound coarse level << 4.  A
// lower nibble of 0 never occurs for a level, so it marks a pair whose round-1 class the fine pass
// settled from its exact levels (class << 4), or, before that, a pair the exact tiles' screen left
// undecided beyond the fix list's capacity (kLvcUndecided).
constexpr uint8_t kLvcUndecided = 0x00;
constexpr uint8_t kLvcResolved = 0x00;  // low nibble of a settled pair; the class is in the high nibble

struct QsrpParams {
    int32_t mode1, all1, L1, U1;           // round 1: equal-bounds mode, "all survivors accepted", k-th bounds
    int32_t n_res1, n_pr1, n_ref1, skip2;  // round-1 counts; skip2: round 1 already produced top-k results
    int32_t mode2, L2, U2, n_elig2;        // round 2
    int32_t exact1, lv_res, lv_pr, lv_m1;  // exact1: count round-1 classes pair by pair; level thresholds
    int32_t crit, cum_before, mask1, mask2;  // critical coarse group, users below it, groups to resolve
    int32_t gneed_lo, gneed_hi, lv_m2, pad1;  // groups 0..31 / 32 the compaction must classify; L2's level
    int32_t cbl, cbu, cum_l, cum_u;        // round 1: critical coarse levels (-1: none needed), counts below
    int32_t amb_l, amb_u, res_fine, ple_fine;  // coarse levels straddling a class threshold; their counts
    int32_t c_res, c_pr, c_m1, w_all;      // coarse-level thresholds of the classes (class1_coarse);
    int32_t w_l, w_u, r2_full, pad4;       // the coarse levels the next fine scan looks for (-1: none), or all;
                                           // r2_full: round 2 needs the full group histogram
};

// The lowest level of coarse level c (its levels are lvt_lo(c) .. lvt_level(c)).
__device__ __forceinline__ int lvt_lo(int c, int S) { return c == 0 ? 0 : lvt_level(c - 1, S) + 1; }
// Every level in coarse level c is <= t / is > t.
__device__ __forceinline__ bool coarse_all_le(int c, int t, int S) { return lvt_level(c, S) <= t; }
__device__ __forceinline__ bool coarse_all_gt(int c, int t, int S) { return lvt_lo(c, S) > t; }
// The coarse level whose levels straddle t (some <= t, some > t), or -1 when none does.
__device__ __forceinline__ int coarse_straddle(int t, int S) {
    if (t < 0 || t > S) return -1;
    const int c = lvt_coarse(t, S);
    return lvt_level(c, S) == t ? -1 : c;
}
// A coarse level of more than one level (a selection inside it needs the exact levels), else -1.
__device__ __forceinline__ int coarse_multi(int c, int S) { return lvt_level(c, S) > lvt_lo(c, S) ? c : -1; }

// Round-1 class from exact levels: rank(level) is non-decreasing in the level, so lb <= U1 is
// lvl_lb <= lv_res, L1 <= ub is lvl_ub >= lv_pr and the equal-bounds test is a test against lv_m1.
__device__ __forceinline__ int class1_lv(const QsrpParams &p, int l, int h) {
    if (p.mode1) return (h <= p.lv_m1 && l <= p.lv_m1) ? kClsResult : kClsIdle;
    if (l <= p.lv_res) return kClsResult;
    if (h >= p.lv_pr) return kClsPrune;
    return p.all1 ? kClsResult : kClsRefine;
}

// The same from a coarse-level byte that no threshold straddles (or that the fine pass settled):
// c_res / c_m1 are the last coarse levels wholly <= lv_res / lv_m1, c_pr the first wholly >= lv_pr.
__device__ __forceinline__ int class1_coarse(const QsrpParams &p, unsigned v) {
    if ((v & 15) == kLvcResolved) {
        const int k = (int) (v >> 4);
        return (k == kClsRefine && p.all1) ? kClsResult : k;
    }
    const int cl = (int) (v & 15), cu = (int) (v >> 4);
    if (p.mode1) return (cu <= p.c_m1 && cl <= p.c_m1) ? kClsResult : kClsIdle;
    if (cl <= p.c_res) return kClsResult;
    if (cu >= p.c_pr) return kClsPrune;
    return p.all1 ? kClsResult : kClsRefine;
}

// The last coarse level wholly <= t (-1 if none) and the first wholly > t (kLvEntries if none).
__device__ __forceinline__ int coarse_last_le(int t, int S) {
    int c = -1;
    while (c + 1 < kLvEntries && lvt_level(c + 1, S) <= t) c++;
    return c;
}
__device__ __forceinline__ int coarse_first_gt(int t, int S) {
    int c = 0;
    while (c < kLvEntries && lvt_lo(c, S) <= t) c++;
    return c;
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

// The reference's round-1 arithmetic for one pair: the SVD-space partial score over the first
// check_dim coordinates (PartDimPartNorm.hpp:62), its bounds -+ the product of the remaining norms,
// and their regression levels (lb | ub << 16).
struct Round1Src {
    const float *svd_user, *qtr, *unorm, *qnorm;
    RegModel m;
    int dim, c;
    __device__ uint32_t levels(int64_t u, int64_t q) const {
        const float left = exact_dot(svd_user + u * dim, qtr + q * dim, c);
        const float right = __fmul_rn(__ldg(unorm + u), __ldg(qnorm + q));
        return regression_levels_exact(m.rec, m.S, m.err_cap, u, __fsub_rn(left, right), __fadd_rn(left, right));
    }
};

// The reference's score of a (query, user) pair, recomputed: a sum over [0, c) and one over
// [c, dim), added once (c == dim: one sum); the user rows are SVD-space for QSRP.
struct QipView {
    const float *urow, *qrow;
    int dim, c;
    int *n_exact;  // recomputed scores (a counter), or nullptr
    __device__ float exact(int64_t u, int64_t q) const {
        const float *ur = urow + u * dim, *qr = qrow + q * dim;
        const float left = exact_dot(ur, qr, c);
        const float v = c < dim ? __fadd_rn(left, exact_dot(ur + c, qr + c, dim - c)) : left;
        if (n_exact) atomicAdd(n_exact, 1);
        return v;
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

// The bucket (inside its coarse group g) of a pair's reference score.
__device__ __forceinline__ int pair_bucket(const QipView &sc, const float *__restrict__ thr, int S, int gs, int g,
                                           int64_t u, int64_t q) {
    return fine_bucket(thr + u * S, S, gs, g, sc.exact(u, q));
}

// Pairs the screen left undecided, resolved by qsrp_fix1_kernel: (query, user, partial score).
// Past the list's capacity the pair's coarse-level byte is written as kLvcUndecided and count keeps
// growing, which sends qsrp_fix1_scan_kernel over the whole batch.
struct FixList {
    int4 *e;
    int *count;
    int cap;
};

// One pair's exact levels into its coarse-level byte; the rank-order anomaly check.
__device__ __forceinline__ uint8_t lvc_of_levels(uint32_t v, const RegModel &m, int *anomaly_q) {
    const int l = (int) (v & 0xffffu), h = (int) (v >> 16);
    if (h > l && level_rank(h, m.rank, m.S, m.n_item) > level_rank(l, m.rank, m.S, m.n_item)) atomicAdd(anomaly_q, 1);
    return (uint8_t) (lvt_coarse(l, m.S) | (lvt_coarse(h, m.S) << 4));
}

// Tiles of 128 users x 128 queries: the partial score over the first check_dim coordinates, the
// bounds partial -+ norms and the coarse values of their regression levels; then the full score and
// the coarse group of its sampled-threshold bucket (the round-2 code of the pair if it reaches
// round 2).
struct Round1Epi {
    static constexpr size_t kExtra = sizeof(float) * kBig;
    static constexpr int kSummStride = ThrSummary::kMaxGroups + 1;
    const float *unorm, *qnorm, *thr_summ;
    RegModel m;
    uint8_t *lvc;  // nullptr: no round 1 (QS, US)
    uint8_t *code;
    int *anomaly;
    int nb;
    int64_t n_user, n_query;
    FixList fix;
    __device__ bool prologue(char *x, int64_t, int64_t b0) const {
        float *qn = reinterpret_cast<float *>(x);
        if (threadIdx.x < kBig) qn[threadIdx.x] = b0 + threadIdx.x < n_query ? __ldg(qnorm + b0 + threadIdx.x) : 0.0f;
        return true;
    }
    __device__ void finish_lo(char *x, const BigResult &res, int64_t a0, int64_t b0) const {
        if (!lvc) return;  // no round 1 (QS, US)
        const float *qn = reinterpret_cast<const float *>(x);
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7, lane = threadIdx.x & 31;
        const int64_t u = a0 + ra;
        const unsigned alive = __ballot_sync(0xffffffffu, u < n_user);
        if (u >= n_user) return;
        const RegUser r = reg_user(m, u);
        const float un = __ldg(unorm + u);
        uint8_t *out = lvc + (b0 + half) * n_user + u;
        const int64_t step = 2 * n_user;
        const int64_t left_rows = (n_query - b0 - half + 1) / 2;
        const int nrow = left_rows < kBig / 2 ? (int) left_rows : kBig / 2;
        // two queries per iteration: their screens are independent chains
        for (int i = 0; i < nrow; i += 2, out += 2 * step) {
            float left[2];
            uint8_t packed[2];
            bool ok[2];
#pragma unroll
            for (int g = 0; g < 2; g++) {
                const int rb = half + 2 * min(i + g, nrow - 1);
                left[g] = res.v[rb][ra];
                const float right = __fmul_rn(un, qn[rb]);
                int l, h;
                ok[g] = regression_levels_fast(r, m.S, __fsub_rn(left[g], right), __fadd_rn(left[g], right), l, h);
                packed[g] = ok[g] ? lvc_of_levels((uint32_t) l | ((uint32_t) h << 16), m,
                                                  anomaly + b0 + half + 2 * min(i + g, nrow - 1))
                                  : kLvcUndecided;
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
        constexpr int G4 = 4;
        for (int i0 = 0; i0 < nrow; i0 += G4) {
            float sv[G4];
            int lo[G4];
#pragma unroll
            for (int g = 0; g < G4; g++) {
                sv[g] = res.v[half + 2 * min(i0 + g, nrow - 1)][ra];
                lo[g] = 0;
            }
#pragma unroll
            for (int st = 16; st >= 1; st >>= 1)
#pragma unroll
                for (int g = 0; g < G4; g++) lo[g] += sm[lo[g] + st - 1] >= sv[g] ? st : 0;
#pragma unroll
            for (int g = 0; g < G4; g++) {
                lo[g] = min(lo[g] + (sm[lo[g]] >= sv[g]), nb);  // a score of -inf passes the padding too
                if (i0 + g < nrow) code[base + (i0 + g) * step] = (uint8_t) lo[g];
            }
        }
    }
};

// The reference's arithmetic for the pairs the screen left undecided (the listed ones).
__global__ void qsrp_fix1_kernel(FixList fix, RegModel m, const float *__restrict__ unorm,
                                 const float *__restrict__ qnorm, int64_t n_user, uint8_t *__restrict__ lvc,
                                 int *__restrict__ anomaly) {
    const int n = min(*fix.count, fix.cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 e = fix.e[i];
        const float left = __int_as_float(e.z);
        const float right = __fmul_rn(__ldg(unorm + e.y), __ldg(qnorm + e.x));
        const uint32_t v =
            regression_levels_exact(m.rec, m.S, m.err_cap, e.y, __fsub_rn(left, right), __fadd_rn(left, right));
        lvc[(int64_t) e.x * n_user + e.y] = lvc_of_levels(v, m, anomaly + e.x);
    }
}

// Undecided pairs beyond the list's capacity: a scan of the batch's coarse-level bytes for
// kLvcUndecided, with the partial score recomputed.  Returns at once when the list held them all.
__global__ void qsrp_fix1_scan_kernel(const int *__restrict__ count, int cap, Round1Src src, int64_t n_user,
                                      int nq, uint8_t *__restrict__ lvc, int *__restrict__ anomaly) {
    if (*count <= cap) return;
    const int64_t n = n_user * nq;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        if (lvc[i] != kLvcUndecided) continue;
        const int64_t q = i / n_user, u = i % n_user;
        lvc[i] = lvc_of_levels(src.levels(u, q), src.m, anomaly + q);
    }
}

// Coarse-level histograms of the exact tiles' batch (the tensor-core kernel counts in its epilogue),
// one CTA per (user chunk, query); the lower side's last coarse level and the upper side's level 0
// are left implicit, as there.
// Coarse-level histograms of a batch from its coarse-level bytes: per query, the pairs at each lower
// coarse level and each upper coarse level (the lower side's level 15 and the upper side's 0, which
// hold most pairs, stay implicit).  Per-thread counters in shared memory, bin-major ([bin][thread]:
// a thread's counters sit in its own bank), so the increments need no atomics and never conflict;
// 16 users per thread and step from aligned words.
__global__ void __launch_bounds__(kHistThreads) lvc_hist_kernel(const uint8_t *__restrict__ lvc, int64_t n_user,
                                                               int64_t chunk, int *__restrict__ lhist) {
    __shared__ int h[2 * kLvEntries * kHistThreads];
    const int q = blockIdx.y, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int b = 0; b < 2 * kLvEntries; b++) h[b * kHistThreads + tid] = 0;
    const uint8_t *row = lvc + (int64_t) q * n_user;
    const int64_t u0 = (int64_t) blockIdx.x * chunk, u1 = min(u0 + chunk, n_user);
    for (int64_t ub = u0 + (int64_t) tid * 16; ub < u1; ub += (int64_t) kHistThreads * 16) {
        const int n = (int) min((int64_t) 16, u1 - ub);
        uint32_t w[4];
        load16_bytes(row + ub, w);
        if (n < 16)  // past the chunk: bytes at both implicit levels, which count nowhere
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int keep = max(0, min(4, n - 4 * i));
                const uint32_t m = keep == 4 ? 0xffffffffu : (1u << (8 * keep)) - 1u;
                w[i] = (w[i] & m) | (0x0f0f0f0fu & ~m);
            }
#pragma unroll
        for (int e = 0; e < 16; e++) {
            const unsigned v = (w[e >> 2] >> (8 * (e & 3))) & 0xffu;
            const int cl = (int) (v & 15), cu = (int) (v >> 4);
            if (cl != kLvEntries - 1) h[cl * kHistThreads + tid]++;
            if (cu != 0) h[(kLvEntries + cu) * kHistThreads + tid]++;
        }
    }
    __syncthreads();
    int *gh = lhist + (int64_t) q * 2 * kLvEntries;
    for (int b = warp; b < 2 * kLvEntries; b += kHistThreads / 32) {
        int sum = 0;
        for (int t = lane; t < kHistThreads; t += 32) sum += h[b * kHistThreads + t];
        sum = __reduce_add_sync(0xffffffffu, sum);
        if (lane == 0 && sum) atomicAdd(gh + b, sum);
    }
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

// Full coarse counts of one side (the implicit bin restored: every pair is counted once).
__device__ __forceinline__ void coarse_counts(const int *__restrict__ h, int implicit, int64_t n_user, int *out) {
    int64_t s = 0;
    for (int b = 0; b < kLvEntries; b++) {
        out[b] = b == implicit ? 0 : h[b];
        s += out[b];
    }
    out[implicit] = (int) (n_user - s);
}

// Round-1 selection, coarse step (PruneCandidateByBound.hpp:36-77 with nothing excluded): the coarse
// levels holding each side's k-th smallest level, and the users below them.  A critical coarse
// level of a single level (0 or S + 1, where most pairs sit) needs no fine step.
__global__ void qsrp_select1c_kernel(const int *__restrict__ lhist, int64_t n_user, KSpec ks, int nq, int S,
                                     QsrpParams *__restrict__ par) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int topk = ks.of(q);
    int hl[kLvEntries], hu[kLvEntries];
    coarse_counts(lhist + (int64_t) q * 2 * kLvEntries, kLvEntries - 1, n_user, hl);
    coarse_counts(lhist + (int64_t) q * 2 * kLvEntries + kLvEntries, 0, n_user, hu);
    QsrpParams p = {};
    int64_t cum = 0;
    p.cbl = kLvEntries - 1;
    for (int b = 0; b < kLvEntries; b++) {
        if (cum + hl[b] >= topk) { p.cbl = b; break; }
        cum += hl[b];
    }
    p.cum_l = (int) cum;
    cum = 0;
    p.cbu = kLvEntries - 1;
    for (int b = 0; b < kLvEntries; b++) {
        if (cum + hu[b] >= topk) { p.cbu = b; break; }
        cum += hu[b];
    }
    p.cum_u = (int) cum;
    p.w_l = coarse_multi(p.cbl, S);
    p.w_u = coarse_multi(p.cbu, S);
    p.amb_l = -1;
    p.amb_u = -1;
    par[q] = p;
}

// Exact levels of the pairs in the coarse levels a query flags (QsrpParams::w_l / w_u / w_all).
// mode 0: the critical coarse levels of the selection that span more than one level, counted by
// exact level (fine histograms [query][2][W], W = lvt_width).  mode 1: the pairs whose coarse level
// straddles a class threshold (every pair of a query whose class counts must be taken pair by pair),
// settled to their exact round-1 class in place (lvc = class << 4) and counted.  A disagreement
// between an exact level and its coarse level is reported (the call fails) instead of counted.
__device__ __forceinline__ void fine1_hit(int mode, QsrpParams *__restrict__ par, const Round1Src &src, int64_t u,
                                          int q, unsigned v, uint8_t *__restrict__ lvc_at, int S, int W,
                                          int *__restrict__ fhist, int *__restrict__ mismatch) {
    const QsrpParams &p = par[q];
    const int cl = (int) (v & 15), cu = (int) (v >> 4);
    const uint32_t lv = src.levels(u, q);
    const int l = (int) (lv & 0xffffu), h = (int) (lv >> 16);
    if (mode == 0) {
        int *fh = fhist + (int64_t) q * 2 * W;
        if (cl == p.w_l) {
            const int i = l - lvt_lo(cl, S);
            if (i >= 0 && l <= lvt_level(cl, S)) atomicAdd(fh + i, 1);
            else atomicAdd(mismatch, 1);
        }
        if (cu == p.w_u) {
            const int i = h - lvt_lo(cu, S);
            if (i >= 0 && h <= lvt_level(cu, S)) atomicAdd(fh + W + i, 1);
            else atomicAdd(mismatch, 1);
        }
        return;
    }
    const int cls = class1_lv(p, l, h);
    if (p.w_all) {
        atomicAdd(cls == kClsResult ? &par[q].n_res1 : (cls == kClsPrune ? &par[q].n_pr1 : &par[q].n_ref1), 1);
    } else {
        if (cl == p.w_l && l <= p.lv_res) atomicAdd(&par[q].res_fine, 1);
        if (cu == p.w_u && h <= p.lv_pr - 1) atomicAdd(&par[q].ple_fine, 1);
    }
    *lvc_at = (uint8_t) ((cls << 4) | kLvcResolved);
}

// Hits of a fine scan: (query << 40 | user << 8 | coarse-level byte); past the capacity the scan
// settles them itself.
struct Fine1List {
    uint64_t *e;
    int *count;
    int cap;
};

// The scan: the batch's coarse-level bytes as one flat [query][user] array, 64 per lane and 2,048 per
// warp and step (a lane's bytes nearly always lie in one query row; a lane across a row's end goes
// byte by byte).
__global__ void __launch_bounds__(256) qsrp_fine1_scan_kernel(uint8_t *__restrict__ lvc, Round1Src src, int64_t n_user,
                                                             int nq, double inv_user, int S, int W, int mode,
                                                             QsrpParams *__restrict__ par, Fine1List fl,
                                                             int *__restrict__ fhist, int *__restrict__ mismatch,
                                                             int *__restrict__ n_hits) {
    constexpr int kLaneBytes = 64, kSeg = 32 * kLaneBytes;  // bytes per lane and per warp step
    const int64_t total = n_user * nq;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = (int64_t) gridDim.x * (blockDim.x / 32) * kSeg;
    // the lane's 64 bytes of a step (zero past the end), as four aligned 16-byte loads
    auto load = [&](int64_t seg, uint4 w[4]) {
        const int64_t base = seg + (int64_t) lane * kLaneBytes;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int64_t b = base + 16 * k;
            if (b + 16 <= total) {
                w[k] = *reinterpret_cast<const uint4 *>(lvc + b);
            } else {
                uint32_t x[4] = {0u, 0u, 0u, 0u};
                for (int j = 0; j < 16; j++)
                    if (b + j < total) x[j >> 2] |= (uint32_t) lvc[b + j] << (8 * (j & 3));
                w[k] = make_uint4(x[0], x[1], x[2], x[3]);
            }
        }
    };
    uint4 wn[4] = {};
    if (warp * kSeg < total) load(warp * kSeg, wn);
    for (int64_t seg = warp * kSeg; seg < total; seg += stride) {
        const int64_t base = seg + (int64_t) lane * kLaneBytes;
        // this step's bytes, and the next step's loads in flight while they are examined
        uint4 cur[4] = {wn[0], wn[1], wn[2], wn[3]};
        if (seg + stride < total) load(seg + stride, wn);
        const uint32_t *w = reinterpret_cast<const uint32_t *>(cur);  // 16 words, byte e in word e >> 2
        // the step's first query and the end of its row, once per warp; a lane's row follows from
        // them by additions
        int64_t qs = 0, e0 = 0;
        if (lane == 0) {
            qs = (int64_t) ((double) seg * inv_user);
            if (qs * n_user > seg) qs--;
            else if ((qs + 1) * n_user <= seg) qs++;
            e0 = (qs + 1) * n_user;
        }
        qs = __shfl_sync(0xffffffffu, qs, 0);
        e0 = __shfl_sync(0xffffffffu, e0, 0);
        uint64_t hits = 0;
        if (base < total) {
            int64_t q = qs, edge = e0;
            while (edge <= base) { q++; edge += n_user; }
            int wl = par[q].w_l, wu = par[q].w_u, wa = par[q].w_all;
            if (base + kLaneBytes <= edge && base + kLaneBytes <= total) {
                // the lane's 64 pairs in one query row: four bytes at a time, the nibbles compared in
                // parallel (a byte of t = nibbles ^ wanted is below 0x20, so t + 0x7f keeps its carry
                // inside the byte: bit 7 is set exactly where the nibble differs)
                if (wa) {
                    hits = ~uint64_t(0);
                } else {
                    const uint32_t ml = (uint32_t) (wl >= 0 ? wl : 16) * 0x01010101u;
                    const uint32_t mu = (uint32_t) (wu >= 0 ? wu : 16) * 0x01010101u;
#pragma unroll
                    for (int i = 0; i < 16; i++) {
                        const uint32_t tl = (w[i] & 0x0f0f0f0fu) ^ ml, tu = ((w[i] >> 4) & 0x0f0f0f0fu) ^ mu;
                        const uint32_t diff = ((tl + 0x7f7f7f7fu) & (tu + 0x7f7f7f7fu)) & 0x80808080u;
                        const uint32_t eq = diff ^ 0x80808080u;  // bit 7 of each byte: a nibble matches
                        hits |= (uint64_t) ((eq * 0x00204081u) >> 28) << (4 * i);
                    }
                }
            } else {
                for (int e = 0; e < kLaneBytes; e++) {
                    const int64_t pos = base + e;
                    if (pos >= total) break;
                    if (pos >= edge) {  // the next query (and the one after, for short rows)
                        while (edge <= pos) { q++; edge += n_user; }
                        wl = par[q].w_l; wu = par[q].w_u; wa = par[q].w_all;
                    }
                    const unsigned v = lvc[pos];  // rare: a lane across a row's end (its words stay in registers)
                    hits |= (uint64_t) (wa || (int) (v & 15) == wl || (int) (v >> 4) == wu) << e;
                }
            }
        }
        if (n_hits) {
            const int c = __popcll(hits);
            const int tot = __reduce_add_sync(0xffffffffu, c);
            if (lane == 0 && tot) atomicAdd(n_hits + mode, tot);
        }
        // one hit per lane and round: warp-aggregated appends
        while (__any_sync(0xffffffffu, hits != 0)) {
            const bool have = hits != 0;
            const int e = have ? __ffsll((long long) hits) - 1 : 0;
            const unsigned want = __ballot_sync(0xffffffffu, have);
            const int leader = __ffs(want) - 1;
            int at = 0;
            if (lane == leader) at = atomicAdd(fl.count, __popc(want));
            at = __shfl_sync(0xffffffffu, at, leader) + __popc(want & ((1u << lane) - 1));
            if (have) {
                const int64_t pos = base + e;
                int64_t qq = qs, eq = e0;
                while (eq <= pos) { qq++; eq += n_user; }
                const int64_t u = pos - (eq - n_user);
                const unsigned v = lvc[pos];
                if (at < fl.cap) fl.e[at] = ((uint64_t) qq << 40) | ((uint64_t) u << 8) | v;
                else fine1_hit(mode, par, src, u, (int) qq, v, lvc + pos, S, W, fhist, mismatch);
                hits &= hits - 1;
            }
        }
    }
}

__global__ void __launch_bounds__(256) qsrp_fine1_list_kernel(uint8_t *__restrict__ lvc, Round1Src src, int64_t n_user,
                                                             int S, int W, int mode, QsrpParams *__restrict__ par,
                                                             Fine1List fl, int *__restrict__ fhist,
                                                             int *__restrict__ mismatch) {
    const int n = min(*fl.count, fl.cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t x = fl.e[i];
        const int q = (int) (x >> 40);
        const int64_t u = (int64_t) ((x >> 8) & 0xffffffffu);
        fine1_hit(mode, par, src, u, q, (unsigned) (x & 0xffu), lvc + (int64_t) q * n_user + u, S, W, fhist, mismatch);
    }
}

// Round-1 selection, exact step, one warp per query: each side's k-th smallest level from the fine
// histogram of its critical coarse level, the bounds (L1, U1), the level thresholds of the classes,
// the coarse levels that straddle them (settled pair by pair by the fine pass), and the counts of the
// whole coarse levels on each side of them.  While every pair has ub <= lb, a result (lb <= U*) and a
// prune (ub >= L*) cannot coincide unless L* == U*, so the class counts follow from the two sides'
// counts; a query with a pair that breaks the order (anomaly) counts its classes pair by pair.
// rank(level) is non-decreasing, so the levels with rank <= X form a prefix and the thresholds are
// counts.
__global__ void qsrp_select1f_kernel(const int *__restrict__ lhist, const int *__restrict__ fhist,
                                     const int *__restrict__ anomaly, int64_t n_user, const int32_t *__restrict__ rank,
                                     int S, int n_item, int W, KSpec ks, int nq, QsrpParams *__restrict__ par) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= nq) return;
    const int topk = ks.of(q);
    QsrpParams p = par[q];
    int kl, kh;
    {
        const int *fh = fhist + (int64_t) q * 2 * W;
        const int wl = lvt_level(p.cbl, S) - lvt_lo(p.cbl, S) + 1, wu = lvt_level(p.cbu, S) - lvt_lo(p.cbu, S) + 1;
        kl = lvt_lo(p.cbl, S) + (wl > 1 ? warp_first_reaching(fh, wl, topk - p.cum_l) : 0);
        kh = lvt_lo(p.cbu, S) + (wu > 1 ? warp_first_reaching(fh + W, wu, topk - p.cum_u) : 0);
    }
    p.L1 = level_rank(kl, rank, S, n_item);
    p.U1 = level_rank(kh, rank, S, n_item);
    p.mode1 = p.L1 == p.U1;
    int64_t c_res = 0, c_m1 = 0, c_lt = 0;
    for (int l = lane; l < S + 2; l += 32) {
        const int rl = level_rank(l, rank, S, n_item);
        c_res += rl <= p.U1;
        c_m1 += rl <= p.L1;
        c_lt += rl < p.L1;
    }
    p.lv_res = (int) warp_sum64(c_res) - 1;
    p.lv_m1 = (int) warp_sum64(c_m1) - 1;
    p.lv_pr = (int) warp_sum64(c_lt);
    p.c_res = coarse_last_le(p.lv_res, S);
    p.c_m1 = coarse_last_le(p.lv_m1, S);
    p.c_pr = coarse_first_gt(p.lv_pr - 1, S);
    p.res_fine = 0;
    p.ple_fine = 0;
    p.n_res1 = 0;
    p.n_pr1 = 0;
    p.n_ref1 = 0;
    if (p.mode1) {
        p.amb_l = coarse_straddle(p.lv_m1, S);
        p.amb_u = coarse_straddle(p.lv_m1, S);
    } else if (anomaly[q]) {
        p.exact1 = 1;
        p.w_all = 1;
    } else {
        p.amb_l = coarse_straddle(p.lv_res, S);
        p.amb_u = coarse_straddle(p.lv_pr - 1, S);
        // the whole coarse levels: lower side <= lv_res, upper side <= lv_pr - 1
        int hl[kLvEntries], hu[kLvEntries];
        coarse_counts(lhist + (int64_t) q * 2 * kLvEntries, kLvEntries - 1, n_user, hl);
        coarse_counts(lhist + (int64_t) q * 2 * kLvEntries + kLvEntries, 0, n_user, hu);
        int64_t nres = 0, nle = 0;
        for (int b = 0; b < kLvEntries; b++) {
            if (coarse_all_le(b, p.lv_res, S)) nres += hl[b];
            if (coarse_all_le(b, p.lv_pr - 1, S)) nle += hu[b];
        }
        p.n_res1 = (int) nres;
        p.n_pr1 = (int) nle;  // until qsrp_final1: users whose upper level is <= lv_pr - 1 (whole levels)
    }
    p.w_l = p.amb_l;
    p.w_u = p.amb_u;
    if (lane == 0) par[q] = p;
}

// Round-1 closing rules (PruneCandidateByBound.hpp:93-94, 139-150).
__global__ void qsrp_final1_kernel(QsrpParams *__restrict__ par, int nq, KSpec ks, int64_t n_user) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int topk = ks.of(q);
    QsrpParams p = par[q];
    if (p.mode1) {
        p.n_res1 = topk;
        p.n_pr1 = 0;
        p.n_ref1 = 0;
    } else {
        if (!p.exact1) {
            p.n_res1 += p.res_fine;
            p.n_pr1 = (int) (n_user - p.n_pr1 - p.ple_fine);
            p.n_ref1 = (int) (n_user - p.n_res1 - p.n_pr1);
        }
        if (p.n_res1 + p.n_ref1 == topk) {
            p.all1 = 1;
            p.n_res1 = topk;
            p.n_ref1 = 0;
        }
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
    p.amb_l = -1;
    p.amb_u = -1;
    par[q] = p;
}

// ---- round 2 -------------------------------------------------------------------------------------

// Round 2 per (user chunk, query): pairs that did not reach round 2 get their round-1 state code in
// place of the group code; the others are counted by group (per-warp shared-memory copies).
// The word of w holding byte e (0 .. 15), without indexing the array by a run-time value.
__device__ __forceinline__ uint32_t word_of(const uint32_t w[4], int e) {
    return e < 8 ? (e < 4 ? w[0] : w[1]) : (e < 12 ? w[2] : w[3]);
}

// Pass 0: the round-1 class of every pair (non-survivors' codes rewritten to kCodeResult1 /
// kCodePruned1), the survivors counted by code for codes below cap only, and the survivors' total at
// index nb + 1 of the row: qsrp_select2c takes the critical group from those low groups and the
// lumped count of the rest, where that is exact, and otherwise flags the query for pass 1.  Most
// codes are at or above cap (at config 2, 89% of pairs), so most bytes cost a few word operations.
// Pass 1 (flagged queries only): every survivor's code counted (codes 0 .. nb; the non-survivors'
// rewritten codes lie above nb).  Row stride of hist_c: nb + 2.
__global__ void __launch_bounds__(kHistThreads) qsrp_round2_kernel(const uint8_t *__restrict__ lvc,
                                                                  uint8_t *__restrict__ code, int64_t n_user,
                                                                  const QsrpParams *__restrict__ par, int nb, int cap,
                                                                  int pass, int64_t chunk, int *__restrict__ hist_c) {
    // per-thread counts, bin-major ([bin][thread]): a thread's counters sit in its own bank, so the
    // increments of a warp never conflict and need no atomics
    extern __shared__ int h[];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q = blockIdx.y;
    if (pass == 1 && !par[q].r2_full) return;
    const int nbin = pass == 0 ? cap : nb + 1;
    QsrpParams p;
    {
        const QsrpParams &g = par[q];
        p.mode1 = g.mode1; p.all1 = g.all1; p.c_res = g.c_res; p.c_pr = g.c_pr; p.c_m1 = g.c_m1;
    }
    const bool all_survive = lvc == nullptr;  // QS and US: no round 1
    // The common classes of round 1 four bytes at a time (nibbles n < 16, so n + k with k <= 0x80
    // keeps its carry inside the byte): cl > c_res is bit 7 of cl + 0x7f - c_res, cu >= c_pr bit 7 of
    // cu + 0x80 - c_pr, and a zero low nibble marks a pair the fine pass resolved.  Bytes flagged by
    // any of the three take class1_coarse; the others are round-2 survivors.  Codes below cap:
    // bit 7 clear in c + 0x80 - cap (codes are at most nb < 0x60 here).
    const bool swar = !all_survive && !p.mode1 && !p.all1;
    const uint32_t kres = (uint32_t) (0x7f - p.c_res) * 0x01010101u;
    const uint32_t kpr = (uint32_t) (0x80 - p.c_pr) * 0x01010101u;
    const uint32_t kcap = (uint32_t) (0x80 - cap) * 0x01010101u;
    for (int b = 0; b < nbin; b++) h[b * kHistThreads + tid] = 0;
    const uint8_t *lrow = lvc ? lvc + (int64_t) q * n_user : nullptr;
    uint8_t *crow = code + (int64_t) q * n_user;
    const int64_t u0 = (int64_t) blockIdx.x * chunk, u1 = min(u0 + chunk, n_user);
    int n_surv = 0;
    // 16 consecutive users per thread and step, their bytes from five aligned words per row
    for (int64_t ub = u0 + (int64_t) tid * 16; ub < u1; ub += (int64_t) kHistThreads * 16) {
        const int n = (int) min((int64_t) 16, u1 - ub);
        const uint32_t valid = n >= 16 ? 0xffffu : (1u << n) - 1u;
        uint32_t cw[4];
        load16_bytes(crow + ub, cw);
        if (pass == 1) {
#pragma unroll
            for (int e = 0; e < 16; e++) {
                const unsigned c = (cw[e >> 2] >> (8 * (e & 3))) & 0xffu;
                if (((valid >> e) & 1u) && c <= (unsigned) nb) h[c * kHistThreads + tid]++;
            }
            continue;
        }
        uint32_t lw[4] = {0u, 0u, 0u, 0u};
        if (!all_survive) load16_bytes(lrow + ub, lw);
        uint32_t flag = 0, low = 0;  // bytes whose class takes class1_coarse; codes below cap
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const uint32_t lt = ((cw[i] + kcap) & 0x80808080u) ^ 0x80808080u;
            low |= ((lt * 0x00204081u) >> 28) << (4 * i);
            if (swar) {
                const uint32_t lo = lw[i] & 0x0f0f0f0fu, hi = (lw[i] >> 4) & 0x0f0f0f0fu;
                const uint32_t le_res = ((lo + kres) & 0x80808080u) ^ 0x80808080u;
                const uint32_t ge_pr = (hi + kpr) & 0x80808080u;
                const uint32_t zero = ((lo + 0x7f7f7f7fu) & 0x80808080u) ^ 0x80808080u;
                flag |= (((le_res | ge_pr | zero) * 0x00204081u) >> 28) << (4 * i);
            }
        }
        if (!all_survive && !swar) flag = 0xffffu;
        flag &= valid;
        low &= valid;
        int n_out = 0;
        for (uint32_t m = flag | low; m; m &= m - 1) {
            const int e = __ffs(m) - 1;
            const unsigned c = (word_of(cw, e) >> (8 * (e & 3))) & 0xffu;
            bool surv = true;
            if ((flag >> e) & 1u) {
                const unsigned v = (word_of(lw, e) >> (8 * (e & 3))) & 0xffu;
                const int k = class1_coarse(p, v);
                surv = k == kClsRefine || k == kClsIdle;
                if (!surv) {
                    crow[ub + e] = k == kClsResult ? kCodeResult1 : kCodePruned1;
                    n_out++;
                }
            }
            if (surv && c < (unsigned) cap) h[c * kHistThreads + tid]++;
        }
        n_surv += n - n_out;
    }
    __syncthreads();
    int *gh = hist_c + (int64_t) q * (nb + 2);
    for (int b = warp; b < nbin; b += kHistThreads / 32) {
        int sum = 0;
        for (int t = lane; t < kHistThreads; t += 32) sum += h[b * kHistThreads + t];
        sum = __reduce_add_sync(0xffffffffu, sum);
        if (lane == 0 && sum) atomicAdd(gh + b, sum);
    }
    if (pass == 0) {
        n_surv = __reduce_add_sync(0xffffffffu, n_surv);
        if (lane == 0 && n_surv) atomicAdd(gh + nb + 1, n_surv);
    }
}

// Round-2 selection, coarse step (second PruneCandidateByBound call, QSRPNormalLP.hpp:187-190):
// the coarse group holding the kp-th smallest bucket among the users that reached round 2
// (kp = topk - round-1 results), or, with fewer such users than kp, the highest occupied group.
// Pass 0 reads the capped histogram of qsrp_round2_kernel's pass 0: when the kp-th smallest code lies
// at least two groups below cap, every group from cap on lies beyond the upper bound of the k-th
// bucket's neighbour (their buckets are pruned, PruneCandidateByBound.hpp:83-150) and their count is
// the survivors' total minus the low groups', kept in group cap; otherwise the query is flagged for
// the full histogram (pass 1 of both kernels).
__global__ void qsrp_select2c_kernel(int *__restrict__ hist_c, int nb, int cap, int pass, const int32_t *__restrict__ rank,
                                     int gs, KSpec ks, int nq, QsrpParams *__restrict__ par,
                                     QueryCounts *__restrict__ counts) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int topk = ks.of(q);
    QsrpParams p = par[q];
    if (pass == 1 && !p.r2_full) return;
    if (pass == 0) p.r2_full = 0;
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
    int *h = hist_c + (int64_t) q * (nb + 2);
    const int kp = topk - p.n_res1;
    if (pass == 0 && cap <= nb - 1) {
        const int64_t total = h[nb + 1];
        int64_t cum = 0;
        int crit = -1;
        if (total >= kp)
            for (int g = 0; g < cap; g++) {
                if (cum + h[g] >= kp) { crit = g; break; }
                cum += h[g];
            }
        const int lo_b = max(0, (crit + 1) * gs - 2);  // at or above the k-th bucket's lower neighbour
        if (crit >= 0 && crit <= cap - 2 && rank[cap * gs] > rank[lo_b]) {
            int64_t low = 0;
            for (int g = 0; g < cap; g++) low += h[g];
            h[cap] = (int) (total - low);
            p.n_elig2 = (int) total;
            p.crit = crit;
            p.cum_before = (int) cum;
            p.r2_full = 0;
            if (p.crit < nb) p.mask1 = (int32_t) (1u << p.crit);
            par[q] = p;
            return;
        }
        // the full histogram: pass 1 recounts every group
        for (int g = 0; g <= nb + 1; g++) h[g] = 0;
        p.r2_full = 1;
        par[q] = p;
        return;
    }
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
                                     const int32_t *__restrict__ rank, int n_item, KSpec ks, int nq,
                                     QsrpParams *__restrict__ par, uint8_t *__restrict__ cls2,
                                     uint8_t *__restrict__ clsg, int *__restrict__ any2) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= nq) return;
    const int topk = ks.of(q);
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
                                   KSpec ks, int nq, const int32_t *__restrict__ reg_rank, int S_reg, int n_item,
                                   QsrpParams *__restrict__ par, uint8_t *__restrict__ cls2, uint8_t *__restrict__ clsg,
                                   QueryCounts *__restrict__ counts) {
    const int q = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (q >= nq) return;
    const int topk = ks.of(q);
    QsrpParams p = par[q];
    if (p.skip2) return;
    if (reg_rank) {
        // the largest regression level whose rank is <= L2 (the equal-bounds rule in level space)
        int64_t c_le = 0;
        for (int l = lane; l < S_reg + 2; l += 32) c_le += level_rank(l, reg_rank, S_reg, n_item) <= p.L2;
        p.lv_m2 = (int) warp_sum64(c_le) - 1;
    }
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
        const int *hc = hist_c + (int64_t) q * (nb + 2);
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
    const uint8_t *lvc;  // coarse round-1 levels (QSRP), or nullptr
    Round1Src src;       // the reference's round-1 levels, recomputed
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
    int kstride;  // row stride of the result arrays (the batch's largest k)
    int32_t *res_user, *res_rank;
    uint8_t *res_fresh;
    int32_t *cand_user, *cand_query, *cand_lb, *cand_ub;
    __device__ bool query_active(int q) const { return true; }
    // Users whose code can make them a result or a candidate: a group the compaction must
    // classify, a round-1 result, or any non-survivor under the equal-bounds rule.
    // The needed users among 16 codes of query q (bit e for w's byte e).
    __device__ uint32_t need_bits(int q, const uint32_t w[4]) const {
        const QsrpParams &p = par[q];
        const uint64_t gneed = (uint64_t) (uint32_t) p.gneed_lo | ((uint64_t) (uint32_t) p.gneed_hi << 32);
        const bool state_any = !p.skip2 && p.mode2;
        uint32_t m = 0;
        if ((gneed & (gneed + 1)) == 0) {
            // the needed groups are 0 .. gmax (the classes rise with the group): four codes at a time.
            // A byte's (c | 0x80) - (gmax + 1) stays inside the byte, bit 7 set exactly when c > gmax;
            // kCodeResult1 is found as a zero byte of c ^ 0xfe; with state_any every code above nb
            // (the two round-1 codes, bit 7 set) is needed too
            const int gmax1 = __popcll(gneed);  // gmax + 1
            const uint32_t g1 = (uint32_t) gmax1 * 0x01010101u;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const uint32_t x = w[i];
                const uint32_t le = (((x | 0x80808080u) - g1) & 0x80808080u) ^ 0x80808080u;
                const uint32_t t = x ^ 0xfefefefeu;
                const uint32_t fe = ~(((t & 0x7f7f7f7fu) + 0x7f7f7f7fu) | t) & 0x80808080u;
                const uint32_t nd = le | fe | (state_any ? (x & 0x80808080u) : 0u);
                m |= ((nd * 0x00204081u) >> 28) << (4 * i);
            }
        } else {
#pragma unroll
            for (int e = 0; e < kCompactPer; e++) m |= (uint32_t) need_byte(q, (w[e >> 2] >> (8 * (e & 3))) & 0xff) << e;
        }
        return m;
    }
    __device__ bool need_byte(int q, unsigned c) const {
        const QsrpParams &p = par[q];
        const uint64_t gneed = (uint64_t) (uint32_t) p.gneed_lo | ((uint64_t) (uint32_t) p.gneed_hi << 32);
        return c <= (unsigned) nb ? (bool) (gneed >> c & 1) : (c == kCodeResult1 || (!p.skip2 && p.mode2));
    }
    __device__ uint32_t need_mask(int q, int64_t u, int n) const {
        uint32_t w[4];
        load16_bytes(code + (int64_t) q * n_user + u, w);
        const uint32_t m = need_bits(q, w);
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
            if (c != kCodeResult1) {
                // the equal-bounds rule scans every user: decided from the coarse levels where no
                // level threshold straddles them
                const unsigned v = lvc[at];
                if ((v & 15) != kLvcResolved) {
                    const int cl = (int) (v & 15), cu = (int) (v >> 4);
                    if (coarse_all_gt(cu, p.lv_m2, S_reg) || coarse_all_gt(cl, p.lv_m2, S_reg)) return 0;
                    if (!with_aux && coarse_all_le(cu, p.lv_m2, S_reg) && coarse_all_le(cl, p.lv_m2, S_reg)) return 1;
                }
            }
            const uint32_t v = src.levels(u, q);
            const int lb1 = level_rank((int) (v & 0xffffu), reg_rank, S_reg, n_item);
            const int ub1 = level_rank((int) (v >> 16), reg_rank, S_reg, n_item);
            aux.rank = lb1; aux.lb = lb1; aux.ub = ub1;
            if (c == kCodeResult1) return 1;
            return (ub1 <= p.L2 && lb1 <= p.L2) ? 1 : 0;
        }
        return 0;
    }
    __device__ void emit_result(int q, int pos, int64_t u, const Aux &aux) const {
        const int64_t i = (int64_t) q * kstride + pos;
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
// score from its latest earlier round-2 query in the batch, else the carried state.  With req_first
// (the first query of each query's request) only the request's own earlier queries count and a
// request starts from a fresh state (zero scores), as a fresh index would.
__global__ void __launch_bounds__(128, 8) qsrp_result_fill_kernel(const QueryCounts *__restrict__ counts, const int32_t *__restrict__ res_user,
                                        const uint8_t *__restrict__ res_fresh, const uint8_t *__restrict__ code,
                                        QipView sc, int64_t n_user, const float *__restrict__ state,
                                        const int32_t *__restrict__ req_first, int kstride,
                                        float *__restrict__ res_qip) {
    const int q = blockIdx.x;
    const int n = counts[q].n_res_emit;
    const int first = req_first ? req_first[q] : 0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int64_t i = (int64_t) q * kstride + k;
        const int u = res_user[i];
        int src = res_fresh[i] ? q : -1;
        for (int qq = q - 1; src < 0 && qq >= first; qq--)
            if (code[(int64_t) qq * n_user + u] < kCodeResult1) src = qq;
        res_qip[i] = src >= 0 ? sc.exact(u, src) : (req_first ? 0.0f : state[u]);
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

// A user shard's round-1 class counts from the fine pass (mode 1), summed over the shards: the
// counters that pass adds to are copied out (their values before it are 0, or the summed whole-level
// counts of qsrp_select1f for n_res1 / n_pr1 when the query is not counted pair by pair), summed,
// and written back.
__global__ void qsrp_shard_counts1_kernel(QsrpParams *__restrict__ par, int nq, int32_t *__restrict__ buf, int unpack) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    QsrpParams &p = par[q];
    int32_t *b = buf + (int64_t) q * 5;
    if (!unpack) {
        b[0] = p.res_fine;
        b[1] = p.ple_fine;
        b[2] = p.w_all ? p.n_res1 : 0;
        b[3] = p.w_all ? p.n_pr1 : 0;
        b[4] = p.w_all ? p.n_ref1 : 0;
        return;
    }
    p.res_fine = b[0];
    p.ple_fine = b[1];
    if (p.w_all) {
        p.n_res1 = b[2];
        p.n_pr1 = b[3];
        p.n_ref1 = b[4];
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

static int shard_sum_counts1(rkr_index *ix, QsrpParams *par, int nq, cudaStream_t st) {
    RKR_TRY(ix->ws_shard.ensure(sizeof(int32_t) * 5 * (size_t) nq));
    int32_t *buf = ix->ws_shard.as<int32_t>();
    qsrp_shard_counts1_kernel<<<(nq + 127) / 128, 128, 0, st>>>(par, nq, buf, 0);
    RKR_CUDA(cudaGetLastError());
    RKR_TRY(shard_sum(ix, buf, 5 * (int64_t) nq, st));
    qsrp_shard_counts1_kernel<<<(nq + 127) / 128, 128, 0, st>>>(par, nq, buf, 1);
    RKR_CUDA(cudaGetLastError());
    return RKR_OK;
}

// Runs a batch's phase 1: eagerly, or, with ix->graphs_on, from a CUDA graph of the same launches.  A
// shape (method, batch size, workspace addresses) runs eagerly the first time -- that sizes every
// buffer it touches -- and is captured the second time and replayed from then on.  A capture that
// fails (an operation not allowed while capturing) turns graphs off for the index and runs eagerly.
template <class F> static int run_phase1(rkr_index *ix, int method, int nq, cudaStream_t st, F &&phase1) {
    if (!ix->graphs_on || ix->prof.on || ix->sharded()) return phase1(false);
    const void *ws[8] = {ix->ws_qtr.p, ix->ws_levels.p, ix->ws_cls.p, ix->ws_counts.p,
                         ix->ws_hist.p, ix->ws_fix.p, ix->ws_sc.p, ix->ws_km.p};
    rkr_index::PhaseGraph *hit = nullptr;
    for (auto &g : ix->graphs)
        if (g.method == method && g.nq == nq && std::equal(ws, ws + 8, g.ws)) hit = &g;
    if (hit && hit->exec) {
        RKR_CUDA(cudaGraphLaunch(hit->exec, st));
        return RKR_OK;
    }
    if (!hit) {
        RKR_TRY(phase1(false));
        rkr_index::PhaseGraph g;
        g.method = method;
        g.nq = nq;
        // the buffers as they are after the eager run
        const void *now[8] = {ix->ws_qtr.p, ix->ws_levels.p, ix->ws_cls.p, ix->ws_counts.p,
                              ix->ws_hist.p, ix->ws_fix.p, ix->ws_sc.p, ix->ws_km.p};
        std::copy(now, now + 8, g.ws);
        g.exec = nullptr;
        ix->graphs.push_back(g);
        return RKR_OK;
    }
    cudaGraph_t graph = nullptr;
    RKR_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = phase1(false);
    const cudaError_t e = cudaStreamEndCapture(st, &graph);
    cudaGraphExec_t exec = nullptr;
    if (rc == RKR_OK && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        cudaGraphDestroy(graph);
        hit->exec = exec;
        RKR_CUDA(cudaGraphLaunch(exec, st));
        return RKR_OK;
    }
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    ix->graphs_on = false;
    return phase1(false);
}

// One chunk of queries.  QSRPNormalLP runs both rounds; QS and US (no regression round, scores
// in the original space) run the scores tile without levels and start at round 2.
int pair_chunk(rkr_index *ix, int method, const float *d_query, int nq, const BatchSpec &bs, rkr_user_rank *d_out,
               rkr_query_stats *d_stats, cudaStream_t st) {
    const bool qsrp = method == RKR_METHOD_QSRP_NORMAL_LP;
    int kmax = bs.topk;
    if (bs.k) kmax = *std::max_element(bs.k, bs.k + nq);
    const int64_t U = ix->n_user;
    const int64_t Ug = ix->n_user_all();  // a user shard selects over every shard's users
    const int dim = ix->dim, c = ix->check_dim, S = ix->n_sample, Sr = ix->n_sample_reg;
    const int n_item = (int) ix->n_item;
    const int gs = thr_group(S), nb = (S + gs - 1) / gs;
    const int W = qsrp ? lvt_width(Sr) : 1;
    const size_t n_lhist = (size_t) nq * 2 * kLvEntries, n_fhist = (size_t) nq * 2 * W;
    RKR_TRY(ix->ws_qtr.ensure(carve_size((size_t) nq * dim, 4) + carve_size(nq, 4) + carve_size(nq, sizeof(QsrpParams)) +
                              carve_size(nq, 4) + carve_size(1, 4) * 3 + carve_size(2, 4) * 3 + carve_size(n_lhist, 4) +
                              carve_size(n_fhist, 4) + carve_size(nq, 4) * 2 + carve_size(nq, 8)));
    uint8_t *p0 = ix->ws_qtr.as<uint8_t>();
    float *qtr = carve<float>(p0, (size_t) nq * dim);
    // per-query k, output offsets and request starts, when given
    KSpec ks;
    ks.kmax = kmax;
    ks.k = nullptr;
    int32_t *d_k = carve<int32_t>(p0, nq);
    int64_t *d_out_off = carve<int64_t>(p0, nq);
    int32_t *d_req_first = carve<int32_t>(p0, nq);
    if (bs.k) {
        std::vector<int64_t> oo(nq);
        int64_t acc = 0;
        for (int q = 0; q < nq; q++) { oo[q] = acc; acc += bs.k[q]; }
        RKR_CUDA(cudaMemcpyAsync(d_k, bs.k, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, st));
        RKR_CUDA(cudaMemcpyAsync(d_out_off, oo.data(), sizeof(int64_t) * nq, cudaMemcpyHostToDevice, st));
        ks.k = d_k;
    }
    if (bs.req_first)
        RKR_CUDA(cudaMemcpyAsync(d_req_first, bs.req_first, sizeof(int32_t) * nq, cudaMemcpyHostToDevice, st));
    float *qnorm = carve<float>(p0, nq);
    QsrpParams *par = carve<QsrpParams>(p0, nq);
    uint8_t *pz = p0;  // from here on zeroed per chunk
    int *anomaly = carve<int>(p0, nq);
    int *fix_count = carve<int>(p0, 1);
    int *any2 = carve<int>(p0, 1);
    int *hit_count = carve<int>(p0, 2);
    int *mismatch = carve<int>(p0, 1);
    int *n_hits = carve<int>(p0, 2);
    int *f1_count = carve<int>(p0, 2);
    int *lhist = carve<int>(p0, n_lhist);
    int *fhist = carve<int>(p0, n_fhist);
    // code [nq][U], then (QSRP) the coarse levels from the next 256-byte boundary (16-byte vector scans)
    const size_t code_bytes = ((size_t) nq * U + 255) & ~size_t(255);
    RKR_TRY(ix->ws_levels.ensure(code_bytes + (qsrp ? (size_t) nq * U + 256 : 0)));
    uint8_t *code = ix->ws_levels.as<uint8_t>();
    uint8_t *lvc = qsrp ? code + code_bytes : nullptr;
    RKR_TRY(ix->ws_cls.ensure(carve_size((size_t) nq * (S + 1), 1) + carve_size((size_t) nq * (nb + 1), 1)));
    RKR_TRY(ix->ws_counts.ensure(sizeof(QueryCounts) * (size_t) nq));
    const size_t n_hist_c = (size_t) nq * (nb + 2), n_hist_f = (size_t) nq * (S + 1);
    RKR_TRY(ix->ws_hist.ensure(carve_size(n_hist_c, 4) + carve_size(n_hist_f, 4)));
    const int fix_cap = (int) std::min<int64_t>(int64_t(1) << 26, std::max<int64_t>(int64_t(1) << 20, U * nq / 64));
    const int hit_cap = 1 << 24;  // fine-pass hits listed per batch (config 4: about 6.6 M per 1,000 queries)
    RKR_TRY(ix->ws_fix.ensure(carve_size(fix_cap, sizeof(int4)) + carve_size(hit_cap, 8) + carve_size(1, 4)));
    uint8_t *pc = ix->ws_cls.as<uint8_t>();
    uint8_t *cls2 = carve<uint8_t>(pc, (size_t) nq * (S + 1));
    uint8_t *clsg = carve<uint8_t>(pc, (size_t) nq * (nb + 1));
    QueryCounts *counts = ix->ws_counts.as<QueryCounts>();
    uint8_t *ph = ix->ws_hist.as<uint8_t>();
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
    int *n_rescored = carve<int>(pm, 1);
    RegModel m;
    m.rec = ix->reg.as<float>();
    m.rank = ix->reg_rank.as<int32_t>();
    m.S = Sr;
    m.err_cap = (double) Sr - 1e-3;
    m.n_item = n_item;
    Round1Src r1;
    r1.svd_user = ix->svd_user.as<float>();
    r1.qtr = qtr;
    r1.unorm = ix->svd_unorm.as<float>();
    r1.qnorm = qnorm;
    r1.m = m;
    r1.dim = dim;
    r1.c = c;
    QipView qv;
    qv.urow = (qsrp ? ix->svd_user : ix->user).as<float>();
    qv.qrow = qsrp ? qtr : d_query;
    qv.dim = dim;
    qv.c = qsrp ? c : dim;
    qv.n_exact = ix->prof.on ? n_rescored : nullptr;
    const float *thr = ix->thr.as<float>();
    const int32_t *srank = ix->sample_rank.as<int32_t>();
    const unsigned fg2 = 148 * 16;
    const double inv_user = 1.0 / (double) U;
    // Phase 1: both bound rounds up to the round-2 class counts.  Its launches have fixed shapes for
    // a given batch size and no host synchronisation, so a caller that serves batches of a few sizes
    // captures it once per size as a CUDA graph and replays it (ix->graphs_on).
    int *sc_status[4] = {nullptr, nullptr, nullptr, nullptr};
    auto phase1 = [&](bool force_exact) -> int {
        RKR_CUDA(cudaMemsetAsync(pz, 0, (size_t) (p0 - pz), st));
        RKR_CUDA(cudaMemsetAsync(n_rescored, 0, sizeof(int), st));
        RKR_CUDA(cudaMemsetAsync(ix->ws_hist.p, 0, (size_t) (ph - ix->ws_hist.as<uint8_t>()), st));

        if (qsrp) {
            timed(ix, st, "transfer_query", [&] {
                transfer_query_kernel<<<nq, 128, 0, st>>>(d_query, ix->transfer_item.as<float>(), dim, c, qtr, qnorm);
            });
            RKR_CUDA(cudaGetLastError());
        } else {
            RKR_CUDA(cudaMemsetAsync(qnorm, 0, sizeof(float) * nq, st));
        }
        // pair codes, coarse levels and their histograms: on the tensor cores with exact resolution of
        // undecided pairs where the shape allows, else on the exact tiles
        bool tc_done = false;
        if (!force_exact) {
            ScoresTcCall call;
            call.qsrp = qsrp;
            call.qrows = qv.qrow;
            call.qnorm = qnorm;
            call.unorm = r1.unorm;
            call.nq = nq;
            call.m = m;
            call.nb = nb;
            call.lvc = lvc;
            call.code = code;
            call.anomaly = qsrp ? anomaly : nullptr;
            call.status = sc_status;
            RKR_TRY(scores_tc(ix, call, st, &tc_done));
        }
        if (!tc_done) {
            // the exact tiles start from clean counts (a tensor-core run that gave up may have left some)
            RKR_CUDA(cudaMemsetAsync(anomaly, 0, sizeof(int) * nq, st));
            Round1Epi e1;
            e1.unorm = r1.unorm;
            e1.qnorm = qnorm;
            e1.thr_summ = ix->thr_summ.as<float>();
            e1.m = m;
            e1.lvc = lvc;
            e1.code = code;
            e1.anomaly = anomaly;
            e1.nb = nb;
            e1.n_user = U;
            e1.n_query = nq;
            e1.fix = fix;
            RKR_TRY(ix->ws_km.ensure(sizeof(float) * (size_t) dim * (size_t) kmajor_ld(nq)));
            RKR_TRY(to_kmajor(qsrp ? qtr : d_query, nullptr, nq, dim, ix->ws_km.as<float>(), st));
            cudaError_t ce = cudaSuccess;
            const KMajor ka = {(qsrp ? ix->svd_user_km : ix->user_km).as<float>(), U, kmajor_ld(U), kmajor_ld(U)};
            const KMajor kb = {ix->ws_km.as<float>(), nq, kmajor_ld(nq), kmajor_ld(nq)};
            // QS / US: one sequential sum over all coordinates (QS.hpp:137-143), seen by finish_hi
            timed(ix, st, "qsrp_scores", [&] { ce = launch_big_split(ka, kb, qsrp ? c : dim, dim, e1, st); });
            RKR_CUDA(ce);
            if (qsrp) {
                timed(ix, st, "qsrp_fix1", [&] {
                    qsrp_fix1_kernel<<<148 * 4, 256, 0, st>>>(fix, m, r1.unorm, qnorm, U, lvc, anomaly);
                });
                RKR_CUDA(cudaGetLastError());
                timed(ix, st, "qsrp_fix1_scan", [&] {
                    qsrp_fix1_scan_kernel<<<148 * 8, 256, 0, st>>>(fix_count, fix_cap, r1, U, nq, lvc, anomaly);
                });
                RKR_CUDA(cudaGetLastError());
            }
        }
        if (qsrp) {
            // the coarse-level histograms, from every pair's final byte
            const int64_t ch = 65536;
            const dim3 g((unsigned) ((U + ch - 1) / ch), (unsigned) nq);
            timed(ix, st, "lvc_hist", [&] { lvc_hist_kernel<<<g, kHistThreads, 0, st>>>(lvc, U, ch, lhist); });
            RKR_CUDA(cudaGetLastError());
            RKR_TRY(shard_sum(ix, lhist, (int64_t) n_lhist, st));
            RKR_TRY(shard_sum(ix, anomaly, nq, st));
        }
        const int64_t chunk = 65536;  // users per round-2 block (its per-thread counters are set up once)
        dim3 hg((unsigned) ((U + chunk - 1) / chunk), (unsigned) nq);
        if (qsrp) {
            timed(ix, st, "qsrp_select1c", [&] {
                qsrp_select1c_kernel<<<(nq + 127) / 128, 128, 0, st>>>(lhist, Ug, ks, nq, Sr, par);
            });
            RKR_CUDA(cudaGetLastError());
            const double inv_u = 1.0 / (double) U;
            Fine1List f1;
            f1.e = hl.e;  // the fine scans of round 2 reuse this list later
            f1.cap = hl.cap;
            f1.count = f1_count;
            timed(ix, st, "qsrp_fine1", [&] {
                qsrp_fine1_scan_kernel<<<148 * 16, 256, 0, st>>>(lvc, r1, U, nq, inv_u, Sr, W, 0, par, f1, fhist, mismatch,
                                                                 ix->prof.on ? n_hits : nullptr);
            });
            RKR_CUDA(cudaGetLastError());
            timed(ix, st, "qsrp_fine1_list", [&] {
                qsrp_fine1_list_kernel<<<148 * 16, 256, 0, st>>>(lvc, r1, U, Sr, W, 0, par, f1, fhist, mismatch);
            });
            RKR_CUDA(cudaGetLastError());
            RKR_TRY(shard_sum(ix, fhist, (int64_t) n_fhist, st));
            timed(ix, st, "qsrp_select1f", [&] {
                qsrp_select1f_kernel<<<(nq + 3) / 4, 128, 0, st>>>(lhist, fhist, anomaly, Ug, m.rank, Sr, n_item, W, ks,
                                                                   nq, par);
            });
            RKR_CUDA(cudaGetLastError());
            f1.count = f1_count + 1;
            timed(ix, st, "qsrp_fine1", [&] {
                qsrp_fine1_scan_kernel<<<148 * 16, 256, 0, st>>>(lvc, r1, U, nq, inv_u, Sr, W, 1, par, f1, fhist, mismatch,
                                                                 ix->prof.on ? n_hits : nullptr);
            });
            RKR_CUDA(cudaGetLastError());
            timed(ix, st, "qsrp_fine1_list", [&] {
                qsrp_fine1_list_kernel<<<148 * 16, 256, 0, st>>>(lvc, r1, U, Sr, W, 1, par, f1, fhist, mismatch);
            });
            RKR_CUDA(cudaGetLastError());
            if (ix->sharded()) RKR_TRY(shard_sum_counts1(ix, par, nq, st));
            timed(ix, st, "qsrp_final1", [&] { qsrp_final1_kernel<<<(nq + 127) / 128, 128, 0, st>>>(par, nq, ks, Ug); });
            RKR_CUDA(cudaGetLastError());
        } else {
            qs_params_kernel<<<(nq + 127) / 128, 128, 0, st>>>(par, nq, Ug);
            RKR_CUDA(cudaGetLastError());
        }
        // round 2's group histogram: the low groups first (pass 0), the full histogram only for the
        // queries whose selection reaches the lumped groups (pass 1)
        const int cap = kRound2Cap <= nb - 1 ? kRound2Cap : nb + 1;  // nb + 1: every group exact in pass 0
        const int32_t *srank_d = ix->sample_rank.as<int32_t>();
        for (int pass = 0; pass < 2; pass++) {
            const size_t smem_r2 = (size_t) (pass == 0 ? cap : nb + 1) * kHistThreads * sizeof(int);
            if (pass == 1) RKR_TRY(shard_snapshot(ix, 0, hist_c, (int64_t) n_hist_c, st));
            timed(ix, st, "qsrp_round2", [&] {
                qsrp_round2_kernel<<<hg, kHistThreads, smem_r2, st>>>(lvc, code, U, par, nb, cap, pass, chunk, hist_c);
            });
            RKR_CUDA(cudaGetLastError());
            RKR_TRY(pass == 0 ? shard_sum(ix, hist_c, (int64_t) n_hist_c, st)
                              : shard_sum_delta(ix, 0, hist_c, (int64_t) n_hist_c, st));
            timed(ix, st, "qsrp_select2c", [&] {
                qsrp_select2c_kernel<<<(nq + 127) / 128, 128, 0, st>>>(hist_c, nb, cap, pass, srank_d, gs, ks, nq, par,
                                                                       counts);
            });
            RKR_CUDA(cudaGetLastError());
        }
        hl.count = hit_count;
        timed(ix, st, "qsrp_fine2", [&] {
            qsrp_fine2_kernel<<<fg2, 256, 0, st>>>(code, qv, U, nq, inv_user, thr, S, gs, par, 0, any2, hl, hist_f);
        });
        RKR_CUDA(cudaGetLastError());
        timed(ix, st, "qsrp_fine2_list", [&] { qsrp_fine2_list_kernel<<<148 * 16, 256, 0, st>>>(hl, qv, U, thr, S, gs, hist_f); });
        RKR_CUDA(cudaGetLastError());
        RKR_TRY(shard_sum(ix, hist_f, (int64_t) n_hist_f, st));
        timed(ix, st, "qsrp_select2f", [&] {
            qsrp_select2f_kernel<<<(nq + 3) / 4, 128, 0, st>>>(hist_f, nb, gs, S, srank, n_item, ks, nq, par, cls2, clsg, any2);
        });
        RKR_CUDA(cudaGetLastError());
        hl.count = hit_count + 1;
        RKR_TRY(shard_snapshot(ix, 1, hist_f, (int64_t) n_hist_f, st));
        timed(ix, st, "qsrp_fine2", [&] {
            qsrp_fine2_kernel<<<fg2, 256, 0, st>>>(code, qv, U, nq, inv_user, thr, S, gs, par, 1, any2, hl, hist_f);
        });
        RKR_CUDA(cudaGetLastError());
        timed(ix, st, "qsrp_fine2_list", [&] { qsrp_fine2_list_kernel<<<148 * 16, 256, 0, st>>>(hl, qv, U, thr, S, gs, hist_f); });
        RKR_CUDA(cudaGetLastError());
        RKR_TRY(shard_sum_delta(ix, 1, hist_f, (int64_t) n_hist_f, st));
        timed(ix, st, "qsrp_final2", [&] {
            qsrp_final2_kernel<<<(nq + 3) / 4, 128, 0, st>>>(hist_c, hist_f, nb, gs, S, ks, nq, qsrp ? m.rank : nullptr, Sr,
                                                             n_item, par, cls2, clsg, counts);
        });
        RKR_CUDA(cudaGetLastError());
        return RKR_OK;
    };
    RKR_TRY(run_phase1(ix, method, nq, st, phase1));
    std::vector<QueryCounts> hc(nq);
    int h_fix = 0, h_mismatch = 0, h_sc[4] = {0, 0, 0, 0};
    RKR_CUDA(cudaMemcpyAsync(hc.data(), counts, sizeof(QueryCounts) * nq, cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaMemcpyAsync(&h_fix, fix_count, sizeof(int), cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaMemcpyAsync(&h_mismatch, mismatch, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (sc_status[0]) {
        RKR_CUDA(cudaMemcpyAsync(&h_sc[0], sc_status[0], sizeof(int), cudaMemcpyDeviceToHost, st));
        for (int i = 1; i < 4; i++)
            RKR_CUDA(cudaMemcpyAsync(&h_sc[i], sc_status[i], sizeof(int), cudaMemcpyDeviceToHost, st));
    }
    RKR_CUDA(cudaStreamSynchronize(st));
    if (ix->prof.on) {
        ix->prof.add_count("screen_undecided_pairs", h_sc[1]);
        ix->prof.add_count("lvt_search_lower_pairs", h_sc[2]);
        ix->prof.add_count("lvt_search_upper_pairs", h_sc[3]);
    }
    int redo = h_sc[0] ? 1 : 0;
    // user shards redo phase 1 together (its counts are summed over them)
    if (ix->sharded()) RKR_TRY(shard_sum_host(ix, redo, &redo, st));
    if (redo) {
        // the tensor-core run gave up (a bounded wait or a full list): the exact tiles redo phase 1
        RKR_TRY(phase1(true));
        h_mismatch = 0;
        RKR_CUDA(cudaMemcpyAsync(hc.data(), counts, sizeof(QueryCounts) * nq, cudaMemcpyDeviceToHost, st));
        RKR_CUDA(cudaMemcpyAsync(&h_fix, fix_count, sizeof(int), cudaMemcpyDeviceToHost, st));
        RKR_CUDA(cudaMemcpyAsync(&h_mismatch, mismatch, sizeof(int), cudaMemcpyDeviceToHost, st));
        RKR_CUDA(cudaStreamSynchronize(st));
    }
    if (h_mismatch) {
        set_error("internal: %d pairs whose exact round-1 level lies outside their coarse level", h_mismatch);
        return RKR_ERR_STATE;
    }
    if (ix->prof.on) ix->prof.add_count("screen_undecided_pairs", h_fix);
    QsrpCompactPolicy pol = {};
    pol.lvc = lvc;
    pol.src = r1;
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
    pol.kstride = kmax;
    if (ix->sharded()) {
        // the candidates of this shard's users (the counts so far are every shard's)
        RKR_TRY(shard_local_counts(ix, pol, nq, counts, st));
        RKR_CUDA(cudaMemcpyAsync(hc.data(), counts, sizeof(QueryCounts) * nq, cudaMemcpyDeviceToHost, st));
        RKR_CUDA(cudaStreamSynchronize(st));
    }
    std::vector<int64_t> off(nq + 1, 0);
    for (int q = 0; q < nq; q++) off[q + 1] = off[q] + hc[q].n_cand;
    const int64_t n_cand = off[nq];
    size_t need = carve_size(nq + 1, 8) + carve_size((size_t) nq * kmax, 4) * 3 + carve_size((size_t) nq * kmax, 1) +
                  carve_size(n_cand, 4) * 5;
    RKR_TRY(ix->ws_cand.ensure(need));
    uint8_t *p = ix->ws_cand.as<uint8_t>();
    int64_t *d_off = carve<int64_t>(p, nq + 1);
    int32_t *res_user = carve<int32_t>(p, (size_t) nq * kmax);
    int32_t *res_rank = carve<int32_t>(p, (size_t) nq * kmax);
    float *res_qip = carve<float>(p, (size_t) nq * kmax);
    uint8_t *res_fresh = carve<uint8_t>(p, (size_t) nq * kmax);
    int32_t *cand_user = carve<int32_t>(p, n_cand);
    int32_t *cand_query = carve<int32_t>(p, n_cand);
    int32_t *cand_lb = carve<int32_t>(p, n_cand);
    int32_t *cand_ub = carve<int32_t>(p, n_cand);
    float *cand_qip = carve<float>(p, n_cand);
    RKR_CUDA(cudaMemcpyAsync(d_off, off.data(), sizeof(int64_t) * (nq + 1), cudaMemcpyHostToDevice, st));
    pol.cand_off = d_off;
    pol.res_user = res_user;
    pol.res_rank = res_rank;
    pol.res_fresh = res_fresh;
    pol.cand_user = cand_user;
    pol.cand_query = cand_query;
    pol.cand_lb = cand_lb;
    pol.cand_ub = cand_ub;
    RKR_TRY(run_compaction(ix, pol, nq, ks, counts, st));
    timed(ix, st, "qsrp_result_fill", [&] {
        qsrp_result_fill_kernel<<<nq, 128, 0, st>>>(counts, res_user, res_fresh, code, qv, U, ix->qip_state.as<float>(),
                                                    bs.req_first ? d_req_first : nullptr, kmax, res_qip);
    });
    RKR_CUDA(cudaGetLastError());
    if (n_cand > 0) {
        timed(ix, st, "qsrp_cand_fill", [&] {
            qsrp_cand_fill_kernel<<<(unsigned) ((n_cand + 255) / 256), 256, 0, st>>>(cand_user, cand_query, n_cand, qv,
                                                                                    cand_qip);
        });
        RKR_CUDA(cudaGetLastError());
    }
    RKR_TRY(refine_and_assemble_pairs(ix, method, d_query, nq, ks, bs.k ? d_out_off : nullptr, counts, res_user,
                                      res_rank, res_qip, n_cand, cand_user, cand_query, cand_lb, cand_ub, cand_qip, d_off,
                                      d_out, d_stats, st));
    // the carried state advances only when requests are not scoped (a scoped request starts fresh)
    if (qsrp && !bs.req_first) timed(ix, st, "qsrp_state", [&] {
        qsrp_state_kernel<<<(unsigned) ((U + 255) / 256), 256, 0, st>>>(code, qv, U, nq, ix->qip_state.as<float>());
    });
    RKR_CUDA(cudaGetLastError());
    if (bs.front) RKR_CUDA(cudaMemcpyAsync(hc.data(), counts, sizeof(QueryCounts) * nq, cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    if (bs.front)
        for (int q = 0; q < nq; q++) bs.front[q] = hc[q].n_res_emit;
    if (ix->prof.on) {
        int h = 0, hh[2] = {0, 0};
        RKR_CUDA(cudaMemcpy(&h, n_rescored, sizeof(int), cudaMemcpyDeviceToHost));
        ix->prof.add_count("rescored_pairs", h);
        if (qsrp) {
            RKR_CUDA(cudaMemcpy(hh, n_hits, sizeof(hh), cudaMemcpyDeviceToHost));
            ix->prof.add_count("fine1_select_pairs", hh[0]);
            ix->prof.add_count("fine1_class_pairs", hh[1]);
        }
    }
    return RKR_OK;
}

}  // namespace rkr
