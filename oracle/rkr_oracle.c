/*
 * rkr_oracle.c -- CPU restatement of the reverse k-ranks index-build and query path of
 * DBGroup-SUSTech/reverse-k-ranks (QSRP), written from the reference's behaviour.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker: only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline / reference legs may load it.  The product path
 * (librkr_b200.so) never links, loads or calls it.
 *
 * Arithmetic contract.  Every float expression below is evaluated in strict IEEE-754 binary32,
 * one rounding per operation, in the reference's source order (no FMA contraction, no
 * reassociation).  That is what the reference's documented build produces (ReadMe.md:23 builds
 * with CMAKE_BUILD_TYPE=Debug, i.e. -O0, CMakeLists.txt:26-28).  Compile this file with
 * -ffp-contract=off and without -ffast-math / -march=native.
 *
 * Every function cites the reference file:line it restates (paths relative to the reference
 * project's root).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "minimax_line.h"

/* ------------------------------------------------------------------------------------------ */
/* basic arithmetic                                                                            */
/* ------------------------------------------------------------------------------------------ */

/* src/include/alg/SpaceInnerProduct.hpp:14-20 -- sequential float dot product. */
static float ip_f32(const float *a, const float *b, int d) {
    float r = 0.0f;
    for (int i = 0; i < d; i++) r += a[i] * b[i];
    return r;
}

float orc_inner_product(const float *a, const float *b, int32_t d) { return ip_f32(a, b, d); }

/* src/include/struct/VectorMatrix.hpp:51-66 -- users are L2-normalised in place; rows whose
 * norm is <= 0.001 are left untouched. */
void orc_normalize(float *v, int64_t n, int32_t d) {
    for (int64_t i = 0; i < n; i++) {
        float *row = v + i * d;
        float l2 = 0.0f;
        for (int j = 0; j < d; j++) l2 += row[j] * row[j];
        l2 = sqrtf(l2);
        if ((double) l2 <= 0.001) continue;
        for (int j = 0; j < d; j++) row[j] /= l2;
    }
}

static int cmp_float_desc(const void *a, const void *b) {
    const float x = *(const float *) a, y = *(const float *) b;
    return (x < y) - (x > y);
}

/* ------------------------------------------------------------------------------------------ */
/* index build                                                                                 */
/* ------------------------------------------------------------------------------------------ */

/* Score rows sorted descending: src/include/score_computation/CPUScoreTable.hpp:372-386
 * (score = InnerProduct(user, item)), ComputeScoreTableBatch.hpp:292-303 (sort, std::greater). */
void orc_score_sort_rows(const float *user, int64_t start_user, int64_t n_rows, const float *item,
                         int64_t n_item, int32_t d, float *rows_out) {
    for (int64_t r = 0; r < n_rows; r++) {
        const float *u = user + (start_user + r) * d;
        float *row = rows_out + r * n_item;
        for (int64_t i = 0; i < n_item; i++) row[i] = ip_f32(u, item + i * d, d);
        qsort(row, (size_t) n_item, sizeof(float), cmp_float_desc);
    }
}

/* Sampled score thresholds: src/app/build-index/BuildSampleIndexByComputation.cpp:111-125 and
 * SampleSearch::LoopPreprocess, src/include/alg/RankBoundRefinement/SampleSearch.hpp:80-85.
 * thr_out[u][j] = j-th sampled position of user u's descending score row. */
void orc_build_thresholds(const float *user, int64_t n_user, const float *item, int64_t n_item,
                          int32_t d, const int32_t *sample_rank, int32_t n_sample, float *thr_out) {
    float *row = (float *) malloc(sizeof(float) * (size_t) n_item);
    for (int64_t u = 0; u < n_user; u++) {
        orc_score_sort_rows(user, u, 1, item, n_item, d, row);
        for (int j = 0; j < n_sample; j++) thr_out[u * n_sample + j] = row[sample_rank[j]];
    }
    free(row);
}

/* Query-rank distribution: src/app/build-index/QueryRankCPU.hpp:357-413 (rank of a sampled item =
 * number of items scoring strictly above it, found by lower_bound with '>' on the sorted row) and
 * src/app/build-index/QueryRankByComputation.hpp:185-191, 231-239 (histogram, then prefix sum).
 * rank_out: [n_user][n_sample_item] (may be NULL); accu_out: [n_sample_item][n_item + 1]. */
void orc_query_rank_distribution(const float *user, int64_t n_user, const float *item, int64_t n_item,
                                 int32_t d, const int32_t *sample_item, int32_t n_sample_item,
                                 int32_t *rank_out, int32_t *accu_out) {
    float *row = (float *) malloc(sizeof(float) * (size_t) n_item);
    memset(accu_out, 0, sizeof(int32_t) * (size_t) n_sample_item * (size_t) (n_item + 1));
    for (int64_t u = 0; u < n_user; u++) {
        const float *uv = user + u * d;
        orc_score_sort_rows(user, u, 1, item, n_item, d, row);
        for (int s = 0; s < n_sample_item; s++) {
            const float sip = ip_f32(uv, item + (int64_t) sample_item[s] * d, d);
            /* std::lower_bound(row, row + n, sip, arr > sip) */
            int64_t lo = 0, len = n_item;
            while (len > 0) {
                int64_t half = len >> 1, mid = lo + half;
                if (row[mid] > sip) { lo = mid + 1; len = len - half - 1; } else { len = half; }
            }
            if (rank_out) rank_out[u * n_sample_item + s] = (int32_t) lo;
            accu_out[(int64_t) s * (n_item + 1) + lo]++;
        }
    }
    for (int s = 0; s < n_sample_item; s++) {
        int32_t *a = accu_out + (int64_t) s * (n_item + 1);
        for (int64_t r = 1; r <= n_item; r++) a[r] += a[r - 1];
    }
    free(row);
}

/* src/app/build-index/QueryRankBySample.hpp:521-541 -- k-th rank of each sampled item: the first
 * rank r with accu[r] >= sample_topk (n_item + 1 if none).  Unsorted order. */
void orc_kth_rank(const int32_t *accu, int64_t n_item, int32_t n_sample_item, int32_t sample_topk,
                  int32_t *kth_out) {
    for (int s = 0; s < n_sample_item; s++) {
        const int32_t *a = accu + (int64_t) s * (n_item + 1);
        int64_t lo = 0, len = n_item + 1;
        while (len > 0) {
            int64_t half = len >> 1, mid = lo + half;
            if (a[mid] < sample_topk) { lo = mid + 1; len = len - half - 1; } else { len = half; }
        }
        kth_out[s] = (int32_t) lo;
    }
}

/* src/include/alg/RankBoundRefinement/FindSampleRank/UniformSample.hpp:17-25 */
void orc_uniform_sample_rank(int32_t n_item, int32_t n_sample, int32_t *out) {
    const int end_sample_rank = n_item - 1;
    const double delta = (end_sample_rank - 0) * 1.0 / n_sample;
    for (int s = 0; s < n_sample; s++) out[s] = (int32_t) floor(s * delta);
}

/* ---- optimal sample ranks (fsr, OptimalPart) ------------------------------------------------ */

typedef struct {
    int64_t n_user, n_item, nsq;
    const int32_t *kth;   /* sorted ascending, [nsq] */
    const int32_t *accu;  /* rows in the same order, [nsq][n_item + 1] */
    int32_t R;
    int32_t *cand;        /* candidate ranks, sorted ascending, unique */
    int32_t *this_last;   /* first query position with kth > cand[r] */
    int32_t *next_first;  /* first query position with kth >= cand[r] + 1 */
} qdist_t;

static int64_t lb_gt(const int32_t *a, int64_t n, int32_t v) { /* first i with a[i] > v */
    int64_t lo = 0, len = n;
    while (len > 0) { int64_t h = len >> 1, m = lo + h; if (a[m] <= v) { lo = m + 1; len -= h + 1; } else len = h; }
    return lo;
}
static int64_t lb_ge(const int32_t *a, int64_t n, int32_t v) { /* first i with a[i] >= v */
    int64_t lo = 0, len = n;
    while (len > 0) { int64_t h = len >> 1, m = lo + h; if (a[m] < v) { lo = m + 1; len -= h + 1; } else len = h; }
    return lo;
}

/* OptimalSampleRank.hpp:300-317 */
static int64_t qd_cost_begin(const qdist_t *q, int r) {
    const int rank = q->cand[r];
    const int end = q->this_last[r];
    int64_t s = 0;
    for (int i = 0; i < end; i++) s += q->accu[(int64_t) i * (q->n_item + 1) + rank];
    return s;
}
/* OptimalSampleRank.hpp:274-298 */
static int64_t qd_cost_end(const qdist_t *q, int r) {
    const int rank = q->cand[r] + 1;
    const int start = q->next_first[r];
    if (start >= q->nsq) return 0;
    int64_t s = 0;
    for (int i = start; i < q->nsq; i++) s += q->n_user - q->accu[(int64_t) i * (q->n_item + 1) + rank - 1];
    return s;
}
/* OptimalSampleRank.hpp:240-272 */
static int64_t qd_cost_between(const qdist_t *q, int r_ub, int r_lb) {
    const int rank_ub = q->cand[r_ub] + 1;
    const int rank_lb = q->cand[r_lb];
    const int begin = q->next_first[r_ub];
    const int end = q->this_last[r_lb];
    if (begin >= q->nsq) return 0;
    if (begin > end) return 0;
    int64_t s = 0;
    for (int i = begin; i < end; i++)
        s += q->accu[(int64_t) i * (q->n_item + 1) + rank_lb] - q->accu[(int64_t) i * (q->n_item + 1) + rank_ub - 1];
    return s;
}
/* OptimalSampleRank.hpp:319-325 */
static int64_t qd_transit(const qdist_t *q, int r_ub, int r_lb) {
    return -qd_cost_end(q, r_ub) + qd_cost_between(q, r_ub, r_lb) + qd_cost_end(q, r_lb);
}

static int cmp_i32(const void *a, const void *b) {
    const int32_t x = *(const int32_t *) a, y = *(const int32_t *) b;
    return (x > y) - (x < y);
}

/* Fill a sorted unique rank set up to n_sample entries, as OptimalSampleRankFast.hpp:289-310 and
 * :412-432 do: first with a double-stepped sweep below last_sample, then with every free rank. */
static int fill_rank_set(int32_t *set, int n_set, int n_sample, int last_sample, int n_item) {
    char *in = (char *) calloc((size_t) n_item + 2, 1);
    for (int i = 0; i < n_set; i++) in[set[i]] = 1;
    const int n_remain = n_sample - n_set;
    const double delta = last_sample * 1.0 / n_remain;
    double ins = 0;
    while (n_set < n_sample && (int) ins < last_sample) {
        if (!in[(int) ins]) { in[(int) ins] = 1; set[n_set++] = (int) ins; ins += delta; }
        else ins += 1;
    }
    int ii = 0;
    while (n_set < n_sample && ii < n_item) {
        if (!in[ii]) { in[ii] = 1; set[n_set++] = ii; }
        ii++;
    }
    free(in);
    qsort(set, (size_t) n_set, sizeof(int32_t), cmp_i32);
    return n_set;
}

/* FindOptimalSampleFast, src/include/alg/RankBoundRefinement/FindSampleRank/OptimalSampleRankFast.hpp:269-451
 * with the "OptimalPart" candidate set of OptimalSampleRank.hpp:49-64 and the position maps of
 * :206-232.  sort_kth: [nsq] ascending; accu_sorted: [nsq][n_item+1] rows in that order.
 * Returns 0 on success, -1 if the set cannot be filled. */
int orc_optimal_sample_rank(int64_t n_user, int64_t n_item, int32_t n_sample, int32_t nsq,
                            const int32_t *sort_kth, const int32_t *accu_sorted,
                            int32_t *out, int64_t *train_cost) {
    qdist_t q;
    q.n_user = n_user; q.n_item = n_item; q.nsq = nsq; q.kth = sort_kth; q.accu = accu_sorted;
    int32_t *tmp = (int32_t *) malloc(sizeof(int32_t) * (size_t) (2 * nsq + 1));
    int nt = 0;
    for (int i = 0; i < nsq; i++) { tmp[nt++] = sort_kth[i]; if (sort_kth[i] != 0) tmp[nt++] = sort_kth[i] - 1; }
    qsort(tmp, (size_t) nt, sizeof(int32_t), cmp_i32);
    int R = 0;
    for (int i = 0; i < nt; i++) if (R == 0 || tmp[R - 1] != tmp[i]) tmp[R++] = tmp[i];
    q.R = R; q.cand = tmp;
    q.this_last = (int32_t *) malloc(sizeof(int32_t) * (size_t) R);
    q.next_first = (int32_t *) malloc(sizeof(int32_t) * (size_t) R);
    for (int r = 0; r < R; r++) {
        q.this_last[r] = (int32_t) lb_gt(sort_kth, nsq, q.cand[r]);
        q.next_first[r] = (int32_t) lb_ge(sort_kth, nsq, q.cand[r] + 1);
    }
    int rc = 0;
    if (train_cost) *train_cost = 0;
    int32_t *set = (int32_t *) malloc(sizeof(int32_t) * (size_t) (n_sample + R + 1));
    if (R <= n_sample) {
        for (int r = 0; r < R; r++) set[r] = q.cand[r];
        const int last = nsq < 500 ? (int) n_item : q.cand[R - 1];
        int n = fill_rank_set(set, R, n_sample, last, (int) n_item);
        if (n != n_sample) rc = -1;
        for (int s = 0; s < n_sample && s < n; s++) out[s] = set[s];
    } else {
        int64_t *cost1 = (int64_t *) malloc(sizeof(int64_t) * (size_t) R);
        for (int r = 0; r < R; r++) cost1[r] = qd_cost_begin(&q, r) + qd_cost_end(&q, r);
        /* transit[lb][ub] for ub < lb, cached as the reference does (OptimalSampleRankFast.hpp:242-252) */
        int64_t *tr = (int64_t *) malloc(sizeof(int64_t) * (size_t) R * (size_t) R);
        for (int lb = 1; lb < R; lb++)
            for (int ub = 0; ub < lb; ub++) tr[(int64_t) lb * R + ub] = qd_transit(&q, ub, lb);
        int64_t *dp = (int64_t *) malloc(sizeof(int64_t) * (size_t) n_sample * (size_t) R);
        int32_t *pos = (int32_t *) malloc(sizeof(int32_t) * (size_t) n_sample * (size_t) R);
        for (int r = 0; r < R; r++) { dp[r] = cost1[r]; pos[r] = r; }
        for (int s = 1; s < n_sample; s++) {
            for (int r = 0; r < R; r++) {
                int64_t best = dp[(int64_t) (s - 1) * R + r];
                int32_t bp = pos[(int64_t) (s - 1) * R + r];
                for (int p = 0; p <= r - 1; p++) {
                    const int64_t c = dp[(int64_t) (s - 1) * R + p] + tr[(int64_t) r * R + p];
                    if (best > c) { best = c; bp = p; }
                }
                dp[(int64_t) s * R + r] = best;
                pos[(int64_t) s * R + r] = bp;
            }
        }
        uint64_t min_cost = UINT64_MAX;
        int idx = -1;
        for (int r = 0; r < R; r++) {
            const uint64_t c = (uint64_t) dp[(int64_t) (n_sample - 1) * R + r];
            if (c < min_cost) { idx = r; min_cost = c; }
        }
        if (train_cost) *train_cost = (int64_t) min_cost;
        for (int s = n_sample - 1; s >= 0; s--) {
            out[s] = q.cand[idx];
            idx = pos[(int64_t) s * R + idx];
        }
        /* redundancy repair, OptimalSampleRankFast.hpp:397-448 */
        int redundant = 0;
        for (int s = 1; s < n_sample && !redundant; s++)
            for (int t = 0; t < s; t++) if (out[t] == out[s]) { redundant = 1; break; }
        if (redundant) {
            int n = 0;
            for (int s = 0; s < n_sample; s++) {
                int seen = 0;
                for (int t = 0; t < n; t++) if (set[t] == out[s]) { seen = 1; break; }
                if (!seen) set[n++] = out[s];
            }
            qsort(set, (size_t) n, sizeof(int32_t), cmp_i32);
            n = fill_rank_set(set, n, n_sample, q.cand[R - 1], (int) n_item);
            if (n != n_sample) rc = -1;
            for (int s = 0; s < n_sample && s < n; s++) out[s] = set[s];
        }
        free(cost1); free(tr); free(dp); free(pos);
    }
    free(set); free(q.this_last); free(q.next_first); free(tmp);
    return rc;
}

/* ---- regression rank-bound model (NormalLinearRegressionLP) ------------------------------- */

/* src/include/util/MathUtil.hpp:10-27 -- ReverseMIPS::sqrt, a Newton-Raphson iteration run until
 * it stops moving.  Inside namespace ReverseMIPS it hides ::sqrt, so it is the function that
 * computes NormalLinearRegressionLP's sqrt_2_ (NormalLinearRegressionLP.hpp:27). */
float orc_sqrt_constexpr(float x) {
    if (!(x >= 0 && x < INFINITY)) return NAN;
    float curr = x, prev = 0.0f;
    while (curr != prev) {
        const float next = (float) (0.5 * (double) (curr + x / curr));
        prev = curr;
        curr = next;
    }
    return curr;
}

/* src/include/alg/RegressionPruning/NormalLinearRegressionLP.hpp:123-143.  Abramowitz & Stegun
 * 7.1.26 approximation of the normal CDF, with the reference's float/double promotions: the
 * constants are float, t and the final expression pass through double, exp() is the double
 * function. */
float orc_cdf_phi(float x) {
    const float a1 = (float) 0.254829592, a2 = (float) -0.284496736, a3 = (float) 1.421413741;
    const float a4 = (float) -1.453152027, a5 = (float) 1.061405429, p = (float) 0.3275911;
    const float sqrt_2 = orc_sqrt_constexpr(2.0f);
    int sign = 1;
    if (x < 0) sign = -1;
    x = fabsf(x) / sqrt_2;
    const float t = (float) (1.0 / (1.0 + (double) (p * x)));
    const float poly_t = (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t;
    const float y = (float) (1.0 - (double) poly_t * exp((double) (-x * x)));
    return (float) (0.5 * (1.0 + (double) ((float) sign * y)));
}

/* Per-user model record: a, b, mu, sigma, err, smax, smin (NormalLinearRegressionLP.hpp:30-35). */

/* NormalLinearRegressionLP::ComputeRankBound, NormalLinearRegressionLP.hpp:326-380. */
void orc_regression_rank_bound(float qlb, float qub, const float *ab, const float *musig, float err,
                               const float *extreme, const int32_t *sample_rank, int32_t n_sample,
                               int64_t n_item, int32_t *rank_lb, int32_t *rank_ub) {
    const float mu = musig[0], sigma = musig[1];
    const float smax = extreme[0], smin = extreme[1];
    if (qlb > smax) *rank_lb = sample_rank[0];
    else if (qlb < smin) *rank_lb = (int32_t) n_item;
    else if ((double) err >= n_sample - 1e-3) *rank_lb = (int32_t) n_item;
    else {
        const float nx = (qlb - mu) / sigma;
        const float ix = orc_cdf_phi(nx);
        const float pred = ix * ab[0] + ab[1];
        const int64_t pr = (int64_t) ceilf(pred + err);
        if (pr >= n_sample) *rank_lb = (int32_t) n_item;
        else if (pr < 0) *rank_lb = sample_rank[0];
        else *rank_lb = sample_rank[pr];
    }
    if (qub > smax) *rank_ub = 0;
    else if (qub < smin) *rank_ub = sample_rank[n_sample - 1];
    else if ((double) err >= n_sample - 1e-3) *rank_ub = 0;
    else {
        const float nx = (qub - mu) / sigma;
        const float ix = orc_cdf_phi(nx);
        const float pred = ix * ab[0] + ab[1];
        const int64_t pr = (int64_t) floorf(pred - err);
        if (pr >= n_sample) *rank_ub = (int32_t) n_item;
        else if (pr < 0) *rank_ub = 0;
        else *rank_ub = sample_rank[pr];
    }
}

/* Level of a rank bound in the engine's encoding: 0 -> rank 0, l in [1, S] -> sample_rank[l - 1],
 * S + 1 -> n_item (the rank bounds ComputeRankBound can return are exactly these). */
static int32_t orc_rank_level(int32_t r, const int32_t *sample_rank, int32_t n_sample, int64_t n_item) {
    if (r == 0) return 0;
    if (r == n_item) return n_sample + 1;
    int32_t lo = 0, hi = n_sample - 1;
    while (lo < hi) {  /* first index with sample_rank[index] >= r */
        const int32_t m = (lo + hi) / 2;
        if (sample_rank[m] < r) lo = m + 1; else hi = m;
    }
    return lo + 1;
}

/* The binary32 values as ordered integers: k(x) < k(y) <=> x < y (no NaN). */
static int64_t orc_fkey(float x) {
    int32_t i;
    memcpy(&i, &x, 4);
    return i >= 0 ? (int64_t) i : -(int64_t) (i & 0x7fffffff);
}
static float orc_fval(int64_t k) {
    const int32_t i = k >= 0 ? (int32_t) k : (int32_t) ((-k) | 0x80000000);
    float x;
    memcpy(&x, &i, 4);
    return x;
}

/* Score boundaries of one user's rank bound, side 0 the lower bound (a function of qlb), side 1 the
 * upper bound (of qub): out[g] = the smallest binary32 score whose level (orc_rank_level of
 * ComputeRankBound, NormalLinearRegressionLP.hpp:326-380) is <= levels[g], g = 0 .. n_out - 1;
 * +inf where no finite score reaches it, -inf where every finite score does.  Bisection on the
 * ordered binary32 values; the level never rises with the score (tests/test_level_monotone.py), so
 * a score's level lies in (levels[g_1], levels[g_0]] for the boundaries g_0, g_1 around it.  A
 * checker for level-boundary tables built on the device; the levels ascend. */
void orc_level_boundaries_at(const float *rec, const int32_t *sample_rank, int32_t n_sample, int64_t n_item,
                             const int32_t *levels, int32_t side, int32_t n_out, float *out) {
    const int64_t klo = orc_fkey(-INFINITY), khi = orc_fkey(INFINITY);
    for (int32_t g = 0; g < n_out; g++) {
        const int32_t L = levels[g];
        /* level(x) <= L is monotone in x: false ... false true ... true; find the first true */
        int64_t lo = klo, hi = khi;  /* invariant: level(fval(hi)) <= L or hi = khi */
        int32_t rl, ru;
        orc_regression_rank_bound(INFINITY, INFINITY, rec, rec + 2, rec[4], rec + 5, sample_rank, n_sample, n_item,
                                  &rl, &ru);
        const int32_t top = orc_rank_level(side ? ru : rl, sample_rank, n_sample, n_item);
        if (top > L) { out[g] = INFINITY; continue; }
        orc_regression_rank_bound(-INFINITY, -INFINITY, rec, rec + 2, rec[4], rec + 5, sample_rank, n_sample, n_item,
                                  &rl, &ru);
        const int32_t bottom = orc_rank_level(side ? ru : rl, sample_rank, n_sample, n_item);
        if (bottom <= L) { out[g] = -INFINITY; continue; }
        while (hi - lo > 1) {
            const int64_t m = lo + (hi - lo) / 2;
            const float x = orc_fval(m);
            orc_regression_rank_bound(x, x, rec, rec + 2, rec[4], rec + 5, sample_rank, n_sample, n_item, &rl, &ru);
            if (orc_rank_level(side ? ru : rl, sample_rank, n_sample, n_item) <= L) hi = m; else lo = m;
        }
        out[g] = orc_fval(hi);
    }
}

/* The same at the levels g * stride, g = 0 .. n_out - 1. */
void orc_level_boundaries(const float *rec, const int32_t *sample_rank, int32_t n_sample, int64_t n_item,
                          int32_t stride, int32_t side, int32_t n_out, float *out) {
    int32_t levels[4096];
    for (int32_t g = 0; g < n_out && g < 4096; g++) levels[g] = g * stride;
    orc_level_boundaries_at(rec, sample_rank, n_sample, n_item, levels, side, n_out < 4096 ? n_out : 4096, out);
}

/* The LP optimum itself (min e s.t. |a x_i + b - y_i| <= e) comes from minimax_line.h.  The
 * reference solves it with a randomised Seidel LP whose constraint order comes from
 * std::random_device (NormalLinearRegressionLP.hpp:97-100), so its (a, b) are not reproducible
 * run to run; the optimal e is. */

/* Fit one user's model from its descending thresholds thr[0..S-1]:
 * AssignCache (NormalLinearRegressionLP.hpp:104-121, 145-179), LinearProgram post-processing
 * (:194-211), and the endpoint-line fallback with CalcError (:215-243, 272-296).
 * rec_out: a, b, mu, sigma, err, smax, smin. */
void orc_fit_regression_user(const float *thr, int32_t S, float *rec_out) {
    float mu = 0.0f;
    for (int s = 0; s < S; s++) mu += thr[s];
    mu = mu / (float) S;
    float sigma = 0.0f;
    for (int s = 0; s < S; s++) { const float m = thr[s] - mu; const float t = m * m; sigma += t; }
    sigma /= (float) S;
    sigma = sqrtf(sigma);
    double *pts = (double *) malloc(sizeof(double) * 4 * (size_t) (S > 1 ? S - 1 : 1));
    int n = 0;
    for (int j = 0; j < S - 1; j++) {
        const float nx = orc_cdf_phi((thr[j + 1] - mu) / sigma);
        const float cx = orc_cdf_phi((thr[j] - mu) / sigma);
        pts[2 * n] = nx; pts[2 * n + 1] = j + 1; n++;
        pts[2 * n] = cx; pts[2 * n + 1] = j + 1; n++;
    }
    double a = 0, b = 0, e = -1;
    if (n > 0) minimax_line(pts, n, &a, &b, &e);
    free(pts);
    float err = (float) e;
    const float fa = (float) a, fb = (float) b;
    if (fa > 0 || fb < 0) err = -1;
    else if (0 < err && err < (float) S) err += 0.01f;
    else err = -1;
    rec_out[0] = fa; rec_out[1] = fb; rec_out[2] = mu; rec_out[3] = sigma;
    rec_out[5] = thr[0]; rec_out[6] = thr[S - 1];
    if (err < 0 || (double) err > S - 1e-3) {
        const float first = orc_cdf_phi((thr[0] - mu) / sigma);
        const float last = orc_cdf_phi((thr[S - 1] - mu) / sigma);
        const float av = (float) (2.0f - (float) S) / (first - last);
        const float bv = ((float) S * first - last) / (first - last);
        rec_out[0] = av; rec_out[1] = bv;
        err = -1;
        for (int j = 0; j < S - 1; j++) {
            const float cdf = orc_cdf_phi((thr[j] - mu) / sigma);
            const float ncdf = orc_cdf_phi((thr[j + 1] - mu) / sigma);
            const float p1 = cdf * av + bv, p2 = ncdf * av + bv;
            const float e1 = fabsf((float) (j + 1) - p1), e2 = fabsf((float) (j + 1) - p2);
            const float te = (e1 > e2 ? e1 : e2) + 0.01f;
            err = te > err ? te : err;
        }
        err = err < (float) S ? err : (float) S;
        err += 0.01f;
    }
    rec_out[4] = err;
}

void orc_fit_regression(const float *thr, int64_t n_user, int32_t S, float *rec_out /* [n_user][7] */) {
    for (int64_t u = 0; u < n_user; u++) orc_fit_regression_user(thr + u * S, S, rec_out + u * 7);
}

/* ------------------------------------------------------------------------------------------ */
/* query                                                                                       */
/* ------------------------------------------------------------------------------------------ */

/* SampleSearch::CoarseBinarySearch, src/include/alg/RankBoundRefinement/SampleSearch.hpp:91-130. */
void orc_sample_search_bound(const float *thr_row, int32_t S, const int32_t *sample_rank, int64_t n_item,
                             float qip, int32_t *rank_lb, int32_t *rank_ub) {
    int64_t lo = 0, len = S; /* std::lower_bound with comp(arr, q) = arr >= q */
    while (len > 0) {
        int64_t h = len >> 1, m = lo + h;
        if (thr_row[m] >= qip) { lo = m + 1; len -= h + 1; } else len = h;
    }
    const unsigned b = (unsigned) lo;
    const unsigned tlb = b == (unsigned) S ? (unsigned) n_item : (unsigned) sample_rank[b];
    const unsigned tub = b == 0 ? 0u : (unsigned) sample_rank[b - 1];
    if (b == (unsigned) S) { *rank_lb = (int32_t) n_item; *rank_ub = (int32_t) tub; }
    else if (b == 0) { *rank_lb = (int32_t) tlb; *rank_ub = 0; }
    else if (tlb - tub <= 1) { *rank_lb = (int32_t) tlb; *rank_ub = (int32_t) tlb; }
    else { *rank_lb = (int32_t) tlb; *rank_ub = (int32_t) tub; }
}

/* k-th smallest by the reference's size-k max-heap scan (PruneCandidateByBound.hpp:36-77): the
 * heap starts zero-filled, so with fewer than k eligible values the result is max(values, 0). */
static int32_t kth_smallest_heap(const int32_t *v, const char *skip, int64_t n, int k) {
    int32_t *buf = (int32_t *) malloc(sizeof(int32_t) * (size_t) n);
    int64_t m = 0;
    for (int64_t i = 0; i < n; i++) if (!skip[i]) buf[m++] = v[i];
    int32_t res;
    if (m < k) {
        res = 0;
        for (int64_t i = 0; i < m; i++) if (buf[i] > res) res = buf[i];
    } else {
        qsort(buf, (size_t) m, sizeof(int32_t), cmp_i32);
        res = buf[k - 1];
    }
    free(buf);
    return res;
}

/* ---- user shards ---------------------------------------------------------------------------- */

/* A user shard: this call holds users [user_offset, user_offset + n_user) of all shards' users, and
 * exchange(ctx, counts, n, NULL) sums n int32 host counts over all shards in place (the engine's
 * rkr_exchange_fn, include/rkr.h).  first: this shard counts the refinement-independent part of
 * ip_cost.  NULL everywhere below: one whole index. */
typedef int (*orc_exchange_fn)(void *ctx, int32_t *counts, int64_t n, void *stream);
typedef struct {
    orc_exchange_fn exchange;
    void *ctx;
    int64_t user_offset, n_user_total;
    int first;
    int failed;
} orc_shard;

static void shard_sum(orc_shard *sh, int32_t *v, int64_t n) {
    if (sh && sh->exchange(sh->ctx, v, n, NULL) != 0) sh->failed = 1;
}

/* The k-th smallest of the eligible values of every shard by the heap rule of kth_smallest_heap,
 * from the per-value counts summed over the shards (rank bounds lie in [0, n_item]). */
static int32_t kth_smallest_shard(const int32_t *v, const char *skip, int64_t n, int k, int64_t n_item,
                                  orc_shard *sh) {
    int32_t *h = (int32_t *) calloc((size_t) n_item + 1, sizeof(int32_t));
    for (int64_t i = 0; i < n; i++)
        if (!skip[i]) {
            if (v[i] < 0 || v[i] > n_item) sh->failed = 1;
            else h[v[i]]++;
        }
    shard_sum(sh, h, n_item + 1);
    int64_t total = 0;
    for (int64_t r = 0; r <= n_item; r++) total += h[r];
    int32_t res = 0;
    if (total < k) {
        for (int64_t r = n_item; r >= 0; r--) if (h[r]) { res = (int32_t) r; break; }
    } else {
        int64_t cum = 0;
        for (int64_t r = 0; r <= n_item; r++) { cum += h[r]; if (cum >= k) { res = (int32_t) r; break; } }
    }
    free(h);
    return res;
}

/* PruneCandidateByBound, src/include/alg/RankBoundRefinement/PruneCandidateByBound.hpp:19-153.
 * Sharded (sh != NULL): the k-th smallest bounds and the class counts are every shard's (summed
 * counts), the classes are set on this shard's users. */
static void prune_sh(const int32_t *rank_lb, const int32_t *rank_ub, int64_t n_user, int32_t topk, int64_t n_item,
                     int32_t *refine_user_size, int32_t *n_result_user, int32_t *n_prune_user, char *prune,
                     char *result, orc_shard *sh) {
    if (*n_result_user >= topk) return;
    const int heap_size = topk - *n_result_user;
    char *skip = (char *) malloc((size_t) n_user);
    for (int64_t u = 0; u < n_user; u++) skip[u] = prune[u] || result[u];
    const int32_t L = sh ? kth_smallest_shard(rank_lb, skip, n_user, heap_size, n_item, sh)
                         : kth_smallest_heap(rank_lb, skip, n_user, heap_size);
    const int32_t U = sh ? kth_smallest_shard(rank_ub, skip, n_user, heap_size, n_item, sh)
                         : kth_smallest_heap(rank_ub, skip, n_user, heap_size);
    free(skip);
    if (L == U) {
        *n_result_user = topk;
        *refine_user_size = 0;
        for (int64_t u = 0; u < n_user; u++)
            if (rank_ub[u] <= L && rank_lb[u] <= L) result[u] = 1;
        return;
    }
    int32_t refine = 0, nres = 0, npr = 0;
    for (int64_t u = 0; u < n_user; u++) {
        if (prune[u] || result[u]) continue;
        if (rank_lb[u] <= U) { result[u] = 1; nres++; }
        else if (L <= rank_ub[u]) { prune[u] = 1; npr++; }
        else refine++;
    }
    if (sh) {
        int32_t c[3] = {nres, npr, refine};
        shard_sum(sh, c, 3);
        nres = c[0]; npr = c[1]; refine = c[2];
    }
    nres += *n_result_user;
    npr += *n_prune_user;
    *n_result_user = nres; *n_prune_user = npr; *refine_user_size = refine;
    if (nres + refine == topk) {
        for (int64_t u = 0; u < n_user; u++) if (!prune[u] && !result[u]) result[u] = 1;
        *refine_user_size = 0;
        *n_result_user = topk;
    }
}

void orc_prune_candidate_by_bound(const int32_t *rank_lb, const int32_t *rank_ub, int64_t n_user, int32_t topk,
                                  int32_t *refine_user_size, int32_t *n_result_user, int32_t *n_prune_user,
                                  char *prune, char *result) {
    prune_sh(rank_lb, rank_ub, n_user, topk, 0, refine_user_size, n_result_user, n_prune_user, prune, result, NULL);
}

/* ---- refinement ----------------------------------------------------------------------------- */

typedef struct { int32_t user_id, rank; float query_ip; } orc_user_rank;

/* Refinement structure of RefineCPUIPBound (src/include/alg/DiskIndex/RefineByComputation/
 * RefineCPUIPBound.hpp:417-467): items sorted by norm descending, with the norm of their last
 * d - check_dim coordinates (RefineCPUPartDimPartNorm.hpp:39-54). */
typedef struct {
    int64_t n_user, n_item; int d, check_dim;
    const float *user;
    float *item_sorted;  /* [n_item][d] */
    float *item_norm;    /* [n_item] descending */
    float *item_rnorm;   /* [n_item] norm of coordinates [check_dim, d) */
    float *user_rnorm;   /* [n_user] */
} refine_t;

typedef struct { float norm; int32_t id; } norm_id;
static int cmp_norm_desc(const void *a, const void *b) {
    const norm_id *x = (const norm_id *) a, *y = (const norm_id *) b;
    if (x->norm != y->norm) return (x->norm < y->norm) - (x->norm > y->norm);
    return (x->id > y->id) - (x->id < y->id);
}

static void refine_init(refine_t *r, const float *user, int64_t n_user, const float *item, int64_t n_item,
                        int d, int check_dim) {
    r->n_user = n_user; r->n_item = n_item; r->d = d; r->check_dim = check_dim; r->user = user;
    norm_id *ni = (norm_id *) malloc(sizeof(norm_id) * (size_t) n_item);
    for (int64_t i = 0; i < n_item; i++) { ni[i].norm = sqrtf(ip_f32(item + i * d, item + i * d, d)); ni[i].id = (int32_t) i; }
    qsort(ni, (size_t) n_item, sizeof(norm_id), cmp_norm_desc);
    r->item_sorted = (float *) malloc(sizeof(float) * (size_t) (n_item * d));
    r->item_norm = (float *) malloc(sizeof(float) * (size_t) n_item);
    r->item_rnorm = (float *) malloc(sizeof(float) * (size_t) n_item);
    r->user_rnorm = (float *) malloc(sizeof(float) * (size_t) n_user);
    const int rd = d - check_dim;
    for (int64_t i = 0; i < n_item; i++) {
        memcpy(r->item_sorted + i * d, item + (int64_t) ni[i].id * d, sizeof(float) * (size_t) d);
        r->item_norm[i] = ni[i].norm;
        const float *v = r->item_sorted + i * d + check_dim;
        r->item_rnorm[i] = sqrtf(ip_f32(v, v, rd));
    }
    for (int64_t u = 0; u < n_user; u++) {
        const float *v = user + u * d + check_dim;
        r->user_rnorm[u] = sqrtf(ip_f32(v, v, rd));
    }
    free(ni);
}
static void refine_free(refine_t *r) {
    free(r->item_sorted); free(r->item_norm); free(r->item_rnorm); free(r->user_rnorm);
}

/* RefineCPUIPBound::RefineRank, RefineCPUIPBound.hpp:93-150 (with RefineCPUPartDimPartNorm's
 * IPBoundNoParallel :83-107 and ComputeRemainDimNoParallel :131-152). */
static int32_t refine_rank_ipbound(const refine_t *r, float qip, int64_t uid, int64_t *n_compute_item,
                                   int64_t *ip_cost) {
    const float lowq = qip - 8e-3f, highq = qip + 8e-3f;
    int64_t lo = 0, len = r->n_item; /* lower_bound(norms, lowq, arr > q) */
    while (len > 0) { int64_t h = len >> 1, m = lo + h; if (r->item_norm[m] > lowq) { lo = m + 1; len -= h + 1; } else len = h; }
    const int64_t n_proc = lo;
    if (n_compute_item) *n_compute_item = n_proc;
    const int c = r->check_dim, d = r->d;
    const float *uv = r->user + uid * d;
    const float unorm = r->user_rnorm[uid];
    int32_t rank = 0;
    int64_t cost = (int) (n_proc * 1.0 * (c + 1) / (int) d);  /* RefineCPUIPBound.hpp:491 */
    for (int64_t i = 0; i < n_proc; i++) {
        const float *iv = r->item_sorted + i * d;
        const float left = ip_f32(uv, iv, c);
        const float right = r->item_rnorm[i] * unorm;
        const float lbv = left - right, ubv = left + right;
        if (lowq > ubv) continue;
        if (highq < lbv) { rank++; continue; }
        const float ip = left + ip_f32(uv + c, iv + c, d - c);
        cost++;  /* RefineCPUIPBound.hpp:518 */
        if (ip >= qip) rank++;
    }
    if (ip_cost) *ip_cost = cost;
    return rank;
}

/* RefineCPU::RefineRank, src/include/alg/DiskIndex/RefineByComputation/RefineCPU.hpp:33-55:
 * number of items scoring strictly above the query score (full-dimension dot product). */
static int32_t refine_rank_all(const float *uv, const float *item, int64_t n_item, int d, float qip) {
    int32_t rank = 0;
    for (int64_t i = 0; i < n_item; i++) if (ip_f32(uv, item + i * d, d) > qip) rank++;
    return rank;
}

static int cmp_user_rank(const void *a, const void *b) { /* UserRankElement::operator<, :257-262 */
    const orc_user_rank *x = (const orc_user_rank *) a, *y = (const orc_user_rank *) b;
    if (x->rank != y->rank) return (x->rank > y->rank) - (x->rank < y->rank);
    return (x->user_id > y->user_id) - (x->user_id < y->user_id);
}

typedef struct { int32_t n_prune, n_result, n_refine, n_candidate; int64_t n_compute_item, ip_cost; } orc_query_stats;

/* ComputeAllIPBound::GetRank (ComputeAllIPBound.hpp:57-137) and ComputeAll::GetRank
 * (ComputeAll.hpp:54-125), then the result assembly of QS.hpp:185-198 / QSRPNormalLP.hpp:213-226 /
 * US.hpp result loop.  cache is the reference's persistent user_topk_cache_l_ ([n_user]). */
static void refine_and_assemble(const refine_t *rf, int use_ipbound, const float *item, const float *qip,
                                const int32_t *lb, const int32_t *ub, const char *prune, const char *result,
                                int64_t n_user, int32_t topk, int32_t n_result, orc_user_rank *cache,
                                orc_user_rank *out, orc_query_stats *st, const orc_shard *sh, int32_t *n_front) {
    const int32_t n_remain = topk - n_result > 0 ? topk - n_result : 0;
    int32_t n_refine = 0, n_cand = 0;
    int64_t n_compute = 0, refine_ip_cost = 0;
    if (n_remain != 0) {
        for (int64_t u = 0; u < n_user; u++) {
            if (prune[u] || result[u]) continue;
            int32_t rank;
            if (lb[u] == ub[u]) rank = lb[u];
            else {
                n_refine++;
                if (use_ipbound) {
                    int64_t nc = 0, ic = 0;
                    rank = refine_rank_ipbound(rf, qip[u], u, &nc, &ic);
                    n_compute += nc;
                    refine_ip_cost += ic;
                } else {
                    rank = refine_rank_all(rf->user + u * rf->d, item, rf->n_item, rf->d, qip[u]);
                    n_compute += rf->n_item;
                    refine_ip_cost += rf->n_item;  /* ComputeAll.hpp:112-116 */
                }
            }
            cache[n_cand].user_id = (int32_t) u; cache[n_cand].rank = rank; cache[n_cand].query_ip = qip[u];
            n_cand++;
        }
        qsort(cache, (size_t) n_cand, sizeof(orc_user_rank), cmp_user_rank);
    }
    int nc = 0;
    for (int64_t u = 0; u < n_user; u++) {
        if (result[u]) { out[nc].user_id = (int32_t) u; out[nc].rank = lb[u]; out[nc].query_ip = qip[u]; nc++; }
        if (nc == topk) break;
    }
    if (!sh) {
        for (int c = nc; c < topk; c++) out[c] = cache[c - nc];
    } else {
        /* a shard's part: its results, then its candidates in order, then unused entries */
        const int64_t off = sh->user_offset;
        *n_front = nc;
        for (int c = 0; c < nc; c++) out[c].user_id += (int32_t) off;
        for (int c = nc; c < topk; c++) {
            if (n_remain != 0 && c - nc < n_cand) {
                out[c] = cache[c - nc];
                out[c].user_id += (int32_t) off;
            } else {
                out[c].user_id = -1; out[c].rank = -1; out[c].query_ip = -1.0f;
            }
        }
    }
    if (st) { st->n_refine = n_refine; st->n_candidate = n_cand; st->n_compute_item = n_compute; st->ip_cost = refine_ip_cost; }
}

/* QS::Index::Retrieval, src/impl/QS.hpp:106-230.
 * user: normalised users [n_user][d]; item: data items [n_item][d]; thr: [n_user][S].
 * out: [n_query][topk]; st: [n_query] or NULL.  Returns 0, or -1 on the reference's error exits. */
static int qs_impl(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                   int32_t check_dim, const int32_t *sample_rank, int32_t S, const float *thr,
                   const float *query, int32_t n_query, int32_t topk, orc_user_rank *out,
                   orc_query_stats *st, orc_shard *sh, int32_t *n_front) {
    if (!sh && topk > n_user) return -1;
    refine_t rf; refine_init(&rf, user, n_user, item, n_item, d, check_dim);
    float *qip = (float *) calloc((size_t) n_user, sizeof(float));
    int32_t *lb = (int32_t *) calloc((size_t) n_user, sizeof(int32_t));
    int32_t *ub = (int32_t *) calloc((size_t) n_user, sizeof(int32_t));
    char *prune = (char *) malloc((size_t) n_user), *result = (char *) malloc((size_t) n_user);
    orc_user_rank *cache = (orc_user_rank *) calloc((size_t) n_user, sizeof(orc_user_rank));
    for (int64_t u = 0; u < n_user; u++) { cache[u].user_id = -1; cache[u].rank = -1; cache[u].query_ip = -1; }
    for (int q = 0; q < n_query; q++) {
        memset(prune, 0, (size_t) n_user); memset(result, 0, (size_t) n_user);
        const float *qv = query + (int64_t) q * d;
        for (int64_t u = 0; u < n_user; u++) qip[u] = ip_f32(qv, user + u * d, d);
        for (int64_t u = 0; u < n_user; u++)
            orc_sample_search_bound(thr + u * S, S, sample_rank, n_item, qip[u], lb + u, ub + u);
        int32_t refine_size = (int32_t) n_user, n_result = 0, n_prune = 0;
        prune_sh(lb, ub, n_user, topk, n_item, &refine_size, &n_result, &n_prune, prune, result, sh);
        orc_query_stats s = {0};
        refine_and_assemble(&rf, 1, item, qip, lb, ub, prune, result, n_user, topk, n_result, cache,
                            out + (int64_t) q * topk, &s, sh, sh ? n_front + q : NULL);
        s.n_prune = n_prune; s.n_result = n_result;
        if (!sh) s.ip_cost += n_user;  /* QS.hpp:146, 221 */
        else if (sh->first) s.ip_cost += sh->n_user_total;
        if (st) st[q] = s;
    }
    free(qip); free(lb); free(ub); free(prune); free(result); free(cache);
    refine_free(&rf);
    return 0;
}

/* US::Index::Retrieval, src/impl/US.hpp:96-213 (the reference answers only the first 100 queries
 * when n_sample <= 1000, US.hpp:113).  Returns the number of queries answered, or -1. */
static int us_impl(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                   const int32_t *sample_rank, int32_t S, const float *thr,
                   const float *query, int32_t n_query, int32_t topk, orc_user_rank *out,
                   orc_query_stats *st, orc_shard *sh, int32_t *n_front) {
    if (!sh && topk > n_user) return -1;
    const int32_t nq = S <= 1000 ? 100 : n_query;
    if (nq > n_query) return -1;
    refine_t rf; memset(&rf, 0, sizeof(rf));
    rf.user = user; rf.n_user = n_user; rf.n_item = n_item; rf.d = d;
    float *qip = (float *) calloc((size_t) n_user, sizeof(float));
    int32_t *lb = (int32_t *) calloc((size_t) n_user, sizeof(int32_t));
    int32_t *ub = (int32_t *) calloc((size_t) n_user, sizeof(int32_t));
    char *prune = (char *) malloc((size_t) n_user), *result = (char *) malloc((size_t) n_user);
    orc_user_rank *cache = (orc_user_rank *) calloc((size_t) n_user, sizeof(orc_user_rank));
    for (int q = 0; q < nq; q++) {
        memset(prune, 0, (size_t) n_user); memset(result, 0, (size_t) n_user);
        const float *qv = query + (int64_t) q * d;
        for (int64_t u = 0; u < n_user; u++) qip[u] = ip_f32(qv, user + u * d, d);
        for (int64_t u = 0; u < n_user; u++)
            orc_sample_search_bound(thr + u * S, S, sample_rank, n_item, qip[u], lb + u, ub + u);
        int32_t refine_size = (int32_t) n_user, n_result = 0, n_prune = 0;
        prune_sh(lb, ub, n_user, topk, n_item, &refine_size, &n_result, &n_prune, prune, result, sh);
        orc_query_stats s = {0};
        refine_and_assemble(&rf, 0, item, qip, lb, ub, prune, result, n_user, topk, n_result, cache,
                            out + (int64_t) q * topk, &s, sh, sh ? n_front + q : NULL);
        s.n_prune = n_prune; s.n_result = n_result;
        if (!sh) s.ip_cost += n_user;  /* US.hpp:134, 188 */
        else if (sh->first) s.ip_cost += sh->n_user_total;
        if (st) st[q] = s;
    }
    free(qip); free(lb); free(ub); free(prune); free(result); free(cache);
    return nq;
}

/* QSRPNormalLP::Index::Retrieval, src/impl/QSRPNormalLP.hpp:116-260.
 * svd_user: SVD-space users [n_user][d] (SVD.hpp transfer_user_); transfer_item: [d][d];
 * reg: [n_user][7] model records (a, b, mu, sigma, err, smax, smin); reg_rank: the model's
 * sample ranks [S_reg].  qip_state: the index's persistent per-user query score vector
 * ([n_user], zero on a fresh index); users accepted by the first (regression) bound are reported
 * with whatever value it holds, as in the reference. */
static int qsrp_impl(const float *user, const float *svd_user, const float *transfer_item, int64_t n_user,
                     const float *item, int64_t n_item, int32_t d, int32_t check_dim,
                     const int32_t *sample_rank, int32_t S, const float *thr,
                     const int32_t *reg_rank, int32_t S_reg, const float *reg,
                     const float *query, int32_t n_query, int32_t topk,
                     float *qip_state, orc_user_rank *out, orc_query_stats *st, orc_shard *sh, int32_t *n_front) {
    if (!sh && topk > n_user) return -1;
    const int c = check_dim, rd = d - check_dim;
    refine_t rf; refine_init(&rf, user, n_user, item, n_item, d, check_dim);
    float *unorm = (float *) malloc(sizeof(float) * (size_t) n_user);      /* PartDimPartNorm::Preprocess :41-50 */
    for (int64_t u = 0; u < n_user; u++) { const float *v = svd_user + u * d + c; unorm[u] = sqrtf(ip_f32(v, v, rd)); }
    float *left = (float *) malloc(sizeof(float) * (size_t) n_user);
    float *qtr = (float *) malloc(sizeof(float) * (size_t) d);
    int32_t *lb = (int32_t *) calloc((size_t) n_user, sizeof(int32_t));
    int32_t *ub = (int32_t *) calloc((size_t) n_user, sizeof(int32_t));
    char *prune = (char *) malloc((size_t) n_user), *result = (char *) malloc((size_t) n_user);
    orc_user_rank *cache = (orc_user_rank *) calloc((size_t) n_user, sizeof(orc_user_rank));
    for (int64_t u = 0; u < n_user; u++) { cache[u].user_id = -1; cache[u].rank = -1; cache[u].query_ip = -1; }
    for (int q = 0; q < n_query; q++) {
        memset(prune, 0, (size_t) n_user); memset(result, 0, (size_t) n_user);
        const float *qv = query + (int64_t) q * d;
        for (int t = 0; t < d; t++) qtr[t] = ip_f32(transfer_item + (int64_t) t * d, qv, d); /* SVD.hpp:156-164 */
        const float qnorm = sqrtf(ip_f32(qtr + c, qtr + c, rd));                           /* PartDimPartNorm.hpp:56-57 */
        for (int64_t u = 0; u < n_user; u++) {
            const float l = ip_f32(svd_user + u * d, qtr, c);
            left[u] = l;
            const float right = unorm[u] * qnorm;
            const float qlb = l - right, qub = l + right;
            orc_regression_rank_bound(qlb, qub, reg + u * 7, reg + u * 7 + 2, reg[u * 7 + 4], reg + u * 7 + 5,
                                      reg_rank, S_reg, n_item, lb + u, ub + u);
        }
        int32_t refine_size = (int32_t) n_user, n_result = 0, n_prune = 0;
        prune_sh(lb, ub, n_user, topk, n_item, &refine_size, &n_result, &n_prune, prune, result, sh);
        const int32_t ip_cost = refine_size;                                                 /* QSRPNormalLP.hpp:177 */
        for (int64_t u = 0; u < n_user; u++) {                                               /* ComputeRemainDim :76-95 */
            if (prune[u] || result[u]) continue;
            qip_state[u] = left[u] + ip_f32(svd_user + u * d + c, qtr + c, rd);
        }
        for (int64_t u = 0; u < n_user; u++) {
            if (prune[u] || result[u]) continue;
            orc_sample_search_bound(thr + u * S, S, sample_rank, n_item, qip_state[u], lb + u, ub + u);
        }
        prune_sh(lb, ub, n_user, topk, n_item, &refine_size, &n_result, &n_prune, prune, result, sh);
        orc_query_stats s = {0};
        refine_and_assemble(&rf, 1, item, qip_state, lb, ub, prune, result, n_user, topk, n_result, cache,
                            out + (int64_t) q * topk, &s, sh, sh ? n_front + q : NULL);
        s.n_prune = n_prune; s.n_result = n_result;
        if (!sh || sh->first) s.ip_cost += ip_cost;
        if (st) st[q] = s;
    }
    free(unorm); free(left); free(qtr); free(lb); free(ub); free(prune); free(result); free(cache);
    refine_free(&rf);
    return 0;
}

int orc_qs_retrieval(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                     int32_t check_dim, const int32_t *sample_rank, int32_t S, const float *thr,
                     const float *query, int32_t n_query, int32_t topk, orc_user_rank *out,
                     orc_query_stats *st) {
    return qs_impl(user, n_user, item, n_item, d, check_dim, sample_rank, S, thr, query, n_query, topk, out, st,
                   NULL, NULL);
}

int orc_us_retrieval(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                     const int32_t *sample_rank, int32_t S, const float *thr,
                     const float *query, int32_t n_query, int32_t topk, orc_user_rank *out,
                     orc_query_stats *st) {
    return us_impl(user, n_user, item, n_item, d, sample_rank, S, thr, query, n_query, topk, out, st, NULL, NULL);
}

int orc_qsrp_retrieval(const float *user, const float *svd_user, const float *transfer_item, int64_t n_user,
                       const float *item, int64_t n_item, int32_t d, int32_t check_dim,
                       const int32_t *sample_rank, int32_t S, const float *thr,
                       const int32_t *reg_rank, int32_t S_reg, const float *reg,
                       const float *query, int32_t n_query, int32_t topk,
                       float *qip_state, orc_user_rank *out, orc_query_stats *st) {
    return qsrp_impl(user, svd_user, transfer_item, n_user, item, n_item, d, check_dim, sample_rank, S, thr, reg_rank,
                     S_reg, reg, query, n_query, topk, qip_state, out, st, NULL, NULL);
}

/* The same three methods on one user shard holding users [user_offset, user_offset + n_user) of
 * n_user_total (first: shard 0): every argument is the shard's (its users' rows of user / svd_user / thr /
 * reg / qip_state), exchange sums counts over the shards (every shard calls with the same queries and
 * topk).  out[q] is the shard's part of row q as rkr_shard_query returns it (n_front[q] results by
 * user id, then its candidates by (rank, user id), unused entries user_id -1); stats carry the global
 * n_prune / n_result and the shard's share of the rest.  Returns the queries answered, or -1 when
 * the exchange failed or a bound lay outside [0, n_item]. */
int orc_qs_retrieval_shard(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                           int32_t check_dim, const int32_t *sample_rank, int32_t S, const float *thr,
                           const float *query, int32_t n_query, int32_t topk, int64_t user_offset,
                           int64_t n_user_total, int32_t first, orc_exchange_fn exchange, void *ctx,
                           orc_user_rank *out, int32_t *n_front, orc_query_stats *st) {
    orc_shard sh = {exchange, ctx, user_offset, n_user_total, first, 0};
    const int rc = qs_impl(user, n_user, item, n_item, d, check_dim, sample_rank, S, thr, query, n_query, topk, out,
                           st, &sh, n_front);
    return sh.failed ? -1 : (rc < 0 ? rc : n_query);
}

int orc_us_retrieval_shard(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                           const int32_t *sample_rank, int32_t S, const float *thr,
                           const float *query, int32_t n_query, int32_t topk, int64_t user_offset,
                           int64_t n_user_total, int32_t first, orc_exchange_fn exchange, void *ctx,
                           orc_user_rank *out, int32_t *n_front, orc_query_stats *st) {
    orc_shard sh = {exchange, ctx, user_offset, n_user_total, first, 0};
    const int rc = us_impl(user, n_user, item, n_item, d, sample_rank, S, thr, query, n_query, topk, out, st, &sh,
                           n_front);
    return sh.failed ? -1 : rc;
}

int orc_qsrp_retrieval_shard(const float *user, const float *svd_user, const float *transfer_item, int64_t n_user,
                             const float *item, int64_t n_item, int32_t d, int32_t check_dim,
                             const int32_t *sample_rank, int32_t S, const float *thr,
                             const int32_t *reg_rank, int32_t S_reg, const float *reg,
                             const float *query, int32_t n_query, int32_t topk, int64_t user_offset,
                             int64_t n_user_total, int32_t first, orc_exchange_fn exchange, void *ctx,
                             float *qip_state, orc_user_rank *out, int32_t *n_front, orc_query_stats *st) {
    orc_shard sh = {exchange, ctx, user_offset, n_user_total, first, 0};
    const int rc = qsrp_impl(user, svd_user, transfer_item, n_user, item, n_item, d, check_dim, sample_rank, S, thr,
                             reg_rank, S_reg, reg, query, n_query, topk, qip_state, out, st, &sh, n_front);
    return sh.failed ? -1 : (rc < 0 ? rc : n_query);
}

/* ------------------------------------------------------------------------------------------ */
/* FP64 ground truth (not the reference's arithmetic; used to report score error)              */
/* ------------------------------------------------------------------------------------------ */

/* rank64[q][u] = #{ i : <u,i> >= <u,q> } with every dot product evaluated in double. */
void orc_exact_rank_f64(const float *user, int64_t n_user, const float *item, int64_t n_item, int32_t d,
                        const float *query, int32_t n_query, int32_t *rank_out) {
    for (int q = 0; q < n_query; q++) {
        const float *qv = query + (int64_t) q * d;
        for (int64_t u = 0; u < n_user; u++) {
            const float *uv = user + u * d;
            double s = 0;
            for (int j = 0; j < d; j++) s += (double) uv[j] * (double) qv[j];
            int32_t r = 0;
            for (int64_t i = 0; i < n_item; i++) {
                const float *iv = item + i * d;
                double t = 0;
                for (int j = 0; j < d; j++) t += (double) uv[j] * (double) iv[j];
                if (t >= s) r++;
            }
            rank_out[(int64_t) q * n_user + u] = r;
        }
    }
}
