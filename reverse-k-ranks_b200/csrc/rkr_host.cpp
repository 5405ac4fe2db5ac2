// rkr_host.cpp -- host-side index-build steps of librkr_b200 (CPU, OpenMP).
//
// These steps are small next to the score passes that run on the device: choosing the sampled
// items and sample ranks, fitting one straight line per user, and the SVD transform.  Float
// arithmetic here follows the reference's expressions operation by operation (this file is compiled
// with -ffp-contract=off), so the models it fits are the models the reference would fit.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <set>
#include <vector>

#include "rkr.h"
#include "rkr_svd_host.h"

namespace rkr {
void set_error(const char *fmt, ...);
}

namespace {

float dot_f32(const float *a, const float *b, int n) {
    float r = 0.0f;
    for (int i = 0; i < n; i++) r += a[i] * b[i];
    return r;
}

// NormalLinearRegressionLP::CDFPhi (NormalLinearRegressionLP.hpp:123-143): float constants and
// polynomial, t and the closing expression in double, the double ::exp; sqrt_2_ is the binary32
// value of ReverseMIPS::sqrt(2.0) (MathUtil.hpp:10-27), i.e. the float nearest sqrt(2).
float cdf_phi(float x) {
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f;
    const float a4 = -1.453152027f, a5 = 1.061405429f, p = 0.3275911f;
    const float sqrt_2 = 1.41421354f;
    int sign = 1;
    if (x < 0) sign = -1;
    x = std::fabs(x) / sqrt_2;
    const float t = (float) (1.0 / (1.0 + (double) (p * x)));
    const float pt = (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t;
    const float y = (float) (1.0 - (double) pt * ::exp((double) (-x * x)));
    return (float) (0.5 * (1.0 + (double) ((float) sign * y)));
}

// Minimax straight line through (x_i, y_i): minimise e = max |a x_i + b - y_i|, the optimum of
// the LP in NormalLinearRegressionLP::LinearProgram (:181-213).  Points arrive sorted by (x, y)
// ascending.  The optimal strip's direction is that of a convex-hull edge; each hull-edge slope s is
// tried and the narrowest vertical strip kept.  The strip's top, max (y - s x), lies on the upper
// hull, whose edge slopes fall along it, at the vertex where they cross s; its bottom, min (y - s x),
// on the lower hull (rising slopes) likewise: both are found by binary search, and the vertices
// around the crossing are evaluated so that rounding in the slopes cannot miss the extreme.  Double
// precision.
void minimax_fit(const std::vector<double> &xs, const std::vector<double> &ys, double &a, double &b, double &e) {
    const size_t n = xs.size();
    std::vector<size_t> lo, up;
    auto cross = [&](size_t o, size_t p, size_t q) {
        return (xs[p] - xs[o]) * (ys[q] - ys[o]) - (ys[p] - ys[o]) * (xs[q] - xs[o]);
    };
    lo.reserve(n);
    up.reserve(n);
    // the lower hull takes the lowest point at each x, the upper hull the highest: the others can only
    // sit on a vertical end edge, whose slope is never a candidate and whose top (bottom) point the
    // other one dominates
    for (size_t i = 0; i < n; i++) {
        if (i == 0 || xs[i] != xs[i - 1]) {
            while (lo.size() >= 2 && cross(lo[lo.size() - 2], lo.back(), i) <= 0) lo.pop_back();
            lo.push_back(i);
        }
        if (i + 1 == n || xs[i + 1] != xs[i]) {
            while (up.size() >= 2 && cross(up[up.size() - 2], up.back(), i) >= 0) up.pop_back();
            up.push_back(i);
        }
    }
    const double inf = std::numeric_limits<double>::infinity();
    // edge slopes (a vertical edge: +inf; only at the upper hull's start or the lower hull's end)
    auto slopes = [&](const std::vector<size_t> &h) {
        std::vector<double> sl(h.size() > 1 ? h.size() - 1 : 0);
        for (size_t k = 0; k + 1 < h.size(); k++) {
            const double dx = xs[h[k + 1]] - xs[h[k]];
            sl[k] = dx != 0 ? (ys[h[k + 1]] - ys[h[k]]) / dx : inf;
        }
        return sl;
    };
    const std::vector<double> s_up = slopes(up), s_lo = slopes(lo);
    constexpr size_t kWin = 3;
    auto top = [&](double s) {  // max (y - s x) over the upper hull
        const size_t k = std::partition_point(s_up.begin(), s_up.end(), [&](double v) { return v > s; }) - s_up.begin();
        double m = -inf;
        for (size_t j = k > kWin ? k - kWin : 0; j < std::min(up.size(), k + kWin + 1); j++)
            m = std::max(m, ys[up[j]] - s * xs[up[j]]);
        return m;
    };
    auto bottom = [&](double s) {  // min (y - s x) over the lower hull
        const size_t k = std::partition_point(s_lo.begin(), s_lo.end(), [&](double v) { return v < s; }) - s_lo.begin();
        double m = inf;
        for (size_t j = k > kWin ? k - kWin : 0; j < std::min(lo.size(), k + kWin + 1); j++)
            m = std::min(m, ys[lo[j]] - s * xs[lo[j]]);
        return m;
    };
    double best = inf, ba = 0, bb = 0;
    for (const auto *h : {&lo, &up})
        for (size_t k = 0; k + 1 < h->size(); k++) {
            const double dx = xs[(*h)[k + 1]] - xs[(*h)[k]];
            if (dx == 0) continue;
            const double s = (ys[(*h)[k + 1]] - ys[(*h)[k]]) / dx;
            const double mx = top(s), mn = bottom(s);
            const double w = 0.5 * (mx - mn);
            if (w < best) { best = w; ba = s; bb = 0.5 * (mx + mn); }
        }
    if (!(best < inf)) {
        double mx = -inf, mn = inf;
        for (size_t i = 0; i < n; i++) { mx = std::max(mx, ys[i]); mn = std::min(mn, ys[i]); }
        ba = 0;
        bb = n ? 0.5 * (mx + mn) : 0;
        best = n ? 0.5 * (mx - mn) : 0;
    }
    a = ba;
    b = bb;
    e = best;
}

// One user's model from its descending thresholds (AssignCache :145-179, the LinearProgram
// post-processing :194-211, and the endpoint-line fallback with CalcError :215-243, 272-296).
void fit_user(const float *thr, int S, float *rec) {
    float mu = 0.0f;
    for (int s = 0; s < S; s++) mu += thr[s];
    mu = mu / (float) S;
    float sigma = 0.0f;
    for (int s = 0; s < S; s++) {
        const float m = thr[s] - mu;
        const float t = m * m;
        sigma += t;
    }
    sigma /= (float) S;
    sigma = std::sqrt(sigma);
    std::vector<float> cdf(S);
    for (int s = 0; s < S; s++) cdf[s] = cdf_phi((thr[s] - mu) / sigma);
    // points (cdf_j, j + 1) and (cdf_{j+1}, j + 1), j = 0 .. S-2; cdf is non-increasing in j, so
    // walking j backwards gives ascending x.
    std::vector<double> xs, ys;
    xs.reserve(2 * S);
    ys.reserve(2 * S);
    for (int j = S - 2; j >= 0; j--) {
        xs.push_back(cdf[j + 1]); ys.push_back(j + 1);
        xs.push_back(cdf[j]); ys.push_back(j + 1);
    }
    // ascending (x, y) order: a stable insertion sort, linear here since the walk above leaves only
    // adjacent equal-x pairs out of order (the same order a stable sort of any input gives)
    std::vector<double> &sx = xs, &sy = ys;
    for (size_t i = 1; i < sx.size(); i++) {
        const double x = sx[i], y = sy[i];
        size_t k = i;
        while (k > 0 && (x < sx[k - 1] || (x == sx[k - 1] && y < sy[k - 1]))) {
            sx[k] = sx[k - 1];
            sy[k] = sy[k - 1];
            k--;
        }
        sx[k] = x;
        sy[k] = y;
    }
    double a = 0, b = 0, e = -1;
    if (!sx.empty()) minimax_fit(sx, sy, a, b, e);
    float err = (float) e;
    const float fa = (float) a, fb = (float) b;
    if (fa > 0 || fb < 0) err = -1;
    else if (0 < err && err < (float) S) err += 0.01f;
    else err = -1;
    rec[0] = fa; rec[1] = fb; rec[2] = mu; rec[3] = sigma;
    rec[5] = thr[0]; rec[6] = thr[S - 1];
    if (err < 0 || (double) err > S - 1e-3) {
        const float first = cdf[0], last = cdf[S - 1];
        const float av = (float) (2.0f - (float) S) / (first - last);
        const float bv = ((float) S * first - last) / (first - last);
        rec[0] = av; rec[1] = bv;
        err = -1;
        for (int j = 0; j < S - 1; j++) {
            const float p1 = cdf[j] * av + bv, p2 = cdf[j + 1] * av + bv;
            const float e1 = std::abs((float) (j + 1) - p1), e2 = std::abs((float) (j + 1) - p2);
            const float te = std::max(e1, e2) + 0.01f;
            err = std::max(te, err);
        }
        err = std::min(err, (float) S);
        err += 0.01f;
    }
    rec[4] = err;
}

}  // namespace

namespace rkr {

// The SVD transform from the Gram matrix G = user^T user ([d][d], full; overwritten): cyclic Jacobi
// rotations to its eigen-decomposition user^T user = E diag(s^2) E^T, the singular values s
// (descending) with their vectors Es (column k for s[k]), transfer_item[r][c] = s_r * E[c][r], and
// check_dim, the first dimension whose cumulative singular value reaches sigma_ratio of the total
// (SVD.hpp:214-226).
void svd_from_gram(std::vector<double> &G, int d, float sigma_ratio, float *transfer_item, std::vector<double> &Es,
                   std::vector<float> &s, int *check_dim) {
    std::vector<double> E((size_t) d * d, 0.0);
    for (int i = 0; i < d; i++) E[(size_t) i * d + i] = 1.0;
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0, diag = 0;
        for (int p = 0; p < d; p++) {
            diag += G[(size_t) p * d + p] * G[(size_t) p * d + p];
            for (int q = p + 1; q < d; q++) off += G[(size_t) p * d + q] * G[(size_t) p * d + q];
        }
        if (off <= 1e-30 * diag) break;
        for (int p = 0; p < d; p++)
            for (int q = p + 1; q < d; q++) {
                const double apq = G[(size_t) p * d + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double th = (G[(size_t) q * d + q] - G[(size_t) p * d + p]) / (2 * apq);
                const double t = (th >= 0 ? 1.0 : -1.0) / (std::fabs(th) + std::sqrt(th * th + 1));
                const double c = 1 / std::sqrt(t * t + 1), s = t * c;
                for (int r = 0; r < d; r++) {
                    const double x = G[(size_t) r * d + p], y = G[(size_t) r * d + q];
                    G[(size_t) r * d + p] = c * x - s * y;
                    G[(size_t) r * d + q] = s * x + c * y;
                }
                for (int r = 0; r < d; r++) {
                    const double x = G[(size_t) p * d + r], y = G[(size_t) q * d + r];
                    G[(size_t) p * d + r] = c * x - s * y;
                    G[(size_t) q * d + r] = s * x + c * y;
                }
                for (int r = 0; r < d; r++) {
                    const double x = E[(size_t) r * d + p], y = E[(size_t) r * d + q];
                    E[(size_t) r * d + p] = c * x - s * y;
                    E[(size_t) r * d + q] = s * x + c * y;
                }
            }
    }
    std::vector<int> ord(d);
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](int a, int b) { return G[(size_t) a * d + a] > G[(size_t) b * d + b]; });
    s.assign(d, 0.0f);
    Es.assign((size_t) d * d, 0.0);
    for (int k = 0; k < d; k++) {
        const int e = ord[k];
        s[k] = (float) std::sqrt(std::max(G[(size_t) e * d + e], 0.0));
        for (int i = 0; i < d; i++) Es[(size_t) i * d + k] = E[(size_t) i * d + e];
    }
    for (int r = 0; r < d; r++)
        for (int c = 0; c < d; c++) transfer_item[(size_t) r * d + c] = (float) (s[r] * (float) Es[(size_t) c * d + r]);
    std::vector<float> cum(d);
    cum[0] = s[0];
    for (int c = 1; c < d; c++) cum[c] = cum[c - 1] + s[c];
    int cdim = 0;
    for (int c = 0; c < d; c++)
        if (cum[c] / cum[d - 1] >= sigma_ratio) { cdim = c; break; }
    *check_dim = cdim;
}

}  // namespace rkr

extern "C" {

int rkr_normalize(float *v, int64_t n, int32_t dim) {
    if (!v || n < 0 || dim <= 0) { rkr::set_error("rkr_normalize: bad argument"); return RKR_ERR_INVALID; }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) {
        float *row = v + i * dim;
        float l2 = 0.0f;
        for (int j = 0; j < dim; j++) l2 += row[j] * row[j];
        l2 = std::sqrt(l2);
        if (l2 <= 0.001) continue;
        for (int j = 0; j < dim; j++) row[j] /= l2;
    }
    return RKR_OK;
}

int rkr_sample_item(int32_t n_item, int32_t n_sample_item, int32_t *out) {
    if (!out || n_item <= 0 || n_sample_item < 0 || n_sample_item > n_item) {
        rkr::set_error("rkr_sample_item: bad argument");
        return RKR_ERR_INVALID;
    }
    std::vector<int> idx(n_item);
    std::iota(idx.begin(), idx.end(), 0);
    std::mt19937 eng(0);
    std::shuffle(idx.begin(), idx.end(), eng);
    for (int s = 0; s < n_sample_item; s++) out[s] = idx[s];
    return RKR_OK;
}

int rkr_sort_kth_rank(const int32_t *accu, int64_t n_item, int32_t n_sample_item, int32_t sample_topk,
                      int32_t *sort_kth_out, int32_t *sort_sample_id_out) {
    if (!accu || !sort_kth_out || !sort_sample_id_out || n_item <= 0 || n_sample_item <= 0 || sample_topk < 0) {
        rkr::set_error("rkr_sort_kth_rank: bad argument");
        return RKR_ERR_INVALID;
    }
    std::vector<int> kth(n_sample_item);
    for (int s = 0; s < n_sample_item; s++) {
        const int32_t *a = accu + (int64_t) s * (n_item + 1);
        kth[s] = (int) (std::lower_bound(a, a + n_item + 1, sample_topk) - a);
    }
    std::vector<int> sid(n_sample_item);
    std::iota(sid.begin(), sid.end(), 0);
    std::sort(sid.begin(), sid.end(), [&kth](int i1, int i2) { return kth[i1] < kth[i2]; });
    for (int s = 0; s < n_sample_item; s++) {
        sort_sample_id_out[s] = sid[s];
        sort_kth_out[s] = kth[sid[s]];
    }
    return RKR_OK;
}

int rkr_uniform_sample_rank(int32_t n_item, int32_t n_sample, int32_t *out) {
    if (!out || n_item <= 1 || n_sample <= 0 || n_sample >= n_item) {
        rkr::set_error("rkr_uniform_sample_rank: bad argument");
        return RKR_ERR_INVALID;
    }
    const double delta = (n_item - 1) * 1.0 / n_sample;
    for (int s = 0; s < n_sample; s++) out[s] = (int32_t) std::floor(s * delta);
    return RKR_OK;
}

// The OptimalPart dynamic program: candidate ranks {kth, kth - 1}, the cost of a sample set being
// the number of training-query users left unpruned (OptimalSampleRank.hpp:234-325), minimised over
// n_sample ranks (OptimalSampleRankFast.hpp:330-395), then the duplicate repair (:397-448).
int rkr_find_optimal_sample_rank(int64_t n_user, int64_t n_item, int32_t n_sample, int32_t nsq, const int32_t *kth,
                                 const int32_t *accu, int32_t *out, int64_t *train_cost) {
    if (!kth || !accu || !out || n_sample <= 0 || nsq <= 0 || n_item <= 0) {
        rkr::set_error("rkr_find_optimal_sample_rank: bad argument");
        return RKR_ERR_INVALID;
    }
    const int64_t W = n_item + 1;
    std::set<int> cs;
    for (int i = 0; i < nsq; i++) {
        cs.insert(kth[i]);
        if (kth[i] != 0) cs.insert(kth[i] - 1);
    }
    std::vector<int> cand(cs.begin(), cs.end());
    const int R = (int) cand.size();
    std::vector<int> this_last(R), next_first(R);
    for (int r = 0; r < R; r++) {
        this_last[r] = (int) (std::upper_bound(kth, kth + nsq, cand[r]) - kth);
        next_first[r] = (int) (std::lower_bound(kth, kth + nsq, cand[r] + 1) - kth);
    }
    auto A = [&](int q, int64_t r) -> int64_t { return accu[(int64_t) q * W + r]; };
    auto cost_end = [&](int r) -> int64_t {
        const int rank = cand[r] + 1, st = next_first[r];
        int64_t s = 0;
        for (int q = st; q < nsq; q++) s += n_user - A(q, rank - 1);
        return s;
    };
    auto cost_begin = [&](int r) -> int64_t {
        int64_t s = 0;
        for (int q = 0; q < this_last[r]; q++) s += A(q, cand[r]);
        return s;
    };
    auto cost_between = [&](int ub, int lb) -> int64_t {
        const int rank_ub = cand[ub] + 1, rank_lb = cand[lb];
        const int b = next_first[ub], e = this_last[lb];
        if (b >= nsq || b > e) return 0;
        int64_t s = 0;
        for (int q = b; q < e; q++) s += A(q, rank_lb) - A(q, rank_ub - 1);
        return s;
    };
    auto fill = [&](std::set<int> &set, int last_sample) {
        const int n_remain = n_sample - (int) set.size();
        const double delta = last_sample * 1.0 / n_remain;
        double ins = 0;
        while ((int) set.size() < n_sample && (int) ins < last_sample) {
            if (!set.count((int) ins)) { set.insert((int) ins); ins += delta; }
            else ins += 1;
        }
        for (int i = 0; (int) set.size() < n_sample && i < n_item; i++) set.insert(i);
    };
    if (train_cost) *train_cost = 0;
    if (R <= n_sample) {
        std::set<int> set(cand.begin(), cand.end());
        fill(set, nsq < 500 ? (int) n_item : cand[R - 1]);
        if ((int) set.size() != n_sample) { rkr::set_error("cannot fill %d sample ranks", n_sample); return RKR_ERR_INVALID; }
        int i = 0;
        for (int r : set) out[i++] = r;
        return RKR_OK;
    }
    std::vector<int64_t> end_cost(R);
    for (int r = 0; r < R; r++) end_cost[r] = cost_end(r);
    std::vector<int64_t> tr((size_t) R * R);
#pragma omp parallel for schedule(dynamic, 4)
    for (int lb = 1; lb < R; lb++)
        for (int ub = 0; ub < lb; ub++) tr[(size_t) lb * R + ub] = -end_cost[ub] + cost_between(ub, lb) + end_cost[lb];
    std::vector<int64_t> dp((size_t) n_sample * R);
    std::vector<int32_t> pos((size_t) n_sample * R);
    for (int r = 0; r < R; r++) { dp[r] = cost_begin(r) + end_cost[r]; pos[r] = r; }
    for (int s = 1; s < n_sample; s++) {
#pragma omp parallel for schedule(static)
        for (int r = 0; r < R; r++) {
            int64_t best = dp[(size_t) (s - 1) * R + r];
            int32_t bp = pos[(size_t) (s - 1) * R + r];
            for (int p = 0; p < r; p++) {
                const int64_t c = dp[(size_t) (s - 1) * R + p] + tr[(size_t) r * R + p];
                if (best > c) { best = c; bp = p; }
            }
            dp[(size_t) s * R + r] = best;
            pos[(size_t) s * R + r] = bp;
        }
    }
    uint64_t min_cost = UINT64_MAX;
    int idx = -1;
    for (int r = 0; r < R; r++) {
        const uint64_t c = (uint64_t) dp[(size_t) (n_sample - 1) * R + r];
        if (c < min_cost) { idx = r; min_cost = c; }
    }
    if (train_cost) *train_cost = (int64_t) min_cost;
    for (int s = n_sample - 1; s >= 0; s--) {
        out[s] = cand[idx];
        idx = pos[(size_t) s * R + idx];
    }
    std::set<int> set(out, out + n_sample);
    if ((int) set.size() != n_sample) {
        fill(set, cand[R - 1]);
        if ((int) set.size() != n_sample) { rkr::set_error("cannot fill %d sample ranks", n_sample); return RKR_ERR_INVALID; }
        int i = 0;
        for (int r : set) out[i++] = r;
    }
    return RKR_OK;
}

int rkr_fit_regression(const float *thr, int64_t n_user, int32_t S, float *rec_out) {
    if (!thr || !rec_out || n_user < 0 || S < 2) { rkr::set_error("rkr_fit_regression: bad argument"); return RKR_ERR_INVALID; }
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t u = 0; u < n_user; u++) fit_user(thr + u * S, S, rec_out + u * 7);
    return RKR_OK;
}

// SVD::PerformSVD (SVD.hpp:62-124) with the thin SVD from the Gram matrix: user^T user = E diag(s^2) E^T,
// transfer_item[r][c] = s_r * E[c][r], svd_user = user E diag(1/s); check_dim from the cumulative
// singular values (:214-226).
int rkr_svd_build(const float *user, int64_t n_user, int32_t dim, float sigma_ratio, float *transfer_item,
                  float *svd_user, int32_t *check_dim_out) {
    if (!user || !transfer_item || !svd_user || !check_dim_out || n_user <= 0 || dim <= 0) {
        rkr::set_error("rkr_svd_build: bad argument");
        return RKR_ERR_INVALID;
    }
    const int d = dim;
    std::vector<double> G((size_t) d * d, 0.0);
    // the Gram matrix's upper triangle, kGramBlock users per pass over a thread's partial sums (each
    // entry still adds the users' products one after another)
    constexpr int kGramBlock = 8;
#pragma omp parallel
    {
        std::vector<double> g((size_t) d * d, 0.0);
        std::vector<double> rb((size_t) kGramBlock * d);
#pragma omp for schedule(static)
        for (int64_t u0 = 0; u0 < n_user; u0 += kGramBlock) {
            const int nb = (int) std::min<int64_t>(kGramBlock, n_user - u0);
            for (int b = 0; b < kGramBlock; b++)
                for (int i = 0; i < d; i++) rb[(size_t) b * d + i] = b < nb ? (double) user[(u0 + b) * d + i] : 0.0;
            for (int i = 0; i < d; i++) {
                double ri[kGramBlock];
                for (int b = 0; b < kGramBlock; b++) ri[b] = rb[(size_t) b * d + i];
                double *gi = g.data() + (size_t) i * d;
#pragma omp simd
                for (int j = i; j < d; j++) {
                    double acc = gi[j];
                    for (int b = 0; b < kGramBlock; b++) acc += ri[b] * rb[(size_t) b * d + j];
                    gi[j] = acc;
                }
            }
        }
#pragma omp critical
        for (size_t k = 0; k < g.size(); k++) G[k] += g[k];
    }
    for (int i = 0; i < d; i++)
        for (int j = 0; j < i; j++) G[(size_t) i * d + j] = G[(size_t) j * d + i];
    std::vector<double> Es;
    std::vector<float> s;
    int check_dim = 0;
    rkr::svd_from_gram(G, d, sigma_ratio, transfer_item, Es, s, &check_dim);
    // svd_user = user Es diag(1/s), kProjBlock users at a time, each output summed over i in order
    constexpr int kProjBlock = 4;
#pragma omp parallel
    {
        std::vector<double> acc((size_t) kProjBlock * d);
#pragma omp for schedule(static)
        for (int64_t u0 = 0; u0 < n_user; u0 += kProjBlock) {
            const int nb = (int) std::min<int64_t>(kProjBlock, n_user - u0);
            std::fill(acc.begin(), acc.end(), 0.0);
            for (int i = 0; i < d; i++) {
                const double *ei = Es.data() + (size_t) i * d;
                for (int b = 0; b < nb; b++) {
                    const double ri = user[(u0 + b) * d + i];
                    double *ab = acc.data() + (size_t) b * d;
#pragma omp simd
                    for (int k = 0; k < d; k++) ab[k] += ri * ei[k];
                }
            }
            for (int b = 0; b < nb; b++)
                for (int k = 0; k < d; k++)
                    svd_user[(u0 + b) * d + k] = s[k] > 0 ? (float) (acc[(size_t) b * d + k] / s[k]) : 0.0f;
        }
    }
    *check_dim_out = check_dim;
    return RKR_OK;
}

}  // extern "C"
