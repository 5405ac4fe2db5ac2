// rkr_regression.cuh -- the regression model's query-time arithmetic (NormalLinearRegressionLP.hpp),
// exact and screened, shared by the scores kernels.
#pragma once

#include "rkr_internal.cuh"

namespace rkr {

// ---- the regression model's arithmetic (NormalLinearRegressionLP.hpp) ------------------------------

// float -> int64 as x86-64 converts it (cvttss2si): NaN and out-of-range values give INT64_MIN.
__device__ __forceinline__ int64_t f2i64_x86(float v) {
    if (!(v >= -9.2233720368547758e18f && v < 9.2233720368547758e18f)) return INT64_MIN;
    return (int64_t) v;
}

// NormalLinearRegressionLP::CDFPhi (:123-143).  Float constants; t and the closing expression pass
// through double; exp is the double ::exp (the query and regression apps never bring the float
// overload into scope).  sqrt_2_ is ReverseMIPS::sqrt(2.0) (MathUtil.hpp:10-27), which equals
// the binary32 nearest to sqrt(2).
__device__ __forceinline__ float cdf_phi(float x) {
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f;
    const float a4 = -1.453152027f, a5 = 1.061405429f, p = 0.3275911f;
    const float sqrt_2 = __int_as_float(0x3fb504f3);
    const int sign = x < 0 ? -1 : 1;
    x = __fdiv_rn(fabsf(x), sqrt_2);
    const float t = __double2float_rn(__ddiv_rn(1.0, __dadd_rn(1.0, (double) __fmul_rn(p, x))));
    float poly = __fadd_rn(__fmul_rn(a5, t), a4);
    poly = __fmul_rn(poly, t);
    poly = __fadd_rn(poly, a3);
    poly = __fadd_rn(__fmul_rn(poly, t), a2);
    poly = __fadd_rn(__fmul_rn(poly, t), a1);
    const float pt = __fmul_rn(poly, t);
    const double e = exp((double) __fmul_rn(-x, x));
    const float y = __double2float_rn(__dsub_rn(1.0, __dmul_rn((double) pt, e)));
    return __double2float_rn(__dmul_rn(0.5, __dadd_rn(1.0, (double) __fmul_rn((float) sign, y))));
}

// The same formula in binary32 with the hardware reciprocal and exponential, for screening.
// Against cdf_phi, with z given as (q - mu) * (1 / sigma) instead of (q - mu) / sigma, it differs
// by less than kCdfFastErr: the argument and x differ by a few ulps (< 1e-7 after the slope of
// the CDF), t by a few ulps (< 4e-7 on pt * e), the fused polynomial and the approximate exp by a
// few ulps more (< 3e-7), and the closing steps by one rounding each.
constexpr float kCdfFastErr = 2.0e-6f;

__device__ __forceinline__ float cdf_phi_fast(float z) {
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f;
    const float a4 = -1.453152027f, a5 = 1.061405429f, p = 0.3275911f;
    const float x = fabsf(z) * 0.70710677f;
    const float t = __fdividef(1.0f, fmaf(p, x, 1.0f));
    const float pt = fmaf(fmaf(fmaf(fmaf(a5, t, a4), t, a3), t, a2), t, a1) * t;
    const float y = fmaf(-pt, __expf(-x * x), 1.0f);
    return fmaf(z < 0.0f ? -0.5f : 0.5f, y, 0.5f);
}

struct RegModel {           // device view of the regression index
    const float *rec;       // [n_user][8]
    const int32_t *rank;    // [S]
    int S;
    double err_cap;         // S - 1e-3
    int n_item;
};

// The reference's float/double evaluation of one side of ComputeRankBound's index arithmetic:
// pr = ceil(pred + err) (upper = 0) or floor(pred - err) (upper = 1), pred = cdf(nx) * a + b.
__device__ __forceinline__ int64_t regression_index_exact(float nx, float a, float b, float err, bool upper) {
    const float ix = cdf_phi(nx);
    const float pred = __fadd_rn(__fmul_rn(ix, a), b);
    return upper ? f2i64_x86(floorf(__fsub_rn(pred, err))) : f2i64_x86(ceilf(__fadd_rn(pred, err)));
}

// One side of ComputeRankBound (:326-380) with the reference's arithmetic at score q: the level of
// rank_lb (upper = false; 1 .. S + 1) or of rank_ub (upper = true; 0 .. S + 1).  capped: the fit
// error reached the cap, so the model is not used.
__device__ __forceinline__ int regression_level_side(float a, float b, float mu, float sigma, float err, float smax,
                                                     float smin, bool capped, int S, float q, bool upper) {
    if (!upper) {
        if (q > smax) return 1;
        if (q < smin || capped) return S + 1;
        const int64_t pr = regression_index_exact(__fdiv_rn(__fsub_rn(q, mu), sigma), a, b, err, false);
        return pr >= S ? S + 1 : (pr < 0 ? 1 : (int) pr + 1);
    }
    if (q > smax) return 0;
    if (q < smin) return S;
    if (capped) return 0;
    const int64_t pr = regression_index_exact(__fdiv_rn(__fsub_rn(q, mu), sigma), a, b, err, true);
    return pr >= S ? S + 1 : (pr < 0 ? 0 : (int) pr + 1);
}

// ComputeRankBound (:326-380) with the reference's arithmetic, returning levels: 0 -> rank 0,
// j + 1 -> rank[j], S + 1 -> n_item.
// Returns lvl_lb | lvl_ub << 16.  Scalar arguments only: a call with a reference to a kernel
// parameter would copy the parameters to local memory.
static __device__ __noinline__ uint32_t regression_levels_exact(const float *__restrict__ rec, int S, double err_cap,
                                                               int64_t u, float qlb, float qub) {
    const float4 r0 = __ldg(reinterpret_cast<const float4 *>(rec + u * 8));
    const float4 r1 = __ldg(reinterpret_cast<const float4 *>(rec + u * 8 + 4));
    const float a = r0.x, b = r0.y, mu = r0.z, sigma = r0.w, err = r1.x, smax = r1.y, smin = r1.z;
    int lvl_lb, lvl_ub;
    if (qlb > smax) lvl_lb = 1;
    else if (qlb < smin) lvl_lb = S + 1;
    else if ((double) err >= err_cap) lvl_lb = S + 1;
    else {
        const int64_t pr = regression_index_exact(__fdiv_rn(__fsub_rn(qlb, mu), sigma), a, b, err, false);
        lvl_lb = pr >= S ? S + 1 : (pr < 0 ? 1 : (int) pr + 1);
    }
    if (qub > smax) lvl_ub = 0;
    else if (qub < smin) lvl_ub = S;
    else if ((double) err >= err_cap) lvl_ub = 0;
    else {
        const int64_t pr = regression_index_exact(__fdiv_rn(__fsub_rn(qub, mu), sigma), a, b, err, true);
        lvl_ub = pr >= S ? S + 1 : (pr < 0 ? 0 : (int) pr + 1);
    }
    return (uint32_t) lvl_lb | ((uint32_t) lvl_ub << 16);
}

// One user's model prepared for the screen.  A user whose fit error reaches the cap (the
// reference then gives up on the model: ComputeRankBound's error test) gets an infinite margin,
// so every one of its pairs goes to the reference's own arithmetic.
struct RegUser {
    float a, b, mu, inv_sigma, err, smax, smin, margin;
};

__device__ __forceinline__ RegUser reg_user(const RegModel &m, int64_t u) {
    const float4 r0 = __ldg(reinterpret_cast<const float4 *>(m.rec + u * 8));
    const float4 r1 = __ldg(reinterpret_cast<const float4 *>(m.rec + u * 8 + 4));
    RegUser r;
    r.a = r0.x; r.b = r0.y; r.mu = r0.z; r.inv_sigma = __frcp_rn(r0.w);
    r.err = r1.x; r.smax = r1.y; r.smin = r1.z;
    // |pred -+ err| moves by at most |a| * kCdfFastErr through the CDF, plus a few roundings of
    // values no larger than |a| + |b| + |err| in either evaluation.
    r.margin = (double) r1.x >= m.err_cap
                   ? INFINITY
                   : fabsf(r.a) * kCdfFastErr + (fabsf(r.a) + fabsf(r.b) + fabsf(r.err)) * 4.8e-7f + 1e-6f;
    return r;
}

// Level of one side from the integral-valued c = ceil (lower bound) or floor (upper bound) of
// pred -+ err: c >= S -> S + 1, c < 0 -> low, else c + 1.
__device__ __forceinline__ int level_of(float c, int S, int low) {
    return c >= (float) S ? S + 1 : (c < 0.0f ? low : (int) c + 1);
}

// Screened ComputeRankBound: the fast CDF decides a side whenever pred -+ err lies farther than
// the margin from an integer, so that the reference's ceil / floor cannot differ (values beyond
// 1e18, where the reference's int64 conversion saturates, are left undecided too).  Returns false
// when a side is undecided (its level is then not meaningful).
__device__ __forceinline__ bool regression_levels_fast(const RegUser &r, int S, float qlb, float qub, int &lvl_lb,
                                                       int &lvl_ub) {
    const float vl = fmaf(cdf_phi_fast(__fsub_rn(qlb, r.mu) * r.inv_sigma), r.a, r.b) + r.err;
    const float vu = fmaf(cdf_phi_fast(__fsub_rn(qub, r.mu) * r.inv_sigma), r.a, r.b) - r.err;
    const bool in_l = !(qlb > r.smax) && !(qlb < r.smin);
    const bool in_u = !(qub > r.smax) && !(qub < r.smin);
    // |v| < 1e18 (the reference's int64 conversion is exact there) folds into the margin test
    const bool ok_l = fabsf(vl - rintf(vl)) > r.margin && fabsf(vl) < 1e18f;
    const bool ok_u = fabsf(vu - rintf(vu)) > r.margin && fabsf(vu) < 1e18f;
    lvl_lb = qlb > r.smax ? 1 : (in_l ? level_of(ceilf(vl), S, 1) : S + 1);
    lvl_ub = qub > r.smax ? 0 : (in_u ? level_of(floorf(vu), S, 0) : S);
    // a capped-error user's margin is infinite: its in-range sides are always left undecided
    return (!in_l || ok_l) && (!in_u || ok_u) && r.margin < INFINITY;
}

// ---- per-user level-boundary tables ------------------------------------------------------------------
//
// For each user and side, the reference's level is a non-increasing step function of the score.
// The table holds, at each of kLvEntries level values L_g (lvt_level: L_0 = 0, then 14 steps of
// about S / 14 up to L_14 = S, and L_15 = S + 1), the smallest binary32 score T_g whose level is
// <= L_g, and a guard band: outside [T_g - band_g, T_g + band_g] the level's relation to L_g is the
// exact-math one (the reference's binary32 evaluation can only differ from it where the model's
// value lies within its rounding error of the crossing integer).  A score's coarse level is the
// number of boundaries above it, c = #{g : q < T_g}: the smallest g with level <= L_g.  Coarse
// level 0 is exactly level 0 and coarse level 15 exactly level S + 1 (the extremes most pairs sit
// at); the others span (L_(c-1), L_c].  The coarse level of q is decided for every score within dq
// of q when (c == kLvEntries - 1 or q - dq >= T_c + band_c) and (c == 0 or q + dq < T_(c-1) -
// band_(c-1)).  Entries are (T_g, band_g); a user whose record is unusable for the tables (a
// non-finite value, sigma <= 0, a slope a >= 0) has NaN entries, so none of its pairs is ever
// decided from them.
constexpr int kLvEntries = 16;

__host__ __device__ __forceinline__ int lvt_level(int g, int S) {  // S < 2^26: 32-bit products
    return g >= kLvEntries - 1 ? S + 1 : (g * S + (kLvEntries - 3)) / (kLvEntries - 2);
}
// coarse level of an exact level: the smallest g with level <= L_g
__host__ __device__ __forceinline__ int lvt_coarse(int l, int S) {
    if (l <= 0) return 0;
    if (l > S) return kLvEntries - 1;
    return (kLvEntries - 2) * (l - 1) / S + 1;
}
// most levels in one coarse level (the fine histograms' width)
__host__ __device__ __forceinline__ int lvt_width(int S) { return (S + kLvEntries - 3) / (kLvEntries - 2) + 1; }

// Coarse level of score q on one side from the table row (entry j of this user at t[j * stride]),
// and whether every score within dq of q has it.  This is the decision rule itself; the pair-scores
// kernel applies it through register-cached boundaries (the lower side) and through the limit and
// verification-pair forms below (lvt_screen_lim, lvt_screen_ver), which decide a subset of its pairs
// with the same levels (restated on the CPU in tests/test_level_tables.py).
__device__ __forceinline__ bool lvt_screen(const float2 *t, int stride, float q, float dq, int &c) {
    int k = 0;
#pragma unroll
    for (int st = 8; st >= 1; st >>= 1) k += q < t[(k + st - 1) * stride].x ? st : 0;
    c = k;
    bool ok = true;
    if (k < kLvEntries - 1) {
        const float2 e = t[k * stride];
        ok = __fsub_rd(q, dq) >= __fadd_ru(e.x, e.y);
    }
    if (k > 0) {
        const float2 e = t[(k - 1) * stride];
        ok = ok && __fadd_ru(q, dq) < __fsub_rd(e.x, e.y);
    }
    return ok;
}

// The same decision from a row of limits (lo_g, hi_g): lo_g at or below T_g - band_g and hi_g at or
// above T_g + band_g, lo non-increasing and hi non-increasing in g (lvt_limits_row), with qm at or
// below q - dq and qp at or above q + dq.  c = #{g : qp < lo_g} (a prefix of the entries, lo being
// monotone), decided when (c == kLvEntries - 1 or qm >= hi_c) and (c == 0 or qp < lo_(c-1)): every
// score s within dq of q then lies above the band of boundary c and below that of boundary c - 1.
__device__ __forceinline__ bool lvt_screen_lim(const float2 *t, int stride, float qm, float qp, int &c) {
    int k = 0;
#pragma unroll
    for (int st = 8; st >= 1; st >>= 1) k += qp < t[(k + st - 1) * stride].x ? st : 0;
    c = k;
    bool ok = k == kLvEntries - 1 || qm >= t[k * stride].y;
    if (k > 0) ok = ok && qp < t[(k - 1) * stride].x;
    return ok;
}

// One user's table row (entry j at t[j * stride], entries (T_j, band_j)) in place as limits: lo_j =
// T_j - band_j rounded down, then the running minimum from entry 0; hi_j = T_j + band_j rounded up,
// then the running maximum from the last entry.  Each limit only moves away from its boundary, so a
// decision lvt_screen_lim makes from them is one the bands allow.  A row with a NaN stays all NaN.
__device__ __forceinline__ void lvt_limits_row(float2 *t, int stride) {
    bool bad = false;
    float lo = INFINITY;
    for (int j = 0; j < kLvEntries; j++) {
        const float2 e = t[j * stride];
        bad = bad || !(e.x == e.x) || !(e.y == e.y);
        lo = fminf(lo, __fsub_rd(e.x, e.y));
        t[j * stride] = make_float2(lo, __fadd_ru(e.x, e.y));
    }
    float hi = -INFINITY;
    for (int j = kLvEntries - 1; j >= 0; j--) {
        hi = fmaxf(hi, t[j * stride].y);
        t[j * stride].y = hi;
    }
    if (bad)
        for (int j = 0; j < kLvEntries; j++) t[j * stride] = make_float2(NAN, NAN);
}

// A row of limits (lvt_limits_row) rewritten in place as verification pairs: entry c = (hi_c,
// lo_(c-1)), lo_(-1) = +inf.  One entry then decides coarse level c (qm >= hi_c and qp < lo_(c-1)),
// and lo_j is entry j + 1's second value.
__device__ __forceinline__ void lvt_verify_row(float2 *t, int stride) {
    for (int j = kLvEntries - 1; j >= 1; j--) t[j * stride] = make_float2(t[j * stride].y, t[(j - 1) * stride].x);
    const float h0 = t[0].y;
    t[0] = make_float2(h0, h0 == h0 ? INFINITY : NAN);
}
// lvt_screen_lim on a row of verification pairs.
__device__ __forceinline__ bool lvt_screen_ver(const float2 *t, int stride, float qm, float qp, int &c) {
    int k = 0;
#pragma unroll
    for (int st = 8; st >= 1; st >>= 1) k += qp < t[(k + st) * stride].y ? st : 0;
    c = k;
    const float2 e = t[k * stride];
    return qm >= e.x && qp < e.y;
}

__device__ __forceinline__ int level_rank(int lvl, const int32_t *rank, int S, int n_item) {
    return lvl == 0 ? 0 : (lvl > S ? n_item : rank[lvl - 1]);
}

// One batch of pair scores for the bound rounds (rkr_scores_tc.cu): coarse levels (QSRP) and coarse
// group codes of every (query, user) pair (their histograms are a separate pass over the bytes).
struct ScoresTcCall {
    bool qsrp;
    const float *qrows, *qnorm, *unorm;  // queries (SVD space for QSRP), remaining-coordinate norms
    int nq;
    RegModel m;
    int nb;
    uint8_t *lvc;    // [nq][n_user] (QSRP)
    uint8_t *code;   // [nq][n_user]
    int *anomaly;    // [nq] (QSRP), zeroed by the caller
    int **status = nullptr;  // if set ([4]): receives device pointers to the run's status (0: complete),
                             // undecided-pair count and the two table-search counts (lower, upper side:
                             // warp passes x 32), and the call does not wait for the device
};
// Runs the tensor-core scores where the shape allows; *done = false leaves the batch to the exact
// tiles (the anomaly counts may then be partial: the caller clears them).  With call.status
// set, *done only says the kernels were launched; the caller checks the status on the device.
int scores_tc(rkr_index *ix, const ScoresTcCall &call, cudaStream_t st, bool *done);

}  // namespace rkr
