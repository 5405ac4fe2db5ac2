// The regression models of the NormalLinearRegressionLP index fitted on the device, from the
// index's resident sampled thresholds (NormalLinearRegressionLP.hpp:72-310: StartPreprocess /
// BatchLoopPreprocess).  One warp per user: the mean and deviation of the user's thresholds, the
// normal CDF of each standardised threshold (CDFPhi, :123-143), the minimax line through the points
// (cdf_j, j + 1), (cdf_{j+1}, j + 1) (the optimum of LinearProgram's LP, :181-213) and the
// endpoint-line fallback with CalcError (:215-243, 272-296).  The arithmetic is the host fit's
// (rkr_host.cpp): every operation spelled with its rounding (no contraction into FMAs), sums in the
// reference's order on one lane, so the records equal the host's.
#include <climits>
#include <cstring>
#include <vector>

#include "rkr_internal.cuh"

namespace rkr {
namespace {

constexpr int kFitMaxWarps = 4;   // users per block (fewer where one user's arrays are large)
constexpr int kFitMaxS = 4096;    // thresholds per user the shared-memory layout holds

struct FitSmem {  // one warp's arrays, S thresholds, n = 2S - 2 points
    float *cdf;      // [S]
    double *xs;      // [n] point x, sorted with ys
    int32_t *ys;     // [n] point y
    uint16_t *lo;    // [n] lower hull (point indices)
    uint16_t *up;    // [n] upper hull
};

__host__ __device__ inline size_t fit_warp_bytes(int S) {
    const size_t n = (size_t) (2 * S - 2 > 0 ? 2 * S - 2 : 1);
    auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
    return al(4 * (size_t) S) + al(8 * n) + al(4 * n) + 2 * al(2 * n);
}

// CDFPhi: float constants and polynomial, t and the closing expression in double, the double exp.
__device__ float fit_cdf_phi(float x) {
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f;
    const float a4 = -1.453152027f, a5 = 1.061405429f, p = 0.3275911f;
    const float sqrt_2 = 1.41421354f;
    int sign = 1;
    if (x < 0) sign = -1;
    x = __fdiv_rn(fabsf(x), sqrt_2);
    const float t = __double2float_rn(__ddiv_rn(1.0, __dadd_rn(1.0, (double) __fmul_rn(p, x))));
    float pt = __fadd_rn(__fmul_rn(a5, t), a4);
    pt = __fadd_rn(__fmul_rn(pt, t), a3);
    pt = __fadd_rn(__fmul_rn(pt, t), a2);
    pt = __fadd_rn(__fmul_rn(pt, t), a1);
    pt = __fmul_rn(pt, t);
    const float y = __double2float_rn(__dsub_rn(1.0, __dmul_rn((double) pt, exp((double) __fmul_rn(-x, x)))));
    return __double2float_rn(__dmul_rn(0.5, __dadd_rn(1.0, (double) __fmul_rn((float) sign, y))));
}

__device__ __forceinline__ double cross3(const double *xs, const int32_t *ys, int o, int p, int q) {
    return __dsub_rn(__dmul_rn(__dsub_rn(xs[p], xs[o]), __dsub_rn((double) ys[q], (double) ys[o])),
                     __dmul_rn(__dsub_rn((double) ys[p], (double) ys[o]), __dsub_rn(xs[q], xs[o])));
}

// Slope of hull edge k (a vertical edge: +inf).
__device__ __forceinline__ double edge_slope(const double *xs, const int32_t *ys, const uint16_t *h, int k) {
    const double dx = __dsub_rn(xs[h[k + 1]], xs[h[k]]);
    return dx != 0 ? __ddiv_rn(__dsub_rn((double) ys[h[k + 1]], (double) ys[h[k]]), dx) : __longlong_as_double(0x7ff0000000000000ll);
}

// max (y - s x) over the upper hull (nu vertices), or min over the lower hull: the vertex where the
// edge slopes cross s, found by binary search, and three vertices either side of it.
template <bool kTop>
__device__ double hull_extreme(const double *xs, const int32_t *ys, const uint16_t *h, int nh, double s) {
    int lo = 0, len = nh - 1;  // partition point over the nh - 1 edge slopes
    while (len > 0) {
        const int half = len >> 1, mid = lo + half;
        const double v = edge_slope(xs, ys, h, mid);
        if (kTop ? v > s : v < s) { lo = mid + 1; len -= half + 1; } else len = half;
    }
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    double m = kTop ? -inf : inf;
    const int j0 = lo > 3 ? lo - 3 : 0, j1 = min(nh, lo + 4);
    for (int j = j0; j < j1; j++) {
        const double v = __dsub_rn((double) ys[h[j]], __dmul_rn(s, xs[h[j]]));
        m = kTop ? ((m < v) ? v : m) : ((v < m) ? v : m);  // std::max / std::min
    }
    return m;
}

__global__ void __launch_bounds__(32 * kFitMaxWarps) fit_regression_kernel(const float *__restrict__ thr,
                                                                          int64_t n_user, int S,
                                                                          float *__restrict__ rec8) {
    extern __shared__ __align__(16) uint8_t fit_smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, n_warps = blockDim.x >> 5;
    const int64_t u = (int64_t) blockIdx.x * n_warps + warp;
    if (u >= n_user) return;
    const int n = 2 * S - 2;
    uint8_t *base = fit_smem + (size_t) warp * fit_warp_bytes(S);
    auto al = [](size_t b) { return (b + 15) & ~size_t(15); };
    FitSmem sm;
    sm.cdf = reinterpret_cast<float *>(base);
    sm.xs = reinterpret_cast<double *>(base + al(4 * (size_t) S));
    sm.ys = reinterpret_cast<int32_t *>(reinterpret_cast<uint8_t *>(sm.xs) + al(8 * (size_t) max(n, 1)));
    sm.lo = reinterpret_cast<uint16_t *>(reinterpret_cast<uint8_t *>(sm.ys) + al(4 * (size_t) max(n, 1)));
    sm.up = reinterpret_cast<uint16_t *>(reinterpret_cast<uint8_t *>(sm.lo) + al(2 * (size_t) max(n, 1)));
    const float *t = thr + u * S;
    // thresholds into shared memory (cdf holds them until the CDFs replace them)
    for (int s = lane; s < S; s += 32) sm.cdf[s] = t[s];
    __syncwarp();
    float mu = 0.0f, sigma = 0.0f;
    if (lane == 0) {
        for (int s = 0; s < S; s++) mu = __fadd_rn(mu, sm.cdf[s]);
        mu = __fdiv_rn(mu, (float) S);
        for (int s = 0; s < S; s++) {
            const float m = __fsub_rn(sm.cdf[s], mu);
            sigma = __fadd_rn(sigma, __fmul_rn(m, m));
        }
        sigma = __fdiv_rn(sigma, (float) S);
        sigma = __fsqrt_rn(sigma);
    }
    mu = __shfl_sync(0xffffffffu, mu, 0);
    sigma = __shfl_sync(0xffffffffu, sigma, 0);
    __syncwarp();
    for (int s = lane; s < S; s += 32) sm.cdf[s] = fit_cdf_phi(__fdiv_rn(__fsub_rn(sm.cdf[s], mu), sigma));
    __syncwarp();
    // points (cdf_{j+1}, j + 1), (cdf_j, j + 1) for j = S-2 .. 0, then sorted by (x, y) ascending
    for (int i = lane; i < n; i += 32) {
        const int j = S - 2 - (i >> 1);
        sm.xs[i] = (double) sm.cdf[(i & 1) ? j : j + 1];
        sm.ys[i] = j + 1;
    }
    __syncwarp();
    int n_lo = 0, n_up = 0;
    if (lane == 0) {
        // insertion sort: the walk leaves only adjacent equal-x points out of order (linear time)
        for (int i = 1; i < n; i++) {
            const double x = sm.xs[i];
            const int32_t y = sm.ys[i];
            int k = i;
            while (k > 0 && (x < sm.xs[k - 1] || (x == sm.xs[k - 1] && y < sm.ys[k - 1]))) {
                sm.xs[k] = sm.xs[k - 1];
                sm.ys[k] = sm.ys[k - 1];
                k--;
            }
            sm.xs[k] = x;
            sm.ys[k] = y;
        }
        // monotone-chain hulls: the lower hull takes the lowest point of each x, the upper the highest
        for (int i = 0; i < n; i++) {
            if (i == 0 || sm.xs[i] != sm.xs[i - 1]) {
                while (n_lo >= 2 && cross3(sm.xs, sm.ys, sm.lo[n_lo - 2], sm.lo[n_lo - 1], i) <= 0) n_lo--;
                sm.lo[n_lo++] = (uint16_t) i;
            }
            if (i + 1 == n || sm.xs[i + 1] != sm.xs[i]) {
                while (n_up >= 2 && cross3(sm.xs, sm.ys, sm.up[n_up - 2], sm.up[n_up - 1], i) >= 0) n_up--;
                sm.up[n_up++] = (uint16_t) i;
            }
        }
    }
    n_lo = __shfl_sync(0xffffffffu, n_lo, 0);
    n_up = __shfl_sync(0xffffffffu, n_up, 0);
    __syncwarp();
    // every hull edge's slope tried (lower hull's edges first, then the upper's: the first narrowest
    // strip in that order is kept, as the host fit keeps it)
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    double best = inf, ba = 0, bb = 0;
    int best_k = INT_MAX;
    const int e_lo = n_lo > 1 ? n_lo - 1 : 0, e_up = n_up > 1 ? n_up - 1 : 0;
    for (int k = lane; k < e_lo + e_up; k += 32) {
        const uint16_t *h = k < e_lo ? sm.lo : sm.up;
        const int kk = k < e_lo ? k : k - e_lo;
        const double dx = __dsub_rn(sm.xs[h[kk + 1]], sm.xs[h[kk]]);
        if (dx == 0) continue;
        const double s = __ddiv_rn(__dsub_rn((double) sm.ys[h[kk + 1]], (double) sm.ys[h[kk]]), dx);
        const double mx = hull_extreme<true>(sm.xs, sm.ys, sm.up, n_up, s);
        const double mn = hull_extreme<false>(sm.xs, sm.ys, sm.lo, n_lo, s);
        const double w = __dmul_rn(0.5, __dsub_rn(mx, mn));
        if (w < best) { best = w; ba = s; bb = __dmul_rn(0.5, __dadd_rn(mx, mn)); best_k = k; }
    }
    // the lane's first narrowest strip; the warp's: the narrowest, the earliest edge among equals
#pragma unroll
    for (int o = 16; o >= 1; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o), oa = __shfl_xor_sync(0xffffffffu, ba, o);
        const double obb = __shfl_xor_sync(0xffffffffu, bb, o);
        const int ok = __shfl_xor_sync(0xffffffffu, best_k, o);
        if (ob < best || (ob == best && ok < best_k)) { best = ob; ba = oa; bb = obb; best_k = ok; }
    }
    if (lane != 0) return;
    if (!(best < inf)) {
        double mx = -inf, mn = inf;
        for (int i = 0; i < n; i++) {
            const double y = (double) sm.ys[i];
            mx = (mx < y) ? y : mx;
            mn = (y < mn) ? y : mn;
        }
        ba = 0;
        bb = n ? __dmul_rn(0.5, __dadd_rn(mx, mn)) : 0;
        best = n ? __dmul_rn(0.5, __dsub_rn(mx, mn)) : 0;
    }
    double e = n ? best : -1.0;
    if (!n) { ba = 0; bb = 0; }
    float err = __double2float_rn(e);
    const float fa = __double2float_rn(ba), fb = __double2float_rn(bb);
    if (fa > 0 || fb < 0) err = -1;
    else if (0 < err && err < (float) S) err = __fadd_rn(err, 0.01f);
    else err = -1;
    float *r = rec8 + u * 8;
    float ra = fa, rb = fb;
    if (err < 0 || (double) err > __dsub_rn((double) S, 1e-3)) {
        const float first = sm.cdf[0], last = sm.cdf[S - 1];
        const float fl = __fsub_rn(first, last);
        const float av = __fdiv_rn(__fsub_rn(2.0f, (float) S), fl);
        const float bv = __fdiv_rn(__fsub_rn(__fmul_rn((float) S, first), last), fl);
        ra = av;
        rb = bv;
        err = -1;
        for (int j = 0; j < S - 1; j++) {
            const float p1 = __fadd_rn(__fmul_rn(sm.cdf[j], av), bv), p2 = __fadd_rn(__fmul_rn(sm.cdf[j + 1], av), bv);
            const float e1 = fabsf(__fsub_rn((float) (j + 1), p1)), e2 = fabsf(__fsub_rn((float) (j + 1), p2));
            const float m12 = (e1 < e2) ? e2 : e1;  // std::max(e1, e2)
            const float te = __fadd_rn(m12, 0.01f);
            err = (te < err) ? err : te;             // std::max(te, err)
        }
        err = ((float) S < err) ? (float) S : err;   // std::min(err, S)
        err = __fadd_rn(err, 0.01f);
    }
    r[0] = ra; r[1] = rb; r[2] = mu; r[3] = sigma; r[4] = err; r[5] = t[0]; r[6] = t[S - 1]; r[7] = 0.0f;
}

}  // namespace

// Models of users [u_begin, u_end) into ix->reg (already holding n_user records).
int fit_regression_device(rkr_index *ix, int64_t u_begin, int64_t u_end, cudaStream_t st) {
    const int S = ix->n_sample;
    int optin = 0;
    RKR_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ix->device));
    const size_t per_warp = fit_warp_bytes(S);
    const int warps = (int) std::max<size_t>(1, std::min<size_t>(kFitMaxWarps, (size_t) optin / per_warp));
    const size_t smem = per_warp * warps;
    if (smem > (size_t) optin) {
        set_error("rkr_index_fit_regression: %d thresholds per user need %zu bytes of shared memory", S, smem);
        return RKR_ERR_INVALID;
    }
    RKR_CUDA(cudaFuncSetAttribute(fit_regression_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    const int64_t nu = u_end - u_begin;
    if (nu <= 0) return RKR_OK;
    const unsigned grid = (unsigned) ((nu + warps - 1) / warps);
    timed(ix, st, "fit_regression", [&] {
        fit_regression_kernel<<<grid, 32 * warps, smem, st>>>(ix->thr.as<float>() + u_begin * S, nu, S,
                                                              ix->reg.as<float>() + u_begin * 8);
    });
    RKR_CUDA(cudaGetLastError());
    return RKR_OK;
}

}  // namespace rkr

using rkr::set_error;

extern "C" int rkr_index_fit_regression(rkr_index *ix, float *records_out) {
    RKR_REQUIRE(ix, "null index");
    if (ix->n_sample <= 0) {
        set_error("rkr_index_fit_regression: the index has no sampled thresholds (load or build them first)");
        return RKR_ERR_STATE;
    }
    RKR_REQUIRE(ix->n_sample >= 2 && ix->n_sample <= rkr::kFitMaxS,
                "rkr_index_fit_regression: n_sample %d outside [2, %d] (rkr_fit_regression fits any size on the host)",
                ix->n_sample, rkr::kFitMaxS);
    RKR_TRY(rkr::ensure_device(ix));
    const int S = ix->n_sample;
    RKR_TRY(ix->reg.ensure(sizeof(float) * 8 * (size_t) ix->n_user));
    RKR_TRY(rkr::fit_regression_device(ix, 0, ix->n_user, ix->stream));
    RKR_TRY(ix->reg_rank.ensure(sizeof(int32_t) * S));
    RKR_CUDA(cudaMemcpyAsync(ix->reg_rank.p, ix->h_sample_rank.data(), sizeof(int32_t) * S, cudaMemcpyHostToDevice,
                             ix->stream));
    ix->n_sample_reg = S;
    RKR_TRY(rkr::level_tables_build(ix));
    if (records_out) {
        std::vector<float> rec8((size_t) ix->n_user * 8);
        RKR_CUDA(cudaMemcpyAsync(rec8.data(), ix->reg.p, sizeof(float) * rec8.size(), cudaMemcpyDeviceToHost,
                                 ix->stream));
        RKR_CUDA(cudaStreamSynchronize(ix->stream));
        for (int64_t u = 0; u < ix->n_user; u++) std::memcpy(records_out + u * 7, &rec8[(size_t) u * 8], 7 * sizeof(float));
    }
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}
