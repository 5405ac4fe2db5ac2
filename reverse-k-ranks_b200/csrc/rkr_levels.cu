// rkr_levels.cu -- per-user level-boundary tables of the regression rank bound.
//
// QSRPNormalLP's first round (src/impl/QSRPNormalLP.hpp:144-165) turns every (query, user) pair's
// bound scores into levels of NormalLinearRegressionLP::ComputeRankBound
// (NormalLinearRegressionLP.hpp:326-398): lower side ceil(pred + err), upper side floor(pred - err),
// pred = a CDFPhi((q - mu) / sigma) + b, with the extreme-score shortcuts at smax / smin.  For one
// user and side that level is a non-increasing step function of the score, so the coarse level of a
// score (which of the table's level intervals holds its level) is the number of table boundaries
// above it.  The tables are built here
// once per regression index, with the reference's own arithmetic (bisection over binary32 scores),
// and each boundary carries a guard band that covers every score where the reference's binary32
// evaluation could disagree with the exact-math model: where |v(q) - n| <= m, v the model's value
// (pred +- err) in exact arithmetic, n the integer it crosses at the boundary and m a bound on the
// reference's rounding of v.  Outside the band the reference's level is the exact-math one, which
// is monotone, so the table decides it (lvt_screen, rkr_regression.cuh).
#include <cmath>

#include "rkr_internal.cuh"
#include "rkr_regression.cuh"

namespace rkr {

namespace {

// Order-preserving map of binary32 values (NaN excluded) onto int32 and back.
__device__ __forceinline__ int32_t f_key(float f) {
    const int32_t b = __float_as_int(f);
    return b >= 0 ? b : b ^ 0x7fffffff;
}
__device__ __forceinline__ float key_f(int32_t k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }

// The model's value v = a Phi(z) + b +- err in double, Phi the reference's approximation
// (Abramowitz & Stegun 7.1.26 with the reference's binary32 constants and sqrt(2), CDFPhi,
// NormalLinearRegressionLP.hpp:123-143) evaluated without its binary32 roundings.
__device__ __forceinline__ double model_value(double a, double b, double mu, double sigma, double err, bool upper,
                                              double q) {
    const double a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f;
    const double a4 = -1.453152027f, a5 = 1.061405429f, p = 0.3275911f;
    const double sqrt_2 = (double) __int_as_float(0x3fb504f3);
    const double z = (q - mu) / sigma;
    const double x = fabs(z) / sqrt_2;
    const double t = 1.0 / (1.0 + p * x);
    const double y = 1.0 - (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t * exp(-x * x);
    const double phi = 0.5 * (1.0 + (z < 0 ? -y : y));
    return a * phi + b + (upper ? -err : err);
}

// Bound on |v_reference - v| for any score in the model's range: the reference's CDFPhi differs
// from the formula without roundings by less than 5e-7 (binary32 polynomial, the argument's two
// roundings through the slope <= 0.25), and pred +- err takes three more roundings of values at
// most |a| + |b| + |err|; the bound below has three times that headroom.
__device__ __forceinline__ double model_margin(float a, float b, float err) {
    const double aa = fabs((double) a), s = aa + fabs((double) b) + fabs((double) err);
    return aa * 1.5e-6 + s * 6e-7 + 1e-6;
}

__global__ void level_table_kernel(const float *__restrict__ rec, int64_t n_user, int S, double err_cap,
                                   float2 *__restrict__ tab) {
    const int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_user * 2 * kLvEntries) return;
    const int64_t u = i / (2 * kLvEntries);
    const int side = (int) (i / kLvEntries) & 1, g = (int) (i % kLvEntries);
    const bool upper = side == 1;
    const float4 r0 = __ldg(reinterpret_cast<const float4 *>(rec + u * 8));
    const float4 r1 = __ldg(reinterpret_cast<const float4 *>(rec + u * 8 + 4));
    const float a = r0.x, b = r0.y, mu = r0.z, sigma = r0.w, err = r1.x, smax = r1.y, smin = r1.z;
    const bool capped = (double) err >= err_cap;
    const bool usable = isfinite(a) && isfinite(b) && isfinite(mu) && isfinite(sigma) && isfinite(err) &&
                        isfinite(smax) && isfinite(smin) && sigma > 0.0f && a < 0.0f && smin <= smax;
    float2 out;
    const int lim = lvt_level(g, S);  // the entry's level value
    if (!usable) {
        out = make_float2(NAN, NAN);
    } else if (g == kLvEntries - 1 || lim >= S + 1) {
        out = make_float2(-INFINITY, 0.0f);  // every level is <= lim
    } else {
        auto ok = [&](float q) { return regression_level_side(a, b, mu, sigma, err, smax, smin, capped, S, q, upper) <= lim; };
        if (!ok(INFINITY)) {
            out = make_float2(INFINITY, 0.0f);  // no score reaches a level <= lim
        } else if (ok(-INFINITY)) {
            out = make_float2(-INFINITY, 0.0f);
        } else {
            // smallest score with level <= lim: bisection on the order of binary32 values
            int64_t lo = f_key(-INFINITY), hi = f_key(INFINITY);  // ok(lo) false, ok(hi) true
            while (hi - lo > 1) {
                const int64_t mid = lo + ((hi - lo) >> 1);
                if (ok(key_f((int32_t) mid))) hi = mid;
                else lo = mid;
            }
            const float T = key_f((int32_t) hi);
            float band = 0.0f;
            if (!capped) {
                // the model's crossing: level <= lim  <=>  v <= lim - 1 (lower side, ceil) or
                // v < lim (upper side, floor); band around T covering the scores in [smin, smax]
                // where |v - n| <= m
                const double n = upper ? (double) lim : (double) (lim - 1);
                const double m = model_margin(a, b, err);
                auto v = [&](double q) { return model_value(a, b, mu, sigma, err, upper, q); };
                const double qa = smin, qb = smax;
                const double va = v(qa), vb = v(qb);  // v decreases with q (a < 0)
                if (!(va < n - m || vb > n + m)) {
                    // zone edges: v(zlo) = n + m, v(zhi) = n - m, clipped to [smin, smax]
                    double zlo = qa, zhi = qb;
                    if (va > n + m) {
                        double l = qa, h = qb;  // v(l) > n + m >= v(h)
                        for (int it = 0; it < 80 && h - l > 0.0; it++) {
                            const double mid = 0.5 * (l + h);
                            if (mid <= l || mid >= h) break;
                            if (v(mid) > n + m) l = mid;
                            else h = mid;
                        }
                        zlo = l;
                    }
                    if (vb < n - m) {
                        double l = qa, h = qb;  // v(l) >= n - m > v(h)
                        for (int it = 0; it < 80 && h - l > 0.0; it++) {
                            const double mid = 0.5 * (l + h);
                            if (mid <= l || mid >= h) break;
                            if (v(mid) >= n - m) l = mid;
                            else h = mid;
                        }
                        zhi = h;
                    }
                    const double w = fmax(fabs((double) T - zlo), fabs(zhi - (double) T));
                    band = __double2float_ru(w * (1.0 + 1e-6) + 1e-30);
                }
            }
            out = make_float2(T, band);
        }
    }
    tab[i] = out;
}

}  // namespace

// Builds the index's level tables for its regression records ([n_user][2][kLvEntries] float2).
int level_tables_build(rkr_index *ix) {
    const int64_t n = ix->n_user * 2 * kLvEntries;
    RKR_TRY(ix->lvt.ensure(sizeof(float2) * (size_t) n));
    const int S = ix->n_sample_reg;
    level_table_kernel<<<(unsigned) ((n + 127) / 128), 128, 0, ix->stream>>>(
        ix->reg.as<float>(), ix->n_user, S, (double) S - 1e-3, ix->lvt.as<float2>());
    RKR_CUDA(cudaGetLastError());
    return RKR_OK;
}

}  // namespace rkr

extern "C" int rkr_index_level_tables(rkr_index *ix, int32_t *levels_out, float *tables_out) {
    using namespace rkr;
    RKR_REQUIRE(ix && levels_out && tables_out, "null argument");
    if (ix->n_sample_reg <= 0 || !ix->lvt.p) {
        set_error("the index has no regression models");
        return RKR_ERR_STATE;
    }
    RKR_TRY(ensure_device(ix));
    for (int g = 0; g < kLvEntries; g++) levels_out[g] = lvt_level(g, ix->n_sample_reg);
    RKR_CUDA(cudaMemcpyAsync(tables_out, ix->lvt.p, sizeof(float2) * (size_t) ix->n_user * 2 * kLvEntries,
                             cudaMemcpyDeviceToHost, ix->stream));
    RKR_CUDA(cudaStreamSynchronize(ix->stream));
    return RKR_OK;
}
