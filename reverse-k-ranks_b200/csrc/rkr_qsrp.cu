// rkr_qsrp.cu -- QSRPNormalLP retrieval on the device (src/impl/QSRPNormalLP.hpp:116-260).
//
// Per query the reference runs two bound/prune rounds before refinement:
//   1. SVD-space partial score on the first check_dim coordinates +- the product of the remaining
//      norms (PartDimPartNorm::IPBound, PartDimPartNorm.hpp:52-74) -> regression rank bounds
//      (NormalLinearRegressionLP::ComputeRankBound, NormalLinearRegressionLP.hpp:326-398) -> prune.
//   2. full SVD-space score for the survivors (ComputeRemainDim, :76-95) -> sampled-threshold
//      bounds (SampleSearch::RankBound) -> prune again.
// Here each round is one pass over all (user, query) pairs of the batch.  The reference keeps its
// per-user score vector across queries; users accepted in round 1 are reported with whatever that
// vector holds for them.  The batch reproduces it: the score a user had at its latest earlier query
// in which it reached round 2, or the index's carried state when there is none.
#include <algorithm>
#include <vector>

#include "rkr_internal.cuh"

namespace rkr {

// launched from rkr_query.cu
int refine_and_assemble_qsrp(rkr_index *ix, const float *d_query, int nq, int topk, const QueryCounts *d_counts,
                             const int32_t *d_res_user, const int32_t *d_res_rank, const float *d_res_qip, int64_t n_cand,
                             int32_t *d_cand_user, int32_t *d_cand_query, int32_t *d_cand_lb, int32_t *d_cand_ub,
                             const float *d_cand_qip, const int64_t *d_cand_off, rkr_user_rank *d_out,
                             rkr_query_stats *d_stats, cudaStream_t st);

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

struct RegModel {           // device view of the regression index
    const float *rec;       // [n_user][8]
    const int32_t *rank;    // [S]
    int S;
    double err_cap;         // S - 1e-3
    int n_item;
};

// The same CDF with every step in binary32 and expf: within 1e-6 of cdf_phi for every input
// (the two differ only in where the last bits of t, the product and the closing sum are rounded).
__device__ __forceinline__ float cdf_phi_f32(float x) {
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f;
    const float a4 = -1.453152027f, a5 = 1.061405429f, p = 0.3275911f;
    const float sign = x < 0 ? -1.0f : 1.0f;
    x = __fdiv_rn(fabsf(x), __int_as_float(0x3fb504f3));
    const float t = __fdiv_rn(1.0f, __fadd_rn(1.0f, __fmul_rn(p, x)));
    const float pt = (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t;
    const float y = 1.0f - pt * expf(-x * x);
    return 0.5f * (1.0f + sign * y);
}

// The reference's float/double evaluation of one side of ComputeRankBound's index arithmetic
// (kept out of line: the float screen below rarely needs it).
__device__ __noinline__ int64_t regression_index_exact(float nx, float a, float b, float err, bool upper) {
    const float ix = cdf_phi(nx);
    const float pred = __fadd_rn(__fmul_rn(ix, a), b);
    return upper ? f2i64_x86(floorf(__fsub_rn(pred, err))) : f2i64_x86(ceilf(__fadd_rn(pred, err)));
}

// One side of ComputeRankBound's index arithmetic: pr = ceil(pred + err) (upper = 0) or
// floor(pred - err) (upper = 1), pred = cdf(nx) * a + b.  The float-only CDF decides it whenever
// pred -+ err lies farther from an integer than that CDF's error can move it (|a| * 4e-6 plus a
// few ulps of the sum); otherwise the reference's own float/double evaluation decides.
__device__ __forceinline__ int64_t regression_index(float nx, float a, float b, float err, bool upper) {
    const float ixf = cdf_phi_f32(nx);
    const float vf = upper ? __fsub_rn(__fadd_rn(__fmul_rn(ixf, a), b), err) : __fadd_rn(__fadd_rn(__fmul_rn(ixf, a), b), err);
    const float margin = fabsf(a) * 4e-6f + 8.0f * fabsf(vf) * 1.2e-7f + 1e-6f;
    const float r = rintf(vf);
    if (isfinite(vf) && fabsf(vf - r) > margin) return (int64_t) (upper ? floorf(vf) : ceilf(vf));
    return regression_index_exact(nx, a, b, err, upper);
}

// ComputeRankBound (:326-380), returning levels: 0 -> rank 0, j + 1 -> rank[j], S + 1 -> n_item.
// r0 = (a, b, mu, sigma), r1 = (err, smax, smin, -) is the user's model record.
__device__ __forceinline__ void regression_levels_rec(const RegModel &m, float4 r0, float4 r1, float qlb, float qub,
                                                      int &lvl_lb, int &lvl_ub) {
    const float a = r0.x, b = r0.y, mu = r0.z, sigma = r0.w, err = r1.x, smax = r1.y, smin = r1.z;
    const int S = m.S;
    if (qlb > smax) lvl_lb = 1;
    else if (qlb < smin) lvl_lb = S + 1;
    else if ((double) err >= m.err_cap) lvl_lb = S + 1;
    else {
        const int64_t pr = regression_index(__fdiv_rn(__fsub_rn(qlb, mu), sigma), a, b, err, false);
        lvl_lb = pr >= S ? S + 1 : (pr < 0 ? 1 : (int) pr + 1);
    }
    if (qub > smax) lvl_ub = 0;
    else if (qub < smin) lvl_ub = S;
    else if ((double) err >= m.err_cap) lvl_ub = 0;
    else {
        const int64_t pr = regression_index(__fdiv_rn(__fsub_rn(qub, mu), sigma), a, b, err, true);
        lvl_ub = pr >= S ? S + 1 : (pr < 0 ? 0 : (int) pr + 1);
    }
}

__device__ __forceinline__ void regression_levels(const RegModel &m, int64_t u, float qlb, float qub, int &lvl_lb,
                                                  int &lvl_ub) {
    regression_levels_rec(m, __ldg(reinterpret_cast<const float4 *>(m.rec + u * 8)),
                          __ldg(reinterpret_cast<const float4 *>(m.rec + u * 8 + 4)), qlb, qub, lvl_lb, lvl_ub);
}

__device__ __forceinline__ int level_rank(int lvl, const int32_t *rank, int S, int n_item) {
    return lvl == 0 ? 0 : (lvl > S ? n_item : rank[lvl - 1]);
}

// ---- kernels ---------------------------------------------------------------------------------------

constexpr uint16_t kStateResult1 = 0xfffe, kStatePruned1 = 0xffff;

struct QsrpParams {
    int32_t mode1, all1, L1, U1;         // round 1: equal-bounds mode, "all survivors accepted", k-th bounds
    int32_t n_res1, n_pr1, n_ref1, skip2; // round-1 counts; skip2: round 1 already produced top-k results
    int32_t mode2, all2, L2, U2;         // round 2
    int32_t n_elig2, pad0, pad1, pad2;
};

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

// Round 1 for every pair: left = InnerProduct(svd_user, qtr, check_dim) (kept for round 2);
// bounds left -+ norms; regression levels of both bounds packed as (lb | ub << 16).
__global__ void __launch_bounds__(kTileThreads) qsrp_round1_kernel(const float *__restrict__ svd_user, int64_t n_user,
                                                                  int dim, const float *__restrict__ unorm,
                                                                  const float *__restrict__ qtr,
                                                                  const float *__restrict__ qnorm, int n_query,
                                                                  int check_dim, RegModel m, uint32_t *__restrict__ lv,
                                                                  float *__restrict__ left) {
    __shared__ TileSmem sm;
    const int64_t b0 = (int64_t) blockIdx.x * kTile;
    const int64_t a0 = (int64_t) blockIdx.y * kTile;
    float lo[4][4], hi[4][4];
    exact_tile(sm, svd_user, nullptr, n_user, dim, a0, qtr, n_query, dim, b0, 0, check_dim, check_dim, lo, hi);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int64_t u = a0 + 4 * tx + i;
        if (u >= n_user) continue;
        const float un = __ldg(unorm + u);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t q = b0 + 4 * ty + j;
            if (q >= n_query) continue;
            const float right = __fmul_rn(un, __ldg(qnorm + q));
            int l, h;
            regression_levels(m, u, __fsub_rn(lo[i][j], right), __fadd_rn(lo[i][j], right), l, h);
            lv[q * n_user + u] = (uint32_t) l | ((uint32_t) h << 16);
            left[q * n_user + u] = lo[i][j];
        }
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
    for (int64_t u = u0 + threadIdx.x; u < u1; u += kHistThreads) {
        const uint32_t v = row[u];
        const int l = v & 0xffff, hh = v >> 16;
        atomicAdd(mine + l, 1);
        atomicAdd(mine + nl + hh, 1);
        my_anom += hh > l && level_rank(hh, rank, S, n_item) > level_rank(l, rank, S, n_item);
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

// Round 1 on 128 x 128 tiles (users x queries): left over the first check_dim coordinates, the
// bounds left -+ norms and their regression levels.
struct Round1Epi {
    static constexpr size_t kExtra = 0;
    const float *unorm, *qnorm;
    RegModel m;
    uint32_t *lv;
    float *left;
    int64_t n_user, n_query;
    __device__ void prologue(char *, int64_t, int64_t) const {}
    __device__ bool active(char *, int64_t, int64_t) const { return true; }
    __device__ void finish(char *, const BigResult &res, int64_t a0, int64_t b0, bool) const {
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7;
        const int64_t u = a0 + ra;
        if (u >= n_user) return;
        const float4 r0 = __ldg(reinterpret_cast<const float4 *>(m.rec + u * 8));
        const float4 r1 = __ldg(reinterpret_cast<const float4 *>(m.rec + u * 8 + 4));
        const float un = __ldg(unorm + u);
#pragma unroll 2
        for (int i = 0; i < kBig / 2; i++) {
            const int rb = half + 2 * i;
            const int64_t q = b0 + rb;
            if (q >= n_query) break;
            const float v = res.v[rb][ra];
            const float right = __fmul_rn(un, __ldg(qnorm + q));
            int l, h;
            regression_levels_rec(m, r0, r1, __fsub_rn(v, right), __fadd_rn(v, right), l, h);
            lv[q * n_user + u] = (uint32_t) l | ((uint32_t) h << 16);
            left[q * n_user + u] = v;
        }
    }
};

// Round-1 k-th smallest bounds per query (PruneCandidateByBound.hpp:36-77 with nothing excluded)
// and the class counts.  While every pair has ub <= lb, a result (lb <= U*) and a prune
// (ub >= L*) cannot coincide unless L* == U*, so the counts follow from the two histograms;
// otherwise qsrp_count1 counts pair by pair.
__global__ void qsrp_select1_kernel(const int *__restrict__ hist_all, const int *__restrict__ anomaly, int64_t n_user,
                                    const int32_t *__restrict__ rank, int S, int n_item, int topk, int nq,
                                    QsrpParams *__restrict__ par) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    const int nl = S + 2;
    const int *h = hist_all + (int64_t) q * 2 * nl;
    int kl = nl - 1, kh = nl - 1;
    int64_t c = 0;
    for (int b = 0; b < nl; b++) { c += h[b]; if (c >= topk) { kl = b; break; } }
    c = 0;
    for (int b = 0; b < nl; b++) { c += h[nl + b]; if (c >= topk) { kh = b; break; } }
    QsrpParams p = {};
    p.L1 = level_rank(kl, rank, S, n_item);
    p.U1 = level_rank(kh, rank, S, n_item);
    p.mode1 = p.L1 == p.U1;
    if (!p.mode1) {
        if (anomaly[q]) {
            p.pad0 = 1;  // exact counting needed
        } else {
            int64_t nres = 0, npr = 0;
            for (int b = 0; b < nl; b++) {
                if (level_rank(b, rank, S, n_item) <= p.U1) nres += h[b];
                if (level_rank(b, rank, S, n_item) >= p.L1) npr += h[nl + b];
            }
            p.n_res1 = (int) nres;
            p.n_pr1 = (int) npr;
            p.n_ref1 = (int) (n_user - nres - npr);
        }
    }
    par[q] = p;
}

__device__ __forceinline__ int class1_of(const QsrpParams &p, int lb, int ub) {
    if (p.mode1) return (ub <= p.L1 && lb <= p.L1) ? kClsResult : kClsIdle;
    if (lb <= p.U1) return kClsResult;
    if (p.L1 <= ub) return kClsPrune;
    return p.all1 ? kClsResult : kClsRefine;
}

// Round-1 class counts pair by pair (the reduction at PruneCandidateByBound.hpp:115-136), for
// queries where the histogram shortcut does not apply.
__global__ void qsrp_count1_kernel(const uint32_t *__restrict__ lv, int64_t n_user, const int32_t *__restrict__ rank,
                                   int S, int n_item, QsrpParams *__restrict__ par) {
    const int q = blockIdx.y;
    const QsrpParams p = par[q];
    if (p.mode1 || !p.pad0) return;
    __shared__ int cnt[3];
    if (threadIdx.x < 3) cnt[threadIdx.x] = 0;
    __syncthreads();
    int c[3] = {0, 0, 0};
    const uint32_t *row = lv + (int64_t) q * n_user;
    for (int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; u < n_user; u += (int64_t) gridDim.x * blockDim.x) {
        const uint32_t v = row[u];
        const int k = class1_of(p, level_rank(v & 0xffff, rank, S, n_item), level_rank(v >> 16, rank, S, n_item));
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

// Does the pair reach round 2 (neither pruned nor accepted in round 1)?
__device__ __forceinline__ bool eligible2(const QsrpParams &p, uint32_t v, const int32_t *rank, int S, int n_item) {
    const int k = class1_of(p, level_rank(v & 0xffff, rank, S, n_item), level_rank(v >> 16, rank, S, n_item));
    return k == kClsRefine || k == kClsIdle;
}

// Round 2: full SVD-space score of each surviving pair, left (round 1) + the remaining dims
// (ComputeRemainDim, PartDimPartNorm.hpp:76-95), and its sampled-threshold bucket.  Pairs that did
// not reach round 2 get a state code instead: kStateResult1 (accepted in round 1) or kStatePruned1.
__global__ void __launch_bounds__(kTileThreads, 3) qsrp_round2_kernel(const float *__restrict__ svd_user, int64_t n_user,
                                                                  int dim, const float *__restrict__ qtr, int n_query,
                                                                  int check_dim, const uint32_t *__restrict__ lv,
                                                                  const float *__restrict__ left,
                                                                  const QsrpParams *__restrict__ par,
                                                                  const int32_t *reg_rank, int S_reg,
                                                                  int n_item, const float *__restrict__ thr, int S,
                                                                  uint16_t *__restrict__ bucket2) {
    __shared__ TileSmem sm;
    __shared__ ThrSummary ts;
    __shared__ QsrpParams par_s[kTile];
    extern __shared__ int32_t rank_s[];  // the regression model's sample ranks
    const int64_t b0 = (int64_t) blockIdx.x * kTile;
    const int64_t a0 = (int64_t) blockIdx.y * kTile;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    if (threadIdx.x < kTile && b0 + threadIdx.x < n_query) par_s[threadIdx.x] = par[b0 + threadIdx.x];
    for (int i = threadIdx.x; i < S_reg; i += blockDim.x) rank_s[i] = reg_rank[i];
    __syncthreads();
    reg_rank = rank_s;
    uint32_t el = 0, r1 = 0;  // bit 4*i + j: reached round 2 / accepted in round 1
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t u = a0 + 4 * tx + i, q = b0 + 4 * ty + j;
            if (u < n_user && q < n_query) {
                const uint32_t v = lv[q * n_user + u];
                const int k = class1_of(par_s[4 * ty + j], level_rank(v & 0xffff, reg_rank, S_reg, n_item),
                                        level_rank(v >> 16, reg_rank, S_reg, n_item));
                if (k == kClsRefine || k == kClsIdle) el |= 1u << (4 * i + j);
                else if (k == kClsResult) r1 |= 1u << (4 * i + j);
            }
        }
    const bool any = __syncthreads_or(el != 0);
    float lo[4][4], hi[4][4];
    if (any) {
        load_thr_summary(ts, thr, n_user, a0, S);
        exact_tile(sm, svd_user, nullptr, n_user, dim, a0, qtr, n_query, dim, b0, check_dim, dim, dim, lo, hi);
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int64_t u = a0 + 4 * tx + i;
        if (u >= n_user) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t q = b0 + 4 * ty + j;
            if (q >= n_query) continue;
            uint16_t b = (r1 >> (4 * i + j) & 1) ? kStateResult1 : kStatePruned1;
            if (el >> (4 * i + j) & 1) {
                const float qip = __fadd_rn(left[q * n_user + u], lo[i][j]);
                b = (uint16_t) bucket_of_2level(ts.v[4 * tx + i], thr + u * S, S, qip);
            }
            bucket2[q * n_user + u] = b;
        }
    }
}

// Round 2 on 128 x 128 tiles: pairs that reached round 2 get left + the remaining coordinates and
// their sampled-threshold bucket; the others their round-1 state code.  Tiles without a surviving
// pair skip the dot products.
struct Round2Epi {
    static constexpr int kMaxRank = 1024;
    static constexpr size_t kExtra = sizeof(float) * kBig * ThrSummary::kMaxGroups + sizeof(QsrpParams) * kBig +
                                     sizeof(int32_t) * kMaxRank;
    const uint32_t *lv;
    const float *left;
    const QsrpParams *par;
    const int32_t *reg_rank;
    int S_reg, n_item;
    const float *thr;
    int S;
    int64_t n_user;
    int n_query;
    uint16_t *bucket2;
    __device__ float *summ(char *x) const { return reinterpret_cast<float *>(x); }
    __device__ QsrpParams *pars(char *x) const {
        return reinterpret_cast<QsrpParams *>(x + sizeof(float) * kBig * ThrSummary::kMaxGroups);
    }
    __device__ const int32_t *ranks(char *x) const {
        return S_reg <= kMaxRank ? reinterpret_cast<const int32_t *>(x + sizeof(float) * kBig * ThrSummary::kMaxGroups +
                                                                    sizeof(QsrpParams) * kBig)
                                 : reg_rank;
    }
    __device__ int klass(char *x, int64_t u, int64_t q, int rb) const {
        const uint32_t v = lv[q * n_user + u];
        const int32_t *rk = ranks(x);
        return class1_of(pars(x)[rb], level_rank(v & 0xffff, rk, S_reg, n_item), level_rank(v >> 16, rk, S_reg, n_item));
    }
    __device__ void prologue(char *x, int64_t a0, int64_t b0) const {
        if (threadIdx.x < kBig && b0 + threadIdx.x < n_query) pars(x)[threadIdx.x] = par[b0 + threadIdx.x];
        if (S_reg <= kMaxRank) {
            int32_t *rk = reinterpret_cast<int32_t *>(x + sizeof(float) * kBig * ThrSummary::kMaxGroups +
                                                      sizeof(QsrpParams) * kBig);
            for (int i = threadIdx.x; i < S_reg; i += blockDim.x) rk[i] = reg_rank[i];
        }
        load_thr_summary_rows(summ(x), kBig, thr, n_user, a0, S);
    }
    __device__ bool active(char *x, int64_t a0, int64_t b0) const {
        bool any = false;
        for (int idx = threadIdx.x; idx < kBig * kBig && !any; idx += kBigThreads) {
            const int rb = idx / kBig, ra = idx % kBig;
            const int64_t u = a0 + ra, q = b0 + rb;
            if (u < n_user && q < n_query) {
                const int k = klass(x, u, q, rb);
                any = k == kClsRefine || k == kClsIdle;
            }
        }
        return __syncthreads_or(any);
    }
    __device__ void finish(char *x, const BigResult &res, int64_t a0, int64_t b0, bool live) const {
        const int ra = threadIdx.x & (kBig - 1), half = threadIdx.x >> 7;
        const int64_t u = a0 + ra;
        if (u >= n_user) return;
        const float *sm = summ(x) + ra * ThrSummary::kMaxGroups;
        const float *row = thr + u * S;
        const int32_t *rk = ranks(x);
        const QsrpParams *ps = pars(x);
        constexpr int G = 8;
        for (int i0 = 0; i0 < kBig / 2; i0 += G) {
            uint32_t v[G];
            float lf[G];
#pragma unroll
            for (int g = 0; g < G; g++) {
                const int64_t q = b0 + half + 2 * (i0 + g);
                v[g] = q < n_query ? lv[q * n_user + u] : 0u;
                lf[g] = q < n_query ? left[q * n_user + u] : 0.0f;
            }
#pragma unroll
            for (int g = 0; g < G; g++) {
                const int rb = half + 2 * (i0 + g);
                const int64_t q = b0 + rb;
                if (q >= n_query) break;
                const int k = class1_of(ps[rb], level_rank(v[g] & 0xffff, rk, S_reg, n_item),
                                        level_rank(v[g] >> 16, rk, S_reg, n_item));
                uint16_t b;
                if (k == kClsRefine || k == kClsIdle) {
                    b = (uint16_t) bucket_of_2level(sm, row, S, __fadd_rn(lf[g], live ? res.v[rb][ra] : 0.0f));
                } else {
                    b = k == kClsResult ? kStateResult1 : kStatePruned1;
                }
                bucket2[q * n_user + u] = b;
            }
        }
    }
};

// Round-2 pruning per query (second PruneCandidateByBound call, QSRPNormalLP.hpp:187-190): users
// excluded in round 1 are skipped by the heap scan and the classification; the equal-bounds rule
// looks at every user's current bounds.
__global__ void qsrp_select2_kernel(const int *__restrict__ hist_all, int S, const int32_t *__restrict__ rank,
                                    int n_item, int topk, int nq, QsrpParams *__restrict__ par,
                                    uint8_t *__restrict__ cls2, QueryCounts *__restrict__ counts) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    QsrpParams p = par[q];
    uint8_t *cq = cls2 + (int64_t) q * (S + 1);
    if (p.skip2) {
        QueryCounts c = {};
        c.n_result = p.n_res1;
        c.n_prune = p.n_pr1;
        c.n_cand = 0;
        c.mode = 2;
        c.ip_base = p.n_ref1;
        counts[q] = c;
        return;
    }
    const int *hist = hist_all + (int64_t) q * (S + 1);
    const int kp = topk - p.n_res1;
    int64_t n_el = 0;
    for (int b = 0; b <= S; b++) n_el += hist[b];
    int L, U;
    if (n_el < kp) {  // the reference's zero-filled heap: max(bounds of eligible users, 0)
        int bmax = -1;
        for (int b = S; b >= 0; b--) if (hist[b]) { bmax = b; break; }
        L = 0; U = 0;
        if (bmax >= 0) {
            int lb, ub;
            bucket_bounds(bmax, S, rank, n_item, lb, ub);
            L = max(lb, 0); U = max(ub, 0);
        }
    } else {
        int bk = S;
        int64_t c = 0;
        for (int b = 0; b <= S; b++) { c += hist[b]; if (c >= kp) { bk = b; break; } }
        bucket_bounds(bk, S, rank, n_item, L, U);
    }
    p.L2 = L; p.U2 = U; p.n_elig2 = (int) n_el;
    QueryCounts c = {};
    c.lstar = L; c.ustar = U;
    c.ip_base = p.n_ref1;  // QSRPNormalLP.hpp:177: refine_user_size after the first prune
    if (L == U) {
        p.mode2 = 1;
        c.mode = 1;
        c.n_result = topk;
        c.n_prune = p.n_pr1;
        c.n_cand = 0;
        for (int b = 0; b <= S; b++) cq[b] = kClsIdle;
    } else {
        int64_t nres = p.n_res1, npr = p.n_pr1, nref = 0;
        for (int b = 0; b <= S; b++) {
            int lb, ub;
            bucket_bounds(b, S, rank, n_item, lb, ub);
            uint8_t k;
            if (lb <= U) { k = kClsResult; nres += hist[b]; }
            else if (L <= ub) { k = kClsPrune; npr += hist[b]; }
            else { k = kClsRefine; nref += hist[b]; }
            cq[b] = k;
        }
        if (nres + nref == topk) {
            for (int b = 0; b <= S; b++) if (cq[b] == kClsRefine) cq[b] = kClsResult;
            p.all2 = 1;
            nres = topk; nref = 0;
        }
        c.mode = 0;
        c.n_result = (int) nres;
        c.n_prune = (int) npr;
        c.n_cand = nres >= topk ? 0 : (int) nref;
    }
    par[q] = p;
    counts[q] = c;
}

// Classification of a pair after both rounds for the ordered compaction: result users carry their
// reported rank (the lower bound in force) and whether their score is this query's; candidates
// carry their round-2 bounds.
struct QsrpCompactPolicy {
    struct Aux { int rank, fresh, lb, ub; };
    const uint32_t *lv;
    const uint16_t *b2;
    int64_t n_user;
    const int32_t *reg_rank, *rank;
    int S_reg, S, n_item;
    const QsrpParams *par;
    const uint8_t *cls2;
    const QueryCounts *counts;
    const int64_t *cand_off;
    int topk;
    int32_t *res_user, *res_rank;
    uint8_t *res_fresh;
    int32_t *cand_user, *cand_query, *cand_lb, *cand_ub;
    __device__ bool query_active(int q) const { return true; }
    __device__ int classify(int q, int64_t u, Aux &aux) const {
        const QsrpParams &p = par[q];
        const uint16_t code = b2[(int64_t) q * n_user + u];
        if (code <= S) {  // reached round 2
            int lb, ub;
            bucket_bounds(code, S, rank, n_item, lb, ub);
            aux.rank = lb; aux.fresh = 1; aux.lb = lb; aux.ub = ub;
            if (p.skip2) return 0;
            if (p.mode2) return (ub <= p.L2 && lb <= p.L2) ? 1 : 0;
            const uint8_t k2 = __ldg(cls2 + (int64_t) q * (S + 1) + code);
            if (k2 == kClsResult) return 1;
            return (k2 == kClsRefine && counts[q].n_cand > 0) ? 2 : 0;
        }
        aux.fresh = 0;
        if (code == kStateResult1 || (!p.skip2 && p.mode2)) {
            const uint32_t v = lv[(int64_t) q * n_user + u];
            const int lb1 = level_rank(v & 0xffff, reg_rank, S_reg, n_item);
            const int ub1 = level_rank(v >> 16, reg_rank, S_reg, n_item);
            aux.rank = lb1; aux.lb = lb1; aux.ub = ub1;
            if (code == kStateResult1) return 1;
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

// Exact SVD-space score of (query, user): checkdim part + remaining part (PartDimPartNorm.hpp:62, 89-92).
__device__ __forceinline__ float qsrp_score(const float *svd_user, const float *qtr, int64_t u, int q, int dim, int c) {
    const float *uv = svd_user + u * dim;
    const float *qv = qtr + (int64_t) q * dim;
    return __fadd_rn(exact_dot(uv, qv, c), exact_dot(uv + c, qv + c, dim - c));
}

// Scores of the emitted result users: this query's score when the user reached round 2, else the
// score from its latest earlier round-2 query in the batch, else the carried state.
__global__ void qsrp_result_fill_kernel(const QueryCounts *__restrict__ counts, const int32_t *__restrict__ res_user,
                                        const uint8_t *__restrict__ res_fresh, const uint16_t *__restrict__ bucket2,
                                        int64_t n_user, const float *__restrict__ svd_user, const float *__restrict__ qtr,
                                        int dim, int check_dim, const float *__restrict__ state, int topk,
                                        float *__restrict__ res_qip) {
    const int q = blockIdx.x;
    const int n = counts[q].n_res_emit;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        const int64_t i = (int64_t) q * topk + k;
        const int u = res_user[i];
        int src = res_fresh[i] ? q : -1;
        for (int qq = q - 1; src < 0 && qq >= 0; qq--)
            if (bucket2[(int64_t) qq * n_user + u] < kStateResult1) src = qq;
        res_qip[i] = src >= 0 ? qsrp_score(svd_user, qtr, u, src, dim, check_dim) : state[u];
    }
}

__global__ void qsrp_cand_fill_kernel(const int32_t *__restrict__ cand_user, const int32_t *__restrict__ cand_query,
                                      int64_t n, const float *__restrict__ svd_user, const float *__restrict__ qtr, int dim,
                                      int check_dim, float *__restrict__ cand_qip) {
    const int64_t e = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    cand_qip[e] = qsrp_score(svd_user, qtr, cand_user[e], cand_query[e], dim, check_dim);
}

// Carried state after the batch: each user's score at its last round-2 query of the batch.
__global__ void qsrp_state_kernel(const uint16_t *__restrict__ bucket2, int64_t n_user, int nq,
                                  const float *__restrict__ svd_user, const float *__restrict__ qtr, int dim, int check_dim,
                                  float *__restrict__ state) {
    const int64_t u = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= n_user) return;
    for (int q = nq - 1; q >= 0; q--)
        if (bucket2[(int64_t) q * n_user + u] < kStateResult1) {
            state[u] = qsrp_score(svd_user, qtr, u, q, dim, check_dim);
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

int qsrp_chunk(rkr_index *ix, const float *d_query, int nq, int topk, rkr_user_rank *d_out, rkr_query_stats *d_stats,
               cudaStream_t st) {
    const int64_t U = ix->n_user;
    const int dim = ix->dim, c = ix->check_dim, S = ix->n_sample, Sr = ix->n_sample_reg;
    const int n_item = (int) ix->n_item;
    const int nl = Sr + 2;
    RKR_TRY(ix->ws_qtr.ensure(carve_size((size_t) nq * dim, 4) + carve_size(nq, 4) + carve_size(nq, sizeof(QsrpParams)) +
                              carve_size(nq, 4)));
    uint8_t *p0 = ix->ws_qtr.as<uint8_t>();
    float *qtr = carve<float>(p0, (size_t) nq * dim);
    float *qnorm = carve<float>(p0, nq);
    QsrpParams *par = carve<QsrpParams>(p0, nq);
    int *anomaly = carve<int>(p0, nq);
    RKR_TRY(ix->ws_levels.ensure((size_t) nq * U * 8));
    RKR_TRY(ix->ws_bucket2.ensure((size_t) nq * U * 2));
    RKR_TRY(ix->ws_cls.ensure((size_t) nq * (S + 1)));
    RKR_TRY(ix->ws_counts.ensure(sizeof(QueryCounts) * (size_t) nq));
    RKR_TRY(ix->ws_hist.ensure(sizeof(int) * (size_t) nq * std::max(2 * nl, S + 1)));
    uint32_t *lv = ix->ws_levels.as<uint32_t>();
    float *left = reinterpret_cast<float *>(lv + (size_t) nq * U);
    uint16_t *b2 = ix->ws_bucket2.as<uint16_t>();
    QueryCounts *counts = ix->ws_counts.as<QueryCounts>();
    int *hist = ix->ws_hist.as<int>();
    RKR_CUDA(cudaMemsetAsync(anomaly, 0, sizeof(int) * nq, st));

    timed(ix, st, "transfer_query", [&] {
        transfer_query_kernel<<<nq, 128, 0, st>>>(d_query, ix->transfer_item.as<float>(), dim, c, qtr, qnorm);
    });
    RKR_CUDA(cudaGetLastError());
    RegModel m;
    m.rec = ix->reg.as<float>();
    m.rank = ix->reg_rank.as<int32_t>();
    m.S = Sr;
    m.err_cap = (double) Sr - 1e-3;
    m.n_item = n_item;
    Round1Epi e1;
    e1.unorm = ix->svd_unorm.as<float>();
    e1.qnorm = qnorm;
    e1.m = m;
    e1.lv = lv;
    e1.left = left;
    e1.n_user = U;
    e1.n_query = nq;
    cudaError_t ce = cudaSuccess;
    timed(ix, st, "qsrp_round1", [&] { ce = launch_big(ix->svd_user.as<float>(), nullptr, U, dim, qtr, nq, dim, 0, c, e1, st); });
    RKR_CUDA(ce);
    const int64_t chunk = 16384;
    dim3 hg((unsigned) ((U + chunk - 1) / chunk), (unsigned) nq);
    RKR_CUDA(cudaMemsetAsync(hist, 0, sizeof(int) * (size_t) nq * 2 * nl, st));
    timed(ix, st, "level_hist", [&] {
        level_hist_kernel<<<hg, kHistThreads, hist_copies(2 * nl) * 2 * nl * sizeof(int), st>>>(lv, U, m.rank, Sr, n_item,
                                                                                               chunk, hist, anomaly);
    });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_select1", [&] {
        qsrp_select1_kernel<<<(nq + 127) / 128, 128, 0, st>>>(hist, anomaly, U, m.rank, Sr, n_item, topk, nq, par);
    });
    RKR_CUDA(cudaGetLastError());
    {
        dim3 g((unsigned) std::min<int64_t>((U + 1023) / 1024, 64), (unsigned) nq);
        timed(ix, st, "qsrp_count1", [&] { qsrp_count1_kernel<<<g, 256, 0, st>>>(lv, U, m.rank, Sr, n_item, par); });
        RKR_CUDA(cudaGetLastError());
    }
    timed(ix, st, "qsrp_final1", [&] { qsrp_final1_kernel<<<(nq + 127) / 128, 128, 0, st>>>(par, nq, topk); });
    RKR_CUDA(cudaGetLastError());
    Round2Epi e2;
    e2.lv = lv;
    e2.left = left;
    e2.par = par;
    e2.reg_rank = m.rank;
    e2.S_reg = Sr;
    e2.n_item = n_item;
    e2.thr = ix->thr.as<float>();
    e2.S = S;
    e2.n_user = U;
    e2.n_query = nq;
    e2.bucket2 = b2;
    timed(ix, st, "qsrp_round2", [&] { ce = launch_big(ix->svd_user.as<float>(), nullptr, U, dim, qtr, nq, dim, c, dim, e2, st); });
    RKR_CUDA(ce);
    RKR_CUDA(cudaMemsetAsync(hist, 0, sizeof(int) * (size_t) nq * (S + 1), st));
    timed(ix, st, "bucket_hist", [&] {
        bucket_hist_kernel<<<hg, kHistThreads, hist_copies(S + 1) * (S + 1) * sizeof(int), st>>>(b2, U, S + 1, chunk, hist);
    });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_select2", [&] {
        qsrp_select2_kernel<<<(nq + 127) / 128, 128, 0, st>>>(hist, S, ix->sample_rank.as<int32_t>(), n_item, topk, nq,
                                                             par, ix->ws_cls.as<uint8_t>(), counts);
    });
    RKR_CUDA(cudaGetLastError());

    std::vector<QueryCounts> hc(nq);
    RKR_CUDA(cudaMemcpyAsync(hc.data(), counts, sizeof(QueryCounts) * nq, cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
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
    pol.b2 = b2;
    pol.n_user = U;
    pol.reg_rank = m.rank;
    pol.rank = ix->sample_rank.as<int32_t>();
    pol.S_reg = Sr;
    pol.S = S;
    pol.n_item = n_item;
    pol.par = par;
    pol.cls2 = ix->ws_cls.as<uint8_t>();
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
        qsrp_result_fill_kernel<<<nq, 128, 0, st>>>(counts, res_user, res_fresh, b2, U, ix->svd_user.as<float>(), qtr,
                                                    dim, c, ix->qip_state.as<float>(), topk, res_qip);
    });
    RKR_CUDA(cudaGetLastError());
    if (n_cand > 0) {
        timed(ix, st, "qsrp_cand_fill", [&] {
            qsrp_cand_fill_kernel<<<(unsigned) ((n_cand + 255) / 256), 256, 0, st>>>(
                cand_user, cand_query, n_cand, ix->svd_user.as<float>(), qtr, dim, c, cand_qip);
        });
        RKR_CUDA(cudaGetLastError());
    }
    RKR_TRY(refine_and_assemble_qsrp(ix, d_query, nq, topk, counts, res_user, res_rank, res_qip, n_cand, cand_user,
                                     cand_query, cand_lb, cand_ub, cand_qip, d_off, d_out, d_stats, st));
    timed(ix, st, "qsrp_state", [&] {
        qsrp_state_kernel<<<(unsigned) ((U + 255) / 256), 256, 0, st>>>(b2, U, nq, ix->svd_user.as<float>(), qtr, dim,
                                                                        c, ix->qip_state.as<float>());
    });
    RKR_CUDA(cudaGetLastError());
    RKR_CUDA(cudaStreamSynchronize(st));
    return RKR_OK;
}

}  // namespace rkr
