// rkr_query.cu -- batched reverse k-ranks retrieval on the device (QS, QSRPNormalLP, US): the
// refinement of candidates and the assembly of results, and the batch driver.
//
// A batch of queries runs as a short pipeline of kernels; every (query, user) decision the
// reference makes one query at a time (src/impl/QS.hpp:127-224, src/impl/QSRPNormalLP.hpp:137-253,
// src/impl/US.hpp:117-201) is made for the whole batch at once.  The bound and prune stages are in
// rkr_qsrp.cu (QS and US are its second round on its own); here:
//
//   refine_prep       candidates: score, norm cut-off, rank when the bounds already agree
//   refine_tc         candidates x items: the reference's per-item test on tensor-core scores with
//                     exact resolution of undecided pairs (rkr_refine_tc.cu); refine_tile, the
//                     exact SIMT tiles, where that path does not apply
//   assemble          per query: results in user-id order, then candidates by (rank, user id)
#include <algorithm>
#include <cstring>
#include <numeric>

#include "rkr_internal.cuh"

namespace rkr {

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
    KSpec ks;                    // per-query k; ks.kmax is the result arrays' row stride
    const int64_t *out_off;      // [n_query] start of each query's output, or nullptr: q * k
    int ipbound, dim, check_dim;
    rkr_user_rank *out;          // k entries per query
    rkr_query_stats *stats;      // [n_query] or nullptr
    int64_t id_offset;           // added to the user ids written (a user shard's first user)
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
    __shared__ int n_refined;
    __shared__ int64_t n_items, ip_refine;
    __shared__ uint64_t thresh;
    const int q = blockIdx.x;
    const QueryCounts c = a.counts[q];
    const int topk = a.ks.of(q);
    rkr_user_rank *out = a.out + (a.out_off ? a.out_off[q] : (int64_t) q * topk);
    const int nres = c.n_res_emit;
    for (int k = threadIdx.x; k < nres; k += blockDim.x) {
        const int64_t i = (int64_t) q * a.ks.kmax + k;
        out[k].user_id = (int32_t) (a.res_user[i] + a.id_offset);
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
                out[nres + lo].user_id = (int32_t) (a.cand_user[off + e] + a.id_offset);
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
static int refine_and_assemble(rkr_index *ix, int method, const float *d_query, int nq, KSpec ks,
                               const int64_t *d_out_off, const QueryCounts *d_counts, const std::vector<QueryCounts> &h_counts,
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
    aa.ks = ks;
    aa.out_off = d_out_off;
    aa.out = d_out;
    aa.stats = d_stats;
    aa.scratch = nullptr;
    aa.id_offset = ix->shard.user_offset;
    timed(ix, st, "assemble", [&] { assemble_kernel<<<nq, 256, 0, st>>>(aa); });
    RKR_CUDA(cudaGetLastError());
    (void) h_counts;
    return RKR_OK;
}

// One chunk of queries, every method (rkr_qsrp.cu).
int pair_chunk(rkr_index *ix, int method, const float *d_query, int nq, const BatchSpec &bs, rkr_user_rank *d_out,
               rkr_query_stats *d_stats, cudaStream_t st);

int refine_and_assemble_pairs(rkr_index *ix, int method, const float *d_query, int nq, KSpec ks,
                              const int64_t *d_out_off, const QueryCounts *d_counts, const int32_t *d_res_user, const int32_t *d_res_rank,
                              const float *d_res_qip, int64_t n_cand, int32_t *d_cand_user, int32_t *d_cand_query,
                              int32_t *d_cand_lb, int32_t *d_cand_ub, const float *d_cand_qip,
                              const int64_t *d_cand_off, rkr_user_rank *d_out, rkr_query_stats *d_stats,
                              cudaStream_t st) {
    std::vector<QueryCounts> unused;
    return refine_and_assemble(ix, method, d_query, nq, ks, d_out_off, d_counts, unused, d_res_user, d_res_rank,
                               d_res_qip, n_cand,
                               d_cand_user, d_cand_query, d_cand_lb, d_cand_ub, d_cand_qip, d_cand_off, d_out, d_stats,
                               st);
}

int query_batch(rkr_index *ix, int method, const float *d_query, int n_query, const BatchSpec &bs,
                rkr_user_rank *d_out, rkr_query_stats *d_stats, cudaStream_t st) {
    // Chunk so the per-pair arrays (coarse levels and group codes: 2 bytes a pair) stay within a
    // bounded slice of device memory.
    const int64_t budget = int64_t(8) << 30;
    // (user shards chunk alike: their counts are summed chunk by chunk)
    const int64_t per_q = ix->n_user_all() * 2 + 4096;
    int chunk = (int) std::max<int64_t>(1, std::min<int64_t>(n_query, budget / per_q));
    chunk = std::min(chunk, kMaxChunkQueries);
    int64_t out_at = 0;
    for (int q0 = 0; q0 < n_query; q0 += chunk) {
        const int nq = std::min(chunk, n_query - q0);
        BatchSpec part = bs;
        std::vector<int32_t> first;
        if (bs.k) part.k = bs.k + q0;
        if (bs.front) part.front = bs.front + q0;
        if (bs.req_first) {
            // a request that started in an earlier chunk continues from this chunk's first query
            first.resize(nq);
            for (int q = 0; q < nq; q++) first[q] = std::max(bs.req_first[q0 + q] - q0, 0);
            part.req_first = first.data();
        }
        const float *dq = d_query + (int64_t) q0 * ix->dim;
        rkr_query_stats *dst = d_stats ? d_stats + q0 : nullptr;
        RKR_TRY(pair_chunk(ix, method, dq, nq, part, d_out + out_at, dst, st));
        if (bs.k) for (int q = 0; q < nq; q++) out_at += bs.k[q0 + q];
        else out_at += (int64_t) nq * bs.topk;
    }
    return RKR_OK;
}

}  // namespace rkr
