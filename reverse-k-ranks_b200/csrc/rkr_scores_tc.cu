// rkr_scores_tc.cu -- the (query, user) scores of the bound rounds on the tensor cores (tcgen05, int8).
//
// The bound rounds only ask, per (query, user) pair, which regression level its partial score falls
// on (QSRPNormalLP round 1: NormalLinearRegressionLP::ComputeRankBound on the bounds of
// PartDimPartNorm::IPBound, PartDimPartNorm.hpp:52-74) and which coarse group of sampled thresholds
// its full score falls in (SampleSearch::RankBound, SampleSearch.hpp:91-156; QS.hpp:137-143 for QS
// and US).  Both are decided from a tensor-core score with a rigorous bound on its distance to the
// reference's binary32 score; pairs whose bound interval reaches a decision boundary are recomputed
// with the reference's own arithmetic inside the same kernel.
//
// Scores.  Each row (user or query) is scaled by a power of two 2^e with every |coordinate| < 2^(e-1)
// and split into four signed 7-bit digits per coordinate, a = 2^e (d1 2^-7 + d2 2^-14 + d3 2^-21 +
// d4 2^-28 + r), |d| <= 64, |r| <= 2^-29 (each digit is the nearest integer of the remainder times
// 128, all steps exact in binary32).  The ten digit products with i + j <= 5 run as int8 MMAs
// (tcgen05.mma kind::i8) into four int32 TMEM accumulators per part (grouped by i + j); integer
// accumulation is exact.  Per part P of n coordinates the computed value differs from the exact
// dot product by at most 2^(ea+eb) n (3.02 2^-30 + 2^-29 + 1.1e-4 2^-24) + 3.002 2^-24 |value|
// (dropped digit products, the remainders, and the three roundings that combine the accumulators),
// and the reference's sequential binary32 sum differs from the exact one by at most about 2^-24
// Wa Wb, W the rows' position-weighted norms (part_coef).
//
// Tiles.  One CTA per 128 users (the MMA's M and the TMEM lanes) holds the users' digits for the
// whole K extent in shared memory and walks the batch's queries in chunks of 32 (the MMA's N), the
// query digits double-buffered by bulk copies and the accumulators double-buffered in TMEM (2 x 8
// accumulators x 32 columns = 512 columns), so that the MMAs of one chunk overlap the epilogue of
// the previous one.  A chunk's four query digit slices follow each other as row groups, so that per
// user slice i and K step one MMA of N = 32 (4 - i) covers the query slices 0 .. 3 - i and fills the
// digit-group accumulators i .. 3 (umma_i8_step: 4 MMAs per K step instead of one per digit pair;
// these small MMAs are bound by their shared-memory operand traffic, which falls by 1.9x).  Warp 16
// runs the copies and the MMAs (one
// elected lane issues); warps 0-15 read TMEM (warp w: lane quadrant w % 4, columns 8 (w / 4) .. + 8
// of each accumulator) and run the epilogue.
#include <cmath>
#include <cstdio>
#include <vector>

#include "rkr_internal.cuh"
#include "rkr_regression.cuh"
#include "rkr_tc_common.cuh"

namespace rkr {

namespace {

constexpr int kScEpiWarps = 16;
constexpr int kScThreads = 32 * (kScEpiWarps + 1);
constexpr int kScListCap = 1024;                   // undecided pairs per CTA resolved in the kernel
constexpr int kScMaxQ = 1024;                      // queries per launch (their data sits in shared memory)
constexpr int kScMaxKp = 224;                      // padded coordinates (both parts): shared memory
constexpr int kUpCache = 10;  // upper-side lower limits held in registers
static_assert(kUpCache % 2 == 0 && kUpCache < kLvEntries - 1, "paired terms; the verification index stays a table entry");
constexpr int kScSummStride = kScM;  // summary transposed: entry j of row r at j * kScM + r (lanes hit distinct banks)

// ---- the tile kernel -----------------------------------------------------------------------------------

struct ScArgs {
    const int8_t *a_sl, *b_sl;     // user tiles (kScM rows), query chunks (kScN rows)
    const float4 *umeta, *qmeta;
    const float *unorm, *qnorm;    // the reference's remaining-coordinate norms (QSRP)
    const float *urow, *qrow;      // exact rows: [n_user][dim], [nq][dim]
    const float *thr_summ;
    RegModel m;
    const float2 *lvt;             // [n_user][2][kLvEntries] level tables; nullptr: no regression round (QS, US)
    uint8_t *lvc;                  // [query][n_user]: coarse lower-bound level | coarse upper-bound level << 4
    uint8_t *code;                 // [query][n_user]: coarse threshold group of the full score
    int *anomaly;                  // [query]: pairs whose upper-bound rank exceeds their lower-bound rank
    float2 *dump;                  // [query][n_user] (estimate of the full score, its bound), or nullptr
    int2 *ovf;                     // undecided pairs, (query, user): each tile's list in one piece
    int *ovf_count, *status, *undecided;
    int *searches;                 // [2]: warp passes that ran the lower / upper side's table search
    int ovf_cap;
    int2 *tile_rng;                // per tile of the launch: (first entry, entries) in ovf
    int2 *spill;                   // undecided pairs past a tile's shared-memory list
    int *spill_count;
    int spill_cap;
    int q_base;                    // the launch's first query in the batch (overflow entries hold batch queries)
    int64_t n_user;
    int nq, dim, c, kp, ksplit, ksteps, two_parts, nb;
    float cl, kl, cr, kr;          // bound coefficients of the two parts
};

// The reference's scores and decisions for one pair: levels, group code and score stored.
// exact_dot with the first operand in shared or global memory (generic loads; __ldg would not
// accept a shared-memory address).
__device__ __forceinline__ float exact_dot_any(const float *a, const float *__restrict__ b, int n) {
    for (int o = 0; o < n; o += 32) prefetch_l1(b + o);  // the second row's lines, requested up front
    if (n > 0) prefetch_l1(b + n - 1);
    float acc = 0.0f;
    int j = 0;
    if (((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 7) == 0) {
        for (; j + 32 <= n; j += 32) {  // 8-byte loads, 32 coordinates ahead of their (ordered) sum
            float2 x[16], y[16];
#pragma unroll
            for (int t = 0; t < 16; t++) {
                x[t] = reinterpret_cast<const float2 *>(a + j)[t];
                y[t] = __ldg(reinterpret_cast<const float2 *>(b + j) + t);
            }
#pragma unroll
            for (int t = 0; t < 16; t++) {
                acc = __fadd_rn(acc, __fmul_rn(x[t].x, y[t].x));
                acc = __fadd_rn(acc, __fmul_rn(x[t].y, y[t].y));
            }
        }
    }
    for (; j + 8 <= n; j += 8) {
        float y[8];
#pragma unroll
        for (int t = 0; t < 8; t++) y[t] = __ldg(b + j + t);
#pragma unroll
        for (int t = 0; t < 8; t++) acc = __fadd_rn(acc, __fmul_rn(a[j + t], y[t]));
    }
    for (; j < n; j++) acc = __fadd_rn(acc, __fmul_rn(a[j], __ldg(b + j)));
    return acc;
}

// One undecided pair by the reference's arithmetic (batch query q): its coarse levels (counted in
// the histograms, checked for the rank-order anomaly) and its group code.  The user's row in shared
// or global memory, its threshold summary in global memory.
__device__ __forceinline__ void exact_pair(const ScArgs &a, int64_t u, int q, const float *summ, const float *ur) {
    const float *qr = a.qrow + (int64_t) q * a.dim;
    const float left = exact_dot_any(ur, qr, a.c);
    float full = left;
    const int64_t o = (int64_t) q * a.n_user + u;
    if (a.lvt) {
        const float right = __fmul_rn(a.unorm[u], a.qnorm[q]);
        const uint32_t v = regression_levels_exact(a.m.rec, a.m.S, a.m.err_cap, u, __fsub_rn(left, right),
                                                   __fadd_rn(left, right));
        const int l = (int) (v & 0xffffu), h = (int) (v >> 16);
        const int cl = lvt_coarse(l, a.m.S), cu = lvt_coarse(h, a.m.S);
        a.lvc[o] = (uint8_t) (cl | (cu << 4));
        if (h > l && level_rank(h, a.m.rank, a.m.S, a.m.n_item) > level_rank(l, a.m.rank, a.m.S, a.m.n_item))
            atomicAdd(a.anomaly + q, 1);
    }
    if (a.c < a.dim) full = __fadd_rn(left, exact_dot_any(ur + a.c, qr + a.c, a.dim - a.c));
    int g = 0;  // the summary entries >= full (descending, -inf padded)
#pragma unroll
    for (int st = 16; st >= 1; st >>= 1) g += __ldg(summ + g + st - 1) >= full ? st : 0;
    g += __ldg(summ + g) >= full;
    a.code[o] = (uint8_t) min(g, a.nb);
}

// The bound scores of the regression round, qlb = partial - right and qub = partial + right
// (PartDimPartNorm::IPBound), and their distances to the reference's binary32 values: the partial
// score's bound and each side's two roundings.
__device__ __forceinline__ void level_bounds(float vl, float dl, float un, float qn, float &qlb, float &qub,
                                             float &dql, float &dqu) {
    const float right = __fmul_rn(un, qn);
    const float2 q = __fadd2_rn(make_float2(vl, vl), make_float2(-right, right));
    const float dq = dl * 1.0001f;
    const float2 e = __ffma2_rn(make_float2(fabsf(q.x), fabsf(q.y)), make_float2(2.4e-7f, 2.4e-7f), make_float2(dq, dq));
    qlb = q.x;
    qub = q.y;
    dql = e.x;
    dqu = e.y;
}

__global__ void __launch_bounds__(kScThreads, 1) scores_tc_kernel(ScArgs a) {
    extern __shared__ __align__(1024) uint8_t sm_raw[];
    __shared__ uint64_t bar_a, bar_b[2], bar_mma[2], bar_free[2];
    __shared__ uint32_t tslot;
    __shared__ int list_n, abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t u0 = (int64_t) blockIdx.x * kScM;
    const int kp = a.kp, nq = a.nq;
    const int nchunks = (nq + kScN - 1) / kScN;
    const bool lev = a.lvt != nullptr;
    // shared memory: the user tile (A), two query chunk buffers (B, slices as consecutive row groups),
    // the threshold summary, the undecided list, the batch's query data, the coarse-level histograms
    // of two chunks and (QSRP) the tile's level tables
    const uint32_t a_bytes = (uint32_t) (kScSlices * kScM * kp), b_bytes = (uint32_t) (kScSlices * kScN * kp);
    uint8_t *sA = sm_raw;
    uint8_t *sB = sA + a_bytes;
    float *summ = reinterpret_cast<float *>(sB + 2 * b_bytes);
    uint32_t *list = reinterpret_cast<uint32_t *>(summ + ThrSummary::kMaxGroups * kScSummStride);
    float4 *sq = reinterpret_cast<float4 *>(list + kScListCap);  // the batch's query data
    float *sqn = reinterpret_cast<float *>(sq + kScMaxQ);
    float2 *stab = reinterpret_cast<float2 *>(sqn + kScMaxQ);  // [2 kLvEntries][kScM]
    volatile int *abort = &abort_flag;

    if (tid == 0) {
        mbar_init(&bar_a, 1);
        for (int b = 0; b < 2; b++) {
            mbar_init(&bar_b[b], 1);
            mbar_init(&bar_mma[b], 1);
            mbar_init(&bar_free[b], kScEpiWarps);
        }
        list_n = 0;
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    for (int idx = tid; idx < kScM * ThrSummary::kMaxGroups; idx += kScThreads) {
        const int rr = idx / ThrSummary::kMaxGroups, j = idx % ThrSummary::kMaxGroups;
        summ[j * kScSummStride + rr] =
            u0 + rr < a.n_user ? __ldg(a.thr_summ + (u0 + rr) * ThrSummary::kMaxGroups + j) : -INFINITY;
    }
    if (lev)
        for (int idx = tid; idx < kScM * 2 * kLvEntries; idx += kScThreads) {
            const int rr = idx / (2 * kLvEntries), j = idx % (2 * kLvEntries);
            stab[j * kScM + rr] = u0 + rr < a.n_user ? __ldg(a.lvt + (u0 + rr) * 2 * kLvEntries + j)
                                                     : make_float2(NAN, NAN);
        }
    for (int i = tid; i < nchunks * kScN; i += kScThreads) {  // the last chunk padded with the last query
        sq[i] = __ldg(a.qmeta + min(i, nq - 1));
        sqn[i] = lev ? __ldg(a.qnorm + min(i, nq - 1)) : 0.0f;
    }
    if (lev) {
        // the level tables as monotone limits (lvt_limits_row): one thread per user and side
        __syncthreads();
        for (int idx = tid; idx < 2 * kScM; idx += kScThreads) {
            float2 *t = stab + (idx & 1) * kLvEntries * kScM + (idx >> 1);
            lvt_limits_row(t, kScM);
            if (idx & 1) lvt_verify_row(t, kScM);  // the upper side: verification pairs
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = tslot;
    const int nacc = a.two_parts ? 8 : 4;
    const uint32_t buf_cols = (uint32_t) (nacc * kScN);

    if (warp == kScEpiWarps) {
        // ---- copies and MMAs: the warp runs the loop (warp-uniform values), one elected lane issues ----
        bool ok = true;
        int last = -1;  // last chunk whose MMAs were committed
        if (elect_one()) {
            mbar_expect_tx(&bar_a, a_bytes);
            bulk_g2s(sA, a.a_sl + (size_t) blockIdx.x * a_bytes, a_bytes, &bar_a);
            for (int j = 0; j < 2 && j < nchunks; j++) {
                mbar_expect_tx(&bar_b[j], b_bytes);
                bulk_g2s(sB + (size_t) j * b_bytes, a.b_sl + (size_t) j * b_bytes, b_bytes, &bar_b[j]);
            }
        }
        __syncwarp();
        ok = __all_sync(0xffffffffu, mbar_wait(&bar_a, 0, abort));
        // descriptors (addresses in 16-byte units, within the 14-bit field: shared memory < 256 KB): A in
        // K blocks of kScM rows (K step s at s * 2 * kScM * 16 bytes, slice i at i * kScM * kp); the
        // query chunk in row groups of kp * 8 bytes (K step s at s * 256 bytes)
        constexpr uint32_t kAChunk = kScM * 16;
        const uint64_t da0 = umma_desc(smem_u32(sA), kAChunk, 128);
        const uint64_t db0 = umma_desc(smem_u32(sB), 128, (uint32_t) kp * 8);
        const uint32_t a_slice = (uint32_t) (kScM * kp) >> 4, b_buf = b_bytes >> 4;
        for (int j = 0; ok && j < nchunks; j++) {
            const int b = j & 1;
            const uint32_t ph = (uint32_t) (j >> 1) & 1u;
            ok = mbar_wait(&bar_b[b], ph, abort);
            if (ok && j >= 2) ok = mbar_wait(&bar_free[b], (uint32_t) ((j - 2) >> 1) & 1u, abort);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t d0 = taddr + (uint32_t) b * buf_cols;
            for (int s = 0; s < a.ksteps; s++) {
                const int part = s < a.ksplit ? 0 : 1;
                const bool first_s = s == 0 || s == a.ksplit;
                const uint64_t das = da0 + ((uint32_t) s * 2 * kAChunk >> 4);
                const uint64_t dbs = db0 + (uint32_t) b * b_buf + (uint32_t) s * 16;
                const uint32_t dp = d0 + (uint32_t) part * 4 * kScN;
                if (elect_one()) umma_i8_step(dp, das, a_slice, dbs, first_s);
                __syncwarp();
            }
            if (elect_one())
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&bar_mma[b]))
                             : "memory");
            __syncwarp();
            last = j;
            if (j >= 1 && j + 1 < nchunks) {
                // the previous chunk's MMAs have read its query digits: refill that buffer with the next
                // chunk while this chunk's MMAs run
                const int pb = (j - 1) & 1;
                ok = __all_sync(0xffffffffu, mbar_wait(&bar_mma[pb], (uint32_t) ((j - 1) >> 1) & 1u, abort));
                if (!ok) break;
                if (elect_one()) {
                    mbar_expect_tx(&bar_b[pb], b_bytes);
                    bulk_g2s(sB + (size_t) pb * b_bytes, a.b_sl + (size_t) (j + 1) * b_bytes, b_bytes, &bar_b[pb]);
                }
                __syncwarp();
            }
        }
        if (!ok && lane == 0) {
            *abort = 1;
            atomicExch(a.status, 1);
        }
        // the MMAs of the last committed chunk finish on their own: wait for them (bounded) before
        // the columns are released
        if (last >= 0)
            for (int it = 0; it < (1 << 22) && !mbar_try(&bar_mma[last & 1], (uint32_t) (last >> 1) & 1u); it++) {
            }
    } else {
        // ---- epilogue ----
        const int quad = warp & 3, cg = warp >> 2;
        const int row = 32 * quad + lane;
        const int64_t u = u0 + row;
        const bool uval = u < a.n_user;
        const float *srow = summ + row;  // entry j at srow[j * kScSummStride]
        const float2 *tl = stab + row, *tu = stab + kLvEntries * kScM + row;  // entry j at t[j * kScM]
        float un = 0.0f;
        float4 um = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        // the common cases in registers, from the tables' limits (lvt_limits_row): the lower side's
        // last three boundaries T_12 .. T_14 (coarse levels 13 .. 15 hold all but about 0.1% of its
        // pairs at configs 2 and 4), the upper side's first kUpCache lower limits, scaled by 2^100
        // (its coarse levels 0 .. kUpCache - 1 hold all but about 0.01% of its pairs at config 2), so
        // that only the rare pairs beyond them take a table search
        float llo[3], lhi[3], ulo[kUpCache];
#pragma unroll
        for (int g = 0; g < 3; g++) { llo[g] = -INFINITY; lhi[g] = INFINITY; }
#pragma unroll
        for (int g = 0; g < kUpCache; g++) ulo[g] = NAN;
        if (uval) {
            um = __ldg(a.umeta + u);
            if (lev) {
                un = __ldg(a.unorm + u);
                // NaN entries (an unusable model): never decided from registers
#pragma unroll
                for (int g = 0; g < 3; g++) {
                    const float2 e = tl[(kLvEntries - 4 + g) * kScM];
                    llo[g] = e.x;
                    lhi[g] = e.y;
                    if (!(llo[g] == llo[g]) || !(lhi[g] == lhi[g])) { llo[g] = -INFINITY; lhi[g] = INFINITY; }
                }
#pragma unroll
                for (int g = 0; g < kUpCache; g++) ulo[g] = tu[(g + 1) * kScM].y * 0x1p100f;
            }
        }
        // the first two steps of the group search from registers
        const float s7 = srow[7 * kScSummStride], s15 = srow[15 * kScSummStride], s23 = srow[23 * kScSummStride];
        const int ue = __float_as_int(um.w);
        const float cl_u = a.cl * um.y, cr_u = a.cr * um.z;
        const uint32_t lane_base = taddr + ((uint32_t) (32 * quad) << 16) + (uint32_t) (8 * cg);
        int n_und = 0, n_slo = 0, n_sup = 0;
        bool dead = false;
        for (int j = 0; j < nchunks; j++) {
            const int b = j & 1;
            const uint32_t ph = (uint32_t) (j >> 1) & 1u;
            if (!dead && !__all_sync(0xffffffffu, mbar_wait(&bar_mma[b], ph, abort))) {
                *abort = 1;
                atomicExch(a.status, 1);
                dead = true;
            }
            if (!dead) {
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                float sl[8], sr[8];
                {
                    uint32_t v0[8], v1[8], v2[8], v3[8];
                    const uint32_t base = lane_base + (uint32_t) b * buf_cols;
                    tmem_ld8(base, v0);
                    tmem_ld8(base + kScN, v1);
                    tmem_ld8(base + 2 * kScN, v2);
                    tmem_ld8(base + 3 * kScN, v3);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    combine4_x8(v0, v1, v2, v3, sl);
                    if (a.two_parts) {
                        tmem_ld8(base + 4 * kScN, v0);
                        tmem_ld8(base + 5 * kScN, v1);
                        tmem_ld8(base + 6 * kScN, v2);
                        tmem_ld8(base + 7 * kScN, v3);
                        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                        combine4_x8(v0, v1, v2, v3, sr);
                    } else {
#pragma unroll
                        for (int i = 0; i < 8; i++) sr[i] = 0.0f;
                    }
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&bar_free[b]);
                uint32_t und_bits = 0;
                // four pairs at a time, in side-effect-free phases so that their chains interleave
#pragma unroll
                for (int i0 = 0; i0 < 8; i0 += 4) {
                    constexpr int G = 4;
                    float vl[G], full[G], dl[G], df[G];
                    int packed[G];
                    bool ok[G];
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        const int i = i0 + g;
                        const float4 qm = sq[j * kScN + 8 * cg + i];
                        const float scale = __int_as_float((ue + __float_as_int(qm.w) - 35 + 127) << 23);
                        // the two parts side by side in paired FP32 instructions (per component the
                        // roundings of the scalar forms)
                        const float ee = um.x * qm.x;
                        const float2 v = __fmul2_rn(make_float2(sl[i], sr[i]), make_float2(scale, scale));
                        const float2 t = __fmul2_rn(make_float2(ee, ee), make_float2(a.kl, a.kr));
                        const float2 d = __ffma2_rn(make_float2(cl_u, cr_u), make_float2(qm.y, qm.z),
                                                    __ffma2_rn(make_float2(fabsf(v.x), fabsf(v.y)),
                                                               make_float2(1.8e-7f, 1.8e-7f), t));
                        vl[g] = v.x;
                        dl[g] = d.x;
                        const float vr = v.y, dr = d.y;
                        full[g] = a.two_parts ? __fadd_rn(vl[g], vr) : vl[g];
                        df[g] = fmaf(fabsf(full[g]), 2.4e-7f, (dl[g] + dr) * 1.0001f);
                        ok[g] = true;
                        packed[g] = 0;
                    }
                    if (lev) {
                        // coarse levels of the bounds partial -+ right (PartDimPartNorm::IPBound) from the
                        // tables; within dq of the reference's bound scores: the partial score's bound and
                        // the two roundings of each side.  The cached limits decide most pairs without
                        // branches; each side's table search runs afterwards, for the whole warp, where
                        // any lane's pair needs one
                        unsigned needl = 0, needu = 0, needx = 0;
#pragma unroll
                        for (int g = 0; g < G; g++) {
                            float qlb, qub, dql, dqu;
                            level_bounds(vl[g], dl[g], un, sqn[j * kScN + 8 * cg + i0 + g], qlb, qub, dql, dqu);
                            // lower side: coarse level 15 below T_14, 14 between T_14 and T_13, 13 between
                            // T_13 and T_12, each surely (outside the bands)
                            int c_l, c_u;
                            bool okl;
                            {
                                const float qml = __fsub_rd(qlb, dql), qpl = __fadd_ru(qlb, dql);
                                const bool b14 = qpl < llo[2], b13 = qpl < llo[1], b12 = qpl < llo[0];
                                okl = b14 || (qml >= lhi[2] && b13) || (qml >= lhi[1] && b12);
                                c_l = b14 ? 15 : (b13 ? 14 : 13);
                            }
                            // upper side: c_u = #{g : qp < lo_g} over the cached limits, counted on the
                            // FMA pipe (each term saturates (lo_g - qp) 2^100 to [0, 1]: 1 when qp < lo_g,
                            // 0 otherwise or for NaN, a fraction only for differences below 2^-100, which
                            // the verification then refuses), and decided by the verification pair of
                            // c_u: qm >= hi_(c_u) and qp < lo_(c_u - 1).  A pair at the last cached limit
                            // may lie beyond it and takes the table search
                            bool oku;
                            {
                                const float qmu = __fsub_rd(qub, dqu), qpu = __fadd_ru(qub, dqu);
                                const float nq = qpu * -0x1p100f;
                                float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
                                for (int e = 0; e + 1 < kUpCache; e += 2)
                                    acc = __fadd2_rn(acc, make_float2(__saturatef(__fadd_rn(ulo[e], nq)),
                                                                      __saturatef(__fadd_rn(ulo[e + 1], nq))));
                                // in [0, kUpCache]: the table index stays in bounds whatever the terms
                                c_u = __float_as_int(__fadd_rn(__fadd_rn(acc.x, acc.y), 12582912.0f)) - 0x4B400000;
                                const float2 ve = tu[c_u * kScM];
                                oku = qmu >= ve.x && qpu < ve.y;
                                needx |= (unsigned) (!oku && c_u == kUpCache) << g;
                            }
                            needl |= (unsigned) !okl << g;
                            needu |= (unsigned) !oku << g;
                            packed[g] = c_l | (c_u << 4);
                        }
                        if (__any_sync(0xffffffffu, needx != 0u)) {
#pragma unroll
                            for (int g = 0; g < G; g++) {
                                const bool wx = (needx >> g) & 1u;
                                if (!__any_sync(0xffffffffu, wx)) continue;
                                n_sup++;
                                float qlb, qub, dql, dqu;
                                level_bounds(vl[g], dl[g], un, sqn[j * kScN + 8 * cg + i0 + g], qlb, qub, dql, dqu);
                                int c;
                                const bool o = lvt_screen_ver(tu, kScM, __fsub_rd(qub, dqu), __fadd_ru(qub, dqu), c);
                                if (wx) {
                                    packed[g] = (packed[g] & 0x0f) | (c << 4);
                                    if (o) needu &= ~(1u << g);
                                }
                            }
                        }
                        if (__any_sync(0xffffffffu, needl != 0u)) {
#pragma unroll
                            for (int g = 0; g < G; g++) {
                                const bool wl = (needl >> g) & 1u;
                                if (!__any_sync(0xffffffffu, wl)) continue;
                                n_slo++;
                                float qlb, qub, dql, dqu;
                                level_bounds(vl[g], dl[g], un, sqn[j * kScN + 8 * cg + i0 + g], qlb, qub, dql, dqu);
                                int c;
                                const bool o = lvt_screen_lim(tl, kScM, __fsub_rd(qlb, dql), __fadd_ru(qlb, dql), c);
                                if (wl) {
                                    packed[g] = (packed[g] & 0xf0) | c;
                                    if (o) needl &= ~(1u << g);
                                }
                            }
                        }
#pragma unroll
                        for (int g = 0; g < G; g++) ok[g] = !(((needl | needu) >> g) & 1u);
                    }
                    // coarse group: the summary entries >= full.  The search runs on key = full + df:
                    // with lo entries >= key, the pair is decided when the next entry lies below
                    // full - df, and then exactly lo entries are >= full (the entries descend)
                    int lo[G];
                    float key[G];
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        key[g] = full[g] + df[g];
                        lo[g] = s15 >= key[g] ? 16 : 0;
                        lo[g] += (lo[g] ? s23 : s7) >= key[g] ? 8 : 0;
                    }
#pragma unroll
                    for (int st = 4; st >= 1; st >>= 1)
#pragma unroll
                        for (int g = 0; g < G; g++) lo[g] += srow[(lo[g] + st - 1) * kScSummStride] >= key[g] ? st : 0;
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        lo[g] += srow[lo[g] * kScSummStride] >= key[g];
                        const bool gok = (lo[g] >= ThrSummary::kMaxGroups || srow[lo[g] * kScSummStride] < full[g] - df[g]) &&
                                         df[g] < 1e30f && full[g] == full[g];
                        ok[g] = ok[g] && gok;
                    }
                    // every pair is stored (the exact pass rewrites the undecided ones)
#pragma unroll
                    for (int g = 0; g < G; g++) {
                        const int qi = 8 * cg + i0 + g, q = j * kScN + qi;
                        if (!uval || q >= nq) continue;
                        const int64_t o = (int64_t) q * a.n_user + u;
                        if (lev) a.lvc[o] = (uint8_t) packed[g];
                        a.code[o] = (uint8_t) min(lo[g], a.nb);
                        if (a.dump) a.dump[o] = make_float2(full[g], df[g]);
                        und_bits |= (uint32_t) !ok[g] << (i0 + g);
                    }
                }
                // the chunk's undecided pairs into the list: one shared-memory atomic per warp
                const int cnt = __popc(und_bits);
                int incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                const int tot = __shfl_sync(0xffffffffu, incl, 31);
                if (tot) {
                    int base = 0;
                    if (lane == 31) base = atomicAdd(&list_n, tot);
                    base = __shfl_sync(0xffffffffu, base, 31);
                    int slot = base + incl - cnt;
                    n_und += cnt;
                    for (uint32_t m = und_bits; m; m &= m - 1, slot++) {
                        const int q = j * kScN + 8 * cg + __ffs(m) - 1;
                        if (slot < kScListCap) {
                            list[slot] = (uint32_t) q | ((uint32_t) row << 16);
                        } else {
                            const int go = atomicAdd(a.spill_count, 1);
                            if (go < a.spill_cap) a.spill[go] = make_int2(a.q_base + q, (int) u);
                            else atomicExch(a.status, 2);
                        }
                    }
                }
            }
        }
        if (n_und) atomicAdd(a.undecided, n_und);
        if (lane == 0 && (n_slo | n_sup)) {
            atomicAdd(a.searches, 32 * n_slo);
            atomicAdd(a.searches + 1, 32 * n_sup);
        }
    }
    // all MMAs have completed once every epilogue warp has passed its last wait (or given up)
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    // the tile's undecided pairs join the batch's list (one global atomic per CTA); a separate kernel
    // with many threads in flight resolves them, hiding the latency of the rows' loads
    __shared__ int list_base;
    const int n_list = min(list_n, kScListCap);
    if (tid == 0) {
        list_base = n_list ? atomicAdd(a.ovf_count, n_list) : 0;
        a.tile_rng[blockIdx.x] = make_int2(list_base, list_base + n_list <= a.ovf_cap ? n_list : 0);
    }
    __syncthreads();
    for (int i = tid; i < n_list; i += kScThreads) {
        const uint32_t e = list[i];
        const int g = list_base + i;
        if (g < a.ovf_cap) a.ovf[g] = make_int2(a.q_base + (int) (e & 0xffffu), (int) (u0 + (e >> 16)));
        else atomicExch(a.status, 2);
    }
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(taddr) : "memory");
    }
}

// The listed (undecided) pairs of one tile of users, by the reference's arithmetic: the tile's user
// rows are staged in shared memory once (they are contiguous in global memory), the queries' rows
// come from L2.
__global__ void __launch_bounds__(256, 2) scores_tc_exact_tile_kernel(ScArgs a, int n_tiles) {
    extern __shared__ __align__(128) float rows[];
    __shared__ uint64_t bar;
    __shared__ int failed;
    const int2 rng = a.tile_rng[(int64_t) blockIdx.y * n_tiles + blockIdx.x];
    if (rng.y == 0) return;
    const int64_t u0 = (int64_t) blockIdx.x * kScM;
    const int64_t n_rows = a.n_user - u0 < kScM ? a.n_user - u0 : kScM;
    const float *src = a.urow + u0 * a.dim;
    // the tile's rows (contiguous, 16-byte aligned: kScM * 4 | 16) in one bulk copy; a tail that is not
    // a whole 16 bytes by plain loads
    const int n_f = (int) n_rows * a.dim, n_v = n_f >> 2;
    const uint32_t bytes = (uint32_t) n_v * 16;
    if (threadIdx.x == 0) {
        failed = 0;
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        if (bytes) {
            mbar_expect_tx(&bar, bytes);
            bulk_g2s(rows, src, bytes, &bar);
        } else {
            mbar_arrive(&bar);
        }
    }
    for (int f = 4 * n_v + threadIdx.x; f < n_f; f += blockDim.x) rows[f] = __ldg(src + f);
    __syncthreads();
    {
        // every thread observes the copy's completion (bounded wait)
        bool ok = false;
        for (int it = 0; it < (1 << 22) && !ok; it++) ok = mbar_try(&bar, 0);
        if (!ok) {
            failed = 1;
            atomicExch(a.status, 1);
        }
    }
    __syncthreads();
    if (failed) return;
    for (int i = threadIdx.x; i < rng.y; i += blockDim.x) {
        const int2 x = a.ovf[rng.x + i];
        exact_pair(a, x.y, x.x, a.thr_summ + (int64_t) x.y * ThrSummary::kMaxGroups, rows + (x.y - u0) * a.dim);
    }
}

// Undecided pairs past the tiles' shared-memory lists (a tile with more than kScListCap of them).
__global__ void __launch_bounds__(256, 2) scores_tc_spill_kernel(ScArgs a) {
    const int n = min(*a.spill_count, a.spill_cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int2 x = a.spill[i];
        exact_pair(a, x.y, x.x, a.thr_summ + (int64_t) x.y * ThrSummary::kMaxGroups, a.urow + (int64_t) x.y * a.dim);
    }
}

}  // namespace

int scores_tc(rkr_index *ix, const ScoresTcCall &call, cudaStream_t st, bool *done) {
    *done = false;
    if (call.status) call.status[0] = nullptr;
    if (!ix->scores_tc_on) return RKR_OK;
    const int dim = ix->dim, nq = call.nq;
    const int c = call.qsrp ? ix->check_dim : dim;
    const int n1 = c, n2 = dim - c;
    if (n1 <= 0 || n1 > kScMaxPart || n2 > kScMaxPart || nq <= 0) return RKR_OK;
    const int cp = round32(n1), kp = cp + round32(n2);
    if (kp > kScMaxKp) return RKR_OK;
    if (call.qsrp && !ix->lvt.p) return RKR_OK;
    const int64_t U = ix->n_user;
    const int64_t n_tiles = (U + kScM - 1) / kScM;
    if (n_tiles > 0x7fffffff) return RKR_OK;
    const size_t smem = (size_t) kScSlices * kp * (kScM + 2 * kScN) + sizeof(float) * ThrSummary::kMaxGroups * kScM +
                        sizeof(uint32_t) * kScListCap + (sizeof(float4) + sizeof(float)) * kScMaxQ +
                        (call.qsrp ? sizeof(float2) * 2 * kLvEntries * kScM : 0);
    if (smem + 1024 > 227 * 1024) return RKR_OK;
    // user digits for this split (built once per split and kept)
    DevBuf &ub = call.qsrp ? ix->sc_user_split : ix->sc_user_full;
    DevBuf &um = call.qsrp ? ix->sc_umeta_split : ix->sc_umeta_full;
    int &key = call.qsrp ? ix->sc_key_split : ix->sc_key_full;
    if (key != c) {
        const int64_t n_pad = n_tiles * kScM;
        RKR_TRY(ub.ensure((size_t) n_pad * kScSlices * kp));
        RKR_TRY(um.ensure(sizeof(float4) * (size_t) n_pad));
        const float *src = (call.qsrp ? ix->svd_user : ix->user).as<float>();
        const unsigned g = (unsigned) ((n_pad * 32 + 255) / 256);
        slice_rows_kernel<<<g, 256, 0, st>>>(src, nullptr, U, n_pad, dim, c, cp, kp, kScM, 0, ub.as<int8_t>(),
                                             um.as<float4>());
        RKR_CUDA(cudaGetLastError());
        key = c;
    }
    // query digits, chunks of kScN
    const int nchunks = (nq + kScN - 1) / kScN;
    const int64_t nq_pad = (int64_t) nchunks * kScN;
    const int ovf_cap = (int) std::min<int64_t>(int64_t(1) << 24, std::max<int64_t>(int64_t(1) << 16, U * nq / 32));
    const size_t b_total = (size_t) nq_pad * kScSlices * kp;
    const int n_launch = (nq + kScMaxQ - 1) / kScMaxQ;
    const int spill_cap = 1 << 20;
    const size_t need = b_total + 256 + sizeof(float4) * (size_t) nq_pad + 256 + sizeof(int2) * (size_t) ovf_cap + 256 +
                        sizeof(int2) * ((size_t) n_launch * n_tiles + spill_cap) + 512 + 64;
    RKR_TRY(ix->ws_sc.ensure(need));
    uint8_t *p = ix->ws_sc.as<uint8_t>();
    auto take = [&](size_t bytes) {
        uint8_t *r = p;
        p += (bytes + 255) & ~size_t(255);
        return r;
    };
    int8_t *b_sl = reinterpret_cast<int8_t *>(take(b_total));
    float4 *qmeta = reinterpret_cast<float4 *>(take(sizeof(float4) * (size_t) nq_pad));
    int2 *ovf = reinterpret_cast<int2 *>(take(sizeof(int2) * (size_t) ovf_cap));
    int2 *tile_rng = reinterpret_cast<int2 *>(take(sizeof(int2) * (size_t) n_launch * n_tiles));
    int2 *spill = reinterpret_cast<int2 *>(take(sizeof(int2) * (size_t) spill_cap));
    // ovf_count, status, undecided, (unused), spill, lower and upper table searches
    int *counters = reinterpret_cast<int *>(take(64));
    RKR_CUDA(cudaMemsetAsync(counters, 0, 7 * sizeof(int), st));
    if (call.status) {
        // the caller reads the status and the counts later (the launches stay free of host
        // synchronisation, so that they can be captured in a graph)
        call.status[0] = counters + 1;
        call.status[1] = counters + 2;
        call.status[2] = counters + 5;
        call.status[3] = counters + 6;
    }
    {
        const unsigned g = (unsigned) ((nq_pad * 32 + 255) / 256);
        timed(ix, st, "scores_tc_prep", [&] {
            slice_rows_kernel<<<g, 256, 0, st>>>(call.qrows, nullptr, nq, nq_pad, dim, c, cp, kp, kScN, 1, b_sl, qmeta);
        });
        RKR_CUDA(cudaGetLastError());
    }
    ScArgs a = {};
    a.a_sl = ub.as<int8_t>();
    a.b_sl = b_sl;
    a.umeta = um.as<float4>();
    a.qmeta = qmeta;
    a.unorm = call.unorm;
    a.qnorm = call.qnorm;
    a.urow = (call.qsrp ? ix->svd_user : ix->user).as<float>();
    a.qrow = call.qrows;
    a.thr_summ = ix->thr_summ.as<float>();
    a.m = call.m;
    a.lvt = call.qsrp ? ix->lvt.as<float2>() : nullptr;
    a.lvc = call.lvc;
    a.code = call.code;
    a.anomaly = call.anomaly;
    a.dump = ix->score_dump;
    a.ovf = ovf;
    a.ovf_count = counters;
    a.status = counters + 1;
    a.undecided = counters + 2;
    a.searches = counters + 5;
    a.ovf_cap = ovf_cap;
    a.spill = spill;
    a.spill_count = counters + 4;
    a.spill_cap = spill_cap;
    a.n_user = U;
    a.nq = nq;
    a.dim = dim;
    a.c = c;
    a.kp = kp;
    a.ksplit = cp / 32;
    a.ksteps = kp / 32;
    a.two_parts = n2 > 0;
    a.nb = call.nb;
    part_coef(n1, a.cl, a.kl);
    part_coef(n2, a.cr, a.kr);
    // function attributes are set outside graph capture (the eager first run of a shape sets them)
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    RKR_CUDA(cudaStreamIsCapturing(st, &capturing));
    if (capturing == cudaStreamCaptureStatusNone)
        RKR_CUDA(cudaFuncSetAttribute(scores_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    // launches of at most kScMaxQ queries (whole chunks): their data sits in shared memory
    for (int q0 = 0; q0 < nq; q0 += kScMaxQ) {
        ScArgs s = a;
        s.q_base = q0;
        s.nq = std::min(kScMaxQ, nq - q0);
        s.b_sl = b_sl + (size_t) (q0 / kScN) * kScSlices * kScN * kp;
        s.qmeta = qmeta + q0;
        s.qnorm = a.qnorm ? a.qnorm + q0 : nullptr;
        s.qrow = a.qrow + (size_t) q0 * dim;
        s.lvc = a.lvc ? a.lvc + (size_t) q0 * U : nullptr;
        s.code = a.code + (size_t) q0 * U;
        s.anomaly = a.anomaly ? a.anomaly + q0 : nullptr;
        s.dump = a.dump ? a.dump + (size_t) q0 * U : nullptr;
        s.tile_rng = tile_rng + (size_t) (q0 / kScMaxQ) * n_tiles;
        timed(ix, st, "qsrp_scores_tc", [&] { scores_tc_kernel<<<(unsigned) n_tiles, kScThreads, smem, st>>>(s); });
        RKR_CUDA(cudaGetLastError());
    }
    a.tile_rng = tile_rng;
    const size_t rows_smem = sizeof(float) * kScM * (size_t) dim;
    if (capturing == cudaStreamCaptureStatusNone)
        RKR_CUDA(cudaFuncSetAttribute(scores_tc_exact_tile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int) rows_smem));
    timed(ix, st, "qsrp_scores_tc_exact", [&] {
        scores_tc_exact_tile_kernel<<<dim3((unsigned) n_tiles, (unsigned) n_launch), 256, rows_smem, st>>>(a, (int) n_tiles);
    });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "qsrp_scores_tc_spill", [&] { scores_tc_spill_kernel<<<148 * 4, 256, 0, st>>>(a); });
    RKR_CUDA(cudaGetLastError());
    *done = true;
    if (call.status) return RKR_OK;
    int h[7] = {0, 0, 0, 0, 0, 0, 0};
    RKR_CUDA(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    if (ix->prof.on) {
        ix->prof.add_count("screen_undecided_pairs", h[2]);
        ix->prof.add_count("lvt_search_lower_pairs", h[5]);
        ix->prof.add_count("lvt_search_upper_pairs", h[6]);
    }
    if (h[1]) {
        // a wait gave up or the overflow list filled: the exact tiles redo the batch from clean counts
        set_error("scores_tc: status %d", h[1]);
        *done = false;
    }
    return RKR_OK;
}

}  // namespace rkr
