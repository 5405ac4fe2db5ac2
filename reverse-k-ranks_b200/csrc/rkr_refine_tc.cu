// rkr_refine_tc.cu -- the counting step of candidate refinement on the tensor cores (tcgen05, int8).
//
// Refinement counts, per candidate (user u, score qv) and item in the norm cut-off, the reference's
// per-item test (RefineCPUIPBound::RefineRank, RefineCPUIPBound.hpp:93-150 with the split sums of
// RefineCPUPartDimPartNorm.hpp:83-152; RefineCPU::RefineRank, RefineCPU.hpp:33-55 without the bound).
// The test only asks on which side of a few thresholds a pair's scores fall: its partial score over
// the first check_dim coordinates against lowq - right and highq + right, and its full score against
// qv.  So the scores come from the int8 digit products of rkr_tc_common.cuh (exact integer
// accumulation, the partial and the remaining coordinates in separate TMEM accumulators), each
// with a rigorous bound on its distance to the reference's binary32 value; a pair whose bound
// interval straddles a threshold is listed and decided by the reference's own arithmetic
// (refine_tc_exact_kernel).
//
// Items in groups.  Items are taken in the norm order (item_sorted; US counts over all items, in any
// order) and cut into groups of 8 that share one power-of-two scale and one set of bound data (the
// largest weighted and plain norms of the group).  A warp's 8 columns of a chunk are one group, so
// each thread turns its candidate's bound and the six thresholds of the test into the digit units of
// its (candidate, group) once per chunk, and a pair costs the combination of its accumulators, one
// product (the reference's right = |item rest| |user rest|), three sums and six comparisons.
//
// Tiles.  A CTA holds the digits of 128 candidates (the MMA's M, TMEM lanes) and walks a strided
// share of the 32-item chunks inside its candidates' norm cut-off; the items' digit chunks are
// bulk-copied and double-buffered, the accumulators double-buffered in TMEM, so that one chunk's
// MMAs overlap the previous chunk's epilogue.  The chunk's four digit slices follow each other as row
// groups, so that per candidate slice i and K step one MMA of N = 32 (4 - i) fills the digit-group
// accumulators i .. 3 (umma_i8_step: 4 MMAs per K step instead of one per digit pair; the operand
// traffic of shared memory, which bounds these small MMAs, falls by 1.9x).  Warp 16 runs the
// copies and the MMAs (one elected lane issues); warps 0-15 run the epilogue (warp w: lane
// quadrant w % 4, columns 8 (w / 4) .. + 8 of each accumulator).
#include <algorithm>
#include <cstdio>

#include "rkr_internal.cuh"
#include "rkr_tc_common.cuh"

namespace rkr {

namespace {

constexpr int kRfEpiWarps = 16;
constexpr int kRfThreads = 32 * (kRfEpiWarps + 1);
constexpr int kRfMaxKp = 224;  // the candidate tile and two item chunks fit in shared memory up to this K
constexpr int kRfGroup = 8;    // items per group (a warp's columns of a chunk)

// Per candidate row, 2 float4: {2^e, weighted norms WL, WR, plain norm NL}, {NR, e (int bits), 0, 0}.
// Per item group, 4 float4: {the reference's rest norms (item_rnorm) of the 8 items}, {2^e, WL max,
// WR max, NL max}, {NR max, rest norm max, e (int bits), 0}.  Weighted norms as in part_coef, plain
// norms the Euclidean norms of the two parts; all rounded up.

// Rows to 4-digit tiles of tr rows, one block of 8 warps per 8 rows.  grouped (items, the B operand):
// the 8 rows share the scale of their largest coordinate, write group data and take the stacked
// layout of digit_off; else (candidates, the A operand) each row has its own scale and writes row data.  A group or row with a non-finite coordinate or a scale
// beyond 2^+-kScMaxExp gets 2^e = inf (its pairs all go to the exact path) and zero digits.
__global__ void __launch_bounds__(256) rf_slice_kernel(const float *__restrict__ src, const int32_t *__restrict__ idx,
                                                       int64_t n, int dim, int c, int cp, int kp, int tr, int grouped,
                                                       const float *__restrict__ rnorm, int8_t *__restrict__ dst,
                                                       float4 *__restrict__ row_meta, float4 *__restrict__ grp_meta) {
    __shared__ float s_mx[kRfGroup], s_v[kRfGroup][5];
    __shared__ int s_bad[kRfGroup];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t r = (int64_t) blockIdx.x * kRfGroup + warp;  // grid covers the padded rows exactly
    const float *row = r < n ? src + (idx ? (int64_t) idx[r] : r) * dim : nullptr;
    float mx = 0.0f;
    int bad = 0;
    if (row)
        for (int k = lane; k < dim; k += 32) {
            const float v = row[k];
            bad |= !isfinite(v);
            mx = fmaxf(mx, fabsf(v));
        }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        bad |= __shfl_xor_sync(0xffffffffu, bad, o);
    }
    if (grouped) {
        if (lane == 0) {
            s_mx[warp] = mx;
            s_bad[warp] = bad;
        }
        __syncthreads();
        mx = 0.0f;
        bad = 0;
#pragma unroll
        for (int w = 0; w < kRfGroup; w++) {
            mx = fmaxf(mx, s_mx[w]);
            bad |= s_bad[w];
        }
    }
    int e = 0;
    if (mx > 0.0f) {
        int x;
        frexpf(mx, &x);  // mx = m 2^x, m in [0.5, 1): mx 2^-(x + 1) < 0.5
        e = x + 1;
    }
    if (e > kScMaxExp || e < -kScMaxExp) bad = 1;
    const float scale = bad ? 0.0f : ldexpf(1.0f, -e);
    double wl = 0.0, wr = 0.0, nl = 0.0, nr = 0.0;
    const size_t slice_bytes = (size_t) tr * kp;
    int8_t *tb = dst + (size_t) (r / tr) * kScSlices * slice_bytes;
    const int rr = (int) (r % tr);
    for (int p = lane; p < kp; p += 32) {
        const int k = p < cp ? (p < c ? p : -1) : (p - cp + c < dim ? p - cp + c : -1);
        float v = 0.0f;
        if (row && k >= 0) {
            v = row[k];
            const int t = k < c ? k : k - c, m = k < c ? c : dim - c;
            const double w = t == 0 ? m : m - t + 1, v2 = (double) v * v;
            if (k < c) { wl += w * v2; nl += v2; }
            else { wr += w * v2; nr += v2; }
        }
        float a = v * scale;  // exact: a power of two
        const size_t off = digit_off(rr, p, tr, kp, grouped);  // items: the stacked B layout
#pragma unroll
        for (int s = 0; s < kScSlices; s++) {
            const float t = a * 128.0f;  // exact
            const float d = rintf(t);    // |t| < 64
            a = t - d;                   // exact, |a| <= 0.5
            tb[s * slice_bytes + off] = (int8_t) (int) d;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        wl += __shfl_xor_sync(0xffffffffu, wl, o);
        wr += __shfl_xor_sync(0xffffffffu, wr, o);
        nl += __shfl_xor_sync(0xffffffffu, nl, o);
        nr += __shfl_xor_sync(0xffffffffu, nr, o);
    }
    const float E = bad ? INFINITY : ldexpf(1.0f, e);
    const float WL = __double2float_ru(sqrt(wl * (1.0 + 1e-12))), WR = __double2float_ru(sqrt(wr * (1.0 + 1e-12)));
    const float NL = __double2float_ru(sqrt(nl * (1.0 + 1e-12))), NR = __double2float_ru(sqrt(nr * (1.0 + 1e-12)));
    if (!grouped) {
        if (lane == 0) {
            row_meta[2 * r] = make_float4(E, WL, WR, NL);
            row_meta[2 * r + 1] = make_float4(NR, __int_as_float(bad ? 0 : e), 0.0f, 0.0f);
        }
        return;
    }
    if (lane == 0) {
        s_v[warp][0] = WL;
        s_v[warp][1] = WR;
        s_v[warp][2] = NL;
        s_v[warp][3] = NR;
        s_v[warp][4] = r < n && rnorm ? rnorm[r] : 0.0f;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float m[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
        for (int w = 0; w < kRfGroup; w++)
            for (int j = 0; j < 5; j++) m[j] = fmaxf(m[j], s_v[w][j]);
        float4 *g = grp_meta + 4 * blockIdx.x;
        g[0] = make_float4(s_v[0][4], s_v[1][4], s_v[2][4], s_v[3][4]);
        g[1] = make_float4(s_v[4][4], s_v[5][4], s_v[6][4], s_v[7][4]);
        g[2] = make_float4(E, m[0], m[1], m[2]);
        g[3] = make_float4(m[3], m[4], __int_as_float(bad ? 0 : e), 0.0f);
    }
}

struct TcArgs {
    const int8_t *cand_sl, *item_sl;           // digit tiles: candidates (kScM rows), items (kScN rows)
    const float4 *cand_meta, *grp_meta;        // row data (2 float4 per candidate), group data (4 per group)
    const float *item_rnorm, *user_rnorm;      // the reference's remaining-coordinate norms (bound test)
    const float *user_rows, *item_rows;        // exact rows for undecided pairs (item_rows: item_sorted)
    const int32_t *ref_idx, *ref_user, *n_ref, *nproc;
    const float *qip;
    int32_t *rank, *undecided;
    int64_t n_item;
    int dim, c, kp, ksplit, ksteps, ipbound;
    float cl, kl, cr, kr;                      // bound coefficients of the two parts (part_coef)
    int4 *list;                                // undecided pairs: (candidate, user, item, mode)
    int *list_count, *status;
    int list_cap;
};

enum : int { kModeFull = 0, kModeCountOnly = 1 };

// The reference's test for one pair (mode full) or its count alone (mode count-only).
__device__ __forceinline__ void exact_pair(const TcArgs &a, int e, int u, int64_t it, int mode, int &cnt, int &und) {
    const float *ur = a.user_rows + (int64_t) u * a.dim, *ir = a.item_rows + it * a.dim;
    const float qv = a.qip[e];
    cnt = 0;
    und = 0;
    if (!a.ipbound) {
        cnt = exact_dot(ur, ir, a.dim) > qv;
        return;
    }
    const float left = exact_dot(ur, ir, a.c), rest = exact_dot(ur + a.c, ir + a.c, a.dim - a.c);
    if (mode == kModeFull) {
        const float lowq = __fsub_rn(qv, 8e-3f), highq = __fadd_rn(qv, 8e-3f);
        const float right = __fmul_rn(a.item_rnorm[it], a.user_rnorm[u]);
        if (lowq > __fadd_rn(left, right)) return;
        if (highq < __fsub_rn(left, right)) { cnt = 1; return; }
        und = 1;
    }
    cnt = __fadd_rn(left, rest) >= qv;
}

// Out of line with a copy of the arguments, so that the kernel's parameters stay where they are and
// the rarely taken path stays out of the epilogue's instruction stream.
__device__ __noinline__ void exact_pair_now(TcArgs a, int e, int u, int64_t it, int mode) {
    int cnt, und;
    exact_pair(a, e, u, it, mode, cnt, und);
    if (cnt) atomicAdd(a.rank + e, cnt);
    if (und) atomicAdd(a.undecided + e, und);
}

// 2^k as a float, k in [-126, 127].
__device__ __forceinline__ float pow2f(int k) { return __int_as_float((k + 127) << 23); }

__global__ void __launch_bounds__(kRfThreads, 1) refine_tc_kernel(TcArgs a) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ uint64_t bar_a, bar_b[2], bar_mma[2], bar_free[2];
    __shared__ uint32_t tslot;
    __shared__ int e_s[kScM], np_s[kScM], u_s[kScM], max_np, abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t r0 = (int64_t) blockIdx.y * kScM;
    const int n_ref = *a.n_ref;
    if (r0 >= n_ref) return;
    volatile int *abort = &abort_flag;
    if (tid < kScM) {
        const int64_t r = r0 + tid;
        int e = -1, np = 0, u = 0;
        if (r < n_ref) {
            e = a.ref_idx[r];
            np = a.nproc[e];
            u = a.ref_user[r];
        }
        e_s[tid] = e; np_s[tid] = np; u_s[tid] = u;
    }
    if (tid == 0) {
        max_np = 0;
        abort_flag = 0;
    }
    __syncthreads();
    if (tid < kScM) atomicMax(&max_np, np_s[tid]);
    __syncthreads();
    // this CTA's item chunks: s, s + gridDim.x, ... below the candidates' largest cut-off
    const int n_chunks = (max_np + kScN - 1) / kScN;
    const int mine = n_chunks > (int) blockIdx.x ? (n_chunks - (int) blockIdx.x + (int) gridDim.x - 1) / (int) gridDim.x : 0;
    if (mine == 0) return;

    const int kp = a.kp;
    // shared memory: the candidate tile (A), then two item chunk buffers (B, slices as consecutive row
    // groups)
    const uint32_t a_bytes = (uint32_t) (kScSlices * kScM * kp), b_bytes = (uint32_t) (kScSlices * kScN * kp);
    uint8_t *sA = tc_smem;
    uint8_t *sB = sA + a_bytes;
    if (tid == 0) {
        mbar_init(&bar_a, 1);
        for (int b = 0; b < 2; b++) {
            mbar_init(&bar_b[b], 1);
            mbar_init(&bar_mma[b], 1);
            mbar_init(&bar_free[b], kRfEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(&tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = tslot;
    const bool has_rest = a.ksteps > a.ksplit;
    const uint32_t buf_cols = (uint32_t) ((has_rest ? 8 : 4) * kScN);

    if (warp == kRfEpiWarps) {
        // ---- copies and MMAs: the warp runs the loop, one elected lane issues ----
        bool ok = true;
        int last = -1;
        if (elect_one()) {
            mbar_expect_tx(&bar_a, a_bytes);
            bulk_g2s(sA, a.cand_sl + (size_t) blockIdx.y * a_bytes, a_bytes, &bar_a);
            for (int i = 0; i < 2 && i < mine; i++) {
                const int t = blockIdx.x + i * gridDim.x;
                mbar_expect_tx(&bar_b[i], b_bytes);
                bulk_g2s(sB + (size_t) i * b_bytes, a.item_sl + (size_t) t * b_bytes, b_bytes, &bar_b[i]);
            }
        }
        __syncwarp();
        ok = __all_sync(0xffffffffu, mbar_wait(&bar_a, 0, abort));
        // descriptors (addresses in 16-byte units, within the 14-bit field: shared memory < 256 KB): A in
        // K blocks of kScM rows (K step s at s * 2 * kScM * 16 bytes, slice i at i * kScM * kp); the
        // item chunk in row groups of kp * 8 bytes (K step s at s * 256 bytes)
        constexpr uint32_t kAChunk = kScM * 16;
        const uint64_t da0 = umma_desc(smem_u32(sA), kAChunk, 128);
        const uint64_t db0 = umma_desc(smem_u32(sB), 128, (uint32_t) kp * 8);
        const uint32_t a_slice = (uint32_t) (kScM * kp) >> 4, b_buf = b_bytes >> 4;
        for (int i = 0; ok && i < mine; i++) {
            const int b = i & 1;
            const uint32_t ph = (uint32_t) (i >> 1) & 1u;
            ok = mbar_wait(&bar_b[b], ph, abort);
            if (ok && i >= 2) ok = mbar_wait(&bar_free[b], (uint32_t) ((i - 2) >> 1) & 1u, abort);
            ok = __all_sync(0xffffffffu, ok);
            if (!ok) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t d0 = taddr + (uint32_t) b * buf_cols;
            for (int s = 0; s < a.ksteps; s++) {
                const int part = s < a.ksplit ? 0 : 1;
                const uint64_t das = da0 + ((uint32_t) s * 2 * kAChunk >> 4);
                const uint64_t dbs = db0 + (uint32_t) b * b_buf + (uint32_t) s * 16;
                if (elect_one()) umma_i8_step(d0 + (uint32_t) part * 4 * kScN, das, a_slice, dbs, s == 0 || s == a.ksplit);
                __syncwarp();
            }
            if (elect_one())
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&bar_mma[b]))
                             : "memory");
            __syncwarp();
            last = i;
            if (i >= 1 && i + 1 < mine) {
                // the previous chunk's MMAs have read its items: refill that buffer
                const int pb = (i - 1) & 1;
                ok = __all_sync(0xffffffffu, mbar_wait(&bar_mma[pb], (uint32_t) ((i - 1) >> 1) & 1u, abort));
                if (!ok) break;
                if (elect_one()) {
                    const int t = blockIdx.x + (i + 1) * gridDim.x;
                    mbar_expect_tx(&bar_b[pb], b_bytes);
                    bulk_g2s(sB + (size_t) pb * b_bytes, a.item_sl + (size_t) t * b_bytes, b_bytes, &bar_b[pb]);
                }
                __syncwarp();
            }
        }
        if (!ok && lane == 0) {
            *abort = 1;
            atomicExch(a.status, 1);
        }
        if (last >= 0)  // the last committed MMAs finish on their own: wait for them (bounded)
            for (int it = 0; it < (1 << 22) && !mbar_try(&bar_mma[last & 1], (uint32_t) (last >> 1) & 1u); it++) {
            }
    } else {
        // ---- epilogue ----
        const int quad = warp & 3, cg = warp >> 2, row = 32 * quad + lane;
        const int e = e_s[row], np = np_s[row], u = u_s[row];
        const float qv = e >= 0 ? a.qip[e] : 0.0f;
        const float un = e >= 0 && a.ipbound ? a.user_rnorm[u] : 0.0f;
        const float4 m0 = a.cand_meta[2 * (r0 + row)], m1 = a.cand_meta[2 * (r0 + row) + 1];
        const float Eu = m0.x, NLu = m0.w, NRu = m1.x;
        const int eu = __float_as_int(m1.y);
        const float cWL = a.cl * m0.y, cWR = a.cr * m0.z;
        const float lowq = __fsub_rn(qv, 8e-3f), highq = __fadd_rn(qv, 8e-3f);
        // The bound in real units, per (candidate, group): the digit products' distance to the
        // reference's sums (part_coef; the combination's roundings as 1.8e-7 |part| with |part| <=
        // plain norm x plain norm), plus kSigma (|left| + right) or (|left| + |rest|) for the
        // rounding of our own sum of the two terms and of the reference's, all times kSafe for the
        // roundings of this arithmetic.
        constexpr float kComb = 1.8e-7f, kSigma = 1.3e-7f, kSafe = 1.0f + 1.0f / 65536.0f;
        int cnt = 0, und = 0;
        const uint32_t lane_base = taddr + ((uint32_t) (32 * quad) << 16) + (uint32_t) (8 * cg);
        // the warp's group data of chunk i, a chunk ahead: float q of the group's 16 in lane q (one
        // coalesced load), handed out by shuffles
        const float *gmeta = reinterpret_cast<const float *>(a.grp_meta);
        auto grp = [&](int i) {
            const int64_t gi = ((int64_t) (blockIdx.x + i * gridDim.x) * kScN + 8 * cg) / kRfGroup;
            return i < mine && lane < 16 ? __ldg(gmeta + 16 * gi + lane) : 0.0f;
        };
        float gn = grp(0);
        for (int i = 0; i < mine; i++) {
            const int b = i & 1;
            const int64_t c0 = (int64_t) (blockIdx.x + i * gridDim.x) * kScN + 8 * cg;
            const float gv = gn;
            gn = grp(i + 1);
            if (!mbar_wait(&bar_mma[b], (uint32_t) (i >> 1) & 1u, abort)) {
                *abort = 1;
                atomicExch(a.status, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float l[8], r[8];
            {
                uint32_t v0[8], v1[8], v2[8], v3[8];
                const uint32_t base = lane_base + (uint32_t) b * buf_cols;
                tmem_ld8(base, v0);
                tmem_ld8(base + kScN, v1);
                tmem_ld8(base + 2 * kScN, v2);
                tmem_ld8(base + 3 * kScN, v3);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                combine4_x8(v0, v1, v2, v3, l);
                if (has_rest) {
                    tmem_ld8(base + 4 * kScN, v0);
                    tmem_ld8(base + 5 * kScN, v1);
                    tmem_ld8(base + 6 * kScN, v2);
                    tmem_ld8(base + 7 * kScN, v3);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    combine4_x8(v0, v1, v2, v3, r);
                } else {
#pragma unroll
                    for (int j = 0; j < 8; j++) r[j] = 0.0f;
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar_free[b]);
            // thresholds of this (candidate, group) in digit units: the scores are 2^(eu + eg - 35)
            // times the combined accumulators, and scaling by a power of two is exact
            const float Eg = __shfl_sync(0xffffffffu, gv, 8), WLg = __shfl_sync(0xffffffffu, gv, 9);
            const float WRg = __shfl_sync(0xffffffffu, gv, 10), NLg = __shfl_sync(0xffffffffu, gv, 11);
            const float NRg = __shfl_sync(0xffffffffu, gv, 12), IRg = __shfl_sync(0xffffffffu, gv, 13);
            const int eg = __float_as_int(__shfl_sync(0xffffffffu, gv, 14));
            const float EE = Eu * Eg;
            const float nl = NLu * NLg;
            const float DL = fmaf(cWL, WLg, fmaf(EE, a.kl, kComb * nl));
            const float inv = pow2f(35 - eu - eg);
            const int nvalid = e < 0 ? 0 : (int) max((int64_t) 0, min((int64_t) 8, (int64_t) np - c0));
            unsigned lmask = 0;  // 2 bits per column: 1 listed in full, 2 listed for its count
            if (a.ipbound) {
                const float DR = fmaf(cWR, WRg, fmaf(EE, a.kr, kComb * NRu * NRg));
                const float Ms = fmaf(kSigma, fmaf(un, IRg, nl), DL) * kSafe;
                const float Mt = fmaf(kSigma, fmaf(NRu, NRg, nl), DL + DR) * kSafe;
                const float t_sk = __fadd_rd(lowq, -Ms) * inv, t_ns = __fadd_ru(lowq, Ms) * inv;
                const float t_ct = __fadd_ru(highq, Ms) * inv, t_fu = __fadd_rd(highq, -Ms) * inv;
                const float t_hi = __fadd_ru(qv, Mt) * inv, t_mi = __fadd_rd(qv, -Mt) * inv;
                const float un_s = un * inv;
                auto pair_test = [&](int j, float s, float d, float t) {
                    const bool act = j < nvalid && !(s < t_sk);          // not surely skipped
                    const bool ns = s >= t_ns;                             // surely not skipped
                    const bool c1 = ns && d > t_ct;                        // surely counted on its bound
                    const bool f1 = ns && !c1 && d <= t_fu;                // surely scored in full
                    const bool hi = t >= t_hi, mi = t < t_mi;
                    cnt += act && (c1 || (f1 && hi));
                    und += act && f1;
                    const unsigned lf = act && !c1 && !f1, lc = act && f1 && !hi && !mi;
                    lmask |= (lf | (lc << 1)) << (2 * j);
                };
#pragma unroll
                for (int j = 0; j < 8; j += 2) {
                    // two columns per paired FP32 instruction (per component the scalar roundings):
                    // s = left + right, d = left - right, t = left + rest
                    const float2 rt2 = __fmul2_rn(make_float2(__shfl_sync(0xffffffffu, gv, j),
                                                              __shfl_sync(0xffffffffu, gv, j + 1)),
                                                  make_float2(un_s, un_s));  // the reference's right, scaled
                    const float2 l2 = make_float2(l[j], l[j + 1]);
                    const float2 s2 = __fadd2_rn(l2, rt2), d2 = __fadd2_rn(l2, make_float2(-rt2.x, -rt2.y));
                    const float2 t2 = __fadd2_rn(l2, make_float2(r[j], r[j + 1]));
                    pair_test(j, s2.x, d2.x, t2.x);
                    pair_test(j + 1, s2.y, d2.y, t2.y);
                }
            } else {
                const float M = fmaf(kSigma, nl, DL) * kSafe;
                const float t_hi = __fadd_ru(qv, M) * inv, t_lo = __fadd_rd(qv, -M) * inv;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const bool act = j < nvalid;
                    cnt += act && l[j] > t_hi;
                    const unsigned lf = act && !(l[j] > t_hi) && !(l[j] <= t_lo);
                    lmask |= lf << (2 * j);
                }
            }
            if (__any_sync(0xffffffffu, lmask != 0)) {
                // the listed pairs, appended by one atomic per column of the warp
#pragma unroll 1
                for (int j = 0; j < 8; j++) {
                    const unsigned m = (lmask >> (2 * j)) & 3u;
                    const unsigned need = __ballot_sync(0xffffffffu, m != 0);
                    if (!need) continue;
                    const int leader = __ffs(need) - 1;
                    int base = 0;
                    if (lane == leader) base = atomicAdd(a.list_count, __popc(need));
                    base = __shfl_sync(0xffffffffu, base, leader);
                    if (m) {
                        const int mode = m == 1 ? kModeFull : kModeCountOnly;
                        const int slot = base + __popc(need & ((1u << lane) - 1));
                        if (slot < a.list_cap) a.list[slot] = make_int4(e, u, (int) (c0 + j), mode);
                        else exact_pair_now(a, e, u, c0 + j, mode);
                    }
                }
            }
        }
        if (e >= 0) {
            if (cnt) atomicAdd(a.rank + e, cnt);
            if (und) atomicAdd(a.undecided + e, und);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(taddr) : "memory");
    }
}

// The listed pairs, by the reference's arithmetic.
__global__ void refine_tc_exact_kernel(TcArgs a) {
    const int n = min(*a.list_count, a.list_cap);
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int4 x = a.list[i];
        int cnt, und;
        exact_pair(a, x.x, x.y, x.z, x.w, cnt, und);
        if (cnt) atomicAdd(a.rank + x.x, cnt);
        if (und) atomicAdd(a.undecided + x.x, und);
    }
}

inline size_t carve_bytes(size_t n) { return ((n + 255) & ~size_t(255)) + 256; }
template <typename T> T *carve_at(uint8_t *&p, size_t n) {
    uintptr_t v = (reinterpret_cast<uintptr_t>(p) + 255) & ~uintptr_t(255);
    T *r = reinterpret_cast<T *>(v);
    p = reinterpret_cast<uint8_t *>(v + n * sizeof(T));
    return r;
}

// Shares of the item chunks per candidate tile: about 6-12 waves of one CTA per SM, the count whose
// last wave is fullest.
int64_t pick_shares(int64_t tiles, int64_t chunks) {
    const int64_t sms = 148;
    int64_t best = 1;
    double best_eff = -1.0;
    for (int64_t w = 6; w <= 12; w++) {
        const int64_t s = std::max<int64_t>(1, std::min<int64_t>((chunks + 7) / 8, sms * w / tiles));
        const int64_t total = s * tiles, waves = (total + sms - 1) / sms;
        const double eff = (double) total / (double) (waves * sms);
        if (eff > best_eff + 1e-9) {
            best_eff = eff;
            best = s;
        }
    }
    return best;
}

}  // namespace

// The items' digit chunks and group data for the refinement split (QS / QSRP: at check_dim, in the
// norm order; US: unsplit), built once per split and kept with the index.
int refine_tc_tiles(rkr_index *ix, bool ipbound, cudaStream_t st) {
    const int dim = ix->dim;
    const int c = ipbound ? ix->check_dim : dim;
    const int n1 = c, n2 = dim - c;
    if (n1 <= 0 || n1 > kScMaxPart || n2 > kScMaxPart) return RKR_OK;
    const int cp = round32(n1), kp = cp + round32(n2);
    if (kp > kRfMaxKp) return RKR_OK;
    const int64_t n_item = ix->n_item, item_pad = (n_item + kScN - 1) / kScN * kScN;
    DevBuf &isl = ipbound ? ix->ri_item_split : ix->ri_item_full;
    DevBuf &imeta = ipbound ? ix->ri_imeta_split : ix->ri_imeta_full;
    int &key = ipbound ? ix->ri_key_split : ix->ri_key_full;
    if (key != c) {
        key = -2;
        RKR_TRY(isl.ensure((size_t) item_pad * kScSlices * kp));
        RKR_TRY(imeta.ensure(sizeof(float4) * 4 * (size_t) (item_pad / kRfGroup)));
        rf_slice_kernel<<<(unsigned) (item_pad / kRfGroup), 256, 0, st>>>(
            ix->item_sorted.as<float>(), nullptr, n_item, dim, c, cp, kp, kScN, 1,
            ipbound ? ix->item_rnorm.as<float>() : nullptr, isl.as<int8_t>(), nullptr, imeta.as<float4>());
        RKR_CUDA(cudaGetLastError());
        key = c;
    }
    return RKR_OK;
}

int refine_tc(rkr_index *ix, const RefineArgs &ra, cudaStream_t st, bool *done) {
    *done = false;
    const int dim = ix->dim;
    const int c = ra.ipbound ? ix->check_dim : dim;
    const int n1 = c, n2 = dim - c;
    if (n1 <= 0 || n1 > kScMaxPart || n2 > kScMaxPart || ra.n_cand <= 0) return RKR_OK;
    const int cp = round32(n1), kp = cp + round32(n2);
    if (kp > kRfMaxKp) return RKR_OK;
    const int64_t n_item = ix->n_item, item_pad = (n_item + kScN - 1) / kScN * kScN;
    const int64_t cand_pad = (ra.n_cand + kScM - 1) / kScM * kScM;
    if (cand_pad / kScM > 65535) return RKR_OK;  // the exact tiles take batches this large
    RKR_TRY(refine_tc_tiles(ix, ra.ipbound != 0, st));
    DevBuf &isl = ra.ipbound ? ix->ri_item_split : ix->ri_item_full;
    DevBuf &imeta = ra.ipbound ? ix->ri_imeta_split : ix->ri_imeta_full;
    // undecided tests (a small fraction of the candidates' items); past the list they are resolved in line
    const int list_cap = (int) std::min<int64_t>(int64_t(1) << 26,
                                                 std::max<int64_t>(int64_t(1) << 20, cand_pad * n_item / 1024));
    RKR_TRY(ix->ws_tc.ensure(carve_bytes((size_t) cand_pad * kScSlices * kp) + carve_bytes(sizeof(float4) * 2 * cand_pad) +
                             carve_bytes(sizeof(int4) * (size_t) list_cap) + carve_bytes(sizeof(int) * 2)));
    uint8_t *p = ix->ws_tc.as<uint8_t>();
    int8_t *cand = carve_at<int8_t>(p, (size_t) cand_pad * kScSlices * kp);
    float4 *cand_meta = carve_at<float4>(p, 2 * cand_pad);
    int4 *list = carve_at<int4>(p, list_cap);
    int *counters = carve_at<int>(p, 2);
    RKR_CUDA(cudaMemsetAsync(counters, 0, sizeof(int) * 2, st));
    // the candidates' rows (users gathered through ref_user, whose entries past n_ref are 0)
    timed(ix, st, "refine_tc_prep", [&] {
        rf_slice_kernel<<<(unsigned) (cand_pad / kRfGroup), 256, 0, st>>>(ra.user, ra.ref_user, ra.n_cand, dim, c, cp,
                                                                          kp, kScM, 0, nullptr, cand, cand_meta,
                                                                          nullptr);
    });
    RKR_CUDA(cudaGetLastError());
    TcArgs a;
    a.cand_sl = cand;
    a.item_sl = isl.as<int8_t>();
    a.cand_meta = cand_meta;
    a.grp_meta = imeta.as<float4>();
    a.item_rnorm = ix->item_rnorm.as<float>();
    a.user_rnorm = ix->user_rnorm.as<float>();
    a.user_rows = ra.user;
    a.item_rows = ix->item_sorted.as<float>();
    a.ref_idx = ra.ref_idx;
    a.ref_user = ra.ref_user;
    a.n_ref = ra.n_ref;
    a.nproc = ra.nproc;
    a.qip = ra.qip;
    a.rank = ra.rank;
    a.undecided = ra.undecided;
    a.n_item = n_item;
    a.dim = dim;
    a.c = c;
    a.kp = kp;
    a.ksplit = cp / 32;
    a.ksteps = kp / 32;
    a.ipbound = ra.ipbound;
    part_coef(n1, a.cl, a.kl);
    part_coef(n2, a.cr, a.kr);
    a.list = list;
    a.list_count = counters;
    a.status = counters + 1;
    a.list_cap = list_cap;
    const size_t smem = (size_t) kScSlices * kp * (kScM + 2 * kScN);
    RKR_CUDA(cudaFuncSetAttribute(refine_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    const int64_t cand_tiles = cand_pad / kScM;
    const dim3 grid((unsigned) pick_shares(cand_tiles, item_pad / kScN), (unsigned) cand_tiles);
    timed(ix, st, "refine_tc", [&] { refine_tc_kernel<<<grid, kRfThreads, smem, st>>>(a); });
    RKR_CUDA(cudaGetLastError());
    timed(ix, st, "refine_tc_exact", [&] { refine_tc_exact_kernel<<<148 * 4, 256, 0, st>>>(a); });
    RKR_CUDA(cudaGetLastError());
    int h[2] = {0, 0};
    RKR_CUDA(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st));
    RKR_CUDA(cudaStreamSynchronize(st));
    if (h[1]) {
        set_error("refine_tc: tensor-core completion wait timed out");
        return RKR_ERR_CUDA;
    }
    if (ix->prof.on) ix->prof.add_count("refine_exact_pairs", h[0]);
    *done = true;
    return RKR_OK;
}

}  // namespace rkr
