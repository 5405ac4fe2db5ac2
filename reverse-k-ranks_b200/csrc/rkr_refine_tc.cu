// rkr_refine_tc.cu -- the counting step of candidate refinement on the tensor cores (tcgen05, TF32).
//
// Refinement counts, per candidate (user u, score qv) and item in the norm cut-off, the reference's
// per-item test (RefineCPUIPBound::RefineRank, RefineCPUIPBound.hpp:93-150 with the split sums of
// RefineCPUPartDimPartNorm.hpp:83-152; RefineCPU::RefineRank, RefineCPU.hpp:33-55 without the bound).
// The test only asks on which side of a few thresholds a pair's scores fall: its partial score over
// the first check_dim coordinates against lowq - right and highq + right, and its full score against
// qv.  So the scores come from TF32 tensor-core passes (the partial and the remaining coordinates in
// two TMEM accumulators), each with a bound on its distance to the reference's binary32 value; a
// pair whose bound interval straddles a threshold is listed and decided by the reference's own
// arithmetic (refine_tc_exact_kernel).
//
// Tiles.  A CTA holds 128 candidates (the MMA's M, TMEM lanes) in shared memory and walks a strided
// share of the item tiles (64 items, the MMA's N) inside its candidates' norm cut-off, the item
// operands double-buffered by bulk copies (items are stored in that tile layout) and the
// accumulators double-buffered in TMEM, so that one tile's MMAs overlap the previous tile's
// epilogue.  Warp 16 issues the copies and the MMAs; warps 0-15 run the epilogue (warp w: lane
// quadrant w % 4, columns 16 (w / 4) .. + 16).
//
// Error bound.  Operands are rounded to TF32 (11 significant bits, round to nearest), so each
// product is within 2^-10 (1 + 2^-12) |a b| of the exact one; the FP32 accumulation of a K step of
// eight products into the accumulator is taken to cost at most 9 ulps of sum |a b| per step (each
// product aligned with less than an ulp lost, one final rounding) plus 8; and the reference's
// sequential sum of n terms at most n * 2^-24 / (1 - n 2^-24) sum |a b|.  Sum |a b| <= |a| |b|
// (Cauchy-Schwarz) over each part.  The TF32 term dominates: the accumulation term is under 3% of it.
#include <algorithm>
#include <cstdio>

#include "rkr_internal.cuh"

namespace rkr {

namespace {

constexpr int kTcTile = 128;     // candidates per CTA (TMEM lanes)
constexpr int kTcN = 64;         // items per tile (MMA N)
constexpr int kTcEpiWarps = 16;  // warp w reads TMEM lane quadrant w % 4, columns 16 (w / 4) + [0, 16)
constexpr int kTcThreads = 32 * (kTcEpiWarps + 1);
constexpr int kTcMaxK = 208;     // the candidate tile and two item tiles fit in shared memory up to this K

__host__ __device__ inline int round8(int x) { return (x + 7) & ~7; }

// Nearest TF32 value (ties to even); infinities and NaN pass through.
__device__ __forceinline__ float tf32_rne(float x) {
    uint32_t u = __float_as_uint(x);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;
    u = (u + 0xfffu + ((u >> 13) & 1u)) & ~0x1fffu;
    return __uint_as_float(u);
}

// Rows [n][dim] (gathered through idx when given) to TF32 rows of kp values: coordinates [0, c) at
// [0, c), coordinates [c, dim) at [c8, c8 + dim - c), zeros elsewhere; rows [n, n_pad) zero.  norms
// gets (|first c coordinates|, |remaining coordinates|) of the unrounded row.  tiled: rows stored
// as tiles of kTcN in the shared-memory layout of an MMA operand (element (r, k) of a tile at
// ((k / 4) * (kTcN / 8) + r / 8) * 32 + (r % 8) * 4 + k % 4), else [n_pad][kp].  One warp per row.
__global__ void tc_operand_kernel(const float *__restrict__ src, const int32_t *__restrict__ idx, int64_t n,
                                  int64_t n_pad, int dim, int c, int c8, int kp, float *__restrict__ dst,
                                  float2 *__restrict__ norms, int tiled) {
    const int64_t r = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n_pad) return;
    const float *row = r < n ? src + (idx ? (int64_t) idx[r] : r) * dim : nullptr;
    float sl = 0.0f, sr = 0.0f;
    for (int p = lane; p < kp; p += 32) {
        const int k = p < c8 ? (p < c ? p : -1) : (p - c8 + c < dim ? p - c8 + c : -1);
        float v = 0.0f;
        if (row && k >= 0) {
            v = row[k];
            if (k < c) sl = fmaf(v, v, sl);
            else sr = fmaf(v, v, sr);
        }
        const int64_t at = tiled ? (r / kTcN) * kTcN * kp + ((p >> 2) * (kTcN / 8) + (r % kTcN) / 8) * 32 +
                                       (r & 7) * 4 + (p & 3)
                                 : r * kp + p;
        dst[at] = tf32_rne(v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        sl += __shfl_xor_sync(0xffffffffu, sl, o);
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
    }
    if (lane == 0) norms[r] = make_float2(sqrtf(sl), sqrtf(sr));
}

// ---- tcgen05 helpers ----------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, K-major without swizzle: 8-row x 16-byte core matrices, lbo the
// byte distance between the two core matrices of a K step, sbo between groups of 8 rows.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t) ((saddr >> 4) & 0x3FFF);
    d |= (uint64_t) ((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t) ((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t) 1 << 46;  // descriptor version of sm_100
    return d;
}

// Instruction descriptor: kind::tf32, A and B K-major TF32, FP32 accumulator, M = 128, N = 64.
constexpr uint32_t kIdescTf32 = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t) (kTcN >> 3) << 17) |
                                ((uint32_t) (kTcTile >> 4) << 24);

__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(d_tmem), "l"(a), "l"(b), "r"(kIdescTf32), "r"(accumulate) : "memory");
}

__device__ __forceinline__ void tmem_ld4(uint32_t addr, uint32_t (&v)[4]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3])
                 : "r"(addr));
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(addr));
}

__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok) : "r"(smem_u32(b)), "r"(parity) : "memory");
    return ok != 0;
}
// Bounded wait; gives up early when another thread of the CTA has given up.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, volatile int *abort) {
    for (int it = 0; it < (1 << 22); it++) {
        if (mbar_try(b, parity)) return true;
        if (*abort) return false;
    }
    return false;
}
// Plain (non-multicast) bulk copy global -> this CTA's shared memory, completing on an mbarrier.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
          "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
          "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(addr));
}

// ---- the tile kernel -------------------------------------------------------------------------------

struct TcArgs {
    const float *cand, *item;                  // TF32 operands, [rows][kp]
    const float2 *cand_norm, *item_norm;       // norms of the two parts
    const float *item_rnorm, *user_rnorm;      // the reference's remaining-coordinate norms (bound test)
    const float *user_rows, *item_rows;        // exact rows for undecided pairs (item_rows in the item order)
    const int32_t *ref_idx, *ref_user, *n_ref, *nproc;
    const float *qip;
    int32_t *rank, *undecided;
    int64_t n_item;
    int dim, c, c8, kp, ipbound;
    float err_l, err_r;                        // bound coefficients of the two parts
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

__global__ void __launch_bounds__(kTcThreads, 1) refine_tc_kernel(TcArgs a) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ uint64_t bar_b[2], bar_mma[2], bar_free[2];
    __shared__ uint32_t tslot;
    __shared__ int e_s[kTcTile], np_s[kTcTile], u_s[kTcTile], max_np, abort_flag;
    __shared__ float qv_s[kTcTile], un_s[kTcTile];
    __shared__ float2 an_s[kTcTile];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t r0 = (int64_t) blockIdx.y * kTcTile;
    const int n_ref = *a.n_ref;
    if (r0 >= n_ref) return;
    volatile int *abort = &abort_flag;
    if (tid < kTcTile) {
        const int64_t r = r0 + tid;
        int e = -1, np = 0, u = 0;
        float qv = 0.0f, un = 0.0f;
        float2 an = make_float2(0.0f, 0.0f);
        if (r < n_ref) {
            e = a.ref_idx[r];
            np = a.nproc[e];
            qv = a.qip[e];
            u = a.ref_user[r];
            un = a.ipbound ? a.user_rnorm[u] : 0.0f;
            an = a.cand_norm[r];
        }
        e_s[tid] = e; np_s[tid] = np; u_s[tid] = u; qv_s[tid] = qv; un_s[tid] = un; an_s[tid] = an;
    }
    if (tid == 0) {
        max_np = 0;
        abort_flag = 0;
    }
    __syncthreads();
    if (tid < kTcTile) atomicMax(&max_np, np_s[tid]);
    __syncthreads();
    // this CTA's item tiles: s, s + gridDim.x, ... below the candidates' largest cut-off
    const int n_tiles = (max_np + kTcN - 1) / kTcN;
    const int my_tiles = n_tiles > (int) blockIdx.x ? (n_tiles - (int) blockIdx.x + (int) gridDim.x - 1) / (int) gridDim.x : 0;
    if (my_tiles == 0) return;

    // candidates into shared memory as K-major core matrices: element (row r, k) at
    // ((k / 4) * 16 + r / 8) * 128 + (r % 8) * 16 + (k % 4) * 4 bytes; then two item tile buffers
    const int kp = a.kp, ch = kp / 4;
    float *sa = reinterpret_cast<float *>(tc_smem);
    uint8_t *sb = reinterpret_cast<uint8_t *>(sa + kTcTile * kp);
    const uint32_t b_bytes = (uint32_t) (sizeof(float) * kTcN * kp);
    for (int idx = tid; idx < kTcTile * ch; idx += kTcThreads) {
        const int r = idx / ch, j = idx % ch;
        const int off = (j * (kTcTile / 8) + (r >> 3)) * 32 + (r & 7) * 4;
        cp_async16(sa + off, a.cand + (r0 + r) * kp + 4 * j, true);
    }
    cp_async_commit();
    cp_async_wait<0>();
    if (tid == 0) {
        for (int b = 0; b < 2; b++) {
            mbar_init(&bar_b[b], 1);
            mbar_init(&bar_mma[b], 1);
            mbar_init(&bar_free[b], kTcEpiWarps);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(&tslot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t taddr = tslot;
    const int ksplit = a.c8 / 8, ksteps = kp / 8;
    const uint8_t *item_tiles = reinterpret_cast<const uint8_t *>(a.item);

    if (warp == kTcEpiWarps) {
        // ---- copies and MMAs (one thread) ----
        if (lane == 0) {
            bool ok = true;
            int last = -1;
            for (int i = 0; i < 2 && i < my_tiles; i++) {
                const int t = blockIdx.x + i * gridDim.x;
                mbar_expect_tx(&bar_b[i], b_bytes);
                bulk_g2s(sb + (size_t) i * b_bytes, item_tiles + (size_t) t * b_bytes, b_bytes, &bar_b[i]);
            }
            constexpr uint32_t kAChunk = (kTcTile / 8) * 128, kBChunk = (kTcN / 8) * 128;  // bytes per 4-value k chunk
            for (int i = 0; ok && i < my_tiles; i++) {
                const int b = i & 1;
                const uint32_t ph = (uint32_t) (i >> 1) & 1u;
                ok = mbar_wait(&bar_b[b], ph, abort);
                if (ok && i >= 2) ok = mbar_wait(&bar_free[b], (uint32_t) ((i - 2) >> 1) & 1u, abort);
                if (!ok) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d0 = taddr + (uint32_t) b * (2 * kTcN);
                const uint32_t sb0 = smem_u32(sb + (size_t) b * b_bytes);
                for (int s = 0; s < ksteps; s++) {
                    const uint64_t da = umma_desc(smem_u32(sa) + (uint32_t) s * 2 * kAChunk, kAChunk, 128);
                    const uint64_t db = umma_desc(sb0 + (uint32_t) s * 2 * kBChunk, kBChunk, 128);
                    if (s < ksplit) umma_tf32(d0, da, db, s > 0);
                    else umma_tf32(d0 + kTcN, da, db, s > ksplit);
                }
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_u32(&bar_mma[b]))
                             : "memory");
                last = i;
                if (i >= 1 && i + 1 < my_tiles) {
                    // the previous tile's MMAs have read their items: refill that buffer
                    const int pb = (i - 1) & 1;
                    ok = mbar_wait(&bar_mma[pb], (uint32_t) ((i - 1) >> 1) & 1u, abort);
                    if (!ok) break;
                    const int t = blockIdx.x + (i + 1) * gridDim.x;
                    mbar_expect_tx(&bar_b[pb], b_bytes);
                    bulk_g2s(sb + (size_t) pb * b_bytes, item_tiles + (size_t) t * b_bytes, b_bytes, &bar_b[pb]);
                }
            }
            if (!ok) {
                *abort = 1;
                atomicExch(a.status, 1);
            }
            if (last >= 0)  // the last committed MMAs finish on their own: wait for them (bounded)
                for (int it = 0; it < (1 << 22) && !mbar_try(&bar_mma[last & 1], (uint32_t) (last >> 1) & 1u); it++) {
                }
        }
    } else {
        // ---- epilogue ----
        const int quad = warp & 3, cg = warp >> 2, row = 32 * quad + lane;
        const int e = e_s[row], np = np_s[row], u = u_s[row];
        const float qv = qv_s[row], un = un_s[row];
        const float2 an = an_s[row];
        const float lowq = __fsub_rn(qv, 8e-3f), highq = __fadd_rn(qv, 8e-3f);
        const bool has_rest = ksteps > ksplit;
        constexpr float kSlack = 4e-7f;  // a few roundings here and in the reference's one add
        int cnt = 0, und = 0;
        const uint32_t lane_base = taddr + ((uint32_t) (32 * quad) << 16) + (uint32_t) (16 * cg);
        // the items' norms of this warp's 16 columns, one column per lane (lanes 0-15), loaded a tile
        // ahead and broadcast by shuffles
        auto col_norms = [&](int i, float &nx, float &ny, float &rn) {
            const int64_t it = (int64_t) (blockIdx.x + i * gridDim.x) * kTcN + 16 * cg + (lane & 15);
            const bool in = i < my_tiles && it < a.n_item;
            const float2 v = in ? __ldg(a.item_norm + it) : make_float2(0.0f, 0.0f);
            nx = v.x;
            ny = v.y;
            rn = in && a.ipbound ? __ldg(a.item_rnorm + it) : 0.0f;
        };
        float nx_next, ny_next, rn_next;
        col_norms(0, nx_next, ny_next, rn_next);
        for (int i = 0; i < my_tiles; i++) {
            const int b = i & 1;
            const int64_t c0 = (int64_t) (blockIdx.x + i * gridDim.x) * kTcN + 16 * cg;
            const float nx_cur = nx_next, ny_cur = ny_next, rn_cur = rn_next;
            col_norms(i + 1, nx_next, ny_next, rn_next);
            if (!mbar_wait(&bar_mma[b], (uint32_t) (i >> 1) & 1u, abort)) {
                *abort = 1;
                atomicExch(a.status, 1);
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t tbase = lane_base + (uint32_t) b * (2 * kTcN);
            // four columns at a time (a compact loop body keeps the instruction cache warm); the
            // accumulators are released after the last of them
#pragma unroll 1
            for (int j0 = 0; j0 < 16; j0 += 4) {
                uint32_t L[4], R[4] = {0u, 0u, 0u, 0u};
                tmem_ld4(tbase + (uint32_t) j0, L);
                if (has_rest) tmem_ld4(tbase + kTcN + (uint32_t) j0, R);
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int jj = 0; jj < 4; jj++) {
                    const int64_t it = c0 + j0 + jj;
                    const bool valid = e >= 0 && it < np;
                    const float left = __uint_as_float(L[jj]);
                    const float2 bn = make_float2(__shfl_sync(0xffffffffu, nx_cur, j0 + jj),
                                                  __shfl_sync(0xffffffffu, ny_cur, j0 + jj));
                    const float irn = __shfl_sync(0xffffffffu, rn_cur, j0 + jj);
                    const float dl = a.err_l * an.x * bn.x;
                    int mode = -1;  // -1: settled here; else the mode of the exact resolution
                    if (a.ipbound) {
                        const float rest = __uint_as_float(R[jj]);
                        const float right = __fmul_rn(irn, un);
                        const float ub_hi = (left + dl) + right, ub_lo = (left - dl) + right;
                        const float lb_hi = (left + dl) - right, lb_lo = (left - dl) - right;
                        const bool skip = lowq > ub_hi + fabsf(ub_hi) * kSlack;       // skipped by the reference
                        const bool noskip = lowq <= ub_lo - fabsf(ub_lo) * kSlack;
                        const bool counted = noskip && highq < lb_lo - fabsf(lb_lo) * kSlack;  // counted on its bound
                        const bool full = noskip && highq >= lb_hi + fabsf(lb_hi) * kSlack;    // scored in full
                        const float tot = left + rest;
                        const float dt = dl + a.err_r * an.y * bn.y + fabsf(tot) * kSlack;
                        const bool hit = tot - dt >= qv, miss = tot + dt < qv;
                        if (valid && !skip) {
                            if (counted) cnt++;
                            else if (full) {
                                und++;
                                cnt += hit;
                                if (!hit && !miss) mode = kModeCountOnly;
                            } else {
                                mode = kModeFull;
                            }
                        }
                    } else {
                        const float d = dl + fabsf(left) * kSlack;
                        if (valid) {
                            if (left - d > qv) cnt++;
                            else if (left + d > qv) mode = kModeFull;
                        }
                    }
                    const unsigned need = __ballot_sync(0xffffffffu, mode >= 0);
                    if (need) {
                        const int leader = __ffs(need) - 1;
                        int base = 0;
                        if (lane == leader) base = atomicAdd(a.list_count, __popc(need));
                        base = __shfl_sync(0xffffffffu, base, leader);
                        if (mode >= 0) {
                            const int slot = base + __popc(need & ((1u << lane) - 1));
                            if (slot < a.list_cap) a.list[slot] = make_int4(e, u, (int) it, mode);
                            else exact_pair_now(a, e, u, it, mode);
                        }
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar_free[b]);
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(taddr) : "memory");
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

// Bound coefficient of a part of n coordinates taken in `steps` tensor-core K steps.
inline float part_err(int n, int steps) {
    const double tf32 = 9.765625e-4 * (1.0 + 1.0 / 4096.0);          // 2^-10 (1 + 2^-12)
    const double acc = (9.0 * steps + 8) * 1.1920928955078125e-7;    // 9 ulps of FP32 per K step, plus 8
    const double ref = n * 5.9604644775390625e-8 / (1.0 - n * 5.96e-8);  // the reference's sequential sum
    return (float) ((tf32 + acc + ref) * 1.01);
}

}  // namespace

int refine_tc(rkr_index *ix, const RefineArgs &ra, cudaStream_t st, bool *done) {
    *done = false;
    const int dim = ix->dim;
    const int c = ra.ipbound ? ix->check_dim : dim;
    const int c8 = round8(c), kp = c8 + round8(dim - c);
    if (kp > kTcMaxK || ra.n_cand <= 0) return RKR_OK;
    const int64_t n_item = ix->n_item, item_pad = (n_item + kTcN - 1) / kTcN * kTcN;
    // item operands for the current check_dim
    if (ix->tc_check_dim != ix->check_dim) {
        const int cs = ix->check_dim, cs8 = round8(cs), kps = cs8 + round8(dim - cs), kpu = round8(dim);
        RKR_TRY(ix->item_tc.ensure(sizeof(float) * (size_t) item_pad * kps));
        RKR_TRY(ix->item_tc_norm.ensure(sizeof(float2) * (size_t) item_pad));
        RKR_TRY(ix->item_tc_us.ensure(sizeof(float) * (size_t) item_pad * kpu));
        RKR_TRY(ix->item_tc_us_norm.ensure(sizeof(float2) * (size_t) item_pad));
        const unsigned g = (unsigned) ((item_pad * 32 + 255) / 256);
        tc_operand_kernel<<<g, 256, 0, st>>>(ix->item_sorted.as<float>(), nullptr, n_item, item_pad, dim, cs, cs8, kps,
                                             ix->item_tc.as<float>(), ix->item_tc_norm.as<float2>(), 1);
        RKR_CUDA(cudaGetLastError());
        tc_operand_kernel<<<g, 256, 0, st>>>(ix->item.as<float>(), nullptr, n_item, item_pad, dim, dim, kpu, kpu,
                                             ix->item_tc_us.as<float>(), ix->item_tc_us_norm.as<float2>(), 1);
        RKR_CUDA(cudaGetLastError());
        ix->tc_check_dim = ix->check_dim;
    }
    const int64_t cand_pad = (ra.n_cand + kTcTile - 1) / kTcTile * kTcTile;
    // undecided tests (about 0.4% of the candidates' items); past the list they are resolved in line
    const int list_cap = (int) std::min<int64_t>(int64_t(1) << 26,
                                                 std::max<int64_t>(int64_t(1) << 22, cand_pad * n_item / 128));
    RKR_TRY(ix->ws_tc.ensure(carve_bytes(sizeof(float) * (size_t) cand_pad * kp) + carve_bytes(sizeof(float2) * cand_pad) +
                             carve_bytes(sizeof(int4) * (size_t) list_cap) + carve_bytes(sizeof(int) * 2)));
    uint8_t *p = ix->ws_tc.as<uint8_t>();
    float *cand = carve_at<float>(p, (size_t) cand_pad * kp);
    float2 *cand_norm = carve_at<float2>(p, cand_pad);
    int4 *list = carve_at<int4>(p, list_cap);
    int *counters = carve_at<int>(p, 2);
    RKR_CUDA(cudaMemsetAsync(counters, 0, sizeof(int) * 2, st));
    timed(ix, st, "refine_tc_prep", [&] {
        tc_operand_kernel<<<(unsigned) ((cand_pad * 32 + 255) / 256), 256, 0, st>>>(ra.user, ra.ref_user, ra.n_cand,
                                                                                    cand_pad, dim, c, c8, kp, cand,
                                                                                    cand_norm, 0);
    });
    RKR_CUDA(cudaGetLastError());
    TcArgs a;
    a.cand = cand;
    a.cand_norm = cand_norm;
    a.item = ra.ipbound ? ix->item_tc.as<float>() : ix->item_tc_us.as<float>();
    a.item_norm = ra.ipbound ? ix->item_tc_norm.as<float2>() : ix->item_tc_us_norm.as<float2>();
    a.item_rnorm = ix->item_rnorm.as<float>();
    a.user_rnorm = ix->user_rnorm.as<float>();
    a.user_rows = ra.user;
    a.item_rows = ra.ipbound ? ix->item_sorted.as<float>() : ix->item.as<float>();
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
    a.c8 = c8;
    a.kp = kp;
    a.ipbound = ra.ipbound;
    a.err_l = part_err(c, c8 / 8);
    a.err_r = part_err(dim - c, (kp - c8) / 8);
    a.list = list;
    a.list_count = counters;
    a.status = counters + 1;
    a.list_cap = list_cap;
    const size_t smem = sizeof(float) * (kTcTile + 2 * kTcN) * (size_t) kp;
    RKR_CUDA(cudaFuncSetAttribute(refine_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem));
    // candidate tiles x strided shares of the item tiles: about two waves of CTAs
    const int64_t cand_tiles = cand_pad / kTcTile;
    const int64_t item_tiles = item_pad / kTcN;
    const int64_t shares = std::max<int64_t>(1, std::min<int64_t>(item_tiles, (2 * 148 + cand_tiles - 1) / cand_tiles));
    const dim3 grid((unsigned) shares, (unsigned) cand_tiles);
    if (grid.y > 65535) return RKR_OK;  // the exact tiles take batches this large
    timed(ix, st, "refine_tc", [&] { refine_tc_kernel<<<grid, kTcThreads, smem, st>>>(a); });
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
