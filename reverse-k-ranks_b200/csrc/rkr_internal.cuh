// rkr_internal.cuh -- shared device code and the index handle of librkr_b200.
//
// Arithmetic contract: every dot product that decides a bound, a prune, a rank or a reported score
// is evaluated exactly as the reference evaluates InnerProduct (src/include/alg/SpaceInnerProduct.hpp:14-20):
// acc = 0; for j in order: acc = acc + a[j]*b[j], each product and sum rounded to binary32 (no FMA,
// no reassociation).  __fmul_rn/__fadd_rn are never contracted by nvcc, so the kernels reproduce
// the reference's float results bit for bit while running as register-tiled SIMT "GEMMs".
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "rkr.h"

namespace rkr {

// ---- errors ---------------------------------------------------------------------------------------

void set_error(const char *fmt, ...);

#define RKR_CUDA(call)                                                                       \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            ::rkr::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call, cudaGetErrorString(e_)); \
            return RKR_ERR_CUDA;                                                             \
        }                                                                                    \
    } while (0)

#define RKR_TRY(expr)                      \
    do {                                   \
        int s_ = (expr);                   \
        if (s_ != RKR_OK) return s_;       \
    } while (0)

#define RKR_REQUIRE(cond, ...)                  \
    do {                                        \
        if (!(cond)) {                          \
            ::rkr::set_error(__VA_ARGS__);      \
            return RKR_ERR_INVALID;             \
        }                                       \
    } while (0)

// ---- device buffers -------------------------------------------------------------------------------

// Grow-only device buffer owned by an index.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    // Grows with 25% headroom so batches of slightly varying size do not reallocate (each
    // reallocation synchronises the device).
    int ensure(size_t want) {
        if (want <= bytes) return RKR_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        if (want == 0) return RKR_OK;
        want += want / 4 + 4096;
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc(%zu) failed: %s", want, cudaGetErrorString(e));
            return RKR_ERR_NOMEM;
        }
        bytes = want;
        return RKR_OK;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    template <typename T> T *as() const { return static_cast<T *>(p); }
};

// ---- exact register-tiled dot-product tiles ----------------------------------------------------------

constexpr int kTile = 64;      // rows of A and columns of B per CTA
constexpr int kKChunk = 32;    // k staged through shared memory per step
constexpr int kPad = 4;        // shared-memory row padding (keeps float4 alignment)
constexpr int kTileThreads = 256;

// Shared operand tiles, k-major so four consecutive rows (or columns) load as one float4.
struct TileSmem {
    float a[kKChunk][kTile + kPad];
    float b[kKChunk][kTile + kPad];
};

// Computes, for the CTA's 64 x 64 block of (row of A, row of B) pairs, the sequential binary32 dot
// products over k in [k_begin, k_split) into `lo` and over [k_split, k_end) into `hi` (each
// accumulated from 0, as the reference accumulates its partial sums).  Rows of A may be gathered through
// a_idx.  Thread (tx, ty) owns rows a0 + 4*tx + i and columns b0 + 4*ty + j.
__device__ __forceinline__ void exact_tile(TileSmem &sm, const float *__restrict__ A, const int32_t *__restrict__ a_idx,
                                          int64_t n_a, int lda, int64_t a0, const float *__restrict__ B, int64_t n_b,
                                          int ldb, int64_t b0, int k_begin, int k_split, int k_end, float lo[4][4],
                                          float hi[4][4]) {
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) lo[i][j] = 0.0f, hi[i][j] = 0.0f;
    for (int k0 = k_begin; k0 < k_end; k0 += kKChunk) {
        const int kc = min(kKChunk, k_end - k0);
        __syncthreads();
        for (int idx = tid; idx < kTile * kKChunk; idx += kTileThreads) {
            const int r = idx / kKChunk, kk = idx % kKChunk;
            float va = 0.0f, vb = 0.0f;
            if (kk < kc) {
                const int64_t ra = a0 + r, rb = b0 + r;
                if (ra < n_a) {
                    const int64_t row = a_idx ? (int64_t) a_idx[ra] : ra;
                    va = __ldg(A + row * lda + k0 + kk);
                }
                if (rb < n_b) vb = __ldg(B + rb * ldb + k0 + kk);
            }
            sm.a[kk][r] = va;
            sm.b[kk][r] = vb;
        }
        __syncthreads();
        // The chunk may straddle k_split: the first part feeds `lo`, the rest `hi`.
        const int ks = min(max(k_split - k0, 0), kc);
        for (int kk = 0; kk < ks; kk++) {
            const float4 a = *reinterpret_cast<const float4 *>(&sm.a[kk][4 * tx]);
            const float4 b = *reinterpret_cast<const float4 *>(&sm.b[kk][4 * ty]);
            const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) lo[i][j] = __fadd_rn(lo[i][j], __fmul_rn(av[i], bv[j]));
        }
        for (int kk = ks; kk < kc; kk++) {
            const float4 a = *reinterpret_cast<const float4 *>(&sm.a[kk][4 * tx]);
            const float4 b = *reinterpret_cast<const float4 *>(&sm.b[kk][4 * ty]);
            const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) hi[i][j] = __fadd_rn(hi[i][j], __fmul_rn(av[i], bv[j]));
        }
    }
}

// ---- 128 x 128 exact tiles ------------------------------------------------------------------------
//
// The bulk form of exact_tile: each CTA computes a 128 x 128 block of dot products over
// k in [k_begin, k_end), each thread an 8 x 8 register block, with the k range staged through a
// double-buffered shared-memory pipeline (cp.async).  Products and sums stay separately rounded and
// in k order, so every value is the reference's InnerProduct bit for bit; zero-filled padding k
// adds +0.0, which leaves a sum that starts at +0.0 unchanged.  The finished block goes through
// shared memory to an epilogue functor that visits the pairs with consecutive threads on
// consecutive A rows, so outputs indexed [b][a] are written coalesced.

constexpr int kBig = 128, kBigK = 16, kBigPad = 4, kBigThreads = 256;
// k steps unrolled per iteration of the inner loop (the body is 128 FP32 instructions per step;
// full unrolling of a stage overflows the instruction cache).
#ifndef RKR_BIG_KK_UNROLL
#define RKR_BIG_KK_UNROLL 4
#endif
constexpr int kBigKUnroll = RKR_BIG_KK_UNROLL;

struct BigOperands {
    float a[2][kBigK][kBig + kBigPad];
    float b[2][kBigK][kBig + kBigPad];
};
struct BigResult {
    float v[kBig][kBig + kBigPad];  // [b row][a row]
};
constexpr size_t kBigSmem = sizeof(BigResult) > sizeof(BigOperands) ? sizeof(BigResult) : sizeof(BigOperands);

__device__ __forceinline__ void cp_async4(float *smem, const float *gmem, bool valid) {
    const unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__device__ __forceinline__ void big_load_stage(BigOperands &op, int buf, const float *__restrict__ A,
                                               const int32_t *__restrict__ a_rows, int64_t n_a, int lda, int64_t a0,
                                               const float *__restrict__ B, int64_t n_b, int ldb, int64_t b0, int k0,
                                               int k_end) {
#pragma unroll 1
    for (int t = 0; t < (kBig * kBigK) / kBigThreads; t++) {
        const int idx = threadIdx.x + t * kBigThreads;
        const int r = idx / kBigK, kk = idx % kBigK;
        const int k = k0 + kk;
        const int64_t ra = a0 + r, rb = b0 + r;
        const bool va = ra < n_a && k < k_end, vb = rb < n_b && k < k_end;
        const int64_t row = va ? (a_rows ? (int64_t) a_rows[r] : ra) : 0;
        cp_async4(&op.a[buf][kk][r], va ? A + row * lda + k : A, va);
        cp_async4(&op.b[buf][kk][r], vb ? B + rb * ldb + k : B, vb);
    }
}

// Accumulates into acc (zeroed here) the thread's 8 x 8 block of dot products over [k_begin, k_end):
// A rows a0 + 4 tx + {0..3, 64..67} (or, with a_rows, the rows a_rows[4 tx + ...] of the tile's
// gather list), B rows b0 + 4 ty + {0..3, 64..67}.  Returns after a barrier, with the operand
// buffers free.  Returns false (no barrier, acc zero) for an empty range.
__device__ __forceinline__ bool big_accumulate(BigOperands &op, float acc[8][8], const float *__restrict__ A,
                                              const int32_t *__restrict__ a_rows, int64_t n_a, int lda, int64_t a0,
                                              const float *__restrict__ B, int64_t n_b, int ldb, int64_t b0, int k_begin,
                                              int k_end) {
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
    const int ns = (k_end - k_begin + kBigK - 1) / kBigK;
    if (ns <= 0) return false;
    big_load_stage(op, 0, A, a_rows, n_a, lda, a0, B, n_b, ldb, b0, k_begin, k_end);
    cp_async_commit();
    for (int s = 0; s < ns; s++) {
        if (s + 1 < ns) {
            big_load_stage(op, (s + 1) & 1, A, a_rows, n_a, lda, a0, B, n_b, ldb, b0, k_begin + (s + 1) * kBigK, k_end);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int buf = s & 1;
#pragma unroll kBigKUnroll
        for (int kk = 0; kk < kBigK; kk++) {
            const float4 a_lo = *reinterpret_cast<const float4 *>(&op.a[buf][kk][4 * tx]);
            const float4 a_hi = *reinterpret_cast<const float4 *>(&op.a[buf][kk][64 + 4 * tx]);
            const float4 b_lo = *reinterpret_cast<const float4 *>(&op.b[buf][kk][4 * ty]);
            const float4 b_hi = *reinterpret_cast<const float4 *>(&op.b[buf][kk][64 + 4 * ty]);
            const float av[8] = {a_lo.x, a_lo.y, a_lo.z, a_lo.w, a_hi.x, a_hi.y, a_hi.z, a_hi.w};
            const float bv[8] = {b_lo.x, b_lo.y, b_lo.z, b_lo.w, b_hi.x, b_hi.y, b_hi.z, b_hi.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(av[i], bv[j]));
        }
        __syncthreads();
    }
    return true;
}

// Writes (add = false) or adds with one binary32 rounding (add = true) the thread's block into res.
__device__ __forceinline__ void big_store(BigResult &res, const float acc[8][8], bool add) {
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int cb = (j < 4 ? 0 : 64) + 4 * ty + (j & 3);
        float4 *lo = reinterpret_cast<float4 *>(&res.v[cb][4 * tx]);
        float4 *hi = reinterpret_cast<float4 *>(&res.v[cb][64 + 4 * tx]);
        float4 l = make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
        float4 h = make_float4(acc[4][j], acc[5][j], acc[6][j], acc[7][j]);
        if (add) {
            const float4 l0 = *lo, h0 = *hi;
            l = make_float4(__fadd_rn(l0.x, l.x), __fadd_rn(l0.y, l.y), __fadd_rn(l0.z, l.z), __fadd_rn(l0.w, l.w));
            h = make_float4(__fadd_rn(h0.x, h.x), __fadd_rn(h0.y, h.y), __fadd_rn(h0.z, h.z), __fadd_rn(h0.w, h.w));
        }
        *lo = l;
        *hi = h;
    }
}

// Fills res with the 128 x 128 block of dot products (A rows a0.., or a_idx[0..127] as a tile-local
// gather list, B rows b0..) over [k_begin, k_end).
__device__ __forceinline__ void exact_big_tile(char *smem, const float *__restrict__ A, const int32_t *__restrict__ a_idx,
                                              int64_t n_a, int lda, int64_t a0, const float *__restrict__ B,
                                              int64_t n_b, int ldb, int64_t b0, int k_begin, int k_end) {
    BigOperands &op = *reinterpret_cast<BigOperands *>(smem);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
    const int ns = (k_end - k_begin + kBigK - 1) / kBigK;
    if (ns > 0) {
        big_load_stage(op, 0, A, a_idx, n_a, lda, a0, B, n_b, ldb, b0, k_begin, k_end);
        cp_async_commit();
    }
    for (int s = 0; s < ns; s++) {
        if (s + 1 < ns) {
            big_load_stage(op, (s + 1) & 1, A, a_idx, n_a, lda, a0, B, n_b, ldb, b0, k_begin + (s + 1) * kBigK, k_end);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int buf = s & 1;
#pragma unroll kBigKUnroll
        for (int kk = 0; kk < kBigK; kk++) {
            const float4 a_lo = *reinterpret_cast<const float4 *>(&op.a[buf][kk][4 * tx]);
            const float4 a_hi = *reinterpret_cast<const float4 *>(&op.a[buf][kk][64 + 4 * tx]);
            const float4 b_lo = *reinterpret_cast<const float4 *>(&op.b[buf][kk][4 * ty]);
            const float4 b_hi = *reinterpret_cast<const float4 *>(&op.b[buf][kk][64 + 4 * ty]);
            const float av[8] = {a_lo.x, a_lo.y, a_lo.z, a_lo.w, a_hi.x, a_hi.y, a_hi.z, a_hi.w};
            const float bv[8] = {b_lo.x, b_lo.y, b_lo.z, b_lo.w, b_hi.x, b_hi.y, b_hi.z, b_hi.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(av[i], bv[j]));
        }
        __syncthreads();
    }
    BigResult &res = *reinterpret_cast<BigResult *>(smem);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const int cb = (j < 4 ? 0 : 64) + 4 * ty + (j & 3);
        *reinterpret_cast<float4 *>(&res.v[cb][4 * tx]) = make_float4(acc[0][j], acc[1][j], acc[2][j], acc[3][j]);
        *reinterpret_cast<float4 *>(&res.v[cb][64 + 4 * tx]) = make_float4(acc[4][j], acc[5][j], acc[6][j], acc[7][j]);
    }
    __syncthreads();
}

// Grid: x over B tiles, y over A tiles.  Epi provides: static constexpr size_t kExtra (extra shared
// bytes), prologue(extra, a0, b0), active(extra, a0, b0) (false skips the dot products) and
// finish(extra, res, a0, b0, live), which reads the block from res.v[b - b0][a - a0].  The usual
// finish is row-owned: thread t takes A row a0 + (t % 128) and B rows b0 + t / 128 + 2 i, so a
// warp writes 32 consecutive A rows of one B row at a time.
template <class Epi>
__global__ void __launch_bounds__(kBigThreads, 2) exact_big_kernel(const float *__restrict__ A,
                                                                   const int32_t *__restrict__ a_idx, int64_t n_a,
                                                                   int lda, const float *__restrict__ B, int64_t n_b,
                                                                   int ldb, int k_begin, int k_end, Epi epi) {
    extern __shared__ __align__(16) char big_smem[];
    char *extra = big_smem + kBigSmem;
    const int64_t b0 = (int64_t) blockIdx.x * kBig;
    const int64_t a0 = (int64_t) blockIdx.y * kBig;
    __shared__ int32_t rows_s[kBig];  // the tile's gathered A rows
    if (a_idx && threadIdx.x < kBig) rows_s[threadIdx.x] = a0 + threadIdx.x < n_a ? a_idx[a0 + threadIdx.x] : 0;
    epi.prologue(extra, a0, b0);
    __syncthreads();
    const bool live = epi.active(extra, a0, b0);
    if (live) exact_big_tile(big_smem, A, a_idx ? rows_s : nullptr, n_a, lda, a0, B, n_b, ldb, b0, k_begin, k_end);
    epi.finish(extra, *reinterpret_cast<const BigResult *>(big_smem), a0, b0, live);
}

template <class Epi>
inline size_t big_kernel_smem() { return kBigSmem + Epi::kExtra; }

// ---- k-major operands -----------------------------------------------------------------------------
//
// A k-major matrix keeps coordinate k of row r at p[k * ld + r], with ld a multiple of 32 and the
// columns [n, ld) zero.  A 16 x 128 stage of the tile pipeline is then 16 contiguous runs of 512
// bytes: two 16-byte cp.async per thread and operand, no transposition and no per-element address
// arithmetic, and a stage can end at any k (the k loop is bounded by the stage's real extent).

struct KMajor {
    const float *p;
    int64_t n;     // rows
    int64_t ld;    // row pitch of a k step, a multiple of 32
    int64_t cols;  // columns readable from p on each k step (ld for a whole matrix; less for a slice)
};

__host__ __device__ inline int64_t kmajor_ld(int64_t n) { return (n + 31) & ~int64_t(31); }

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem, bool valid) {
    const unsigned s = (unsigned) __cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0));
}

__device__ __forceinline__ void big_load_stage_km(BigOperands &op, int buf, const KMajor &A, int64_t a0,
                                                  const KMajor &B, int64_t b0, int k0, int k_end) {
#pragma unroll
    for (int t = 0; t < (kBig * kBigK / 4) / kBigThreads; t++) {
        const int c = threadIdx.x + t * kBigThreads;
        const int kk = c >> 5, col = (c & 31) * 4;
        const int k = k0 + kk;
        const bool va = k < k_end && a0 + col < A.cols, vb = k < k_end && b0 + col < B.cols;
        cp_async16(&op.a[buf][kk][col], va ? A.p + (int64_t) k * A.ld + a0 + col : A.p, va);
        cp_async16(&op.b[buf][kk][col], vb ? B.p + (int64_t) k * B.ld + b0 + col : B.p, vb);
    }
}

// big_accumulate over k-major operands: the same products and sums in the same k order.
__device__ __forceinline__ bool big_accumulate_km(BigOperands &op, float acc[8][8], const KMajor &A, int64_t a0,
                                                 const KMajor &B, int64_t b0, int k_begin, int k_end) {
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < 8; j++) acc[i][j] = 0.0f;
    const int ns = (k_end - k_begin + kBigK - 1) / kBigK;
    if (ns <= 0) return false;
    big_load_stage_km(op, 0, A, a0, B, b0, k_begin, k_end);
    cp_async_commit();
    for (int s = 0; s < ns; s++) {
        if (s + 1 < ns) {
            big_load_stage_km(op, (s + 1) & 1, A, a0, B, b0, k_begin + (s + 1) * kBigK, k_end);
            cp_async_commit();
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const int buf = s & 1;
        const int kc = min(kBigK, k_end - k_begin - s * kBigK);
#pragma unroll kBigKUnroll
        for (int kk = 0; kk < kc; kk++) {
            const float4 a_lo = *reinterpret_cast<const float4 *>(&op.a[buf][kk][4 * tx]);
            const float4 a_hi = *reinterpret_cast<const float4 *>(&op.a[buf][kk][64 + 4 * tx]);
            const float4 b_lo = *reinterpret_cast<const float4 *>(&op.b[buf][kk][4 * ty]);
            const float4 b_hi = *reinterpret_cast<const float4 *>(&op.b[buf][kk][64 + 4 * ty]);
            const float av[8] = {a_lo.x, a_lo.y, a_lo.z, a_lo.w, a_hi.x, a_hi.y, a_hi.z, a_hi.w};
            const float bv[8] = {b_lo.x, b_lo.y, b_lo.z, b_lo.w, b_hi.x, b_hi.y, b_hi.z, b_hi.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 8; j++) acc[i][j] = __fadd_rn(acc[i][j], __fmul_rn(av[i], bv[j]));
        }
        __syncthreads();
    }
    return true;
}

// Split form: the block of partial sums over [0, k_split) goes to epi.finish_lo(extra, res, a0, b0),
// then the sums over [k_split, k_end) -- each accumulated from 0, as the reference keeps a partial
// score and its remainder apart -- are added to them with one rounding and
// epi.finish_hi(extra, res, a0, b0, spare) sees the totals; spare is the operand buffers'
// sizeof(BigOperands) bytes, free by then.  Operands (k-major) and result have separate shared
// memory, so the second range's loads do not wait for finish_lo.  Epi also provides kExtra and
// prologue(extra, a0, b0), which returns whether the tile has work (the same answer in every
// thread; false ends the CTA).  Every thread calls each hook (they may synchronise the block).
template <class Epi>
__global__ void __launch_bounds__(kBigThreads, 2) exact_big_split_kernel(KMajor A, KMajor B, int k_split, int k_end,
                                                                         Epi epi) {
    extern __shared__ __align__(16) char big_smem[];
    BigOperands &op = *reinterpret_cast<BigOperands *>(big_smem);
    BigResult &res = *reinterpret_cast<BigResult *>(big_smem + sizeof(BigOperands));
    char *extra = big_smem + sizeof(BigOperands) + sizeof(BigResult);
    const int64_t b0 = (int64_t) blockIdx.x * kBig;
    const int64_t a0 = (int64_t) blockIdx.y * kBig;
    if (!epi.prologue(extra, a0, b0)) return;
    float acc[8][8];
    big_accumulate_km(op, acc, A, a0, B, b0, 0, k_split);
    big_store(res, acc, false);
    __syncthreads();
    epi.finish_lo(extra, res, a0, b0);
    // big_accumulate_km's first barrier orders finish_lo's reads of res before the adds below
    if (!big_accumulate_km(op, acc, A, a0, B, b0, k_split, k_end)) __syncthreads();
    big_store(res, acc, true);
    __syncthreads();
    epi.finish_hi(extra, res, a0, b0, big_smem);
}

template <class Epi>
inline cudaError_t launch_big_split(const KMajor &A, const KMajor &B, int k_split, int k_end, const Epi &epi,
                                    cudaStream_t st) {
    const size_t smem = sizeof(BigOperands) + sizeof(BigResult) + Epi::kExtra;
    // set outside graph capture (an eager run of the same launch sets it first)
    cudaStreamCaptureStatus capturing = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &capturing);
    if (e != cudaSuccess) return e;
    if (capturing == cudaStreamCaptureStatusNone) {
        e = cudaFuncSetAttribute(exact_big_split_kernel<Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
        if (e != cudaSuccess) return e;
    }
    dim3 grid((unsigned) ((B.n + kBig - 1) / kBig), (unsigned) ((A.n + kBig - 1) / kBig));
    exact_big_split_kernel<Epi><<<grid, kBigThreads, smem, st>>>(A, B, k_split, k_end, epi);
    return cudaGetLastError();
}

// Row-major [n][dim] rows (gathered through idx when given) to k-major [dim][ld], zeroing the
// columns [n, ld).  Grid (ld / 32, ceil(dim / 32)), block (32, 8).
__global__ void to_kmajor_kernel(const float *__restrict__ src, const int32_t *__restrict__ idx, int64_t n, int dim,
                                 int64_t ld, float *__restrict__ dst);
int to_kmajor(const float *src, const int32_t *idx, int64_t n, int dim, float *dst, cudaStream_t st);

// Launches exact_big_kernel<Epi> over n_a x n_b pairs on stream st.
template <class Epi>
inline cudaError_t launch_big(const float *A, const int32_t *a_idx, int64_t n_a, int lda, const float *B, int64_t n_b,
                              int ldb, int k_begin, int k_end, const Epi &epi, cudaStream_t st) {
    const size_t smem = big_kernel_smem<Epi>();
    cudaError_t e = cudaFuncSetAttribute(exact_big_kernel<Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
    if (e != cudaSuccess) return e;
    dim3 grid((unsigned) ((n_b + kBig - 1) / kBig), (unsigned) ((n_a + kBig - 1) / kBig));
    exact_big_kernel<Epi><<<grid, kBigThreads, smem, st>>>(A, a_idx, n_a, lda, B, n_b, ldb, k_begin, k_end, epi);
    return cudaGetLastError();
}

// Sequential binary32 dot product of one pair (thread-serial), same arithmetic as exact_tile.
__device__ __forceinline__ void prefetch_l1(const void *p) { asm volatile("prefetch.global.L1 [%0];" ::"l"(p)); }

__device__ __forceinline__ float exact_dot(const float *__restrict__ a, const float *__restrict__ b, int n) {
    // every 128-byte line of both rows requested up front, so that the ordered sum below waits for
    // one memory latency instead of one per line
    for (int o = 0; o < n; o += 32) {
        prefetch_l1(a + o);
        prefetch_l1(b + o);
    }
    if (n > 0) {
        prefetch_l1(a + n - 1);
        prefetch_l1(b + n - 1);
    }
    float acc = 0.0f;
    int j = 0;
    if (((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 7) == 0) {
        // 8-byte loads, sixteen coordinates ahead of their (ordered) sum: per-thread rows are read
        // with half the memory transactions
        for (; j + 16 <= n; j += 16) {
            float2 x[8], y[8];
#pragma unroll
            for (int t = 0; t < 8; t++) {
                x[t] = __ldg(reinterpret_cast<const float2 *>(a + j) + t);
                y[t] = __ldg(reinterpret_cast<const float2 *>(b + j) + t);
            }
#pragma unroll
            for (int t = 0; t < 8; t++) {
                acc = __fadd_rn(acc, __fmul_rn(x[t].x, y[t].x));
                acc = __fadd_rn(acc, __fmul_rn(x[t].y, y[t].y));
            }
        }
    }
    for (; j + 8 <= n; j += 8) {  // loads of eight coordinates ahead of their (ordered) sum
        float x[8], y[8];
#pragma unroll
        for (int t = 0; t < 8; t++) {
            x[t] = __ldg(a + j + t);
            y[t] = __ldg(b + j + t);
        }
#pragma unroll
        for (int t = 0; t < 8; t++) acc = __fadd_rn(acc, __fmul_rn(x[t], y[t]));
    }
    for (; j < n; j++) acc = __fadd_rn(acc, __fmul_rn(__ldg(a + j), __ldg(b + j)));
    return acc;
}

// std::lower_bound(row, row + S, q, [](float arr, float q) { return arr >= q; }) on a descending
// row: the number of leading thresholds >= q (SampleSearch.hpp:99-102).
__device__ __forceinline__ int bucket_of(const float *__restrict__ row, int S, float q) {
    int lo = 0, len = S;
    while (len > 0) {
        const int h = len >> 1, m = lo + h;
        if (__ldg(row + m) >= q) {
            lo = m + 1;
            len -= h + 1;
        } else {
            len = h;
        }
    }
    return lo;
}

// Inclusive warp scan of an int.
__device__ __forceinline__ int warp_incl_scan(int v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int n = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += n;
    }
    return v;
}

// Exclusive block scan (blockDim.x == 256); returns the exclusive prefix, *total gets the sum.
__device__ __forceinline__ int block_excl_scan(int v, int *warp_tot, int *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int incl = warp_incl_scan(v);
    if (lane == 31) warp_tot[w] = incl;
    __syncthreads();
    if (w == 0) {
        int t = lane < 8 ? warp_tot[lane] : 0;
        const int ti = warp_incl_scan(t);
        if (lane < 8) warp_tot[lane] = ti - t;
        if (lane == 7) warp_tot[8] = ti;
    }
    __syncthreads();
    const int r = warp_tot[w] + incl - v;
    *total = warp_tot[8];
    __syncthreads();
    return r;
}

// Two-level form of bucket_of for a block of users: the CTA keeps every g-th threshold of each of
// its users in shared memory (the last element of each group of g), finds the first group whose
// last (smallest) threshold is below q there, and counts the thresholds >= q inside that group
// with independent loads.  On a descending row this is the same count std::lower_bound returns.
struct ThrSummary {
    static constexpr int kMaxGroups = 32;
    float v[kTile][kMaxGroups];
};

__host__ __device__ __forceinline__ int thr_group(int S) {
    const int g = (S + ThrSummary::kMaxGroups - 1) / ThrSummary::kMaxGroups;
    return g < 16 ? 16 : g;
}

__device__ __forceinline__ void load_thr_summary(ThrSummary &ts, const float *__restrict__ thr, int64_t n_user,
                                                 int64_t a0, int S) {
    const int g = thr_group(S), nb = (S + g - 1) / g;
    for (int idx = threadIdx.x; idx < kTile * nb; idx += blockDim.x) {
        const int r = idx / nb, j = idx % nb;
        const int64_t u = a0 + r;
        ts.v[r][j] = u < n_user ? __ldg(thr + u * S + min(g * j + g - 1, S - 1)) : 0.0f;
    }
}

// Threshold summaries for `rows` users starting at a0 into dst[rows][kMaxGroups].
__device__ __forceinline__ void load_thr_summary_rows(float *dst, int rows, const float *__restrict__ thr,
                                                      int64_t n_user, int64_t a0, int S) {
    const int g = thr_group(S), nb = (S + g - 1) / g;
    for (int idx = threadIdx.x; idx < rows * nb; idx += blockDim.x) {
        const int r = idx / nb, j = idx % nb;
        const int64_t u = a0 + r;
        dst[r * ThrSummary::kMaxGroups + j] = u < n_user ? __ldg(thr + u * S + min(g * j + g - 1, S - 1)) : 0.0f;
    }
}

__device__ __forceinline__ int bucket_of_2level(const float *__restrict__ summ, const float *__restrict__ row, int S,
                                                float q) {
    const int g = thr_group(S), nb = (S + g - 1) / g;
    int lo = 0, len = nb;
    while (len > 0) {
        const int h = len >> 1, m = lo + h;
        if (summ[m] >= q) { lo = m + 1; len -= h + 1; } else len = h;
    }
    if (lo == nb) return S;
    const int base = g * lo, end = min(base + g, S);
    int c = 0;
    if ((g & 15) == 0 && end - base == g && (S & 3) == 0) {
        const float4 *p = reinterpret_cast<const float4 *>(row + base);
        for (int t = 0; t < g / 16; t++, p += 4) {
            const float4 x0 = __ldg(p), x1 = __ldg(p + 1), x2 = __ldg(p + 2), x3 = __ldg(p + 3);
            c += (x0.x >= q) + (x0.y >= q) + (x0.z >= q) + (x0.w >= q) + (x1.x >= q) + (x1.y >= q) + (x1.z >= q) +
                 (x1.w >= q) + (x2.x >= q) + (x2.y >= q) + (x2.z >= q) + (x2.w >= q) + (x3.x >= q) + (x3.y >= q) +
                 (x3.z >= q) + (x3.w >= q);
        }
    } else {
        for (int i = base; i < end; i++) c += __ldg(row + i) >= q;
    }
    return base + c;
}

// Rank bounds of bucket b (SampleSearch::CoarseBinarySearch, SampleSearch.hpp:107-125).
__device__ __host__ __forceinline__ void bucket_bounds(int b, int S, const int32_t *rank, int n_item, int &lb, int &ub) {
    const unsigned tlb = b == S ? (unsigned) n_item : (unsigned) rank[b];
    const unsigned tub = b == 0 ? 0u : (unsigned) rank[b - 1];
    if (b == S) {
        lb = n_item;
        ub = (int) tub;
    } else if (b == 0) {
        lb = (int) tlb;
        ub = 0;
    } else if (tlb - tub <= 1) {
        lb = (int) tlb;
        ub = (int) tlb;
    } else {
        lb = (int) tlb;
        ub = (int) tub;
    }
}

// Per-query outcome of the pruning steps, written by the select kernels.
struct QueryCounts {
    int32_t n_result;        // results after pruning (the reference's n_result_user)
    int32_t n_prune;         // pruned users (n_prune_user)
    int32_t n_cand;          // candidates handed to refinement (0 when n_result >= topk)
    int32_t n_res_emit;      // result users emitted (min(number flagged, topk))
    int32_t mode;            // 0: normal, 1: k-th bounds equal, 2: refinement skipped
    int32_t bk;              // bucket of the k-th smallest bound
    int32_t lstar, ustar;    // k-th smallest lower / upper rank bound
    int32_t ip_base;         // the reference's ip_cost before refinement (QS/US: n_user; QSRP: round-2 users)
    int32_t pad;
};

// Pair classes produced by the pruning step (PruneCandidateByBound.hpp:83-150).
enum : uint8_t { kClsRefine = 0, kClsResult = 1, kClsPrune = 2, kClsIdle = 3 };

// Histogram of small unsigned values per query (values >= n_bins are skipped), one CTA per
// (user chunk, query).  Each warp counts into its own shared-memory copy (plain atomics, no warp
// matching), the copies are summed, and the non-zero bins are added to the global histogram.
constexpr int kHistThreads = 256;

__host__ __device__ inline int hist_copies(int n_bins) {
    int c = 98304 / (4 * n_bins);
    return c < 1 ? 1 : (c > 8 ? 8 : c);
}

template <typename T>
__global__ void __launch_bounds__(kHistThreads) bucket_hist_kernel(const T *__restrict__ vals, int64_t n_user,
                                                                  int n_bins, int64_t chunk, int *__restrict__ hist) {
    extern __shared__ int h[];
    const int copies = hist_copies(n_bins);
    const int q = blockIdx.y;
    for (int b = threadIdx.x; b < copies * n_bins; b += blockDim.x) h[b] = 0;
    __syncthreads();
    int *mine = h + ((threadIdx.x >> 5) % copies) * n_bins;
    const T *row = vals + (int64_t) q * n_user;
    const int64_t u0 = (int64_t) blockIdx.x * chunk, u1 = min(u0 + chunk, n_user);
    int64_t u = u0 + threadIdx.x;
    for (; u + 3 * kHistThreads < u1; u += 4 * kHistThreads) {
        const unsigned v0 = row[u], v1 = row[u + kHistThreads], v2 = row[u + 2 * kHistThreads],
                       v3 = row[u + 3 * kHistThreads];
        if (v0 < (unsigned) n_bins) atomicAdd(mine + v0, 1);
        if (v1 < (unsigned) n_bins) atomicAdd(mine + v1, 1);
        if (v2 < (unsigned) n_bins) atomicAdd(mine + v2, 1);
        if (v3 < (unsigned) n_bins) atomicAdd(mine + v3, 1);
    }
    for (; u < u1; u += kHistThreads) {
        const unsigned v = row[u];
        if (v < (unsigned) n_bins) atomicAdd(mine + v, 1);
    }
    __syncthreads();
    int *g = hist + (int64_t) q * n_bins;
    for (int b = threadIdx.x; b < n_bins; b += blockDim.x) {
        int s = 0;
        for (int c = 0; c < copies; c++) s += h[c * n_bins + b];
        if (s) atomicAdd(g + b, s);
    }
}

// ---- ordered compaction of result users and candidates ---------------------------------------------
//
// Per query the reference lists result users in user-id order (QS.hpp:185-194) and collects the
// refinement candidates (ComputeAllIPBound.hpp:306-313).  Users are cut into chunks of
// kCompactChunk; pass 1 counts per (query, chunk), a scan turns the counts into offsets, pass 2
// writes each chunk's entries at its offset -- so the lists come out in user-id order while every
// chunk runs in parallel.  Thread t of a chunk owns kCompactPer consecutive users.  A policy P
// gives, for a thread's users, the mask of those that can be a result or a candidate
// (need_mask(q, u, n)), classifies such a (query, user) pair (0 none, 1 result, 2 candidate;
// with_aux asks for the entry's fields too, which only the emitting pass needs) and writes the
// entries.

// The top-k of each query of a batch: k[q] when per-query values are given, else kmax for every
// query; kmax is also the row stride of the batch's per-query result arrays.
struct KSpec {
    const int32_t *k;  // [nq] on the device, or nullptr
    int kmax;
    __host__ __device__ int of(int q) const { return k ? k[q] : kmax; }
};

constexpr int kCompactThreads = 256;
constexpr int kCompactPer = 16;
constexpr int64_t kCompactChunk = (int64_t) kCompactThreads * kCompactPer;

// The 16 bytes p[0..15] as four words (little-endian order), from five aligned 4-byte loads; bytes
// past the buffer's end are read only inside its allocation slack and must be masked by the caller.
__device__ __forceinline__ void load16_bytes(const uint8_t *p, uint32_t w[4]) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uint32_t *base = reinterpret_cast<const uint32_t *>(a & ~uintptr_t(3));
    const unsigned sh = (unsigned) (a & 3) * 8;
    uint32_t x[5];
#pragma unroll
    for (int i = 0; i < 5; i++) x[i] = __ldg(base + i);
#pragma unroll
    for (int i = 0; i < 4; i++) w[i] = __funnelshift_r(x[i], x[i + 1], sh);
}

template <class P>
__global__ void __launch_bounds__(kCompactThreads) compact_count_kernel(P p, int64_t n_user, int nchunks,
                                                                      int2 *__restrict__ cnt,
                                                                      const int32_t *__restrict__ qmap) {
    __shared__ int warp_tot[9];
    const int qi = blockIdx.y, q = qmap ? qmap[qi] : qi;
    const int64_t u0 = (int64_t) blockIdx.x * kCompactChunk + (int64_t) threadIdx.x * kCompactPer;
    int r = 0, c = 0;
    if (u0 < n_user) {
        const int n = (int) (n_user - u0 < kCompactPer ? n_user - u0 : kCompactPer);
        uint32_t need = p.need_mask(q, u0, n);
        while (need) {
            const int e = __ffs(need) - 1;
            need &= need - 1;
            typename P::Aux aux;
            const int k = p.classify(q, u0 + e, aux, false);
            r += k == 1;
            c += k == 2;
        }
    }
    int tot;
    block_excl_scan(r | (c << 16), warp_tot, &tot);
    if (threadIdx.x == 0) cnt[(int64_t) qi * nchunks + blockIdx.x] = make_int2(tot & 0xffff, tot >> 16);
}

// Offsets per (query, chunk); n_res_emit = min(results, topk); flags a candidate-count mismatch.  With
// qmap the kernels of this form run on the listed queries only (slot qi holds query qmap[qi]).
static __global__ void compact_scan_kernel(const int2 *__restrict__ cnt, int nchunks, int nq, KSpec ks, int2 *__restrict__ off,
                                    QueryCounts *__restrict__ counts, int *__restrict__ err,
                                    const int32_t *__restrict__ qmap) {
    const int qi = blockIdx.x * blockDim.x + threadIdx.x;
    if (qi >= nq) return;
    const int q = qmap ? qmap[qi] : qi;
    int r = 0, c = 0;
    for (int i = 0; i < nchunks; i++) {
        const int2 v = cnt[(int64_t) qi * nchunks + i];
        off[(int64_t) qi * nchunks + i] = make_int2(r, c);
        r += v.x;
        c += v.y;
    }
    const int topk = ks.of(q);
    counts[q].n_res_emit = r < topk ? r : topk;
    if (c != counts[q].n_cand) atomicAdd(err, 1);
}

template <class P>
__global__ void __launch_bounds__(kCompactThreads) compact_write_kernel(P p, int64_t n_user, int nchunks,
                                                                      const int2 *__restrict__ cnt,
                                                                      const int2 *__restrict__ off, KSpec ks,
                                                                      const int32_t *__restrict__ qmap) {
    __shared__ int warp_tot[9];
    const int qi = blockIdx.y, q = qmap ? qmap[qi] : qi;
    const int topk = ks.of(q);
    const int2 cc = cnt[(int64_t) qi * nchunks + blockIdx.x];
    const int2 oo = off[(int64_t) qi * nchunks + blockIdx.x];
    if ((cc.x == 0 || oo.x >= topk) && cc.y == 0) return;
    // thread t owns users u0 + t*kCompactPer .. + kCompactPer - 1, so prefix order is user-id order
    const int64_t u0 = (int64_t) blockIdx.x * kCompactChunk + (int64_t) threadIdx.x * kCompactPer;
    uint32_t need = 0;
    if (u0 < n_user) need = p.need_mask(q, u0, (int) (n_user - u0 < kCompactPer ? n_user - u0 : kCompactPer));
    int r = 0, c = 0;
    uint32_t hit = 0, is_res = 0;
    for (uint32_t m = need; m; m &= m - 1) {
        const int e = __ffs(m) - 1;
        typename P::Aux aux;
        const int k = p.classify(q, u0 + e, aux, false);
        r += k == 1;
        c += k == 2;
        if (k) hit |= 1u << e;
        if (k == 1) is_res |= 1u << e;
    }
    int tot;
    const int pre = block_excl_scan(r | (c << 16), warp_tot, &tot);
    if (!hit) return;
    int pr = oo.x + (pre & 0xffff), pc = oo.y + (pre >> 16);
    for (uint32_t m = hit; m; m &= m - 1) {
        const int e = __ffs(m) - 1;
        if ((is_res >> e & 1) && pr >= topk) { pr++; continue; }
        typename P::Aux aux;
        const int k = p.classify(q, u0 + e, aux, true);
        if (k == 1) {
            if (pr < topk) p.emit_result(q, pr, u0 + e, aux);
            pr++;
        } else if (k == 2) {
            p.emit_cand(q, pc, u0 + e, aux);
            pc++;
        }
    }
}

// ---- sparse form of the same compaction -------------------------------------------------------------
//
// The users a query must classify are few (a few hundred of the 480 K at config 2), so the sparse
// form streams the codes once: compact_need_flat_kernel appends each query's flagged users to its
// list (in no particular order), and compact_emit_kernel, one block per query, sorts
// the list by user id and runs the ordered classification and emission of compact_write_kernel on
// it.  A query whose list outgrows kNeedCap is listed and takes the two-pass form above.

constexpr int kNeedBits = 12;               // bits of a list position in the sort keys
constexpr int kNeedCap = 1 << kNeedBits;    // flagged users per query on the sparse path

// The flagged users' lists from one flat pass over the batch's codes ([query][user] as one array): 512 bytes
// per warp and step in aligned 16-byte loads, the next step's load in flight while a step is
// examined; a lane whose 16 codes lie in one query takes the policy's word-wise need_bits, one that
// straddles a query boundary goes byte by byte.  Hits are few: one atomic per lane with hits.
template <class P>
__global__ void __launch_bounds__(256) compact_need_flat_kernel(P p, int64_t n_user, int nq, double inv_user,
                                                               int32_t *__restrict__ need_n,
                                                               int32_t *__restrict__ need_u) {
    const uint8_t *code = p.code;
    const int64_t total = n_user * nq;
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t stride = (int64_t) gridDim.x * blockDim.x * 16;
    auto load = [&](int64_t seg, uint32_t w[4]) {
        const int64_t base = seg + (int64_t) lane * 16;
        if (base + 16 <= total) {
            const uint4 x = __ldg(reinterpret_cast<const uint4 *>(code + base));
            w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                w[i] = 0;
                for (int j = 0; j < 4; j++)
                    if (base + 4 * i + j < total) w[i] |= (uint32_t) code[base + 4 * i + j] << (8 * j);
            }
        }
    };
    uint32_t wn[4] = {0u, 0u, 0u, 0u};
    if (warp * 512 < total) load(warp * 512, wn);
    for (int64_t seg = warp * 512; seg < total; seg += stride) {
        uint32_t w[4] = {wn[0], wn[1], wn[2], wn[3]};
        if (seg + stride < total) load(seg + stride, wn);
        const int64_t base = seg + (int64_t) lane * 16;
        int64_t qs = 0;
        if (lane == 0) {
            qs = (int64_t) ((double) seg * inv_user);
            if (qs * n_user > seg) qs--;
            else if ((qs + 1) * n_user <= seg) qs++;
        }
        qs = __shfl_sync(0xffffffffu, qs, 0);
        if (base >= total) continue;
        int64_t q = qs;
        while ((q + 1) * n_user <= base) q++;
        if (base + 16 <= (q + 1) * n_user && base + 16 <= total) {
            uint32_t m = p.need_bits((int) q, w);
            if (!m) continue;
            int at = atomicAdd(need_n + q, __popc(m));
            int32_t *list = need_u + q * kNeedCap;
            const int64_t u0 = base - q * n_user;
            for (; m; m &= m - 1, at++)
                if (at < kNeedCap) list[at] = (int32_t) (u0 + __ffs(m) - 1);
        } else {
            for (int e = 0; e < 16; e++) {
                const int64_t pos = base + e;
                if (pos >= total) break;
                while ((q + 1) * n_user <= pos) q++;
                if (!p.need_byte((int) q, (w[e >> 2] >> (8 * (e & 3))) & 0xffu)) continue;
                const int at = atomicAdd(need_n + q, 1);
                if (at < kNeedCap) need_u[q * kNeedCap + at] = (int32_t) (pos - q * n_user);
            }
        }
    }
}

// Every listed user classified at once (one thread per list entry over all queries, so that the
// reference-arithmetic recomputations of many queries overlap), with the data its emission needs.
template <class P>
__global__ void __launch_bounds__(256) compact_classify_kernel(P p, int nq, const int32_t *__restrict__ need_n,
                                                              const int32_t *__restrict__ need_u,
                                                              int8_t *__restrict__ cls, typename P::Aux *__restrict__ aux) {
    const int64_t total = (int64_t) nq * kNeedCap;
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t) gridDim.x * blockDim.x) {
        const int q = (int) (idx / kNeedCap), i = (int) (idx % kNeedCap);
        const int n = need_n[q];
        if (n > kNeedCap || i >= n) continue;  // unused slot, or a query left to the two-pass form
        typename P::Aux a;
        cls[idx] = (int8_t) p.classify(q, need_u[idx], a, true);
        aux[idx] = a;
    }
}

// One block per query: its list sorted by user id (the order the reference lists users in), then
// the ordered emission from the classes compact_classify_kernel stored.
template <class P>
__global__ void __launch_bounds__(kCompactThreads) compact_emit_kernel(P p, KSpec ks, const int32_t *__restrict__ need_n,
                                                                     const int32_t *__restrict__ need_u,
                                                                     const int8_t *__restrict__ cls,
                                                                     const typename P::Aux *__restrict__ aux_l,
                                                                     QueryCounts *__restrict__ counts, int *__restrict__ err,
                                                                     int32_t *__restrict__ ovf_q) {
    extern __shared__ __align__(16) unsigned char emit_smem[];
    uint64_t *s = reinterpret_cast<uint64_t *>(emit_smem);  // [kNeedCap]: user id << kNeedBits | list position
    __shared__ int warp_tot[9];
    const int q = blockIdx.x, tid = threadIdx.x;
    const int n = need_n[q], topk = ks.of(q);
    if (n > kNeedCap) {  // listed for the two-pass form
        if (tid == 0) ovf_q[atomicAdd(err + 1, 1)] = q;
        return;
    }
    int pn = 1;
    while (pn < n) pn <<= 1;
    const int64_t row = (int64_t) q * kNeedCap;
    for (int i = tid; i < pn; i += kCompactThreads)
        s[i] = i < n ? ((uint64_t) (uint32_t) need_u[row + i] << kNeedBits) | (uint64_t) i : ~uint64_t(0);
    __syncthreads();
    // bitonic sort, ascending user id
    for (int k = 2; k <= pn; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = tid; i < pn; i += kCompactThreads) {
                const int ij = i ^ j;
                if (ij > i) {
                    const uint64_t a = s[i], b = s[ij];
                    if ((a > b) == ((i & k) == 0)) {
                        s[i] = b;
                        s[ij] = a;
                    }
                }
            }
            __syncthreads();
        }
    int pr = 0, pc = 0;  // results and candidates before this tile
    for (int t0 = 0; t0 < n; t0 += kCompactThreads) {
        const int i = t0 + tid;
        int k = 0;
        int64_t u = 0, at = 0;
        if (i < n) {
            u = (int64_t) (s[i] >> kNeedBits);
            at = row + (int64_t) (s[i] & (kNeedCap - 1));
            k = cls[at];
        }
        int tot;
        const int pre = block_excl_scan((k == 1) | ((k == 2) << 16), warp_tot, &tot);
        const int rpos = pr + (pre & 0xffff), cpos = pc + (pre >> 16);
        if (k == 1 && rpos < topk) p.emit_result(q, rpos, u, aux_l[at]);
        else if (k == 2) p.emit_cand(q, cpos, u, aux_l[at]);
        pr += tot & 0xffff;
        pc += tot >> 16;
    }
    if (tid == 0) {
        counts[q].n_res_emit = pr < topk ? pr : topk;
        if (pc != counts[q].n_cand) atomicAdd(err, 1);
    }
}

}  // namespace rkr

// ---- per-kernel timing (opt-in) -------------------------------------------------------------------

namespace rkr {
// CUDA-event pairs around each kernel launch on its own stream, resolved when read.
struct Profiler {
    bool on = false;
    std::vector<std::string> names;
    std::vector<double> total_ms;
    std::vector<int64_t> launches;
    struct Pending { int id; cudaEvent_t a, b; };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get_event() {
        if (!pool.empty()) { cudaEvent_t e = pool.back(); pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
    // A counter reported beside the kernels (no time; `launches` carries the count).
    void add_count(const char *n, int64_t v) { launches[id_of(n)] += v; }
    int id_of(const char *n) {
        for (size_t i = 0; i < names.size(); i++) if (names[i] == n) return (int) i;
        names.emplace_back(n);
        total_ms.push_back(0);
        launches.push_back(0);
        return (int) names.size() - 1;
    }
    void resolve() {
        for (auto &p : pending) {
            float ms = 0;
            if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
                total_ms[p.id] += ms;
                launches[p.id] += 1;
            }
            pool.push_back(p.a);
            pool.push_back(p.b);
        }
        pending.clear();
    }
    void release() {
        resolve();
        for (auto e : pool) cudaEventDestroy(e);
        pool.clear();
    }
};
}  // namespace rkr

// ---- the index handle --------------------------------------------------------------------------------

struct rkr_index {
    int device = 0;
    cudaStream_t stream = nullptr;
    int64_t n_user = 0, n_item = 0;
    int dim = 0;
    int check_dim = -1;
    // resident data
    rkr::DevBuf user;          // [n_user][dim], normalised
    rkr::DevBuf item;          // [n_item][dim], original order
    rkr::DevBuf item_sorted;   // [n_item][dim], by norm, descending
    rkr::DevBuf item_km;       // k-major copies: [dim][kmajor_ld(n_item)] of item ...
    rkr::DevBuf item_sorted_km;  // ... and of item_sorted
    rkr::DevBuf item_norm;     // [n_item], descending
    rkr::DevBuf item_rnorm;    // [n_item], norm of dims [check_dim, dim) of item_sorted
    rkr::DevBuf user_rnorm;    // [n_user], norm of dims [check_dim, dim) of user
    // tensor-core refinement: item digit tiles, built on first use, of item_sorted split at check_dim
    // (QS, QSRP) and of item unsplit (US)
    bool refine_tc_on = true;                 // refinement counts on the tensor cores where the shape fits
    int ri_key_split = -2, ri_key_full = -2;  // the split the tiles were built for (-2: none)
    rkr::DevBuf ri_item_split, ri_imeta_split, ri_item_full, ri_imeta_full;
    // tensor-core pair scores: user digit tiles for the SVD split at check_dim (QSRP) and unsplit (QS, US)
    bool scores_tc_on = true;
    bool compact_sparse_on = true;            // the sparse ordered compaction (else two-pass for every query)
    int sc_key_split = -2, sc_key_full = -2;  // the split the tiles were built for (-2: none)
    rkr::DevBuf sc_user_split, sc_umeta_split, sc_user_full, sc_umeta_full, sc_cdf_tab;
    std::vector<float> h_item_norm_sorted;
    std::vector<int32_t> h_item_order;
    // SampleSearch
    int n_sample = 0;
    rkr::DevBuf sample_rank;   // [n_sample]
    rkr::DevBuf thr;           // [n_user][n_sample]
    rkr::DevBuf thr_summ;      // [n_user][ThrSummary::kMaxGroups]: last (smallest) threshold of each group
    std::vector<int32_t> h_sample_rank;
    // NormalLinearRegressionLP
    int n_sample_reg = 0;
    rkr::DevBuf reg_rank;      // [n_sample_reg]
    rkr::DevBuf reg;           // [n_user][8]: a, b, mu, sigma, err, smax, smin, 0
    rkr::DevBuf lvt;           // [n_user][2][kLvEntries] float2: level-boundary tables (rkr_levels.cu)
    // SVD
    bool has_svd = false;
    rkr::DevBuf transfer_item; // [dim][dim]
    rkr::DevBuf svd_user;      // [n_user][dim]
    rkr::DevBuf svd_user_km;   // k-major copy: [dim][kmajor_ld(n_user)]
    rkr::DevBuf user_km;       // k-major copy of user: [dim][kmajor_ld(n_user)]
    rkr::DevBuf svd_unorm;     // [n_user], norm of dims [check_dim, dim) of svd_user
    rkr::DevBuf qip_state;     // [n_user], QSRPNormalLP's carried query scores
    // per-call workspace
    rkr::DevBuf ws_query, ws_qtr, ws_qnorm, ws_bucket, ws_bucket2, ws_levels, ws_cls, ws_counts, ws_hist;
    rkr::DevBuf ws_res, ws_cand, ws_cand_off, ws_refine, ws_rank, ws_out, ws_stats, ws_misc, ws_fix, ws_km, ws_tc, ws_sc;
    rkr::DevBuf ws_defer;  // rows the streaming row selection left to the scatter form
    rkr::DevBuf ws_emit;   // the sparse compaction's classes and emission data per list entry
    rkr::DevBuf ws_shard;  // a user shard's counts on their way to the exchange
    rkr::DevBuf ws_snap[2];  // ... and its copies of summed counts before a second pass adds to them
    // Every per-call workspace buffer: a serving worker's shadow of the index owns its own (the
    // resident data it shares), and destruction releases them.
    std::vector<rkr::DevBuf *> workspaces() {
        return {&ws_query, &ws_qtr, &ws_qnorm, &ws_bucket, &ws_bucket2, &ws_levels, &ws_cls, &ws_counts, &ws_hist,
                &ws_res, &ws_cand, &ws_cand_off, &ws_refine, &ws_rank, &ws_out, &ws_stats, &ws_misc, &ws_fix,
                &ws_km, &ws_tc, &ws_sc, &ws_defer, &ws_emit, &ws_shard, &ws_snap[0], &ws_snap[1]};
    }
    // User shard (rkr_index_set_shard): this index holds users [user_offset, user_offset + n_user)
    // of n_user_total, and the per-query counts each selection reads are summed over the shards
    // through fn (rkr_shard.cu).
    struct Shard {
        int32_t index = 0, count = 1;
        int64_t user_offset = 0, n_user_total = 0;
        rkr_exchange_fn fn = nullptr;
        void *ctx = nullptr;
    } shard;
    bool sharded() const { return shard.fn != nullptr; }
    int64_t n_user_all() const { return shard.fn ? shard.n_user_total : n_user; }
    std::vector<uint8_t> h_scratch;
    rkr::Profiler prof;
    // CUDA graphs of a batch's phase 1 (rkr_qsrp.cu), one per (method, batch size, workspace
    // addresses), captured on the second batch of a shape and replayed after; off unless set
    bool graphs_on = false;
    struct PhaseGraph {
        int method, nq;
        const void *ws[8];
        cudaGraphExec_t exec;  // nullptr: the shape ran once eagerly (its buffers are sized)
    };
    std::vector<PhaseGraph> graphs;
    float2 *score_dump = nullptr;  // diagnostics (rkr_score_estimates): where the pair scores' estimates go
};

namespace rkr {
// Runs `launch` (one kernel launch on stream st) and, when profiling is on, times it with events.
template <typename F> inline void timed(rkr_index *ix, cudaStream_t st, const char *name, F &&launch) {
    if (!ix->prof.on) { launch(); return; }
    Profiler::Pending p;
    p.id = ix->prof.id_of(name);
    p.a = ix->prof.get_event();
    p.b = ix->prof.get_event();
    cudaEventRecord(p.a, st);
    launch();
    cudaEventRecord(p.b, st);
    ix->prof.pending.push_back(p);
}
// Ordered compaction driver shared by QS and QSRP: the sparse form (streaming pass, per-query sorted
// lists), and the two-pass form (count, scan, write) for the queries that flag more than kNeedCap users.
template <class P>
inline int run_compaction(rkr_index *ix, P p, int nq, KSpec ks, QueryCounts *counts, cudaStream_t st) {
    const int64_t U = ix->n_user;
    const int nchunks = (int) ((U + kCompactChunk - 1) / kCompactChunk);
    const size_t sparse = sizeof(int32_t) * ((size_t) nq * kNeedCap + 2 * (size_t) nq) + 256;
    const size_t two_pass = sizeof(int2) * 2 * (size_t) nq * nchunks + 256;
    RKR_TRY(ix->ws_cand_off.ensure(sparse + two_pass));
    int32_t *need_n = ix->ws_cand_off.as<int32_t>();
    int32_t *ovf_q = need_n + nq;
    int32_t *need_u = ovf_q + nq;
    int2 *cnt = reinterpret_cast<int2 *>(ix->ws_cand_off.as<uint8_t>() + sparse);
    int2 *off = cnt + (size_t) nq * nchunks;
    int *err = reinterpret_cast<int *>(off + (size_t) nq * nchunks);
    RKR_CUDA(cudaMemsetAsync(err, 0, 2 * sizeof(int), st));
    int h_err[2] = {0, 0};
    int n_two = nq;                  // queries on the two-pass form
    const int32_t *qmap = nullptr;   // which ones (nullptr: all)
    if (ix->compact_sparse_on) {
        RKR_CUDA(cudaMemsetAsync(need_n, 0, sizeof(int32_t) * nq, st));
        timed(ix, st, "compact_need", [&] {
            compact_need_flat_kernel<P><<<148 * 8, 256, 0, st>>>(p, U, nq, 1.0 / (double) U, need_n, need_u);
        });
        RKR_CUDA(cudaGetLastError());
        RKR_TRY(ix->ws_emit.ensure((sizeof(int8_t) + sizeof(typename P::Aux)) * (size_t) nq * kNeedCap + 256));
        int8_t *cls = ix->ws_emit.as<int8_t>();
        auto *aux = reinterpret_cast<typename P::Aux *>(ix->ws_emit.as<uint8_t>() +
                                                        (((size_t) nq * kNeedCap + 255) & ~size_t(255)));
        timed(ix, st, "compact_classify", [&] {
            compact_classify_kernel<P><<<148 * 16, 256, 0, st>>>(p, nq, need_n, need_u, cls, aux);
        });
        RKR_CUDA(cudaGetLastError());
        timed(ix, st, "compact_emit", [&] {
            compact_emit_kernel<P><<<(unsigned) nq, kCompactThreads, sizeof(uint64_t) * kNeedCap, st>>>(p, ks, need_n, need_u, cls, aux, counts,
                                                                             err, ovf_q);
        });
        RKR_CUDA(cudaGetLastError());
        RKR_CUDA(cudaMemcpyAsync(h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, st));
        RKR_CUDA(cudaStreamSynchronize(st));
        n_two = h_err[1];
        qmap = ovf_q;
        if (ix->prof.on && n_two) {
            // how far past the list the two-pass queries' flagged users go
            std::vector<int32_t> nn((size_t) nq);
            RKR_CUDA(cudaMemcpy(nn.data(), need_n, sizeof(int32_t) * nq, cudaMemcpyDeviceToHost));
            int64_t le8 = 0, le16 = 0, le64 = 0, more = 0;
            for (int32_t v : nn) {
                if (v <= kNeedCap) continue;
                if (v <= 2 * kNeedCap) le8++;
                else if (v <= 4 * kNeedCap) le16++;
                else if (v <= 16 * kNeedCap) le64++;
                else more++;
            }
            ix->prof.add_count("two_pass_need_to_2x_queries", le8);
            ix->prof.add_count("two_pass_need_to_4x_queries", le16);
            ix->prof.add_count("two_pass_need_to_16x_queries", le64);
            ix->prof.add_count("two_pass_need_beyond_queries", more);
        }
    }
    if (n_two) {
        const dim3 g2((unsigned) nchunks, (unsigned) n_two);
        timed(ix, st, "compact_count", [&] { compact_count_kernel<P><<<g2, kCompactThreads, 0, st>>>(p, U, nchunks, cnt, qmap); });
        RKR_CUDA(cudaGetLastError());
        timed(ix, st, "compact_scan", [&] {
            compact_scan_kernel<<<(n_two + 127) / 128, 128, 0, st>>>(cnt, nchunks, n_two, ks, off, counts, err, qmap);
        });
        RKR_CUDA(cudaGetLastError());
        timed(ix, st, "compact_write", [&] {
            compact_write_kernel<P><<<g2, kCompactThreads, 0, st>>>(p, U, nchunks, cnt, off, ks, qmap);
        });
        RKR_CUDA(cudaGetLastError());
        RKR_CUDA(cudaMemcpyAsync(h_err, err, sizeof(int), cudaMemcpyDeviceToHost, st));
        RKR_CUDA(cudaStreamSynchronize(st));
    }
    if (ix->prof.on) ix->prof.add_count("two_pass_compaction_queries", n_two);
    if (h_err[0]) {
        set_error("internal: candidate count mismatch in %d queries", h_err[0]);
        return RKR_ERR_STATE;
    }
    return RKR_OK;
}

// ---- user shards (rkr_shard.cu) ----
// counts[0..n) summed over the shards in place (no-op on a whole index).
int shard_sum(rkr_index *ix, int32_t *counts, int64_t n, cudaStream_t st);
// A buffer whose counts were already summed and to which a second pass then added this shard's
// counts: copy it before the second pass (shard_snapshot), then shard_sum_delta sums the added
// counts only.
int shard_snapshot(rkr_index *ix, int slot, const int32_t *counts, int64_t n, cudaStream_t st);
int shard_sum_delta(rkr_index *ix, int slot, int32_t *counts, int64_t n, cudaStream_t st);
// Sum over the shards of a host value (waits for the stream).
int shard_sum_host(rkr_index *ix, int32_t v, int32_t *sum, cudaStream_t st);
// counts[q].n_cand from the shard's (code, class) pairs, and ip_base kept on shard 0 only.
__global__ void shard_local_counts_kernel(const int2 *__restrict__ cnt, int nchunks, int nq, int keep_base,
                                          QueryCounts *__restrict__ counts);

// A user shard's candidate count per query: the global selection (counts as summed) decides each
// user's class, the shard counts its own users of the refinement class; the ordered compaction and
// refinement then run on the shard's candidates.  The results are counted by the compaction itself.
template <class P>
inline int shard_local_counts(rkr_index *ix, P p, int nq, QueryCounts *counts, cudaStream_t st) {
    const int64_t U = ix->n_user;
    const int nchunks = (int) ((U + kCompactChunk - 1) / kCompactChunk);
    RKR_TRY(ix->ws_cand_off.ensure(sizeof(int2) * (size_t) nq * nchunks + 256));
    int2 *cnt = reinterpret_cast<int2 *>(ix->ws_cand_off.p);
    const dim3 g((unsigned) nchunks, (unsigned) nq);
    timed(ix, st, "compact_count", [&] { compact_count_kernel<P><<<g, kCompactThreads, 0, st>>>(p, U, nchunks, cnt, nullptr); });
    RKR_CUDA(cudaGetLastError());
    shard_local_counts_kernel<<<(nq + 127) / 128, 128, 0, st>>>(cnt, nchunks, nq, ix->shard.index == 0, counts);
    RKR_CUDA(cudaGetLastError());
    return RKR_OK;
}

// Candidate refinement (refine_prep_kernel, then the per-item counting on tiles).
struct RefineArgs {
    const float *user;        // rows refined against the items (raw users)
    const float *query;       // [n_query][dim] (QS/US: the score is recomputed from it)
    const float *cand_qip;    // QSRP: score per candidate given; else nullptr
    const int32_t *cand_user;
    const int32_t *cand_query;
    const int32_t *cand_lb, *cand_ub;
    int64_t n_cand;
    int dim;
    int ipbound;              // 1: RefineCPUIPBound (QS, QSRP); 0: RefineCPU (US)
    const float *item_norm;   // descending (ipbound)
    int64_t n_item;
    // outputs
    float *qip;               // [n_cand]
    int32_t *rank;            // [n_cand]
    int32_t *nproc;           // [n_cand]
    int32_t *ref_idx;         // refined candidates (compacted)
    int32_t *ref_user;        // their users
    int32_t *n_ref;           // device counter
    int32_t *undecided;       // [n_cand] items whose score had to be computed in full
};

int ensure_device(const rkr_index *ix);
// Counting step of the refinement on the tensor cores; sets *done = false (and does nothing) where
// the shape does not fit it, leaving the exact tiles to run.
int refine_tc(rkr_index *ix, const RefineArgs &ra, cudaStream_t st, bool *done);
// Builds (once per split) the item tiles refine_tc reads.
int refine_tc_tiles(rkr_index *ix, bool ipbound, cudaStream_t st);
int thr_summary_build(rkr_index *ix);
// Regression models of users [u_begin, u_end) fitted on the device into ix->reg (rkr_fit.cu).
int fit_regression_device(rkr_index *ix, int64_t u_begin, int64_t u_end, cudaStream_t st);
// The SVD transform built on the device over all users and made the index's (rkr_svd.cu).
int svd_build_device(rkr_index *ix, float sigma_ratio, float *transfer_item_out, float *svd_user_out,
                     int32_t *check_dim_out);
// Thresholds of users [u_begin, u_end) for the index's sample ranks into ix->thr (rkr_build.cu).
int build_thresholds_range(rkr_index *ix, int64_t u_begin, int64_t u_end);
int level_tables_build(rkr_index *ix);
int refine_prepare_norms(rkr_index *ix);
// What a batch of queries asks for: top-k `topk` for every query (k null; outputs [n_query][topk]),
// or k[q] per query (host array; query q's outputs start at the sum of the earlier k's).  req_first
// (host, or null) scopes QSRPNormalLP's carried scores to requests: query q belongs to the request
// that starts at query req_first[q] of the batch, only that request's earlier queries carry scores
// to it, and a request starts from zero scores, as on a fresh index (the index's carried state is
// neither read nor advanced).
constexpr int kMaxChunkQueries = 4096;  // queries per device pass (a larger batch runs in chunks)
struct BatchSpec {
    int topk = 0;
    const int32_t *k = nullptr;
    const int32_t *req_first = nullptr;
    int32_t *front = nullptr;  // user shard (host, [n_query]): the result users at the front of each row
};
int query_batch(rkr_index *ix, int method, const float *d_query, int n_query, const BatchSpec &bs,
                rkr_user_rank *d_out, rkr_query_stats *d_stats, cudaStream_t st);
int build_sample_search(rkr_index *ix, const int32_t *sample_rank, int n_sample);
int score_sort_rows(rkr_index *ix, int64_t start, int64_t n_rows, float *h_rows);
int query_rank_distribution(rkr_index *ix, const int32_t *sample_item, int n_sample_item, int32_t *h_accu);
}  // namespace rkr
