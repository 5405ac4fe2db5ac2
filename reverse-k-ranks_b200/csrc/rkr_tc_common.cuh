// rkr_tc_common.cuh -- pieces shared by the int8 tensor-core kernels (pair scores, refinement):
// the digit operands, tcgen05 / mbarrier / bulk-copy helpers, and the digit arithmetic's bound.
//
// Digits.  Each row is scaled by a power of two 2^e with every |coordinate| < 2^(e-1) and split into
// four signed 7-bit digits per coordinate, a = 2^e (d1 2^-7 + d2 2^-14 + d3 2^-21 + d4 2^-28 + r),
// |d| <= 64, |r| <= 2^-29 (each digit the nearest integer of the remainder times 128, all steps exact
// in binary32).  The ten digit products with i + j <= 5 run as int8 MMAs (tcgen05.mma kind::i8)
// into four int32 TMEM accumulators per part; integer accumulation is exact.
#pragma once

#include <cmath>

#include "rkr_internal.cuh"

namespace rkr {
namespace {

constexpr int kScSlices = 4;                       // digits per coordinate
constexpr int kScMaxExp = 40;                      // rows scaled beyond 2^+-40 go to the exact path
constexpr int kScMaxPart = 240;                    // coordinates per part: digit sums stay below 2^22
constexpr int kScN = 32;                           // rows per B tile (the MMA's N)
constexpr int kScM = 128;                          // rows per A tile (the MMA's M, TMEM lanes)

__host__ __device__ inline int round32(int x) { return (x + 31) & ~31; }

// ---- operands ----------------------------------------------------------------------------------------

// Byte offset of (row rr, coordinate p) within one digit slice of a tile of tr rows, as 8-row x
// 16-byte core matrices: K blocks outermost ([kp / 16][tr / 8][8][16], the resident A tiles), or row
// groups outermost ([tr / 8][kp / 16][8][16], the stacked B tiles, whose slices then follow each other
// as whole 8-row groups).
__host__ __device__ inline size_t digit_off(int rr, int p, int tr, int kp, bool rows_outer) {
    return rows_outer ? (size_t) (rr >> 3) * (kp * 8) + (p >> 4) * 128 + (rr & 7) * 16 + (p & 15)
                      : (size_t) (p >> 4) * (tr * 16) + (rr >> 3) * 128 + (rr & 7) * 16 + (p & 15);
}

// Rows [n][dim] (gathered through idx when given) to the digit layout of the tiles: per tile of tr rows,
// 4 slices in the layout of digit_off; coordinates [0, c) at k in [0, c), [c, dim) at
// [cp, cp + dim - c), zeros elsewhere and in rows [n, n_pad).  meta[r] = {2^e, upper bounds of the
// weighted norms (sum_t w(t) x_t^2)^(1/2) of the two parts, e (as int bits)}; a row with a non-finite
// coordinate or a scale beyond 2^+-kScMaxExp gets 2^e = inf, which sends all of its pairs to the
// exact path.  One warp per row.
__global__ void slice_rows_kernel(const float *__restrict__ src, const int32_t *__restrict__ idx, int64_t n,
                                  int64_t n_pad, int dim, int c, int cp, int kp, int tr, int rows_outer,
                                  int8_t *__restrict__ dst, float4 *__restrict__ meta) {
    const int64_t r = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (r >= n_pad) return;
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
    int e = 0;
    if (mx > 0.0f) {
        int x;
        frexpf(mx, &x);  // mx = m 2^x, m in [0.5, 1): mx 2^-(x + 1) < 0.5
        e = x + 1;
    }
    if (e > kScMaxExp || e < -kScMaxExp) bad = 1;
    const float scale = bad ? 0.0f : ldexpf(1.0f, -e);
    double sl = 0.0, sr = 0.0;
    const size_t slice_bytes = (size_t) tr * kp;
    int8_t *tb = dst + (size_t) (r / tr) * kScSlices * slice_bytes;
    const int rr = (int) (r % tr);
    for (int p = lane; p < kp; p += 32) {
        const int k = p < cp ? (p < c ? p : -1) : (p - cp + c < dim ? p - cp + c : -1);
        float v = 0.0f;
        if (row && k >= 0) {
            v = row[k];
            // position t of the coordinate in its part's sequential sum, weight w(t) (see part_coef)
            const int t = k < c ? k : k - c, n = k < c ? c : dim - c;
            const double w = t == 0 ? n : n - t + 1;
            if (k < c) sl += w * v * v;
            else sr += w * v * v;
        }
        float a = v * scale;  // exact: a power of two
        const size_t off = digit_off(rr, p, tr, kp, rows_outer);
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
        sl += __shfl_xor_sync(0xffffffffu, sl, o);
        sr += __shfl_xor_sync(0xffffffffu, sr, o);
    }
    if (lane == 0) {
        float4 m;
        m.x = bad ? INFINITY : ldexpf(1.0f, e);
        m.y = __double2float_ru(sqrt(sl * (1.0 + 1e-12)));
        m.z = __double2float_ru(sqrt(sr * (1.0 + 1e-12)));
        m.w = __int_as_float(bad ? 0 : e);
        meta[r] = m;
    }
}

// ---- tcgen05 / mbarrier helpers ----------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t) __cvta_generic_to_shared(p); }

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

// Shared-memory matrix descriptor, K-major without swizzle: 8-row x 16-byte core matrices, lbo the
// byte distance between the two core matrices of one K step, sbo between groups of 8 rows.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t) ((saddr >> 4) & 0x3FFF);
    d |= (uint64_t) ((lbo >> 4) & 0x3FFF) << 16;
    d |= (uint64_t) ((sbo >> 4) & 0x3FFF) << 32;
    d |= (uint64_t) 1 << 46;  // descriptor version of sm_100
    return d;
}

// Instruction descriptor: kind::i8, A and B signed 8-bit K-major, int32 accumulator, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
    return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t) (n >> 3) << 17) | ((uint32_t) (kScM >> 4) << 24);
}
constexpr uint32_t kIdescI8 = idesc_i8(kScN);

__device__ __forceinline__ void umma_i8(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate,
                                        uint32_t idesc = kIdescI8) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t"
        "}\n" ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate) : "memory");
}

// The ten digit products of one K step as four MMAs: A slice i (a + i * a_slice) against B slices
// 0 .. 3 - i, which follow each other as row groups from b (the row-group-outer layout of digit_off),
// with N = 32 (4 - i) into the accumulators from column block i on (d + 32 i): column block g gets
// the products of digit pair (i, g - i).  Slice 0 writes all four blocks first (accumulate = 0 at a
// part's first K step).
__device__ __forceinline__ void umma_i8_step(uint32_t d, uint64_t a, uint32_t a_slice, uint64_t b, bool first) {
    umma_i8(d, a, b, !first, idesc_i8(4 * kScN));
    umma_i8(d + kScN, a + a_slice, b, 1u, idesc_i8(3 * kScN));
    umma_i8(d + 2 * kScN, a + 2 * a_slice, b, 1u, idesc_i8(2 * kScN));
    umma_i8(d + 3 * kScN, a + 3 * a_slice, b, 1u, idesc_i8(kScN));
}

// One lane of the (fully active) warp: the issuing lane of the copies, MMAs and commits, while the
// whole warp runs the loop around them (its values stay warp-uniform).
__device__ __forceinline__ bool elect_one() {
    uint32_t pred = 0;
    asm volatile("{\n\t.reg .pred p;\n\telect.sync _|p, 0xffffffff;\n\tselp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(pred));
    return pred != 0;
}

__device__ __forceinline__ void tmem_ld8(uint32_t addr, uint32_t (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(addr));
}

// int32 of magnitude below 2^22 to binary32, exactly (the value sits in the significand of 1.5 2^23).
__device__ __forceinline__ float i2f_small(uint32_t x) {
    return __fsub_rn(__int_as_float((int) x + 0x4B400000), 12582912.0f);
}
// 2^35 times the digit-product value of one part: a0 2^21 + a1 2^14 + a2 2^7 + a3.
__device__ __forceinline__ float combine4(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3) {
    return fmaf(fmaf(fmaf(i2f_small(a0), 128.0f, i2f_small(a1)), 128.0f, i2f_small(a2)), 128.0f, i2f_small(a3));
}
// The same for the eight columns of a tcgen05.ld, two columns per paired FP32 instruction
// (__fadd2_rn / __ffma2_rn round each component as __fadd_rn / __fmaf_rn do: the results are
// combine4's, bit for bit).
__device__ __forceinline__ void combine4_x8(const uint32_t a0[8], const uint32_t a1[8], const uint32_t a2[8],
                                            const uint32_t a3[8], float out[8]) {
    const float2 off = make_float2(-12582912.0f, -12582912.0f), k128 = make_float2(128.0f, 128.0f);
    auto f2 = [&](const uint32_t *a, int i) {
        return __fadd2_rn(make_float2(__int_as_float((int) a[i] + 0x4B400000), __int_as_float((int) a[i + 1] + 0x4B400000)),
                          off);
    };
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        float2 r = __ffma2_rn(f2(a0, i), k128, f2(a1, i));
        r = __ffma2_rn(r, k128, f2(a2, i));
        r = __ffma2_rn(r, k128, f2(a3, i));
        out[i] = r.x;
        out[i + 1] = r.y;
    }
}

// Bound coefficients of a part of n coordinates: (on the product of the rows' weighted norms, on
// 2^(ea + eb)).  The reference's sequential binary32 sum of p_t = a_t b_t (t = 1..n, one rounding
// per product and per addition) differs from the exact sum by at most u (1 + gamma_n) / (1 - u)
// sum_t w_t |p_t|, w_1 = n, w_t = n - t + 2 (each product's rounding, plus the rounding of every
// partial sum that contains it), and sum_t w_t |a_t b_t| <= Wa Wb with W = (sum_t w_t x_t^2)^(1/2)
// (Cauchy-Schwarz).  The digits: dropped products 3.02 n 2^-30, remainders n 2^-29, and the tails
// of the three roundings that combine the accumulators n 1.1e-4 u (their leading part, 3.002 u
// times the computed value, is added per pair).
inline void part_coef(int n, float &cn, float &ke) {
    if (n <= 0) {
        cn = ke = 0.0f;
        return;
    }
    const double u = 5.9604644775390625e-8;  // 2^-24
    const double gamma = n * u / (1.0 - n * u);
    cn = (float) (u * (1.0 + gamma) / (1.0 - u) * 1.0001);
    ke = (float) (n * (3.02 * 9.313225746154785e-10 + 1.862645149230957e-9 + 1.1e-4 * u) * 1.01);
}

}  // namespace
}  // namespace rkr
