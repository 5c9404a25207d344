// Device arithmetic of the SCMF engine: counter-based Philox4x32-10, uniform
// and Gaussian variates (a tabulated inverse normal CDF), and a project-written
// log.
//
// Every routine is IEEE single precision built from +, -, *, correctly rounded
// division and sqrt, and explicit __fmaf_rn; the translation unit is compiled
// with --fmad=false -prec-div=true -prec-sqrt=true so nothing else is fused.
// The results are therefore a pure function of the inputs and identical to a
// host build of the same expressions with -ffp-contract=off.
//
// The reference draws from a stateful cuRAND Philox4_32_10 per chain
// (device_function.cu:12-24, 683, 749) seeded by time(NULL)
// (init_config.cu:864).  Here the stream is stateless: the counter is
// (chain, bead, step, draw) and the key is the 64-bit seed, so any bead move
// can be replayed in any order.
#pragma once
#include <stdint.h>

#include "scmf_internal.h"

namespace scmf {

// Philox4x32-10: Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC'11.  Round multipliers 0xD2511F53 / 0xCD9E8D57, key
// increments 0x9E3779B9 / 0xBB67AE85.  Each 32x32->64 product is one wide
// multiply.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// philox4x32_10 with the round keys taken from a schedule (PhiloxKeys, the
// same bits).
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, const PhiloxKeys& ks) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ ks.k[2 * r], (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ ks.k[2 * r + 1],
                       (uint32_t)p0);
    }
    return c;
}

// philox4x32_10 with the first key word advanced in a register and the
// second word's round keys from a schedule (the same bits): for launches whose
// systems share the upper 32 bits of their seed.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, const PhiloxKeys& ks) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
        c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ ks.k[2 * r + 1],
                       (uint32_t)p0);
        k0 += 0x9E3779B9u;
    }
    return c;
}

// Uniform in (0, 1] from bits 9..31: 2 - 1.m with the 23 bits as mantissa
// (exact in FP32; no integer-to-float conversion).
__device__ __forceinline__ float u01(uint32_t w) {
    return __fsub_rn(2.0f, __uint_as_float(0x3F800000u | (w >> 9)));
}

// log(x) for normal x > 0.  x = 2^e m with m in [sqrt(1/2), sqrt(2));
// log m = log1p(t) = t + t^2 Q(t), t = m - 1 (exact), Q of degree 8 fitted by
// weighted least squares on Chebyshev nodes (gen_log_poly.py); e ln2 with a
// 12-bit head of ln2 so that e * head is exact.  No division, no branch.
__device__ __forceinline__ float log_f(float x) {
    const uint32_t ix = __float_as_uint(x);
    int e = (int)(ix >> 23) - 127;
    uint32_t mb = (ix & 0x007FFFFFu) | 0x3F800000u;
    const bool hi = mb > 0x3FB504F3u;
    mb = hi ? mb - 0x00800000u : mb;
    e = hi ? e + 1 : e;
    const float t = __fsub_rn(__uint_as_float(mb), 1.0f);
    float q = -0x1.321a4cp-4f;
    q = __fmaf_rn(q, t, 0x1.068b2ap-3f);
    q = __fmaf_rn(q, t, -0x1.0f9b0cp-3f);
    q = __fmaf_rn(q, t, 0x1.22bf86p-3f);
    q = __fmaf_rn(q, t, -0x1.5424e0p-3f);
    q = __fmaf_rn(q, t, 0x1.999fc2p-3f);
    q = __fmaf_rn(q, t, -0x1.000422p-2f);
    q = __fmaf_rn(q, t, 0x1.555558p-2f);
    q = __fmaf_rn(q, t, -0x1.fffff8p-2f);
    const float lm = __fmaf_rn(__fmul_rn(t, t), q, t);
    const float fe = __int2float_rn(e);
    return __fmaf_rn(fe, 0x1.62ep-1f, __fmaf_rn(fe, 0x1.0bfbe8p-15f, lm));
}

// A lower bound of log_f(u), linear in the bits of u: for u = 2^e (1 + f),
// f in [0, 1), log2(1 + f) >= f (the chord of a concave function), so
// (bits(u) 2^-23 - 127) ln2 <= log u; one conversion and one fma, less a
// slack of 2^-12 that covers their rounding and log_f's own error (checked
// for all 2^23 values u01 yields against the oracle's log by the oracle
// tests).  It lies 0.04 below log u on average (the exponent alone, e ln2,
// lies 0.39 below), so fewer trials need the logarithm or the omega reads.
__device__ __forceinline__ float log_lower(float u) {
    return __fmaf_rn(__uint2float_rn(__float_as_uint(u)), 0x1.62e43p-24f, -0x1.601ea8p+6f);
}

// One standard normal from one 32-bit word by the inverse normal CDF: bit 31
// is the sign, bits 0..30 give f = 2 (w mod 2^31) + 1 rounded to FP32 (in
// [1, 2^32]) and the magnitude is the half-normal quantile h(f 2^-32),
// h(v) = -Phi^-1(v / 2), from a table of 513 cubic segments (16 per binade
// of f, picked by the exponent and the top four mantissa bits; the local
// coordinate t in [-2^-5, 2^-5) is the low 19 mantissa bits, exactly).  The
// table (scmf_normal_table.h, written by gen_normal_table.py) is within
// 1.3e-7 relative of the quantile, and reaches 6.34 sigma.  `tab` points at
// the global table, or at a lane's copy in shared memory where STRIDE copies
// are entry-interleaved; the bits are the same.
template <int STRIDE = 1>
__device__ __forceinline__ float normal_of(uint32_t w, const float4* __restrict__ tab) {
    const uint32_t b = __float_as_uint(__uint2float_rn((w << 1) | 1u));
    const float4 c = tab[((b >> 19) - (127u << 4)) * STRIDE];
    const float t = __fsub_rn(__uint_as_float((b & 0x7FFFFu) | 0x3F800000u), 1.03125f);
    float z = __fmaf_rn(c.w, t, c.z);
    z = __fmaf_rn(z, t, c.y);
    z = __fmaf_rn(z, t, c.x);
    return __uint_as_float(__float_as_uint(z) ^ (w & 0x80000000u));
}

// The three normals of a move from words x, y, z of its Philox block.
template <int STRIDE = 1>
__device__ __forceinline__ void normals3(uint4 w, const float4* __restrict__ tab, float& n0, float& n1, float& n2) {
    n0 = normal_of<STRIDE>(w.x, tab);
    n1 = normal_of<STRIDE>(w.y, tab);
    n2 = normal_of<STRIDE>(w.z, tab);
}

// The Metropolis word of a move: word w of the same block (u01 reads its bits
// 9..31).
__device__ __forceinline__ uint32_t accept_word(uint4 w) { return w.w; }

// floor(x * inv_d) mod n, in [0, n), for |x * inv_d| < 2^22 (beyond that the
// index stays in [0, n) but need not be the floor).  FP32 restatement of the
// periodic fold in coord_to_index_unified_high (device_function.cu:313-360).
// floor(t) of the exact product t = x * inv_d, for |t| < 2^22, in one fused
// multiply-add and no conversion instruction: x * inv_d + 1.5*2^23 rounded
// down (once, __fmaf_rd) is 1.5*2^23 + floor(t) exactly, an integer-valued
// float whose mantissa holds the floor.
// One box away is folded with selects; the general modulo only runs for
// coordinates more than one box length outside the primary box.
__device__ __forceinline__ int fold(float x, float inv_d, int n) {
    int i = __float_as_int(__fmaf_rd(x, inv_d, 0x1.8p23f)) - 0x4B400000;
    i = i < 0 ? i + n : i;
    i = i >= n ? i - n : i;
    if ((unsigned)i >= (unsigned)n) {
        i %= n;
        if (i < 0) i += n;
    }
    return i;
}

// The same fold for 2 <= n <= 256 without selects or branches.  The floor is
// read with a bias B = n * ceil(2^22 / n) folded into the integer offset
// (off = 0x4B400000 - B), so j = floor(t) + B lies in [0, 2^23 + n) for
// |t| < 2^22, and j mod n = j - n * umulhi(j, mag) with mag = ceil(2^32 / n),
// exact for every j < 2^24 and n <= 256 (Granlund and Montgomery, "Division
// by invariant integers using multiplication", PLDI 1994; checked for all
// such j and n).  Clamping j below 2^24 keeps every input, NaN included,
// inside [0, n).  off and mag come from a table indexed by n.
__device__ __forceinline__ int fold_magic(float x, float inv_d, int n, int off, uint32_t mag) {
    uint32_t j = (uint32_t)(__float_as_int(__fmaf_rd(x, inv_d, 0x1.8p23f)) - off);
    j = min(j, 0x00FFFFFFu);
    return (int)(j - __umulhi(j, mag) * (uint32_t)n);
}

// The same fold for a power-of-two n: the low log2(n) bits of the mantissa
// of t + 1.5*2^23 (rounded down once) are floor(t) mod n, because 0x4B400000, the
// offset of that mantissa, has no bits below 2^22.  Exact for |t| < 2^22.
__device__ __forceinline__ int fold_pow2(float x, float inv_d, int mask) {
    return __float_as_int(__fmaf_rd(x, inv_d, 0x1.8p23f)) & mask;
}

}  // namespace scmf
