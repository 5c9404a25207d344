// Device arithmetic of the SCMF engine: counter-based Philox4x32-10, uniform
// and Gaussian variates, and project-written log / sin / cos.
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

// A lower bound of log_f(u) from the exponent alone: u in [2^e, 2^(e+1))
// gives log_f(u) >= e ln2 - 2^-10 (log_f rounds within ~2e-6 of log, and
// log u >= e ln2; checked for all 2^23 values u01 yields by the oracle test).
__device__ __forceinline__ float log_floor(float u) {
    const int e = (int)(__float_as_uint(u) >> 23) - 127;
    return __fmaf_rn(__int2float_rn(e), 0x1.62e430p-1f, -0x1p-10f);
}

// -2 ln u for u in (0, 1]: the squared Box-Muller radius.  u = 2^k m with m in
// [sqrt(1/2), sqrt(2)) split off in integers (k from the bits of u minus those
// of sqrt(1/2)), t = m - 1 exact, -2 log1p(t) = -2t + t^2 Q2(t) with Q2 = -2 Q
// of log_f (the same fit, scaled by -2 exactly), and -2 k ln2 added with
// -2 ln2 rounded to FP32 (at most 9e-8 off for the k >= -23 that u01 yields).
__device__ __forceinline__ float rad2_f(float u) {
    const uint32_t ix = __float_as_uint(u) - 0x3F3504F3u;
    const int k = (int)ix >> 23;
    const float t = __fsub_rn(__uint_as_float((ix & 0x007FFFFFu) + 0x3F3504F3u), 1.0f);
    float q = 0x1.321a4cp-3f;
    q = __fmaf_rn(q, t, -0x1.068b2ap-2f);
    q = __fmaf_rn(q, t, 0x1.0f9b0cp-2f);
    q = __fmaf_rn(q, t, -0x1.22bf86p-2f);
    q = __fmaf_rn(q, t, 0x1.5424e0p-2f);
    q = __fmaf_rn(q, t, -0x1.999fc2p-2f);
    q = __fmaf_rn(q, t, 0x1.000422p-1f);
    q = __fmaf_rn(q, t, -0x1.555558p-1f);
    q = __fmaf_rn(q, t, 0x1.fffff8p-1f);
    const float r2 = __fmaf_rn(__fmul_rn(t, t), q, __fmul_rn(-2.0f, t));
    return __fmaf_rn(__int2float_rn(k), -0x1.62e430p+0f, r2);
}

// sin and cos of 2 pi (2j+1) 2^-24 with j = w >> 9: the quadrant is removed in
// integers, the remainder g in [-1/2, 1/2) of a quadrant goes through
// sin(pi g / 2) = g S(g^2) (to g^7) and cos(pi g / 2) = 1 + g^2 C(g^2) (to g^8),
// S and C fitted by least squares on Chebyshev nodes (gen_sincos_poly.py;
// at most 1e-7 absolute error in FP32).
__device__ __forceinline__ void sincos_turn(uint32_t w, float& s, float& c) {
    const int32_t v = (int32_t)(((w >> 9) << 1) | 1u);
    const int32_t qv = (v + (1 << 21)) >> 22;
    const int32_t r = v - (qv << 22);
    const int q = qv & 3;
    const float g = __fmul_rn(__int2float_rn(r), 0x1p-22f);
    const float g2 = __fmul_rn(g, g);
    float sp = -0x1.2cf598p-8f;
    sp = __fmaf_rn(sp, g2, 0x1.465a3cp-4f);
    sp = __fmaf_rn(sp, g2, -0x1.4abba8p-1f);
    sp = __fmaf_rn(sp, g2, 0x1.921fb4p+0f);
    const float sa = __fmul_rn(g, sp);
    float cp = 0x1.d9f188p-11f;
    cp = __fmaf_rn(cp, g2, -0x1.55c64ap-6f);
    cp = __fmaf_rn(cp, g2, 0x1.03c1dep-2f);
    cp = __fmaf_rn(cp, g2, -0x1.3bd3ccp+0f);
    const float ca = __fmaf_rn(cp, g2, 1.0f);
    const bool odd = q & 1, neg_s = q & 2, neg_c = (q == 1) || (q == 2);
    const float s0 = odd ? ca : sa;
    const float c0 = odd ? sa : ca;
    s = neg_s ? -s0 : s0;
    c = neg_c ? -c0 : c0;
}

// Three standard normals from one Philox block (Box-Muller on (w.x, w.y) and
// on (w.z, w.w), the last sine unused).  Only bits 8..31 of each word are
// read; the low bytes feed accept_word().
__device__ __forceinline__ void normals3(uint4 w, float& n0, float& n1, float& n2) {
    float s, c;
    const float r0 = __fsqrt_rn(rad2_f(u01(w.x)));
    sincos_turn(w.y, s, c);
    n0 = __fmul_rn(r0, c);
    n1 = __fmul_rn(r0, s);
    const float r1 = __fsqrt_rn(rad2_f(u01(w.z)));
    sincos_turn(w.w, s, c);
    n2 = __fmul_rn(r1, c);
}

// normals3 that also returns the spare sine of its second Box-Muller pair
// (the first normal of the next, odd, bead).
__device__ __forceinline__ void normals3_spare(uint4 w, float& n0, float& n1, float& n2, float& spare) {
    float s, c;
    const float r0 = __fsqrt_rn(rad2_f(u01(w.x)));
    sincos_turn(w.y, s, c);
    n0 = __fmul_rn(r0, c);
    n1 = __fmul_rn(r0, s);
    const float r1 = __fsqrt_rn(rad2_f(u01(w.z)));
    sincos_turn(w.w, s, c);
    n2 = __fmul_rn(r1, c);
    spare = __fmul_rn(r1, s);
}

// The spare sine of bead b-1's block, for an odd bead b whose even partner is
// not at hand.
__device__ __forceinline__ float spare_of(uint4 wp) {
    float s, c;
    const float r1 = __fsqrt_rn(rad2_f(u01(wp.z)));
    sincos_turn(wp.w, s, c);
    return __fmul_rn(r1, s);
}

// Normals of an odd bead: the spare sine of bead b-1, then Box-Muller on
// (w.x, w.y) of its own block.  Three Box-Muller pairs per two beads.
__device__ __forceinline__ void normals3_odd(float spare, uint4 w, float& n0, float& n1, float& n2) {
    float s, c;
    const float r = __fsqrt_rn(rad2_f(u01(w.x)));
    sincos_turn(w.y, s, c);
    n0 = spare;
    n1 = __fmul_rn(r, c);
    n2 = __fmul_rn(r, s);
}

// The Metropolis uniform of a move: the low bytes of w.y, w.z, w.w of the
// block that gave its normals (bits the normals never read).
__device__ __forceinline__ uint32_t accept_word(uint4 w) {
    return ((w.y & 0xFFu) << 24) | ((w.z & 0xFFu) << 16) | ((w.w & 0xFFu) << 8);
}

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
