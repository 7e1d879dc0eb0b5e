// Device modular arithmetic for 60-bit RNS limbs.
//
// All values are uint64 residues. Products of two residues are formed as
// 128-bit (hi, lo) pairs with __umul64hi; reductions are exact. The lazy
// Shoup product returns a value in [0, 2q) for any 64-bit input, which the
// NTT butterflies keep below 4q (requires q < 2^62).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace kbfv {

struct u128 {
    uint64_t lo, hi;
};

__device__ __forceinline__ u128 mul_wide(uint64_t a, uint64_t b) {
    u128 r;
    r.lo = a * b;
    r.hi = __umul64hi(a, b);
    return r;
}

// acc += a * b (128-bit, no overflow handling beyond 2^128), from 64-bit
// multiplies (mac32 below computes the same from 32-bit partial products)
__device__ __forceinline__ void mac64(u128& acc, uint64_t a, uint64_t b) {
    uint64_t lo = a * b;
    uint64_t hi = __umul64hi(a, b);
    asm("add.cc.u64 %0, %0, %2;\n\taddc.u64 %1, %1, %3;"
        : "+l"(acc.lo), "+l"(acc.hi)
        : "l"(lo), "l"(hi));
}

// acc += a * b from 32-bit partial products with carry chains (mad.lo/hi.cc
// on 32-bit halves) instead of 64-bit multiplies: eight 32-bit multiplies and
// two carry adds. Same result as mac() while the sum stays below 2^128.
__device__ __forceinline__ void mac32(u128& acc, uint64_t a, uint64_t b) {
    const uint32_t a0 = (uint32_t)a, a1 = (uint32_t)(a >> 32), b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    uint32_t r0 = (uint32_t)acc.lo, r1 = (uint32_t)(acc.lo >> 32), r2 = (uint32_t)acc.hi,
             r3 = (uint32_t)(acc.hi >> 32);
    asm("mad.lo.cc.u32  %0, %4, %6, %0;\n\t"
        "madc.hi.cc.u32 %1, %4, %6, %1;\n\t"
        "madc.lo.cc.u32 %2, %5, %7, %2;\n\t"
        "madc.hi.u32    %3, %5, %7, %3;\n\t"
        "mad.lo.cc.u32  %1, %4, %7, %1;\n\t"
        "madc.hi.cc.u32 %2, %4, %7, %2;\n\t"
        "addc.u32       %3, %3, 0;\n\t"
        "mad.lo.cc.u32  %1, %5, %6, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %6, %2;\n\t"
        "addc.u32       %3, %3, 0;"
        : "+r"(r0), "+r"(r1), "+r"(r2), "+r"(r3)
        : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
    acc.lo = ((uint64_t)r1 << 32) | r0;
    acc.hi = ((uint64_t)r3 << 32) | r2;
}

// the multiply-accumulate of the kernels: mac32 (25% more per cycle than mac64
// on the B200 in isolated register chains)
__device__ __forceinline__ void mac(u128& acc, uint64_t a, uint64_t b) { mac32(acc, a, b); }

__device__ __forceinline__ void sub128(u128& acc, uint64_t v) {
    asm("sub.cc.u64 %0, %0, %2;\n\tsubc.u64 %1, %1, 0;" : "+l"(acc.lo), "+l"(acc.hi) : "l"(v));
}

__device__ __forceinline__ uint64_t csub(uint64_t a, uint64_t q) { return a >= q ? a - q : a; }
__device__ __forceinline__ uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) { return csub(a + b, q); }
__device__ __forceinline__ uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) { return csub(a + q - b, q); }

// Shoup: b * w mod q with ws = floor(w * 2^64 / q); result in [0, 2q)
__device__ __forceinline__ uint64_t shoup_lazy(uint64_t b, uint64_t w, uint64_t ws, uint64_t q) {
    return b * w - __umul64hi(b, ws) * q;
}
__device__ __forceinline__ uint64_t shoup(uint64_t b, uint64_t w, uint64_t ws, uint64_t q) {
    return csub(shoup_lazy(b, w, ws, q), q);
}

// Barrett reduction of a 128-bit value with mu = floor(2^128 / q) = (mu_hi, mu_lo).
// The quotient estimate drops the low carry of lo*mu_lo and errs low by at
// most 2; two conditional subtractions make the result exact for q < 2^62.
__device__ __forceinline__ uint64_t barrett128(u128 x, uint64_t q, uint64_t mu_hi, uint64_t mu_lo) {
    // quotient ~ floor(x * mu / 2^128)
    uint64_t t1 = __umul64hi(x.lo, mu_lo);
    uint64_t a_lo = x.lo * mu_hi, a_hi = __umul64hi(x.lo, mu_hi);
    uint64_t b_lo = x.hi * mu_lo, b_hi = __umul64hi(x.hi, mu_lo);
    // middle word = t1 + a_lo + b_lo; only its carries reach the quotient
    uint64_t m1 = t1 + a_lo;
    uint64_t c1 = m1 < t1;
    uint64_t m2 = m1 + b_lo;
    uint64_t c2 = m2 < m1;
    uint64_t quot = x.hi * mu_hi + a_hi + b_hi + c1 + c2;
    uint64_t r = x.lo - quot * q;
    r = csub(r, q);
    r = csub(r, q);
    return r;
}

// Product-sized values, x < 2^(2k+2) with k = bit length of q (k <= 60): the
// quotient comes from one 64x64 high product, t = floor(x / 2^(k-2)) and
// mu = floor(2^(62+k) / q) < 2^64; the estimate is low by at most 3, so two
// conditional subtractions (2q, then q) give [0, q).
__device__ __forceinline__ uint64_t barrett_prod(u128 x, uint64_t q, uint64_t mu) {
    const int s = 62 - __clzll(q);  // k - 2
    const uint64_t t = (x.lo >> s) | (x.hi << (64 - s));
    uint64_t r = x.lo - __umul64hi(t, mu) * q;
    r = csub(r, q << 1);
    return csub(r, q);
}
__device__ __forceinline__ uint64_t mul_mod_prod(uint64_t a, uint64_t b, uint64_t q, uint64_t mu) {
    return barrett_prod(mul_wide(a, b), q, mu);
}

// 64-bit value mod q with the high word of mu: floor(a * mu_hi / 2^64) errs by at most 1
__device__ __forceinline__ uint64_t barrett64(uint64_t a, uint64_t q, uint64_t mu_hi) {
    uint64_t r = a - __umul64hi(a, mu_hi) * q;
    return csub(r, q);
}

__device__ __forceinline__ uint64_t mul_mod(uint64_t a, uint64_t b, uint64_t q, uint64_t mu_hi, uint64_t mu_lo) {
    return barrett128(mul_wide(a, b), q, mu_hi, mu_lo);
}

}  // namespace kbfv
