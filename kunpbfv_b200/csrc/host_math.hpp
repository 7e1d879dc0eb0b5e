// Host-side number theory for parameter-set construction (no external big-int library).
//
// The reference builds these with NTL and SEAL-style helpers
// (include/BFVcontext.cuh:130-542, include/uintarith_bfv.h); here they are
// plain 64/128-bit integer routines and a small fixed-width multiword type.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace kbfv {
namespace host {

typedef unsigned __int128 u128;

inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
inline uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = mulmod(r, a, q);
        a = mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}
inline uint64_t invmod(uint64_t a, uint64_t q) { return powmod(a % q, q - 2, q); }
inline uint64_t shoup(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }
inline int bit_count(uint64_t x) {
    int b = 0;
    while (x) { b++; x >>= 1; }
    return b;
}
// floor(2^128 / q) as (hi, lo)
inline void barrett_mu(uint64_t q, uint64_t& hi, uint64_t& lo) {
    // 2^128 / q = (2^128 - 1) / q unless q divides 2^128 (q odd prime: never)
    u128 all = ~(u128)0;
    u128 m = all / q;
    hi = (uint64_t)(m >> 64);
    lo = (uint64_t)m;
}

inline bool is_prime(uint64_t n) {
    if (n < 2) return false;
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (uint64_t p : small) {
        if (n == p) return true;
        if (n % p == 0) return false;
    }
    uint64_t d = n - 1;
    int s = 0;
    while ((d & 1) == 0) { d >>= 1; s++; }
    for (uint64_t a : small) {
        uint64_t x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool comp = true;
        for (int r = 1; r < s; r++) {
            x = mulmod(x, x, n);
            if (x == n - 1) { comp = false; break; }
        }
        if (comp) return false;
    }
    return true;
}

// Primitive-root search with the reference's factorisation loop bound
// (include/Utils.cuh:54-88): the trial divisor runs while i < sqrt(remaining).
inline uint64_t primitive_root(uint64_t q) {
    std::vector<uint64_t> fac;
    uint64_t number = q - 1;
    if (number % 2 == 0) {
        fac.push_back(2);
        while (number % 2 == 0) number /= 2;
    }
    for (uint64_t i = 3; (double)i < std::sqrt((double)number); i++) {
        if (number % i == 0) {
            fac.push_back(i);
            while (number % i == 0) number /= i;
        }
    }
    if (number > 2) {
        bool dup = false;
        for (uint64_t f : fac) dup |= (f == number);
        if (!dup) fac.push_back(number);
    }
    const uint64_t phi = q - 1;
    for (uint64_t r = 2; r <= phi; r++) {
        bool bad = false;
        for (uint64_t f : fac)
            if (powmod(r, phi / f, q) == 1) { bad = true; break; }
        if (!bad) return r;
    }
    return ~(uint64_t)0;
}

// findMthRootOfUnity(2N, q) (include/Utils.cuh:90-101)
inline uint64_t root_2n(uint64_t q, uint64_t n) {
    uint64_t m = 2 * n;
    if ((q - 1) % m != 0) return ~(uint64_t)0;
    return powmod(primitive_root(q), (q - 1) / m, q);
}
inline bool root_ok(uint64_t psi, uint64_t q, uint64_t n) {
    return psi != ~(uint64_t)0 && powmod(psi, n, q) == q - 1;
}

// get_primes_below (include/uintarith_bfv.h:983-1016), skipping primes whose
// 2N-th root is not primitive.
inline std::vector<uint64_t> primes_below(uint64_t n, uint64_t upper, size_t count) {
    std::vector<uint64_t> out;
    uint64_t factor = 2 * n;
    uint64_t value = upper - factor;
    uint64_t lower = (uint64_t)1 << (bit_count(upper) - 1);
    while (out.size() < count && value > lower) {
        if (is_prime(value) && root_ok(root_2n(value, n), value, n)) out.push_back(value);
        value -= factor;
    }
    return out;
}

// Largest primes below 2^bits that are 1 mod 2N with a primitive 2N-th root.
inline std::vector<uint64_t> primes_bits(uint64_t n, int bits, size_t count, const std::vector<uint64_t>& skip) {
    std::vector<uint64_t> out;
    uint64_t factor = 2 * n;
    uint64_t value = ((uint64_t)1 << bits) + 1 - factor;
    uint64_t lower = (uint64_t)1 << (bits - 1);
    while (out.size() < count && value > lower) {
        bool ex = false;
        for (uint64_t s : skip) ex |= (s == value);
        if (!ex && is_prime(value) && root_ok(root_2n(value, n), value, n)) out.push_back(value);
        value -= factor;
    }
    return out;
}

// fixed-width multiword unsigned integer, little-endian 64-bit words
struct Big {
    static const int W = 24;
    uint64_t w[W];
    explicit Big(uint64_t v = 0) { std::memset(w, 0, sizeof w); w[0] = v; }
    void mul_word(uint64_t m) {
        u128 c = 0;
        for (int i = 0; i < W; i++) {
            u128 t = (u128)w[i] * m + c;
            w[i] = (uint64_t)t;
            c = t >> 64;
        }
    }
    uint64_t mod_word(uint64_t m) const {
        u128 r = 0;
        for (int i = W - 1; i >= 0; i--) r = ((r << 64) | w[i]) % m;
        return (uint64_t)r;
    }
    Big div_word(uint64_t m) const {
        Big q;
        u128 r = 0;
        for (int i = W - 1; i >= 0; i--) {
            u128 cur = (r << 64) | w[i];
            q.w[i] = (uint64_t)(cur / m);
            r = cur % m;
        }
        return q;
    }
    int cmp(const Big& o) const {
        for (int i = W - 1; i >= 0; i--)
            if (w[i] != o.w[i]) return w[i] > o.w[i] ? 1 : -1;
        return 0;
    }
    void add(const Big& o) {
        u128 c = 0;
        for (int i = 0; i < W; i++) {
            u128 t = (u128)w[i] + o.w[i] + c;
            w[i] = (uint64_t)t;
            c = t >> 64;
        }
    }
    void sub(const Big& o) {
        uint64_t br = 0;
        for (int i = 0; i < W; i++) {
            uint64_t x = w[i], y = o.w[i];
            uint64_t d = x - y - br;
            br = (x < y) || (x - y < br);
            w[i] = d;
        }
    }
    double log2v() const {
        int top = W - 1;
        while (top > 0 && w[top] == 0) top--;
        if (top == 0 && w[0] == 0) return -INFINITY;
        double v = (double)w[top];
        if (top > 0) v += (double)w[top - 1] / 18446744073709551616.0;
        return std::log2(v) + 64.0 * top;
    }
};

}  // namespace host
}  // namespace kbfv
