// Minimal stand-in for NTL::ZZ covering what kunpBFV's context precompute uses
// (construction from an integer, shifts, +,-,*,/ and % by words, products,
// comparisons, to_ulong). Fixed width: 32 x 64-bit words, unsigned.
// Test infrastructure for the reference-kernel harness only.
#pragma once
#include <cstdint>
#include <cstring>
#include <ostream>

namespace NTL {

class ZZ {
public:
    static const int W = 32;
    uint64_t w[W];
    ZZ() { std::memset(w, 0, sizeof w); }
    ZZ(long v) { std::memset(w, 0, sizeof w); w[0] = (uint64_t)v; }
    ZZ(unsigned long v) { std::memset(w, 0, sizeof w); w[0] = v; }
    ZZ(unsigned long long v) { std::memset(w, 0, sizeof w); w[0] = v; }
    ZZ(int v) { std::memset(w, 0, sizeof w); w[0] = (uint64_t)(int64_t)v; }

    ZZ& operator<<=(int s) { *this = *this << s; return *this; }
    ZZ operator<<(int s) const {
        ZZ r;
        int ws = s / 64, bs = s % 64;
        for (int i = W - 1; i >= ws; i--) {
            uint64_t v = w[i - ws] << bs;
            if (bs && i - ws - 1 >= 0) v |= w[i - ws - 1] >> (64 - bs);
            r.w[i] = v;
        }
        return r;
    }
    ZZ operator>>(int s) const {
        ZZ r;
        int ws = s / 64, bs = s % 64;
        for (int i = 0; i + ws < W; i++) {
            uint64_t v = w[i + ws] >> bs;
            if (bs && i + ws + 1 < W) v |= w[i + ws + 1] << (64 - bs);
            r.w[i] = v;
        }
        return r;
    }
    ZZ& operator*=(uint64_t m) {
        unsigned __int128 c = 0;
        for (int i = 0; i < W; i++) {
            unsigned __int128 t = (unsigned __int128)w[i] * m + c;
            w[i] = (uint64_t)t;
            c = t >> 64;
        }
        return *this;
    }
    ZZ& operator*=(const ZZ& o) { *this = *this * o; return *this; }
    ZZ operator*(const ZZ& o) const {
        ZZ r;
        for (int i = 0; i < W; i++) {
            unsigned __int128 c = 0;
            for (int j = 0; i + j < W; j++) {
                unsigned __int128 t = (unsigned __int128)w[i] * o.w[j] + r.w[i + j] + c;
                r.w[i + j] = (uint64_t)t;
                c = t >> 64;
            }
        }
        return r;
    }
    ZZ operator*(long m) const { ZZ r = *this; r *= (uint64_t)m; return r; }
    ZZ operator*(int m) const { ZZ r = *this; r *= (uint64_t)m; return r; }
    ZZ operator*(unsigned long m) const { ZZ r = *this; r *= (uint64_t)m; return r; }
    ZZ operator*(unsigned long long m) const { ZZ r = *this; r *= (uint64_t)m; return r; }
    ZZ& operator/=(uint64_t m) {
        unsigned __int128 r = 0;
        for (int i = W - 1; i >= 0; i--) {
            unsigned __int128 cur = (r << 64) | w[i];
            w[i] = (uint64_t)(cur / m);
            r = cur % m;
        }
        return *this;
    }
    long operator%(uint64_t m) const {
        unsigned __int128 r = 0;
        for (int i = W - 1; i >= 0; i--) r = ((r << 64) | w[i]) % m;
        return (long)(uint64_t)r;
    }
    ZZ operator-(const ZZ& o) const {
        ZZ r;
        uint64_t br = 0;
        for (int i = 0; i < W; i++) {
            uint64_t x = w[i], y = o.w[i];
            uint64_t d = x - y - br;
            br = (x < y) || (x - y < br);
            r.w[i] = d;
        }
        return r;
    }
    bool operator>(const ZZ& o) const {
        for (int i = W - 1; i >= 0; i--)
            if (w[i] != o.w[i]) return w[i] > o.w[i];
        return false;
    }
};

inline unsigned long to_ulong(const ZZ& a) { return (unsigned long)a.w[0]; }
inline std::ostream& operator<<(std::ostream& os, const ZZ&) { return os << "<ZZ>"; }

}  // namespace NTL
