// Batched negacyclic NTT / inverse NTT over 60-bit primes for sm_100a.
//
// Convention (the reference's, include/ntt_60bit.cuh and include/Utils.cuh:171-191):
// forward Cooley-Tukey with psi_br[i] = psi^brv(i); output index k holds
// A(psi^(2*brv(k)+1)), fully reduced. Inverse Gentleman-Sande with
// psi^-brv(i), n^-1 folded into the last stage; output fully reduced.
//
// Shape: one CTA transforms one block of 2^LOGB points held in shared memory
// (N = 2^14 -> 1024 threads x 16 points, 136 KiB of padded smem). Each thread
// runs register groups of 16 points through 4 butterfly stages between
// shared-memory exchanges (N = 2^14: stages 4 + 4 + 4 + 2, three exchanges). Larger rings (2^15, 2^16),
// and launches of few rows at 2^14, add one elementwise radix-2^RC column pass in
// front of (forward) or behind (inverse) 2^12-point block kernels (the launch
// code picks the split). Moduli must be below 2^60 (lazy range 8q < 2^63).
//
// Rows are described by Src/Dst functors: src.prime(row) (or src.tables(row,
// inverse), see RowTab) and src.bind(row) -> {load(j), store(j, v)}. This lets pipeline stages fuse their per-element
// prologue (e.g. a tensor product) and epilogue (e.g. a key product) into the
// transform's first load and last store, which are always coalesced
// (consecutive threads touch consecutive j).
#pragma once
#include <type_traits>
#include <utility>

#include "arith.cuh"

namespace kbfv {

typedef ulonglong2 tw_t;  // (w, floor(w * 2^64 / q))

// The twiddle table and modulus of one row. By default they come from the
// launch's prime table (tw_all + prime(row) * N, mods[prime(row)]); a functor
// whose rows belong to different parameter sets (the levels of a mixed-level
// batch) provides `tables(row, inverse)` itself.
struct RowTab {
    const tw_t* tw;
    uint64_t q;
};
template <class T, class = void>
struct has_row_tables : std::false_type {};
template <class T>
struct has_row_tables<T, std::void_t<decltype(std::declval<const T&>().tables(0, false))>> : std::true_type {};

template <class Src>
__device__ __forceinline__ RowTab row_tab(const Src& s, int row, bool inverse, const tw_t* __restrict__ tw_all,
                                          const uint64_t* __restrict__ mods, int logn) {
    if constexpr (has_row_tables<Src>::value) {
        return s.tables(row, inverse);
    } else {
        const int p = s.prime(row);
        return RowTab{tw_all + ((size_t)p << logn), mods[p]};
    }
}

// The two constants of the inverse transform's last stage (n^-1 and
// psi_br^-1[1] * n^-1, with their Shoup companions): tw[0] and tw[1] of the
// row's table, unless the store target scales its row by a constant c, in
// which case `fold(row)` points to the same two constants times c (the
// product comes out scaled at no extra multiply).
template <class T, class = void>
struct has_fold : std::false_type {};
template <class T>
struct has_fold<T, std::void_t<decltype(std::declval<const T&>().fold(0))>> : std::true_type {};

template <class Dst>
__device__ __forceinline__ const tw_t* fold_tab(const Dst& d, int row, const tw_t* tw) {
    if constexpr (has_fold<Dst>::value) return d.fold(row);
    else return tw;
}

// A source that can name its rows' input ranges (`prefetch(row, off, n)`)
// lets a block kernel ask L2 for the block that starts one wave of CTAs after
// its own: the copy runs while this CTA computes, and the later CTA's first
// pass reads L2 instead of waiting on HBM (one CTA per SM at N = 2^14, so
// its load phase is otherwise not overlapped with any computation).
template <class T, class = void>
struct has_prefetch : std::false_type {};
template <class T>
struct has_prefetch<T, std::void_t<decltype(std::declval<const T&>().prefetch(0, 0, 0))>> : std::true_type {};

// asynchronous copy of `bytes` (a multiple of 16, 16-byte aligned) into L2
__device__ __forceinline__ void l2_prefetch(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// the block `ahead` CTAs after this one (ahead = CTAs resident at once; 0: none)
template <int LOGB, class Src>
__device__ __forceinline__ void prefetch_next(const Src& src, int ahead, int nblk) {
    if constexpr (has_prefetch<Src>::value) {
        if (ahead > 0 && threadIdx.x == 0) {
            const unsigned nxt = blockIdx.x + (unsigned)ahead;
            if (nxt < gridDim.x) src.prefetch((int)(nxt / nblk), (int)(nxt % nblk) << LOGB, 1 << LOGB);
        }
    }
}

__device__ __forceinline__ int spad(int j) { return j + (j >> 4); }

// Shoup product with a quotient estimate from three 32-bit partial products
// of b * ws (b1*w1, hi(b1*w0), hi(b0*w1)): the dropped terms make the
// estimate low by at most 3, so the result is b*w mod q plus at most 3q,
// i.e. in [0, 4q). Any 64-bit b is allowed.
__device__ __forceinline__ uint64_t shoup4_64(uint64_t b, uint64_t w, uint64_t ws, uint64_t q) {
    const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    const uint32_t w0 = (uint32_t)ws, w1 = (uint32_t)(ws >> 32);
    const uint64_t est = (uint64_t)b1 * w1 + (uint64_t)__umulhi(b1, w0) + (uint64_t)__umulhi(b0, w1);
    return b * w - est * q;
}

// shoup4 written with 32-bit multiplies only (mul/mad .lo/.hi .u32 with carry
// chains): the same value as shoup4 for every input. The low 64 bits of b*w
// and est*q each take one high and three low 32-bit products instead of a
// 32x32->64 wide product and two low ones.
__device__ __forceinline__ uint64_t shoup4_32(uint64_t b, uint64_t w, uint64_t ws, uint64_t q) {
    const uint32_t b0 = (uint32_t)b, b1 = (uint32_t)(b >> 32);
    const uint32_t w0 = (uint32_t)w, w1 = (uint32_t)(w >> 32);
    const uint32_t s0 = (uint32_t)ws, s1 = (uint32_t)(ws >> 32);
    const uint32_t q0 = (uint32_t)q, q1 = (uint32_t)(q >> 32);
    uint32_t e0, e1, r0, r1, f0, f1;
    asm("mul.lo.u32      %0, %7, %11;\n\t"     // est = b1*s1
        "mul.hi.u32      %1, %7, %11;\n\t"
        "mad.hi.cc.u32   %0, %7, %10, %0;\n\t" // + hi(b1*s0)
        "addc.u32        %1, %1, 0;\n\t"
        "mad.hi.cc.u32   %0, %6, %11, %0;\n\t" // + hi(b0*s1)
        "addc.u32        %1, %1, 0;\n\t"
        "mul.lo.u32      %2, %6, %8;\n\t"      // lo64(b*w)
        "mul.hi.u32      %3, %6, %8;\n\t"
        "mad.lo.u32      %3, %6, %9, %3;\n\t"
        "mad.lo.u32      %3, %7, %8, %3;\n\t"
        "mul.lo.u32      %4, %0, %12;\n\t"     // lo64(est*q)
        "mul.hi.u32      %5, %0, %12;\n\t"
        "mad.lo.u32      %5, %0, %13, %5;\n\t"
        "mad.lo.u32      %5, %1, %12, %5;\n\t"
        "sub.cc.u32      %2, %2, %4;\n\t"
        "subc.u32        %3, %3, %5;"
        : "=&r"(e0), "=&r"(e1), "=&r"(r0), "=&r"(r1), "=&r"(f0), "=&r"(f1)
        : "r"(b0), "r"(b1), "r"(w0), "r"(w1), "r"(s0), "r"(s1), "r"(q0), "r"(q1));
    return ((uint64_t)r1 << 32) | r0;
}

// the Shoup product of the butterflies: the 32-bit form (8% more butterflies
// per cycle than shoup4_64 in register chains on the B200)
__device__ __forceinline__ uint64_t shoup4(uint64_t b, uint64_t w, uint64_t ws, uint64_t q) {
    return shoup4_32(b, w, ws, q);
}

// a - c if that is non-negative, else a; a, c < 2^63
__device__ __forceinline__ uint64_t csub63(uint64_t a, uint64_t c) {
    const int64_t t = (int64_t)(a - c);
    return t < 0 ? a : (uint64_t)t;
}

// Forward Cooley-Tukey butterfly; values stay in [0, 8q) (q < 2^60 keeps 8q < 2^63).
__device__ __forceinline__ void ct_bfly(uint64_t& a, uint64_t& b, tw_t w, uint64_t q, uint64_t q4) {
    const uint64_t v = shoup4(b, w.x, w.y, q);  // [0, 4q)
    a = csub63(a, q4);                          // [0, 4q)
    b = a + q4 - v;                             // (0, 8q)
    a = a + v;                                  // [0, 8q)
}

// Inverse Gentleman-Sande butterfly; values stay in [0, 4q).
__device__ __forceinline__ void gs_bfly(uint64_t& a, uint64_t& b, tw_t w, uint64_t q, uint64_t q4) {
    const uint64_t t = a + q4 - b;   // (0, 8q)
    a = csub63(a + b, q4);           // [0, 4q)
    b = shoup4(t, w.x, w.y, q);      // [0, 4q)
}

__device__ __forceinline__ uint64_t reduce_from(uint64_t v, uint64_t q, int log_mult) {
    // v < 2^log_mult * q -> [0, q)
    for (int m = log_mult - 1; m >= 0; m--) v = csub63(v, q << m);
    return v;
}

// R forward stages on 2^R registers; stage s0+u uses psi_br[2^(s0+u) + (hi << u) + h].
// Stage and butterfly loops are expanded by template recursion so that every
// register index is a compile-time constant.
template <int R, int U, int H>
__device__ __forceinline__ void fwd_stage_h(uint64_t* x, const tw_t* __restrict__ tw, int bidx, uint64_t q,
                                            uint64_t q4) {
    if constexpr (H < (1 << U)) {
        constexpr int half = 1 << (R - 1 - U);
        const tw_t w = tw[bidx + H];
#pragma unroll
        for (int k = 0; k < half; k++) ct_bfly(x[H * 2 * half + k], x[H * 2 * half + k + half], w, q, q4);
        fwd_stage_h<R, U, H + 1>(x, tw, bidx, q, q4);
    }
}
template <int R, int U>
__device__ __forceinline__ void fwd_stages(uint64_t* x, const tw_t* __restrict__ tw, int s0, int hi, uint64_t q,
                                           uint64_t q4) {
    if constexpr (U < R) {
        fwd_stage_h<R, U, 0>(x, tw, (1 << (s0 + U)) + (hi << U), q, q4);
        fwd_stages<R, U + 1>(x, tw, s0, hi, q, q4);
    }
}
template <int R>
__device__ __forceinline__ void fwd_group(uint64_t* x, const tw_t* __restrict__ tw, int s0, int hi,
                                          uint64_t q, uint64_t q4) {
    fwd_stages<R, 0>(x, tw, s0, hi, q, q4);
}

// R inverse stages (reverse order). `fold` (only with s0 == 0, hi == 0) applies
// n^-1 at global stage 0 using ftw[0] = n^-1, ftw[1] = psi_br^-1[1] * n^-1
// (ftw = tw, or a scaled pair: fold_tab) and fully reduces.
template <int R, int U, int H>
__device__ __forceinline__ void inv_stage_h(uint64_t* x, const tw_t* __restrict__ tw, int bidx, uint64_t q,
                                            uint64_t q4) {
    if constexpr (H < (1 << U)) {
        constexpr int half = 1 << (R - 1 - U);
        const tw_t w = tw[bidx + H];
#pragma unroll
        for (int k = 0; k < half; k++) gs_bfly(x[H * 2 * half + k], x[H * 2 * half + k + half], w, q, q4);
        inv_stage_h<R, U, H + 1>(x, tw, bidx, q, q4);
    }
}
template <int R, int U>
__device__ __forceinline__ void inv_stages(uint64_t* x, const tw_t* __restrict__ tw, int s0, int hi, uint64_t q,
                                           uint64_t q4, bool fold, const tw_t* __restrict__ ftw) {
    if constexpr (U >= 0) {
        constexpr int half = 1 << (R - 1 - U);
        if (U == 0 && fold) {
            const tw_t ni = ftw[0];
            const tw_t w1 = ftw[1];
#pragma unroll
            for (int k = 0; k < half; k++) {
                const uint64_t a = x[k], b = x[k + half];
                x[k] = reduce_from(shoup4(a + b, ni.x, ni.y, q), q, 2);
                x[k + half] = reduce_from(shoup4(a + q4 - b, w1.x, w1.y, q), q, 2);
            }
        } else {
            inv_stage_h<R, U, 0>(x, tw, (1 << (s0 + U)) + (hi << U), q, q4);
        }
        inv_stages<R, U - 1>(x, tw, s0, hi, q, q4, fold, ftw);
    }
}
template <int R>
__device__ __forceinline__ void inv_group(uint64_t* x, const tw_t* __restrict__ tw, int s0, int hi,
                                          uint64_t q, uint64_t q4, bool fold, const tw_t* __restrict__ ftw = nullptr) {
    inv_stages<R, R - 1>(x, tw, s0, hi, q, q4, fold, ftw ? ftw : tw);
}

// ---------------------------------------------------------------------------
// Block kernels. The CTA handles block `blk` of row `row`; the block holds
// global indices [blk << LOGB, (blk + 1) << LOGB) of a length-2^logn transform
// and runs global stages [logn - LOGB, logn). With logn == LOGB this is the
// whole transform. T = 2^LOGB / 16 threads, each owning 16 points; a pass of
// R <= RAD stages processes 16 / 2^R register groups per thread. Group gi of a
// pass starting at local stage S0 holds the points
//   ((gi >> lb) << (lb + R)) | (gi & (2^lb - 1)) + k * 2^lb,  lb = LOGB - S0 - R,
// and thread t takes gi = g * T + t; with one pad word per 16 points every
// shared-memory access of every pass is free of bank conflicts.
// ---------------------------------------------------------------------------
template <int LOGB>
struct BlockShape {
    static constexpr int NB = 1 << LOGB;
    static constexpr int THREADS = NB / 16;
    static constexpr int SMEM_BYTES = (NB + NB / 16) * 8;
    // radix of the register groups: 16 points (the template-expanded groups keep
    // a 1024-thread block within 64 registers)
    static constexpr int RAD = 4;
};

// Teams. After the forward transform's first radix-16 pass (before the
// inverse's last) the block splits into independent sub-blocks of 2^(LOGB-4)
// points, each held by 2^(LOGB-8) consecutive threads in every later pass. A
// team of 128 threads owns 2048 contiguous points and synchronises those
// passes with a named barrier of its own (ids 1..COUNT), so teams drift apart
// and one team's shared-memory exchange overlaps the others' arithmetic. Blocks
// of at most 2048 points are one team (the CTA barrier).
template <int LOGB>
struct Teams {
    static constexpr int T = (1 << LOGB) / 16;
    static constexpr int SIZE = T < 128 ? T : 128;
    static constexpr int COUNT = T / SIZE;
    static constexpr int TB = LOGB - 8;  // log2 of the threads of one sub-block
};

template <int LOGB>
__device__ __forceinline__ void team_sync() {
    if constexpr (Teams<LOGB>::COUNT == 1) {
        __syncthreads();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(1 + (int)threadIdx.x / Teams<LOGB>::SIZE), "n"(Teams<LOGB>::SIZE)
                     : "memory");
    }
}

// group index of register group g of thread t in a pass of R stages whose
// groups are 2^R adjacent points (lb = 0, NG = 16 / 2^R groups per thread):
// with teams, a thread's groups stay inside its own sub-block
template <int LOGB, int R>
__device__ __forceinline__ int adjacent_group(int g, int t) {
    if constexpr (Teams<LOGB>::COUNT == 1) {
        return g * Teams<LOGB>::T + t;
    } else {
        constexpr int TB = Teams<LOGB>::TB;
        return ((t >> TB) << (LOGB - 4 - R)) | (g << TB) | (t & ((1 << TB) - 1));
    }
}

// point k of thread t in a coalesced sweep of the block (k < 16): with teams,
// the sweep covers the thread's own team's 2048 points
template <int LOGB>
__device__ __forceinline__ int sweep_index(int t, int k) {
    constexpr int S = Teams<LOGB>::SIZE;
    if constexpr (Teams<LOGB>::COUNT == 1) return t + k * Teams<LOGB>::T;
    else return (t / S) * (S * 16) + (t % S) + k * S;
}

// Resident CTAs per SM a block kernel is compiled for (0: left to ptxas). The
// 2^13-point blocks (512 threads, 68 KiB of shared memory) get two, i.e. 64
// registers a thread: left to itself ptxas gives them 88 and one CTA per SM
// (N = 8192 multiply, 64 pairs: 0.825 -> 0.760 ms). Capping the 2^12-point
// blocks at 64 registers as well (four CTAs) measured mixed (-1% for the
// N = 32768 multiply, +3.5% for a two-pair multiply at N = 16384), so they,
// and the 1024-thread 2^14 blocks (64 registers either way), keep ptxas's choice.
template <int LOGB>
constexpr int block_min_ctas() {
    return LOGB == 13 ? 2 : 0;
}

struct PassCtx {
    uint64_t* sm;
    const tw_t* tw;
    int t, sbase, goff, logn;
    uint64_t q, q4;
};

// padded index of lbase + (k << lb); for lb >= 4 the offset is a constant
template <int LB>
__device__ __forceinline__ int spad_off(int pbase, int lbase, int k) {
    if constexpr (LB >= 4) return pbase + k * ((1 << LB) + (1 << (LB - 4)));
    else return spad(lbase + (k << LB));
}

template <int LOGB, int S0, int R>
__device__ __forceinline__ int group_base(int gi) {
    constexpr int lb = LOGB - S0 - R;
    return ((gi >> lb) << (lb + R)) | (gi & ((1 << lb) - 1));
}

// one forward pass over shared memory (a pass after the first: team-local)
template <int LOGB, int S0, int R>
__device__ __forceinline__ void fwd_pass_smem(const PassCtx& c) {
    constexpr int T = (1 << LOGB) / 16, G = 1 << R, NG = 16 / G, lb = LOGB - S0 - R;
    static_assert(NG == 1 || lb == 0, "only the last pass holds several groups per thread");
#pragma unroll
    for (int g = 0; g < NG; g++) {
        const int lbase = group_base<LOGB, S0, R>(NG == 1 ? c.t : adjacent_group<LOGB, R>(g, c.t));
        const int pbase = spad(lbase);
        uint64_t x[G];
#pragma unroll
        for (int k = 0; k < G; k++) x[k] = c.sm[spad_off<lb>(pbase, lbase, k)];
        const int s0 = c.sbase + S0;
        fwd_group<R>(x, c.tw, s0, (c.goff + lbase) >> (c.logn - s0), c.q, c.q4);
#pragma unroll
        for (int k = 0; k < G; k++) c.sm[spad_off<lb>(pbase, lbase, k)] = x[k];
    }
    team_sync<LOGB>();
}

template <int LOGB, int RAD, int S0>
__device__ __forceinline__ void fwd_passes(const PassCtx& c) {
    if constexpr (S0 < LOGB) {
        constexpr int R = (LOGB - S0) < RAD ? (LOGB - S0) : RAD;
        fwd_pass_smem<LOGB, S0, R>(c);
        fwd_passes<LOGB, RAD, S0 + R>(c);
    }
}

// one inverse pass over shared memory; FULL: the last one before the first
// pass (which spans the whole block) ends with the CTA barrier, the others
// with their team's
template <int LOGB, int S0, int R, bool FULL>
__device__ __forceinline__ void inv_pass_smem(const PassCtx& c) {
    constexpr int T = (1 << LOGB) / 16, G = 1 << R, NG = 16 / G, lb = LOGB - S0 - R;
    static_assert(NG == 1 || lb == 0, "only the last pass holds several groups per thread");
    // groups one after another: keeps the 1024-thread variant within 64 registers
#pragma unroll 1
    for (int g = 0; g < NG; g++) {
        const int lbase = group_base<LOGB, S0, R>(NG == 1 ? c.t : adjacent_group<LOGB, R>(g, c.t));
        const int pbase = spad(lbase);
        uint64_t x[G];
#pragma unroll
        for (int k = 0; k < G; k++) x[k] = c.sm[spad_off<lb>(pbase, lbase, k)];
        const int s0 = c.sbase + S0;
        inv_group<R>(x, c.tw, s0, (c.goff + lbase) >> (c.logn - s0), c.q, c.q4, false);
#pragma unroll
        for (int k = 0; k < G; k++) c.sm[spad_off<lb>(pbase, lbase, k)] = x[k];
    }
    if constexpr (FULL) __syncthreads();
    else team_sync<LOGB>();
}

// inverse passes with S0 >= first, run from the last stages back to `first`
// (the pass at `first` = R0 precedes the whole-block first pass)
template <int LOGB, int RAD, int S0>
__device__ __forceinline__ void inv_passes(const PassCtx& c) {
    if constexpr (S0 < LOGB) {
        constexpr int R = (LOGB - S0) < RAD ? (LOGB - S0) : RAD;
        constexpr int R0 = RAD < LOGB ? RAD : LOGB;
        inv_passes<LOGB, RAD, S0 + R>(c);
        inv_pass_smem<LOGB, S0, R, S0 == R0>(c);
    }
}

// The first inverse pass (the block's last local stages, lb = 0: groups of
// 2^R adjacent points) loads its inputs straight from the row: no staging of
// the row in shared memory and one barrier less (4.7% faster inverse NTT at
// N=2^14 than a coalesced load-in; the loads of adjacent points hit the same
// cache lines).
template <int LOGB, int S0, int R, class SRow, bool FULL>
__device__ __forceinline__ void inv_pass_load(const PassCtx& c, const SRow& s) {
    constexpr int G = 1 << R, NG = 16 / G;
    static_assert(LOGB - S0 - R == 0, "the loading pass holds the last stages");
#pragma unroll 1
    for (int g = 0; g < NG; g++) {
        const int lbase = adjacent_group<LOGB, R>(g, c.t) << R;
        uint64_t x[G];
#pragma unroll
        for (int k = 0; k < G; k++) x[k] = s.load(c.goff + lbase + k);
        const int s0 = c.sbase + S0;
        inv_group<R>(x, c.tw, s0, (c.goff + lbase) >> (c.logn - s0), c.q, c.q4, false);
#pragma unroll
        for (int k = 0; k < G; k++) c.sm[spad(lbase + k)] = x[k];
    }
    if constexpr (FULL) __syncthreads();
    else team_sync<LOGB>();
}
template <int LOGB, int RAD, int S0, class SRow>
__device__ __forceinline__ void inv_passes_load(const PassCtx& c, const SRow& s) {
    constexpr int R = (LOGB - S0) < RAD ? (LOGB - S0) : RAD;
    constexpr int R0 = RAD < LOGB ? RAD : LOGB;
    if constexpr (S0 + R < LOGB) {
        inv_passes_load<LOGB, RAD, S0 + R>(c, s);
        inv_pass_smem<LOGB, S0, R, S0 == R0>(c);
    } else {
        inv_pass_load<LOGB, S0, R, SRow, S0 == R0>(c, s);
    }
}

// Direct loads for groups of up to 4 adjacent points (32-byte lane stride);
// wider groups (the 2^12-point blocks' last pass holds 16) load coalesced into
// shared memory first.
template <int LOGB, int RAD>
__device__ __forceinline__ constexpr bool inv_direct_load() {
    constexpr int rest = (LOGB - (RAD < LOGB ? RAD : LOGB)) % RAD;
    return (rest == 0 ? RAD : rest) <= 2;
}

// FULL: fully reduce the output to [0, q); otherwise outputs are in [0, 8q).
template <int LOGB, class Src, class Dst, bool FULL = true>
static __global__ void __launch_bounds__(1 << (LOGB - 4), block_min_ctas<LOGB>())
ntt_fwd_block_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all, const uint64_t* __restrict__ mods,
                     int logn, int ahead) {
    constexpr int NB = 1 << LOGB, T = NB / 16, RAD = BlockShape<LOGB>::RAD;
    constexpr int R0 = RAD < LOGB ? RAD : LOGB, G0 = 1 << R0, lb0 = LOGB - R0;
    extern __shared__ uint64_t sm[];
    const int nblk = 1 << (logn - LOGB);
    const int row = blockIdx.x / nblk;
    const int blk = blockIdx.x % nblk;
    const int t = threadIdx.x;
    const RowTab rt = row_tab(src, row, false, tw_all, mods, logn);
    const auto s = src.bind(row);
    const uint64_t q = rt.q, q4 = q << 2;
    PassCtx c{sm, rt.tw, t, logn - LOGB, blk << LOGB, logn, q, q4};
    prefetch_next<LOGB>(src, ahead, nblk);

    // pass 0 straight from global memory: groups gi + k * 2^lb0 (consecutive lanes, coalesced);
    // groups one after another so fused loaders keep their temporaries in registers
#pragma unroll 1
    for (int g = 0; g < 16 / G0; g++) {
        const int gi = g * T + t;
        uint64_t x[G0];
#pragma unroll
        for (int k = 0; k < G0; k++) x[k] = s.load(c.goff + gi + (k << lb0));
        fwd_group<R0>(x, c.tw, c.sbase, c.goff >> LOGB, q, q4);
        const int pg = spad(gi);
#pragma unroll
        for (int k = 0; k < G0; k++) sm[spad_off<lb0>(pg, gi, k)] = x[k];
    }
    __syncthreads();
    fwd_passes<LOGB, RAD, R0>(c);
    // coalesced write-out (a last pass storing its groups of adjacent points
    // straight to the row measured 14% slower here); the store target is bound
    // here, so a fused store's operands hold no registers during the transform
    const auto d = dst.bind(row);
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int j = sweep_index<LOGB>(t, k);
        const uint64_t v = sm[spad(j)];
        d.store(c.goff + j, FULL ? reduce_from(v, q, 3) : v);
    }
}

// WHOLE: the block is the whole ring (logn == LOGB), so n^-1 is applied here.
template <int LOGB, class Src, class Dst, bool WHOLE = true>
static __global__ void __launch_bounds__(1 << (LOGB - 4), block_min_ctas<LOGB>())
ntt_inv_block_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all, const uint64_t* __restrict__ mods,
                     int logn, int ahead) {
    constexpr int NB = 1 << LOGB, T = NB / 16, RAD = BlockShape<LOGB>::RAD;
    constexpr int R0 = RAD < LOGB ? RAD : LOGB, G0 = 1 << R0, lb0 = LOGB - R0;
    extern __shared__ uint64_t sm[];
    const int nblk = 1 << (logn - LOGB);
    const int row = blockIdx.x / nblk;
    const int blk = blockIdx.x % nblk;
    const int t = threadIdx.x;
    const RowTab rt = row_tab(src, row, true, tw_all, mods, logn);
    const auto s = src.bind(row);
    const uint64_t q = rt.q, q4 = q << 2;
    PassCtx c{sm, rt.tw, t, logn - LOGB, blk << LOGB, logn, q, q4};
    prefetch_next<LOGB>(src, ahead, nblk);

    if constexpr (inv_direct_load<LOGB, RAD>()) {
        inv_passes_load<LOGB, RAD, R0>(c, s);
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            const int j = sweep_index<LOGB>(t, k);
            sm[spad(j)] = s.load(c.goff + j);
        }
        team_sync<LOGB>();
        inv_passes<LOGB, RAD, R0>(c);
    }
    // pass 0 (local stages 0..R0-1), coalesced stores
    const auto d = dst.bind(row);
    const tw_t* ftw = fold_tab(dst, row, c.tw);
#pragma unroll 1
    for (int g = 0; g < 16 / G0; g++) {
        const int gi = g * T + t;
        uint64_t x[G0];
        const int pg = spad(gi);
#pragma unroll
        for (int k = 0; k < G0; k++) x[k] = sm[spad_off<lb0>(pg, gi, k)];
        inv_group<R0>(x, c.tw, c.sbase, c.goff >> LOGB, q, q4, WHOLE, ftw);
#pragma unroll
        for (int k = 0; k < G0; k++) d.store(c.goff + gi + (k << lb0), x[k]);
    }
}

// ---------------------------------------------------------------------------
// Column pass for rings larger than one block: the first (forward) or last
// (inverse) RC = logn - LOGB stages, elementwise over 2^RC-point columns.
// Forward outputs are in [0, 8q); inverse inputs may be in [0, 4q).
// ---------------------------------------------------------------------------
template <int RC, class Src, class Dst>
__device__ __forceinline__ void ntt_fwd_col(const Src& src, const Dst& dst, const tw_t* __restrict__ tw_all,
                                            const uint64_t* __restrict__ mods, int logn, size_t gid) {
    const int cols = 1 << (logn - RC);
    const int row = (int)(gid >> (logn - RC)), c = (int)(gid & (cols - 1));
    const RowTab rt = row_tab(src, row, false, tw_all, mods, logn);
    const auto s = src.bind(row);
    const auto d = dst.bind(row);
    const uint64_t q = rt.q, q4 = q << 2;
    const tw_t* tw = rt.tw;
    uint64_t x[1 << RC];
#pragma unroll
    for (int k = 0; k < (1 << RC); k++) x[k] = s.load(c + k * cols);
    fwd_group<RC>(x, tw, 0, 0, q, q4);
#pragma unroll
    for (int k = 0; k < (1 << RC); k++) d.store(c + k * cols, x[k]);
}

template <int RC, class Src, class Dst>
__device__ __forceinline__ void ntt_inv_col(const Src& src, const Dst& dst, const tw_t* __restrict__ tw_all,
                                            const uint64_t* __restrict__ mods, int logn, size_t gid) {
    const int cols = 1 << (logn - RC);
    const int row = (int)(gid >> (logn - RC)), c = (int)(gid & (cols - 1));
    const RowTab rt = row_tab(src, row, true, tw_all, mods, logn);
    const auto s = src.bind(row);
    const auto d = dst.bind(row);
    const uint64_t q = rt.q, q4 = q << 2;
    const tw_t* tw = rt.tw;
    uint64_t x[1 << RC];
#pragma unroll
    for (int k = 0; k < (1 << RC); k++) x[k] = s.load(c + k * cols);
    inv_group<RC>(x, tw, 0, 0, q, q4, true, fold_tab(dst, row, tw));
#pragma unroll
    for (int k = 0; k < (1 << RC); k++) d.store(c + k * cols, x[k]);
}

// grid-stride over all columns of all rows (more than 2^31 columns allowed)
template <int RC, class Src, class Dst>
static __global__ void ntt_fwd_col_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all,
                                   const uint64_t* __restrict__ mods, int logn, size_t ncol_total) {
    for (size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gid < ncol_total;
         gid += (size_t)gridDim.x * blockDim.x)
        ntt_fwd_col<RC>(src, dst, tw_all, mods, logn, gid);
}

template <int RC, class Src, class Dst>
static __global__ void ntt_inv_col_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all,
                                   const uint64_t* __restrict__ mods, int logn, size_t ncol_total) {
    for (size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gid < ncol_total;
         gid += (size_t)gridDim.x * blockDim.x)
        ntt_inv_col<RC>(src, dst, tw_all, mods, logn, gid);
}

// The radix-16 column pass (N = 2^16 ahead of / behind 2^12-point blocks)
// holds 16 points a thread: compiled for three 256-thread CTAs per SM (80
// registers) instead of ptxas's own 104 registers and two CTAs (forward
// 0.881 -> 0.838 ms, inverse 0.894 -> 0.846 ms per 1024 rows at N = 65536).
// Launched with 256 threads.
template <int RC, class Src, class Dst>
static __global__ void __launch_bounds__(256, 3)
ntt_fwd_col16_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all, const uint64_t* __restrict__ mods, int logn,
                     size_t ncol_total) {
    for (size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gid < ncol_total;
         gid += (size_t)gridDim.x * blockDim.x)
        ntt_fwd_col<RC>(src, dst, tw_all, mods, logn, gid);
}

template <int RC, class Src, class Dst>
static __global__ void __launch_bounds__(256, 3)
ntt_inv_col16_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all, const uint64_t* __restrict__ mods, int logn,
                     size_t ncol_total) {
    for (size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x; gid < ncol_total;
         gid += (size_t)gridDim.x * blockDim.x)
        ntt_inv_col<RC>(src, dst, tw_all, mods, logn, gid);
}

// ---------------------------------------------------------------------------
// Row functors: prime(row), bind(row) -> {load(j), store(j, v)}
// ---------------------------------------------------------------------------
struct PtrRow {
    uint64_t* p;
    __device__ __forceinline__ void prefetch(int off, int n) const { l2_prefetch(p + off, (uint32_t)n * 8); }
    __device__ __forceinline__ uint64_t load(int j) const { return p[j]; }
    __device__ __forceinline__ void store(int j, uint64_t v) const { p[j] = v; }
};

// Contiguous rows: row r at base + r*N, prime index p0 + (r % period).
struct RowsIO {
    uint64_t* base;
    int logn;
    int p0;
    int period;
    __device__ __forceinline__ int prime(int row) const { return p0 + row % period; }
    __device__ __forceinline__ PtrRow bind(int row) const { return PtrRow{base + ((size_t)row << logn)}; }
    __device__ __forceinline__ void prefetch(int row, int off, int n) const { bind(row).prefetch(off, n); }
};

}  // namespace kbfv
