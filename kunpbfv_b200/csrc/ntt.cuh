// Batched negacyclic NTT / inverse NTT over 60-bit primes for sm_100a.
//
// Convention (the reference's, include/ntt_60bit.cuh and include/Utils.cuh:171-191):
// forward Cooley-Tukey with psi_br[i] = psi^brv(i); output index k holds
// A(psi^(2*brv(k)+1)), fully reduced. Inverse Gentleman-Sande with
// psi^-brv(i), n^-1 folded into the last stage; output fully reduced.
//
// Shape: one CTA transforms one block of 2^LOGB points held in shared memory
// (N = 2^14 -> 1024 threads x 16 points, 136 KiB of padded smem). Each thread
// runs radix-16 groups (4 butterfly stages in registers) between shared-memory
// exchanges. Larger rings (N = 2^15, 2^16) add one elementwise radix-2/4 column
// pass in front of (forward) or behind (inverse) the block kernels.
//
// Rows are described by Src/Dst functors: src.prime(row), s.load(j),
// d.store(j, v). This lets pipeline stages fuse their per-element
// prologue (e.g. a tensor product) and epilogue (e.g. a key product) into the
// transform's first load and last store, which are always coalesced
// (consecutive threads touch consecutive j).
#pragma once
#include "arith.cuh"

namespace kbfv {

typedef ulonglong2 tw_t;  // (w, floor(w * 2^64 / q))

__device__ __forceinline__ int spad(int j) { return j + (j >> 4); }

__device__ __forceinline__ void ct_bfly(uint64_t& a, uint64_t& b, tw_t w, uint64_t q, uint64_t q2) {
    uint64_t v = shoup_lazy(b, w.x, w.y, q);
    a = a >= q2 ? a - q2 : a;
    b = a + q2 - v;
    a = a + v;
}

__device__ __forceinline__ void gs_bfly(uint64_t& a, uint64_t& b, tw_t w, uint64_t q, uint64_t q2) {
    uint64_t t = a + q2 - b;
    uint64_t s = a + b;
    a = s >= q2 ? s - q2 : s;
    b = shoup_lazy(t, w.x, w.y, q);
}

// R forward stages on 2^R registers; stage s0+u uses psi_br[2^(s0+u) + (hi << u) + h].
template <int R>
__device__ __forceinline__ void fwd_group(uint64_t* x, const tw_t* __restrict__ tw, int s0, int hi,
                                          uint64_t q, uint64_t q2) {
#pragma unroll
    for (int u = 0; u < R; u++) {
        const int half = 1 << (R - 1 - u);
        const int bidx = (1 << (s0 + u)) + (hi << u);
#pragma unroll
        for (int h = 0; h < (1 << u); h++) {
            const tw_t w = tw[bidx + h];
#pragma unroll
            for (int k = 0; k < half; k++) {
                const int i0 = h * 2 * half + k;
                ct_bfly(x[i0], x[i0 + half], w, q, q2);
            }
        }
    }
}

// R inverse stages (reverse order); `fold` applies n^-1 at global stage 0
// using tw[0] = n^-1 and tw[1] = psi^-1 * n^-1, and fully reduces.
template <int R>
__device__ __forceinline__ void inv_group(uint64_t* x, const tw_t* __restrict__ tw, int s0, int hi,
                                          uint64_t q, uint64_t q2, bool fold) {
#pragma unroll
    for (int u = R - 1; u >= 0; u--) {
        const int half = 1 << (R - 1 - u);
        const int bidx = (1 << (s0 + u)) + (hi << u);
        if (fold && u == 0) {
            // s0 == 0 and hi == 0 here: a single butterfly column with psi^-1 at index 1
            const tw_t ni = tw[0];
            const tw_t w1 = tw[1];
#pragma unroll
            for (int k = 0; k < half; k++) {
                uint64_t a = x[k], b = x[k + half];
                uint64_t s = a + b;
                uint64_t t = a + q2 - b;
                x[k] = csub(shoup_lazy(s, ni.x, ni.y, q), q);
                x[k + half] = csub(shoup_lazy(t, w1.x, w1.y, q), q);
            }
        } else {
#pragma unroll
            for (int h = 0; h < (1 << u); h++) {
                const tw_t w = tw[bidx + h];
#pragma unroll
                for (int k = 0; k < half; k++) {
                    const int i0 = h * 2 * half + k;
                    gs_bfly(x[i0], x[i0 + half], w, q, q2);
                }
            }
        }
    }
}

__device__ __forceinline__ uint64_t reduce4q(uint64_t v, uint64_t q, uint64_t q2) {
    v = v >= q2 ? v - q2 : v;
    return v >= q ? v - q : v;
}

// ---------------------------------------------------------------------------
// Block kernels. The CTA handles block `blk` of row `row`; the block holds
// global indices [blk << LOGB, (blk + 1) << LOGB) of a length-2^logn transform
// and runs global stages [logn - LOGB, logn). With logn == LOGB this is the
// whole transform.
// ---------------------------------------------------------------------------
template <int LOGB>
struct BlockShape {
    static constexpr int NB = 1 << LOGB;
    static constexpr int THREADS = NB / 16;
    static constexpr int SMEM_BYTES = (NB + NB / 16) * 8;
};

template <int LOGB, class Src, class Dst>
__global__ void __launch_bounds__(1 << (LOGB - 4))
ntt_fwd_block_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all, const uint64_t* __restrict__ mods,
                     int logn) {
    constexpr int NB = 1 << LOGB, T = NB / 16;
    extern __shared__ uint64_t sm[];
    const int nblk = 1 << (logn - LOGB);
    const int row = blockIdx.x / nblk;
    const int blk = blockIdx.x % nblk;
    const int t = threadIdx.x;
    const int pidx = src.prime(row);
    const auto s = src.bind(row);
    const auto d = dst.bind(row);
    const uint64_t q = mods[pidx], q2 = q << 1;
    const tw_t* tw = tw_all + ((size_t)pidx << logn);
    const int sbase = logn - LOGB;   // first global stage handled here
    const int goff = blk << LOGB;    // global index of local 0
    uint64_t x[16];

    // pass 0: local stride NB/16, elements t + k*T (coalesced loads)
#pragma unroll
    for (int k = 0; k < 16; k++) x[k] = s.load(goff + t + k * T);
    fwd_group<4>(x, tw, sbase, goff >> (logn - sbase), q, q2);
#pragma unroll
    for (int k = 0; k < 16; k++) sm[spad(t + k * T)] = x[k];
    __syncthreads();

    // middle passes (full radix-16)
#pragma unroll
    for (int ls0 = 4; ls0 + 4 <= LOGB; ls0 += 4) {
        const int lowbits = LOGB - ls0 - 4;
        const int stride = 1 << lowbits;
        const int lbase = ((t >> lowbits) << (lowbits + 4)) | (t & (stride - 1));
        const int s0 = sbase + ls0;
#pragma unroll
        for (int k = 0; k < 16; k++) x[k] = sm[spad(lbase + k * stride)];
        fwd_group<4>(x, tw, s0, (goff + lbase) >> (logn - s0), q, q2);
#pragma unroll
        for (int k = 0; k < 16; k++) sm[spad(lbase + k * stride)] = x[k];
        __syncthreads();
    }

    // tail pass: remaining R = LOGB % 4 stages on consecutive groups
    constexpr int R = LOGB % 4;
    if (R > 0) {
        constexpr int RR = R > 0 ? R : 1;
        constexpr int G = 16 >> RR;
        const int s0 = sbase + LOGB - RR;
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int gidx = g * T + t;  // group index within block
            uint64_t y[1 << RR];
#pragma unroll
            for (int k = 0; k < (1 << RR); k++) y[k] = sm[spad((gidx << RR) + k)];
            fwd_group<RR>(y, tw, s0, (goff >> RR) + gidx, q, q2);
#pragma unroll
            for (int k = 0; k < (1 << RR); k++) sm[spad((gidx << RR) + k)] = y[k];
        }
        __syncthreads();
    }

    // coalesced write-out with full reduction
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int j = t + k * T;
        d.store(goff + j, reduce4q(sm[spad(j)], q, q2));
    }
}

template <int LOGB, class Src, class Dst>
__global__ void __launch_bounds__(1 << (LOGB - 4))
ntt_inv_block_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all, const uint64_t* __restrict__ mods,
                     int logn) {
    constexpr int NB = 1 << LOGB, T = NB / 16;
    extern __shared__ uint64_t sm[];
    const int nblk = 1 << (logn - LOGB);
    const int row = blockIdx.x / nblk;
    const int blk = blockIdx.x % nblk;
    const int t = threadIdx.x;
    const int pidx = src.prime(row);
    const auto s = src.bind(row);
    const auto d = dst.bind(row);
    const uint64_t q = mods[pidx], q2 = q << 1;
    const tw_t* tw = tw_all + ((size_t)pidx << logn);
    const int sbase = logn - LOGB;
    const int goff = blk << LOGB;
    const bool whole = (sbase == 0);
    uint64_t x[16];

#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int j = t + k * T;
        sm[spad(j)] = s.load(goff + j);
    }
    __syncthreads();

    constexpr int R = LOGB % 4;
    if (R > 0) {
        constexpr int RR = R > 0 ? R : 1;
        constexpr int G = 16 >> RR;
        const int s0 = sbase + LOGB - RR;
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int gidx = g * T + t;
            uint64_t y[1 << RR];
#pragma unroll
            for (int k = 0; k < (1 << RR); k++) y[k] = sm[spad((gidx << RR) + k)];
            inv_group<RR>(y, tw, s0, (goff >> RR) + gidx, q, q2, false);
#pragma unroll
            for (int k = 0; k < (1 << RR); k++) sm[spad((gidx << RR) + k)] = y[k];
        }
        __syncthreads();
    }

    // middle passes, last stages first
#pragma unroll
    for (int ls0 = ((LOGB - R) - 4); ls0 >= 4; ls0 -= 4) {
        const int lowbits = LOGB - ls0 - 4;
        const int stride = 1 << lowbits;
        const int lbase = ((t >> lowbits) << (lowbits + 4)) | (t & (stride - 1));
        const int s0 = sbase + ls0;
#pragma unroll
        for (int k = 0; k < 16; k++) x[k] = sm[spad(lbase + k * stride)];
        inv_group<4>(x, tw, s0, (goff + lbase) >> (logn - s0), q, q2, false);
#pragma unroll
        for (int k = 0; k < 16; k++) sm[spad(lbase + k * stride)] = x[k];
        __syncthreads();
    }

    // pass 0 (local stages 0..3), coalesced stores
#pragma unroll
    for (int k = 0; k < 16; k++) x[k] = sm[spad(t + k * T)];
    inv_group<4>(x, tw, sbase, goff >> (logn - sbase), q, q2, whole);
#pragma unroll
    for (int k = 0; k < 16; k++) d.store(goff + t + k * T, x[k]);
}

// ---------------------------------------------------------------------------
// Column pass for rings larger than one block: the first (forward) or last
// (inverse) RC = logn - LOGB stages, elementwise over 2^RC-point columns.
// ---------------------------------------------------------------------------
template <int RC, class Src, class Dst>
__global__ void ntt_fwd_col_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all,
                                   const uint64_t* __restrict__ mods, int logn, int ncol_total) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= ncol_total) return;
    const int cols = 1 << (logn - RC);
    const int row = gid / cols, c = gid % cols;
    const int pidx = src.prime(row);
    const auto s = src.bind(row);
    const auto d = dst.bind(row);
    const uint64_t q = mods[pidx], q2 = q << 1;
    const tw_t* tw = tw_all + ((size_t)pidx << logn);
    uint64_t x[1 << RC];
#pragma unroll
    for (int k = 0; k < (1 << RC); k++) x[k] = s.load(c + k * cols);
    fwd_group<RC>(x, tw, 0, 0, q, q2);
#pragma unroll
    for (int k = 0; k < (1 << RC); k++) d.store(c + k * cols, x[k]);
}

template <int RC, class Src, class Dst>
__global__ void ntt_inv_col_kernel(Src src, Dst dst, const tw_t* __restrict__ tw_all,
                                   const uint64_t* __restrict__ mods, int logn, int ncol_total) {
    const int gid = blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= ncol_total) return;
    const int cols = 1 << (logn - RC);
    const int row = gid / cols, c = gid % cols;
    const int pidx = src.prime(row);
    const auto s = src.bind(row);
    const auto d = dst.bind(row);
    const uint64_t q = mods[pidx], q2 = q << 1;
    const tw_t* tw = tw_all + ((size_t)pidx << logn);
    uint64_t x[1 << RC];
#pragma unroll
    for (int k = 0; k < (1 << RC); k++) x[k] = s.load(c + k * cols);
    inv_group<RC>(x, tw, 0, 0, q, q2, true);
#pragma unroll
    for (int k = 0; k < (1 << RC); k++) d.store(c + k * cols, x[k]);
}

// ---------------------------------------------------------------------------
// Row functors: prime(row), bind(row) -> {load(j), store(j, v)}
// ---------------------------------------------------------------------------
struct PtrRow {
    uint64_t* p;
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
};

}  // namespace kbfv
