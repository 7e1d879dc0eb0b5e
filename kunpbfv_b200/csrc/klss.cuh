// The reference's key switch over the auxiliary T base (KLSS), for parity with
// kunpBFV at its own parameter sets:
//   lift of Qj blocks into T   modUpQjtoT_23   include/BasisConv.cuh:86-151
//   lift of Ri blocks into T   modUpPQtoT_23   include/BasisConv.cuh:11-79   (key conversion)
//   external product over T    external_product_T  include/ExternalProduct.cuh:11-112
//   exact centred T -> P|Q     modUpTtoPQl_23  include/BasisConv.cuh:159-226
// A block of primes B lifts x mod B into each T prime by approximate CRT with a
// single-precision quotient estimate: rb_j = x_j * (B/b_j)^-1 mod b_j,
// v = (int) sum rb_j / b_j (float division and addition in order),
// out_k = sum rb_j * (B/b_j mod t_k) - v * (B mod t_k) mod t_k.
#pragma once
#include "kernels.cuh"

namespace kbfv {

// reference-order index over P|Q -> row in this library's Q|P order (= prime index)
__host__ __device__ __forceinline__ int ref_to_row(int i, int np, int nq) { return i < np ? nq + i : i - np; }

// Lift blocks into T. which = 0: Qj blocks of a Q polynomial (rows 0..nq-1);
// which = 1: Ri blocks of a Q|P polynomial (rows in Q|P order).
// grid: (N/128, blocks, items); out item layout [block][nt].
static __global__ void klss_block_to_t_kernel(DevConsts c, KlssConsts kc, const uint64_t* __restrict__ in,
                                       uint64_t* __restrict__ out, int which, size_t in_item_stride,
                                       size_t out_item_stride) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    const uint64_t* src = in + blockIdx.z * in_item_stride;
    uint64_t* dst = out + blockIdx.z * out_item_stride + (((size_t)b * kc.nt) << c.logn);
    int width, first;
    const uint64_t *hinv, *hinvs, *hat_t, *mod_t;
    if (which == 0) {
        first = b * c.np;
        width = min(c.np, c.nq - first);
        hinv = kc.qj_hatinv + (size_t)b * c.np;
        hinvs = kc.qj_hatinvs + (size_t)b * c.np;
        hat_t = kc.qj_hat_t + (size_t)b * kc.nt * c.np;
        mod_t = kc.qj_mod_t + (size_t)b * kc.nt;
    } else {
        first = b * kc.gamma;
        width = min(kc.gamma, c.np + c.nq - first);
        hinv = kc.ri_hatinv + (size_t)b * kc.gamma;
        hinvs = kc.ri_hatinvs + (size_t)b * kc.gamma;
        hat_t = kc.ri_hat_t + (size_t)b * kc.nt * kc.gamma;
        mod_t = kc.ri_mod_t + (size_t)b * kc.nt;
    }
    const int stride_hat = which == 0 ? c.np : kc.gamma;
    uint64_t rb[kMaxBlk];
    float vv = 0.f;
#pragma unroll
    for (int j = 0; j < kMaxBlk; j++) {
        if (j < width) {
            const int row = which == 0 ? first + j : ref_to_row(first + j, c.np, c.nq);
            const uint64_t qj = c.mods[row];  // prime index == row in Q|P order
            rb[j] = shoup(src[((size_t)row << c.logn) + k], hinv[j], hinvs[j], qj);
            vv = __fadd_rn(vv, __fdiv_rn(__ull2float_rn(rb[j]), __ull2float_rn(qj)));
        }
    }
    const uint64_t vf = (uint64_t)__float2int_rz(vv);
    for (int t = 0; t < kc.nt; t++) {
        const int pt = c.idx_t + t;
        u128 acc{0, 0};
#pragma unroll
        for (int j = 0; j < kMaxBlk; j++)
            if (j < width) mac(acc, rb[j], hat_t[t * stride_hat + j]);
        sub128(acc, vf * mod_t[t]);
        dst[((size_t)t << c.logn) + k] = barrett128(acc, c.mods[pt], c.mu_hi[pt], c.mu_lo[pt]);
    }
}

// Exact centred T -> P|Q: one polynomial's Ri blocks over T (coefficient form)
// to its P|Q limbs (rows in Q|P order). in: [poly][nri][nt]; out: [poly][npq].
// grid: (N/128, nri, polys)
static __global__ void klss_t_to_pq_kernel(DevConsts c, KlssConsts kc, const uint64_t* __restrict__ in,
                                    uint64_t* __restrict__ out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int b = blockIdx.y;
    const uint64_t* src = in + (((size_t)blockIdx.z * kc.nri + b) * kc.nt << c.logn);
    uint64_t* dst = out + ((size_t)blockIdx.z * c.npq << c.logn);
    uint64_t rb[kMaxT];
    float vv = 0.f;
#pragma unroll
    for (int t = 0; t < kMaxT; t++) {
        if (t < kc.nt) {
            const uint64_t tt = c.mods[c.idx_t + t];
            // (x + T/2) mod t_k without reduction, as the reference adds before its Shoup product
            const uint64_t ra = src[((size_t)t << c.logn) + k] + kc.halft_t[t];
            rb[t] = shoup(ra, kc.thatinv[t], kc.thatinvs[t], tt);
            vv = __fadd_rn(vv, __fdiv_rn(__ull2float_rn(rb[t]), __ull2float_rn(tt)));
        }
    }
    const uint64_t vf = (uint64_t)__float2int_rz(vv);
    const int first = b * kc.gamma;
    const int width = min(kc.gamma, c.np + c.nq - first);
    for (int j = 0; j < width; j++) {
        const int m = first + j;                    // reference order
        const int row = ref_to_row(m, c.np, c.nq);  // prime index / output row
        const uint64_t ri = c.mods[row];
        u128 acc{0, 0};
#pragma unroll
        for (int t = 0; t < kMaxT; t++)
            if (t < kc.nt) mac(acc, rb[t], kc.that_pq[(size_t)m * kc.nt + t]);
        sub128(acc, vf * kc.t_pq[m]);
        uint64_t r = barrett128(acc, ri, c.mu_hi[row], c.mu_lo[row]);
        r = csub(r + ri - kc.halft_pq[m], ri);
        dst[((size_t)row << c.logn) + k] = r;
    }
}

// External product over T (NTT form), fused into the inverse NTT's load:
// row (item, h, b, t): sum over digits i of dig[item][i][t] * key[h][i][b][t] mod t_t.
struct ExtProdRow {
    const uint64_t* dig;   // digit 0, T prime t
    const uint64_t* key;   // half h, digit 0, block b, T prime t
    size_t ds, ks;
    int ndig;
    uint64_t q, mh, ml;
    __device__ __forceinline__ uint64_t load(int j) const {
        u128 acc{0, 0};
        for (int i = 0; i < ndig; i++) mac(acc, dig[i * ds + j], key[i * ks + j]);
        return barrett128(acc, q, mh, ml);
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct ExtProdSrc {
    const uint64_t* dig;   // [item][nqj][nt]
    const uint64_t* key;   // [2][dnum][nri][nt]
    DevConsts dc;
    int nt, nri, nqj, kdnum;
    __device__ __forceinline__ int prime(int row) const { return dc.idx_t + row % nt; }
    __device__ __forceinline__ ExtProdRow bind(int row) const {
        const int per = 2 * nri * nt;
        const int item = row / per, w = row % per;
        const int h = w / (nri * nt), b = (w / nt) % nri, t = w % nt;
        const int logn = dc.logn;
        ExtProdRow r;
        r.dig = dig + (((size_t)item * nqj * nt + t) << logn);
        r.key = key + ((((size_t)h * kdnum * nri + b) * nt + t) << logn);
        r.ds = (size_t)nt << logn;
        r.ks = (size_t)nri * nt << logn;
        r.ndig = nqj;
        const int pi = dc.idx_t + t;
        r.q = dc.mods[pi]; r.mh = dc.mu_hi[pi]; r.ml = dc.mu_lo[pi];
        return r;
    }
};

}  // namespace kbfv
