// K5 of the multiply pipeline, per coefficient: t/Q scale-and-round Q|R -> R,
// the base extension R -> Q and the key-switch digit lift; and K3 with the
// Q -> R base extension in its loader (q2r_ntt.cuh). Each bucket of the
// prime count (MAXQ) is instantiated in its own translation unit
// (k5_m<MAXQ>.cu) so that the unrolled variants compile in parallel.
#pragma once
#include "mixed.cuh"
#include "q2r_ntt.cuh"

// K5 in one kernel, for launches of one or two pairs (one launch less on the
// per-call path): scale-and-round to R, R -> Q, and (mode 1) the key-switch
// lift of a1*a2.
// mode 0: all three outputs over Q to out0 ([item][3][nq]).
// mode 1: a1*a2 lifted into sd2 ([item][dnum][npq]); cross, b1*b2 to sd ([item][2][nq]).
// mode 2: a1*a2 over Q into sd2 ([item][nq]); cross, b1*b2 to sd (T-base key switch).
template <int MAXQ>
static __global__ void k5_round_kernel(DevConsts c, const uint64_t* __restrict__ sc, uint64_t* __restrict__ out0,
                                uint64_t* __restrict__ sd, uint64_t* __restrict__ sd2, int mode) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int poly = blockIdx.y, item = poly / 3, which = poly % 3;
    const uint64_t* src = sc + ((size_t)poly * c.nqr << c.logn);
    uint64_t xq[MAXQ], xr[MAXQ + 1], rr[MAXQ + 1];
#pragma unroll
    for (int i = 0; i < MAXQ; i++)
        if (i < c.nq) xq[i] = src[((size_t)i << c.logn) + k];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) xr[j] = src[((size_t)(c.nq + j) << c.logn) + k];
    scale_round_coeff<MAXQ>(c, xq, xr, rr);
    // R -> Q
    const BconvTables tb = r2q_tables(c);
    uint64_t y[MAXQ + 1];
    const long long v = bconv_prep<MAXQ + 1>(y, rr, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
#pragma unroll
    for (int i = 0; i < MAXQ; i++) {
        if (i < c.nq)
            xq[i] = bconv_out<MAXQ + 1>(y, tb.nin, tb.hat + (size_t)i * tb.nin, tb.alpha[v * tb.nout + i],
                                        c.mods[i], c.mu_hi[i], c.mu_lo[i]);
    }
    if (mode == 0) {
        uint64_t* dst = out0 + ((size_t)poly * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    } else if (which == 0 && mode == 2) {  // a1*a2 over Q, coefficient form, to sd2 ([item][nq])
        uint64_t* dst = sd2 + ((size_t)item * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    } else if (which == 0) {
        modup_coeff<MAXQ>(c, xq, sd2 + ((size_t)item * c.dnum * c.npq << c.logn), k);
    } else {
        uint64_t* dst = sd + (((size_t)item * 2 + (which - 1)) * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    }
}

// K5, in two kernels so that each holds fewer registers (more warps per SM):
// K5a: t/Q scale-and-round Q|R -> R of each tensor polynomial into rr ([poly][nr]).
template <int MAXQ>
static __global__ void k5_scale_kernel(DevConsts c, const uint64_t* __restrict__ sc, uint64_t* __restrict__ rr_out,
                                       int ahead) {
    prefetch_chunk_ahead(sc, (size_t)c.nqr << c.logn, c.nqr, c.logn, blockDim.x, ahead);
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int poly = blockIdx.y;
    const uint64_t* src = sc + ((size_t)poly * c.nqr << c.logn);
    uint64_t xq[MAXQ], xr[MAXQ + 1], rr[MAXQ + 1];
#pragma unroll
    for (int i = 0; i < MAXQ; i++)
        if (i < c.nq) xq[i] = src[((size_t)i << c.logn) + k];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) xr[j] = src[((size_t)(c.nq + j) << c.logn) + k];
    scale_round_coeff<MAXQ>(c, xq, xr, rr);
    uint64_t* dst = rr_out + ((size_t)poly * c.nr << c.logn);
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) dst[((size_t)j << c.logn) + k] = rr[j];
}

// K5b: R -> Q, and (mode 1) the key-switch lift of a1*a2.
// mode 0: all three outputs over Q to out0 ([item][3][nq]).
// mode 1: a1*a2 lifted into sd2 ([item][dnum][npq]); cross, b1*b2 to sd ([item][2][nq]).
// mode 2: a1*a2 over Q into sd2 ([item][nq]); cross, b1*b2 to sd (T-base key switch).
template <int MAXQ>
static __global__ void k5_lift_kernel(DevConsts c, const uint64_t* __restrict__ rr_in, uint64_t* __restrict__ out0,
                               uint64_t* __restrict__ sd, uint64_t* __restrict__ sd2, int mode, int ahead) {
    prefetch_chunk_ahead(rr_in, (size_t)c.nr << c.logn, c.nr, c.logn, blockDim.x, ahead);
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int poly = blockIdx.y, item = poly / 3, which = poly % 3;
    const uint64_t* src = rr_in + ((size_t)poly * c.nr << c.logn);
    uint64_t rr[MAXQ + 1], xq[MAXQ];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) rr[j] = src[((size_t)j << c.logn) + k];
    const BconvTables tb = r2q_tables(c);
    uint64_t y[MAXQ + 1];
    const long long v = bconv_prep<MAXQ + 1>(y, rr, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
#pragma unroll
    for (int i = 0; i < MAXQ; i++) {
        if (i < c.nq)
            xq[i] = bconv_out<MAXQ + 1>(y, tb.nin, tb.hat + (size_t)i * tb.nin, tb.alpha[v * tb.nout + i],
                                        c.mods[i], c.mu_hi[i], c.mu_lo[i]);
    }
    if (mode == 0) {
        uint64_t* dst = out0 + ((size_t)poly * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    } else if (which == 0 && mode == 2) {  // a1*a2 over Q, coefficient form, to sd2 ([item][nq])
        uint64_t* dst = sd2 + ((size_t)item * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    } else if (which == 0) {
        modup_coeff<MAXQ>(c, xq, sd2 + ((size_t)item * c.dnum * c.npq << c.logn), k);
    } else {
        uint64_t* dst = sd + (((size_t)item * 2 + (which - 1)) * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    }
}

template <int MAXQ>
void k5_launch_m(const DevConsts& dc, int count, const MulScratch& m, uint64_t* out0, int mode, cudaStream_t st) {
    const int threads = dc.shape.k5_threads;
    dim3 grid((unsigned)((1u << dc.logn) / threads), (unsigned)(count * 3));
    // the R limbs of the inputs (m.sb, 4 x nr limbs per pair) are dead after K4:
    // they hold the scale-and-round results (3 x nr limbs per pair)
    if (count <= dc.shape.k5_fused_pairs) {
        k5_round_kernel<MAXQ><<<grid, threads, 0, st>>>(dc, m.sc, out0, m.sd, m.sd2, mode);
    } else {
        static int res_scale[4] = {0, 0, 0, 0}, res_lift[4] = {0, 0, 0, 0};
        const int a = dc.shape.l2_prefetch ? resident_ctas_at((const void*)k5_scale_kernel<MAXQ>, threads, 0, res_scale) : 0;
        const int b = dc.shape.l2_prefetch ? resident_ctas_at((const void*)k5_lift_kernel<MAXQ>, threads, 0, res_lift) : 0;
        k5_scale_kernel<MAXQ><<<grid, threads, 0, st>>>(dc, m.sc, m.sb, a);
        k5_lift_kernel<MAXQ><<<grid, threads, 0, st>>>(dc, m.sb, out0, m.sd, m.sd2, mode, b);
    }
    check_launch("k5_round");
}

// ---- mixed-level batches (see mixed.cuh): the level of each CTA's item
// chooses the constants; scratch has the top level's per-item layout ----------

// K5a over a mixed batch: grid.y = item x 3 tensor polynomials
template <int MAXQ>
static __global__ void k5_scale_mixed_kernel(Groups G, const uint64_t* __restrict__ sc, uint64_t* __restrict__ rr_out) {
    __shared__ DevConsts c;
    const int item = blockIdx.y / 3, which = blockIdx.y % 3, g = G.group_of_item(item);
    load_level_consts(c, G.lv[g]);
    const int logn = G.logn;
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = sc + (((size_t)item * 3 * G.top_nqr + (size_t)which * c.nqr) << logn);
    uint64_t xq[MAXQ], xr[MAXQ + 1], rr[MAXQ + 1];
#pragma unroll
    for (int i = 0; i < MAXQ; i++)
        if (i < c.nq) xq[i] = src[((size_t)i << logn) + k];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) xr[j] = src[((size_t)(c.nq + j) << logn) + k];
    scale_round_coeff<MAXQ>(c, xq, xr, rr);
    uint64_t* dst = rr_out + (((size_t)item * 3 * G.top_nr + (size_t)which * c.nr) << logn);
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) dst[((size_t)j << logn) + k] = rr[j];
}

// K5b over a mixed batch: R -> Q; a1*a2 lifted into the digits (sd2), the cross
// term and b1*b2 to sd
template <int MAXQ>
static __global__ void k5_lift_mixed_kernel(Groups G, const uint64_t* __restrict__ rr_in, uint64_t* __restrict__ sd,
                                            uint64_t* __restrict__ sd2) {
    __shared__ DevConsts c;
    const int item = blockIdx.y / 3, which = blockIdx.y % 3, g = G.group_of_item(item);
    load_level_consts(c, G.lv[g]);
    const int logn = G.logn;
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = rr_in + (((size_t)item * 3 * G.top_nr + (size_t)which * c.nr) << logn);
    uint64_t rr[MAXQ + 1], xq[MAXQ];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) rr[j] = src[((size_t)j << logn) + k];
    const BconvTables tb = r2q_tables(c);
    uint64_t y[MAXQ + 1];
    const long long v = bconv_prep<MAXQ + 1>(y, rr, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
#pragma unroll
    for (int i = 0; i < MAXQ; i++) {
        if (i < c.nq)
            xq[i] = bconv_out<MAXQ + 1>(y, tb.nin, tb.hat + (size_t)i * tb.nin, tb.alpha[v * tb.nout + i],
                                        c.mods[i], c.mu_hi[i], c.mu_lo[i]);
    }
    if (which == 0) {
        modup_coeff<MAXQ>(c, xq, sd2 + (((size_t)item * G.top_dnum * G.top_npq) << logn), k);
    } else {
        uint64_t* dst = sd + (((size_t)item * 2 * G.top_nq + (size_t)(which - 1) * c.nq) << logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << logn) + k] = xq[i];
    }
}

// K2 (Q -> R) of a mixed batch; MAXQ bounds the top level's ciphertext primes + 1
template <int MAXQ>
void bconv_mixed_launch_m(const Groups& G, const LaunchShape& sh, int count, const MulScratch& m, cudaStream_t st) {
    const int threads = sh.bconv_threads;
    dim3 grid((unsigned)((1u << G.logn) / threads), (unsigned)(count * 4));
    const size_t smem = (size_t)G.top_nq * G.top_nr * 8;
    bconv_mixed_kernel<MAXQ><<<grid, threads, smem, st>>>(G, m.sa, m.sb);
    check_launch("bconv_mixed");
}

// K5a + K5b of a mixed batch
template <int MAXQ>
void k5_mixed_launch_m(const Groups& G, const LaunchShape& sh, int count, const MulScratch& m, cudaStream_t st) {
    const int threads = sh.k5_threads;
    dim3 grid((unsigned)((1u << G.logn) / threads), (unsigned)(count * 3));
    k5_scale_mixed_kernel<MAXQ><<<grid, threads, 0, st>>>(G, m.sc, m.sb);
    k5_lift_mixed_kernel<MAXQ><<<grid, threads, 0, st>>>(G, m.sb, m.sd, m.sd2);
    check_launch("k5_mixed");
}
