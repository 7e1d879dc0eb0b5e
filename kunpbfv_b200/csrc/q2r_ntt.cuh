// K3 with the Q -> R base extension in its loader: each row of the forward
// NTT over R (polynomial, output prime r) computes its input coefficients from
// the polynomial's Q limbs instead of reading limbs that a separate
// base-conversion launch wrote (kernels.cuh: bconv_prep + bconv_out, the HPS
// Q -> R extension of include/poly_arithmetic.cuh's base conversion kernels).
// The inverse NTT over Q before it (K1) stores y_i = [x_i (Q/q_i)^-1]_{q_i}
// (QHatRowsIO), so a row's loader only accumulates
//   sum_i y_i * (Q/q_i mod r) - alpha_v * (Q mod r),  v = round(sum_i y_i / q_i),
// with the same operations, in the same order, as the two-kernel form: the
// R limbs are bit-identical. The R rows of one polynomial are adjacent CTAs,
// so their reads of the polynomial's Q limbs after the first are L2 hits.
#pragma once
#include "pipeline.cuh"

template <int MAXQ>
struct Q2RRow {
    const uint64_t* y;      // limb 0 of the polynomial's y rows (limb stride N)
    const uint64_t* hat;    // [nq]: Q/q_i mod r
    const uint64_t* alpha;  // column r of the alpha table (row stride nr)
    const double* binv;     // [nq]: 1/q_i
    int logn, nq, nr;
    uint64_t o, mh, ml;
    __device__ __forceinline__ uint64_t load(int j) const {
        double frac = 0.0;
        u128 acc{0, 0};
#pragma unroll
        for (int i = 0; i < MAXQ; i++) {
            if (i < nq) {
                const uint64_t v = y[((size_t)i << logn) + j];
                frac = __fma_rn(__ull2double_rn(v), binv[i], frac);
                mac(acc, v, hat[i]);
            }
        }
        return sub_mod(barrett128(acc, o, mh, ml), alpha[llround(frac) * nr], o);
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};

template <int MAXQ>
struct Q2RSrc {
    const uint64_t* y;  // [poly][nq] rows of y_i
    const uint64_t *hat, *alpha, *mods, *mu_hi, *mu_lo;
    const double* binv;
    int logn, nq, nr, idx_r;
    __device__ __forceinline__ int prime(int row) const { return idx_r + row % nr; }
    __device__ __forceinline__ Q2RRow<MAXQ> bind(int row) const {
        const int poly = row / nr, r = row % nr;
        Q2RRow<MAXQ> w;
        w.y = y + (((size_t)poly * nq) << logn);
        w.hat = hat + (size_t)r * nq;
        w.alpha = alpha + r;
        w.binv = binv;
        w.logn = logn; w.nq = nq; w.nr = nr;
        w.o = mods[idx_r + r]; w.mh = mu_hi[idx_r + r]; w.ml = mu_lo[idx_r + r];
        return w;
    }
};

template <int MAXQ>
void q2r_ntt_launch_m(const DevConsts& dc, const uint64_t* y, uint64_t* out, int polys, cudaStream_t st) {
    const Q2RSrc<MAXQ> src{y, dc.q2r_hat, dc.q2r_alpha, dc.mods, dc.mu_hi, dc.mu_lo, dc.q2r_inv,
                           dc.logn, dc.nq, dc.nr, dc.idx_r};
    ntt_fwd<Q2RSrc<MAXQ>, RowsIO, true>(dc, src, rows_io(dc, out, dc.idx_r, dc.nr), polys * dc.nr, st);
}
