// Non-NTT kernels: HPS base extension and rounding, key-switch lift / mod-down,
// XSalsa20 samplers and limb-wise arithmetic.
//
// Floating-point steps restate the reference bit for bit: the double sums of
// the HPS steps are fused multiply-adds (the reference's nvcc build contracts
// `acc += (double)x * c`), the key-switch quotient estimate is single-precision
// division and addition in source order (include/BasisConv.cuh:100-108).
#pragma once
#include "context.cuh"

namespace kbfv {

// ===========================================================================
// HPS base extension (BaseConverter::bConv_HPS, include/BasisConv_QR.cuh:191-207;
// include/poly_arithmetic.cuh:1078-1178): centred lift of x mod B into O.
// ===========================================================================
// Per-coefficient kernels over a 2-D grid (x: chunks of `chunk` coefficients,
// y: polynomials of `nrows` limbs, `poly_stride` words apart): threads
// 0 .. nrows-1 ask L2 for their limb's chunk of the CTA `ahead` places later in
// launch order (ahead = CTAs resident at once; 0: none), so that CTA's loads
// hit L2 instead of waiting on HBM.
__device__ __forceinline__ void prefetch_chunk_ahead(const uint64_t* in, size_t poly_stride, int nrows, int logn,
                                                     int chunk, int ahead) {
    if (ahead <= 0 || (int)threadIdx.x >= nrows) return;
    const unsigned lin = blockIdx.y * gridDim.x + blockIdx.x + (unsigned)ahead;
    if (lin >= gridDim.x * gridDim.y) return;
    const unsigned bx = lin % gridDim.x, by = lin / gridDim.x;
    l2_prefetch(in + by * poly_stride + ((size_t)threadIdx.x << logn) + (size_t)bx * chunk, (uint32_t)chunk * 8);
}

template <int MAXIN>
__device__ __forceinline__ long long bconv_prep(uint64_t* y, const uint64_t* x, int nin,
                                                const uint64_t* __restrict__ in_mods,
                                                const uint64_t* __restrict__ hatinv,
                                                const uint64_t* __restrict__ hatinvs,
                                                const double* __restrict__ binv) {
    double frac = 0.0;
#pragma unroll
    for (int i = 0; i < MAXIN; i++) {
        if (i < nin) {
            y[i] = shoup(x[i], hatinv[i], hatinvs[i], in_mods[i]);
            frac = __fma_rn(__ull2double_rn(y[i]), binv[i], frac);
        }
    }
    return llround(frac);
}

template <int MAXIN>
__device__ __forceinline__ uint64_t bconv_out(const uint64_t* y, int nin, const uint64_t* hat_row,
                                              uint64_t alpha_v, uint64_t o, uint64_t mh, uint64_t ml) {
    u128 acc{0, 0};
#pragma unroll
    for (int i = 0; i < MAXIN; i++)
        if (i < nin) mac(acc, y[i], hat_row[i]);
    return sub_mod(barrett128(acc, o, mh, ml), alpha_v, o);
}

struct BconvTables {
    const uint64_t* in_mods;
    const uint64_t* out_mods;
    const uint64_t* out_mu_hi;
    const uint64_t* out_mu_lo;
    const uint64_t* hatinv;
    const uint64_t* hatinvs;
    const uint64_t* hat;     // [nout][nin]
    const uint64_t* alpha;   // [nin+1][nout]
    const double* binv;
    int nin, nout;
};

__host__ __device__ inline BconvTables q2r_tables(const DevConsts& c) {
    return BconvTables{c.mods, c.mods + c.idx_r, c.mu_hi + c.idx_r, c.mu_lo + c.idx_r,
                       c.q2r_hatinv, c.q2r_hatinvs, c.q2r_hat, c.q2r_alpha, c.q2r_inv, c.nq, c.nr};
}
__host__ __device__ inline BconvTables r2q_tables(const DevConsts& c) {
    return BconvTables{c.mods + c.idx_r, c.mods, c.mu_hi, c.mu_lo,
                       c.r2q_hatinv, c.r2q_hatinvs, c.r2q_hat, c.r2q_alpha, c.r2q_inv, c.nr, c.nq};
}

// one thread per coefficient; grid.y = polynomial
template <int MAXIN>
static __global__ void bconv_kernel(BconvTables tb, const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                             int logn, size_t in_stride, size_t out_stride, int ahead) {
    extern __shared__ uint64_t sh_hat[];
    prefetch_chunk_ahead(in, in_stride, tb.nin, logn, blockDim.x, ahead);
    for (int i = threadIdx.x; i < tb.nin * tb.nout; i += blockDim.x) sh_hat[i] = tb.hat[i];
    __syncthreads();
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = in + blockIdx.y * in_stride;
    uint64_t* dst = out + blockIdx.y * out_stride;
    uint64_t x[MAXIN], y[MAXIN];
#pragma unroll
    for (int i = 0; i < MAXIN; i++)
        if (i < tb.nin) x[i] = src[((size_t)i << logn) + k];
    long long v = bconv_prep<MAXIN>(y, x, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
    for (int j = 0; j < tb.nout; j++) {
        dst[((size_t)j << logn) + k] = bconv_out<MAXIN>(y, tb.nin, sh_hat + j * tb.nin, tb.alpha[v * tb.nout + j],
                                                        tb.out_mods[j], tb.out_mu_hi[j], tb.out_mu_lo[j]);
    }
}

// Two coefficients per thread (k and k + 1: 16-byte loads and stores): the
// table reads of each output prime (the hat row in shared memory, modulus,
// Barrett constants) serve both, and the two multiply-accumulate chains are
// independent. Per coefficient the arithmetic is bconv_kernel's.
template <int MAXIN>
static __global__ void bconv2_kernel(BconvTables tb, const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                     int logn, size_t in_stride, size_t out_stride, int ahead) {
    extern __shared__ uint64_t sh_hat[];
    prefetch_chunk_ahead(in, in_stride, tb.nin, logn, 2 * blockDim.x, ahead);
    for (int i = threadIdx.x; i < tb.nin * tb.nout; i += blockDim.x) sh_hat[i] = tb.hat[i];
    __syncthreads();
    const size_t k = 2 * ((size_t)blockIdx.x * blockDim.x + threadIdx.x);
    const uint64_t* src = in + blockIdx.y * in_stride;
    uint64_t* dst = out + blockIdx.y * out_stride;
    uint64_t y0[MAXIN], y1[MAXIN];
#pragma unroll
    for (int i = 0; i < MAXIN; i++) {
        if (i < tb.nin) {
            const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(src + ((size_t)i << logn) + k);
            y0[i] = v.x;
            y1[i] = v.y;
        }
    }
    const long long v0 = bconv_prep<MAXIN>(y0, y0, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
    const long long v1 = bconv_prep<MAXIN>(y1, y1, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
    for (int j = 0; j < tb.nout; j++) {
        const uint64_t* hr = sh_hat + j * tb.nin;
        const uint64_t o = tb.out_mods[j], mh = tb.out_mu_hi[j], ml = tb.out_mu_lo[j];
        u128 a0{0, 0}, a1{0, 0};
#pragma unroll
        for (int i = 0; i < MAXIN; i++) {
            if (i < tb.nin) {
                const uint64_t h = hr[i];
                mac(a0, y0[i], h);
                mac(a1, y1[i], h);
            }
        }
        ulonglong2 r;
        r.x = sub_mod(barrett128(a0, o, mh, ml), tb.alpha[v0 * tb.nout + j], o);
        r.y = sub_mod(barrett128(a1, o, mh, ml), tb.alpha[v1 * tb.nout + j], o);
        *reinterpret_cast<ulonglong2*>(dst + ((size_t)j << logn) + k) = r;
    }
}

// ===========================================================================
// t/Q scale-and-round Q|R -> R (scaleAndRound_HPS_QR_R_kernel,
// include/poly_arithmetic.cuh:1263-1307). x: nq values then nr values.
// ===========================================================================
template <int MAXQ>
__device__ __forceinline__ void scale_round_coeff(const DevConsts& c, const uint64_t* xq, const uint64_t* xr,
                                                  uint64_t* out_r) {
    double nu = 0.5;
#pragma unroll
    for (int i = 0; i < MAXQ; i++)
        if (i < c.nq) nu = __fma_rn(__ull2double_rn(xq[i]), c.sr_frac[i], nu);
    const uint64_t alpha = __double2ull_rz(nu);
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++) {
        if (j < c.nr) {
            const uint64_t* cj = c.sr_c + (size_t)j * (c.nq + 1);
            u128 acc{0, 0};
#pragma unroll
            for (int i = 0; i < MAXQ; i++)
                if (i < c.nq) mac(acc, xq[i], cj[i]);
            mac(acc, xr[j], cj[c.nq]);
            const int pj = c.idx_r + j;
            const uint64_t rj = c.mods[pj];
            const uint64_t v = barrett128(acc, rj, c.mu_hi[pj], c.mu_lo[pj]);
            // alpha is reduced mod each r_j on its own (the reference chains the
            // reduction across r_0, r_1, ..., which breaks the R residues)
            out_r[j] = add_mod(v, barrett64(alpha, rj, c.mu_hi[pj]), rj);
        }
    }
}

template <int MAXQ>
static __global__ void scale_round_kernel(DevConsts c, const uint64_t* __restrict__ in, uint64_t* __restrict__ out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = in + ((size_t)blockIdx.y * c.nqr << c.logn);
    uint64_t* dst = out + ((size_t)blockIdx.y * c.nr << c.logn);
    uint64_t xq[MAXQ], xr[MAXQ + 1], rr[MAXQ + 1];
#pragma unroll
    for (int i = 0; i < MAXQ; i++)
        if (i < c.nq) xq[i] = src[((size_t)i << c.logn) + k];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) xr[j] = src[((size_t)(c.nq + j) << c.logn) + k];
    scale_round_coeff<MAXQ>(c, xq, xr, rr);
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) dst[((size_t)j << c.logn) + k] = rr[j];
}

// ===========================================================================
// key-switch digit lift (modUpQjtoT_23's estimate, include/BasisConv.cuh:86-135,
// retargeted to the primes of Q|P outside the digit)
// ===========================================================================
template <int MAXQ>
__device__ __forceinline__ void modup_coeff(const DevConsts& c, const uint64_t* xq, uint64_t* __restrict__ out,
                                            size_t k) {
    // out: [dnum][npq] rows of N. Register arrays are indexed by unrolled
    // prime positions only; digit membership is a runtime test.
    for (int d = 0; d < c.dnum; d++) {
        const int lo = d * c.alpha;
        const int hi = min(lo + c.alpha, c.nq);
        uint64_t rb[MAXQ];
        float vv = 0.f;
#pragma unroll
        for (int i = 0; i < MAXQ; i++) {
            rb[i] = 0;
            if (i >= lo && i < hi) {
                const uint64_t qi = c.mods[i];
                rb[i] = shoup(xq[i], c.dig_hatinv[i], c.dig_hatinvs[i], qi);
                vv = __fadd_rn(vv, __fdiv_rn(__ull2float_rn(rb[i]), __ull2float_rn(qi)));
            }
        }
        const int vf = min(__float2int_rz(vv), c.alpha);
        const uint64_t* vq = c.dig_vq_mod + ((size_t)d * (c.alpha + 1) + vf) * c.npq;
        uint64_t* o = out + ((size_t)d * c.npq << c.logn);
        // the digit's own primes: the input residues
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i >= lo && i < hi) o[((size_t)i << c.logn) + k] = xq[i];
        // every other prime of Q|P: approximate CRT of the digit
        for (int m = 0; m < c.npq; m++) {
            if (m >= lo && m < hi) continue;
            const uint64_t* hm = c.dig_hat_mod + ((size_t)d * c.npq + m) * c.alpha - lo;
            u128 acc{0, 0};
#pragma unroll
            for (int i = 0; i < MAXQ; i++)
                if (i >= lo && i < hi) mac(acc, rb[i], hm[i]);
            // subtract v * Q_d after reducing: the sum can be below v * Q_d (one-prime digits)
            o[((size_t)m << c.logn) + k] = sub_mod(barrett128(acc, c.mods[m], c.mu_hi[m], c.mu_lo[m]), vq[m], c.mods[m]);
        }
    }
}

template <int MAXQ>
static __global__ void modup_kernel(DevConsts c, const uint64_t* __restrict__ in, uint64_t* __restrict__ out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = in + ((size_t)blockIdx.y * c.nq << c.logn);
    uint64_t* dst = out + ((size_t)blockIdx.y * c.dnum * c.npq << c.logn);
    uint64_t xq[MAXQ];
#pragma unroll
    for (int i = 0; i < MAXQ; i++)
        if (i < c.nq) xq[i] = src[((size_t)i << c.logn) + k];
    modup_coeff<MAXQ>(c, xq, dst, k);
}

// (x_q - conv_{P->q}(x_P)) * P^-1 mod q (modDownPQltoQl_23_{alpha1_,}multi_kernel,
// include/BasisConv.cuh:229-300); x points at limb 0 of a Q|P polynomial.
__device__ __forceinline__ uint64_t moddown_elem(const DevConsts& c, const uint64_t* x, int l, size_t k) {
    const uint64_t ql = c.mods[l];
    uint64_t conv;
    if (c.np == 1) {
        conv = barrett64(x[((size_t)c.nq << c.logn) + k], ql, c.mu_hi[l]);
    } else {
        u128 acc{0, 0};
        for (int kk = 0; kk < c.np; kk++) {
            const int pk = c.idx_p + kk;
            uint64_t rb = shoup(x[((size_t)(c.nq + kk) << c.logn) + k], c.phatinv_p[kk], c.phatinv_ps[kk], c.mods[pk]);
            mac(acc, rb, c.phat_mod_q[(size_t)l * c.np + kk]);
        }
        conv = barrett128(acc, ql, c.mu_hi[l], c.mu_lo[l]);
    }
    const uint64_t v = ql - conv + x[((size_t)l << c.logn) + k];
    return shoup(v, c.pinv_q[l], c.pinv_qs[l], ql);
}

static __global__ void moddown_kernel(DevConsts c, const uint64_t* __restrict__ in, uint64_t* __restrict__ out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* x = in + ((size_t)blockIdx.y * c.npq << c.logn);
    uint64_t* y = out + ((size_t)blockIdx.y * c.nq << c.logn);
    for (int l = 0; l < c.nq; l++) y[((size_t)l << c.logn) + k] = moddown_elem(c, x, l, k);
}

// ===========================================================================
// decrypt rounding (hps_decrypt_scale_and_round_kernel_*, include/poly_arithmetic.cuh:930-1075)
// ===========================================================================
template <int MAXQ>
__device__ __forceinline__ uint64_t decrypt_round_coeff(const DevConsts& c, const uint64_t* __restrict__ src,
                                                       size_t k) {
    const uint64_t t = c.t;
    const int hf = c.qmsbhf;
    const uint64_t mask = ((uint64_t)1 << hf) - 1;
    const double tinv = __drcp_rn((double)t);
    double ds = 0.0;
    uint64_t is = 0;
#pragma unroll
    for (int i = 0; i < MAXQ; i++) {
        if (i >= c.nq) break;
        const uint64_t x = src[((size_t)i << c.logn) + k];
        switch (c.dec_variant) {
            case 0:
                ds = __fma_rn(__ull2double_rn(x), c.dec_frac[i], ds);
                is += shoup(x, c.dec_mod_t[i], c.dec_mod_t_s[i], t);
                break;
            case 1:
                ds = __fma_rn(__ull2double_rn(x), c.dec_frac[i], ds);
                is += x * c.dec_mod_t[i];
                break;
            case 2: {
                const uint64_t hi = x >> hf, lo = x & mask;
                ds = __fma_rn(__ull2double_rn(lo), c.dec_frac[i], ds);
                ds = __fma_rn(__ull2double_rn(hi), c.dec_fracB[i], ds);
                is += shoup(lo, c.dec_mod_t[i], c.dec_mod_t_s[i], t);
                is += shoup(hi, c.dec_modB_t[i], c.dec_modB_t_s[i], t);
                break;
            }
            default: {
                const uint64_t hi = x >> hf, lo = x & mask;
                ds = __fma_rn(__ull2double_rn(lo), c.dec_frac[i], ds);
                ds = __fma_rn(__ull2double_rn(hi), c.dec_fracB[i], ds);
                is += lo * c.dec_mod_t[i];
                is += hi * c.dec_modB_t[i];
                break;
            }
        }
    }
    ds = __dadd_rn(ds, __ull2double_rn(is));
    const uint64_t quot = __double2ull_rz(__dmul_rn(ds, tinv));
    ds = __dsub_rn(ds, __ull2double_rn(t * quot));
    return (uint64_t)llround(ds);
}

template <int MAXQ>
static __global__ void decrypt_round_kernel(DevConsts c, const uint64_t* __restrict__ in, uint64_t* __restrict__ out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = in + ((size_t)blockIdx.y * c.nq << c.logn);
    out[((size_t)blockIdx.y << c.logn) + k] = decrypt_round_coeff<MAXQ>(c, src, k);
}

// ===========================================================================
// limb-wise arithmetic. Index space: items x polys x limbs x N; the prime of a
// limb is prime0 + limb.
// ===========================================================================
struct LimbIdx {
    int logn, limbs;
    __device__ __forceinline__ int limb(size_t i) const { return (int)((i >> logn) % (size_t)limbs); }
};

// ceil(Q*m/t) per limb (bfv_add_timesQ_overt_kernel, include/poly_arithmetic.cuh:902-927)
static __global__ void delta_m_kernel(DevConsts c, const uint64_t* __restrict__ m, uint64_t* __restrict__ out, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const size_t n = (size_t)1 << c.logn;
    const int l = (int)((i >> c.logn) % c.nq);
    const size_t poly = i / (n * c.nq);
    const uint64_t mv = m[poly * n + (i & (n - 1))];
    const uint64_t mq = shoup(mv, c.negq_mod_t, c.negq_mod_t_s, c.t);
    out[i] = shoup(mq, c.tinv_q[l], c.tinv_qs[l], c.mods[l]);
}

static __global__ void add_kernel(DevConsts c, const uint64_t* __restrict__ x, const uint64_t* __restrict__ y,
                           uint64_t* __restrict__ out, size_t total, int limbs) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int l = (int)((i >> c.logn) % limbs);
    out[i] = add_mod(x[i], y[i], c.mods[l]);
}

// limb-wise linear ops over ciphertexts (rows of N, limb = row % limbs):
// op 0: out = x - y; 1: out = -x; 2: out = x * c_l; 3: out = y + x * c_l
// (c_l = cnst mod q_l with its Shoup constant, passed by value)
struct ScalarTab {
    uint64_t c[kMaxQ], cs[kMaxQ];
};
static __global__ void linear_kernel(DevConsts c, const uint64_t* x, const uint64_t* y, uint64_t* out, size_t total,
                              int limbs, int op, ScalarTab tab) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int l = (int)((i >> c.logn) % limbs);
    const uint64_t q = c.mods[l];
    uint64_t v;
    if (op == 0) v = sub_mod(x[i], y[i], q);
    else if (op == 1) v = x[i] ? q - x[i] : 0;
    else if (op == 2) v = shoup(x[i], tab.c[l], tab.cs[l], q);
    else v = add_mod(y[i], shoup(x[i], tab.c[l], tab.cs[l], q), q);
    out[i] = v;
}

// ct (items x 2 x nq) times pt (items x nq)
static __global__ void mul_plain_kernel(DevConsts c, const uint64_t* __restrict__ ct, const uint64_t* __restrict__ pt,
                                 uint64_t* __restrict__ out, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const size_t lq = (size_t)c.nq << c.logn;
    const int l = (int)((i >> c.logn) % c.nq);
    const size_t item = i / (2 * lq);
    const uint64_t p = pt[item * lq + (i % lq)];
    out[i] = mul_mod(ct[i], p, c.mods[l], c.mu_hi[l], c.mu_lo[l]);
}

// tensor over Q|R for the C-ABI building block: pairs of [a|b] (nqr limbs each)
static __global__ void tensor_qr_kernel(DevConsts c, const uint64_t* __restrict__ c1, const uint64_t* __restrict__ c2,
                                 uint64_t* __restrict__ out, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;  // total = pairs * nqr * N
    const size_t lqr = (size_t)c.nqr << c.logn;
    const size_t pair = i / lqr, w = i % lqr;
    const int l = (int)(w >> c.logn);
    const int pi = l < c.nq ? l : c.idx_r + (l - c.nq);
    const uint64_t q = c.mods[pi], mh = c.mu_hi[pi], ml = c.mu_lo[pi];
    const uint64_t a1 = c1[pair * 2 * lqr + w], b1 = c1[pair * 2 * lqr + lqr + w];
    const uint64_t a2 = c2[pair * 2 * lqr + w], b2 = c2[pair * 2 * lqr + lqr + w];
    u128 cr = mul_wide(a1, b2);
    mac(cr, b1, a2);
    out[pair * 3 * lqr + w] = mul_mod(a1, a2, q, mh, ml);
    out[pair * 3 * lqr + lqr + w] = barrett128(cr, q, mh, ml);
    out[pair * 3 * lqr + 2 * lqr + w] = mul_mod(b1, b2, q, mh, ml);
}

// ===========================================================================
// XSalsa20 (corrected Salsa20/20 of include/RNG_impl.cuh:70-176) and samplers
// ===========================================================================
struct SalsaKey {
    uint32_t k[8];
    uint32_t sigma[4];
};

__device__ __forceinline__ uint32_t rotl32(uint32_t u, int c) { return __funnelshift_l(u, u, c); }

__device__ __forceinline__ void salsa_block(const SalsaKey& key, uint32_t n0, uint32_t n1, uint64_t ctr,
                                            uint32_t out[16]) {
    uint32_t j[16], x[16];
    j[0] = key.sigma[0]; j[5] = key.sigma[1]; j[10] = key.sigma[2]; j[15] = key.sigma[3];
    j[1] = key.k[0]; j[2] = key.k[1]; j[3] = key.k[2]; j[4] = key.k[3];
    j[11] = key.k[4]; j[12] = key.k[5]; j[13] = key.k[6]; j[14] = key.k[7];
    j[6] = n0; j[7] = n1; j[8] = (uint32_t)ctr; j[9] = (uint32_t)(ctr >> 32);
#pragma unroll
    for (int i = 0; i < 16; i++) x[i] = j[i];
#pragma unroll
    for (int r = 0; r < 10; r++) {
        x[4] ^= rotl32(x[0] + x[12], 7);   x[8] ^= rotl32(x[4] + x[0], 9);
        x[12] ^= rotl32(x[8] + x[4], 13);  x[0] ^= rotl32(x[12] + x[8], 18);
        x[9] ^= rotl32(x[5] + x[1], 7);    x[13] ^= rotl32(x[9] + x[5], 9);
        x[1] ^= rotl32(x[13] + x[9], 13);  x[5] ^= rotl32(x[1] + x[13], 18);
        x[14] ^= rotl32(x[10] + x[6], 7);  x[2] ^= rotl32(x[14] + x[10], 9);
        x[6] ^= rotl32(x[2] + x[14], 13);  x[10] ^= rotl32(x[6] + x[2], 18);
        x[3] ^= rotl32(x[15] + x[11], 7);  x[7] ^= rotl32(x[3] + x[15], 9);
        x[11] ^= rotl32(x[7] + x[3], 13);  x[15] ^= rotl32(x[11] + x[7], 18);
        x[1] ^= rotl32(x[0] + x[3], 7);    x[2] ^= rotl32(x[1] + x[0], 9);
        x[3] ^= rotl32(x[2] + x[1], 13);   x[0] ^= rotl32(x[3] + x[2], 18);
        x[6] ^= rotl32(x[5] + x[4], 7);    x[7] ^= rotl32(x[6] + x[5], 9);
        x[4] ^= rotl32(x[7] + x[6], 13);   x[5] ^= rotl32(x[4] + x[7], 18);
        x[11] ^= rotl32(x[10] + x[9], 7);  x[8] ^= rotl32(x[11] + x[10], 9);
        x[9] ^= rotl32(x[8] + x[11], 13);  x[10] ^= rotl32(x[9] + x[8], 18);
        x[12] ^= rotl32(x[15] + x[14], 7); x[13] ^= rotl32(x[12] + x[15], 9);
        x[14] ^= rotl32(x[13] + x[12], 13); x[15] ^= rotl32(x[14] + x[13], 18);
    }
#pragma unroll
    for (int i = 0; i < 16; i++) out[i] = x[i] + j[i];
}

// raw keystream: block b of the stream written at byte 64*b (tail truncated)
static __global__ void salsa_stream_kernel(SalsaKey key, uint32_t n0, uint32_t n1, uint64_t block0, uint8_t* out,
                                    size_t nbytes) {
    const size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b * 64 >= nbytes) return;
    uint32_t w[16];
    salsa_block(key, n0, n1, block0 + b, w);
    const size_t m = nbytes - b * 64 < 64 ? nbytes - b * 64 : 64;
    const uint8_t* wb = reinterpret_cast<const uint8_t*>(w);
    for (size_t i = 0; i < m; i++) out[b * 64 + i] = wb[i];
}

// uniform residues: coefficient (limb l, k) of item i <- bytes [(l*N + k)*16, +16)
// of stream (id0 + i); value floor(u128 * q / 2^128). One thread = 4 coefficients.
static __global__ void sample_uniform_kernel(DevConsts c, SalsaKey key, uint64_t id0, int prime0, int limbs,
                                      uint64_t* __restrict__ out, size_t item_stride, int items) {
    const size_t n = (size_t)1 << c.logn;
    const size_t per_item = (size_t)limbs * n / 4;
    const size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= per_item * items) return;
    const size_t item = gid / per_item, b = gid % per_item;
    const uint64_t id = id0 + item;
    uint32_t w[16];
    salsa_block(key, (uint32_t)id, (uint32_t)(id >> 32), b, w);
#pragma unroll
    for (int s = 0; s < 4; s++) {
        const size_t coef = b * 4 + s;  // = l*N + k
        const int l = (int)(coef >> c.logn);
        const uint64_t q = c.mods[prime0 + l];
        const uint64_t lo = (uint64_t)w[4 * s] | ((uint64_t)w[4 * s + 1] << 32);
        const uint64_t hi = (uint64_t)w[4 * s + 2] | ((uint64_t)w[4 * s + 3] << 32);
        const uint64_t a1 = __umul64hi(lo, q);
        // floor((hi*q + a1) / 2^64)
        const uint64_t plo = hi * q;
        const uint64_t phi = __umul64hi(hi, q);
        const uint64_t sum = plo + a1;
        out[item * item_stride + coef] = phi + (sum < plo);
    }
}

// small polynomials (ternary: 4 bytes/coef, Gaussian: 8 bytes/coef), written
// as residues over `limbs` consecutive primes from prime0.
template <int KIND>
__device__ __forceinline__ void sample_small_block(const DevConsts& c, const SalsaKey& key, uint64_t id, size_t b,
                                                   int prime0, int limbs, uint64_t* __restrict__ out) {
    constexpr int PER = KIND == 0 ? 16 : 8;
    uint32_t w[16];
    salsa_block(key, (uint32_t)id, (uint32_t)(id >> 32), b, w);
#pragma unroll
    for (int s = 0; s < PER; s++) {
        int v;
        if (KIND == 0) {
            const uint32_t r = (uint32_t)(((uint64_t)w[s] * 3) >> 32);
            v = r == 0 ? 0 : (r == 1 ? 1 : -1);
        } else {
            const uint64_t u = (uint64_t)w[2 * s] | ((uint64_t)w[2 * s + 1] << 32);
            v = -c.gauss_bound;
            for (int j = 0; j < 2 * c.gauss_bound; j++) v += (u >= c.gauss_cdt[j]);
        }
        const size_t k = b * PER + s;
        for (int l = 0; l < limbs; l++) {
            const uint64_t q = c.mods[prime0 + l];
            out[((size_t)l << c.logn) + k] = v < 0 ? q - (uint64_t)(-v) : (uint64_t)v;
        }
    }
}

template <int KIND>
static __global__ void sample_small_kernel(DevConsts c, SalsaKey key, uint64_t id0, int prime0, int limbs,
                                    uint64_t* __restrict__ out, size_t item_stride, int items) {
    constexpr int PER = KIND == 0 ? 16 : 8;
    const size_t per_item = ((size_t)1 << c.logn) / PER;
    const size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= per_item * items) return;
    const size_t item = gid / per_item, b = gid % per_item;
    sample_small_block<KIND>(c, key, id0 + item, b, prime0, limbs, out + item * item_stride);
}

// the same with one stream id per item (ids passed by value)
struct IdTable {
    uint64_t v[128];
};
template <int KIND>
static __global__ void sample_small_ids_kernel(DevConsts c, SalsaKey key, IdTable ids, int prime0, int limbs,
                                        uint64_t* __restrict__ out, size_t item_stride, int items) {
    constexpr int PER = KIND == 0 ? 16 : 8;
    const size_t per_item = ((size_t)1 << c.logn) / PER;
    const size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= per_item * items) return;
    const size_t item = gid / per_item, b = gid % per_item;
    sample_small_block<KIND>(c, key, ids.v[item], b, prime0, limbs, out + item * item_stride);
}

// Hamming-weight-h ternary secret (convert_HWT, include/Sampler_impl.cuh:68-87):
// h positions from u32 & (N-1), sign from a byte >= 128; a later draw at the
// same position overwrites. One thread per item; `out` must be zeroed.
static __global__ void sample_hwt_kernel(DevConsts c, SalsaKey key, uint64_t id0, int h, int prime0, int limbs,
                                  uint64_t* __restrict__ out, size_t item_stride, int items) {
    const int item = blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= items) return;
    const uint64_t id = id0 + item;
    const size_t n = (size_t)1 << c.logn;
    auto byte_at = [&](size_t pos, uint32_t* cache, uint64_t& cached) -> uint8_t {
        const uint64_t blk = pos / 64;
        if (blk != cached) {
            salsa_block(key, (uint32_t)id, (uint32_t)(id >> 32), blk, cache);
            cached = blk;
        }
        return reinterpret_cast<const uint8_t*>(cache)[pos % 64];
    };
    uint32_t cache[16];
    uint64_t cached = ~(uint64_t)0;
    for (int i = 0; i < h; i++) {
        uint32_t p = 0;
        for (int b = 0; b < 4; b++) p |= (uint32_t)byte_at((size_t)4 * i + b, cache, cached) << (8 * b);
        const uint8_t sb = byte_at((size_t)4 * h + i, cache, cached);
        const size_t pos = p & (uint32_t)(n - 1);
        const bool plus = (float)sb / 128.0f >= 1.0f;
        for (int l = 0; l < limbs; l++) {
            const uint64_t q = c.mods[prime0 + l];
            out[item * item_stride + ((size_t)l << c.logn) + pos] = plus ? 1 : q - 1;
        }
    }
}

// ===========================================================================
// keygen / encrypt combinations (NTT domain)
// ===========================================================================
// pk.b = e - a*s over Q (addEncKey, include/BFVScheme.cuh:67-78)
static __global__ void pk_combine_kernel(DevConsts c, const uint64_t* __restrict__ a, const uint64_t* __restrict__ s,
                                  uint64_t* __restrict__ eb, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int l = (int)(i >> c.logn);
    eb[i] = sub_mod(eb[i], mul_mod(a[i], s[i], c.mods[l], c.mu_hi[l], c.mu_lo[l]), c.mods[l]);
}

// rlk digit d: b = e - a*s (+ P*s^2 on the digit's primes) over Q|P
// (addMultKey_23, include/KeySwitch_23.cuh:35-53)
static __global__ void rlk_combine_kernel(DevConsts c, const uint64_t* __restrict__ a, const uint64_t* __restrict__ s,
                                   uint64_t* __restrict__ eb, int digit, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int l = (int)(i >> c.logn);
    const uint64_t q = c.mods[l], mh = c.mu_hi[l], ml = c.mu_lo[l];
    uint64_t v = sub_mod(eb[i], mul_mod(a[i], s[i], q, mh, ml), q);
    const int lo = digit * c.alpha, hi = min(lo + c.alpha, c.nq);
    if (l >= lo && l < hi) {
        const uint64_t s2 = mul_mod(s[i], s[i], q, mh, ml);
        v = add_mod(v, mul_mod(s2, c.p_mod_q[l], q, mh, ml), q);
    }
    eb[i] = v;
}

// gadget key component: b = e - a*s + [l == prime] * g * s^2 (g = P * 2^{wj} mod q_prime)
static __global__ void gk_combine_kernel(DevConsts c, const uint64_t* __restrict__ a, const uint64_t* __restrict__ s,
                                  uint64_t* __restrict__ eb, int prime, uint64_t g, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int l = (int)(i >> c.logn);
    const uint64_t q = c.mods[l], mh = c.mu_hi[l], ml = c.mu_lo[l];
    uint64_t v = sub_mod(eb[i], mul_mod(a[i], s[i], q, mh, ml), q);
    if (l == prime) v = add_mod(v, mul_mod(mul_mod(s[i], s[i], q, mh, ml), g, q, mh, ml), q);
    eb[i] = v;
}

// ---------------------------------------------------------------------------
// The reference's conversions of random words into samples
// (include/Sampler_impl.cuh:13-108), restated operation for operation so that
// the same random words give the same samples: double arithmetic for the
// uniform one, float arithmetic and CUDA's normcdfinvf for the Gaussian one.
// ---------------------------------------------------------------------------
static __global__ void compat_uniform_kernel(DevConsts c, const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                      int prime0, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const uint64_t q = c.mods[prime0 + (int)(i >> c.logn)];
    double d = __ull2double_rn(in[i]);
    d = __ddiv_rn(d, 18446744073709551615.0);  // UINT64_MAX as a double (2^64)
    d = __dmul_rn(d, __ull2double_rn(q - 1));
    out[i] = __double2ull_rz(d);
}
static __global__ void compat_gauss_kernel(DevConsts c, const uint32_t* __restrict__ in, uint64_t* __restrict__ out,
                                    int prime0, int limbs) {
    const size_t n = (size_t)1 << c.logn;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float d = __uint2float_rn(in[i]);
    d = __fdiv_rn(d, 4294967296.0f);  // 4294967295 rounds to 2^32 as a float
    if (d == 0.f) d = __fadd_rn(d, 1.192092896e-07F);
    else if (d == 1.f) d = __fsub_rn(d, 1.192092896e-07F);
    d = normcdfinvf(d);
    d = __fmaf_rn(d, 3.2f, 0.0f);  // d * stdev + mean, contracted as nvcc does
    if ((double)d > 19.2) d = 19.2f;
    else if ((double)d < -19.2) d = -19.2f;
    const int dd = __float2int_rz(d);
    for (int t = 0; t < limbs; t++) {
        const uint64_t q = c.mods[prime0 + t];
        out[t * n + i] = dd < 0 ? q + (int64_t)dd : (uint64_t)dd;
    }
}
static __global__ void compat_zo_kernel(DevConsts c, const uint8_t* __restrict__ in, uint64_t* __restrict__ out,
                                 int prime0, int limbs, double probability) {
    const size_t n = (size_t)1 << c.logn;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double d = (double)(float)in[i];
    for (int t = 0; t < limbs; t++) {
        const uint64_t q = c.mods[prime0 + t];
        uint64_t v;
        if (d < 256.0 * probability) v = 0;
        else if (d < 256.0 * (1 + probability) / 2) v = 1;
        else v = q - 1;
        out[t * n + i] = v;
    }
}
// one block per limb, h threads: position word, then sign byte (out pre-zeroed)
static __global__ void compat_hwt_kernel(DevConsts c, const uint8_t* __restrict__ in, uint64_t* __restrict__ out,
                                  int prime0, int h) {
    const int t = blockIdx.x, j = threadIdx.x;
    if (j >= h) return;
    const uint32_t pos = ((const uint32_t*)in)[j] & (((uint32_t)1 << c.logn) - 1);
    const float d = __fdiv_rn((float)in[(size_t)h * 4 + j], 128.0f);
    out[((size_t)t << c.logn) + pos] = d >= 1.f ? 1 : c.mods[prime0 + t] - 1;
}

// Galois automorphism X -> X^g in NTT form: index i holds A(psi^(2 brv(i) + 1)),
// so the automorphism reads index perm(i) with 2 brv(perm(i)) + 1 = (2 brv(i) + 1) g mod 2N.
__device__ __forceinline__ uint32_t galois_perm(uint32_t i, uint64_t g, int logn) {
    const uint32_t bi = __brev(i) >> (32 - logn);
    const uint64_t e = ((2 * (uint64_t)bi + 1) * g) & ((2ULL << logn) - 1);
    return __brev((uint32_t)(e >> 1)) >> (32 - logn);
}
// out[poly][l][i] = in[poly][l][perm(i)]  (polys x limbs rows of N; out != in)
static __global__ void galois_ntt_kernel(DevConsts c, const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                                  uint64_t g, size_t total) {
    const size_t x = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= total) return;
    const size_t row = x >> c.logn;
    const uint32_t i = (uint32_t)(x & (((size_t)1 << c.logn) - 1));
    out[x] = in[(row << c.logn) + galois_perm(i, g, c.logn)];
}
// key-switch key component for a target polynomial t (NTT form over Q|P):
// b = e - a*s + [l in digit] * P * t
static __global__ void ksk_combine_kernel(DevConsts c, const uint64_t* __restrict__ a, const uint64_t* __restrict__ s,
                                   const uint64_t* __restrict__ target, uint64_t* __restrict__ eb, int digit,
                                   size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int l = (int)(i >> c.logn);
    const uint64_t q = c.mods[l], mh = c.mu_hi[l], ml = c.mu_lo[l];
    uint64_t v = sub_mod(eb[i], mul_mod(a[i], s[i], q, mh, ml), q);
    const int lo = digit * c.alpha, hi = min(lo + c.alpha, c.nq);
    if (l >= lo && l < hi) v = add_mod(v, mul_mod(target[i], c.p_mod_q[l], q, mh, ml), q);
    eb[i] = v;
}

// encrypt: a = v*pk.a + e0, b = v*pk.b + e1 + dm (encryptZero/encryptMsg,
// include/BFVScheme.cuh:87-146). work: items x [v | e0 | e1 | dm] x nq (NTT form)
static __global__ void enc_combine_kernel(DevConsts c, const uint64_t* __restrict__ pk, const uint64_t* __restrict__ work,
                                   uint64_t* __restrict__ ct, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;  // items * nq * N
    const size_t lq = (size_t)c.nq << c.logn;
    const size_t item = i / lq, w = i % lq;
    const int l = (int)(w >> c.logn);
    const uint64_t q = c.mods[l], mh = c.mu_hi[l], ml = c.mu_lo[l];
    const uint64_t* wk = work + item * 4 * lq;
    const uint64_t v = wk[w], e0 = wk[lq + w], e1 = wk[2 * lq + w], dm = wk[3 * lq + w];
    ct[item * 2 * lq + w] = add_mod(mul_mod(v, pk[w], q, mh, ml), e0, q);
    ct[item * 2 * lq + lq + w] = add_mod(add_mod(mul_mod(v, pk[lq + w], q, mh, ml), e1, q), dm, q);
}

}  // namespace kbfv
