// Row functors of the fused multiply pipeline (sources and store targets of
// the NTT kernels that carry the tensor product, key products, mod down and
// output epilogues) and the host functions that launch the pipeline's steps.
#pragma once
#include "internal.cuh"

// Pointer arrays must be device-readable: the batched entry points pass
// PtrBatch by value as a kernel parameter, so functors point into it through
// this wrapper kernel-parameter view.
struct PairQRowsP {
    PtrBatch pb;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const int item = row / (4 * nq), w = row % (4 * nq), p = w / nq, l = w % nq;
        const uint64_t* base = p < 2 ? pb.a[item] : pb.b[item];
        return PtrRow{const_cast<uint64_t*>(base) + (((size_t)(p & 1) * nq + l) << logn)};
    }
    __device__ __forceinline__ void prefetch(int row, int off, int n) const { bind(row).prefetch(off, n); }
};

// K1 store target when the Q -> R base extension runs inside K3: rows over Q
// (RowsIO layout) holding y_i = [x_i (Q/q_i)^-1]_{q_i}, the scale folded into
// the inverse transform's last-stage constants
struct QHatRowsIO {
    uint64_t* base;
    int logn, nq;
    const tw_t* fold_base;  // DevConsts::q2r_fold
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const { return PtrRow{base + ((size_t)row << logn)}; }
    __device__ __forceinline__ const tw_t* fold(int row) const { return fold_base + 2 * (row % nq); }
};

// rows of consecutive Q|R polynomials; limb l of Q|R uses prime l (Q) or idx_r + l - nq (R)
struct QRRowsIO {
    uint64_t* base;
    int logn, nq, nqr, idx_r;
    __device__ __forceinline__ int prime(int row) const {
        const int l = row % nqr;
        return l < nq ? l : idx_r + (l - nq);
    }
    __device__ __forceinline__ PtrRow bind(int row) const { return PtrRow{base + ((size_t)row << logn)}; }
};

// K4 source: tensor product of the pair at limb l of Q|R, one of three outputs
struct TensorRow {
    const uint64_t *a1, *b1, *a2, *b2;
    int k;
    uint64_t q, mh, ml;  // mh: barrett_prod constant (inputs are fully reduced)
    __device__ __forceinline__ uint64_t load(int j) const {
        if (k == 0) return mul_mod_prod(a1[j], a2[j], q, mh);
        if (k == 2) return mul_mod_prod(b1[j], b2[j], q, mh);
        u128 acc = mul_wide(a1[j], b2[j]);
        mac(acc, b1[j], a2[j]);  // < 2 q^2
        return barrett_prod(acc, q, mh);
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct TensorSrc {
    PtrBatch pb;
    const uint64_t* sb;  // NTT-form R limbs: [item][4][nr]
    DevConsts dc;
    __device__ __forceinline__ int prime(int row) const {
        const int l = row % dc.nqr;
        return l < dc.nq ? l : dc.idx_r + (l - dc.nq);
    }
    __device__ __forceinline__ TensorRow bind(int row) const {
        const int nqr = dc.nqr, nq = dc.nq, nr = dc.nr, logn = dc.logn;
        const int item = row / (3 * nqr), w = row % (3 * nqr), k = w / nqr, l = w % nqr;
        TensorRow t;
        t.k = k;
        const int pi = l < nq ? l : dc.idx_r + (l - nq);
        t.q = dc.mods[pi]; t.mh = dc.mu_prod[pi]; t.ml = 0;
        if (l < nq) {
            const uint64_t* A = pb.a[item];
            const uint64_t* B = pb.b[item];
            t.a1 = A + ((size_t)l << logn); t.b1 = A + ((size_t)(nq + l) << logn);
            t.a2 = B + ((size_t)l << logn); t.b2 = B + ((size_t)(nq + l) << logn);
        } else {
            const int r = l - nq;
            const uint64_t* base = sb + (((size_t)item * 4 * nr) << logn);
            t.a1 = base + ((size_t)(0 * nr + r) << logn); t.b1 = base + ((size_t)(1 * nr + r) << logn);
            t.a2 = base + ((size_t)(2 * nr + r) << logn); t.b2 = base + ((size_t)(3 * nr + r) << logn);
        }
        return t;
    }
};

// K6b source: inner product with the relinearisation key over Q|P
struct KeyIPRow {
    const uint64_t* dig;  // limb m of digit 0 (digit stride ds)
    const uint64_t* key;  // limb m, half h of digit 0 (digit stride ks)
    size_t ds, ks;
    int dnum;
    uint64_t q, mh, ml, mp;
    __device__ __forceinline__ uint64_t load(int j) const {
        if (dnum == 1) return mul_mod_prod(dig[j], key[j], q, mp);  // digits fully reduced
        u128 acc{0, 0};
        for (int d = 0; d < dnum; d++) mac(acc, dig[d * ds + j], key[d * ks + j]);
        return barrett128(acc, q, mh, ml);
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct KeyIPSrc {
    const uint64_t* sd2;  // [item][ndig][npq]
    const uint64_t* rlk;  // [ndig][2][npq]
    DevConsts dc;
    int ndig;             // digits: dnum (hybrid) or q_count * pieces (gadget)
    int m0 = 0, nm = 0;   // rows cover limbs m0 .. m0+nm-1 of Q|P (nm = 0: all of Q|P)
    __device__ __forceinline__ int prime(int row) const { return m0 + row % (nm ? nm : dc.npq); }
    __device__ __forceinline__ KeyIPRow bind(int row) const {
        const int npq = dc.npq, logn = dc.logn, per = nm ? nm : npq;
        const int item = row / (2 * per), w = row % (2 * per), h = w / per, m = m0 + w % per;
        KeyIPRow r;
        r.dig = sd2 + (((size_t)item * ndig * npq + m) << logn);
        // key limbs: [digit][a|b][Q|P] of the top level; a level reads its live Q limbs and P
        const int km = m < dc.nq ? m : dc.key_nq + (m - dc.nq);
        r.key = rlk + (((size_t)h * dc.key_npq + km) << logn);
        r.ds = (size_t)npq << logn;
        r.ks = (size_t)2 * dc.key_npq << logn;
        r.dnum = ndig;
        r.q = dc.mods[m]; r.mh = dc.mu_hi[m]; r.ml = dc.mu_lo[m]; r.mp = dc.mu_prod[m];
        return r;
    }
};

// Gadget decomposition source: rows (item, digit g = i*J + j, m) -> the j-th
// w-bit piece of limb i of a1*a2 (coefficient form), the same small integer in
// every prime m of Q|P.
struct GadgetRow {
    const uint64_t* x;
    int shift;
    uint64_t mask;
    __device__ __forceinline__ uint64_t load(int j) const { return (x[j] >> shift) & mask; }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct GadgetDigitSrc {
    const uint64_t* sd2;  // [item][nq]
    DevConsts dc;
    int pieces, w;
    __device__ __forceinline__ int prime(int row) const { return row % dc.npq; }
    __device__ __forceinline__ GadgetRow bind(int row) const {
        const int ndig = dc.nq * pieces;
        const int item = row / (ndig * dc.npq), g = (row / dc.npq) % ndig;
        GadgetRow r;
        r.x = sd2 + (((size_t)item * dc.nq + g / pieces) << dc.logn);
        r.shift = w * (g % pieces);
        r.mask = (w >= 64) ? ~0ULL : (((uint64_t)1 << w) - 1);
        return r;
    }
};

// K7 source: mod down P|Q -> q_l and add the tensor term (coefficient form)
struct ModDownAddRow {
    const uint64_t* x;    // limb l of the Q|P polynomial, or null (Q part added in the NTT domain)
    const uint64_t* xp;   // limb 0 of its P part
    const uint64_t* add;  // limb l of the term to add, or null
    const uint64_t* pmods;
    const uint64_t* phatinv;
    const uint64_t* phatinvs;
    const uint64_t* phat;  // row l of (P/p_k) mod q_l
    size_t limb;
    int np;
    uint64_t q, mh, ml, pinv, pinvs;
    __device__ __forceinline__ uint64_t load(int j) const {
        uint64_t conv;
        if (np == 1) {
            conv = barrett64(xp[j], q, mh);
        } else {
            u128 acc{0, 0};
            for (int kk = 0; kk < np; kk++) {
                uint64_t rb = shoup(xp[kk * limb + j], phatinv[kk], phatinvs[kk], pmods[kk]);
                mac(acc, rb, phat[kk]);
            }
            conv = barrett128(acc, q, mh, ml);
        }
        uint64_t v = shoup(q - conv + (x ? x[j] : 0), pinv, pinvs, q);
        if (add) v = add_mod(v, add[j], q);
        return v;
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct ModDownAddSrc {
    const uint64_t* se;   // [item][2][npq]
    const uint64_t* sd;   // [item][2][nq] or null
    DevConsts dc;
    bool p_only = false;  // se holds only the P limbs (OutCtKeyDst adds the Q part)
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ ModDownAddRow bind(int row) const {
        const int nq = dc.nq, npq = dc.npq, logn = dc.logn;
        const int item = row / (2 * nq), w = row % (2 * nq), h = w / nq, l = w % nq;
        ModDownAddRow r;
        const uint64_t* poly = se + (((size_t)item * 2 + h) * npq << logn);
        r.x = p_only ? nullptr : poly + ((size_t)l << logn);
        r.xp = poly + ((size_t)nq << logn);
        r.add = sd ? sd + (((size_t)(item * 2 + h) * nq + l) << logn) : nullptr;
        r.pmods = dc.mods + dc.idx_p;
        r.phatinv = dc.phatinv_p;
        r.phatinvs = dc.phatinv_ps;
        r.phat = dc.phat_mod_q + (size_t)l * dc.np;
        r.limb = (size_t)1 << logn;
        r.np = dc.np;
        r.q = dc.mods[l]; r.mh = dc.mu_hi[l]; r.ml = dc.mu_lo[l];
        r.pinv = dc.pinv_q[l]; r.pinvs = dc.pinv_qs[l];
        return r;
    }
};

// ModDownAddSrc for one special prime: [x_P]_q is x_P mod q, so the row needs
// no conversion tables (fewer live registers in the transform's first pass)
struct ModDownAdd1Row {
    const uint64_t* x;    // limb l of the Q|P polynomial, or null
    const uint64_t* xp;   // its P limb
    const uint64_t* add;  // limb l of the term to add, or null
    uint64_t q, mh, pinv, pinvs;
    __device__ __forceinline__ uint64_t load(int j) const {
        const uint64_t conv = barrett64(xp[j], q, mh);
        uint64_t v = shoup(q - conv + (x ? x[j] : 0), pinv, pinvs, q);
        if (add) v = add_mod(v, add[j], q);
        return v;
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct ModDownAdd1Src {
    const uint64_t* se;   // [item][2][npq]
    const uint64_t* sd;   // [item][2][nq] or null
    DevConsts dc;
    bool p_only = false;
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ ModDownAdd1Row bind(int row) const {
        const int nq = dc.nq, npq = dc.npq, logn = dc.logn;
        const int item = row / (2 * nq), w = row % (2 * nq), h = w / nq, l = w % nq;
        const uint64_t* poly = se + (((size_t)item * 2 + h) * npq << logn);
        ModDownAdd1Row r;
        r.x = p_only ? nullptr : poly + ((size_t)l << logn);
        r.xp = poly + ((size_t)nq << logn);
        r.add = sd ? sd + (((size_t)(item * 2 + h) * nq + l) << logn) : nullptr;
        r.q = dc.mods[l]; r.mh = dc.mu_hi[l];
        r.pinv = dc.pinv_q[l]; r.pinvs = dc.pinv_qs[l];
        return r;
    }
};

struct OutCtDst {  // rows: (item, h, l) -> out[item] + (h*nq + l)*N
    PtrBatch pb;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const int item = row / (2 * nq), w = row % (2 * nq);
        return PtrRow{pb.o[item] + ((size_t)w << logn)};
    }
};

// rows (item, h, k) -> limb nq + k (P part) of se ([item][2][npq])
struct SeRowsP {
    uint64_t* se;
    int logn, nq, np, npq;
    __device__ __forceinline__ int prime(int row) const { return nq + row % np; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const int item = row / (2 * np), w = row % (2 * np), h = w / np, k = w % np;
        return PtrRow{se + (((size_t)(item * 2 + h) * npq + nq + k) << logn)};
    }
};

// Output store of the key-switch tail: adds P^-1 * sum_d digit_d * key_d[h] at
// limb l of Q (all NTT form, fully reduced) to the transformed value.
struct OutKeyRow {
    uint64_t* p;
    const uint64_t* dig;  // limb l of digit 0, digit stride ds
    const uint64_t* key;  // limb l of half h of digit 0, digit stride ks
    size_t ds, ks;
    int ndig;
    uint64_t q, mh, ml, mp, pinv, pinvs;
    __device__ __forceinline__ uint64_t load(int j) const { return p[j]; }
    __device__ __forceinline__ void store(int j, uint64_t v) const {
        uint64_t ip;
        if (ndig == 1) {
            ip = mul_mod_prod(dig[j], key[j], q, mp);
        } else {
            u128 acc{0, 0};
            for (int d = 0; d < ndig; d++) mac(acc, dig[d * ds + j], key[d * ks + j]);
            ip = barrett128(acc, q, mh, ml);
        }
        p[j] = add_mod(v, shoup(ip, pinv, pinvs, q), q);
    }
};
struct OutCtKeyDst {  // rows: (item, h, l) -> out[item] + (h*nq + l)*N
    PtrBatch pb;
    const uint64_t* sd2;  // NTT-form digits [item][ndig][npq]
    const uint64_t* rlk;  // [ndig][2][Q|P] of the top level
    DevConsts dc;
    int ndig;
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ OutKeyRow bind(int row) const {
        const int nq = dc.nq, logn = dc.logn;
        const int item = row / (2 * nq), w = row % (2 * nq), h = w / nq, l = w % nq;
        OutKeyRow r;
        r.p = pb.o[item] + ((size_t)w << logn);
        r.dig = sd2 + (((size_t)item * ndig * dc.npq + l) << logn);
        r.key = rlk + (((size_t)h * dc.key_npq + l) << logn);
        r.ds = (size_t)dc.npq << logn;
        r.ks = (size_t)2 * dc.key_npq << logn;
        r.ndig = ndig;
        r.q = dc.mods[l]; r.mh = dc.mu_hi[l]; r.ml = dc.mu_lo[l]; r.mp = dc.mu_prod[l];
        r.pinv = dc.pinv_q[l]; r.pinvs = dc.pinv_qs[l];
        return r;
    }
};
// the column pass of a split transform writes plain values; only the block
// kernel's final store runs the epilogue
static inline OutCtDst plain_of(const OutCtKeyDst& d) { return OutCtDst{d.pb, d.dc.logn, d.dc.nq}; }

// rows (item, limb) of the first polynomial of consecutive 3-polynomial tensors
struct TensorA2 {
    const uint64_t* tz;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const int item = row / nq, l = row % nq;
        return PtrRow{const_cast<uint64_t*>(tz) + (((size_t)item * 3 * nq + l) << logn)};
    }
};

// decrypt: INTT over Q of (a*s + b), then the rounding
struct DecSrc {
    const uint64_t* ct;
    const uint64_t* sk;
    DevConsts dc;
    struct Row {
        const uint64_t *a, *b, *s;
        uint64_t q, mh, ml;
        // a and s fully reduced: one-high-product Barrett (mh holds its constant)
        __device__ __forceinline__ uint64_t load(int j) const { return add_mod(mul_mod_prod(a[j], s[j], q, mh), b[j], q); }
        __device__ __forceinline__ void store(int, uint64_t) const {}
    };
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ Row bind(int row) const {
        const int item = row / dc.nq, l = row % dc.nq;
        const size_t lq = (size_t)dc.nq << dc.logn;
        Row r;
        r.a = ct + item * 2 * lq + ((size_t)l << dc.logn);
        r.b = r.a + lq;
        r.s = sk + ((size_t)l << dc.logn);
        r.q = dc.mods[l]; r.mh = dc.mu_prod[l]; r.ml = 0;
        return r;
    }
};


// INTT over Q of the four input polynomials, Q -> R, NTT over R, fused tensor +
// INTT over Q|R: steps shared by kbfv_mul and the fused multiply-relinearise.
void mul_front(const DevConsts& dc, const PtrBatch& pb, int count, const MulScratch& m, cudaStream_t st);
// K5: scale-and-round, R -> Q and (mode 1) the key-switch digit lift
template <int MAXQ>
void k5_launch_m(const DevConsts& dc, int count, const MulScratch& m, uint64_t* out0, int mode, cudaStream_t st);
// K3 with the Q -> R base extension in its loader: `polys` polynomials of y
// rows over Q (QHatRowsIO layout) -> NTT-form R limbs, fully reduced
template <int MAXQ>
void q2r_ntt_launch_m(const DevConsts& dc, const uint64_t* y, uint64_t* out, int polys, cudaStream_t st);
void k5_launch(const DevConsts& dc, int count, const MulScratch& m, uint64_t* out0, int mode, cudaStream_t st);
// key-switch tail: key product, mod down and add, written to the outputs of pb
void ks_tail(const DevConsts& dc, const uint64_t* sd2, const uint64_t* key, int ndig, uint64_t* se,
             const uint64_t* add, const PtrBatch& pb, int count, cudaStream_t st);
// the auxiliary streams and fork / join events of the sub-batches (created once)
void ensure_branch_streams(Context& c);
// the whole multiply + relinearise of one sub-batch (9 launches)
void mul_relin_chunk(const DevConsts& dc, const uint64_t* rlk, const PtrBatch& pb, int count, const MulScratch& m,
                     cudaStream_t st);
// The constants with the launch shapes of a multiply that runs as one stream
// (no sibling sub-batch on another stream to fill the SMs): 2^14-point
// transforms of up to shape.split_rows_alone rows run split.
static inline DevConsts alone_consts(const Context& c) {
    DevConsts d = c.dc;
    d.shape.split_rows14 = d.shape.split_rows_alone;
    return d;
}
