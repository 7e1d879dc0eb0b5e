// Mixed-level batches: ciphertext pairs at different levels (numbers of live
// ciphertext primes) multiplied and relinearised by ONE launch sequence of the
// pipeline (the reference's key switch has a batch axis for this,
// include/BasisConv.cuh:73, but no levels).
//
// The pairs are ordered by level on the host and split into level groups. A
// row of any pipeline stage locates its group, item and local row from the
// stage's per-group row starts (at most kMaxGroups comparisons); its constants
// (moduli, Barrett and base-extension tables, twiddles) come from its level's
// DevConsts, which the top-level context keeps in device memory (one slot per
// level). Scratch keeps the top level's per-item layout, so every item's region
// holds its own level's limbs. Each level's arithmetic is the level context's
// own, so the products are bit-identical to multiplying each group on its own
// level context.
#pragma once
#include "pipeline.cuh"

constexpr int kMaxGroups = 8;

// x / d and x % d for x * d < 2^32 from m = ceil(2^32 / d): floor(x * m / 2^32)
// exceeds x / d by less than x / 2^32 < 1 / d, which never reaches the next
// integer (the column passes locate their row per thread; a hardware-free
// division there would cost as much as the butterflies).
struct FastDiv {
    uint32_t d;
    uint64_t m;
    __host__ __device__ __forceinline__ uint32_t div(uint32_t x) const { return (uint32_t)((x * m) >> 32); }
    __host__ __device__ __forceinline__ uint32_t mod(uint32_t x) const { return x - div(x) * d; }
};
inline FastDiv fast_div(uint32_t d) { return FastDiv{d, (((uint64_t)1 << 32) + d - 1) / d}; }

struct Groups {
    int ng;                                   // level groups in this launch
    int first[kMaxGroups + 1];                // items of group g: [first[g], first[g+1])
    int nq[kMaxGroups], nr[kMaxGroups], npq[kMaxGroups], nqr[kMaxGroups], dnum[kMaxGroups];
    FastDiv dq[kMaxGroups], dr[kMaxGroups], dpq[kMaxGroups], dqr[kMaxGroups];  // division by nq, nr, npq, nqr
    FastDiv dp;                               // division by np
    const DevConsts* lv[kMaxGroups];          // the group's level constants (device memory)
    int logn, np;
    int top_nq, top_nr, top_npq, top_nqr, top_dnum;  // scratch layout per item (top level's)
    int key_nq, key_npq;                      // limb layout of the top-level key
    __device__ __forceinline__ int group_of_item(int item) const {
        int g = 0;
        while (g + 1 < ng && item >= first[g + 1]) g++;
        return g;
    }
};

// rows of one pipeline stage: group g's rows start at start[g], per[g] rows per item
struct StageRows {
    int start[kMaxGroups + 1];
    FastDiv per[kMaxGroups];
};

struct RowLoc {
    int g, item, local;
};

__device__ __forceinline__ RowLoc locate(const Groups& G, const StageRows& R, int row) {
    int g = 0;
    while (g + 1 < G.ng && row >= R.start[g + 1]) g++;
    const uint32_t rel = (uint32_t)(row - R.start[g]);
    const uint32_t q = R.per[g].div(rel);
    return RowLoc{g, G.first[g] + (int)q, (int)(rel - q * R.per[g].d)};
}

// twiddle table and modulus of prime `p` of a level's own prime table
__device__ __forceinline__ RowTab level_tab(const DevConsts* lv, int p, bool inverse, int logn) {
    return RowTab{(inverse ? lv->tw_inv : lv->tw_fwd) + ((size_t)p << logn), lv->mods[p]};
}

// Scratch rows with the top level's per-item stride, the item's rows packed by
// its own level. kind: 0 Q limbs of consecutive polynomials; 1 R limbs; 2 Q|P
// limbs (digits of the key switch); 3 Q|R limbs (tensor outputs).
struct MixedRows {
    uint64_t* base;
    size_t item_limbs;
    Groups G;
    StageRows R;
    int kind;
    __device__ __forceinline__ int prime_of(const RowLoc& L) const {
        const int g = L.g;
        switch (kind) {
            case 0: return (int)G.dq[g].mod(L.local);
            case 1: return G.nq[g] + G.np + (int)G.dr[g].mod(L.local);
            case 2: return (int)G.dpq[g].mod(L.local);
            default: {
                const int l = (int)G.dqr[g].mod(L.local);
                return l < G.nq[g] ? l : G.nq[g] + G.np + (l - G.nq[g]);
            }
        }
    }
    __device__ __forceinline__ int prime(int row) const { return prime_of(locate(G, R, row)); }
    __device__ __forceinline__ RowTab tables(int row, bool inverse) const {
        const RowLoc L = locate(G, R, row);
        return level_tab(G.lv[L.g], prime_of(L), inverse, G.logn);
    }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const RowLoc L = locate(G, R, row);
        return PtrRow{base + (((size_t)L.item * item_limbs + L.local) << G.logn)};
    }
};

// K1 source: the Q limbs of [a1, b1, a2, b2] of each pair, in the pair's own
// layout ([a | b], its level's live primes each)
struct MixedPairQRows {
    PtrBatch pb;
    Groups G;
    StageRows R;
    __device__ __forceinline__ int prime(int row) const {
        const RowLoc L = locate(G, R, row);
        return (int)G.dq[L.g].mod(L.local);
    }
    __device__ __forceinline__ RowTab tables(int row, bool inverse) const {
        const RowLoc L = locate(G, R, row);
        return level_tab(G.lv[L.g], (int)G.dq[L.g].mod(L.local), inverse, G.logn);
    }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const RowLoc L = locate(G, R, row);
        const int nq = G.nq[L.g], p = (int)G.dq[L.g].div(L.local), l = L.local - p * nq;
        const uint64_t* base = p < 2 ? pb.a[L.item] : pb.b[L.item];
        return PtrRow{const_cast<uint64_t*>(base) + (((size_t)(p & 1) * nq + l) << G.logn)};
    }
};

// K4 source: the tensor product at limb l of Q|R (see TensorSrc)
struct MixedTensorSrc {
    PtrBatch pb;
    const uint64_t* sb;  // NTT-form R limbs: item region of 4 x top_nr limbs, [4][nr] packed
    Groups G;
    StageRows R;
    __device__ __forceinline__ int prime_of(const RowLoc& L) const {
        const int l = (int)G.dqr[L.g].mod(L.local);
        return l < G.nq[L.g] ? l : G.nq[L.g] + G.np + (l - G.nq[L.g]);
    }
    __device__ __forceinline__ int prime(int row) const { return prime_of(locate(G, R, row)); }
    __device__ __forceinline__ RowTab tables(int row, bool inverse) const {
        const RowLoc L = locate(G, R, row);
        return level_tab(G.lv[L.g], prime_of(L), inverse, G.logn);
    }
    __device__ __forceinline__ TensorRow bind(int row) const {
        const RowLoc L = locate(G, R, row);
        const int g = L.g, nq = G.nq[g], nr = G.nr[g], nqr = G.nqr[g], logn = G.logn;
        const int k = (int)G.dqr[g].div(L.local), l = L.local - k * nqr;
        const DevConsts* lv = G.lv[g];
        const int pi = prime_of(L);
        TensorRow t;
        t.k = k;
        t.q = lv->mods[pi];
        t.mh = lv->mu_prod[pi];
        t.ml = 0;
        if (l < nq) {
            const uint64_t* A = pb.a[L.item];
            const uint64_t* B = pb.b[L.item];
            t.a1 = A + ((size_t)l << logn); t.b1 = A + ((size_t)(nq + l) << logn);
            t.a2 = B + ((size_t)l << logn); t.b2 = B + ((size_t)(nq + l) << logn);
        } else {
            const int r = l - nq;
            const uint64_t* base = sb + (((size_t)L.item * 4 * G.top_nr) << logn);
            t.a1 = base + ((size_t)(0 * nr + r) << logn); t.b1 = base + ((size_t)(1 * nr + r) << logn);
            t.a2 = base + ((size_t)(2 * nr + r) << logn); t.b2 = base + ((size_t)(3 * nr + r) << logn);
        }
        return t;
    }
};

// K6b source: inner product of the digits with the top-level key over P (see KeyIPSrc)
struct MixedKeyIPSrc {
    const uint64_t* sd2;  // item region of top_dnum x top_npq limbs, [dnum][npq] packed
    const uint64_t* rlk;  // [digit][a|b][Q|P] of the top level
    Groups G;
    StageRows R;          // 2 x np rows per item
    __device__ __forceinline__ int limb(const RowLoc& L) const { return G.nq[L.g] + (int)G.dp.mod(L.local); }
    __device__ __forceinline__ int prime(int row) const { return limb(locate(G, R, row)); }
    __device__ __forceinline__ RowTab tables(int row, bool inverse) const {
        const RowLoc L = locate(G, R, row);
        return level_tab(G.lv[L.g], limb(L), inverse, G.logn);
    }
    __device__ __forceinline__ KeyIPRow bind(int row) const {
        const RowLoc L = locate(G, R, row);
        const int g = L.g, logn = G.logn, h = (int)G.dp.div(L.local), k = L.local - h * G.np, m = G.nq[g] + k;
        const DevConsts* lv = G.lv[g];
        KeyIPRow r;
        r.dig = sd2 + (((size_t)L.item * G.top_dnum * G.top_npq + m) << logn);
        r.key = rlk + (((size_t)h * G.key_npq + G.key_nq + k) << logn);
        r.ds = (size_t)G.npq[g] << logn;
        r.ks = (size_t)2 * G.key_npq << logn;
        r.dnum = G.dnum[g];
        r.q = lv->mods[m]; r.mh = lv->mu_hi[m]; r.ml = lv->mu_lo[m]; r.mp = lv->mu_prod[m];
        return r;
    }
};

// K6b destination: the P limbs of se (item region of 2 x top_npq limbs, [2][npq] packed)
struct MixedSeRowsP {
    uint64_t* se;
    Groups G;
    StageRows R;
    __device__ __forceinline__ int limb(const RowLoc& L) const { return G.nq[L.g] + (int)G.dp.mod(L.local); }
    __device__ __forceinline__ int prime(int row) const { return limb(locate(G, R, row)); }
    __device__ __forceinline__ RowTab tables(int row, bool inverse) const {
        const RowLoc L = locate(G, R, row);
        return level_tab(G.lv[L.g], limb(L), inverse, G.logn);
    }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const RowLoc L = locate(G, R, row);
        const int h = (int)G.dp.div(L.local);
        return PtrRow{se + (((size_t)L.item * 2 * G.top_npq + h * G.npq[L.g] + limb(L)) << G.logn)};
    }
};

// K7 source: mod down of the P part and the add term (see ModDownAdd1Src /
// ModDownAddSrc); rows (item, h, l), 2 x nq rows per item
template <bool ONE_P>
struct MixedModDownSrc {
    const uint64_t* se;
    const uint64_t* sd;  // item region of 2 x top_nq limbs, [2][nq] packed
    Groups G;
    StageRows R;
    __device__ __forceinline__ int prime(int row) const {
        const RowLoc L = locate(G, R, row);
        return (int)G.dq[L.g].mod(L.local);
    }
    __device__ __forceinline__ RowTab tables(int row, bool inverse) const {
        const RowLoc L = locate(G, R, row);
        return level_tab(G.lv[L.g], (int)G.dq[L.g].mod(L.local), inverse, G.logn);
    }
    __device__ __forceinline__ auto bind(int row) const {
        const RowLoc L = locate(G, R, row);
        const int g = L.g, nq = G.nq[g], logn = G.logn, h = (int)G.dq[g].div(L.local), l = L.local - h * nq;
        const DevConsts* lv = G.lv[g];
        const uint64_t* poly = se + (((size_t)L.item * 2 * G.top_npq + (size_t)h * G.npq[g]) << logn);
        const uint64_t* add = sd + (((size_t)L.item * 2 * G.top_nq + (size_t)h * nq + l) << logn);
        if constexpr (ONE_P) {
            ModDownAdd1Row r;
            r.x = nullptr;  // the Q part is added in the NTT domain at K7's store
            r.xp = poly + ((size_t)nq << logn);
            r.add = add;
            r.q = lv->mods[l]; r.mh = lv->mu_hi[l];
            r.pinv = lv->pinv_q[l]; r.pinvs = lv->pinv_qs[l];
            return r;
        } else {
            ModDownAddRow r;
            r.x = nullptr;
            r.xp = poly + ((size_t)nq << logn);
            r.add = add;
            r.pmods = lv->mods + lv->idx_p;
            r.phatinv = lv->phatinv_p;
            r.phatinvs = lv->phatinv_ps;
            r.phat = lv->phat_mod_q + (size_t)l * lv->np;
            r.limb = (size_t)1 << logn;
            r.np = lv->np;
            r.q = lv->mods[l]; r.mh = lv->mu_hi[l]; r.ml = lv->mu_lo[l];
            r.pinv = lv->pinv_q[l]; r.pinvs = lv->pinv_qs[l];
            return r;
        }
    }
};

// K7's plain rows: out[item] + (h * nq + l) * N (the column pass of a split transform)
struct MixedOutCtDst {
    PtrBatch pb;
    Groups G;
    StageRows R;
    __device__ __forceinline__ int prime(int row) const {
        const RowLoc L = locate(G, R, row);
        return (int)G.dq[L.g].mod(L.local);
    }
    __device__ __forceinline__ RowTab tables(int row, bool inverse) const {
        const RowLoc L = locate(G, R, row);
        return level_tab(G.lv[L.g], (int)G.dq[L.g].mod(L.local), inverse, G.logn);
    }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const RowLoc L = locate(G, R, row);
        return PtrRow{pb.o[L.item] + ((size_t)L.local << G.logn)};
    }
};

// K7 destination: the output ciphertexts, the key product over Q times P^-1
// added at the store (see OutCtKeyDst)
struct MixedOutCtKeyDst {
    PtrBatch pb;
    const uint64_t* sd2;
    const uint64_t* rlk;
    Groups G;
    StageRows R;
    __device__ __forceinline__ int prime(int row) const {
        const RowLoc L = locate(G, R, row);
        return (int)G.dq[L.g].mod(L.local);
    }
    __device__ __forceinline__ RowTab tables(int row, bool inverse) const {
        const RowLoc L = locate(G, R, row);
        return level_tab(G.lv[L.g], (int)G.dq[L.g].mod(L.local), inverse, G.logn);
    }
    __device__ __forceinline__ OutKeyRow bind(int row) const {
        const RowLoc L = locate(G, R, row);
        const int g = L.g, nq = G.nq[g], logn = G.logn, h = (int)G.dq[g].div(L.local), l = L.local - h * nq;
        const DevConsts* lv = G.lv[g];
        OutKeyRow r;
        r.p = pb.o[L.item] + ((size_t)L.local << logn);
        r.dig = sd2 + (((size_t)L.item * G.top_dnum * G.top_npq + l) << logn);
        r.key = rlk + (((size_t)h * G.key_npq + l) << logn);
        r.ds = (size_t)G.npq[g] << logn;
        r.ks = (size_t)2 * G.key_npq << logn;
        r.ndig = G.dnum[g];
        r.q = lv->mods[l]; r.mh = lv->mu_hi[l]; r.ml = lv->mu_lo[l]; r.mp = lv->mu_prod[l];
        r.pinv = lv->pinv_q[l]; r.pinvs = lv->pinv_qs[l];
        return r;
    }
};
static inline MixedOutCtDst plain_of(const MixedOutCtKeyDst& d) { return MixedOutCtDst{d.pb, d.G, d.R}; }

// K2 and K5 of a mixed batch (instantiated per MAXQ bucket in k5_m<MAXQ>.cu)
template <int MAXQ>
void bconv_mixed_launch_m(const Groups& G, const LaunchShape& sh, int count, const MulScratch& m, cudaStream_t st);
template <int MAXQ>
void k5_mixed_launch_m(const Groups& G, const LaunchShape& sh, int count, const MulScratch& m, cudaStream_t st);

// The level constants of item `item` copied into shared memory by the CTA (one
// item per CTA row of the per-coefficient kernels), so that the kernels' reads
// of them cannot alias their global stores.
__device__ __forceinline__ void load_level_consts(DevConsts& dst, const DevConsts* src) {
    static_assert(sizeof(DevConsts) % 8 == 0, "DevConsts copies as 8-byte words");
    const uint64_t* s = reinterpret_cast<const uint64_t*>(src);
    uint64_t* d = reinterpret_cast<uint64_t*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(DevConsts) / 8); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

// K2 over a mixed batch: Q -> R of [a1, b1, a2, b2] per item (grid.y = item x 4)
template <int MAXIN>
static __global__ void bconv_mixed_kernel(Groups G, const uint64_t* __restrict__ sa, uint64_t* __restrict__ sb) {
    __shared__ DevConsts c;
    extern __shared__ uint64_t sh_hat[];
    const int item = blockIdx.y / 4, p = blockIdx.y % 4, g = G.group_of_item(item);
    load_level_consts(c, G.lv[g]);
    const BconvTables tb = q2r_tables(c);
    for (int i = threadIdx.x; i < tb.nin * tb.nout; i += blockDim.x) sh_hat[i] = tb.hat[i];
    __syncthreads();
    const int logn = G.logn;
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = sa + (((size_t)item * 4 * G.top_nq + (size_t)p * tb.nin) << logn);
    uint64_t* dst = sb + (((size_t)item * 4 * G.top_nr + (size_t)p * tb.nout) << logn);
    uint64_t x[MAXIN], y[MAXIN];
#pragma unroll
    for (int i = 0; i < MAXIN; i++)
        if (i < tb.nin) x[i] = src[((size_t)i << logn) + k];
    const long long v = bconv_prep<MAXIN>(y, x, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
    for (int j = 0; j < tb.nout; j++)
        dst[((size_t)j << logn) + k] = bconv_out<MAXIN>(y, tb.nin, sh_hat + j * tb.nin, tb.alpha[v * tb.nout + j],
                                                        tb.out_mods[j], tb.out_mu_hi[j], tb.out_mu_lo[j]);
}
