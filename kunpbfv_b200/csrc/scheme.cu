// libkbfv: randomness (XSalsa20 sub-keys and samplers), key generation,
// encoding, encryption, decryption and the linear and plaintext operations.
#include "pipeline.cuh"

// ---- randomness helpers ----
static void hsalsa_host(const uint8_t key[32], const uint8_t nonce16[16], uint32_t out[8]);
static SalsaKey subkey_for(const uint8_t seed[32], uint32_t domain, uint32_t sub) {
    uint8_t n16[16] = {0};
    for (int i = 0; i < 4; i++) { n16[i] = (uint8_t)(domain >> (8 * i)); n16[4 + i] = (uint8_t)(sub >> (8 * i)); }
    SalsaKey k;
    hsalsa_host(seed, n16, k.k);
    static const char* sig = "expand 32-byte k";
    for (int i = 0; i < 4; i++) std::memcpy(&k.sigma[i], sig + 4 * i, 4);
    return k;
}

static inline uint32_t rl(uint32_t u, int c) { return (u << c) | (u >> (32 - c)); }
static inline uint32_t ld32(const uint8_t* x) {
    return (uint32_t)x[0] | ((uint32_t)x[1] << 8) | ((uint32_t)x[2] << 16) | ((uint32_t)x[3] << 24);
}
static void hsalsa_host(const uint8_t key[32], const uint8_t nonce16[16], uint32_t out[8]) {
    static const char* sig = "expand 32-byte k";
    uint32_t x[16];
    x[0] = ld32((const uint8_t*)sig); x[5] = ld32((const uint8_t*)sig + 4);
    x[10] = ld32((const uint8_t*)sig + 8); x[15] = ld32((const uint8_t*)sig + 12);
    for (int i = 0; i < 4; i++) { x[1 + i] = ld32(key + 4 * i); x[11 + i] = ld32(key + 16 + 4 * i); }
    for (int i = 0; i < 4; i++) x[6 + i] = ld32(nonce16 + 4 * i);
    for (int r = 0; r < 10; r++) {
        x[4] ^= rl(x[0] + x[12], 7);   x[8] ^= rl(x[4] + x[0], 9);
        x[12] ^= rl(x[8] + x[4], 13);  x[0] ^= rl(x[12] + x[8], 18);
        x[9] ^= rl(x[5] + x[1], 7);    x[13] ^= rl(x[9] + x[5], 9);
        x[1] ^= rl(x[13] + x[9], 13);  x[5] ^= rl(x[1] + x[13], 18);
        x[14] ^= rl(x[10] + x[6], 7);  x[2] ^= rl(x[14] + x[10], 9);
        x[6] ^= rl(x[2] + x[14], 13);  x[10] ^= rl(x[6] + x[2], 18);
        x[3] ^= rl(x[15] + x[11], 7);  x[7] ^= rl(x[3] + x[15], 9);
        x[11] ^= rl(x[7] + x[3], 13);  x[15] ^= rl(x[11] + x[7], 18);
        x[1] ^= rl(x[0] + x[3], 7);    x[2] ^= rl(x[1] + x[0], 9);
        x[3] ^= rl(x[2] + x[1], 13);   x[0] ^= rl(x[3] + x[2], 18);
        x[6] ^= rl(x[5] + x[4], 7);    x[7] ^= rl(x[6] + x[5], 9);
        x[4] ^= rl(x[7] + x[6], 13);   x[5] ^= rl(x[4] + x[7], 18);
        x[11] ^= rl(x[10] + x[9], 7);  x[8] ^= rl(x[11] + x[10], 9);
        x[9] ^= rl(x[8] + x[11], 13);  x[10] ^= rl(x[9] + x[8], 18);
        x[12] ^= rl(x[15] + x[14], 7); x[13] ^= rl(x[12] + x[15], 9);
        x[14] ^= rl(x[13] + x[12], 13); x[15] ^= rl(x[14] + x[13], 18);
    }
    out[0] = x[0]; out[1] = x[5]; out[2] = x[10]; out[3] = x[15];
    out[4] = x[6]; out[5] = x[7]; out[6] = x[8]; out[7] = x[9];
}

enum { DOM_SK = 1, DOM_PK_A = 2, DOM_PK_E = 3, DOM_RLK_A = 4, DOM_RLK_E = 5, DOM_ENC_V = 6, DOM_ENC_E0 = 7,
       DOM_ENC_E1 = 8, DOM_GK_A = 9, DOM_GK_E = 10, DOM_GAL_A = 11, DOM_GAL_E = 12 };

static void sample_small(Context& c, const uint8_t seed[32], uint32_t domain, uint64_t id0, int kind, int prime0,
                         int limbs, uint64_t* out, size_t item_stride, int items, cudaStream_t st) {
    SalsaKey k = subkey_for(seed, domain, 0);
    const int per = kind == 0 ? 16 : 8;
    const size_t total = (size_t)items * (c.n / per);
    if (kind == 0)
        sample_small_kernel<0><<<blocks_for(total, 128), 128, 0, st>>>(c.dc, k, id0, prime0, limbs, out, item_stride, items);
    else
        sample_small_kernel<1><<<blocks_for(total, 128), 128, 0, st>>>(c.dc, k, id0, prime0, limbs, out, item_stride, items);
    check_launch("sample_small");
}

static void sample_uniform(Context& c, const uint8_t seed[32], uint32_t domain, uint32_t sub, uint64_t id0, int prime0,
                           int limbs, uint64_t* out, size_t item_stride, int items, cudaStream_t st) {
    SalsaKey k = subkey_for(seed, domain, sub);
    const size_t total = (size_t)items * limbs * c.n / 4;
    sample_uniform_kernel<<<blocks_for(total, 128), 128, 0, st>>>(c.dc, k, id0, prime0, limbs, out, item_stride, items);
    check_launch("sample_uniform");
}

// ---- pointer-table variants of encryption, decryption and addition ----------
// delta * m of item i (plaintext pb.a[i]) into its work slot
__global__ void delta_m_ptr_kernel(DevConsts c, PtrBatch pb, uint64_t* __restrict__ work, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const size_t lq = (size_t)c.nq << c.logn;
    const size_t item = i / lq, w = i % lq;
    const int l = (int)(w >> c.logn);
    const uint64_t mv = pb.a[item][w & (((size_t)1 << c.logn) - 1)];
    const uint64_t mq = shoup(mv, c.negq_mod_t, c.negq_mod_t_s, c.t);
    work[item * 4 * lq + 3 * lq + w] = shoup(mq, c.tinv_q[l], c.tinv_qs[l], c.mods[l]);
}
__global__ void enc_combine_ptr_kernel(DevConsts c, const uint64_t* __restrict__ pk, const uint64_t* __restrict__ work,
                                       PtrBatch pb, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const size_t lq = (size_t)c.nq << c.logn;
    const size_t item = i / lq, w = i % lq;
    const int l = (int)(w >> c.logn);
    const uint64_t q = c.mods[l], mh = c.mu_hi[l], ml = c.mu_lo[l];
    const uint64_t* wk = work + item * 4 * lq;
    const uint64_t v = wk[w], e0 = wk[lq + w], e1 = wk[2 * lq + w], dm = wk[3 * lq + w];
    uint64_t* ct = pb.o[item];
    ct[w] = add_mod(mul_mod(v, pk[w], q, mh, ml), e0, q);
    ct[lq + w] = add_mod(add_mod(mul_mod(v, pk[lq + w], q, mh, ml), e1, q), dm, q);
}
// x = pb.a[item], y = pb.b[item], out = pb.o[item]: 2 x nq limbs each; grid.y = item
__global__ void add_ptr_kernel(DevConsts c, PtrBatch pb, size_t per_item) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= per_item) return;
    const int item = blockIdx.y;
    const int l = (int)((i >> c.logn) % c.nq);
    pb.o[item][i] = add_mod(pb.a[item][i], pb.b[item][i], c.mods[l]);
}
// decryption source with ciphertexts at pb.a[item]
struct DecSrcP {
    PtrBatch pb;
    const uint64_t* sk;
    DevConsts dc;
    struct Row {
        const uint64_t *a, *b, *s;
        uint64_t q, mp;
        __device__ __forceinline__ uint64_t load(int j) const { return add_mod(mul_mod_prod(a[j], s[j], q, mp), b[j], q); }
        __device__ __forceinline__ void store(int, uint64_t) const {}
    };
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ Row bind(int row) const {
        const int item = row / dc.nq, l = row % dc.nq;
        Row r;
        r.a = pb.a[item] + ((size_t)l << dc.logn);
        r.b = r.a + ((size_t)dc.nq << dc.logn);
        r.s = sk + ((size_t)l << dc.logn);
        r.q = dc.mods[l];
        r.mp = dc.mu_prod[l];
        return r;
    }
};
template <int MAXQ>
__global__ void decrypt_round_ptr_kernel(DevConsts c, const uint64_t* __restrict__ in, PtrBatch pb) {
    // the rounding of decrypt_round_kernel, written to pb.o[item]
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = in + ((size_t)blockIdx.y * c.nq << c.logn);
    pb.o[blockIdx.y][k] = decrypt_round_coeff<MAXQ>(c, src, k);
}

extern "C" {

int kbfv_keygen_secret(kbfv_context* ctx, const uint8_t seed[32], int secret_kind, uint32_t h, uint64_t* d_sk,
                       kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk, KBFV_ERR_INVALID, "null argument");
        const int npq = c.nq + c.np;
        cudaStream_t st = S(stream);
        if (secret_kind == 1) {
            KB_CHECK_CUDA(cudaMemsetAsync(d_sk, 0, (size_t)npq * c.n * 8, st));
            SalsaKey k = subkey_for(seed, DOM_SK, 0);
            sample_hwt_kernel<<<1, 32, 0, st>>>(c.dc, k, 0, (int)h, 0, npq, d_sk, 0, 1);
            check_launch("sample_hwt");
        } else {
            sample_small(c, seed, DOM_SK, 0, 0, 0, npq, d_sk, 0, 1, st);
        }
        RowsIO io = rows_io(c.dc, d_sk, 0, npq);
        ntt_fwd(c.dc, io, io, npq, st);
    });
}

int kbfv_keygen_public(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t* d_pk,
                       kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk && d_pk, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        uint64_t* a = d_pk;
        uint64_t* b = d_pk + lq;
        sample_uniform(c, seed, DOM_PK_A, 0, 0, 0, c.nq, a, 0, 1, st);
        sample_small(c, seed, DOM_PK_E, 0, 1, 0, c.nq, b, 0, 1, st);
        RowsIO io = rows_io(c.dc, b, 0, c.nq);
        ntt_fwd(c.dc, io, io, c.nq, st);
        pk_combine_kernel<<<blocks_for(lq, 256), 256, 0, st>>>(c.dc, a, d_sk, b, lq);
        check_launch("pk_combine");
    });
}

int kbfv_keygen_relin(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t* d_rlk,
                      kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk && d_rlk, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const int npq = c.nq + c.np;
        const size_t lpq = (size_t)npq * c.n;
        for (int d = 0; d < c.dnum; d++) {
            uint64_t* a = d_rlk + (size_t)d * 2 * lpq;
            uint64_t* b = a + lpq;
            sample_uniform(c, seed, DOM_RLK_A, (uint32_t)d, 0, 0, npq, a, 0, 1, st);
            SalsaKey k = subkey_for(seed, DOM_RLK_E, (uint32_t)d);
            const size_t total = c.n / 8;
            sample_small_kernel<1><<<blocks_for(total, 128), 128, 0, st>>>(c.dc, k, 0, 0, npq, b, 0, 1);
            check_launch("sample_gauss");
            RowsIO io = rows_io(c.dc, b, 0, npq);
            ntt_fwd(c.dc, io, io, npq, st);
            rlk_combine_kernel<<<blocks_for(lpq, 256), 256, 0, st>>>(c.dc, a, d_sk, b, d, lpq);
            check_launch("rlk_combine");
        }
    });
}

int kbfv_keygen_relin_gadget(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint32_t log_base,
                             uint64_t* d_gk, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk && d_gk, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(log_base >= 4 && log_base <= 30, KBFV_ERR_INVALID, "gadget base 2^w needs 4 <= w <= 30");
        const int w = (int)log_base, J = gadget_pieces(w);
        cudaStream_t st = S(stream);
        const int npq = c.nq + c.np;
        const size_t lpq = (size_t)npq * c.n;
        for (int i = 0; i < c.nq; i++) {
            uint64_t pm = 1;  // P mod q_i
            for (int k = 0; k < c.np; k++) pm = H::mulmod(pm, c.mods[c.nq + k] % c.mods[i], c.mods[i]);
            for (int j = 0; j < J; j++) {
                const uint32_t sub = (uint32_t)(i * J + j);
                uint64_t* a = d_gk + (size_t)sub * 2 * lpq;
                uint64_t* b = a + lpq;
                sample_uniform(c, seed, DOM_GK_A, sub, 0, 0, npq, a, 0, 1, st);
                SalsaKey k = subkey_for(seed, DOM_GK_E, sub);
                sample_small_kernel<1><<<blocks_for(c.n / 8, 128), 128, 0, st>>>(c.dc, k, 0, 0, npq, b, 0, 1);
                check_launch("sample_gauss");
                RowsIO io = rows_io(c.dc, b, 0, npq);
                ntt_fwd(c.dc, io, io, npq, st);
                const uint64_t g = H::mulmod(pm, H::powmod(2, (uint64_t)w * j, c.mods[i]), c.mods[i]);
                gk_combine_kernel<<<blocks_for(lpq, 256), 256, 0, st>>>(c.dc, a, d_sk, b, i, g, lpq);
                check_launch("gk_combine");
            }
        }
    });
}

int kbfv_encode(kbfv_context* ctx, const uint64_t* d_slots, uint64_t* d_m, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!count) return;
        if (d_m != d_slots)
            KB_CHECK_CUDA(cudaMemcpyAsync(d_m, d_slots, (size_t)count * c.n * 8, cudaMemcpyDeviceToDevice, S(stream)));
        RowsIO io = rows_io(c.dc, d_m, c.dc.idx_pt, 1);
        ntt_inv(c.dc, io, io, (int)count, S(stream));
    });
}

int kbfv_decode(kbfv_context* ctx, const uint64_t* d_m, uint64_t* d_slots, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!count) return;
        if (d_m != d_slots)
            KB_CHECK_CUDA(cudaMemcpyAsync(d_slots, d_m, (size_t)count * c.n * 8, cudaMemcpyDeviceToDevice, S(stream)));
        RowsIO io = rows_io(c.dc, d_slots, c.dc.idx_pt, 1);
        ntt_fwd(c.dc, io, io, (int)count, S(stream));
    });
}

// values (< t) as polynomial coefficients, replicated over Q and transformed
struct ReplicateSrc {
    const uint64_t* vals;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        return PtrRow{const_cast<uint64_t*>(vals) + ((size_t)(row / nq) << logn)};
    }
};

int kbfv_encode_ntt(kbfv_context* ctx, const uint64_t* d_vals, uint64_t* d_pt_ntt, uint32_t count,
                    kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!count) return;
        require_batchable(c);
        ntt_fwd(c.dc, ReplicateSrc{d_vals, c.logn, c.nq}, rows_io(c.dc, d_pt_ntt, 0, c.nq), (int)(count * c.nq),
                S(stream));
    });
}

int kbfv_encrypt(kbfv_context* ctx, const uint8_t seed[32], uint64_t enc_id, const uint64_t* d_pk, const uint64_t* d_m,
                 uint64_t* d_ct, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_pk && d_m && d_ct, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint64_t* work = (uint64_t*)ensure_scratch(c, (size_t)cnt * 4 * lq * 8);
            const uint64_t id0 = enc_id + off;
            // [v | e0 | e1 | dm] per item
            sample_small(c, seed, DOM_ENC_V, id0, 0, 0, c.nq, work, 4 * lq, cnt, st);
            sample_small(c, seed, DOM_ENC_E0, id0, 1, 0, c.nq, work + lq, 4 * lq, cnt, st);
            sample_small(c, seed, DOM_ENC_E1, id0, 1, 0, c.nq, work + 2 * lq, 4 * lq, cnt, st);
            for (int i = 0; i < cnt; i++) {
                const size_t tot = lq;
                delta_m_kernel<<<blocks_for(tot, 256), 256, 0, st>>>(c.dc, d_m + (size_t)(off + i) * c.n,
                                                                      work + (size_t)i * 4 * lq + 3 * lq, tot);
            }
            check_launch("delta_m");
            RowsIO io = rows_io(c.dc, work, 0, c.nq);
            ntt_fwd(c.dc, io, io, cnt * 4 * c.nq, st);
            const size_t total = (size_t)cnt * lq;
            enc_combine_kernel<<<stride_blocks(total, 256), 256, 0, st>>>(c.dc, d_pk, work, d_ct + (size_t)off * 2 * lq, total);
            check_launch("enc_combine");
        }
    });
}

int kbfv_decrypt(kbfv_context* ctx, const uint64_t* d_sk, const uint64_t* d_ct, uint64_t* d_m, uint32_t count,
                 kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_sk && d_ct && d_m, KBFV_ERR_INVALID, "null argument");
        require_batchable(c);
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint64_t* work = (uint64_t*)ensure_scratch(c, (size_t)cnt * lq * 8);
            ntt_inv(c.dc, DecSrc{d_ct + (size_t)off * 2 * lq, d_sk, c.dc}, rows_io(c.dc, work, 0, c.nq), cnt * c.nq, st);
            dim3 grid((unsigned)(c.n / 128), (unsigned)cnt);
#define L_DR(M) decrypt_round_kernel<M><<<grid, 128, 0, st>>>(c.dc, work, d_m + (size_t)off * c.n)
            DISPATCH_MAXQ(c.nq, L_DR);
#undef L_DR
            check_launch("decrypt_round");
        }
    });
}

int kbfv_add(kbfv_context* ctx, const uint64_t* d_x, const uint64_t* d_y, uint64_t* d_out, uint32_t count,
             kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        const size_t total = (size_t)count * 2 * c.nq * c.n;
        if (!total) return;
        add_kernel<<<blocks_for(total, 256), 256, 0, S(stream)>>>(c.dc, d_x, d_y, d_out, total, c.nq);
        check_launch("add");
    });
}

int kbfv_mul_plain(kbfv_context* ctx, const uint64_t* d_ct, const uint64_t* d_pt_ntt, uint64_t* d_out, uint32_t count,
                   kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        const size_t total = (size_t)count * 2 * c.nq * c.n;
        if (!total) return;
        mul_plain_kernel<<<blocks_for(total, 256), 256, 0, S(stream)>>>(c.dc, d_ct, d_pt_ntt, d_out, total);
        check_launch("mul_plain");
    });
}

int kbfv_add_plain(kbfv_context* ctx, const uint64_t* d_ct, const uint64_t* d_m, uint64_t* d_out, uint32_t count,
                   kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_ct && d_m && d_out, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint64_t* dm = (uint64_t*)ensure_scratch(c, (size_t)cnt * lq * 8);
            delta_m_kernel<<<blocks_for((size_t)cnt * lq, 256), 256, 0, st>>>(c.dc, d_m + (size_t)off * c.n, dm,
                                                                             (size_t)cnt * lq);
            check_launch("delta_m");
            RowsIO io = rows_io(c.dc, dm, 0, c.nq);
            ntt_fwd(c.dc, io, io, cnt * c.nq, st);
            for (int i = 0; i < cnt; i++) {
                const uint64_t* src = d_ct + (size_t)(off + i) * 2 * lq;
                uint64_t* dst = d_out + (size_t)(off + i) * 2 * lq;
                if (dst != src) KB_CHECK_CUDA(cudaMemcpyAsync(dst, src, lq * 8, cudaMemcpyDeviceToDevice, st));
                add_kernel<<<blocks_for(lq, 256), 256, 0, st>>>(c.dc, src + lq, dm + (size_t)i * lq, dst + lq, lq,
                                                                c.nq);
            }
            check_launch("add_plain");
        }
    });
}

// ---- Galois automorphisms (rotations, conjugation) ---------------------------
uint64_t kbfv_galois_element(const kbfv_context* ctx, int64_t rot_slots) {
    if (!ctx) return 0;
    const Context& c = const_cast<kbfv_context*>(ctx)->c;
    const uint64_t m = 2 * c.n;
    if (rot_slots < 0) return m - 1;  // conjugation
    uint64_t g = 1;
    for (int64_t i = 0; i < rot_slots; i++) g = g * 5 % m;
    return g;
}

int kbfv_keygen_galois(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t galois_elt,
                       uint64_t* d_gk, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk && d_gk, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE((galois_elt & 1) && galois_elt < 2 * c.n, KBFV_ERR_INVALID, "Galois element must be odd and below 2N");
        cudaStream_t st = S(stream);
        const int npq = c.nq + c.np;
        const size_t lpq = (size_t)npq * c.n;
        uint64_t* sg = (uint64_t*)ensure_scratch(c, lpq * 8);
        galois_ntt_kernel<<<blocks_for(lpq, 256), 256, 0, st>>>(c.dc, d_sk, sg, galois_elt, lpq);
        check_launch("galois_sk");
        for (int d = 0; d < c.dnum; d++) {
            uint64_t* a = d_gk + (size_t)d * 2 * lpq;
            uint64_t* b = a + lpq;
            sample_uniform(c, seed, DOM_GAL_A, (uint32_t)d, galois_elt, 0, npq, a, 0, 1, st);
            SalsaKey k = subkey_for(seed, DOM_GAL_E, (uint32_t)d);
            sample_small_kernel<1><<<blocks_for(c.n / 8, 128), 128, 0, st>>>(c.dc, k, galois_elt, 0, npq, b, 0, 1);
            check_launch("sample_gauss");
            RowsIO io = rows_io(c.dc, b, 0, npq);
            ntt_fwd(c.dc, io, io, npq, st);
            ksk_combine_kernel<<<blocks_for(lpq, 256), 256, 0, st>>>(c.dc, a, d_sk, sg, b, d, lpq);
            check_launch("ksk_combine");
        }
    });
}

// ---- scalar and linear ops (BFVScheme.cuh:246-330: multConstAndEqual(uint64),
// multConstAndAddCipherEqual, sub / subAndEqual, negateAndEqual) -------------
static int linear_op(kbfv_context* ctx, const uint64_t* x, const uint64_t* y, uint64_t* out, uint64_t cnst,
                     int op, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(x && out && (op == 1 || op == 2 || y), KBFV_ERR_INVALID, "null argument");
        const size_t total = (size_t)count * 2 * c.nq * c.n;
        if (!total) return;
        ScalarTab tab{};
        for (int l = 0; op >= 2 && l < c.nq; l++) {
            tab.c[l] = cnst % c.mods[l];
            tab.cs[l] = H::shoup(tab.c[l], c.mods[l]);
        }
        linear_kernel<<<blocks_for(total, 256), 256, 0, S(stream)>>>(c.dc, x, y, out, total, c.nq, op, tab);
        check_launch("linear");
    });
}
int kbfv_sub(kbfv_context* ctx, const uint64_t* d_x, const uint64_t* d_y, uint64_t* d_out, uint32_t count,
             kbfv_stream stream) {
    return linear_op(ctx, d_x, d_y, d_out, 0, 0, count, stream);
}
int kbfv_negate(kbfv_context* ctx, const uint64_t* d_x, uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return linear_op(ctx, d_x, nullptr, d_out, 0, 1, count, stream);
}
int kbfv_mul_scalar(kbfv_context* ctx, const uint64_t* d_x, uint64_t cnst, uint64_t* d_out, uint32_t count,
                    kbfv_stream stream) {
    return linear_op(ctx, d_x, nullptr, d_out, cnst, 2, count, stream);
}
int kbfv_mul_scalar_add(kbfv_context* ctx, const uint64_t* d_x, uint64_t cnst, uint64_t* d_acc, uint32_t count,
                        kbfv_stream stream) {
    return linear_op(ctx, d_x, d_acc, d_acc, cnst, 3, count, stream);
}

int kbfv_sample_compat(kbfv_context* ctx, int kind, const void* d_rand, uint64_t* d_out, uint32_t prime0,
                       uint32_t limbs, uint32_t h, double probability, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_rand && d_out, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(limbs >= 1 && prime0 + limbs <= c.mods.size(), KBFV_ERR_INVALID, "prime range out of table");
        cudaStream_t st = S(stream);
        const size_t n = c.n;
        switch (kind) {
            case 0:
                compat_uniform_kernel<<<blocks_for(limbs * n, 256), 256, 0, st>>>(
                    c.dc, (const uint64_t*)d_rand, d_out, (int)prime0, limbs * n);
                break;
            case 1:
                compat_gauss_kernel<<<blocks_for(n, 256), 256, 0, st>>>(c.dc, (const uint32_t*)d_rand, d_out,
                                                                       (int)prime0, (int)limbs);
                break;
            case 2:
                compat_zo_kernel<<<blocks_for(n, 256), 256, 0, st>>>(c.dc, (const uint8_t*)d_rand, d_out, (int)prime0,
                                                                    (int)limbs, probability);
                break;
            case 3:
                KB_REQUIRE(h >= 1 && h <= 1024 && h <= n, KBFV_ERR_INVALID, "Hamming weight out of range");
                KB_CHECK_CUDA(cudaMemsetAsync(d_out, 0, limbs * n * 8, st));
                compat_hwt_kernel<<<limbs, h, 0, st>>>(c.dc, (const uint8_t*)d_rand, d_out, (int)prime0, (int)h);
                break;
            default:
                throw KbfvError(KBFV_ERR_INVALID, "unknown sampler kind");
        }
        check_launch("sample_compat");
    });
}

// ---- batches at arbitrary addresses (HOST arrays of device pointers) ---------
int kbfv_encrypt_batch(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* enc_ids, const uint64_t* d_pk,
                       const uint64_t* const* d_m, uint64_t* const* d_ct, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(enc_ids && d_pk && d_m && d_ct, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            PtrBatch pb = make_batch(d_m + off, d_m + off, d_ct + off, cnt);
            IdTable ids{};
            for (int i = 0; i < cnt; i++) ids.v[i] = enc_ids[off + i];
            uint64_t* work = (uint64_t*)ensure_scratch(c, (size_t)cnt * 4 * lq * 8);
            const size_t per = c.n / 16, per8 = c.n / 8;
            const SalsaKey kv = subkey_for(seed, DOM_ENC_V, 0), k0 = subkey_for(seed, DOM_ENC_E0, 0),
                           k1 = subkey_for(seed, DOM_ENC_E1, 0);
            sample_small_ids_kernel<0><<<blocks_for(per * cnt, 128), 128, 0, st>>>(c.dc, kv, ids, 0, c.nq, work, 4 * lq, cnt);
            sample_small_ids_kernel<1><<<blocks_for(per8 * cnt, 128), 128, 0, st>>>(c.dc, k0, ids, 0, c.nq, work + lq, 4 * lq, cnt);
            sample_small_ids_kernel<1><<<blocks_for(per8 * cnt, 128), 128, 0, st>>>(c.dc, k1, ids, 0, c.nq, work + 2 * lq, 4 * lq, cnt);
            check_launch("sample_small");
            const size_t total = (size_t)cnt * lq;
            delta_m_ptr_kernel<<<stride_blocks(total, 256), 256, 0, st>>>(c.dc, pb, work, total);
            check_launch("delta_m");
            RowsIO io = rows_io(c.dc, work, 0, c.nq);
            ntt_fwd(c.dc, io, io, cnt * 4 * c.nq, st);
            enc_combine_ptr_kernel<<<stride_blocks(total, 256), 256, 0, st>>>(c.dc, d_pk, work, pb, total);
            check_launch("enc_combine");
        }
    });
}

int kbfv_decrypt_batch(kbfv_context* ctx, const uint64_t* d_sk, const uint64_t* const* d_ct, uint64_t* const* d_m,
                       uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_sk && d_ct && d_m, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            PtrBatch pb = make_batch(d_ct + off, d_ct + off, d_m + off, cnt);
            uint64_t* work = (uint64_t*)ensure_scratch(c, (size_t)cnt * lq * 8);
            ntt_inv(c.dc, DecSrcP{pb, d_sk, c.dc}, rows_io(c.dc, work, 0, c.nq), cnt * c.nq, st);
            dim3 grid((unsigned)(c.n / 128), (unsigned)cnt);
#define L_DR(M) decrypt_round_ptr_kernel<M><<<grid, 128, 0, st>>>(c.dc, work, pb)
            DISPATCH_MAXQ(c.nq, L_DR);
#undef L_DR
            check_launch("decrypt_round");
        }
    });
}

int kbfv_add_batch(kbfv_context* ctx, const uint64_t* const* d_x, const uint64_t* const* d_y, uint64_t* const* d_out,
                   uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_x && d_y && d_out, KBFV_ERR_INVALID, "null argument");
        const size_t per = (size_t)2 * c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            PtrBatch pb = make_batch(d_x + off, d_y + off, d_out + off, cnt);
            add_ptr_kernel<<<dim3(blocks_for(per, 256), (unsigned)cnt), 256, 0, S(stream)>>>(c.dc, pb, per);
            check_launch("add_batch");
        }
    });
}

int kbfv_salsa20_stream(const uint8_t key[32], const uint8_t nonce[24], uint64_t block0, uint8_t* d_out, size_t nbytes,
                        int compat, kbfv_stream stream) {
    return guarded([&] {
        KB_REQUIRE(key && nonce && d_out, KBFV_ERR_INVALID, "null argument");
        SalsaKey k;
        uint32_t n0, n1;
        size_t len = nbytes;
        if (compat) {
            // the reference's VecCrypt: zero constants, raw key, nonce word 1 always 0,
            // partial tail block left zero (include/RNG.cuh:18-51, include/RNG_impl.cuh:70-176)
            for (int i = 0; i < 8; i++) k.k[i] = ld32(key + 4 * i);
            for (int i = 0; i < 4; i++) k.sigma[i] = 0;
            n0 = ld32(nonce);
            n1 = 0;
            KB_CHECK_CUDA(cudaMemsetAsync(d_out, 0, nbytes, S(stream)));
            len = nbytes / 64 * 64;
        } else {
            hsalsa_host(key, nonce, k.k);
            static const char* sig = "expand 32-byte k";
            for (int i = 0; i < 4; i++) std::memcpy(&k.sigma[i], sig + 4 * i, 4);
            n0 = ld32(nonce + 16);
            n1 = ld32(nonce + 20);
        }
        if (!len) return;
        const size_t blocks = (len + 63) / 64;
        salsa_stream_kernel<<<blocks_for(blocks, 128), 128, 0, S(stream)>>>(k, n0, n1, block0, d_out, len);
        check_launch("salsa20");
    });
}

}  // extern "C"
