// libkbfv: levels (contexts for fewer live primes), the BFV modulus switch,
// multiplies of batches at mixed levels, key switching over a gadget
// decomposition, and Galois automorphisms.
#include "pipeline.cuh"

// ---- modulus switch (divide by the last prime and round) ---------------------
struct LastLimbSrc {  // row = polynomial: its last limb
    const uint64_t* ct;
    int logn, nq;
    __device__ __forceinline__ int prime(int) const { return nq - 1; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        return PtrRow{const_cast<uint64_t*>(ct) + (((size_t)row * nq + nq - 1) << logn)};
    }
};
struct ModSwitchRow {
    const uint64_t* last;
    uint64_t ql, half, q, mh, half_i;
    // [x + floor(ql/2)]_ql - floor(ql/2), taken mod q_i: the rounding correction
    __device__ __forceinline__ uint64_t load(int j) const {
        const uint64_t x = csub(last[j] + half, ql);
        return sub_mod(barrett64(x, q, mh), half_i, q);
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct ModSwitchSrc {  // rows (poly, i < nq-1)
    const uint64_t* last;  // [poly][N], coefficient form, < q_last
    DevConsts dc;
    __device__ __forceinline__ int prime(int row) const { return row % (dc.nq - 1); }
    __device__ __forceinline__ ModSwitchRow bind(int row) const {
        const int nout = dc.nq - 1, poly = row / nout, i = row % nout;
        ModSwitchRow r;
        r.last = last + ((size_t)poly << dc.logn);
        r.ql = dc.mods[dc.nq - 1];
        r.half = dc.ms_half;
        r.q = dc.mods[i]; r.mh = dc.mu_hi[i];
        r.half_i = dc.ms_half_mod[i];
        return r;
    }
};
// out[poly][i] = (ct[poly][i] - corr[poly][i]) * q_last^-1 mod q_i
__global__ void mod_switch_combine_kernel(DevConsts c, const uint64_t* __restrict__ ct,
                                          const uint64_t* __restrict__ corr, uint64_t* __restrict__ out,
                                          size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int nout = c.nq - 1;
    const size_t row = i >> c.logn, j = i & (((size_t)1 << c.logn) - 1);
    const size_t poly = row / nout;
    const int l = (int)(row % nout);
    const uint64_t q = c.mods[l];
    const uint64_t x = ct[((poly * c.nq + l) << c.logn) + j];
    out[i] = shoup(x + q - corr[i], c.ms_qlinv[l], c.ms_qlinvs[l], q);
}

// rows (item, l) of the a-part of ciphertexts, read through the Galois permutation
struct GaloisRow {
    const uint64_t* p;
    uint64_t g;
    int logn;
    __device__ __forceinline__ uint64_t load(int j) const { return p[galois_perm((uint32_t)j, g, logn)]; }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct GaloisASrc {
    const uint64_t* ct;  // [item][a|b][nq]
    uint64_t g;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ GaloisRow bind(int row) const {
        const int item = row / nq, l = row % nq;
        return GaloisRow{ct + (((size_t)item * 2 * nq + l) << logn), g, logn};
    }
};

extern "C" {

// ---- levels ---------------------------------------------------------------
int kbfv_context_at_level(kbfv_context* ctx, uint32_t live_q, kbfv_context** out) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(out, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(!c.parent, KBFV_ERR_INVALID, "levels are taken from the top-level context");
        KB_REQUIRE(live_q >= 1 && live_q <= (uint32_t)c.nq, KBFV_ERR_LEVEL, "live prime count out of range");
        if (live_q == (uint32_t)c.nq) {
            *out = ctx;
            return;
        }
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.levels.size() < (size_t)c.nq) c.levels.resize(c.nq, nullptr);
        if (!c.levels[live_q]) {
            kbfv_params prm;
            std::memset(&prm, 0, sizeof prm);
            prm.log_n = (uint32_t)c.logn;
            prm.plain_modulus = c.t;
            prm.q_count = live_q;
            prm.q = c.mods.data();
            prm.p_count = (uint32_t)c.np;
            prm.p = c.mods.data() + c.nq;
            prm.digit_primes = (uint32_t)c.alpha;
            auto* h = new kbfv_context();
            try {
                build_context(h->c, prm);
            } catch (...) {
                if (h->c.pool) cudaFree(h->c.pool);
                delete h;
                throw;
            }
            h->c.parent = &c;
            h->c.dc.key_nq = c.nq;
            h->c.dc.key_npq = c.nq + c.np;
            std::memcpy(h->c.seed, c.seed, 32);
            c.levels[live_q] = h;
        }
        *out = (kbfv_context*)c.levels[live_q];
    });
}

int kbfv_mod_switch(kbfv_context* ctx, const uint64_t* d_ct, uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(c.nq >= 2, KBFV_ERR_LEVEL, "a ciphertext with one live prime cannot be switched down");
        KB_REQUIRE(d_ct && d_out, KBFV_ERR_INVALID, "null argument");
        const size_t in_words = (size_t)count * 2 * c.nq * c.n, out_words = (size_t)count * 2 * (c.nq - 1) * c.n;
        KB_REQUIRE(d_out + out_words <= d_ct || d_ct + in_words <= d_out, KBFV_ERR_INVALID,
                   "output must not overlap the input");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const int nout = c.nq - 1;
        const uint32_t chunk = 32;
        for (uint32_t off = 0; off < count; off += chunk) {
            const int cnt = (int)std::min<uint32_t>(chunk, count - off);
            const int polys = cnt * 2;
            uint64_t* last = (uint64_t*)ensure_scratch(c, (size_t)polys * (1 + nout) * c.n * 8);
            uint64_t* corr = last + ((size_t)polys << c.logn);
            const uint64_t* in = d_ct + (size_t)off * 2 * c.nq * c.n;
            uint64_t* o = d_out + (size_t)off * 2 * nout * c.n;
            ntt_inv(dc, LastLimbSrc{in, c.logn, c.nq}, rows_io(dc, last, c.nq - 1, 1), polys, st);
            ntt_fwd(dc, ModSwitchSrc{last, dc}, rows_io(dc, corr, 0, nout), polys * nout, st);
            const size_t total = (size_t)polys * nout * c.n;
            mod_switch_combine_kernel<<<stride_blocks(total, 256), 256, 0, st>>>(dc, in, corr, o, total);
            check_launch("mod_switch");
        }
    });
}

int kbfv_mul_relin_levels(kbfv_context* ctx, const uint64_t* d_rlk, const uint32_t* live_q,
                          const uint64_t* const* ct_a, const uint64_t* const* ct_b, uint64_t* const* out,
                          uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(!c.parent, KBFV_ERR_INVALID, "call on the top-level context");
        KB_REQUIRE(live_q && ct_a && ct_b && out, KBFV_ERR_INVALID, "null pointer array");
        std::map<uint32_t, std::vector<uint32_t>> groups;
        for (uint32_t i = 0; i < count; i++) {
            KB_REQUIRE(live_q[i] >= 1 && live_q[i] <= (uint32_t)c.nq, KBFV_ERR_LEVEL, "live prime count out of range");
            groups[live_q[i]].push_back(i);
        }
        // the level groups run concurrently: the first on the caller's stream, the
        // next ones on the context's lane streams (forked from and joined back into
        // the caller's stream); each level context has its own scratch arena
        cudaStream_t st = S(stream);
        const int ng = (int)groups.size();
        const int lanes = std::min(ng, 4);
        if (lanes > 1) {
            if (!c.lane_fork) {
                for (int k = 0; k < 3; k++) {
                    KB_CHECK_CUDA(cudaStreamCreateWithFlags(&c.lane[k], cudaStreamNonBlocking));
                    KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.lane_join[k], cudaEventDisableTiming));
                }
                KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.lane_fork, cudaEventDisableTiming));
            }
            KB_CHECK_CUDA(cudaEventRecord(c.lane_fork, st));
            for (int k = 1; k < lanes; k++) KB_CHECK_CUDA(cudaStreamWaitEvent(c.lane[k - 1], c.lane_fork, 0));
        }
        int g = 0;
        for (auto it = groups.rbegin(); it != groups.rend(); ++it, ++g) {  // highest level first
            kbfv_context* lv = nullptr;
            int rc = kbfv_context_at_level(ctx, it->first, &lv);
            if (rc != KBFV_OK) throw KbfvError(rc, g_last_error);
            std::vector<const uint64_t*> A, B;
            std::vector<uint64_t*> O;
            for (uint32_t i : it->second) {
                A.push_back(ct_a[i]);
                B.push_back(ct_b[i]);
                O.push_back(out[i]);
            }
            const int lane = g % lanes;
            cudaStream_t ls = lane == 0 ? st : c.lane[lane - 1];
            rc = kbfv_mul_relin_batch(lv, d_rlk, A.data(), B.data(), O.data(), (uint32_t)A.size(), (kbfv_stream)ls);
            if (rc != KBFV_OK) throw KbfvError(rc, g_last_error);
        }
        for (int k = 1; k < lanes; k++) {
            KB_CHECK_CUDA(cudaEventRecord(c.lane_join[k - 1], c.lane[k - 1]));
            KB_CHECK_CUDA(cudaStreamWaitEvent(st, c.lane_join[k - 1], 0));
        }
    });
}

// ---- key switching over a gadget decomposition ------------------------------
// G1: pieces of a1*a2 (coefficient form, sd2) fused into the forward NTT over Q|P;
// G2/G3: the key-switch tail (ks_tail) with the gadget key, written to the outputs.
static size_t gadget_sg_bytes(const Context& c, int count, int w) {
    return (size_t)count * c.nq * gadget_pieces(w) * (c.nq + c.np) * c.n * 8;
}
static int gadget_chunk(const Context& c, int w) {
    const size_t per = gadget_sg_bytes(c, 1, w);
    return (int)std::max<size_t>(1, std::min<size_t>(kMaxBatch, ((size_t)4 << 30) / per));
}

static void gadget_keyswitch(Context& c, const uint64_t* gk, int w, int count, const MulScratch& m, uint64_t* sg,
                             const uint64_t* add, const PtrBatch& pb, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    const int J = gadget_pieces(w), ndig = c.nq * J;
    // fully reduced NTT outputs: the key product sums ndig terms below q^2
    ntt_fwd<GadgetDigitSrc, RowsIO, true>(dc, GadgetDigitSrc{m.sd2, dc, J, w}, rows_io(dc, sg, 0, dc.npq),
                                         count * ndig * dc.npq, st);
    ks_tail(dc, sg, gk, ndig, m.se, add, pb, count, st);
}

int kbfv_relinearize_gadget(kbfv_context* ctx, const uint64_t* d_gk, uint32_t log_base, const uint64_t* d_tensor,
                            uint64_t* d_ct, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_gk, KBFV_ERR_NO_KEY, "gadget key missing");
        KB_REQUIRE(log_base >= 4 && log_base <= 30, KBFV_ERR_INVALID, "gadget base 2^w needs 4 <= w <= 30");
        KB_REQUIRE(c.nq * gadget_pieces((int)log_base) < 256, KBFV_ERR_INVALID, "too many gadget digits");
        const int w = (int)log_base;
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const size_t lq = (size_t)c.nq * c.n;
        const int chunk = gadget_chunk(c, w);
        for (uint32_t off = 0; off < count; off += chunk) {
            const int cnt = (int)std::min<uint32_t>(chunk, count - off);
            const size_t mb = mul_scratch_layout(c, cnt, nullptr).bytes;
            uint8_t* base = ensure_scratch(c, mb + gadget_sg_bytes(c, cnt, w));
            MulScratch m = mul_scratch_layout(c, cnt, base);
            uint64_t* sg = (uint64_t*)(base + mb);
            const uint64_t* tz = d_tensor + (size_t)off * 3 * lq;
            uint64_t* out = d_ct + (size_t)off * 2 * lq;
            ntt_inv(dc, TensorA2{tz, dc.logn, dc.nq}, rows_io(dc, m.sd2, 0, dc.nq), cnt * dc.nq, st);
            std::vector<uint64_t*> O(cnt);
            std::vector<const uint64_t*> Z(cnt);
            for (int i = 0; i < cnt; i++) { O[i] = out + (size_t)i * 2 * lq; Z[i] = nullptr; }
            PtrBatch pb = make_batch(Z.data(), Z.data(), O.data(), cnt);
            gadget_keyswitch(c, d_gk, w, cnt, m, sg, nullptr, pb, st);
            for (int i = 0; i < cnt; i++) {
                const size_t tot = 2 * lq;
                add_kernel<<<blocks_for(tot, 256), 256, 0, st>>>(dc, out + (size_t)i * 2 * lq, tz + (size_t)i * 3 * lq + lq,
                                                                 out + (size_t)i * 2 * lq, tot, dc.nq);
            }
            check_launch("relin_add");
        }
    });
}

int kbfv_mul_relin_gadget(kbfv_context* ctx, const uint64_t* d_gk, uint32_t log_base, const uint64_t* d_ct_a,
                          const uint64_t* d_ct_b, uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_gk, KBFV_ERR_NO_KEY, "gadget key missing");
        KB_REQUIRE(log_base >= 4 && log_base <= 30, KBFV_ERR_INVALID, "gadget base 2^w needs 4 <= w <= 30");
        KB_REQUIRE(c.nq * gadget_pieces((int)log_base) < 256, KBFV_ERR_INVALID, "too many gadget digits");
        const int w = (int)log_base;
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        const int chunk = gadget_chunk(c, w);
        for (uint32_t off = 0; off < count; off += chunk) {
            const int cnt = (int)std::min<uint32_t>(chunk, count - off);
            std::vector<const uint64_t*> A(cnt), B(cnt);
            std::vector<uint64_t*> O(cnt);
            for (int i = 0; i < cnt; i++) {
                A[i] = d_ct_a + (size_t)(off + i) * 2 * lq;
                B[i] = d_ct_b + (size_t)(off + i) * 2 * lq;
                O[i] = d_out + (size_t)(off + i) * 2 * lq;
            }
            PtrBatch pb = make_batch(A.data(), B.data(), O.data(), cnt);
            const size_t mb = mul_scratch_layout(c, cnt, nullptr).bytes;
            uint8_t* base = ensure_scratch(c, mb + gadget_sg_bytes(c, cnt, w));
            MulScratch m = mul_scratch_layout(c, cnt, base);
            uint64_t* sg = (uint64_t*)(base + mb);
            mul_front(c, pb, cnt, m, st);
            k5_launch(c, cnt, m, nullptr, 2, st);
            gadget_keyswitch(c, d_gk, w, cnt, m, sg, m.sd, pb, st);
        }
    });
}

int kbfv_apply_galois(kbfv_context* ctx, const uint64_t* d_gk, uint64_t galois_elt, const uint64_t* d_ct,
                      uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_gk, KBFV_ERR_NO_KEY, "Galois key missing");
        KB_REQUIRE(d_ct && d_out, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE((galois_elt & 1) && galois_elt < 2 * c.n, KBFV_ERR_INVALID, "Galois element must be odd and below 2N");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
            MulScratch m = mul_scratch_layout(c, cnt, base);
            const uint64_t* in = d_ct + (size_t)off * 2 * lq;
            uint64_t* out = d_out + (size_t)off * 2 * lq;
            // g(b) first (the output may overwrite the input): sb holds [item][nq]
            for (int i = 0; i < cnt; i++)
                galois_ntt_kernel<<<blocks_for(lq, 256), 256, 0, st>>>(dc, in + (size_t)i * 2 * lq + lq,
                                                                        m.sb + (size_t)i * lq, galois_elt, lq);
            check_launch("galois_b");
            // g(a) read through the permutation by the inverse NTT, then the hybrid key switch
            ntt_inv(dc, GaloisASrc{in, galois_elt, dc.logn, dc.nq}, rows_io(dc, m.sa, 0, dc.nq), cnt * dc.nq, st);
            dim3 grid((unsigned)(c.n / 128), (unsigned)cnt);
#define L_MU(M) modup_kernel<M><<<grid, 128, 0, st>>>(dc, m.sa, m.sd2)
            DISPATCH_MAXQ(dc.nq, L_MU);
#undef L_MU
            check_launch("modup");
            ntt_fwd<RowsIO, RowsIO, true>(dc, rows_io(dc, m.sd2, 0, dc.npq), rows_io(dc, m.sd2, 0, dc.npq),
                                          cnt * dc.dnum * dc.npq, st);
            std::vector<uint64_t*> O(cnt);
            std::vector<const uint64_t*> Z(cnt);
            for (int i = 0; i < cnt; i++) { O[i] = out + (size_t)i * 2 * lq; Z[i] = nullptr; }
            PtrBatch pb = make_batch(Z.data(), Z.data(), O.data(), cnt);
            ks_tail(dc, m.sd2, d_gk, dc.dnum, m.se, nullptr, pb, cnt, st);
            for (int i = 0; i < cnt; i++)
                add_kernel<<<blocks_for(lq, 256), 256, 0, st>>>(dc, out + (size_t)i * 2 * lq + lq, m.sb + (size_t)i * lq,
                                                                out + (size_t)i * 2 * lq + lq, lq, dc.nq);
            check_launch("galois_add");
        }
    });
}

}  // extern "C"
