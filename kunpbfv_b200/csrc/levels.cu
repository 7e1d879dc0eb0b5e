// libkbfv: levels (contexts for fewer live primes), the BFV modulus switch,
// multiplies of batches at mixed levels, key switching over a gadget
// decomposition, and Galois automorphisms.
#include <numeric>

#include "mixed.cuh"

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

// ---- multiplies of batches at mixed levels (see mixed.cuh) -------------------
// The DevConsts of the level with `live` primes in the top context's device
// array: the level context is built and its constants uploaded on first use
// (synchronous copies: make a first call per level before any stream capture).
static const DevConsts* level_consts(kbfv_context* top_h, Context& top, int live) {
    if (!top.d_level_consts) {
        KB_CHECK_CUDA(cudaMalloc(&top.d_level_consts, sizeof(DevConsts) * (size_t)(top.nq + 1)));
        top.level_uploaded.assign((size_t)top.nq + 1, 0);
    }
    if (!top.level_uploaded[live]) {
        kbfv_context* lv = nullptr;
        const int rc = kbfv_context_at_level(top_h, (uint32_t)live, &lv);
        if (rc != KBFV_OK) throw KbfvError(rc, g_last_error);
        KB_CHECK_CUDA(cudaMemcpy(top.d_level_consts + live, &lv->c.dc, sizeof(DevConsts), cudaMemcpyHostToDevice));
        top.level_uploaded[live] = 1;
    }
    return top.d_level_consts + live;
}

static Groups groups_header(const Context& top) {
    Groups G;
    std::memset(&G, 0, sizeof G);
    G.logn = top.logn;
    G.np = top.np;
    G.top_nq = top.nq;
    G.top_nr = top.nr;
    G.top_npq = top.nq + top.np;
    G.top_nqr = top.nq + top.nr;
    G.top_dnum = top.dnum;
    G.key_nq = top.nq;
    G.key_npq = top.nq + top.np;
    G.dp = fast_div((uint32_t)top.np);
    return G;
}

// open group G.ng for level `lvl`, its first item `first`
static void add_group(kbfv_context* top_h, Context& top, Groups& G, int lvl, int first) {
    const int g = G.ng++;
    G.first[g] = first;
    G.lv[g] = level_consts(top_h, top, lvl);
    G.nq[g] = lvl;
    G.nr[g] = lvl + 1;
    G.npq[g] = lvl + top.np;
    G.nqr[g] = 2 * lvl + 1;
    G.dnum[g] = (lvl + top.alpha - 1) / top.alpha;  // the level keeps the top level's digit size
    G.dq[g] = fast_div((uint32_t)G.nq[g]);
    G.dr[g] = fast_div((uint32_t)G.nr[g]);
    G.dpq[g] = fast_div((uint32_t)G.npq[g]);
    G.dqr[g] = fast_div((uint32_t)G.nqr[g]);
}

// rows of a stage with per(g) rows per item of group g
template <class F>
static StageRows stage_rows(const Groups& G, F per, int* total) {
    StageRows R;
    std::memset(&R, 0, sizeof R);
    int acc = 0;
    for (int g = 0; g < G.ng; g++) {
        R.start[g] = acc;
        R.per[g] = fast_div((uint32_t)per(g));
        acc += (G.first[g + 1] - G.first[g]) * per(g);
    }
    R.start[G.ng] = acc;
    *total = acc;
    return R;
}

// The hybrid multiply + relinearise of a mixed batch (items ordered by level as
// G describes) as one launch sequence: the stages of mul_relin_chunk, each over
// all items, every row with its own level's constants.
static void mul_relin_mixed(Context& top, const uint64_t* rlk, const PtrBatch& pb, const Groups& G, int count,
                            const MulScratch& m, cudaStream_t st) {
    const DevConsts& dc = top.dc;  // ring degree and launch shapes; rows take their level's tables
    int n = 0;
    // K1: INTT over Q of [a1, b1, a2, b2]
    const StageRows r1 = stage_rows(G, [&](int g) { return 4 * G.nq[g]; }, &n);
    ntt_inv(dc, MixedPairQRows{pb, G, r1}, MixedRows{m.sa, (size_t)4 * G.top_nq, G, r1, 0}, n, st);
    // K2: Q -> R
#define L_BM(M) bconv_mixed_launch_m<M>(G, dc.shape, count, m, st)
    DISPATCH_MAXQ(G.top_nq + 1, L_BM);
#undef L_BM
    // K3: NTT over R in place, fully reduced
    const StageRows r3 = stage_rows(G, [&](int g) { return 4 * G.nr[g]; }, &n);
    const MixedRows rrows{m.sb, (size_t)4 * G.top_nr, G, r3, 1};
    ntt_fwd<MixedRows, MixedRows, true>(dc, rrows, rrows, n, st);
    // K4: tensor fused into INTT over Q|R
    const StageRows r4 = stage_rows(G, [&](int g) { return 3 * G.nqr[g]; }, &n);
    ntt_inv(dc, MixedTensorSrc{pb, m.sb, G, r4}, MixedRows{m.sc, (size_t)3 * G.top_nqr, G, r4, 3}, n, st);
    // K5: scale-and-round, R -> Q, digit lift
#define L_KM(M) k5_mixed_launch_m<M>(G, dc.shape, count, m, st)
    DISPATCH_MAXQ(G.top_nq + 1, L_KM);
#undef L_KM
    // K6a: NTT over Q|P of the digits in place, fully reduced
    const StageRows r6 = stage_rows(G, [&](int g) { return G.dnum[g] * G.npq[g]; }, &n);
    const MixedRows drows{m.sd2, (size_t)G.top_dnum * G.top_npq, G, r6, 2};
    ntt_fwd<MixedRows, MixedRows, true>(dc, drows, drows, n, st);
    // K6b: key product over P fused into INTT over P
    const StageRows r6b = stage_rows(G, [&](int) { return 2 * G.np; }, &n);
    ntt_inv(dc, MixedKeyIPSrc{m.sd2, rlk, G, r6b}, MixedSeRowsP{m.se, G, r6b}, n, st);
    // K7: mod down + add fused into NTT over Q, the key product over Q added at its store
    const StageRows r7 = stage_rows(G, [&](int g) { return 2 * G.nq[g]; }, &n);
    const MixedOutCtKeyDst dst{pb, m.sd2, rlk, G, r7};
    if (G.np == 1)
        ntt_fwd(dc, MixedModDownSrc<true>{m.se, m.sd, G, r7}, dst, n, st);
    else
        ntt_fwd(dc, MixedModDownSrc<false>{m.se, m.sd, G, r7}, dst, n, st);
}

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
            h->c.dc.shape = c.dc.shape;
            h->c.branches = c.branches;
            h->c.min_branch_pairs = c.min_branch_pairs;
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
        require_batchable(c);
        KB_REQUIRE(d_rlk, KBFV_ERR_NO_KEY, "relinearisation key missing");
        KB_REQUIRE(live_q && ct_a && ct_b && out, KBFV_ERR_INVALID, "null pointer array");
        for (uint32_t i = 0; i < count; i++) {
            KB_REQUIRE(live_q[i] >= 1 && live_q[i] <= (uint32_t)c.nq, KBFV_ERR_LEVEL, "live prime count out of range");
            KB_REQUIRE(ct_a[i] && ct_b[i] && out[i], KBFV_ERR_INVALID, "null ciphertext pointer");
        }
        // pairs ordered by level, highest first (stable); each product still goes
        // to its own output pointer
        std::vector<uint32_t> order(count);
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return live_q[x] > live_q[y]; });
        cudaStream_t st = S(stream);
        for (uint32_t off = 0; off < count;) {
            // one chunk: up to kMaxBatch pairs in up to kMaxGroups levels
            uint32_t end = off;
            int levels_seen = 0;
            while (end < count && end - off < (uint32_t)kMaxBatch) {
                if (end == off || live_q[order[end]] != live_q[order[end - 1]]) {
                    if (levels_seen == kMaxGroups) break;
                    levels_seen++;
                }
                end++;
            }
            const int cnt = (int)(end - off);
            // sub-batches on the caller's stream and auxiliary streams (as in
            // kbfv_mul_relin_batch); pairs dealt round-robin, so each sub-batch
            // keeps the level order and a similar mix of levels
            const int nb = branch_count(c, cnt);
            const int per = (cnt + nb - 1) / nb;
            const size_t region = branch_region_bytes(c, per);
            uint8_t* base = ensure_scratch(c, region * nb);
            if (nb > 1) {
                ensure_branch_streams(c);
                KB_CHECK_CUDA(cudaEventRecord(c.fork_ev, st));
                for (int k = 1; k < nb; k++) KB_CHECK_CUDA(cudaStreamWaitEvent(c.aux[k - 1], c.fork_ev, 0));
            }
            for (int k = 0; k < nb; k++) {
                Groups G = groups_header(c);
                PtrBatch pb;
                std::memset(&pb, 0, sizeof pb);
                int n = 0;
                for (int j = k; j < cnt; j += nb) {
                    const uint32_t it = order[off + j];
                    const int lvl = (int)live_q[it];
                    if (G.ng == 0 || G.nq[G.ng - 1] != lvl) add_group(ctx, c, G, lvl, n);
                    pb.a[n] = ct_a[it];
                    pb.b[n] = ct_b[it];
                    pb.o[n] = out[it];
                    n++;
                }
                G.first[G.ng] = n;
                if (n == 0) continue;
                mul_relin_mixed(c, d_rlk, pb, G, n, mul_scratch_layout(c, n, base + (size_t)k * region),
                                k == 0 ? st : c.aux[k - 1]);
            }
            for (int k = 1; k < nb; k++) {
                KB_CHECK_CUDA(cudaEventRecord(c.join_ev[k - 1], c.aux[k - 1]));
                KB_CHECK_CUDA(cudaStreamWaitEvent(st, c.join_ev[k - 1], 0));
            }
            off = end;
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
            mul_front(c.dc, pb, cnt, m, st);
            k5_launch(c.dc, cnt, m, nullptr, 2, st);
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
