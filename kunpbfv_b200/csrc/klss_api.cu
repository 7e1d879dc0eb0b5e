// libkbfv: the reference's key switch over the auxiliary T base (KLSS) and its
// pieces as entry points.
#include "pipeline.cuh"

// T-base key switch (the reference's KLSS, include/KeySwitch_23.cuh:244-330) of
// a1*a2 given in coefficient form over Q (sd2, [item][nq]); writes the P|Q
// results into se ([item][2][npq]).
static void klss_keyswitch(Context& c, const uint64_t* rlk_t, int count, const MulScratch& m, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    const KlssConsts& kc = c.kc;
    // Qj blocks -> T (modUpQjtoT_23)
    klss_block_to_t_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)kc.nqj, (unsigned)count), 128, 0, st>>>(
        dc, kc, m.sd2, m.st1, 0, (size_t)c.nq << c.logn, (size_t)kc.nqj * c.nt << c.logn);
    check_launch("klss_qj_to_t");
    // NTT over T
    ntt_fwd<RowsIO, RowsIO, true>(dc, rows_io(dc, m.st1, dc.idx_t, c.nt), rows_io(dc, m.st1, dc.idx_t, c.nt),
                                   count * kc.nqj * c.nt, st);
    // external product over T fused into INTT over T (external_product_T)
    ntt_inv(dc, ExtProdSrc{m.st1, rlk_t, dc, c.nt, kc.nri, kc.nqj, kc.nqj}, rows_io(dc, m.st2, dc.idx_t, c.nt),
            count * 2 * kc.nri * c.nt, st);
    // centred T -> P|Q (modUpTtoPQl_23)
    klss_t_to_pq_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)kc.nri, (unsigned)(count * 2)), 128, 0, st>>>(
        dc, kc, m.st2, m.se);
    check_launch("klss_t_to_pq");
}

static void mul_relin_klss_chunk(Context& c, const uint64_t* rlk_t, const PtrBatch& pb, int count,
                                 const MulScratch& m, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    mul_front(c.dc, pb, count, m, st);
    k5_launch(c.dc, count, m, nullptr, 2, st);
    klss_keyswitch(c, rlk_t, count, m, st);
    ntt_fwd(dc, ModDownAddSrc{m.se, m.sd, dc}, OutCtDst{pb, dc.logn, dc.nq}, count * 2 * dc.nq, st);
}

extern "C" {

// ---- T-base key switch (the reference's KLSS) ------------------------------
int kbfv_context_klss(const kbfv_context* ctx, uint32_t* ri_blocks, uint32_t* qj_blocks, uint64_t* key_words) {
    return guarded([&] {
        const Context& c = CX(const_cast<kbfv_context*>(ctx));
        require_klss(c);
        if (ri_blocks) *ri_blocks = (uint32_t)c.kc.nri;
        if (qj_blocks) *qj_blocks = (uint32_t)c.kc.nqj;
        if (key_words) *key_words = (uint64_t)2 * c.kc.nqj * c.kc.nri * c.nt * c.n;
    });
}

int kbfv_rlk_to_klss(kbfv_context* ctx, const uint64_t* d_rlk, uint64_t* d_rlk_t, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(d_rlk && d_rlk_t, KBFV_ERR_INVALID, "null key pointer");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const KlssConsts& kc = c.kc;
        const int npq = dc.npq;
        uint64_t* coef = (uint64_t*)ensure_scratch(c, (size_t)c.dnum * 2 * npq * c.n * 8);
        // key [digit][a|b][Q|P] in NTT form -> coefficient form
        ntt_inv(dc, rows_io(dc, const_cast<uint64_t*>(d_rlk), 0, npq), rows_io(dc, coef, 0, npq),
                c.dnum * 2 * npq, st);
        // Ri blocks -> T (modUpPQtoT_23), written as [a|b][digit][Ri][T]
        for (int h = 0; h < 2; h++) {
            klss_block_to_t_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)kc.nri, (unsigned)c.dnum), 128, 0, st>>>(
                dc, kc, coef + ((size_t)h * npq << c.logn), d_rlk_t + ((size_t)h * c.dnum * kc.nri * c.nt << c.logn), 1,
                (size_t)2 * npq << c.logn, (size_t)kc.nri * c.nt << c.logn);
            check_launch("klss_pq_to_t");
        }
        RowsIO io = rows_io(dc, d_rlk_t, dc.idx_t, c.nt);
        ntt_fwd(dc, io, io, 2 * c.dnum * kc.nri * c.nt, st);
    });
}

int kbfv_klss_modup_qj_to_t(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                            kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(polys <= 65535, KBFV_ERR_INVALID, "at most 65535 polynomials per call");
        if (!polys) return;
        klss_block_to_t_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)c.kc.nqj, polys), 128, 0, S(stream)>>>(
            c.dc, c.kc, d_in, d_out, 0, (size_t)c.nq << c.logn, (size_t)c.kc.nqj * c.nt << c.logn);
        check_launch("klss_qj_to_t");
    });
}

int kbfv_klss_modup_pq_to_t(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                            kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(polys <= 65535, KBFV_ERR_INVALID, "at most 65535 polynomials per call");
        if (!polys) return;
        klss_block_to_t_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)c.kc.nri, polys), 128, 0, S(stream)>>>(
            c.dc, c.kc, d_in, d_out, 1, (size_t)c.dc.npq << c.logn, (size_t)c.kc.nri * c.nt << c.logn);
        check_launch("klss_pq_to_t");
    });
}

int kbfv_klss_external_product(kbfv_context* ctx, const uint64_t* d_digits, const uint64_t* d_rlk_t,
                               uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(d_rlk_t, KBFV_ERR_NO_KEY, "T-base relinearisation key missing");
        const KlssConsts& kc = c.kc;
        ntt_inv(c.dc, ExtProdSrc{d_digits, d_rlk_t, c.dc, c.nt, kc.nri, kc.nqj, kc.nqj},
                rows_io(c.dc, d_out, c.dc.idx_t, c.nt), (int)count * 2 * kc.nri * c.nt, S(stream));
    });
}

int kbfv_klss_t_to_pq(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(polys <= 65535, KBFV_ERR_INVALID, "at most 65535 polynomials per call");
        if (!polys) return;
        klss_t_to_pq_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)c.kc.nri, polys), 128, 0, S(stream)>>>(
            c.dc, c.kc, d_in, d_out);
        check_launch("klss_t_to_pq");
    });
}

int kbfv_relinearize_klss(kbfv_context* ctx, const uint64_t* d_rlk_t, const uint64_t* d_tensor, uint64_t* d_ct,
                          uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(d_rlk_t, KBFV_ERR_NO_KEY, "T-base relinearisation key missing");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
            MulScratch m = mul_scratch_layout(c, cnt, base);
            const uint64_t* tz = d_tensor + (size_t)off * 3 * lq;
            uint64_t* out = d_ct + (size_t)off * 2 * lq;
            ntt_inv(dc, TensorA2{tz, dc.logn, dc.nq}, rows_io(dc, m.sd2, 0, dc.nq), cnt * dc.nq, st);
            klss_keyswitch(c, d_rlk_t, cnt, m, st);
            std::vector<uint64_t*> O(cnt);
            std::vector<const uint64_t*> Z(cnt);
            for (int i = 0; i < cnt; i++) { O[i] = out + (size_t)i * 2 * lq; Z[i] = nullptr; }
            PtrBatch pb = make_batch(Z.data(), Z.data(), O.data(), cnt);
            ntt_fwd(dc, ModDownAddSrc{m.se, nullptr, dc}, OutCtDst{pb, dc.logn, dc.nq}, cnt * 2 * dc.nq, st);
            for (int i = 0; i < cnt; i++) {
                const size_t tot = 2 * lq;
                add_kernel<<<blocks_for(tot, 256), 256, 0, st>>>(dc, out + (size_t)i * 2 * lq, tz + (size_t)i * 3 * lq + lq,
                                                                 out + (size_t)i * 2 * lq, tot, dc.nq);
            }
            check_launch("relin_add");
        }
    });
}

int kbfv_mul_relin_klss(kbfv_context* ctx, const uint64_t* d_rlk_t, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                        uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(d_rlk_t, KBFV_ERR_NO_KEY, "T-base relinearisation key missing");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            std::vector<const uint64_t*> A(cnt), B(cnt);
            std::vector<uint64_t*> O(cnt);
            for (int i = 0; i < cnt; i++) {
                A[i] = d_ct_a + (size_t)(off + i) * 2 * lq;
                B[i] = d_ct_b + (size_t)(off + i) * 2 * lq;
                O[i] = d_out + (size_t)(off + i) * 2 * lq;
            }
            PtrBatch pb = make_batch(A.data(), B.data(), O.data(), cnt);
            uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
            MulScratch m = mul_scratch_layout(c, cnt, base);
            mul_relin_klss_chunk(c, d_rlk_t, pb, cnt, m, st);
        }
    });
}

}  // extern "C"
