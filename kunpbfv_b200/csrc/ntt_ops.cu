// libkbfv: the standalone transforms (rows and pointer batches, with the tuned
// radix split) and the standalone per-step kernels of the multiply path.
#include "pipeline.cuh"

// Standalone NTT of plain rows with a chosen radix split for rings above 2^lb:
// a column pass of logn - lb stages (forward: first; inverse: last) and block
// kernels of 2^lb points, lb in 12..14 (0: the built-in shapes of ntt_fwd/inv).
template <int RC, int LB>
static void ntt_rows_split(const DevConsts& dc, RowsIO io, int rows, bool fwd, cudaStream_t st) {
    const size_t total = (size_t)rows << LB;
    if (fwd) {
        if constexpr (RC == 4)
            ntt_fwd_col16_kernel<RC, RowsIO, RowsIO><<<stride_blocks(total, 256), 256, 0, st>>>(io, io, dc.tw_fwd,
                                                                                            dc.mods, dc.logn, total);
        else
            ntt_fwd_col_kernel<RC, RowsIO, RowsIO><<<stride_blocks(total, 256), 256, 0, st>>>(io, io, dc.tw_fwd,
                                                                                          dc.mods, dc.logn, total);
        launch_fwd_block<LB, RowsIO, RowsIO, true>(dc, io, io, rows, dc.logn, st);
    } else {
        launch_inv_block<LB, RowsIO, RowsIO, false>(dc, io, io, rows, dc.logn, st);
        if constexpr (RC == 4)
            ntt_inv_col16_kernel<RC, RowsIO, RowsIO><<<stride_blocks(total, 256), 256, 0, st>>>(io, io, dc.tw_inv,
                                                                                            dc.mods, dc.logn, total);
        else
            ntt_inv_col_kernel<RC, RowsIO, RowsIO><<<stride_blocks(total, 256), 256, 0, st>>>(io, io, dc.tw_inv,
                                                                                          dc.mods, dc.logn, total);
    }
    check_launch(fwd ? "ntt_fwd" : "ntt_inv");
}
static void ntt_rows(const Context& c, RowsIO io, int rows, bool fwd, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    if (rows <= 0) return;
    const int lb = c.ntt_block_log;
    if (lb == 0 || lb >= dc.logn) {  // built-in shapes
        if (fwd) ntt_fwd(dc, io, io, rows, st);
        else ntt_inv(dc, io, io, rows, st);
        return;
    }
    switch (dc.logn * 100 + lb) {
        case 1312: ntt_rows_split<1, 12>(dc, io, rows, fwd, st); break;
        case 1412: ntt_rows_split<2, 12>(dc, io, rows, fwd, st); break;
        case 1413: ntt_rows_split<1, 13>(dc, io, rows, fwd, st); break;
        case 1512: ntt_rows_split<3, 12>(dc, io, rows, fwd, st); break;
        case 1513: ntt_rows_split<2, 13>(dc, io, rows, fwd, st); break;
        case 1514: ntt_rows_split<1, 14>(dc, io, rows, fwd, st); break;
        case 1612: ntt_rows_split<4, 12>(dc, io, rows, fwd, st); break;
        case 1613: ntt_rows_split<3, 13>(dc, io, rows, fwd, st); break;
        case 1614: ntt_rows_split<2, 14>(dc, io, rows, fwd, st); break;
        default: throw KbfvError(KBFV_ERR_INVALID, "unsupported NTT split");
    }
}

void launch_bconv(const DevConsts& dc, const BconvTables& tb, const uint64_t* in, uint64_t* out, int polys,
                         size_t in_stride, size_t out_stride, cudaStream_t st) {
    if (polys <= 0) return;
    const int threads = dc.shape.bconv_threads, cpt = dc.shape.bconv_cpt;
    dim3 grid((unsigned)((1u << dc.logn) / (threads * cpt)), (unsigned)polys);
    const size_t sh = (size_t)tb.nin * tb.nout * 8;
#define L_BC(M)                                                                                            \
    do {                                                                                                   \
        static int res1[4] = {0, 0, 0, 0}, res2[4] = {0, 0, 0, 0};                                         \
        if (cpt == 2) {                                                                                    \
            const int a = dc.shape.l2_prefetch ? resident_ctas_at((const void*)bconv2_kernel<M>, threads, (int)sh, res2) : 0; \
            bconv2_kernel<M><<<grid, threads, sh, st>>>(tb, in, out, dc.logn, in_stride, out_stride, a);   \
        } else {                                                                                           \
            const int a = dc.shape.l2_prefetch ? resident_ctas_at((const void*)bconv_kernel<M>, threads, (int)sh, res1) : 0; \
            bconv_kernel<M><<<grid, threads, sh, st>>>(tb, in, out, dc.logn, in_stride, out_stride, a);    \
        }                                                                                                  \
    } while (0)
    DISPATCH_MAXQ(tb.nin, L_BC);
#undef L_BC
    check_launch("bconv");
}

// rows of polynomials at arbitrary addresses: row (item, limb) -> pb.o[item] + limb*N
struct PtrPolysIO {
    PtrBatch pb;
    int logn, limbs, p0;
    __device__ __forceinline__ int prime(int row) const { return p0 + row % limbs; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        return PtrRow{pb.o[row / limbs] + ((size_t)(row % limbs) << logn)};
    }
};

extern "C" {

int kbfv_ntt_fwd(kbfv_context* ctx, uint64_t* d_rows, uint32_t rows, uint32_t prime0, uint32_t period,
                 kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_rows && period >= 1 && prime0 + period <= c.mods.size(), KBFV_ERR_INVALID, "bad NTT rows");
        KB_REQUIRE(rows <= (1u << 27), KBFV_ERR_INVALID, "at most 2^27 rows per call");
        RowsIO io = rows_io(c.dc, d_rows, (int)prime0, (int)period);
        ntt_rows(c, io, (int)rows, true, S(stream));
    });
}

int kbfv_ntt_inv(kbfv_context* ctx, uint64_t* d_rows, uint32_t rows, uint32_t prime0, uint32_t period,
                 kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_rows && period >= 1 && prime0 + period <= c.mods.size(), KBFV_ERR_INVALID, "bad NTT rows");
        KB_REQUIRE(rows <= (1u << 27), KBFV_ERR_INVALID, "at most 2^27 rows per call");
        RowsIO io = rows_io(c.dc, d_rows, (int)prime0, (int)period);
        ntt_rows(c, io, (int)rows, false, S(stream));
    });
}

int kbfv_bconv_q_to_r(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        launch_bconv(c.dc, q2r_tables(c.dc), d_in, d_out, (int)polys, (size_t)c.nq << c.logn,
                     (size_t)c.nr << c.logn, S(stream));
    });
}

int kbfv_bconv_r_to_q(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        launch_bconv(c.dc, r2q_tables(c.dc), d_in, d_out, (int)polys, (size_t)c.nr << c.logn,
                     (size_t)c.nq << c.logn, S(stream));
    });
}

int kbfv_tensor_qr(kbfv_context* ctx, const uint64_t* d_ct1, const uint64_t* d_ct2, uint64_t* d_out, uint32_t pairs,
                   kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        const size_t total = (size_t)pairs * c.dc.nqr * c.n;
        if (!total) return;
        tensor_qr_kernel<<<blocks_for(total, 256), 256, 0, S(stream)>>>(c.dc, d_ct1, d_ct2, d_out, total);
        check_launch("tensor_qr");
    });
}

int kbfv_scale_round_qr_r(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                          kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!polys) return;
        dim3 grid((unsigned)(c.n / 128), polys);
#define L_SR(M) scale_round_kernel<M><<<grid, 128, 0, S(stream)>>>(c.dc, d_in, d_out)
        DISPATCH_MAXQ(c.nq, L_SR);
#undef L_SR
        check_launch("scale_round");
    });
}

int kbfv_decrypt_round(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!polys) return;
        dim3 grid((unsigned)(c.n / 128), polys);
#define L_DR(M) decrypt_round_kernel<M><<<grid, 128, 0, S(stream)>>>(c.dc, d_in, d_out)
        DISPATCH_MAXQ(c.nq, L_DR);
#undef L_DR
        check_launch("decrypt_round");
    });
}

int kbfv_delta_m(kbfv_context* ctx, const uint64_t* d_m, uint64_t* d_out, uint32_t polys, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        const size_t total = (size_t)polys * c.nq * c.n;
        if (!total) return;
        delta_m_kernel<<<blocks_for(total, 256), 256, 0, S(stream)>>>(c.dc, d_m, d_out, total);
        check_launch("delta_m");
    });
}

int kbfv_modup(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!polys) return;
        dim3 grid((unsigned)(c.n / 128), polys);
#define L_MU(M) modup_kernel<M><<<grid, 128, 0, S(stream)>>>(c.dc, d_in, d_out)
        DISPATCH_MAXQ(c.nq, L_MU);
#undef L_MU
        check_launch("modup");
    });
}

int kbfv_moddown(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!polys) return;
        dim3 grid((unsigned)(c.n / 128), polys);
        moddown_kernel<<<grid, 128, 0, S(stream)>>>(c.dc, d_in, d_out);
        check_launch("moddown");
    });
}

static int ntt_batch(kbfv_context* ctx, uint64_t* const* d_polys, uint32_t count, uint32_t limbs, uint32_t prime0,
                     kbfv_stream stream, bool fwd) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_polys || !count, KBFV_ERR_INVALID, "null pointer array");
        KB_REQUIRE(limbs >= 1 && prime0 + limbs <= c.mods.size(), KBFV_ERR_INVALID, "prime range out of table");
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            PtrBatch pb{};
            for (int i = 0; i < cnt; i++) {
                KB_REQUIRE(d_polys[off + i], KBFV_ERR_INVALID, "null polynomial pointer");
                pb.o[i] = d_polys[off + i];
            }
            PtrPolysIO io{pb, c.logn, (int)limbs, (int)prime0};
            if (fwd) ntt_fwd(c.dc, io, io, cnt * (int)limbs, S(stream));
            else ntt_inv(c.dc, io, io, cnt * (int)limbs, S(stream));
        }
    });
}

int kbfv_ntt_fwd_batch(kbfv_context* ctx, uint64_t* const* d_polys, uint32_t count, uint32_t limbs, uint32_t prime0,
                       kbfv_stream stream) {
    return ntt_batch(ctx, d_polys, count, limbs, prime0, stream, true);
}

int kbfv_ntt_inv_batch(kbfv_context* ctx, uint64_t* const* d_polys, uint32_t count, uint32_t limbs, uint32_t prime0,
                       kbfv_stream stream) {
    return ntt_batch(ctx, d_polys, count, limbs, prime0, stream, false);
}

}  // extern "C"
