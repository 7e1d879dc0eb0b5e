// libkbfv: the fused batched multiply + relinearise pipeline (HPS tensor and
// hybrid key switch), its entry points on device and host memory, and the
// allocation-free variant.
#include <cuda.h>

#include "pipeline.cuh"

// Key-switch tail over NTT-form digits (sd2, [item][ndig][npq]) and a key
// ([ndig][2][Q|P] of the top level), written to the outputs of pb:
//   out_h = add_h + P^-1 (x_h,Q - [x_h,P]_Q),  x_h = sum_d digit_d * key_d[h].
// Only the P limbs of x are brought back to coefficient form (inverse NTT over
// P, the key product fused into its loads) for the conversion to Q. The Q limbs
// stay in the NTT domain, where the forward NTT's store adds them:
//   NTT(add - P^-1 [x_P]_Q) + P^-1 x_Q,  with x_Q computed at the store.
void ks_tail(const DevConsts& dc, const uint64_t* sd2, const uint64_t* key, int ndig, uint64_t* se,
                    const uint64_t* add, const PtrBatch& pb, int count, cudaStream_t st) {
    ntt_inv(dc, KeyIPSrc{sd2, key, dc, ndig, dc.nq, dc.np}, SeRowsP{se, dc.logn, dc.nq, dc.np, dc.npq},
            count * 2 * dc.np, st);
    const OutCtKeyDst dst{pb, sd2, key, dc, ndig};
    if (dc.np == 1)
        ntt_fwd(dc, ModDownAdd1Src{se, add, dc, true}, dst, count * 2 * dc.nq, st);
    else
        ntt_fwd(dc, ModDownAddSrc{se, add, dc, true}, dst, count * 2 * dc.nq, st);
}

void mul_front(const DevConsts& dc, const PtrBatch& pb, int count, const MulScratch& m, cudaStream_t st) {
    if (count <= dc.shape.fuse_q2r_pairs) {
        // K1 stores y_i = [x_i (Q/q_i)^-1]_{q_i}; K3's loader extends them to R
        ntt_inv(dc, PairQRowsP{pb, dc.logn, dc.nq}, QHatRowsIO{m.sa, dc.logn, dc.nq, dc.q2r_fold},
                count * 4 * dc.nq, st);
#define L_Q2R(M) q2r_ntt_launch_m<M>(dc, m.sa, m.sb, count * 4, st)
        DISPATCH_MAXQ(dc.nq, L_Q2R);
#undef L_Q2R
    } else {
        // K1: INTT over Q of [a1, b1, a2, b2]
        ntt_inv(dc, PairQRowsP{pb, dc.logn, dc.nq}, rows_io(dc, m.sa, 0, dc.nq), count * 4 * dc.nq, st);
        // K2: Q -> R (centred)
        launch_bconv(dc, q2r_tables(dc), m.sa, m.sb, count * 4, (size_t)dc.nq << dc.logn, (size_t)dc.nr << dc.logn, st);
        // K3: NTT over R in place, fully reduced (the tensor's products use barrett_prod)
        ntt_fwd<RowsIO, RowsIO, true>(dc, rows_io(dc, m.sb, dc.idx_r, dc.nr), rows_io(dc, m.sb, dc.idx_r, dc.nr),
                                       count * 4 * dc.nr, st);
    }
    // K4: tensor (Q part from the NTT-form inputs, R part from K3) fused into INTT over Q|R
    TensorSrc ts{pb, m.sb, dc};
    ntt_inv(dc, ts, QRRowsIO{m.sc, dc.logn, dc.nq, dc.nqr, dc.idx_r}, count * 3 * dc.nqr, st);
}

void k5_launch(const DevConsts& dc, int count, const MulScratch& m, uint64_t* out0, int mode, cudaStream_t st) {
#define L_K5(M) k5_launch_m<M>(dc, count, m, out0, mode, st)
    DISPATCH_MAXQ(dc.nq + 1, L_K5);
#undef L_K5
}

void mul_relin_chunk(const DevConsts& dc, const uint64_t* rlk, const PtrBatch& pb, int count, const MulScratch& m,
                     cudaStream_t st) {
    mul_front(dc, pb, count, m, st);
    k5_launch(dc, count, m, nullptr, 1, st);
    // K6a: NTT over Q|P of the lifted digits, in place, fully reduced (key product uses barrett_prod)
    ntt_fwd<RowsIO, RowsIO, true>(dc, rows_io(dc, m.sd2, 0, dc.npq), rows_io(dc, m.sd2, 0, dc.npq),
                                   count * dc.dnum * dc.npq, st);
    // K6b: key product over P fused into INTT over P; K7: mod down + add (cross |
    // b1b2) fused into NTT over Q, the key product over Q added at its store
    ks_tail(dc, m.sd2, rlk, dc.dnum, m.se, m.sd, pb, count, st);
}

void ensure_branch_streams(Context& c) {
    if (c.fork_ev) return;
    for (int i = 0; i < 3; i++) {
        KB_CHECK_CUDA(cudaStreamCreateWithFlags(&c.aux[i], cudaStreamNonBlocking));
        KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.join_ev[i], cudaEventDisableTiming));
    }
    KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.fork_ev, cudaEventDisableTiming));
}

extern "C" {

int kbfv_mul(kbfv_context* ctx, const uint64_t* d_ct1, const uint64_t* d_ct2, uint64_t* d_tensor, uint32_t count,
             kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            std::vector<const uint64_t*> A(cnt), B(cnt);
            for (int i = 0; i < cnt; i++) {
                A[i] = d_ct1 + (size_t)(off + i) * 2 * lq;
                B[i] = d_ct2 + (size_t)(off + i) * 2 * lq;
            }
            PtrBatch pb = make_batch(A.data(), B.data(), nullptr, cnt);
            uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
            MulScratch m = mul_scratch_layout(c, cnt, base);
            uint64_t* out = d_tensor + (size_t)off * 3 * lq;
            const DevConsts dc = alone_consts(c);  // one stream: no sibling sub-batch fills the SMs
            mul_front(dc, pb, cnt, m, st);
            k5_launch(dc, cnt, m, out, 0, st);
            RowsIO io = rows_io(dc, out, 0, c.nq);
            ntt_fwd(dc, io, io, cnt * 3 * c.nq, st);
        }
    });
}

int kbfv_relinearize(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* d_tensor, uint64_t* d_ct, uint32_t count,
                     kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_rlk, KBFV_ERR_NO_KEY, "relinearisation key missing");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
            MulScratch m = mul_scratch_layout(c, cnt, base);
            const uint64_t* tz = d_tensor + (size_t)off * 3 * lq;
            uint64_t* out = d_ct + (size_t)off * 2 * lq;
            // INTT of a1*a2 into sa: rows (item, limb) read from the tensor's first poly
            ntt_inv(dc, TensorA2{tz, dc.logn, dc.nq}, rows_io(dc, m.sa, 0, dc.nq), cnt * dc.nq, st);
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
            ks_tail(dc, m.sd2, d_rlk, dc.dnum, m.se, nullptr, pb, cnt, st);
            // add [cross | b1b2] (NTT form)
            for (int i = 0; i < cnt; i++) {
                const size_t tot = 2 * lq;
                add_kernel<<<blocks_for(tot, 256), 256, 0, st>>>(dc, out + (size_t)i * 2 * lq, tz + (size_t)i * 3 * lq + lq,
                                                                 out + (size_t)i * 2 * lq, tot, dc.nq);
            }
            check_launch("relin_add");
        }
    });
}

int kbfv_mul_relin_batch(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* const* ct_a,
                         const uint64_t* const* ct_b, uint64_t* const* out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_rlk, KBFV_ERR_NO_KEY, "relinearisation key missing");
        KB_REQUIRE(ct_a && ct_b && out, KBFV_ERR_INVALID, "null pointer array");
        cudaStream_t st = S(stream);
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            for (int i = 0; i < cnt; i++)
                KB_REQUIRE(ct_a[off + i] && ct_b[off + i] && out[off + i], KBFV_ERR_INVALID, "null ciphertext pointer");
            const int nb = branch_count(c, cnt);
            if (nb == 1) {
                PtrBatch pb = make_batch(ct_a + off, ct_b + off, out + off, cnt);
                uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
                MulScratch m = mul_scratch_layout(c, cnt, base);
                mul_relin_chunk(alone_consts(c), d_rlk, pb, cnt, m, st);
                continue;
            }
            // sub-batches on the caller's stream and auxiliary streams, each with its
            // own scratch region, forked from and joined back into the caller's stream
            const int per = (cnt + nb - 1) / nb;
            const size_t each = branch_region_bytes(c, per);
            uint8_t* base = ensure_scratch(c, each * nb);
            ensure_branch_streams(c);
            KB_CHECK_CUDA(cudaEventRecord(c.fork_ev, st));
            for (int b = 1; b < nb; b++) KB_CHECK_CUDA(cudaStreamWaitEvent(c.aux[b - 1], c.fork_ev, 0));
            for (int b = 0; b < nb; b++) {
                const int lo = b * per, n = std::min(per, cnt - lo);
                if (n <= 0) break;
                PtrBatch pb = make_batch(ct_a + off + lo, ct_b + off + lo, out + off + lo, n);
                MulScratch m = mul_scratch_layout(c, n, base + b * each);
                mul_relin_chunk(c.dc, d_rlk, pb, n, m, b == 0 ? st : c.aux[b - 1]);
            }
            for (int b = 1; b < nb; b++) {
                KB_CHECK_CUDA(cudaEventRecord(c.join_ev[b - 1], c.aux[b - 1]));
                KB_CHECK_CUDA(cudaStreamWaitEvent(st, c.join_ev[b - 1], 0));
            }
        }
    });
}

int kbfv_mul_relin(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                   uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        const size_t lq = (size_t)c.nq * c.n;
        std::vector<const uint64_t*> A(count), B(count);
        std::vector<uint64_t*> O(count);
        for (uint32_t i = 0; i < count; i++) {
            A[i] = d_ct_a + (size_t)i * 2 * lq;
            B[i] = d_ct_b + (size_t)i * 2 * lq;
            O[i] = d_out + (size_t)i * 2 * lq;
        }
        int rc = kbfv_mul_relin_batch(ctx, d_rlk, A.data(), B.data(), O.data(), count, stream);
        if (rc != KBFV_OK) throw KbfvError(rc, g_last_error);
    });
}

// ---- multiply of ciphertexts held in host memory ----------------------------
// The pairs stream through kHostSlots device staging slots in chunks: chunk j's
// inputs are copied in on hs[0] while chunk j-1 is multiplied on hs[1 + (j-1)%2]
// and chunk j-2's products are copied out on hs[3]. Host-to-device and
// device-to-host copies use separate copy engines, so the step costs about the
// larger of the two copy times plus one chunk's multiply and copy-out.
constexpr int kHostSlots = 4;
static void ensure_host_streams(Context& c) {
    if (c.hfork) return;
    for (int i = 0; i < 4; i++) {
        KB_CHECK_CUDA(cudaStreamCreateWithFlags(&c.hs[i], cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&c.hjoin[i], &c.hin[i], &c.hcomp[i], &c.hout[i]})
            KB_CHECK_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.hfork, cudaEventDisableTiming));
}
// default chunk: about 32 MiB of input ciphertexts (8 pairs at N=16384 with 7
// primes, the fastest of 6-24 pairs on a B200 with PCIe 5 at ~55 GB/s each way)
static int host_chunk_default(const Context& c) {
    const size_t pair_bytes = (size_t)4 * c.nq * c.n * 8;
    return (int)std::max<size_t>(1, std::min<size_t>(kMaxBatch, ((size_t)32 << 20) / pair_bytes));
}
// chunk sizes for `count` pairs, none above `chunk`: the first two and the last
// three taper (chunk/4, chunk/2, ..., chunk/2, chunk/4, 1) so the first multiply
// waits for a short copy-in and the step ends with a short multiply and copy-out
static std::vector<int> host_chunks(uint32_t count, int chunk) {
    std::vector<int> head, tail, sizes;
    if (chunk >= 4) {
        head = {chunk / 4, chunk / 2};
        tail = {chunk / 2, chunk / 4, 1};
    }
    size_t ends = 0;
    for (int x : head) ends += x;
    for (int x : tail) ends += x;
    if (head.empty() || count < ends + (size_t)chunk) {
        head.clear();
        tail.clear();
        ends = 0;
    }
    sizes = head;
    for (size_t r = count - ends; r > 0;) {
        const int x = (int)std::min<size_t>(r, chunk);
        sizes.push_back(x);
        r -= x;
    }
    sizes.insert(sizes.end(), tail.begin(), tail.end());
    return sizes;
}

int kbfv_mul_relin_host(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* h_ct_a, const uint64_t* h_ct_b,
                        uint64_t* h_out, uint32_t count, uint32_t chunk_pairs, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_rlk, KBFV_ERR_NO_KEY, "relinearisation key missing");
        KB_REQUIRE(h_ct_a && h_ct_b && h_out, KBFV_ERR_INVALID, "null host buffer");
        KB_REQUIRE(chunk_pairs <= (uint32_t)kMaxBatch, KBFV_ERR_INVALID, "chunk_pairs must be 0..128");
        if (count == 0) return;
        const int want = chunk_pairs ? (int)chunk_pairs : c.host_chunk ? c.host_chunk : host_chunk_default(c);
        const int chunk = (int)std::min<uint32_t>(count, (uint32_t)want);
        const size_t ctw = (size_t)2 * c.nq * c.n;  // words of one ciphertext
        const size_t region = branch_region_bytes(c, chunk);
        const size_t slot_bytes = ((size_t)3 * chunk * ctw * 8 + 255) & ~(size_t)255;
        uint8_t* base = ensure_scratch(c, 2 * region + kHostSlots * slot_bytes);
        ensure_host_streams(c);
        cudaStream_t st = S(stream), h2d = c.hs[0], d2h = c.hs[3];
        KB_CHECK_CUDA(cudaEventRecord(c.hfork, st));
        for (int i = 0; i < 4; i++) KB_CHECK_CUDA(cudaStreamWaitEvent(c.hs[i], c.hfork, 0));
        // slot s: [a x chunk | b x chunk | out x chunk]
        auto slot = [&](int s) { return (uint64_t*)(base + 2 * region + (size_t)s * slot_bytes); };
        const std::vector<int> sizes = host_chunks(count, chunk);
        std::vector<size_t> first(sizes.size());  // first pair of each chunk
        for (size_t j = 1; j < sizes.size(); j++) first[j] = first[j - 1] + sizes[j - 1];
        auto copy_out = [&](size_t j) {
            const int s = (int)(j % kHostSlots);
            KB_CHECK_CUDA(cudaStreamWaitEvent(d2h, c.hcomp[s], 0));
            KB_CHECK_CUDA(cudaMemcpyAsync(h_out + first[j] * ctw, slot(s) + 2 * chunk * ctw,
                                          (size_t)sizes[j] * ctw * 8, cudaMemcpyDeviceToHost, d2h));
            KB_CHECK_CUDA(cudaEventRecord(c.hout[s], d2h));
        };
        const size_t chunks = sizes.size();
        std::vector<const uint64_t*> A(chunk), B(chunk);
        std::vector<uint64_t*> O(chunk);
        for (size_t j = 0; j < chunks; j++) {
            const int s = (int)(j % kHostSlots), k = (int)(j & 1), n = sizes[j];
            cudaStream_t comp = c.hs[1 + k];
            uint64_t* da = slot(s);
            uint64_t* db = da + chunk * ctw;
            uint64_t* dout = db + chunk * ctw;
            // the slot's inputs are free once the multiply of chunk j - kHostSlots read them
            if (j >= kHostSlots) KB_CHECK_CUDA(cudaStreamWaitEvent(h2d, c.hcomp[s], 0));
            const size_t off = first[j] * ctw, bytes = (size_t)n * ctw * 8;
            KB_CHECK_CUDA(cudaMemcpyAsync(da, h_ct_a + off, bytes, cudaMemcpyHostToDevice, h2d));
            KB_CHECK_CUDA(cudaMemcpyAsync(db, h_ct_b + off, bytes, cudaMemcpyHostToDevice, h2d));
            KB_CHECK_CUDA(cudaEventRecord(c.hin[s], h2d));
            KB_CHECK_CUDA(cudaStreamWaitEvent(comp, c.hin[s], 0));
            // ... and its products once chunk j - kHostSlots was copied out
            if (j >= kHostSlots) KB_CHECK_CUDA(cudaStreamWaitEvent(comp, c.hout[s], 0));
            for (int i = 0; i < n; i++) {
                A[i] = da + i * ctw;
                B[i] = db + i * ctw;
                O[i] = dout + i * ctw;
            }
            PtrBatch pb = make_batch(A.data(), B.data(), O.data(), n);
            MulScratch m = mul_scratch_layout(c, n, base + k * region);
            mul_relin_chunk(c.dc, d_rlk, pb, n, m, comp);
            KB_CHECK_CUDA(cudaEventRecord(c.hcomp[s], comp));
            if (j >= 1) copy_out(j - 1);
        }
        copy_out(chunks - 1);
        for (int i = 0; i < 4; i++) {
            KB_CHECK_CUDA(cudaEventRecord(c.hjoin[i], c.hs[i]));
            KB_CHECK_CUDA(cudaStreamWaitEvent(st, c.hjoin[i], 0));
        }
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// allocation-free multiply: scratch in a static device array
// ---------------------------------------------------------------------------
static __device__ __align__(256) uint8_t g_noalloc_scratch[KBFV_NOALLOC_SCRATCH_BYTES];

// The array's device address is a property of the CUDA context that loaded
// the library's module, not of the device ordinal: a device reset, or another
// context made current on the same device, loads the module again at another
// address. So the address is resolved once per context, keyed by the driver's
// process-unique context id (a handle value can be reused after a reset; the
// id is not). The driver calls come through the runtime's entry-point query,
// so the library needs no link-time dependency on libcuda.
struct NoallocSlot {
    unsigned long long ctx_id;
    void* addr;
};
constexpr int kNoallocSlots = 64;
static NoallocSlot g_noalloc_slots[kNoallocSlots];
static int g_noalloc_used = 0, g_noalloc_next = 0;
static std::mutex g_noalloc_mu;

template <class Fn>
static Fn driver_entry(const char* name) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion(name, &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
        p = nullptr;
    return (Fn)p;
}

static unsigned long long current_context_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static const GetCurrent get_current = driver_entry<GetCurrent>("cuCtxGetCurrent");
    static const GetId get_id = driver_entry<GetId>("cuCtxGetId");
    KB_REQUIRE(get_current && get_id, KBFV_ERR_CUDA, "driver entry points cuCtxGetCurrent / cuCtxGetId unavailable");
    CUcontext cx = nullptr;
    unsigned long long id = 0;
    KB_REQUIRE(get_current(&cx) == CUDA_SUCCESS && cx, KBFV_ERR_CUDA, "no current CUDA context");
    KB_REQUIRE(get_id(cx, &id) == CUDA_SUCCESS, KBFV_ERR_CUDA, "cuCtxGetId failed");
    return id;
}

// Device address of the static scratch in the current context: looked up in a
// fixed table (no allocation), resolved with cudaGetSymbolAddress the first
// time a context is seen (the host-side symbol is only a handle, never a
// device address). With lazy module loading that first resolution also loads
// the module if no multiply kernel has run in the context yet.
static uint8_t* noalloc_scratch() {
    const unsigned long long id = current_context_id();
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    for (int i = 0; i < g_noalloc_used; i++)
        if (g_noalloc_slots[i].ctx_id == id) return (uint8_t*)g_noalloc_slots[i].addr;
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        throw KbfvError(KBFV_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
    const int slot = g_noalloc_used < kNoallocSlots ? g_noalloc_used++ : (g_noalloc_next++ % kNoallocSlots);
    g_noalloc_slots[slot] = NoallocSlot{id, p};
    return (uint8_t*)p;
}

extern "C" {

int kbfv_mul_relin_noalloc(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                           uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_rlk, KBFV_ERR_NO_KEY, "relinearisation key missing");
        KB_REQUIRE(d_ct_a && d_ct_b && d_out, KBFV_ERR_INVALID, "null ciphertext pointer");
        if (count == 0) return;
        KB_REQUIRE(count <= (uint32_t)kMaxBatch, KBFV_ERR_INVALID, "too many pairs for one allocation-free call");
        const size_t need = mul_scratch_layout(c, (int)count, nullptr).bytes;
        if (need > KBFV_NOALLOC_SCRATCH_BYTES)
            throw KbfvError(KBFV_ERR_INVALID, "kbfv_mul_relin_noalloc: " + std::to_string(count) + " pair(s) need " +
                                                  std::to_string(need) + " bytes of scratch; the static array holds " +
                                                  std::to_string((size_t)KBFV_NOALLOC_SCRATCH_BYTES));
        int dev = -1;
        KB_CHECK_CUDA(cudaGetDevice(&dev));
        KB_REQUIRE(dev == c.device, KBFV_ERR_INVALID, "the context's device is not current");
        MulScratch m = mul_scratch_layout(c, (int)count, noalloc_scratch());
        // every scratch word is written before it is read: nothing to clear
        PtrBatch pb;
        std::memset(&pb, 0, sizeof pb);
        const size_t stride = (size_t)2 * c.nq * c.n;
        for (uint32_t i = 0; i < count; i++) {
            pb.a[i] = d_ct_a + i * stride;
            pb.b[i] = d_ct_b + i * stride;
            pb.o[i] = d_out + i * stride;
        }
        mul_relin_chunk(c.dc, d_rlk, pb, (int)count, m, S(stream));
    });
}

}  // extern "C"
