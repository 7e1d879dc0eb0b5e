// Native timing of the multiply's per-call forms through the C ABI, with no
// interpreter between calls (bench.py runs it beside its own measurements):
//
//   perop_bench [pairs] [reps]
//
// N = 16384, 7 x 60-bit ciphertext primes + 1 special prime, t = 65537, dnum 1.
// Prints one JSON line with, per pair: the fused one-pair call (kbfv_mul_relin,
// count 1), the same call replayed from a captured plan (kbfv_plan_launch of a
// one-pair plan bound to fixed buffers), the plain form (one kernel per
// building block: INTT, Q -> R, NTT, copies into the Q|R layout, tensor, six
// INTTs, scale-and-round, R -> Q, NTT, then kbfv_relinearize), and the batched
// call over all pairs. Each form runs `reps` timed rounds after one warm-up
// round (CUDA events on one stream); the plan's and the plain form's products
// of the first pair are compared with the fused one's.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "../../include/kbfv.h"

static void ok(int rc, const char* what) {
    if (rc != KBFV_OK) {
        std::fprintf(stderr, "%s: %d %s\n", what, rc, kbfv_last_error());
        std::exit(1);
    }
}
static void cu(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        std::exit(1);
    }
}
static uint64_t* dalloc(size_t words) {
    uint64_t* p = nullptr;
    cu(cudaMalloc(&p, words * 8), "cudaMalloc");
    return p;
}

int main(int argc, char** argv) {
    const int pairs = argc > 1 ? std::atoi(argv[1]) : 64;
    const int reps = argc > 2 ? std::atoi(argv[2]) : 3;
    if (pairs < 1 || pairs > 128 || reps < 1) {
        std::fprintf(stderr, "usage: perop_bench [pairs 1..128] [reps >= 1]\n");
        return 2;
    }
    const uint32_t qb[7] = {60, 60, 60, 60, 60, 60, 60}, pb[1] = {60};
    kbfv_params* prm = nullptr;
    ok(kbfv_params_create(14, qb, 7, pb, 1, 65537, 1, &prm), "params");
    kbfv_context* ctx = nullptr;
    ok(kbfv_context_create(prm, &ctx), "context");
    kbfv_params_destroy(prm);
    uint64_t n64 = 0;
    uint32_t nq = 0, np = 0, nr = 0, nt = 0, dnum = 0, alpha = 0;
    ok(kbfv_context_info(ctx, &n64, &nq, &np, &nr, &nt, &dnum, &alpha), "info");
    const size_t N = n64, npq = nq + np, nqr = nq + nr, ctw = 2 * nq * N;
    const uint32_t idx_r = nq + np;
    cudaStream_t st;
    cu(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
    kbfv_stream S = (kbfv_stream)st;

    uint8_t seed[32];
    for (int i = 0; i < 32; i++) seed[i] = (uint8_t)(17 * i + 5);
    uint64_t* sk = dalloc(npq * N);
    uint64_t* pk = dalloc(2 * nq * N);
    uint64_t* rlk = dalloc((size_t)dnum * 2 * npq * N);
    ok(kbfv_keygen_secret(ctx, seed, 0, 64, sk, S), "keygen secret");
    ok(kbfv_keygen_public(ctx, seed, sk, pk, S), "keygen public");
    ok(kbfv_keygen_relin(ctx, seed, sk, rlk, S), "keygen relin");
    std::vector<uint64_t> slots((size_t)2 * pairs * N);
    uint64_t x = 88172645463325252ULL;
    for (auto& v : slots) {  // xorshift64: uniform slots mod t
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        v = x % 65537;
    }
    uint64_t* d_slots = dalloc(slots.size());
    uint64_t* d_m = dalloc(slots.size());
    cu(cudaMemcpy(d_slots, slots.data(), slots.size() * 8, cudaMemcpyHostToDevice), "copy slots");
    ok(kbfv_encode(ctx, d_slots, d_m, 2 * pairs, S), "encode");
    uint64_t* a = dalloc(pairs * ctw);
    uint64_t* b = dalloc(pairs * ctw);
    uint64_t* o = dalloc(pairs * ctw);
    ok(kbfv_encrypt(ctx, seed, 0, pk, d_m, a, pairs, S), "encrypt a");
    ok(kbfv_encrypt(ctx, seed, 1000, pk, d_m + (size_t)pairs * N, b, pairs, S), "encrypt b");
    ok(kbfv_reserve(ctx, pairs), "reserve");

    cudaEvent_t e0, e1;
    cu(cudaEventCreate(&e0), "event");
    cu(cudaEventCreate(&e1), "event");
    auto timed = [&](auto&& round) {
        round();  // warm-up
        cu(cudaStreamSynchronize(st), "sync");
        cu(cudaEventRecord(e0, st), "record");
        for (int r = 0; r < reps; r++) round();
        cu(cudaEventRecord(e1, st), "record");
        cu(cudaEventSynchronize(e1), "sync");
        float ms = 0.f;
        cu(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        return (double)ms / reps;
    };

    // fused pipeline, one pair per call
    const double fused_ms = timed([&] {
        for (int i = 0; i < pairs; i++)
            ok(kbfv_mul_relin(ctx, rlk, a + i * ctw, b + i * ctw, o + i * ctw, 1, S), "mul_relin");
    });
    std::vector<uint64_t> want(ctw), got(ctw);
    cu(cudaStreamSynchronize(st), "sync");
    cu(cudaMemcpy(want.data(), o, ctw * 8, cudaMemcpyDeviceToHost), "copy product");

    // captured plan: one pair bound to fixed buffers (pair 0), replayed per call
    uint64_t* po1 = dalloc(ctw);
    kbfv_plan* plan = nullptr;
    ok(kbfv_plan_mul_relin(ctx, rlk, a, b, po1, 1, &plan), "plan");
    const double plan_ms = timed([&] {
        for (int i = 0; i < pairs; i++) ok(kbfv_plan_launch(plan, S), "plan launch");
    });
    cu(cudaStreamSynchronize(st), "sync");
    cu(cudaMemcpy(got.data(), po1, ctw * 8, cudaMemcpyDeviceToHost), "copy product");
    const bool plan_matches = std::memcmp(got.data(), want.data(), ctw * 8) == 0;
    uint64_t plan_launches = 0, plan_captures = 0;
    ok(kbfv_plan_info(plan, &plan_launches, &plan_captures), "plan info");
    ok(kbfv_plan_destroy(plan), "plan destroy");

    // plain: one kernel per building block
    uint64_t* x4 = dalloc(4 * nq * N);
    uint64_t* r4 = dalloc(4 * nr * N);
    uint64_t* qr = dalloc(2 * 2 * nqr * N);
    uint64_t* tz = dalloc(3 * nqr * N);
    uint64_t* sr = dalloc(3 * nr * N);
    uint64_t* d3 = dalloc(3 * nq * N);
    uint64_t* po = dalloc(2 * nq * N);
    auto cp = [&](uint64_t* dst, const uint64_t* src, size_t words) {
        cu(cudaMemcpyAsync(dst, src, words * 8, cudaMemcpyDeviceToDevice, st), "copy");
    };
    auto plain_pair = [&](int i, uint64_t* out) {
        const uint64_t* A = a + i * ctw;
        const uint64_t* B = b + i * ctw;
        cp(x4, A, 2 * nq * N);
        cp(x4 + 2 * nq * N, B, 2 * nq * N);
        ok(kbfv_ntt_inv(ctx, x4, 4 * nq, 0, nq, S), "intt");
        ok(kbfv_bconv_q_to_r(ctx, x4, r4, 4, S), "q->r");
        ok(kbfv_ntt_fwd(ctx, r4, 4 * nr, idx_r, nr, S), "ntt r");
        for (int c = 0; c < 2; c++)
            for (int p = 0; p < 2; p++) {
                uint64_t* poly = qr + ((size_t)(c * 2 + p) * nqr) * N;
                cp(poly, (c == 0 ? A : B) + p * nq * N, nq * N);
                cp(poly + nq * N, r4 + (size_t)(c * 2 + p) * nr * N, nr * N);
            }
        ok(kbfv_tensor_qr(ctx, qr, qr + 2 * nqr * N, tz, 1, S), "tensor");
        for (int k = 0; k < 3; k++) {
            ok(kbfv_ntt_inv(ctx, tz + k * nqr * N, nq, 0, nq, S), "intt q");
            ok(kbfv_ntt_inv(ctx, tz + (k * nqr + nq) * N, nr, idx_r, nr, S), "intt r");
        }
        ok(kbfv_scale_round_qr_r(ctx, tz, sr, 3, S), "scale-round");
        ok(kbfv_bconv_r_to_q(ctx, sr, d3, 3, S), "r->q");
        ok(kbfv_ntt_fwd(ctx, d3, 3 * nq, 0, nq, S), "ntt q");
        ok(kbfv_relinearize(ctx, rlk, d3, out, 1, S), "relinearize");
    };
    const double plain_ms = timed([&] {
        for (int i = 0; i < pairs; i++) plain_pair(i, po);
    });
    plain_pair(0, po);
    cu(cudaStreamSynchronize(st), "sync");  // st does not synchronise with the legacy default stream
    cu(cudaMemcpy(got.data(), po, ctw * 8, cudaMemcpyDeviceToHost), "copy product");
    const bool plain_matches = std::memcmp(got.data(), want.data(), ctw * 8) == 0;

    // batched: all pairs in one call
    const double batch_ms = timed([&] { ok(kbfv_mul_relin(ctx, rlk, a, b, o, pairs, S), "mul_relin batch"); });

    std::printf("{\"pairs\": %d, \"reps\": %d, \"fused_per_call_ms_per_pair\": %.5f, "
                "\"plan_per_call_ms_per_pair\": %.5f, "
                "\"plain_per_op_ms_per_pair\": %.5f, \"batched_ms_per_call\": %.5f, "
                "\"fused_per_call_ct_per_s\": %.1f, \"plan_per_call_ct_per_s\": %.1f, "
                "\"plain_per_op_ct_per_s\": %.1f, \"batched_ct_per_s\": %.1f, "
                "\"plain_matches_fused\": %s, \"plan_matches_fused\": %s, \"plan_captures\": %llu}\n",
                pairs, reps, fused_ms / pairs, plan_ms / pairs, plain_ms / pairs, batch_ms, pairs / fused_ms * 1e3,
                pairs / plan_ms * 1e3, pairs / plain_ms * 1e3, pairs / batch_ms * 1e3,
                plain_matches ? "true" : "false", plan_matches ? "true" : "false",
                (unsigned long long)plan_captures);
    for (uint64_t* p : {sk, pk, rlk, d_slots, d_m, a, b, o, x4, r4, qr, tz, sr, d3, po, po1}) cudaFree(p);
    kbfv_context_destroy(ctx);
    return plain_matches && plan_matches ? 0 : 1;
}
