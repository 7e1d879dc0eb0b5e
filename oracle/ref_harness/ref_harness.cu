// Reference-kernel harness (test infrastructure).
//
// Compiles kunpBFV's own headers, where they lie, for sm_100a and runs its
// kernels and launchers on seeded inputs, writing a manifest line (length,
// 64-bit digest, first values) for every input and output. The committed script
// tests/golden/make_ref_fixtures.py turns one run into the fixtures that
// pin the CPU oracle. Build: `make -C oracle ref` (nvcc; NTL replaced by the
// header in ntl_shim/, which covers the context precompute's big-integer use).
//
// Only calls that are safe to run are made: the reference's encryptMsg /
// addConstAndEqual pass a host std::vector pointer to a kernel
// (include/BFVScheme.cuh:138), so the harness launches that kernel itself
// with a device copy of the moduli.
//
// Usage: ref_harness <logN 14|15> <outdir> [raw_limit_words] [time_reps]
// With time_reps > 0 it also times the genuine multiply (one pair per call,
// CUDA events) and prints {"logN", "reps", "ms_per_mult"} on stdout.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "include/Plaintext.cuh"
#include "include/Ciphertext.cuh"
#include "include/BFVScheme.cuh"
#include "include/BFVcontext.cuh"

static std::string g_out;
static FILE* g_manifest = nullptr;

static void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "CUDA error at %s: %s\n", what, cudaGetErrorString(e));
        exit(2);
    }
}

static uint64_tt splitmix(uint64_tt& s) {
    uint64_tt z = (s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// limb l of a seeded input: N draws of splitmix64 from state (seed << 20) + l, reduced mod mods[l]
static std::vector<uint64_tt> gen(uint64_tt seed, const std::vector<uint64_tt>& mods, size_t N) {
    std::vector<uint64_tt> v(mods.size() * N);
    for (size_t l = 0; l < mods.size(); l++) {
        uint64_tt s = (seed << 20) + l;
        for (size_t k = 0; k < N; k++) v[l * N + k] = splitmix(s) % mods[l];
    }
    return v;
}

// Order-dependent 64-bit digest: sum over i of mix(x_i ^ (i * gamma)), mix being
// splitmix64's finaliser. tests/golden/refgen.py computes the same digest.
static uint64_tt mix64(uint64_tt z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Writes one manifest line per array: name, length, digest, first 8 values.
// Arrays up to `g_raw_limit` words are also written raw (<name>.bin).
static size_t g_raw_limit = 0;
static int g_time_reps = 0;  // > 0: also time the genuine multiply over this many calls
static void dump_host(const std::string& name, const uint64_tt* p, size_t count) {
    uint64_tt h = 0;
    for (size_t i = 0; i < count; i++) h += mix64(p[i] ^ ((uint64_tt)i * 0x9E3779B97F4A7C15ULL));
    fprintf(g_manifest, "%s %zu %llu", name.c_str(), count, (unsigned long long)h);
    for (size_t i = 0; i < 8 && i < count; i++) fprintf(g_manifest, " %llu", (unsigned long long)p[i]);
    fprintf(g_manifest, "\n");
    if (count <= g_raw_limit) {
        std::string path = g_out + "/" + name + ".bin";
        FILE* f = fopen(path.c_str(), "wb");
        fwrite(p, 8, count, f);
        fclose(f);
    }
}

static void dump_dev(const std::string& name, const uint64_tt* d, size_t count) {
    std::vector<uint64_tt> h(count);
    ck(cudaDeviceSynchronize(), name.c_str());
    ck(cudaMemcpy(h.data(), d, count * 8, cudaMemcpyDeviceToHost), name.c_str());
    dump_host(name, h.data(), count);
}

static uint64_tt* up(const std::vector<uint64_tt>& v) {
    uint64_tt* d;
    ck(cudaMalloc(&d, v.size() * 8), "malloc");
    ck(cudaMemcpy(d, v.data(), v.size() * 8, cudaMemcpyHostToDevice), "upload");
    return d;
}

static std::vector<uint64_tt> rep(const std::vector<uint64_tt>& m, int times) {
    std::vector<uint64_tt> r;
    for (int i = 0; i < times; i++) r.insert(r.end(), m.begin(), m.end());
    return r;
}

int main(int argc, char** argv) {
    if (argc < 3) {
        fprintf(stderr, "usage: %s <logN> <outdir>\n", argv[0]);
        return 1;
    }
    const int logN = atoi(argv[1]);
    g_out = argv[2];
    g_manifest = fopen((g_out + "/manifest.txt").c_str(), "w");
    g_raw_limit = argc > 3 ? (size_t)atoll(argv[3]) : 64;
    g_time_reps = argc > 4 ? atoi(argv[4]) : 0;
    const size_t N = (size_t)1 << logN;

    BFVContext context(N);
    BFVScheme scheme(context);
    SecretKey sk(context);
    scheme.mallocMemory();
    scheme.addEncKey(sk);
    scheme.addMultKey_23(sk);
    ck(cudaDeviceSynchronize(), "setup");

    const int L = context.L, K = context.K, t_num = context.t_num;
    const int q_num = context.q_num, r_num = context.r_num, dnum = context.dnum;
    const int Ri = context.Ri_blockNum, Qj = context.Qj_blockNum;
    std::vector<uint64_tt> info = {(uint64_tt)logN, context.plain_modulus, (uint64_tt)q_num, (uint64_tt)K,
                                  (uint64_tt)t_num, (uint64_tt)r_num, (uint64_tt)dnum, (uint64_tt)context.gamma,
                                  (uint64_tt)Ri, (uint64_tt)Qj, context.plainModPsi};
    dump_host("info", info.data(), info.size());
    dump_host("qVec", context.qVec.data(), context.qVec.size());
    dump_host("pVec", context.pVec.data(), context.pVec.size());
    dump_host("tVec", context.tVec.data(), context.tVec.size());
    dump_host("rVec", context.rVec.data(), context.rVec.size());
    dump_host("pqtPsi", context.pqtPsi.data(), context.pqtPsi.size());
    dump_host("qrPsi", context.qrPsi.data(), context.qrPsi.size());

    const std::vector<uint64_tt>& pqt = context.pqtVec;  // [P | Q | T]
    const std::vector<uint64_tt>& qr = context.qrVec;    // [Q | R]
    const std::vector<uint64_tt> Q(context.qVec), R(context.rVec), T(context.tVec);
    std::vector<uint64_tt> PQ(pqt.begin(), pqt.begin() + K + q_num);
    const int npqt = (int)pqt.size(), nqr = (int)qr.size();

    // ---- NTT over P|Q|T (ToNTTInplace / FromNTTInplace, BFVcontext.cuh:1513-1552)
    {
        auto x = gen(1, pqt, N);
        dump_host("ntt_pqt_in", x.data(), x.size());
        uint64_tt* d = up(x);
        context.ToNTTInplace(d, 0, 0, 1, npqt, npqt);
        dump_dev("ntt_pqt_out", d, x.size());
        auto y = gen(2, pqt, N);
        dump_host("intt_pqt_in", y.data(), y.size());
        ck(cudaMemcpy(d, y.data(), y.size() * 8, cudaMemcpyHostToDevice), "up");
        context.FromNTTInplace(d, 0, 0, 1, npqt, npqt);
        dump_dev("intt_pqt_out", d, y.size());
        cudaFree(d);
    }
    // ---- NTT over Q|R (BFVcontext.cuh:1719-1757)
    {
        auto x = gen(3, qr, N);
        dump_host("ntt_qr_in", x.data(), x.size());
        uint64_tt* d = up(x);
        context.ToNTTInplace_for_QR(d, 0, 0, 1, nqr, nqr);
        dump_dev("ntt_qr_out", d, x.size());
        auto y = gen(4, qr, N);
        dump_host("intt_qr_in", y.data(), y.size());
        ck(cudaMemcpy(d, y.data(), y.size() * 8, cudaMemcpyHostToDevice), "up");
        context.FromNTTInplace_for_QR(d, 0, 0, 1, nqr, nqr);
        dump_dev("intt_qr_out", d, y.size());
        cudaFree(d);
    }
    // ---- NTT mod t (encode / decode transforms, BFVcontext.cuh:1634-1677)
    {
        std::vector<uint64_tt> tm = {context.plain_modulus};
        auto x = gen(5, tm, N);
        dump_host("bfv_enc_in", x.data(), x.size());
        uint64_tt* d = up(x);
        context.FromNTTInplace_for_BFV(d, 0, 0, 0, 0, 1);
        dump_dev("bfv_enc_out", d, N);
        auto y = gen(6, tm, N);
        dump_host("bfv_dec_in", y.data(), y.size());
        ck(cudaMemcpy(d, y.data(), N * 8, cudaMemcpyHostToDevice), "up");
        context.ToNTTInplace_for_BFV(d, 0, 0, 0, 0, 1);
        dump_dev("bfv_dec_out", d, N);
        cudaFree(d);
    }
    // ---- HPS base conversions (BasisConv_QR.cuh:191-207)
    {
        auto x = gen(7, Q, N);
        dump_host("bconv_qr_in", x.data(), x.size());
        uint64_tt* d = up(x);
        uint64_tt* o;
        ck(cudaMalloc(&o, r_num * N * 8), "m");
        context.QtoR.bConv_HPS(o, d, N, 0);
        dump_dev("bconv_qr_out", o, r_num * N);
        auto y = gen(8, R, N);
        dump_host("bconv_rq_in", y.data(), y.size());
        uint64_tt* d2 = up(y);
        uint64_tt* o2;
        ck(cudaMalloc(&o2, q_num * N * 8), "m");
        context.RtoQ.bConv_HPS(o2, d2, N, 0);
        dump_dev("bconv_rq_out", o2, q_num * N);
    }
    // ---- t/Q scale-and-round Q|R -> R (poly_arithmetic.cuh:1263-1316)
    {
        auto x = gen(9, qr, N);
        dump_host("sr_in", x.data(), x.size());
        uint64_tt* d = up(x);
        uint64_tt* o;
        ck(cudaMalloc(&o, r_num * N * 8), "m");
        scaleAndRound_HPS_QR_R(o, d, context.RtoQ.get_ibase(), context.RtoQ.get_ibase_Mu_high(),
                               context.RtoQ.get_ibase_Mu_low(), context.tRSHatInvModsDivsModr_,
                               context.tRSHatInvModsDivsFrac_, q_num, r_num, N, 0);
        dump_dev("sr_out", o, r_num * N);
    }
    // ---- decrypt scale-and-round (BFVcontext.cuh:1680-1717); first limb of the output
    {
        auto x = gen(10, Q, N);
        dump_host("decr_in", x.data(), x.size());
        uint64_tt* d = up(x);
        uint64_tt* o;
        ck(cudaMalloc(&o, q_num * N * 8), "m");
        ck(cudaMemset(o, 0, q_num * N * 8), "z");
        context.hps_decrypt_scale_and_round(o, d, 0);
        dump_dev("decr_out", o, N);
    }
    // ---- tensor over Q|R (poly_arithmetic.cuh:1180-1219)
    {
        auto a = gen(11, rep(qr, 2), N), b = gen(12, rep(qr, 2), N);
        dump_host("tensor_in1", a.data(), a.size());
        dump_host("tensor_in2", b.data(), b.size());
        uint64_tt *da = up(a), *db = up(b), *o;
        ck(cudaMalloc(&o, 3 * nqr * N * 8), "m");
        uint64_tt grid = N * nqr / blockDimGlb.x;
        tensor_prod_2x2_rns_poly<<<grid, blockDimGlb>>>(da, db, context.QR_mod, context.QR_Mu_high,
                                                       context.QR_Mu_low, o, N, nqr);
        dump_dev("tensor_out", o, 3 * nqr * N);
    }
    // ---- delta * m (poly_arithmetic.cuh:902-927) with a device copy of the moduli
    {
        std::vector<uint64_tt> tm = {context.plain_modulus};
        auto m = gen(13, tm, N);
        dump_host("delta_in", m.data(), N);
        std::vector<uint64_tt> mm = rep(m, q_num);
        uint64_tt* d = up(mm);
        uint64_tt* dq = up(Q);
        uint64_tt grid = N * q_num / blockDimGlb.x;
        bfv_add_timesQ_overt_kernel<<<grid, blockDimGlb>>>(d, d, context.negQl_mod_t, context.negQl_mod_t_shoup,
                                                          context.tInv_mod_q, context.tInv_mod_q_shoup, dq,
                                                          context.plain_modulus, N, q_num);
        dump_dev("delta_out", d, q_num * N);
    }
    // ---- KLSS key-switch conversions (BasisConv.cuh, ExternalProduct.cuh)
    {
        auto x = gen(14, Q, N);
        dump_host("modup_qj_t_in", x.data(), x.size());
        uint64_tt* d = up(x);
        uint64_tt* o;
        ck(cudaMalloc(&o, Qj * t_num * N * 8), "m");
        context.modUpQjtoT_23(o, d, L, 1);
        dump_dev("modup_qj_t_out", o, Qj * t_num * N);

        auto y = gen(15, PQ, N);
        dump_host("modup_pq_t_in", y.data(), y.size());
        uint64_tt* dy = up(y);
        uint64_tt* oy;
        ck(cudaMalloc(&oy, Ri * t_num * N * 8), "m");
        context.modUpPQtoT_23(oy, dy, L, 1);
        dump_dev("modup_pq_t_out", oy, Ri * t_num * N);

        auto dg = gen(16, rep(T, Qj), N);
        auto key = gen(17, rep(T, 2 * dnum * Ri), N);
        dump_host("extprod_digits", dg.data(), dg.size());
        dump_host("extprod_key", key.data(), key.size());
        uint64_tt *ddg = up(dg), *dkey = up(key), *oe;
        ck(cudaMalloc(&oe, 2 * Ri * t_num * N * 8), "m");
        context.external_product_T(oe, ddg, dkey, L);
        dump_dev("extprod_out", oe, 2 * Ri * t_num * N);

        auto z = gen(18, rep(T, 2 * Ri), N);
        dump_host("modup_t_pq_in", z.data(), z.size());
        uint64_tt* dz = up(z);
        uint64_tt* oz;
        ck(cudaMalloc(&oz, 2 * Ri * t_num * N * 8), "m");
        ck(cudaMemset(oz, 0, 2 * Ri * t_num * N * 8), "z");
        context.modUpTtoPQl_23(oz, dz, L, 2);
        dump_dev("modup_t_pq_out", oz, 2 * Ri * t_num * N);

        // mod down: per cipher Ri*t_num limbs whose first K+L+1 hold [P | Q] values
        std::vector<uint64_tt> md(2 * Ri * t_num * N, 0);
        auto pqv = gen(19, rep(PQ, 2), N);
        for (int c = 0; c < 2; c++)
            for (size_t i = 0; i < PQ.size() * N; i++) md[c * Ri * t_num * N + i] = pqv[c * PQ.size() * N + i];
        dump_host("moddown_in", pqv.data(), pqv.size());
        uint64_tt* dm = up(md);
        uint64_tt* om;
        ck(cudaMalloc(&om, 2 * q_num * N * 8), "m");
        context.modDownPQltoQl_23(om, dm, L, 2);
        dump_dev("moddown_out", om, 2 * q_num * N);
    }
    // ---- Salsa20 keystream (RNG.cuh:18-51, RNG_impl.cuh:70-176)
    {
        uint64_tt s = 20;
        uint8_t key[32];
        for (int i = 0; i < 32; i++) key[i] = (uint8_t)splitmix(s);
        std::vector<uint64_tt> kw(4);
        memcpy(kw.data(), key, 32);
        dump_host("rng_key", kw.data(), 4);
        const uint64_tt nonce = splitmix(s) & 0xffffffffULL;
        std::vector<uint64_tt> nv = {nonce};
        dump_host("rng_nonce", nv.data(), 1);
        const size_t nbytes = 64 * 40;
        uint8_t* d;
        ck(cudaMalloc(&d, nbytes), "m");
        ck(cudaMemcpyToSymbol(RNG::key, key, 32), "key");
        ck(cudaMemset(d, 0, nbytes), "z");
        RNG::VecCrypt<<<(40 + THREADS_PER_BLOCK - 1) / THREADS_PER_BLOCK, THREADS_PER_BLOCK>>>(d, 40, nbytes,
                                                                                              nonce, 1);
        dump_dev("rng_out", (uint64_tt*)d, nbytes / 8);
    }
    // ---- sampler conversions (Sampler.cuh:16-45, Sampler_impl.cuh:13-108) on
    // seeded random words, over the P|Q primes (pqt_cons order)
    {
        const int npq = K + L + 1;
        const std::vector<uint64_tt> raw = {~0ULL};
        auto ru = gen(26, rep(raw, npq), N);  // one 64-bit word per output
        dump_host("samp_uniform_in", ru.data(), ru.size());
        uint64_tt* du = up(ru);
        uint64_tt* ou;
        ck(cudaMalloc(&ou, (size_t)npq * N * 8), "m");
        Sampler::uniformSampler_xq((uint8_tt*)du, ou, N, 0, 0, npq);
        dump_dev("samp_uniform_out", ou, (size_t)npq * N);
        auto rg = gen(27, raw, N / 2);  // N 32-bit words
        uint64_tt* dg = up(rg);
        Sampler::gaussianSampler_xq((uint8_tt*)dg, ou, N, 0, 0, npq);
        dump_dev("samp_gauss_out", ou, (size_t)npq * N);
        auto rz = gen(28, raw, N / 8);  // N bytes
        uint64_tt* dz = up(rz);
        Sampler::ZOSampler((uint8_tt*)dz, ou, N, 0.5, 0, 0, npq);
        dump_dev("samp_zo_out", ou, (size_t)npq * N);
        auto rh = gen(29, raw, 40);  // 64 positions (32-bit) then 64 sign bytes
        uint64_tt* dh = up(rh);
        ck(cudaMemset(ou, 0, (size_t)npq * N * 8), "z");
        Sampler::HWTSampler((uint8_tt*)dh, ou, logN, 64, 0, 0, npq);
        dump_dev("samp_hwt_out", ou, (size_t)npq * N);
    }
    // ---- the multiply path without the secret-key shortcut: HPS tensor then
    // the KLSS key switch, as multAndEqual_23 (KeySwitch_23.cuh:244-305) runs
    // them, omitting only its final copy of mult_scale_buffer into cipher1.
    {
        // key material over P|Q in NTT form (reference order), converted to the
        // KLSS layout exactly as addMultKey_23 does (KeySwitch_23.cuh:55-65)
        auto ka = gen(21, rep(PQ, dnum), N), kb = gen(22, rep(PQ, dnum), N);
        dump_host("mult_key_a", ka.data(), ka.size());
        dump_host("mult_key_b", kb.data(), kb.size());
        Key_decomp* rlk = scheme.rlk_23;
        const size_t slot = (size_t)N * t_num * Ri;
        for (int i = 0; i < dnum; i++) {
            ck(cudaMemcpy(rlk->ax_device + i * slot, ka.data() + i * PQ.size() * N, PQ.size() * N * 8,
                          cudaMemcpyHostToDevice), "ka");
            ck(cudaMemcpy(rlk->bx_device + i * slot, kb.data() + i * PQ.size() * N, PQ.size() * N * 8,
                          cudaMemcpyHostToDevice), "kb");
        }
        context.FromNTTInplace(rlk->ax_device, 0, 0, dnum, K + L + 1, t_num * Ri);
        context.FromNTTInplace(rlk->bx_device, 0, 0, dnum, K + L + 1, t_num * Ri);
        for (int i = 0; i < dnum; i++) {
            ck(cudaMemcpy(scheme.modUp_RitoT_temp, rlk->ax_device + i * slot, sizeof(uint64_tt) * N * (K + L + 1),
                          cudaMemcpyDeviceToDevice), "t");
            context.modUpPQtoT_23(rlk->ax_device + i * slot, scheme.modUp_RitoT_temp, L, 1);
            ck(cudaMemcpy(scheme.modUp_RitoT_temp, rlk->bx_device + i * slot, sizeof(uint64_tt) * N * (K + L + 1),
                          cudaMemcpyDeviceToDevice), "t");
            context.modUpPQtoT_23(rlk->bx_device + i * slot, scheme.modUp_RitoT_temp, L, 1);
        }
        context.ToNTTInplace(rlk->cipher_device, 0, K + L + 1, dnum * Ri * 2, t_num, t_num);
        dump_dev("mult_key_t", rlk->cipher_device, 2 * slot * dnum);

        auto a = gen(23, rep(Q, 2), N), b = gen(24, rep(Q, 2), N);
        dump_host("mult_ct1", a.data(), a.size());
        dump_host("mult_ct2", b.data(), b.size());
        Ciphertext c1(N, L, L, context.slots), c2(N, L, L, context.slots);
        ck(cudaMemcpy(c1.cipher_device, a.data(), a.size() * 8, cudaMemcpyHostToDevice), "c1");
        ck(cudaMemcpy(c2.cipher_device, b.data(), b.size() * 8, cudaMemcpyHostToDevice), "c2");

        const int l = L;
        const int swk_blockNum = (int)ceil(double(K + l + 1) / context.gamma);
        const int cipher_blockNum = (int)ceil(double(l + 1) / K);
        // tensor, then the key switch of a1*a2 and the add-back into c1
        auto tensor = [&]() { scheme.compute_t_QInv_c0c1c2(scheme.axbx1_mul, scheme.axax_mul, scheme.bxbx_mul, c1, c2); };
        auto key_switch = [&]() {
            context.FromNTTInplace(scheme.axax_mul, 0, K, 1, l + 1, L + 1);
            context.modUpQjtoT_23(scheme.modUp_QjtoT_temp, scheme.axax_mul, l, 1);
            context.ToNTTInplace(scheme.modUp_QjtoT_temp, 0, K + L + 1, cipher_blockNum, t_num, t_num);
            context.external_product_T(scheme.exProduct_T_temp, scheme.modUp_QjtoT_temp, rlk->cipher_device, l);
            context.FromNTTInplace_for_externalProduct(scheme.exProduct_T_temp, 0, K + L + 1, swk_blockNum, t_num,
                                                       t_num, Ri * t_num, 2);
            context.modUpTtoPQl_23(scheme.modUp_TtoQj_buffer, scheme.exProduct_T_temp, l, 2);
            context.modDownPQltoQl_23(c1.cipher_device, scheme.modUp_TtoQj_buffer, l, 2);
            context.ToNTTInplace(c1.cipher_device, 0, K, 2, l + 1, L + 1);
            cipher_add_axbx_batch_device(c1.cipher_device, scheme.axbx1_mul, scheme.bxbx_mul, N, K, l + 1, L + 1);
        };
        tensor();
        dump_dev("mult_axax", scheme.axax_mul, q_num * N);
        dump_dev("mult_axbx", scheme.axbx1_mul, q_num * N);
        dump_dev("mult_bxbx", scheme.bxbx_mul, q_num * N);
        key_switch();
        dump_dev("mult_out", c1.cipher_device, 2 * q_num * N);
        // timing of the same genuine multiply, one pair per call as the reference
        // runs it (its tensor step allocates device memory on every call); the
        // values keep changing in place, which does not change the work
        if (g_time_reps > 0) {
            for (int r = 0; r < 2; r++) { tensor(); key_switch(); }
            cudaEvent_t e0, e1;
            ck(cudaEventCreate(&e0), "event");
            ck(cudaEventCreate(&e1), "event");
            ck(cudaDeviceSynchronize(), "warm-up");
            ck(cudaEventRecord(e0), "record");
            for (int r = 0; r < g_time_reps; r++) { tensor(); key_switch(); }
            ck(cudaEventRecord(e1), "record");
            ck(cudaEventSynchronize(e1), "sync");
            float ms = 0.f;
            ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
            printf("{\"logN\": %d, \"reps\": %d, \"ms_per_mult\": %.5f}\n", logN, g_time_reps, ms / g_time_reps);
        }
    }
    ck(cudaDeviceSynchronize(), "end");
    fclose(g_manifest);
    printf("ref_harness logN=%d done\n", logN);
    return 0;
}
