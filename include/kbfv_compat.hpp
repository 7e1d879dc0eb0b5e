// kbfv_compat.hpp -- kunpBFV's class API (BFVContext, BFVScheme, Plaintext,
// Ciphertext, SecretKey) rebuilt on the C ABI in kbfv.h, so drivers written for
// kunpBFV (correct_mult.cu, perf_mult.cu, ...) run on the B200 path. Unmodified
// drivers compile against the include tree include/kunpbfv/ (its include/*.cuh
// forward the reference's header names here and put the classes in the global
// namespace); new code can include this header and use namespace kbfv_compat.
// Header-only; link libkbfv.so and cudart.
//
// Behaviour kept from the reference: encode() overwrites its input with the
// plaintext coefficients (include/Encoder.cuh:32), encode_ntt() takes
// coefficients, errors throw std::invalid_argument / std::runtime_error.
// Behaviour not kept: multAndEqual_23 computes a genuine relinearised product
// (the reference overwrites it with ct1 * Dec(ct2), include/KeySwitch_23.cuh:308).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <random>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "kbfv.h"

namespace kbfv_compat {

typedef unsigned long long uint64_tt;

inline void check(int rc) {
    if (rc == KBFV_OK) return;
    std::string m = kbfv_last_error();
    if (rc == KBFV_ERR_INVALID || rc == KBFV_ERR_LEVEL || rc == KBFV_ERR_NO_KEY) throw std::invalid_argument(m);
    throw std::runtime_error(m);
}

inline void check_cuda(cudaError_t e) {
    if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
}

class BFVContext;

// A device buffer of `words` uint64 words that copies deeply: copy construction
// and assignment allocate their own buffer (reallocating when the size differs)
// and copy the contents device to device, like the reference's Plaintext and
// Ciphertext (include/Plaintext.cuh:21-48, include/Ciphertext.cuh:42-78);
// moves hand the buffer over.
struct DeviceWords {
    uint64_tt* p = nullptr;
    size_t words = 0;
    DeviceWords() = default;
    explicit DeviceWords(size_t n, bool zero) { reset(n, zero); }
    DeviceWords(const DeviceWords& o) { copy_from(o); }
    DeviceWords(DeviceWords&& o) noexcept : p(o.p), words(o.words) { o.p = nullptr; o.words = 0; }
    DeviceWords& operator=(const DeviceWords& o) {
        if (this != &o) copy_from(o);
        return *this;
    }
    DeviceWords& operator=(DeviceWords&& o) noexcept {
        if (this != &o) {
            release();
            p = o.p; words = o.words;
            o.p = nullptr; o.words = 0;
        }
        return *this;
    }
    ~DeviceWords() { release(); }
    void reset(size_t n, bool zero) {
        if (n != words) {
            release();
            if (n) check_cuda(cudaMalloc(&p, sizeof(uint64_tt) * n));
            words = n;
        }
        if (zero && n) check_cuda(cudaMemset(p, 0, sizeof(uint64_tt) * n));
    }
    void copy_from(const DeviceWords& o) {
        reset(o.words, false);
        if (o.words) check_cuda(cudaMemcpy(p, o.p, sizeof(uint64_tt) * o.words, cudaMemcpyDeviceToDevice));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        words = 0;
    }
};

class Plaintext {
    DeviceWords buf_;

public:
    uint64_tt* mx_device = nullptr;  // (L+1) x N words: coefficients in the first N, or NTT form over Q
    int N = 0, L = 0, l = 0, slots = 0;
    Plaintext() = default;
    Plaintext(int N_, int L_, int l_, int slots_)
        : buf_((size_t)N_ * (L_ + 1), true), N(N_), L(L_), l(l_), slots(slots_) {
        mx_device = buf_.p;
    }
    // host values (N x (L+1) words) copied in (include/Plaintext.cuh:13-18)
    Plaintext(uint64_tt* m_host, int N_, int L_, int l_, int slots_) : Plaintext(N_, L_, l_, slots_) {
        check_cuda(cudaMemcpy(mx_device, m_host, sizeof(uint64_tt) * buf_.words, cudaMemcpyHostToDevice));
    }
    Plaintext(const Plaintext& o) : buf_(o.buf_), N(o.N), L(o.L), l(o.l), slots(o.slots) { mx_device = buf_.p; }
    Plaintext(Plaintext&& o) noexcept : buf_(std::move(o.buf_)), N(o.N), L(o.L), l(o.l), slots(o.slots) {
        mx_device = buf_.p;
        o.mx_device = nullptr;
    }
    Plaintext& operator=(const Plaintext& o) {
        if (this == &o) return *this;
        buf_ = o.buf_;
        N = o.N; L = o.L; l = o.l; slots = o.slots;
        mx_device = buf_.p;
        return *this;
    }
    Plaintext& operator=(Plaintext&& o) noexcept {
        if (this == &o) return *this;
        buf_ = std::move(o.buf_);
        N = o.N; L = o.L; l = o.l; slots = o.slots;
        mx_device = buf_.p;
        o.mx_device = nullptr;
        return *this;
    }
    virtual ~Plaintext() = default;
};

class Ciphertext {
    DeviceWords buf_;
    void bind() {
        cipher_device = buf_.p;
        ax_device = cipher_device;
        bx_device = cipher_device ? cipher_device + (size_t)N * (L + 1) : nullptr;
    }

public:
    uint64_tt* cipher_device = nullptr;  // [ax | bx], (L+1) x N words each, NTT form over Q
    uint64_tt* ax_device = nullptr;
    uint64_tt* bx_device = nullptr;
    int N = 0, L = 0, l = 0, slots = 0;
    Ciphertext() = default;
    Ciphertext(int N_, int L_, int l_, int slots_)
        : buf_((size_t)N_ * (L_ + 1) * 2, false), N(N_), L(L_), l(l_), slots(slots_) {
        bind();
    }
    Ciphertext(const Ciphertext& o) : buf_(o.buf_), N(o.N), L(o.L), l(o.l), slots(o.slots) { bind(); }
    Ciphertext(Ciphertext&& o) noexcept : buf_(std::move(o.buf_)), N(o.N), L(o.L), l(o.l), slots(o.slots) {
        bind();
        o.bind();
    }
    Ciphertext& operator=(const Ciphertext& o) {
        if (this == &o) return *this;
        buf_ = o.buf_;
        N = o.N; L = o.L; l = o.l; slots = o.slots;
        bind();
        return *this;
    }
    Ciphertext& operator=(Ciphertext&& o) noexcept {
        if (this == &o) return *this;
        buf_ = std::move(o.buf_);
        N = o.N; L = o.L; l = o.l; slots = o.slots;
        bind();
        o.bind();
        return *this;
    }
    virtual ~Ciphertext() = default;
};

class BFVContext {
public:
    kbfv_context* handle = nullptr;
    long N = 0;
    int logN = 0, L = 0, K = 0, slots = 0, q_num = 0, p_num = 0, dnum = 0;
    uint64_tt plain_modulus = 0;

    // the reference's parameter set for this ring degree (include/Params.cuh)
    explicit BFVContext(size_t poly_modulus_degree) {
        const int lg = (int)std::lround(std::log2((double)poly_modulus_degree));
        check(kbfv_context_create_reference((uint32_t)lg, &handle));
        fill();
    }
    explicit BFVContext(const kbfv_params& p) {
        check(kbfv_context_create(&p, &handle));
        fill();
    }
    BFVContext(const BFVContext&) = delete;
    BFVContext& operator=(const BFVContext&) = delete;
    ~BFVContext() { if (handle) kbfv_context_destroy(handle); }

    // INTT mod t into msg; like the reference, `vals` is overwritten with the coefficients
    void encode(uint64_tt* vals, Plaintext& msg) {
        check(kbfv_encode(handle, reinterpret_cast<const uint64_t*>(vals), reinterpret_cast<uint64_t*>(msg.mx_device),
                          1, 0));
        check_cuda(cudaMemcpy(vals, msg.mx_device, sizeof(uint64_tt) * N, cudaMemcpyDeviceToDevice));
    }
    // coefficients -> NTT form over Q (for multConstAndEqual)
    void encode_ntt(uint64_tt* vals, Plaintext& msg) {
        check(kbfv_encode_ntt(handle, reinterpret_cast<const uint64_t*>(vals),
                              reinterpret_cast<uint64_t*>(msg.mx_device), 1, 0));
    }
    void decode(Plaintext& msg, uint64_tt* vals) {
        check(kbfv_decode(handle, reinterpret_cast<const uint64_t*>(msg.mx_device), reinterpret_cast<uint64_t*>(vals),
                          1, 0));
    }

private:
    void fill() {
        uint64_t n;
        uint32_t nq, np, nr, nt, dn, al;
        check(kbfv_context_info(handle, &n, &nq, &np, &nr, &nt, &dn, &al));
        N = (long)n;
        logN = (int)std::lround(std::log2((double)n));
        q_num = (int)nq;
        p_num = (int)np;
        L = q_num - 1;
        K = p_num;
        dnum = (int)dn;
        slots = (int)N;
        plain_modulus = kbfv_context_plain_modulus(handle);
    }
};

class SecretKey {
    DeviceWords buf_;

public:
    uint64_tt* sx_device = nullptr;  // (K+L+1) x N words, NTT form over Q|P
    int N = 0, L = 0, K = 0;
    uint8_t seed[32];
    // Hamming-weight-64 ternary secret as in the reference (include/SecretKey.cuh:31);
    // the seed is drawn from std::random_device unless given
    explicit SecretKey(BFVContext& ctx, cudaStream_t stream = 0, const uint8_t* seed_in = nullptr)
        : N((int)ctx.N), L(ctx.L), K(ctx.K) {
        if (seed_in) std::memcpy(seed, seed_in, 32);
        else {
            std::random_device rd;
            for (int i = 0; i < 32; i++) seed[i] = (uint8_t)rd();
        }
        buf_.reset((size_t)N * (K + L + 1), false);
        sx_device = buf_.p;
        check(kbfv_keygen_secret(ctx.handle, seed, 1, 64, reinterpret_cast<uint64_t*>(sx_device), stream));
    }
    // deep copies (the reference's SecretKey copies shallowly and frees twice)
    SecretKey(const SecretKey& o) : buf_(o.buf_), N(o.N), L(o.L), K(o.K) {
        sx_device = buf_.p;
        std::memcpy(seed, o.seed, 32);
    }
    SecretKey& operator=(const SecretKey& o) {
        if (this == &o) return *this;
        buf_ = o.buf_;
        N = o.N; L = o.L; K = o.K;
        std::memcpy(seed, o.seed, 32);
        sx_device = buf_.p;
        return *this;
    }
    virtual ~SecretKey() = default;
};

class BFVScheme {
public:
    BFVContext& context;
    uint64_tt* publicKey = nullptr;
    uint64_tt* rlk_23 = nullptr;
    std::map<uint64_t, uint64_tt*> galoisKeys;  // rotKey_vec_23 and ConjKey_23, by Galois element
    Ciphertext cipher_const_1;                  // kept for callers that read it (bfv_demo.cu); unused here
    uint64_t enc_counter = 0;
    uint8_t seed[32];

    explicit BFVScheme(BFVContext& ctx) : context(ctx) {
        std::random_device rd;
        for (int i = 0; i < 32; i++) seed[i] = (uint8_t)rd();
    }
    BFVScheme(const BFVScheme&) = delete;
    BFVScheme& operator=(const BFVScheme&) = delete;
    ~BFVScheme() {
        if (publicKey) cudaFree(publicKey);
        if (rlk_23) cudaFree(rlk_23);
        for (auto& kv : galoisKeys) cudaFree(kv.second);
    }

    void mallocMemory() { check(kbfv_reserve(context.handle, 1)); }

    void addEncKey(SecretKey& sk, cudaStream_t stream = 0) {
        if (!publicKey) check_cuda(cudaMalloc(&publicKey, sizeof(uint64_tt) * context.N * context.q_num * 2));
        check(kbfv_keygen_public(context.handle, seed, reinterpret_cast<const uint64_t*>(sk.sx_device),
                                 reinterpret_cast<uint64_t*>(publicKey), stream));
    }
    void addMultKey_23(SecretKey& sk, cudaStream_t stream = 0) {
        if (rlk_23) return;
        const size_t words = (size_t)context.dnum * 2 * (context.q_num + context.p_num) * context.N;
        check_cuda(cudaMalloc(&rlk_23, sizeof(uint64_tt) * words));
        check(kbfv_keygen_relin(context.handle, seed, reinterpret_cast<const uint64_t*>(sk.sx_device),
                                reinterpret_cast<uint64_t*>(rlk_23), stream));
    }
    // rotation / conjugation keys (KeySwitch_23.cuh:71-166): Galois element 5^r or 2N - 1
    void addGaloisKey(SecretKey& sk, uint64_t g, cudaStream_t stream = 0) {
        if (galoisKeys.count(g)) return;
        uint64_tt* key = nullptr;
        const size_t words = (size_t)context.dnum * 2 * (context.q_num + context.p_num) * context.N;
        check_cuda(cudaMalloc(&key, sizeof(uint64_tt) * words));
        check(kbfv_keygen_galois(context.handle, seed, reinterpret_cast<const uint64_t*>(sk.sx_device), g,
                                 reinterpret_cast<uint64_t*>(key), stream));
        galoisKeys[g] = key;
    }
    void addLeftRotKey_23(SecretKey& sk, long rot_num, cudaStream_t stream = 0) {
        addGaloisKey(sk, kbfv_galois_element(context.handle, rot_num), stream);
    }
    void addConjKey_23(SecretKey& sk, cudaStream_t stream = 0) { addGaloisKey(sk, 2 * (uint64_t)context.N - 1, stream); }
    void applyGalois(Ciphertext& cipher, uint64_t g) {
        auto it = galoisKeys.find(g);
        if (it == galoisKeys.end()) throw std::invalid_argument("rotKey_23 not exists");
        check(kbfv_apply_galois(context.handle, reinterpret_cast<const uint64_t*>(it->second), g,
                                reinterpret_cast<const uint64_t*>(cipher.cipher_device),
                                reinterpret_cast<uint64_t*>(cipher.cipher_device), 1, 0));
    }
    void leftRotateAndEqual_23(Ciphertext& cipher, long rotSlots) {
        applyGalois(cipher, kbfv_galois_element(context.handle, rotSlots));
    }
    // the reference's conversion (KeySwitch_23.cuh:580-584)
    void rightRotateAndEqual_23(Ciphertext& cipher, long rotSlots) {
        leftRotateAndEqual_23(cipher, context.N / 2 - (1L << rotSlots));
    }
    void conjugate_23(Ciphertext& cipher) { applyGalois(cipher, 2 * (uint64_t)context.N - 1); }

    void encryptMsg(Ciphertext& cipher, Plaintext& message, cudaStream_t stream = 0) {
        if (!publicKey) throw std::invalid_argument("public key not generated");
        cipher.l = message.l;
        check(kbfv_encrypt(context.handle, seed, enc_counter++, reinterpret_cast<const uint64_t*>(publicKey),
                           reinterpret_cast<const uint64_t*>(message.mx_device),
                           reinterpret_cast<uint64_t*>(cipher.cipher_device), 1, stream));
    }
    void decryptMsg(Plaintext& plain, SecretKey& sk, Ciphertext& cipher, cudaStream_t stream = 0) {
        plain.l = cipher.l;
        check(kbfv_decrypt(context.handle, reinterpret_cast<const uint64_t*>(sk.sx_device),
                           reinterpret_cast<const uint64_t*>(cipher.cipher_device),
                           reinterpret_cast<uint64_t*>(plain.mx_device), 1, stream));
    }
    void add(Ciphertext& res, Ciphertext& c1, Ciphertext& c2) {
        res.l = std::min(c1.l, c2.l);
        check(kbfv_add(context.handle, reinterpret_cast<const uint64_t*>(c1.cipher_device),
                       reinterpret_cast<const uint64_t*>(c2.cipher_device),
                       reinterpret_cast<uint64_t*>(res.cipher_device), 1, 0));
    }
    void addAndEqual(Ciphertext& c1, Ciphertext& c2) { add(c1, c1, c2); }
    // adds the constant c to every slot (BFVScheme.cuh:220-224)
    void addConstAndEqual(Ciphertext& cipher, uint64_tt c) {
        uint64_tt* d = nullptr;
        check_cuda(cudaMalloc(&d, sizeof(uint64_tt) * context.N));
        std::vector<uint64_tt> h((size_t)context.N, c % context.plain_modulus);
        check_cuda(cudaMemcpy(d, h.data(), sizeof(uint64_tt) * context.N, cudaMemcpyHostToDevice));
        int rc = kbfv_encode(context.handle, reinterpret_cast<const uint64_t*>(d), reinterpret_cast<uint64_t*>(d), 1, 0);
        if (rc == KBFV_OK)
            rc = kbfv_add_plain(context.handle, reinterpret_cast<const uint64_t*>(cipher.cipher_device),
                                reinterpret_cast<const uint64_t*>(d), reinterpret_cast<uint64_t*>(cipher.cipher_device),
                                1, 0);
        cudaFree(d);
        check(rc);
    }
    // b += NTT(Delta * m) with m the plaintext's coefficients (BFVScheme.cuh:192-217)
    void addConstAndEqual(Ciphertext& cipher, Plaintext& cnst) {
        cipher.l = std::min(cipher.l, cnst.l);
        check(kbfv_add_plain(context.handle, reinterpret_cast<const uint64_t*>(cipher.cipher_device),
                             reinterpret_cast<const uint64_t*>(cnst.mx_device),
                             reinterpret_cast<uint64_t*>(cipher.cipher_device), 1, 0));
    }
    void multConstAndEqual(Ciphertext& cipher, Plaintext& cnst) {
        if (cipher.l == 0) throw std::invalid_argument("Ciphertexts are on level 0");
        check(kbfv_mul_plain(context.handle, reinterpret_cast<const uint64_t*>(cipher.cipher_device),
                             reinterpret_cast<const uint64_t*>(cnst.mx_device),
                             reinterpret_cast<uint64_t*>(cipher.cipher_device), 1, 0));
    }
    void mult_23(Ciphertext& res, Ciphertext& c1, Ciphertext& c2) {
        if (c1.l == 0 || c2.l == 0) throw std::invalid_argument("Ciphertexts are on level 0");
        if (!rlk_23) throw std::invalid_argument("rotKey_23 not exists");
        res.l = std::min(c1.l, c2.l);
        check(kbfv_mul_relin(context.handle, reinterpret_cast<const uint64_t*>(rlk_23),
                             reinterpret_cast<const uint64_t*>(c1.cipher_device),
                             reinterpret_cast<const uint64_t*>(c2.cipher_device),
                             reinterpret_cast<uint64_t*>(res.cipher_device), 1, 0));
    }
    void multAndEqual_23(Ciphertext& c1, Ciphertext& c2) { mult_23(c1, c1, c2); }
};

}  // namespace kbfv_compat
