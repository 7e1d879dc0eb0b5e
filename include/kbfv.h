/*
 * kbfv.h -- C ABI of the B200-native BFV multiply path (libkbfv.so).
 *
 * kunpBFV exposes its multiply path as a header-only C++ class API
 * (BFVContext / BFVScheme / Plaintext / Ciphertext / SecretKey / Key_decomp)
 * compiled into the caller. This header is the flat boundary underneath an
 * equivalent API: opaque context handle, plain device pointers and sizes,
 * int status codes, caller-supplied CUDA stream (0 = legacy default stream).
 * kbfv_compat.hpp rebuilds the reference's class names on top of it.
 *
 * Data layout (all device memory, uint64 residues, limb-major poly[limb][coeff]):
 *   ciphertext  [a | b], each q_count limbs, NTT form over Q  (decrypts as b + a*s)
 *   tensor      [a1*a2 | a1*b2 + b1*a2 | b1*b2], each q_count limbs, NTT form
 *   secret key  q_count + p_count limbs, NTT form over Q|P
 *   public key  [a | b], q_count limbs each, NTT form
 *   relin key   dnum x [a | b], (q_count + p_count) limbs each, NTT form over Q|P
 *   plaintext   N coefficients mod t (coefficient form)
 *   slots       N values mod t (batch encoding: slot k <-> NTT index k mod t)
 * Prime table order inside a context: [ Q | P | R (HPS base) | T (KLSS) | t ].
 *
 * Every function returns KBFV_OK or a negative kbfv_status; kbfv_last_error()
 * describes the most recent failure on the calling thread.
 *
 * Threads and streams: calls on different contexts are independent. A context
 * owns one scratch arena and its helper streams, so calls on the same context
 * must be issued in order from one host thread (or under the caller's lock)
 * and ordered on the GPU through one caller stream; the request server
 * (kbfv_serve.h) drives each ring's context from its one scheduler thread, so
 * a context handed to a running server is not used by other threads.
 */
#ifndef KBFV_H
#define KBFV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    KBFV_OK = 0,
    KBFV_ERR_INVALID = -1,    /* bad argument (std::invalid_argument in the reference) */
    KBFV_ERR_PARAMS = -2,     /* parameter set cannot be built (logic_error in the reference) */
    KBFV_ERR_CUDA = -3,       /* a CUDA call failed */
    KBFV_ERR_NOMEM = -4,      /* device allocation failed */
    KBFV_ERR_NO_KEY = -5,     /* key missing ("rotKey_23 not exists" in the reference) */
    KBFV_ERR_LEVEL = -6,      /* ciphertext level unsupported ("Ciphertexts are on level 0") */
    KBFV_ERR_UNSUPPORTED = -7
} kbfv_status;

typedef struct kbfv_context kbfv_context;
typedef void* kbfv_stream; /* cudaStream_t */

/* Parameter set. Explicit primes win over bit sizes; R (the HPS base) is
 * always derived: q_count + 1 primes below min(q) that are 1 mod 2N.
 * Replaces the hard-coded BFVContext::getPrimeBFV (include/Params.cuh:7-149). */
typedef struct {
    uint32_t log_n;           /* ring degree N = 2^log_n, 10..16 */
    uint64_t plain_modulus;   /* t, prime, 1 mod 2N for batching */
    uint32_t q_count;
    const uint64_t* q;        /* q_count primes, or NULL to generate q_bits-sized primes */
    uint32_t q_bits;
    uint32_t p_count;
    const uint64_t* p;        /* special primes or NULL (generated with p_bits, largest first) */
    uint32_t p_bits;
    uint32_t dnum;            /* key-switch digits; digit size alpha = ceil(q_count / dnum) */
    uint32_t t_count;         /* optional KLSS base (reference key switch), may be 0 */
    const uint64_t* t_primes;
    uint32_t gamma;           /* KLSS Ri block size */
    uint32_t digit_primes;    /* key-switch digit size alpha; 0 = ceil(q_count / dnum) */
} kbfv_params;

/* Parameter set from per-prime bit sizes (SEAL-style coeff_modulus sizes):
 * p_count special primes of p_bits[i] bits, then q_count ciphertext primes of
 * q_bits[i] bits, all distinct, 1 mod 2N, largest first within each size.
 * Replaces the hard-coded prime lists of include/Params.cuh:7-149. Free with
 * kbfv_params_destroy. */
int kbfv_params_create(uint32_t log_n, const uint32_t* q_bits, uint32_t q_count, const uint32_t* p_bits,
                       uint32_t p_count, uint64_t plain_modulus, uint32_t dnum, kbfv_params** out);
int kbfv_params_destroy(kbfv_params* params);

const char* kbfv_last_error(void);
const char* kbfv_version(void);
/* Throughput of one 64-bit modular primitive on the current device (Gop/s):
 * independent register chains, no memory traffic. kind 0: 64x64->128
 * multiply-accumulate, 1: mul.lo.u64, 2: mul.hi.u64, 3: forward NTT butterfly
 * with the Shoup product from 64-bit multiplies,
 * 4: Shoup product, 5: 128-bit Barrett, 6: one-high-product Barrett,
 * 7: 32x32->64 multiply-add, 8: 32x32 high product, 9: 32-bit multiply-add,
 * 10: 64x64->128 multiply-accumulate from 32-bit partial products with carry
 * chains, 11: forward NTT butterfly from 32-bit partial products (the one the
 * NTT kernels use), 12: 32-bit multiply-add issue rate (16 dependent
 * multiply-adds per chain step: the IMAD pipe's peak), 13: the same for
 * 32x32->64 multiply-adds, 14: 60x60-bit multiply-accumulate from 30-bit
 * halves (four 32x32->64 multiply-adds into three column sums), 15: the same
 * as 12 for 32-bit high multiply-adds. The roofline of the IMAD-bound
 * kernels. */
int kbfv_probe_arith(int kind, uint32_t iters, double* gops);

/* ---- context ---------------------------------------------------------
 * BFVContext::BFVContext(size_t N) (include/BFVcontext.cuh:13-101):
 * precompute on the host, tables to the device. One context per parameter
 * set; any number of contexts may coexist in a process (no __constant__ state). */
int kbfv_context_create(const kbfv_params* params, kbfv_context** out);
/* the reference's own parameter sets, logN = 14 or 15 (include/Params.cuh:31-145) */
int kbfv_context_create_reference(uint32_t log_n, kbfv_context** out);
int kbfv_context_destroy(kbfv_context* ctx);
/* sizes: N, q_count, p_count, r_count, t_count, dnum, alpha */
int kbfv_context_info(const kbfv_context* ctx, uint64_t* n, uint32_t* q_count, uint32_t* p_count,
                      uint32_t* r_count, uint32_t* t_count, uint32_t* dnum, uint32_t* alpha);
/* full prime table [Q|P|R|T|t]; count receives its length (primes may be NULL) */
int kbfv_context_primes(const kbfv_context* ctx, uint64_t* primes, uint32_t* count);
uint64_t kbfv_context_plain_modulus(const kbfv_context* ctx);
/* decrypt rounding variant chosen by bit sizes (0 small, 1 small_lazy, 2 large, 3 large_lazy) */
int kbfv_context_decrypt_variant(const kbfv_context* ctx);
/* bytes of device scratch a batched multiply of `count` pairs uses */
size_t kbfv_mul_relin_scratch_bytes(const kbfv_context* ctx, uint32_t count);
/* pre-size the context's scratch arena (no allocation happens later for <= count pairs) */
int kbfv_reserve(kbfv_context* ctx, uint32_t pairs);
/* bytes of device memory the context's scratch arena holds now: 0 until a call
 * needs scratch or kbfv_reserve sizes it (no counterpart in the reference, whose
 * scratch is allocated per call; lets a caller audit what the context holds) */
size_t kbfv_context_arena_bytes(const kbfv_context* ctx);

/* seed for keygen / encryption calls that pass seed = NULL (the reference
 * seeds its RNG once per scheme, include/RNG.cuh:18-51) */
int kbfv_set_seed(kbfv_context* ctx, const uint8_t seed[32]);

/* ---- NTT over the context's prime table --------------------------------
 * ToNTTInplace / FromNTTInplace (include/BFVcontext.cuh:1513-1552) and the
 * _for_QR / _for_BFV / _for_externalProduct variants (1554-1757): rows are
 * consecutive N-coefficient limbs; row r uses prime index
 * prime0 + (r % period). In place. */
int kbfv_ntt_fwd(kbfv_context* ctx, uint64_t* d_rows, uint32_t rows, uint32_t prime0, uint32_t period,
                 kbfv_stream stream);
int kbfv_ntt_inv(kbfv_context* ctx, uint64_t* d_rows, uint32_t rows, uint32_t prime0, uint32_t period,
                 kbfv_stream stream);
/* the same over `count` polynomials at arbitrary addresses (HOST array of
 * device pointers), each `limbs` rows using primes prime0 .. prime0+limbs-1 */
int kbfv_ntt_fwd_batch(kbfv_context* ctx, uint64_t* const* d_polys, uint32_t count, uint32_t limbs,
                       uint32_t prime0, kbfv_stream stream);
int kbfv_ntt_inv_batch(kbfv_context* ctx, uint64_t* const* d_polys, uint32_t count, uint32_t limbs,
                       uint32_t prime0, kbfv_stream stream);

/* ---- HPS building blocks (per polynomial, coefficient form) ------------
 * BaseConverter::bConv_HPS (include/BasisConv_QR.cuh:191-207): centred base
 * extension Q -> R and R -> Q. */
int kbfv_bconv_q_to_r(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                      kbfv_stream stream);
int kbfv_bconv_r_to_q(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                      kbfv_stream stream);
/* tensor_prod_2x2_rns_poly (include/poly_arithmetic.cuh:1180-1219): pairs of
 * [a|b] over Q|R (NTT form) -> [a1a2 | cross | b1b2] over Q|R */
int kbfv_tensor_qr(kbfv_context* ctx, const uint64_t* d_ct1, const uint64_t* d_ct2, uint64_t* d_out,
                   uint32_t pairs, kbfv_stream stream);
/* scaleAndRound_HPS_QR_R (include/poly_arithmetic.cuh:1263-1316): Q|R -> R */
int kbfv_scale_round_qr_r(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                          kbfv_stream stream);
/* hps_decrypt_scale_and_round (include/BFVcontext.cuh:1680-1717): Q -> N values */
int kbfv_decrypt_round(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                       kbfv_stream stream);
/* bfv_add_timesQ_overt_kernel (include/poly_arithmetic.cuh:902-927): m -> ceil(Q*m/t) over Q */
int kbfv_delta_m(kbfv_context* ctx, const uint64_t* d_m, uint64_t* d_out, uint32_t polys,
                 kbfv_stream stream);

/* ---- key-switch building blocks (coefficient form) ---------------------
 * digit lift of one polynomial over Q into dnum polynomials over Q|P; the
 * quotient estimate restates modUpQjtoT_23 (include/BasisConv.cuh:86-151) */
int kbfv_modup(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
               kbfv_stream stream);
/* modDownPQltoQl_23 (include/BasisConv.cuh:229-319): Q|P -> Q */
int kbfv_moddown(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                 kbfv_stream stream);

/* ---- keys --------------------------------------------------------------
 * SecretKey::SecretKey (include/SecretKey.cuh:20-37), BFVScheme::addEncKey
 * (include/BFVScheme.cuh:57-85), BFVScheme::addMultKey_23
 * (include/KeySwitch_23.cuh:21-66). All randomness comes from XSalsa20 keyed
 * by `seed` (32 bytes; NULL = the context seed, kbfv_set_seed); the same seed
 * reproduces the same keys. kbfv_encrypt takes seeds the same way.
 * secret_kind: 0 = ternary uniform, 1 = Hamming weight h (the reference's HWT). */
int kbfv_keygen_secret(kbfv_context* ctx, const uint8_t seed[32], int secret_kind, uint32_t h,
                       uint64_t* d_sk, kbfv_stream stream);
int kbfv_keygen_public(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t* d_pk,
                       kbfv_stream stream);
int kbfv_keygen_relin(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t* d_rlk,
                      kbfv_stream stream);

/* ---- encoder -----------------------------------------------------------
 * BFVContext::encode / decode (include/Encoder.cuh:23-112): INTT / NTT mod t.
 * Unlike the reference, encode does not overwrite its input. */
int kbfv_encode(kbfv_context* ctx, const uint64_t* d_slots, uint64_t* d_m, uint32_t count,
                kbfv_stream stream);
int kbfv_decode(kbfv_context* ctx, const uint64_t* d_m, uint64_t* d_slots, uint32_t count,
                kbfv_stream stream);
/* BFVContext::encode_ntt (include/Encoder.cuh:64-79): values as coefficients, NTT over Q */
int kbfv_encode_ntt(kbfv_context* ctx, const uint64_t* d_vals, uint64_t* d_pt_ntt, uint32_t count,
                    kbfv_stream stream);

/* ---- scheme ------------------------------------------------------------
 * BFVScheme::encryptMsg / decryptMsg (include/BFVScheme.cuh:87-166).
 * Encrypts `count` plaintexts (consecutive, N words each) into `count`
 * consecutive ciphertexts; ciphertext i uses randomness stream enc_id + i. */
int kbfv_encrypt(kbfv_context* ctx, const uint8_t seed[32], uint64_t enc_id, const uint64_t* d_pk,
                 const uint64_t* d_m, uint64_t* d_ct, uint32_t count, kbfv_stream stream);
int kbfv_decrypt(kbfv_context* ctx, const uint64_t* d_sk, const uint64_t* d_ct, uint64_t* d_m,
                 uint32_t count, kbfv_stream stream);
/* encryption, decryption and addition of `count` objects at arbitrary addresses
 * (HOST arrays of device pointers, as kbfv_mul_relin_batch): item i of
 * kbfv_encrypt_batch uses encryption id enc_ids[i] (HOST array) and equals
 * kbfv_encrypt(ctx, seed, enc_ids[i], ...) of that item alone. */
int kbfv_encrypt_batch(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* enc_ids, const uint64_t* d_pk,
                       const uint64_t* const* d_m, uint64_t* const* d_ct, uint32_t count, kbfv_stream stream);
int kbfv_decrypt_batch(kbfv_context* ctx, const uint64_t* d_sk, const uint64_t* const* d_ct, uint64_t* const* d_m,
                       uint32_t count, kbfv_stream stream);
int kbfv_add_batch(kbfv_context* ctx, const uint64_t* const* d_x, const uint64_t* const* d_y, uint64_t* const* d_out,
                   uint32_t count, kbfv_stream stream);
/* BFVScheme::add / addAndEqual (include/BFVScheme.cuh:169-190); polys per item = 2 */
int kbfv_add(kbfv_context* ctx, const uint64_t* d_x, const uint64_t* d_y, uint64_t* d_out,
             uint32_t count, kbfv_stream stream);
/* BFVScheme::addConstAndEqual(Ciphertext&, Plaintext&) (include/BFVScheme.cuh:192-217):
 * b += NTT(Delta * m) for plaintexts m of N coefficients mod t */
int kbfv_add_plain(kbfv_context* ctx, const uint64_t* d_ct, const uint64_t* d_m, uint64_t* d_out,
                   uint32_t count, kbfv_stream stream);
/* limb-wise ops on `count` ciphertexts (2 x q_count limbs each, NTT form):
 * sub / subAndEqual, negateAndEqual, multConstAndEqual(Ciphertext&, uint64_tt) and
 * multConstAndAddCipherEqual (include/BFVScheme.cuh:246-330); the scalar is taken
 * mod each q_l. d_out may equal an input. */
int kbfv_sub(kbfv_context* ctx, const uint64_t* d_x, const uint64_t* d_y, uint64_t* d_out, uint32_t count,
             kbfv_stream stream);
int kbfv_negate(kbfv_context* ctx, const uint64_t* d_x, uint64_t* d_out, uint32_t count, kbfv_stream stream);
int kbfv_mul_scalar(kbfv_context* ctx, const uint64_t* d_x, uint64_t cnst, uint64_t* d_out, uint32_t count,
                    kbfv_stream stream);
/* d_acc += d_x * cnst */
int kbfv_mul_scalar_add(kbfv_context* ctx, const uint64_t* d_x, uint64_t cnst, uint64_t* d_acc, uint32_t count,
                        kbfv_stream stream);
/* BFVScheme::multConstAndEqual (include/BFVScheme.cuh:226-245) with an encode_ntt plaintext */
int kbfv_mul_plain(kbfv_context* ctx, const uint64_t* d_ct, const uint64_t* d_pt_ntt, uint64_t* d_out,
                   uint32_t count, kbfv_stream stream);
/* compute_t_QInv_c0c1c2 (include/KeySwitch_23.cuh:703-926) without its
 * secret-key shortcut: HPS tensor of `count` ciphertext pairs -> tensors */
int kbfv_mul(kbfv_context* ctx, const uint64_t* d_ct1, const uint64_t* d_ct2, uint64_t* d_tensor,
             uint32_t count, kbfv_stream stream);
/* key switch of the a1*a2 term (include/KeySwitch_23.cuh:277-305): tensors -> ciphertexts */
int kbfv_relinearize(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* d_tensor, uint64_t* d_ct,
                     uint32_t count, kbfv_stream stream);
/* BFVScheme::multAndEqual_23 / mult_23 (include/KeySwitch_23.cuh:192-310) as
 * one fused batched launch sequence: out[i] = relin(ct_a[i] * ct_b[i]).
 * Arrays are HOST arrays of device pointers. */
int kbfv_mul_relin_batch(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* const* ct_a,
                         const uint64_t* const* ct_b, uint64_t* const* out, uint32_t count,
                         kbfv_stream stream);
/* Batches of 2 or more pairs (2 x KBFV_TUNE_MIN_BRANCH_PAIRS) run as sub-batches on the caller's stream and on
 * auxiliary streams of the context, forked from and joined back into the
 * caller's stream with events (the call stays ordered on `stream`); the partial
 * last wave of one sub-batch's kernels then overlaps the others'. branches: 1..4
 * sub-batches (default 2; 1 disables). No counterpart in the reference. */
int kbfv_set_branches(kbfv_context* ctx, uint32_t branches);
/* ---- tuning ---------------------------------------------------------------
 * Per-context knobs that change speed only, never results. The Python module
 * kunpbfv_b200.tune picks them by timing the candidates on the device and
 * caches the choice per device and parameter set. No counterpart in the
 * reference (its shapes are fixed at compile time). */
typedef enum {
    KBFV_TUNE_NTT_BLOCK_LOG = 0, /* 0 (default: built-in shapes) or 12..14: kbfv_ntt_fwd/inv on
                                    rings above 2^v points run as a column pass of log_n - v
                                    stages and blocks of 2^v points */
    KBFV_TUNE_BRANCHES = 1,      /* 1..4 (default 2): sub-batches of a batched multiply */
    KBFV_TUNE_HOST_CHUNK = 2,    /* 0..128 (default 0 = ~32 MiB of inputs): pairs per chunk of
                                    kbfv_mul_relin_host when its chunk_pairs is 0 */
    KBFV_TUNE_SPLIT_ROWS = 3,    /* 0..2^20 (default 48): at N = 2^14, transforms of at most this
                                    many rows (inside the multiply pipeline too) run as a radix-4
                                    column pass and 2^12-point blocks instead of one block per row */
    KBFV_TUNE_BCONV_THREADS = 4, /* 64, 128, 256 (default) or 512: CTA size of the base conversion
                                    Q -> R (the multiply's K2 and kbfv_bconv_*) */
    KBFV_TUNE_K5_THREADS = 5,    /* 64, 128 (default) or 256: CTA size of the multiply's
                                    scale-and-round / R -> Q / digit-lift kernels (K5) */
    KBFV_TUNE_K5_FUSED_PAIRS = 6, /* 0..128 (default 2): batches of at most this many pairs run K5
                                    as one kernel, larger ones as two (fewer registers each) */
    KBFV_TUNE_BCONV_CPT = 7,     /* 1 or 2 (default): coefficients per thread of the Q -> R base
                                    conversion (2: 16-byte loads and stores, table reads shared by
                                    two independent multiply-accumulate chains) */
    KBFV_TUNE_FUSE_Q2R_PAIRS = 8, /* 0..128 (default 1): multiplies of at most this many pairs (per
                                    sub-batch) run the Q -> R base extension in the loader of the
                                    forward NTT over R: the inverse NTT over Q stores its outputs
                                    scaled by (Q/q_i)^-1, and there is no base-conversion launch
                                    and no HBM round trip of the R limbs; each R row then reads
                                    all q_count Q limbs, which larger batches pay for in L2 traffic */
    KBFV_TUNE_L2_PREFETCH = 9,   /* 0 or 1 (default): NTT block kernels whose input is plain rows
                                    (standalone transforms, the multiply's INTT of its inputs and
                                    its NTTs over R and Q|P) ask L2 for the block one wave of CTAs
                                    ahead of their own */
    KBFV_TUNE_SPLIT_ROWS_ALONE = 10, /* 0..2^20 (default 148): KBFV_TUNE_SPLIT_ROWS for a multiply
                                    that runs as one stream (batches too small for sub-batches,
                                    kbfv_mul), where no sibling sub-batch fills idle SMs */
    KBFV_TUNE_MIN_BRANCH_PAIRS = 11 /* 1..64 (default 1): a batched multiply splits into
                                    KBFV_TUNE_BRANCHES sub-batches only with at least this many
                                    pairs in each */
} kbfv_tune_knob;
int kbfv_tune_set(kbfv_context* ctx, int knob, int64_t value);
int kbfv_tune_get(const kbfv_context* ctx, int knob, int64_t* value);
/* same for consecutive ciphertexts (stride 2*q_count*N words) */
int kbfv_mul_relin(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                   uint64_t* d_out, uint32_t count, kbfv_stream stream);
/* kbfv_mul_relin on ciphertexts in HOST memory (same layout): the pairs move
 * through device staging slots in chunks of at most `chunk_pairs` (0: the
 * context's KBFV_TUNE_HOST_CHUNK, else about 32 MiB of inputs; at most 128;
 * the first and last chunks are smaller), the
 * copy-in of one chunk overlapping the multiply of the previous and the
 * copy-out of the one before that. The copies
 * overlap only when the host buffers are page-locked (cudaHostAlloc /
 * cudaHostRegister). Ordered on `stream` like every call: the copies start after
 * the work queued on it, and h_out holds the products once `stream` has passed
 * the call. The reference multiplies device ciphertexts only (its callers copy
 * them in and out); no counterpart in the reference. */
int kbfv_mul_relin_host(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* h_ct_a, const uint64_t* h_ct_b,
                        uint64_t* h_out, uint32_t count, uint32_t chunk_pairs, kbfv_stream stream);

/* ---- key switching over a gadget decomposition of base 2^w --------------
 * No counterpart in the reference. a1*a2 = sum_i [a1*a2]_{q_i} * g_i (mod Q),
 * g_i = Q/q_i * [(Q/q_i)^-1]_{q_i}; each residue is cut into J = ceil(60 / w)
 * pieces of w bits (small integers, the same in every prime), so no base
 * conversion is needed and the key-switch noise is about J * q_count * 2^w *
 * sigma * N / P. Key: q_count * J components [a|b] over Q|P (NTT form, layout
 * [i*J + j][a|b][Q|P]): b = e - a*s + 2^{wj} * P * [prime == q_i] * s^2.
 * 4 <= w <= 30. Works at levels (kbfv_context_at_level) with the top-level key. */
int kbfv_keygen_relin_gadget(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint32_t log_base,
                             uint64_t* d_gk, kbfv_stream stream);
int kbfv_relinearize_gadget(kbfv_context* ctx, const uint64_t* d_gk, uint32_t log_base, const uint64_t* d_tensor,
                            uint64_t* d_ct, uint32_t count, kbfv_stream stream);
int kbfv_mul_relin_gadget(kbfv_context* ctx, const uint64_t* d_gk, uint32_t log_base, const uint64_t* d_ct_a,
                          const uint64_t* d_ct_b, uint64_t* d_out, uint32_t count, kbfv_stream stream);

/* ---- Galois automorphisms: rotations and conjugation ---------------------
 * BFVScheme::addLeftRotKey_23 / leftRotateAndEqual_23 / rightRotateAndEqual_23 /
 * addConjKey_23 (include/KeySwitch_23.cuh:71-166, 544-584): the automorphism
 * X -> X^g (g = 5^r mod 2N for a left rotation by r, the reference's rotGroups,
 * include/BFVcontext.cuh:788-799; g = 2N - 1 for conjugation) followed by a key
 * switch from s(X^g) back to s. In NTT form the automorphism is a permutation
 * of the evaluation points. The key (layout of the relinearisation key) encrypts
 * P * s(X^g) per digit. The reference applies the coefficient-domain automorphism
 * to its NTT-form secret key when it builds rotation keys (KeySwitch_23.cuh:133),
 * so its rotations do not decrypt; these do.
 * kbfv_galois_element: 5^rot_slots mod 2N, or 2N - 1 for rot_slots < 0. */
uint64_t kbfv_galois_element(const kbfv_context* ctx, int64_t rot_slots);
int kbfv_keygen_galois(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t galois_elt,
                       uint64_t* d_gk, kbfv_stream stream);
/* out = key_switch(automorphism(ct)); out may equal ct */
int kbfv_apply_galois(kbfv_context* ctx, const uint64_t* d_gk, uint64_t galois_elt, const uint64_t* d_ct,
                      uint64_t* d_out, uint32_t count, kbfv_stream stream);

/* ---- wire format ----------------------------------------------------------
 * No counterpart in the reference (it has no serialization). A 56-byte header
 * (magic "KBFVWIRE", version 1, kind, log_n, q_count, p_count, count, aux, a
 * digest of the context's Q, P and t, payload words per object) followed by the
 * objects' words, little-endian, in the device layout. Kinds: 1 ciphertext,
 * 2 plaintext coefficients, 3 secret key, 4 public key, 5 relinearisation key,
 * 6 Galois key (aux = Galois element), 7 gadget key (aux = log2 of the base),
 * 8 T-base key. Loading checks the header against the context (a ciphertext at
 * a lower level loads into that level's context) and fails with
 * KBFV_ERR_INVALID on any mismatch or truncation. */
size_t kbfv_wire_bytes(const kbfv_context* ctx, int kind, uint64_t aux, uint32_t count);
int kbfv_wire_save(kbfv_context* ctx, int kind, uint64_t aux, const uint64_t* d_obj, uint32_t count, void* h_buf,
                   size_t h_bytes, kbfv_stream stream);
int kbfv_wire_load(kbfv_context* ctx, int kind, const void* h_buf, size_t h_bytes, uint64_t* d_obj, uint32_t max_count,
                   uint32_t* count, uint64_t* aux, kbfv_stream stream);

/* ---- levels: fewer live ciphertext primes --------------------------------
 * A ciphertext at level l holds the first l primes of Q (2 x l limbs, NTT form).
 * kbfv_context_at_level: the context for l live primes (l = q_count returns
 * ctx itself); owned by ctx and freed with it. It shares the top level's keys:
 * its multiply reads the top-level relinearisation key through a limb map (digit
 * d keeps the top level's primes [d*alpha, (d+1)*alpha) that are still live,
 * plus P), its decryption the top-level secret key. Keys and encryptions are made
 * on the top-level context. No counterpart in the reference (its rescale is
 * CKKS-style flooring, include/BFVScheme.cuh:400-502). */
int kbfv_context_at_level(kbfv_context* ctx, uint32_t live_q, kbfv_context** out);
/* BFV modulus switch: divide by the last live prime and round, c' = round(c / q_l),
 * in NTT form (SEAL's divide_and_round_q_last). ctx_level is the input's level
 * context (q_count >= 2); d_out receives count ciphertexts of q_count - 1 limbs
 * and must not overlap d_ct. */
int kbfv_mod_switch(kbfv_context* ctx_level, const uint64_t* d_ct, uint64_t* d_out, uint32_t count,
                    kbfv_stream stream);
/* Multiply + relinearise a batch whose pairs sit at different levels: pair i has
 * live_q[i] live primes (both inputs and the output at that level). One call on
 * one stream: up to 128 pairs in up to 8 levels run as ONE launch sequence of
 * the multiply pipeline (every kernel takes its items' level constants from a
 * per-level table; the top-level key is read through a limb map), larger
 * batches as several. d_rlk is the top-level key. */
int kbfv_mul_relin_levels(kbfv_context* ctx, const uint64_t* d_rlk, const uint32_t* live_q,
                          const uint64_t* const* ct_a, const uint64_t* const* ct_b, uint64_t* const* out,
                          uint32_t count, kbfv_stream stream);

/* ---- key switch over the auxiliary T base (the reference's own method) ---
 * Available when the context has T primes (kbfv_params.t_count), q_count is a
 * multiple of p_count and dnum == q_count / p_count (the reference's parameter
 * sets: kbfv_context_create_reference). Layouts (N words per limb):
 *   T-form key    [a|b][digit][Ri block][T prime], NTT form over T
 *   Qj digits     [poly][Qj block][T prime]
 *   Ri blocks     [poly][Ri block][T prime]
 * Qj block i = Q primes [i*p_count, (i+1)*p_count); Ri block b = P|Q primes in
 * the reference's order (P first) [b*gamma, (b+1)*gamma).
 * kbfv_context_klss: block counts and the T-form key size in words. */
int kbfv_context_klss(const kbfv_context* ctx, uint32_t* ri_blocks, uint32_t* qj_blocks, uint64_t* key_words);
/* addMultKey_23's key conversion (include/KeySwitch_23.cuh:55-65):
 * relinearisation key [digit][a|b][Q|P] (NTT) -> T-form key */
int kbfv_rlk_to_klss(kbfv_context* ctx, const uint64_t* d_rlk, uint64_t* d_rlk_t, kbfv_stream stream);
/* modUpQjtoT_23 (include/BasisConv.cuh:86-151): [poly][Q] coefficient form -> Qj digits over T */
int kbfv_klss_modup_qj_to_t(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                            kbfv_stream stream);
/* modUpPQtoT_23 (include/BasisConv.cuh:11-79): [poly][Q|P] coefficient form -> Ri blocks over T */
int kbfv_klss_modup_pq_to_t(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                            kbfv_stream stream);
/* external_product_T (include/ExternalProduct.cuh:11-112) of NTT-form digits
 * [count][Qj][T] with the T-form key, returned in COEFFICIENT form
 * ([count][a|b][Ri][T]; the inverse NTT over T is fused) */
int kbfv_klss_external_product(kbfv_context* ctx, const uint64_t* d_digits, const uint64_t* d_rlk_t,
                               uint64_t* d_out, uint32_t count, kbfv_stream stream);
/* modUpTtoPQl_23 (include/BasisConv.cuh:159-226): centred exact Ri blocks over T
 * (coefficient form) -> [poly][Q|P] */
int kbfv_klss_t_to_pq(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                      kbfv_stream stream);
/* key switch of a1*a2 as multAndEqual_23 does it (include/KeySwitch_23.cuh:277-305):
 * tensors -> ciphertexts, with the T-form key */
int kbfv_relinearize_klss(kbfv_context* ctx, const uint64_t* d_rlk_t, const uint64_t* d_tensor, uint64_t* d_ct,
                          uint32_t count, kbfv_stream stream);
/* multAndEqual_23 (include/KeySwitch_23.cuh:244-310) with the reference's key
 * switch, as one batched launch sequence (consecutive ciphertexts) */
int kbfv_mul_relin_klss(kbfv_context* ctx, const uint64_t* d_rlk_t, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                        uint64_t* d_out, uint32_t count, kbfv_stream stream);

/* ---- multiply without allocating -------------------------------------
 * No counterpart in the reference. Same result as kbfv_mul_relin, for callers
 * that must not allocate device memory during a call: services that fix their
 * device-memory budget at start-up and cannot risk an out-of-memory failure in
 * the middle of a request, code running inside another framework's allocator
 * or memory-pool hook (where calling cudaMalloc again is forbidden), and
 * latency-bound paths that cannot afford the implicit device synchronisation of
 * cudaMalloc / cudaFree. Its scratch is a statically sized device array inside
 * libkbfv.so of KBFV_NOALLOC_SCRATCH_BYTES (40 MiB).
 * Limit: one call of `count` pairs needs
 *   count * N * 8 * (4q + 4r + 3(q + r) + 2q + (dnum + 2)(q + p) [+ nqj*nt + 2*nri*nt with a T base])
 * bytes (q ciphertext primes, r = q + 1, p special primes; the bracket only for
 * contexts built with T-base primes): 143 limbs of 128 KiB = 17.9 MiB per pair
 * at N=16384 with 7 + 1 primes and dnum 1, so 2 pairs; with dnum 7 one pair.
 * For a single pair kbfv_mul_relin_scratch_bytes(ctx, count) returns the same
 * figure (from 2 x KBFV_TUNE_MIN_BRANCH_PAIRS pairs on, 2 by default, it counts
 * the batched multiply's sub-batches).
 * Larger requests return KBFV_ERR_INVALID and launch nothing; nothing on this
 * path calls cudaMalloc, cudaFree or any allocating routine, and the
 * context's own scratch arena is never touched (kbfv_context_arena_bytes
 * stays where it was).
 * The array is part of the library's multiply module. The CUDA runtime
 * allocates it when it loads that module in a context: with lazy module
 * loading (the default since CUDA 12.2) at the first call in that context of
 * kbfv_mul_relin, kbfv_mul_relin_batch, kbfv_mul_relin_host, kbfv_mul,
 * kbfv_relinearize or of this entry point (or of the gadget, T-base and
 * Galois key switches built on them; kbfv_mul_relin_levels runs kernels of
 * another module); with eager loading when the context is created. It is held until the process exits (or
 * the context is destroyed). A caller with a fixed budget makes one multiply
 * call on each device during start-up, before any stream capture and before
 * taking its budget snapshot. The first call of this entry point in each CUDA
 * context also resolves the array's device address (cudaGetSymbolAddress),
 * which is why that first call belongs before any stream capture too; later
 * calls only look the address up. The context's device must be current.
 * All calls share the one array: calls that overlap on the GPU (several
 * streams or contexts) race and must be serialised by the caller. Every scratch
 * word is written before it is read, so nothing needs clearing between calls;
 * the array keeps the last call's intermediate values. */
#define KBFV_NOALLOC_SCRATCH_BYTES ((size_t)40 << 20)
int kbfv_mul_relin_noalloc(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                           uint64_t* d_out, uint32_t count, kbfv_stream stream);

/* ---- captured multiplies -------------------------------------------------
 * No counterpart in the reference. A plan binds a multiply (the same operation
 * and product as kbfv_mul_relin) to fixed device buffers: `count` consecutive
 * pairs at d_ct_a / d_ct_b, products to d_out. kbfv_plan_launch multiplies
 * whatever the buffers hold at launch time. Its first launch runs the multiply
 * eagerly on `stream` and records the same launch sequence into a CUDA graph
 * (recording executes nothing); later launches replay that graph with one
 * cudaGraphLaunch (one pair per call at N=16384: about 135 instead of 160 us,
 * the ~14 kernel launches of the eager path issued as one). A launch after
 * the context's scratch arena moved or its tuning knobs changed records the
 * graph again (eagerly, as the first). Creating a plan sizes the context's
 * arena for `count` pairs (kbfv_reserve). Plans of one context share that
 * arena with every other call on the context, so their launches must be
 * ordered with those calls (one stream, or events), as for kbfv_mul_relin.
 * A plan refers to its context and buffers: destroy it before them. */
typedef struct kbfv_plan kbfv_plan;
int kbfv_plan_mul_relin(kbfv_context* ctx, const uint64_t* d_rlk, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                        uint64_t* d_out, uint32_t count, kbfv_plan** plan);
int kbfv_plan_launch(kbfv_plan* plan, kbfv_stream stream);
/* The same for a batch at mixed levels (kbfv_mul_relin_levels' arguments; the
 * arrays are copied, the buffers they point to are bound): each launch replays
 * the whole uneven batch as one CUDA graph launch. */
int kbfv_plan_mul_relin_levels(kbfv_context* ctx, const uint64_t* d_rlk, const uint32_t* live_q,
                               const uint64_t* const* ct_a, const uint64_t* const* ct_b, uint64_t* const* out,
                               uint32_t count, kbfv_plan** plan);
/* launches so far and how many of them recorded the graph */
int kbfv_plan_info(const kbfv_plan* plan, uint64_t* launches, uint64_t* captures);
int kbfv_plan_destroy(kbfv_plan* plan);

/* invariant noise budget in bits of one ciphertext (host-side diagnostic, synchronous) */
int kbfv_noise_budget(kbfv_context* ctx, const uint64_t* d_sk, const uint64_t* d_ct, double* bits);

/* ---- randomness ---------------------------------------------------------
 * XSalsa20 keystream (the reference's RNG::generateRandom_device,
 * include/RNG.cuh:18-51, corrected: "expand 32-byte k" constants, HSalsa20
 * subkey, 64-bit nonce). compat != 0 reproduces the reference's variant
 * (zero constants, 32-bit nonce from nonce[0..3], no HSalsa20). */
int kbfv_salsa20_stream(const uint8_t key[32], const uint8_t nonce[24], uint64_t block0, uint8_t* d_out,
                        size_t nbytes, int compat, kbfv_stream stream);
/* The reference's sampler conversions (include/Sampler_impl.cuh:13-108) applied
 * to caller-supplied random words, restated bit for bit (so the same words give
 * the reference's samples): kind 0 uniform (limbs x N 64-bit words; double
 * scaling, biased like the reference's), 1 Gaussian sigma 3.2 (N 32-bit words;
 * normcdfinvf, clamp +-19.2, truncation), 2 ternary (N bytes; `probability` of 0),
 * 3 Hamming weight h (h 32-bit positions then h sign bytes; collisions keep the
 * last writer, as in the reference). Output: limbs x N residues for primes
 * prime0 .. prime0+limbs-1 of the context's table. */
int kbfv_sample_compat(kbfv_context* ctx, int kind, const void* d_rand, uint64_t* d_out, uint32_t prime0,
                       uint32_t limbs, uint32_t h, double probability, kbfv_stream stream);

#ifdef __cplusplus
}
#endif
#endif /* KBFV_H */
