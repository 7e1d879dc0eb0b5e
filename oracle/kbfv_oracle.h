/*
 * kbfv_oracle.h -- CPU restatement of kunpBFV's BFV homomorphic-multiply path.
 *
 * TEST INFRASTRUCTURE. This library is the checker for the CUDA product in
 * kunpbfv_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it. Nothing in the product links or calls it.
 *
 * Every function restates an algorithm of the reference (file:line cited in
 * kbfv_oracle.c). Layout everywhere is limb-major uint64: poly[limb][coeff].
 * Prime indices refer to the oracle context's prime table, ordered
 *   [ Q (nq) | P (np) | R (nq+1) | T (nt) | plain modulus t ].
 */
#ifndef KBFV_ORACLE_H
#define KBFV_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* ---- primes and roots ------------------------------------------------- */
int      orc_is_prime(uint64_t n);
/* get_primes_below: candidates upper-2N, upper-4N, ... above 2^(bits(upper)-1).
 * require_root != 0 additionally skips primes whose 2N-th root (by the
 * reference's primitive-root search) is not primitive. Returns count found. */
size_t   orc_primes_below(uint64_t n, uint64_t upper, size_t count, uint64_t* out, int require_root);
size_t   orc_primes_bits(uint64_t n, int bits, size_t count, const uint64_t* skip, size_t nskip,
                         uint64_t* out);
uint64_t orc_primitive_root(uint64_t q);
uint64_t orc_root_2n(uint64_t q, uint64_t n);
int      orc_root_is_primitive(uint64_t psi, uint64_t q, uint64_t n);

/* ---- context ----------------------------------------------------------- */
/* q: nq ciphertext primes; p: np special primes; dnum: key-switch digits
 * (dnum < 0: digit size alpha = -dnum primes, digits = ceil(nq / alpha));
 * tk: optional KLSS T primes (nt may be 0), gamma: KLSS Ri block size.
 * The R base is derived here by the reference rule (nq+1 primes below min q). */
orc_ctx* orc_create(uint32_t log_n, uint64_t t, const uint64_t* q, int nq,
                    const uint64_t* p, int np, int dnum,
                    const uint64_t* tk, int nt, int gamma);
void     orc_destroy(orc_ctx* c);
/* 1: mul_tensor reproduces the reference's in-place alpha reduction (see scale_round_qr_r_ref) */
void     orc_set_ref_compat(orc_ctx* c, int on);
int      orc_prime_count(const orc_ctx* c);          /* total entries in the prime table */
void     orc_primes(const orc_ctx* c, uint64_t* out);
uint64_t orc_psi(const orc_ctx* c, int prime_idx);

/* ---- NTT (in place, one row of N per call, rows consecutive) ------------ */
void orc_ntt_fwd(const orc_ctx* c, int prime_idx, uint64_t* rows, int nrows);
void orc_ntt_inv(const orc_ctx* c, int prime_idx, uint64_t* rows, int nrows);

/* ---- HPS pieces -------------------------------------------------------- */
void orc_bconv_q_to_r(const orc_ctx* c, const uint64_t* in_q, uint64_t* out_r);
void orc_bconv_r_to_q(const orc_ctx* c, const uint64_t* in_r, uint64_t* out_q);
/* ct1, ct2: 2 polys x (nq+nr) limbs in NTT form over Q|R; out: 3 polys */
void orc_tensor_qr(const orc_ctx* c, const uint64_t* ct1, const uint64_t* ct2, uint64_t* out);
void orc_scale_round_qr_r(const orc_ctx* c, const uint64_t* in_qr, uint64_t* out_r);
/* the reference's variant: alpha reduced in place across the R primes */
void orc_scale_round_qr_r_ref(const orc_ctx* c, const uint64_t* in_qr, uint64_t* out_r);
/* variant: -1 = select by bit sizes as the reference does, else 0..3 */
void orc_decrypt_round(const orc_ctx* c, const uint64_t* in_q, uint64_t* out, int variant);
int  orc_decrypt_variant(const orc_ctx* c);
void orc_delta_m(const orc_ctx* c, const uint64_t* m, uint64_t* out_q);

/* ---- key switching ----------------------------------------------------- */
/* d2: nq limbs coefficient form -> dnum polys of (nq+np) limbs, coefficient form */
void orc_modup(const orc_ctx* c, const uint64_t* d2, uint64_t* out);
/* in: 2 polys x (nq+np) limbs coefficient form -> 2 polys x nq limbs */
void orc_moddown(const orc_ctx* c, const uint64_t* in, uint64_t* out, int npoly);
/* key switching over a gadget decomposition of base 2^w (J = ceil(60 / w) pieces
 * per ciphertext prime); gk: nq * J x [a | b] x (nq+np) limbs, NTT form */
int  orc_gadget_pieces(int w);
void orc_keygen_relin_gadget(const orc_ctx* c, const uint8_t key[32], const uint64_t* sk, int w, uint64_t* gk);
void orc_relinearize_gadget(const orc_ctx* c, const uint64_t* d, const uint64_t* gk, int w, uint64_t* ct);
/* Galois automorphism X -> X^g on NTT-form limbs; key switching key from s(X^g)
 * to s (layout of the relinearisation key); automorphism + key switch of a ciphertext */
void orc_galois_ntt(const orc_ctx* c, uint64_t g, const uint64_t* in, uint64_t* out, int nlimbs);
void orc_keygen_galois(const orc_ctx* c, const uint8_t key[32], const uint64_t* sk, uint64_t g, uint64_t* gk);
void orc_apply_galois(const orc_ctx* c, const uint64_t* gk, uint64_t g, const uint64_t* ct, uint64_t* out);
/* BFV modulus switch by the last prime: npoly polys of nq limbs (NTT) -> nq - 1 limbs */
void orc_mod_switch(const orc_ctx* c, const uint64_t* ct, uint64_t* out, int npoly);
/* KLSS restatement (reference's own key-switch base conversions) */
int  orc_klss_ri_blocks(const orc_ctx* c);
int  orc_klss_qj_blocks(const orc_ctx* c);
void orc_klss_modup_qj_to_t(const orc_ctx* c, const uint64_t* d2, uint64_t* out);
void orc_klss_modup_pq_to_t(const orc_ctx* c, const uint64_t* in_pq_ref_order, uint64_t* out);
void orc_klss_external_product(const orc_ctx* c, const uint64_t* digits_t, const uint64_t* key_t,
                               uint64_t* out);
void orc_klss_modup_t_to_pq(const orc_ctx* c, const uint64_t* in_t, uint64_t* out_pq_ref_order, int npoly);
void orc_klss_moddown(const orc_ctx* c, const uint64_t* in_pq_ref_order, uint64_t* out_q, int npoly);
/* the reference's full KLSS relinearisation of a tensor [a1a2|cross|b1b2] (NTT form) */
void orc_klss_relinearize(const orc_ctx* c, const uint64_t* d, const uint64_t* key_t, uint64_t* ct);

/* ---- randomness and samplers ------------------------------------------ */
void orc_hsalsa20(const uint8_t key[32], const uint8_t nonce16[16], uint8_t out[32]);
void orc_xsalsa20_stream(const uint8_t key[32], const uint8_t nonce[24], uint64_t block0,
                         uint8_t* out, size_t nbytes);
/* the reference's quirky Salsa20 variant: zero sigma, 32-bit nonce, no HSalsa20 */
void orc_salsa20_compat_stream(const uint8_t key[32], uint64_t nonce, uint8_t* out, size_t nbytes);
void orc_gaussian_cdt(double sigma, int bound, uint64_t* table /* 2*bound+1 */);
/* deterministic sample streams: domain/id/sub select the XSalsa20 nonce */
void orc_sample_uniform(const orc_ctx* c, const uint8_t key[32], uint32_t domain, uint64_t id,
                        uint32_t sub, const int* prime_idx, int nlimbs, uint64_t* out);
void orc_sample_ternary(const orc_ctx* c, const uint8_t key[32], uint32_t domain, uint64_t id,
                        uint32_t sub, int64_t* out);
void orc_sample_gaussian(const orc_ctx* c, const uint8_t key[32], uint32_t domain, uint64_t id,
                         uint32_t sub, int64_t* out);
void orc_sample_hwt(const orc_ctx* c, const uint8_t key[32], uint32_t domain, uint64_t id,
                    uint32_t sub, int h, int64_t* out);

/* ---- scheme ------------------------------------------------------------ */
/* secret: nq+np limbs NTT form. secret_kind 0 = ternary uniform, 1 = HWT(h) */
void orc_keygen_secret(const orc_ctx* c, const uint8_t key[32], int secret_kind, int h, uint64_t* sk);
/* pk: [a | b] each nq limbs NTT form */
void orc_keygen_public(const orc_ctx* c, const uint8_t key[32], const uint64_t* sk, uint64_t* pk);
/* rlk: dnum x [a | b] each (nq+np) limbs NTT form */
void orc_keygen_relin(const orc_ctx* c, const uint8_t key[32], const uint64_t* sk, uint64_t* rlk);
void orc_encode(const orc_ctx* c, const uint64_t* slots, uint64_t* m);   /* INTT mod t */
void orc_decode(const orc_ctx* c, const uint64_t* m, uint64_t* slots);   /* NTT mod t */
/* ct: [a | b] each nq limbs NTT form */
void orc_encrypt(const orc_ctx* c, const uint8_t key[32], uint64_t enc_id, const uint64_t* pk,
                 const uint64_t* m, uint64_t* ct);
void orc_decrypt(const orc_ctx* c, const uint64_t* sk, const uint64_t* ct, uint64_t* m);
void orc_add(const orc_ctx* c, const uint64_t* x, const uint64_t* y, uint64_t* out, int npoly);
void orc_mul_plain(const orc_ctx* c, const uint64_t* ct, const uint64_t* pt_ntt, uint64_t* out);
/* HPS tensor + scale-and-round: 2 cts -> 3 polys [a1*a2 | a1*b2+b1*a2 | b1*b2], NTT form over Q */
void orc_mul_tensor(const orc_ctx* c, const uint64_t* ct1, const uint64_t* ct2, uint64_t* d);
void orc_relinearize(const orc_ctx* c, const uint64_t* d, const uint64_t* rlk, uint64_t* ct);
void orc_mul_relin(const orc_ctx* c, const uint64_t* ct1, const uint64_t* ct2, const uint64_t* rlk,
                   uint64_t* ct);
/* invariant noise budget in bits (SEAL's definition), <0 means decryption failure */
double orc_noise_budget(const orc_ctx* c, const uint64_t* sk, const uint64_t* ct);

#ifdef __cplusplus
}
#endif
#endif
