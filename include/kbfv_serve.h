/*
 * kbfv_serve.h -- request serving over the B200 multiply path.
 *
 * No counterpart in kunpBFV (its drivers run one operation at a time from one
 * host thread, perf_mult.cu / correct_mult.cu). A server owns one scheduler
 * thread and, per registered ring (one kbfv_context with its keys), a CUDA
 * stream. Requests are chains of multiply+relinearise and add operations on
 * fresh encryptions:
 *
 *     acc = Enc(x_0);  for i in 0..n_ops-1:  acc = acc (op_i) Enc(x_{i+1});
 *     result = Decode(Dec(acc))
 *
 * Scheduling is continuous batching at operation granularity: every scheduler
 * iteration admits waiting requests while the device budget has room (their
 * plaintexts, ciphertexts and result live in one block of a device slab of
 * hbm_budget_bytes), then advances EVERY admitted request of a ring by one
 * operation: all multiplies of the iteration go to the GPU as batched
 * kbfv_mul_relin_batch launches (pointer arrays, requests at different chain
 * positions side by side), adds follow, finished chains are decrypted and read
 * back. Each ring's iterations are queued on its own stream, so rings of
 * different N overlap on the device; up to inflight_iterations iterations per
 * ring are queued ahead of the GPU. Encryption of request r uses the ring's
 * seed and ids enc_id .. enc_id + n_ops, so a request's ciphertexts and result
 * do not depend on what else is being served.
 *
 * Thread safety: submit / wait / stats may be called from any host threads.
 * While a server runs, its rings' contexts must not be used by other callers.
 */
#ifndef KBFV_SERVE_H
#define KBFV_SERVE_H

#include <stdint.h>

#include "kbfv.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct kbfv_server kbfv_server;

typedef struct {
    uint64_t hbm_budget_bytes;     /* device bytes for request state; admission waits when full */
    uint64_t pinned_bytes;         /* pinned host staging for inputs and results (0 = 256 MiB) */
    uint32_t max_batch;            /* ciphertext pairs per batched multiply launch, 1..128 */
    uint32_t max_active;           /* admitted requests per ring, 0 = limited by the budget only */
    uint32_t inflight_iterations;  /* iterations queued ahead per ring, 1..8 (0 = 2) */
} kbfv_server_config;

enum { KBFV_OP_MUL = 0, KBFV_OP_ADD = 1 };
enum { KBFV_REQ_RETURN_CT = 1 };  /* also copy the final ciphertext back */

typedef struct {
    uint64_t submitted, completed, failed;
    uint64_t iterations;           /* scheduler iterations issued (all rings) */
    uint64_t mul_launches;         /* batched multiply calls */
    uint64_t mul_ops, add_ops;     /* operations executed */
    uint64_t bytes_in_use, bytes_peak;  /* device slab */
    uint32_t pending, active;      /* right now, all rings */
} kbfv_server_stats;

int kbfv_server_create(const kbfv_server_config* cfg, kbfv_server** out);
/* register a ring: the context and its device-resident keys (public key
 * [a|b] over Q, relinearisation key, secret key), all owned by the caller and
 * valid until kbfv_server_destroy. Reserves the context's scratch for
 * max_batch pairs. Must precede kbfv_server_start. */
int kbfv_server_add_ring(kbfv_server* s, kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_pk,
                         const uint64_t* d_rlk, const uint64_t* d_sk, uint32_t* ring_id);
int kbfv_server_start(kbfv_server* s);
/* h_slots: (n_ops + 1) x N slot values mod t (copied before return);
 * ops: n_ops entries of KBFV_OP_MUL / KBFV_OP_ADD, 1 <= n_ops <= 8. */
int kbfv_server_submit(kbfv_server* s, uint32_t ring, const uint64_t* h_slots, uint32_t n_ops, const uint8_t* ops,
                       uint64_t enc_id, uint32_t flags, uint64_t* request_id);
/* Wait for a request (timeout_ms < 0: no limit; KBFV_ERR_UNSUPPORTED on
 * timeout), copy its N result slots and, if it was submitted with
 * KBFV_REQ_RETURN_CT, its final ciphertext (2 x q_count x N words); latency
 * is submit-to-result in milliseconds. Each request is waited on once. */
int kbfv_server_wait(kbfv_server* s, uint64_t request_id, int64_t timeout_ms, uint64_t* h_slots_out,
                     uint64_t* h_ct_out, double* latency_ms);
int kbfv_server_get_stats(kbfv_server* s, kbfv_server_stats* out);
/* message of the last failed kbfv_server_wait on this thread */
const char* kbfv_server_last_error(void);
/* finishes every submitted request, stops the scheduler, frees the server */
int kbfv_server_destroy(kbfv_server* s);

#ifdef __cplusplus
}
#endif
#endif
