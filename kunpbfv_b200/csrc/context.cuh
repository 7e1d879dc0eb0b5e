// Parameter-set context: host precompute and the device-side constant view.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "ntt.cuh"

namespace kbfv {

constexpr int kMaxPrimes = 96;   // whole prime table [Q|P|R|T|t]
constexpr int kMaxQ = 32;        // ciphertext primes per context
constexpr int kMaxP = 8;         // special primes

// Launch shapes of the multiply pipeline (speed only; kbfv_tune_set). Set by
// build_context; kernels never read them.
struct LaunchShape {
    int split_rows14;    // N = 2^14 transforms of at most this many rows: column pass + 2^12-point blocks
    int bconv_threads;   // CTA size of the Q -> R base conversion
    int bconv_cpt;       // coefficients per thread of the base conversion (1 or 2)
    int k5_threads;      // CTA size of K5
    int k5_fused_pairs;  // batches of at most this many pairs run K5 as one kernel
    int fuse_q2r_pairs;  // batches of at most this many pairs run the Q -> R base extension in the
                         // loader of the NTT over R (no K2 launch)
    int l2_prefetch;     // 1: block kernels ask L2 for the block one wave of CTAs ahead
    int split_rows_alone;  // split_rows14 for a multiply that runs as one stream
};

// Everything a kernel needs, passed by value (all pointers into one device pool).
struct DevConsts {
    int logn;
    int nq, np, nr, nt, dnum, alpha, npq, nqr;
    int idx_p, idx_r, idx_t, idx_pt;   // prime-table offsets of P, R, T, plain modulus
    uint64_t t;
    const uint64_t* mods;
    const uint64_t* mu_hi;
    const uint64_t* mu_lo;
    const uint64_t* mu_prod;  // floor(2^(62+k) / q), k = bit length (barrett_prod)
    const tw_t* tw_fwd;   // [prime][N]
    const tw_t* tw_inv;   // [prime][N]; [0] = n^-1, [1] = psi_br^-1[1] * n^-1
    // HPS base extension Q -> R
    const uint64_t *q2r_hatinv, *q2r_hatinvs, *q2r_hat, *q2r_alpha;
    const double* q2r_inv;
    const tw_t* q2r_fold;  // [nq][2]: the inverse NTT's last-stage constants times (Q/q_i)^-1 mod q_i
    // HPS base extension R -> Q
    const uint64_t *r2q_hatinv, *r2q_hatinvs, *r2q_hat, *r2q_alpha;
    const double* r2q_inv;
    // t/Q scale-and-round Q|R -> R
    const double* sr_frac;       // [nq]
    const uint64_t* sr_c;        // [nr][nq+1]
    // decrypt rounding
    const uint64_t *dec_mod_t, *dec_mod_t_s, *dec_modB_t, *dec_modB_t_s;
    const double *dec_frac, *dec_fracB;
    int dec_variant, qmsbhf;
    // delta * m
    uint64_t negq_mod_t, negq_mod_t_s;
    const uint64_t *tinv_q, *tinv_qs;
    // key switching
    const uint64_t *p_mod_q, *pinv_q, *pinv_qs, *phatinv_p, *phatinv_ps, *phat_mod_q;
    const uint64_t *dig_hatinv, *dig_hatinvs, *dig_hat_mod, *dig_q_mod;
    const uint64_t* dig_vq_mod;  // [d][v = 0..alpha][npq]: v * Q_d mod p_m
    int key_nq, key_npq;         // limb layout of the relinearisation key (top level's Q and Q|P counts)
    // modulus switch: q_last^-1 mod q_i (+ Shoup), floor(q_last / 2) mod q_i, for i < nq - 1
    const uint64_t *ms_qlinv, *ms_qlinvs, *ms_half_mod;
    uint64_t ms_half;
    // Gaussian table
    const uint64_t* gauss_cdt;
    int gauss_bound;
    LaunchShape shape;
};

constexpr int kMaxBlk = 16;  // primes per block of the T-base key switch (p_count or gamma)
constexpr int kMaxT = 12;    // T primes

// Constants of the reference's key switch over the auxiliary T base (KLSS).
// Qj blocks: block i = Q primes [i*np, (i+1)*np). Ri blocks: the P|Q primes in
// the reference's order (P first, then Q), gamma per block.
struct KlssConsts {
    int nt, gamma, nri, nqj;
    const uint64_t *qj_hatinv, *qj_hatinvs;  // [nqj][np]
    const uint64_t* qj_hat_t;                // [nqj][nt][np]
    const uint64_t* qj_mod_t;                // [nqj][nt]
    const uint64_t *ri_hatinv, *ri_hatinvs;  // [nri][gamma]
    const uint64_t* ri_hat_t;                // [nri][nt][gamma]
    const uint64_t* ri_mod_t;                // [nri][nt]
    const uint64_t *thatinv, *thatinvs;      // [nt]: (T/t_k)^-1 mod t_k
    const uint64_t* that_pq;                 // [npq][nt]: T/t_k mod r_m, m in reference order
    const uint64_t* t_pq;                    // [npq]: T mod r_m
    const uint64_t* halft_t;                 // [nt]: floor(T/2) mod t_k
    const uint64_t* halft_pq;                // [npq]: floor(T/2) mod r_m
};

struct Context {
    // parameters
    int logn = 0;
    uint64_t n = 0;
    uint64_t t = 0;
    int nq = 0, np = 0, nr = 0, nt = 0, gamma = 1, dnum = 1, alpha = 1;
    std::vector<uint64_t> mods;  // Q | P | R | T | t
    int dec_variant = 0;

    // device
    void* pool = nullptr;       // constants
    DevConsts dc{};
    // host copies used by host-side diagnostics
    std::vector<uint64_t> h_q2r_hatinv;

    // scratch arena (grows; never shrinks while the context lives)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // device pointer tables for batched calls
    uint64_t** d_ptrs = nullptr;
    size_t d_ptrs_cap = 0;
    uint64_t** h_ptrs = nullptr;  // pinned staging
    cudaEvent_t ptrs_event = nullptr;
    std::mutex mu;
    int device = 0;
    // T-base key switch: available when T primes are given and its blocks
    // line up with the hybrid digits (alpha == p_count, dnum == q_count / p_count)
    bool klss_ok = false;
    KlssConsts kc{};
    // seed used by keygen / encryption calls that pass no seed (kbfv_set_seed)
    uint8_t seed[32] = {0};
    // levels: contexts for fewer live primes, owned by the top level (index = live primes)
    const Context* parent = nullptr;
    std::vector<void*> levels;
    // batched multiplies run as `branches` sub-batches on the caller's stream and
    // auxiliary streams (forked and joined with events), so one sub-batch's
    // partial last wave overlaps the others' kernels
    int branches = 2;
    int min_branch_pairs = 1;  // pairs per sub-batch at least (smaller batches run as one stream)
    // tuning knobs (kbfv_tune_set): block size 2^ntt_block_log of the standalone
    // NTT on rings above it (the rest runs as a column pass of logn - ntt_block_log
    // stages); pairs per chunk of the host-memory multiply (0: by bytes)
    int ntt_block_log = 0;  // 0: built-in shapes
    int host_chunk = 0;
    cudaStream_t aux[3] = {nullptr, nullptr, nullptr};
    cudaEvent_t fork_ev = nullptr, join_ev[3] = {nullptr, nullptr, nullptr};
    // multiplies of ciphertexts in host memory: copy-in, two compute and
    // copy-out streams (hs[0..3]); per staging slot the events that mark its
    // inputs copied in, its product computed and its product copied out
    cudaStream_t hs[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t hfork = nullptr, hjoin[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t hin[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t hcomp[4] = {nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t hout[4] = {nullptr, nullptr, nullptr, nullptr};
    // batches of pairs at several levels run as one launch sequence: slot l of
    // this device array holds the DevConsts of the level with l live primes (the
    // top level's own in slot nq), uploaded when that level is first used
    DevConsts* d_level_consts = nullptr;
    std::vector<uint8_t> level_uploaded;
};

}  // namespace kbfv
