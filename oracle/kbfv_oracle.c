/*
 * kbfv_oracle.c -- CPU restatement of kunpBFV's BFV homomorphic-multiply path.
 *
 * TEST INFRASTRUCTURE: this is the checker for the CUDA product. Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Build with -ffp-contract=off: every floating-point step below is written
 * out explicitly. The reference's CUDA build (nvcc default -fmad=true)
 * contracts `acc += (double)x * c` into a fused multiply-add, so those steps
 * are restated with fma(); the single-precision divisions and sums of the
 * key-switch lift are plain IEEE operations in source order.
 *
 * Parity anchors (reference file:line, paths inside the kunpBFV project):
 *   NTT convention      include/Utils.cuh:54-101 (root search), :171-191 (tables),
 *                       include/ntt_60bit.cuh:289-313 (CT/GS butterflies)
 *   HPS base conversion include/BasisConv_QR.cuh:53-207, include/poly_arithmetic.cuh:1078-1178
 *   HPS tensor          include/poly_arithmetic.cuh:1180-1219
 *   QR->R scale-round   include/poly_arithmetic.cuh:1263-1316, include/BFVcontext.cuh:1267-1389
 *   decrypt round       include/poly_arithmetic.cuh:930-1075, include/BFVcontext.cuh:1680-1717,
 *                       constants include/BFVcontext.cuh:1030-1156
 *   delta * m           include/poly_arithmetic.cuh:902-927, include/BFVcontext.cuh:881-926
 *   key-switch lift     include/BasisConv.cuh:86-135 (float estimate), :229-319 (mod down)
 *   KLSS conversions    include/BasisConv.cuh:11-226, include/ExternalProduct.cuh:11-53
 *   encode / decode     include/Encoder.cuh:23-112
 *   encrypt / decrypt   include/BFVScheme.cuh:57-166
 *   relin key layout    include/KeySwitch_23.cuh:21-66
 *   samplers            include/Sampler_impl.cuh:13-108, include/RNG_impl.cuh:70-176
 */
#include "kbfv_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef unsigned __int128 u128;

/* ======================================================================= */
/* scalar modular arithmetic                                               */
/* ======================================================================= */
static inline u64 mulmod(u64 a, u64 b, u64 q) { return (u64)(((u128)a * b) % q); }
static inline u64 addmod(u64 a, u64 b, u64 q) { u64 c = a + b; return c >= q ? c - q : c; }
static inline u64 submod(u64 a, u64 b, u64 q) { return a >= b ? a - b : a + q - b; }
static u64 powmod(u64 a, u64 e, u64 q) {
    u64 r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = mulmod(r, a, q);
        a = mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}
/* modinv128 (include/Utils.cuh:45-51): Fermat inverse, q prime */
static u64 invmod(u64 a, u64 q) { return powmod(a % q, q - 2, q); }
/* x_Shoup (include/Utils.cuh:38-43) */
static inline u64 shoup(u64 w, u64 q) { return (u64)(((u128)w << 64) / q); }
/* multiply_and_reduce_shoup (include/uintarith_bfv.h:960-969): exact a*w mod q */
static inline u64 mulshoup(u64 a, u64 w, u64 ws, u64 q) {
    u64 hi = (u64)(((u128)a * ws) >> 64);
    u64 r = a * w - hi * q;
    return r >= q ? r - q : r;
}
static int bit_count(u64 x) { int b = 0; while (x) { b++; x >>= 1; } return b; }

/* ======================================================================= */
/* primes and roots                                                        */
/* ======================================================================= */
int orc_is_prime(u64 n) {
    if (n < 2) return 0;
    static const u64 small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    for (int i = 0; i < 12; i++) {
        if (n == small[i]) return 1;
        if (n % small[i] == 0) return 0;
    }
    u64 d = n - 1; int s = 0;
    while ((d & 1) == 0) { d >>= 1; s++; }
    for (int i = 0; i < 12; i++) {
        u64 x = powmod(small[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int comp = 1;
        for (int r = 1; r < s; r++) {
            x = mulmod(x, x, n);
            if (x == n - 1) { comp = 0; break; }
        }
        if (comp) return 0;
    }
    return 1;
}

/* findPrimeFactors (include/Utils.cuh:54-69), including its loop bound
 * `i < sqrt(number)` evaluated on the shrinking cofactor. */
static int prime_factors_ref(u64 number, u64* fac) {
    int nf = 0;
    int has2 = 0;
    while (number % 2 == 0) { has2 = 1; number /= 2; }
    if (has2) fac[nf++] = 2;
    for (u64 i = 3; (double)i < sqrt((double)number); i++) {
        int hit = 0;
        while (number % i == 0) { hit = 1; number /= i; }
        if (hit) fac[nf++] = i;
    }
    if (number > 2) {
        int dup = 0;
        for (int k = 0; k < nf; k++) if (fac[k] == number) dup = 1;
        if (!dup) fac[nf++] = number;
    }
    return nf;
}

/* findPrimitiveRoot (include/Utils.cuh:71-88) */
u64 orc_primitive_root(u64 q) {
    u64 fac[64];
    u64 phi = q - 1;
    int nf = prime_factors_ref(phi, fac);
    for (u64 r = 2; r <= phi; r++) {
        int flag = 0;
        for (int k = 0; k < nf; k++)
            if (powmod(r, phi / fac[k], q) == 1) { flag = 1; break; }
        if (!flag) return r;
    }
    return (u64)-1;
}

/* findMthRootOfUnity(M = 2N, q) (include/Utils.cuh:90-101) */
u64 orc_root_2n(u64 q, u64 n) {
    u64 g = orc_primitive_root(q);
    u64 m = 2 * n;
    if ((q - 1) % m != 0) return (u64)-1;
    return powmod(g, (q - 1) / m, q);
}

int orc_root_is_primitive(u64 psi, u64 q, u64 n) {
    return psi != (u64)-1 && powmod(psi, n, q) == q - 1;
}

/* get_primes_below (include/uintarith_bfv.h:983-1016) */
size_t orc_primes_below(u64 n, u64 upper, size_t count, u64* out, int require_root) {
    u64 factor = 2 * n;
    u64 value = upper - factor;
    u64 lower = (u64)1 << (bit_count(upper) - 1);
    size_t got = 0;
    while (got < count && value > lower) {
        if (orc_is_prime(value)) {
            if (!require_root || orc_root_is_primitive(orc_root_2n(value, n), value, n))
                out[got++] = value;
        }
        value -= factor;
    }
    return got;
}

/* Chain primes of a given size: the largest primes below 2^bits that are
 * 1 mod 2N and have a primitive 2N-th root by the reference's search,
 * skipping `nskip` excluded values. */
size_t orc_primes_bits(u64 n, int bits, size_t count, const u64* skip, size_t nskip, u64* out) {
    u64 factor = 2 * n;
    u64 value = ((u64)1 << bits) + 1 - factor;
    u64 lower = (u64)1 << (bits - 1);
    size_t got = 0;
    while (got < count && value > lower) {
        int excluded = 0;
        for (size_t i = 0; i < nskip; i++) if (skip[i] == value) excluded = 1;
        if (!excluded && orc_is_prime(value) && orc_root_is_primitive(orc_root_2n(value, n), value, n))
            out[got++] = value;
        value -= factor;
    }
    return got;
}

/* ======================================================================= */
/* minimal multi-word unsigned integers (little-endian u64 words)          */
/* ======================================================================= */
#define BIGW 24
typedef struct { u64 w[BIGW]; } big;
static void big_set(big* a, u64 v) { memset(a, 0, sizeof *a); a->w[0] = v; }
static void big_mul_word(big* a, u64 m) {
    u128 carry = 0;
    for (int i = 0; i < BIGW; i++) {
        u128 t = (u128)a->w[i] * m + carry;
        a->w[i] = (u64)t;
        carry = t >> 64;
    }
}
static u64 big_mod_word(const big* a, u64 m) {
    u128 r = 0;
    for (int i = BIGW - 1; i >= 0; i--) r = ((r << 64) | a->w[i]) % m;
    return (u64)r;
}
static void big_div_word(const big* a, u64 m, big* q) {
    u128 r = 0;
    for (int i = BIGW - 1; i >= 0; i--) {
        u128 cur = (r << 64) | a->w[i];
        q->w[i] = (u64)(cur / m);
        r = cur % m;
    }
}
static int big_cmp(const big* a, const big* b) {
    for (int i = BIGW - 1; i >= 0; i--) {
        if (a->w[i] != b->w[i]) return a->w[i] > b->w[i] ? 1 : -1;
    }
    return 0;
}
static void big_add(big* a, const big* b) {
    u128 c = 0;
    for (int i = 0; i < BIGW; i++) {
        u128 t = (u128)a->w[i] + b->w[i] + c;
        a->w[i] = (u64)t;
        c = t >> 64;
    }
}
static void big_sub(big* a, const big* b) { /* a -= b, requires a >= b */
    u64 br = 0;
    for (int i = 0; i < BIGW; i++) {
        u64 x = a->w[i], y = b->w[i];
        u64 d = x - y - br;
        br = (x < y) || (x - y < br);
        a->w[i] = d;
    }
}
static double big_log2(const big* a) {
    int top = BIGW - 1;
    while (top > 0 && a->w[top] == 0) top--;
    if (top == 0 && a->w[0] == 0) return -INFINITY;
    double v = (double)a->w[top];
    if (top > 0) v += (double)a->w[top - 1] / 18446744073709551616.0;
    return log2(v) + 64.0 * top;
}

/* ======================================================================= */
/* context                                                                 */
/* ======================================================================= */
typedef struct {
    u64 q;
    u64* psi;    /* psi^brv(i) */
    u64* psis;   /* Shoup companions */
    u64* ipsi;   /* psi^-brv(i) */
    u64* ipsis;
    u64 ninv, ninvs;
    u64 root;
} prime_tab;

typedef struct {
    int nin, nout;
    u64 *in, *out;
    u64 *hatinv, *hatinvs;   /* ((B/b_i) mod b_i)^-1 */
    u64 *hat_mod_out;        /* [j][i] (B/b_i) mod o_j */
    u64 *alphaB_mod_out;     /* [a][j] a*(B mod o_j) mod o_j, a in [0, nin] */
    double* binv;            /* 1.0 / b_i */
} bconv_t;

struct orc_ctx {
    u64 n; int logn; u64 t;
    int nq, np, nr, nt, gamma, dnum, alpha;
    int nall;                 /* nq+np+nr+nt+1 */
    u64* mods;                /* prime table, order Q|P|R|T|t */
    prime_tab* tab;
    bconv_t q2r, r2q;
    /* decrypt round (BFVcontext.cuh:1030-1156) */
    int qmsb, sizeqmsb, tmsb, dec_variant;
    u64 *dec_mod_t, *dec_mod_t_s, *dec_modB_t, *dec_modB_t_s;
    double *dec_frac, *dec_fracB;
    /* QR -> R scale-round (BFVcontext.cuh:1267-1389) */
    double* sr_frac;          /* [i in Q] */
    u64* sr_c;                /* [j][nq+1] */
    /* encrypt */
    u64 negQ_mod_t, negQ_mod_t_s;
    u64 *tinv_q, *tinv_qs;
    /* hybrid key switch */
    u64 *p_mod_q, *pinv_q, *pinv_qs;            /* P mod q_i, P^-1 mod q_i */
    u64 *phatinv_p, *phatinv_ps;                /* ((P/p_k) mod p_k)^-1 */
    u64 *phat_mod_q;                            /* [i][k] (P/p_k) mod q_i */
    /* per digit lift constants: digit d covers primes [d*alpha, min((d+1)*alpha, nq)) */
    u64 *dig_hatinv, *dig_hatinvs;              /* [q index] */
    u64 *dig_hat_mod;                           /* [d][target m in 0..nq+np)][j in digit] */
    u64 *dig_Q_mod;                             /* [d][target m] */
    uint64_t gauss_cdt[64]; int gauss_bound;
    int ref_compat;            /* 1: reproduce the reference's scale-round quirk in mul_tensor */
};

static u64 brv(u64 x, int bits) {
    u64 r = 0;
    for (int i = 0; i < bits; i++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}

static void build_tab(prime_tab* pt, u64 q, u64 n, int logn) {
    pt->q = q;
    pt->root = orc_root_2n(q, n);
    u64 psi = pt->root, ipsi = invmod(psi, q);
    pt->psi = malloc(n * 8); pt->psis = malloc(n * 8);
    pt->ipsi = malloc(n * 8); pt->ipsis = malloc(n * 8);
    /* fillTablePsi128_special order (include/Utils.cuh:171-182) without the n^-1 fold */
    for (u64 i = 0; i < n; i++) {
        u64 e = brv(i, logn);
        pt->psi[i] = powmod(psi, e, q);
        pt->ipsi[i] = powmod(ipsi, e, q);
        pt->psis[i] = shoup(pt->psi[i], q);
        pt->ipsis[i] = shoup(pt->ipsi[i], q);
    }
    pt->ninv = invmod(n % q, q);
    pt->ninvs = shoup(pt->ninv, q);
}

/* BaseConverter::init (include/BasisConv_QR.cuh:53-189) */
static void build_bconv(bconv_t* b, const u64* in, int nin, const u64* out, int nout) {
    b->nin = nin; b->nout = nout;
    b->in = malloc(nin * 8); memcpy(b->in, in, nin * 8);
    b->out = malloc(nout * 8); memcpy(b->out, out, nout * 8);
    b->hatinv = malloc(nin * 8); b->hatinvs = malloc(nin * 8);
    b->binv = malloc(nin * sizeof(double));
    b->hat_mod_out = malloc((size_t)nin * nout * 8);
    b->alphaB_mod_out = malloc((size_t)(nin + 1) * nout * 8);
    for (int i = 0; i < nin; i++) {
        u64 h = 1;
        for (int k = 0; k < nin; k++) if (k != i) h = mulmod(h, in[k] % in[i], in[i]);
        b->hatinv[i] = nin > 1 ? invmod(h, in[i]) : 1;
        b->hatinvs[i] = shoup(b->hatinv[i], in[i]);
        b->binv[i] = 1.0 / (double)in[i];
    }
    for (int j = 0; j < nout; j++) {
        u64 o = out[j];
        u64 bmod = 1;
        for (int i = 0; i < nin; i++) {
            u64 h = 1;
            for (int k = 0; k < nin; k++) if (k != i) h = mulmod(h, in[k] % o, o);
            b->hat_mod_out[(size_t)j * nin + i] = h;
            bmod = mulmod(bmod, in[i] % o, o);
        }
        for (int a = 0; a <= nin; a++) b->alphaB_mod_out[(size_t)a * nout + j] = mulmod((u64)a, bmod, o);
    }
}

static void free_bconv(bconv_t* b) {
    free(b->in); free(b->out); free(b->hatinv); free(b->hatinvs); free(b->binv);
    free(b->hat_mod_out); free(b->alphaB_mod_out);
}

static void build_gauss(orc_ctx* c, double sigma, int bound) {
    orc_gaussian_cdt(sigma, bound, c->gauss_cdt);
    c->gauss_bound = bound;
}

orc_ctx* orc_create(uint32_t log_n, u64 t, const u64* q, int nq, const u64* p, int np, int dnum,
                    const u64* tk, int nt, int gamma) {
    orc_ctx* c = calloc(1, sizeof *c);
    c->n = (u64)1 << log_n; c->logn = (int)log_n; c->t = t;
    c->nq = nq; c->np = np; c->nr = nq + 1; c->nt = nt; c->gamma = gamma > 0 ? gamma : 1;
    if (dnum < 0) {  /* digit size given: alpha = -dnum */
        c->alpha = -dnum;
        c->dnum = (nq + c->alpha - 1) / c->alpha;
    } else {
        c->dnum = dnum > 0 ? dnum : 1;
        c->alpha = (nq + c->dnum - 1) / c->dnum;
    }
    c->nall = nq + np + c->nr + nt + 1;
    c->mods = malloc(c->nall * 8);
    int k = 0;
    for (int i = 0; i < nq; i++) c->mods[k++] = q[i];
    for (int i = 0; i < np; i++) c->mods[k++] = p[i];
    /* R base: r_num = q_num + 1 primes below min q (include/BFVcontext.cuh:56-58) */
    u64 qmin = q[0];
    for (int i = 1; i < nq; i++) if (q[i] < qmin) qmin = q[i];
    size_t got = orc_primes_below(c->n, qmin, c->nr, c->mods + k, 1);
    if ((int)got != c->nr) { free(c->mods); free(c); return NULL; }
    k += c->nr;
    for (int i = 0; i < nt; i++) c->mods[k++] = tk[i];
    c->mods[k++] = t;

    c->tab = calloc(c->nall, sizeof(prime_tab));
    for (int i = 0; i < c->nall; i++) build_tab(&c->tab[i], c->mods[i], c->n, c->logn);

    const u64* Q = c->mods;
    const u64* R = c->mods + nq + np;
    build_bconv(&c->q2r, Q, nq, R, c->nr);
    build_bconv(&c->r2q, R, c->nr, Q, nq);

    /* ---- decrypt constants (include/BFVcontext.cuh:1030-1156) ---- */
    u64 qmax = Q[0];
    for (int i = 1; i < nq; i++) if (Q[i] > qmax) qmax = Q[i];
    c->qmsb = bit_count(qmax);
    c->sizeqmsb = bit_count((u64)nq);
    c->tmsb = bit_count(t);
    c->dec_mod_t = calloc(nq, 8); c->dec_mod_t_s = calloc(nq, 8);
    c->dec_modB_t = calloc(nq, 8); c->dec_modB_t_s = calloc(nq, 8);
    c->dec_frac = calloc(nq, sizeof(double)); c->dec_fracB = calloc(nq, sizeof(double));
    int qmsbhf = c->qmsb >> 1;
    for (int i = 0; i < nq; i++) {
        u64 qi = Q[i];
        u64 hinv = c->q2r.hatinv[i];
        u128 big_t = (u128)t * hinv;
        u128 quo = big_t / qi;
        u64 rem = (u64)(big_t % qi);
        c->dec_mod_t[i] = (u64)(quo % t);
        c->dec_mod_t_s[i] = shoup(c->dec_mod_t[i], t);
        c->dec_frac[i] = (double)rem / (double)qi;
        if (c->qmsb + c->sizeqmsb >= 52) {
            u64 hb = (u64)(((u128)hinv << qmsbhf) % qi);
            u128 bigB = (u128)t * hb;
            u128 quoB = bigB / qi;
            u64 remB = (u64)(bigB % qi);
            c->dec_modB_t[i] = (u64)(quoB % t);
            c->dec_modB_t_s[i] = shoup(c->dec_modB_t[i], t);
            c->dec_fracB[i] = (double)remB / (double)qi;
        }
    }
    /* variant selection (include/BFVcontext.cuh:1680-1717) */
    if (c->qmsb + c->sizeqmsb < 52)
        c->dec_variant = (c->qmsb + c->tmsb + c->sizeqmsb) < 52 ? 1 /*small_lazy*/ : 0 /*small*/;
    else
        c->dec_variant = (qmsbhf + c->tmsb + c->sizeqmsb) < 52 ? 3 /*large_lazy*/ : 2 /*large*/;

    /* ---- QR -> R scale-round constants (include/BFVcontext.cuh:1267-1389) ---- */
    {
        int nqr = nq + c->nr;
        const u64* S = c->mods; /* Q then (after P) R: build a contiguous QR list */
        u64* qr = malloc(nqr * 8);
        for (int i = 0; i < nq; i++) qr[i] = S[i];
        for (int j = 0; j < c->nr; j++) qr[nq + j] = R[j];
        big tR; big_set(&tR, t);
        for (int j = 0; j < c->nr; j++) big_mul_word(&tR, R[j]);
        c->sr_frac = malloc(nq * sizeof(double));
        c->sr_c = malloc((size_t)c->nr * (nq + 1) * 8);
        big* divs = malloc(nqr * sizeof(big));
        for (int i = 0; i < nqr; i++) {
            u64 si = qr[i];
            u64 h = 1;
            for (int kk = 0; kk < nqr; kk++) if (kk != i) h = mulmod(h, qr[kk] % si, si);
            u64 shinv = invmod(h, si);
            big v = tR;
            big_mul_word(&v, shinv);
            if (i < nq) c->sr_frac[i] = (double)big_mod_word(&v, si) / (double)si;
            big_div_word(&v, si, &divs[i]);
        }
        for (int j = 0; j < c->nr; j++) {
            for (int i = 0; i < nq; i++) c->sr_c[(size_t)j * (nq + 1) + i] = big_mod_word(&divs[i], R[j]);
            c->sr_c[(size_t)j * (nq + 1) + nq] = big_mod_word(&divs[nq + j], R[j]);
        }
        free(divs); free(qr);
    }

    /* ---- encrypt constants (include/BFVcontext.cuh:881-926) ---- */
    {
        u64 qmod_t = 1;
        for (int i = 0; i < nq; i++) qmod_t = mulmod(qmod_t, Q[i] % t, t);
        c->negQ_mod_t = t - qmod_t;
        c->negQ_mod_t_s = shoup(c->negQ_mod_t, t);
        c->tinv_q = malloc(nq * 8); c->tinv_qs = malloc(nq * 8);
        for (int i = 0; i < nq; i++) {
            c->tinv_q[i] = invmod(t % Q[i], Q[i]);
            c->tinv_qs[i] = shoup(c->tinv_q[i], Q[i]);
        }
    }

    /* ---- key-switch constants ---- */
    if (np > 0) {
        const u64* P = c->mods + nq;
        c->p_mod_q = malloc(nq * 8); c->pinv_q = malloc(nq * 8); c->pinv_qs = malloc(nq * 8);
        c->phat_mod_q = malloc((size_t)nq * np * 8);
        c->phatinv_p = malloc(np * 8); c->phatinv_ps = malloc(np * 8);
        for (int i = 0; i < nq; i++) {
            u64 pm = 1;
            for (int kk = 0; kk < np; kk++) pm = mulmod(pm, P[kk] % Q[i], Q[i]);
            c->p_mod_q[i] = pm;
            c->pinv_q[i] = invmod(pm, Q[i]);
            c->pinv_qs[i] = shoup(c->pinv_q[i], Q[i]);
            for (int kk = 0; kk < np; kk++) {
                u64 h = 1;
                for (int m = 0; m < np; m++) if (m != kk) h = mulmod(h, P[m] % Q[i], Q[i]);
                c->phat_mod_q[(size_t)i * np + kk] = h;
            }
        }
        for (int kk = 0; kk < np; kk++) {
            u64 h = 1;
            for (int m = 0; m < np; m++) if (m != kk) h = mulmod(h, P[m] % P[kk], P[kk]);
            c->phatinv_p[kk] = invmod(h, P[kk]);
            c->phatinv_ps[kk] = shoup(c->phatinv_p[kk], P[kk]);
        }
        int npq = nq + np;
        c->dig_hatinv = malloc(nq * 8); c->dig_hatinvs = malloc(nq * 8);
        c->dig_hat_mod = calloc((size_t)c->dnum * npq * c->alpha, 8);
        c->dig_Q_mod = calloc((size_t)c->dnum * npq, 8);
        for (int d = 0; d < c->dnum; d++) {
            int lo = d * c->alpha, hi = lo + c->alpha; if (hi > nq) hi = nq;
            for (int j = lo; j < hi; j++) {
                u64 h = 1;
                for (int kk = lo; kk < hi; kk++) if (kk != j) h = mulmod(h, Q[kk] % Q[j], Q[j]);
                c->dig_hatinv[j] = invmod(h, Q[j]);
                c->dig_hatinvs[j] = shoup(c->dig_hatinv[j], Q[j]);
            }
            for (int m = 0; m < npq; m++) {
                u64 mod = c->mods[m];
                u64 qm = 1;
                for (int j = lo; j < hi; j++) {
                    u64 h = 1;
                    for (int kk = lo; kk < hi; kk++) if (kk != j) h = mulmod(h, Q[kk] % mod, mod);
                    c->dig_hat_mod[((size_t)d * npq + m) * c->alpha + (j - lo)] = h;
                    qm = mulmod(qm, Q[j] % mod, mod);
                }
                c->dig_Q_mod[(size_t)d * npq + m] = qm;
            }
        }
    }
    build_gauss(c, 3.2, 19);
    return c;
}

void orc_destroy(orc_ctx* c) {
    if (!c) return;
    for (int i = 0; i < c->nall; i++) {
        free(c->tab[i].psi); free(c->tab[i].psis); free(c->tab[i].ipsi); free(c->tab[i].ipsis);
    }
    free(c->tab); free(c->mods);
    free_bconv(&c->q2r); free_bconv(&c->r2q);
    free(c->dec_mod_t); free(c->dec_mod_t_s); free(c->dec_modB_t); free(c->dec_modB_t_s);
    free(c->dec_frac); free(c->dec_fracB); free(c->sr_frac); free(c->sr_c);
    free(c->tinv_q); free(c->tinv_qs);
    free(c->p_mod_q); free(c->pinv_q); free(c->pinv_qs); free(c->phat_mod_q);
    free(c->phatinv_p); free(c->phatinv_ps);
    free(c->dig_hatinv); free(c->dig_hatinvs); free(c->dig_hat_mod); free(c->dig_Q_mod);
    free(c);
}

int orc_prime_count(const orc_ctx* c) { return c->nall; }
void orc_set_ref_compat(orc_ctx* c, int on) { c->ref_compat = on; }
void orc_primes(const orc_ctx* c, u64* out) { memcpy(out, c->mods, c->nall * 8); }
u64 orc_psi(const orc_ctx* c, int i) { return c->tab[i].root; }

/* ======================================================================= */
/* NTT                                                                     */
/* ======================================================================= */
/* Forward negacyclic NTT, Cooley-Tukey with bit-reversed powers of psi
 * (include/ntt_60bit.cuh:289-300, 414-601): output index k holds
 * A(psi^(2*brv(k)+1)), fully reduced to [0, q). */
static void ntt_fwd_row(const prime_tab* pt, u64* a, u64 n) {
    u64 q = pt->q;
    for (u64 m = 1, t = n >> 1; m < n; m <<= 1, t >>= 1) {
        for (u64 i = 0; i < m; i++) {
            u64 w = pt->psi[m + i], ws = pt->psis[m + i];
            u64* x = a + 2 * i * t;
            for (u64 j = 0; j < t; j++) {
                u64 u = x[j];
                u64 v = mulshoup(x[j + t], w, ws, q);
                x[j] = addmod(u, v, q);
                x[j + t] = submod(u, v, q);
            }
        }
    }
}

/* Inverse, Gentleman-Sande with psi^-1 tables and a final n^-1
 * (include/ntt_60bit.cuh:302-313, 603-823). */
static void ntt_inv_row(const prime_tab* pt, u64* a, u64 n) {
    u64 q = pt->q;
    for (u64 m = n >> 1, t = 1; m >= 1; m >>= 1, t <<= 1) {
        for (u64 i = 0; i < m; i++) {
            u64 w = pt->ipsi[m + i], ws = pt->ipsis[m + i];
            u64* x = a + 2 * i * t;
            for (u64 j = 0; j < t; j++) {
                u64 u = x[j], v = x[j + t];
                x[j] = addmod(u, v, q);
                x[j + t] = mulshoup(submod(u, v, q), w, ws, q);
            }
        }
    }
    for (u64 j = 0; j < n; j++) a[j] = mulshoup(a[j], pt->ninv, pt->ninvs, q);
}

void orc_ntt_fwd(const orc_ctx* c, int pi, u64* rows, int nrows) {
    for (int r = 0; r < nrows; r++) ntt_fwd_row(&c->tab[pi], rows + (size_t)r * c->n, c->n);
}
void orc_ntt_inv(const orc_ctx* c, int pi, u64* rows, int nrows) {
    for (int r = 0; r < nrows; r++) ntt_inv_row(&c->tab[pi], rows + (size_t)r * c->n, c->n);
}
/* apply over consecutive limbs starting at prime index p0 */
static void ntt_fwd_limbs(const orc_ctx* c, int p0, u64* poly, int nl) {
    for (int l = 0; l < nl; l++) ntt_fwd_row(&c->tab[p0 + l], poly + (size_t)l * c->n, c->n);
}
static void ntt_inv_limbs(const orc_ctx* c, int p0, u64* poly, int nl) {
    for (int l = 0; l < nl; l++) ntt_inv_row(&c->tab[p0 + l], poly + (size_t)l * c->n, c->n);
}

/* ======================================================================= */
/* HPS base conversion (BaseConverter::bConv_HPS, BasisConv_QR.cuh:191-207;
 * bconv_mult_unroll2_kernel + base_convert_matmul_hps_unroll2_kernel,
 * poly_arithmetic.cuh:1078-1178). Output is the centred lift of x mod B. */
/* ======================================================================= */
static void bconv_apply(const bconv_t* b, u64 n, const u64* in, u64* out) {
    u64 y[64];
    for (u64 k = 0; k < n; k++) {
        double frac = 0.0;
        for (int i = 0; i < b->nin; i++) {
            y[i] = mulshoup(in[(size_t)i * n + k], b->hatinv[i], b->hatinvs[i], b->in[i]);
            frac = fma((double)y[i], b->binv[i], frac);
        }
        long long v = llround(frac);
        for (int j = 0; j < b->nout; j++) {
            u64 o = b->out[j];
            u128 acc = 0;
            for (int i = 0; i < b->nin; i++) acc += (u128)y[i] * b->hat_mod_out[(size_t)j * b->nin + i];
            u64 r = (u64)(acc % o);
            out[(size_t)j * n + k] = submod(r, b->alphaB_mod_out[(size_t)v * b->nout + j], o);
        }
    }
}
void orc_bconv_q_to_r(const orc_ctx* c, const u64* in_q, u64* out_r) { bconv_apply(&c->q2r, c->n, in_q, out_r); }
void orc_bconv_r_to_q(const orc_ctx* c, const u64* in_r, u64* out_q) { bconv_apply(&c->r2q, c->n, in_r, out_q); }

/* prime index of the l-th limb of a Q|R polynomial */
static int qr_prime(const orc_ctx* c, int l) { return l < c->nq ? l : c->nq + c->np + (l - c->nq); }

/* tensor_prod_2x2_rns_poly (poly_arithmetic.cuh:1180-1219): Karatsuba, results exact mod s */
void orc_tensor_qr(const orc_ctx* c, const u64* ct1, const u64* ct2, u64* out) {
    int nqr = c->nq + c->nr;
    size_t cnt = (size_t)nqr * c->n;
    for (int l = 0; l < nqr; l++) {
        u64 s = c->mods[qr_prime(c, l)];
        for (u64 k = 0; k < c->n; k++) {
            size_t id = (size_t)l * c->n + k;
            u64 a0 = ct1[id], a1 = ct1[id + cnt], b0 = ct2[id], b1 = ct2[id + cnt];
            u64 d0 = mulmod(a0, b0, s), d2 = mulmod(a1, b1, s);
            u64 d1 = mulmod(addmod(a0, a1, s), addmod(b0, b1, s), s);
            d1 = submod(submod(d1, d0, s), d2, s);
            out[id] = d0; out[id + cnt] = d1; out[id + 2 * cnt] = d2;
        }
    }
}

/* scaleAndRound_HPS_QR_R_kernel (poly_arithmetic.cuh:1263-1307).
 * chain_alpha != 0 reproduces the reference exactly: its
 * barrett_reduce_uint64_uint64 takes alpha by reference (uint128.cuh:156-163,
 * called at poly_arithmetic.cuh:1299), so alpha is reduced mod r_0, then that
 * mod r_1, ... and the R residues stop describing one integer once alpha
 * exceeds an R prime. chain_alpha == 0 reduces alpha mod each r_j (correct). */
static void scale_round_impl(const orc_ctx* c, const u64* in, u64* out, int chain_alpha) {
    u64 n = c->n;
    const u64* R = c->mods + c->nq + c->np;
    for (u64 k = 0; k < n; k++) {
        double nu = 0.5;
        for (int i = 0; i < c->nq; i++) nu = fma((double)in[(size_t)i * n + k], c->sr_frac[i], nu);
        u64 alpha = (u64)nu;
        for (int j = 0; j < c->nr; j++) {
            const u64* cj = c->sr_c + (size_t)j * (c->nq + 1);
            u128 acc = 0;
            for (int i = 0; i < c->nq; i++) acc += (u128)in[(size_t)i * n + k] * cj[i];
            acc += (u128)in[(size_t)(c->nq + j) * n + k] * cj[c->nq];
            u64 r = (u64)(acc % R[j]);
            u64 a;
            if (chain_alpha) { alpha %= R[j]; a = alpha; }
            else a = alpha % R[j];
            out[(size_t)j * n + k] = addmod(r, a, R[j]);
        }
    }
}
void orc_scale_round_qr_r(const orc_ctx* c, const u64* in, u64* out) { scale_round_impl(c, in, out, 0); }
void orc_scale_round_qr_r_ref(const orc_ctx* c, const u64* in, u64* out) { scale_round_impl(c, in, out, 1); }

/* hps_decrypt_scale_and_round_kernel_{small,small_lazy,large,large_lazy}
 * (poly_arithmetic.cuh:930-1075). Returns the rounded value; for inputs that
 * decrypt a zero slot with negative noise this is t itself, as in the
 * reference -- the decoder's NTT mod t absorbs it. */
int orc_decrypt_variant(const orc_ctx* c) { return c->dec_variant; }
void orc_decrypt_round(const orc_ctx* c, const u64* in, u64* out, int variant) {
    if (variant < 0) variant = c->dec_variant;
    u64 n = c->n, t = c->t;
    int hf = c->qmsb >> 1;
    u64 mask = ((u64)1 << hf) - 1;
    double tinv = 1. / (double)t;
    for (u64 k = 0; k < n; k++) {
        double ds = 0.0;
        u64 is = 0;
        for (int i = 0; i < c->nq; i++) {
            u64 x = in[(size_t)i * n + k];
            if (variant <= 1) {
                ds = fma((double)x, c->dec_frac[i], ds);
                if (variant == 0) is += mulshoup(x, c->dec_mod_t[i], c->dec_mod_t_s[i], t);
                else is += x * c->dec_mod_t[i];
            } else {
                u64 hi = x >> hf, lo = x & mask;
                ds = fma((double)lo, c->dec_frac[i], ds);
                ds = fma((double)hi, c->dec_fracB[i], ds);
                if (variant == 2) {
                    is += mulshoup(lo, c->dec_mod_t[i], c->dec_mod_t_s[i], t);
                    is += mulshoup(hi, c->dec_modB_t[i], c->dec_modB_t_s[i], t);
                } else {
                    is += lo * c->dec_mod_t[i];
                    is += hi * c->dec_modB_t[i];
                }
            }
        }
        ds += (double)is;
        u64 quot = (u64)(ds * tinv);
        ds -= (double)(t * quot);
        out[k] = (u64)llround(ds);
    }
}

/* bfv_add_timesQ_overt_kernel (poly_arithmetic.cuh:902-927): ceil(Q*m/t) per limb */
void orc_delta_m(const orc_ctx* c, const u64* m, u64* out) {
    u64 n = c->n, t = c->t;
    for (int i = 0; i < c->nq; i++) {
        u64 qi = c->mods[i];
        for (u64 k = 0; k < n; k++) {
            u64 mq = mulshoup(m[k], c->negQ_mod_t, c->negQ_mod_t_s, t);
            out[(size_t)i * n + k] = mulshoup(mq, c->tinv_q[i], c->tinv_qs[i], qi);
        }
    }
}

/* ======================================================================= */
/* hybrid key switching                                                    */
/* ======================================================================= */
/* Digit lift: restates modUpQjtoT_23_kernel's approximate CRT with the
 * single-precision quotient estimate (BasisConv.cuh:86-135), targeting the
 * primes of P and of Q outside the digit instead of the T base. One change:
 * v * (Q_d mod p) is subtracted after reducing the sum, not from the 128-bit
 * sum. The reference subtracts first; when a digit has one prime the sum is
 * x < q_j, the float estimate can round x / q_j up to 1, and the 128-bit
 * subtraction wraps, giving a residue inconsistent with the other primes. */
void orc_modup(const orc_ctx* c, const u64* d2, u64* out) {
    u64 n = c->n;
    int nq = c->nq, np = c->np, npq = nq + np;
    for (int d = 0; d < c->dnum; d++) {
        int lo = d * c->alpha, hi = lo + c->alpha; if (hi > nq) hi = nq;
        u64* o = out + (size_t)d * npq * n;
        for (u64 k = 0; k < n; k++) {
            u64 rb[64];
            float vv = 0;
            for (int j = lo; j < hi; j++) {
                u64 qj = c->mods[j];
                rb[j - lo] = mulshoup(d2[(size_t)j * n + k], c->dig_hatinv[j], c->dig_hatinvs[j], qj);
                float rr = (float)rb[j - lo];
                vv += rr / (float)qj;
            }
            int vf = (int)vv;
            for (int m = 0; m < npq; m++) {
                u64 mod = c->mods[m];
                if (m >= lo && m < hi) { o[(size_t)m * n + k] = d2[(size_t)m * n + k]; continue; }
                u128 acc = 0;
                const u64* hm = c->dig_hat_mod + ((size_t)d * npq + m) * c->alpha;
                for (int j = lo; j < hi; j++) acc += (u128)rb[j - lo] * hm[j - lo];
                u64 sub = (u64)(((u128)(u64)vf * c->dig_Q_mod[(size_t)d * npq + m]) % mod);
                u64 r = (u64)(acc % mod);
                o[(size_t)m * n + k] = r >= sub ? r - sub : r + mod - sub;
            }
        }
    }
}

/* modDownPQltoQl_23_{alpha1_,}multi_kernel (BasisConv.cuh:229-319):
 * (x_q - conv_P->q(x_P)) * P^-1 mod q, no rounding correction. */
void orc_moddown(const orc_ctx* c, const u64* in, u64* out, int npoly) {
    u64 n = c->n;
    int nq = c->nq, np = c->np, npq = nq + np;
    const u64* P = c->mods + nq;
    for (int pl = 0; pl < npoly; pl++) {
        const u64* x = in + (size_t)pl * npq * n;
        u64* y = out + (size_t)pl * nq * n;
        for (u64 k = 0; k < n; k++) {
            u64 rb[16];
            for (int kk = 0; kk < np; kk++)
                rb[kk] = mulshoup(x[(size_t)(nq + kk) * n + k], c->phatinv_p[kk], c->phatinv_ps[kk], P[kk]);
            for (int i = 0; i < nq; i++) {
                u64 qi = c->mods[i];
                u64 conv;
                if (np == 1) conv = x[(size_t)nq * n + k] % qi;
                else {
                    u128 acc = 0;
                    for (int kk = 0; kk < np; kk++) acc += (u128)rb[kk] * c->phat_mod_q[(size_t)i * np + kk];
                    conv = (u64)(acc % qi);
                }
                u64 v = qi - conv + x[(size_t)i * n + k];
                y[(size_t)i * n + k] = mulshoup(v, c->pinv_q[i], c->pinv_qs[i], qi);
            }
        }
    }
}

/* BFV modulus switch by the last prime q_l: c' = round(c / q_l) over the
 * remaining primes, in NTT form. Restates SEAL's divide_and_round_q_last_ntt
 * (the reference has only a CKKS-style flooring rescale, BFVScheme.cuh:400-502):
 * x = INTT(c_l); r_i = ([x + floor(q_l/2)]_{q_l} - floor(q_l/2)) mod q_i;
 * c'_i = (c_i - NTT_i(r_i)) * q_l^-1 mod q_i. */
void orc_mod_switch(const orc_ctx* c, const u64* ct, u64* out, int npoly) {
    u64 n = c->n;
    int nq = c->nq, nout = nq - 1;
    u64 ql = c->mods[nq - 1], half = ql >> 1;
    u64* last = malloc(n * 8);
    u64* corr = malloc(n * 8);
    for (int pl = 0; pl < npoly; pl++) {
        const u64* x = ct + (size_t)pl * nq * n;
        u64* y = out + (size_t)pl * nout * n;
        memcpy(last, x + (size_t)(nq - 1) * n, n * 8);
        ntt_inv_limbs(c, nq - 1, last, 1);
        for (int i = 0; i < nout; i++) {
            u64 qi = c->mods[i], hi = half % qi, inv = invmod(ql % qi, qi);
            for (u64 k = 0; k < n; k++) {
                u64 v = (last[k] + half) % ql % qi;
                corr[k] = v >= hi ? v - hi : v + qi - hi;
            }
            ntt_fwd_limbs(c, i, corr, 1);
            for (u64 k = 0; k < n; k++) {
                u64 d = x[(size_t)i * n + k] + qi - corr[k];
                if (d >= qi) d -= qi;
                y[(size_t)i * n + k] = mulmod(d, inv, qi);
            }
        }
    }
    free(last); free(corr);
}

/* ======================================================================= */
/* KLSS restatement (the reference's own key switch). Reference limb order  */
/* for PQ polynomials is [P | Q]; T blocks are [block][t_num].             */
/* ======================================================================= */
int orc_klss_ri_blocks(const orc_ctx* c) { return (c->np + c->nq + c->gamma - 1) / c->gamma; }
int orc_klss_qj_blocks(const orc_ctx* c) { return (c->nq + c->np - 1) / c->np; }
static u64 ref_pq_mod(const orc_ctx* c, int i) { return i < c->np ? c->mods[c->nq + i] : c->mods[i - c->np]; }
static u64 t_mod(const orc_ctx* c, int k) { return c->mods[c->nq + c->np + c->nr + k]; }

/* approximate CRT of a block of primes into every T prime (BasisConv.cuh:11-59, 86-135) */
static void klss_block_to_t(const orc_ctx* c, const u64* const* rows, const u64* blk, int nb,
                            u64 n, u64* out_blk /* nt rows */) {
    u64 hinv[16], hmod[16][16], bmod[16];
    for (int j = 0; j < nb; j++) {
        u64 h = 1;
        for (int kk = 0; kk < nb; kk++) if (kk != j) h = mulmod(h, blk[kk] % blk[j], blk[j]);
        hinv[j] = invmod(h, blk[j]);
    }
    for (int tk = 0; tk < c->nt; tk++) {
        u64 tm = t_mod(c, tk);
        u64 bm = 1;
        for (int j = 0; j < nb; j++) {
            u64 h = 1;
            for (int kk = 0; kk < nb; kk++) if (kk != j) h = mulmod(h, blk[kk] % tm, tm);
            hmod[tk][j] = h;
            bm = mulmod(bm, blk[j] % tm, tm);
        }
        bmod[tk] = bm;
    }
    for (u64 k = 0; k < n; k++) {
        u64 rb[16];
        float vv = 0;
        for (int j = 0; j < nb; j++) {
            rb[j] = mulshoup(rows[j][k], hinv[j], shoup(hinv[j], blk[j]), blk[j]);
            float rr = (float)rb[j];
            vv += rr / (float)blk[j];
        }
        int vf = (int)vv;
        for (int tk = 0; tk < c->nt; tk++) {
            u64 tm = t_mod(c, tk);
            u128 acc = 0;
            for (int j = 0; j < nb; j++) acc += (u128)rb[j] * hmod[tk][j];
            acc -= (u128)((u64)vf * bmod[tk]);
            out_blk[(size_t)tk * n + k] = (u64)(acc % tm);
        }
    }
}

/* modUpQjtoT_23 (BasisConv.cuh:86-151): d2 (nq limbs, coefficient) -> Qj blocks x T */
void orc_klss_modup_qj_to_t(const orc_ctx* c, const u64* d2, u64* out) {
    int nb = orc_klss_qj_blocks(c);
    for (int b = 0; b < nb; b++) {
        const u64* rows[16]; u64 blk[16]; int cnt = 0;
        for (int j = 0; j < c->np && b * c->np + j < c->nq; j++) {
            rows[cnt] = d2 + (size_t)(b * c->np + j) * c->n;
            blk[cnt] = c->mods[b * c->np + j];
            cnt++;
        }
        klss_block_to_t(c, rows, blk, cnt, c->n, out + (size_t)b * c->nt * c->n);
    }
}

/* modUpPQtoT_23 (BasisConv.cuh:11-79): PQ poly (reference order) -> Ri blocks x T */
void orc_klss_modup_pq_to_t(const orc_ctx* c, const u64* in, u64* out) {
    int nb = orc_klss_ri_blocks(c), npq = c->np + c->nq;
    for (int b = 0; b < nb; b++) {
        const u64* rows[16]; u64 blk[16]; int cnt = 0;
        for (int j = 0; j < c->gamma && b * c->gamma + j < npq; j++) {
            rows[cnt] = in + (size_t)(b * c->gamma + j) * c->n;
            blk[cnt] = ref_pq_mod(c, b * c->gamma + j);
            cnt++;
        }
        klss_block_to_t(c, rows, blk, cnt, c->n, out + (size_t)b * c->nt * c->n);
    }
}

/* external_product_T_kernel (ExternalProduct.cuh:11-53): in NTT form over T.
 * digits_t: [Qj block][T]; key_t: [ax|bx][digit][Ri block][T]; out: [2][Ri block][T] */
void orc_klss_external_product(const orc_ctx* c, const u64* digits_t, const u64* key_t, u64* out) {
    int nri = orc_klss_ri_blocks(c), nqj = orc_klss_qj_blocks(c);
    int dnum = c->nq / c->np;
    u64 n = c->n;
    size_t half = (size_t)dnum * nri * c->nt * n;
    for (int h = 0; h < 2; h++)
        for (int b = 0; b < nri; b++)
            for (int tk = 0; tk < c->nt; tk++) {
                u64 tm = t_mod(c, tk);
                for (u64 k = 0; k < n; k++) {
                    u128 acc = 0;
                    for (int i = 0; i < nqj; i++) {
                        u64 ra = digits_t[((size_t)i * c->nt + tk) * n + k];
                        u64 rb = key_t[h * half + (((size_t)i * nri + b) * c->nt + tk) * n + k];
                        acc += (u128)ra * rb;
                    }
                    out[(((size_t)h * nri + b) * c->nt + tk) * n + k] = (u64)(acc % tm);
                }
            }
}

/* modUpTtoPQl_23_kernel (BasisConv.cuh:159-213): centred exact T -> each PQ prime */
void orc_klss_modup_t_to_pq(const orc_ctx* c, const u64* in, u64* out, int npoly) {
    int nri = orc_klss_ri_blocks(c), npq = c->np + c->nq, nt = c->nt;
    u64 n = c->n;
    u64 thinv[16], thinvs[16];
    big halfT; big_set(&halfT, 1);
    for (int k = 0; k < nt; k++) big_mul_word(&halfT, t_mod(c, k));
    { big h2; big_div_word(&halfT, 2, &h2); halfT = h2; }
    for (int i = 0; i < nt; i++) {
        u64 ti = t_mod(c, i), h = 1;
        for (int k = 0; k < nt; k++) if (k != i) h = mulmod(h, t_mod(c, k) % ti, ti);
        thinv[i] = invmod(h, ti); thinvs[i] = shoup(thinv[i], ti);
    }
    for (int pl = 0; pl < npoly; pl++)
        for (int b = 0; b < nri; b++)
            for (u64 k = 0; k < n; k++) {
                u64 rb[16]; float vv = 0;
                for (int i = 0; i < nt; i++) {
                    u64 ti = t_mod(c, i);
                    u64 ra = in[(((size_t)pl * nri + b) * nt + i) * n + k] + big_mod_word(&halfT, ti);
                    rb[i] = mulshoup(ra, thinv[i], thinvs[i], ti);
                    float rr = (float)rb[i];
                    vv += rr / (float)ti;
                }
                int vf = (int)vv;
                for (int j = 0; j < c->gamma && b * c->gamma + j < npq; j++) {
                    int ip = b * c->gamma + j;
                    u64 ri = ref_pq_mod(c, ip);
                    u128 acc = 0;
                    u64 tmod = 1;
                    for (int i = 0; i < nt; i++) {
                        u64 h = 1;
                        for (int kk = 0; kk < nt; kk++) if (kk != i) h = mulmod(h, t_mod(c, kk) % ri, ri);
                        acc += (u128)rb[i] * h;
                        tmod = mulmod(tmod, t_mod(c, i) % ri, ri);
                    }
                    acc -= (u128)((u64)vf * tmod);
                    u64 r = (u64)(acc % ri);
                    r = r + ri - big_mod_word(&halfT, ri);
                    if (r >= ri) r -= ri;
                    /* output limb index in [P|Q] order within the poly's Ri*T-sized slot */
                    out[((size_t)pl * nri * nt + ip) * n + k] = r;
                }
            }
}

/* modDownPQltoQl_23 on reference-ordered input ([P|Q] per poly, poly stride Ri*T limbs) */
void orc_klss_moddown(const orc_ctx* c, const u64* in, u64* out, int npoly) {
    int nri = orc_klss_ri_blocks(c), nq = c->nq, np = c->np, npq = nq + np;
    u64 n = c->n;
    u64* tmp = malloc((size_t)npq * n * 8);
    for (int pl = 0; pl < npoly; pl++) {
        const u64* x = in + (size_t)pl * nri * c->nt * n;
        for (int i = 0; i < nq; i++) memcpy(tmp + (size_t)i * n, x + (size_t)(np + i) * n, n * 8);
        for (int k = 0; k < np; k++) memcpy(tmp + (size_t)(nq + k) * n, x + (size_t)k * n, n * 8);
        orc_moddown(c, tmp, out + (size_t)pl * nq * n, 1);
    }
    free(tmp);
}

/* ======================================================================= */
/* Salsa20 / XSalsa20                                                      */
/* ======================================================================= */
static inline uint32_t rotl(uint32_t u, int c) { return (u << c) | (u >> (32 - c)); }
static inline uint32_t ld32(const uint8_t* x) {
    return (uint32_t)x[0] | ((uint32_t)x[1] << 8) | ((uint32_t)x[2] << 16) | ((uint32_t)x[3] << 24);
}
static inline void st32(uint8_t* x, uint32_t v) { x[0] = v; x[1] = v >> 8; x[2] = v >> 16; x[3] = v >> 24; }

/* 20-round double-round sequence (RNG_impl.cuh:117-150, the Salsa20 core) */
static void salsa_rounds(uint32_t x[16]) {
    for (int i = 20; i > 0; i -= 2) {
        x[4] ^= rotl(x[0] + x[12], 7);   x[8] ^= rotl(x[4] + x[0], 9);
        x[12] ^= rotl(x[8] + x[4], 13);  x[0] ^= rotl(x[12] + x[8], 18);
        x[9] ^= rotl(x[5] + x[1], 7);    x[13] ^= rotl(x[9] + x[5], 9);
        x[1] ^= rotl(x[13] + x[9], 13);  x[5] ^= rotl(x[1] + x[13], 18);
        x[14] ^= rotl(x[10] + x[6], 7);  x[2] ^= rotl(x[14] + x[10], 9);
        x[6] ^= rotl(x[2] + x[14], 13);  x[10] ^= rotl(x[6] + x[2], 18);
        x[3] ^= rotl(x[15] + x[11], 7);  x[7] ^= rotl(x[3] + x[15], 9);
        x[11] ^= rotl(x[7] + x[3], 13);  x[15] ^= rotl(x[11] + x[7], 18);
        x[1] ^= rotl(x[0] + x[3], 7);    x[2] ^= rotl(x[1] + x[0], 9);
        x[3] ^= rotl(x[2] + x[1], 13);   x[0] ^= rotl(x[3] + x[2], 18);
        x[6] ^= rotl(x[5] + x[4], 7);    x[7] ^= rotl(x[6] + x[5], 9);
        x[4] ^= rotl(x[7] + x[6], 13);   x[5] ^= rotl(x[4] + x[7], 18);
        x[11] ^= rotl(x[10] + x[9], 7);  x[8] ^= rotl(x[11] + x[10], 9);
        x[9] ^= rotl(x[8] + x[11], 13);  x[10] ^= rotl(x[9] + x[8], 18);
        x[12] ^= rotl(x[15] + x[14], 7); x[13] ^= rotl(x[12] + x[15], 9);
        x[14] ^= rotl(x[13] + x[12], 13); x[15] ^= rotl(x[14] + x[13], 18);
    }
}

static const uint8_t SIGMA[16] = {'e','x','p','a','n','d',' ','3','2','-','b','y','t','e',' ','k'};

void orc_hsalsa20(const uint8_t key[32], const uint8_t nonce16[16], uint8_t out[32]) {
    uint32_t x[16];
    x[0] = ld32(SIGMA); x[5] = ld32(SIGMA + 4); x[10] = ld32(SIGMA + 8); x[15] = ld32(SIGMA + 12);
    for (int i = 0; i < 4; i++) { x[1 + i] = ld32(key + 4 * i); x[11 + i] = ld32(key + 16 + 4 * i); }
    for (int i = 0; i < 4; i++) x[6 + i] = ld32(nonce16 + 4 * i);
    salsa_rounds(x);
    st32(out + 0, x[0]); st32(out + 4, x[5]); st32(out + 8, x[10]); st32(out + 12, x[15]);
    st32(out + 16, x[6]); st32(out + 20, x[7]); st32(out + 24, x[8]); st32(out + 28, x[9]);
}

static void salsa20_block(const uint8_t sigma[16], const uint8_t key[32], uint32_t n0, uint32_t n1,
                          uint64_t ctr, uint8_t out[64]) {
    uint32_t j[16], x[16];
    j[0] = ld32(sigma); j[5] = ld32(sigma + 4); j[10] = ld32(sigma + 8); j[15] = ld32(sigma + 12);
    for (int i = 0; i < 4; i++) { j[1 + i] = ld32(key + 4 * i); j[11 + i] = ld32(key + 16 + 4 * i); }
    j[6] = n0; j[7] = n1; j[8] = (uint32_t)ctr; j[9] = (uint32_t)(ctr >> 32);
    memcpy(x, j, sizeof x);
    salsa_rounds(x);
    for (int i = 0; i < 16; i++) st32(out + 4 * i, x[i] + j[i]);
}

void orc_xsalsa20_stream(const uint8_t key[32], const uint8_t nonce[24], uint64_t block0,
                         uint8_t* out, size_t nbytes) {
    uint8_t sub[32], blk[64];
    orc_hsalsa20(key, nonce, sub);
    uint32_t n0 = ld32(nonce + 16), n1 = ld32(nonce + 20);
    for (size_t off = 0; off < nbytes; off += 64) {
        salsa20_block(SIGMA, sub, n0, n1, block0 + off / 64, blk);
        size_t m = nbytes - off < 64 ? nbytes - off : 64;
        memcpy(out + off, blk, m);
    }
}

/* The reference's VecCrypt (RNG_impl.cuh:70-176): sigma constant never
 * written (all zero), nonce truncated to 32 bits, no HSalsa20, tail bytes
 * of a partial block left zero. */
void orc_salsa20_compat_stream(const uint8_t key[32], uint64_t nonce, uint8_t* out, size_t nbytes) {
    static const uint8_t zero_sigma[16] = {0};
    uint8_t blk[64];
    memset(out, 0, nbytes);
    for (size_t b = 0; b < nbytes / 64; b++) {
        salsa20_block(zero_sigma, key, (uint32_t)nonce, 0, b, blk);
        memcpy(out + b * 64, blk, 64);
    }
}

/* ======================================================================= */
/* samplers                                                                */
/* ======================================================================= */
/* Discrete Gaussian on [-B, B] by cumulative table: table[k] = floor(2^64 * P(X <= -B + k)),
 * k = 0..2B-1; a 64-bit uniform u maps to -B + #{k : u >= table[k]}. */
void orc_gaussian_cdt(double sigma, int bound, uint64_t* table) {
    long double w[128], z = 0;
    for (int x = -bound; x <= bound; x++) {
        w[x + bound] = expl(-(long double)x * x / (2.0L * (long double)sigma * sigma));
        z += w[x + bound];
    }
    long double acc = 0;
    for (int k = 0; k < 2 * bound; k++) {
        acc += w[k];
        long double v = acc / z * 18446744073709551616.0L;
        table[k] = v >= 18446744073709551615.0L ? UINT64_MAX : (uint64_t)v;
    }
    table[2 * bound] = UINT64_MAX;
}

/* nonce = [domain | sub | 0 | 0 | id_lo | id_hi] (little-endian words): the
 * HSalsa20 subkey depends on (key, domain, sub) only; the item id is the
 * Salsa20 nonce, so every item of a batch draws an independent stream. */
static void make_nonce(uint32_t domain, uint64_t id, uint32_t sub, uint8_t nonce[24]) {
    memset(nonce, 0, 24);
    st32(nonce, domain);
    st32(nonce + 4, sub);
    st32(nonce + 16, (uint32_t)id);
    st32(nonce + 20, (uint32_t)(id >> 32));
}

static uint8_t* stream_bytes(const uint8_t key[32], uint32_t domain, uint64_t id, uint32_t sub, size_t nbytes) {
    uint8_t nonce[24];
    make_nonce(domain, id, sub, nonce);
    uint8_t* buf = malloc(nbytes + 64);
    orc_xsalsa20_stream(key, nonce, 0, buf, nbytes);
    return buf;
}
static inline u64 ld64(const uint8_t* p) { return (u64)ld32(p) | ((u64)ld32(p + 4) << 32); }

/* uniform mod q from 16 bytes: floor(u128 * q / 2^128) */
void orc_sample_uniform(const orc_ctx* c, const uint8_t key[32], uint32_t domain, uint64_t id,
                        uint32_t sub, const int* prime_idx, int nl, u64* out) {
    u64 n = c->n;
    uint8_t* b = stream_bytes(key, domain, id, sub, (size_t)nl * n * 16);
    for (int l = 0; l < nl; l++) {
        u64 q = c->mods[prime_idx[l]];
        for (u64 k = 0; k < n; k++) {
            const uint8_t* p = b + ((size_t)l * n + k) * 16;
            u64 lo = ld64(p), hi = ld64(p + 8);
            u128 a1 = ((u128)lo * q) >> 64;
            out[(size_t)l * n + k] = (u64)((((u128)hi * q) + a1) >> 64);
        }
    }
    free(b);
}

/* ternary uniform {0, 1, -1} from 4 bytes: (u32 * 3) >> 32 */
void orc_sample_ternary(const orc_ctx* c, const uint8_t key[32], uint32_t domain, uint64_t id,
                        uint32_t sub, int64_t* out) {
    uint8_t* b = stream_bytes(key, domain, id, sub, c->n * 4);
    for (u64 k = 0; k < c->n; k++) {
        uint32_t v = (uint32_t)(((u64)ld32(b + 4 * k) * 3) >> 32);
        out[k] = v == 0 ? 0 : (v == 1 ? 1 : -1);
    }
    free(b);
}

void orc_sample_gaussian(const orc_ctx* c, const uint8_t key[32], uint32_t domain, uint64_t id,
                         uint32_t sub, int64_t* out) {
    uint8_t* b = stream_bytes(key, domain, id, sub, c->n * 8);
    int B = c->gauss_bound;
    for (u64 k = 0; k < c->n; k++) {
        u64 u = ld64(b + 8 * k);
        int x = -B;
        for (int j = 0; j < 2 * B; j++) x += (u >= c->gauss_cdt[j]);
        out[k] = x;
    }
    free(b);
}

/* convert_HWT (Sampler_impl.cuh:68-87): h positions from u32 & (N-1), sign from a byte;
 * colliding positions resolve to the later draw. */
void orc_sample_hwt(const orc_ctx* c, const uint8_t key[32], uint32_t domain, uint64_t id,
                    uint32_t sub, int h, int64_t* out) {
    uint8_t* b = stream_bytes(key, domain, id, sub, (size_t)h * 5);
    memset(out, 0, c->n * sizeof(int64_t));
    for (int i = 0; i < h; i++) {
        uint32_t pos = ld32(b + 4 * i) & (uint32_t)(c->n - 1);
        float d = (float)b[4 * h + i];
        d /= (256.0f / 2);
        out[pos] = d >= 1 ? 1 : -1;
    }
    free(b);
}

/* ======================================================================= */
/* scheme                                                                  */
/* ======================================================================= */
enum { DOM_SK = 1, DOM_PK_A = 2, DOM_PK_E = 3, DOM_RLK_A = 4, DOM_RLK_E = 5,
       DOM_ENC_V = 6, DOM_ENC_E0 = 7, DOM_ENC_E1 = 8, DOM_GK_A = 9, DOM_GK_E = 10, DOM_GAL_A = 11, DOM_GAL_E = 12 };

static void small_to_rns(const orc_ctx* c, const int64_t* s, int p0, int nl, u64* out) {
    for (int l = 0; l < nl; l++) {
        u64 q = c->mods[p0 + l];
        for (u64 k = 0; k < c->n; k++) out[(size_t)l * c->n + k] = s[k] < 0 ? q - (u64)(-s[k]) : (u64)s[k];
    }
}

void orc_keygen_secret(const orc_ctx* c, const uint8_t key[32], int kind, int h, u64* sk) {
    int64_t* s = malloc(c->n * sizeof(int64_t));
    if (kind == 1) orc_sample_hwt(c, key, DOM_SK, 0, 0, h, s);
    else orc_sample_ternary(c, key, DOM_SK, 0, 0, s);
    int npq = c->nq + c->np;
    small_to_rns(c, s, 0, npq, sk);
    ntt_fwd_limbs(c, 0, sk, npq);
    free(s);
}

/* addEncKey (BFVScheme.cuh:57-85): a uniform in NTT form, b = e - a*s */
void orc_keygen_public(const orc_ctx* c, const uint8_t key[32], const u64* sk, u64* pk) {
    u64 n = c->n;
    int nq = c->nq;
    int idx[64] = {0};
    for (int i = 0; i < nq; i++) idx[i] = i;
    u64* a = pk;
    u64* b = pk + (size_t)nq * n;
    orc_sample_uniform(c, key, DOM_PK_A, 0, 0, idx, nq, a);
    int64_t* e = malloc(n * sizeof(int64_t));
    orc_sample_gaussian(c, key, DOM_PK_E, 0, 0, e);
    small_to_rns(c, e, 0, nq, b);
    ntt_fwd_limbs(c, 0, b, nq);
    for (int l = 0; l < nq; l++) {
        u64 q = c->mods[l];
        for (u64 k = 0; k < n; k++) {
            size_t id = (size_t)l * n + k;
            b[id] = submod(b[id], mulmod(a[id], sk[id], q), q);
        }
    }
    free(e);
}

/* addMultKey_23's key material (KeySwitch_23.cuh:21-56), kept over PQ:
 * digit d: a_d uniform, b_d = -a_d*s + e_d + P*s^2 on the digit's primes. */
void orc_keygen_relin(const orc_ctx* c, const uint8_t key[32], const u64* sk, u64* rlk) {
    u64 n = c->n;
    int nq = c->nq, np = c->np, npq = nq + np;
    int idx[128];
    for (int i = 0; i < npq; i++) idx[i] = i;
    int64_t* e = malloc(n * sizeof(int64_t));
    for (int d = 0; d < c->dnum; d++) {
        int lo = d * c->alpha, hi = lo + c->alpha; if (hi > nq) hi = nq;
        u64* a = rlk + (size_t)d * 2 * npq * n;
        u64* b = a + (size_t)npq * n;
        orc_sample_uniform(c, key, DOM_RLK_A, 0, (uint32_t)d, idx, npq, a);
        orc_sample_gaussian(c, key, DOM_RLK_E, 0, (uint32_t)d, e);
        small_to_rns(c, e, 0, npq, b);
        ntt_fwd_limbs(c, 0, b, npq);
        for (int l = 0; l < npq; l++) {
            u64 q = c->mods[l];
            for (u64 k = 0; k < n; k++) {
                size_t id = (size_t)l * n + k;
                u64 v = submod(b[id], mulmod(a[id], sk[id], q), q);
                if (l >= lo && l < hi) {
                    u64 s2 = mulmod(sk[id], sk[id], q);
                    v = addmod(v, mulmod(s2, c->p_mod_q[l], q), q);
                }
                b[id] = v;
            }
        }
    }
    free(e);
}

void orc_encode(const orc_ctx* c, const u64* slots, u64* m) {
    memcpy(m, slots, c->n * 8);
    ntt_inv_row(&c->tab[c->nall - 1], m, c->n);
}
void orc_decode(const orc_ctx* c, const u64* m, u64* slots) {
    /* the decrypt round may leave the value t itself; the NTT works modulo t */
    for (u64 k = 0; k < c->n; k++) slots[k] = m[k] % c->t;
    ntt_fwd_row(&c->tab[c->nall - 1], slots, c->n);
}

/* encryptZero + encryptMsg (BFVScheme.cuh:87-146) with ternary v and Gaussian e0, e1 */
void orc_encrypt(const orc_ctx* c, const uint8_t key[32], uint64_t id, const u64* pk,
                 const u64* m, u64* ct) {
    u64 n = c->n;
    int nq = c->nq;
    int64_t* s = malloc(n * sizeof(int64_t));
    u64* v = malloc((size_t)nq * n * 8);
    u64* e = malloc((size_t)nq * n * 8);
    u64* dm = malloc((size_t)nq * n * 8);
    orc_sample_ternary(c, key, DOM_ENC_V, id, 0, s);
    small_to_rns(c, s, 0, nq, v);
    ntt_fwd_limbs(c, 0, v, nq);
    u64* a = ct;
    u64* b = ct + (size_t)nq * n;
    const u64* pa = pk;
    const u64* pb = pk + (size_t)nq * n;
    orc_sample_gaussian(c, key, DOM_ENC_E0, id, 0, s);
    small_to_rns(c, s, 0, nq, e);
    ntt_fwd_limbs(c, 0, e, nq);
    for (size_t i = 0; i < (size_t)nq * n; i++) {
        u64 q = c->mods[i / n];
        a[i] = addmod(mulmod(v[i], pa[i], q), e[i], q);
    }
    orc_sample_gaussian(c, key, DOM_ENC_E1, id, 0, s);
    small_to_rns(c, s, 0, nq, e);
    ntt_fwd_limbs(c, 0, e, nq);
    orc_delta_m(c, m, dm);
    ntt_fwd_limbs(c, 0, dm, nq);
    for (size_t i = 0; i < (size_t)nq * n; i++) {
        u64 q = c->mods[i / n];
        b[i] = addmod(addmod(mulmod(v[i], pb[i], q), e[i], q), dm[i], q);
    }
    free(s); free(v); free(e); free(dm);
}

/* decryptMsg (BFVScheme.cuh:148-166): round(t/Q * [b + a*s]) */
void orc_decrypt(const orc_ctx* c, const u64* sk, const u64* ct, u64* m) {
    u64 n = c->n;
    int nq = c->nq;
    u64* x = malloc((size_t)nq * n * 8);
    for (size_t i = 0; i < (size_t)nq * n; i++) {
        u64 q = c->mods[i / n];
        x[i] = addmod(mulmod(ct[i], sk[i], q), ct[(size_t)nq * n + i], q);
    }
    ntt_inv_limbs(c, 0, x, nq);
    orc_decrypt_round(c, x, m, -1);
    free(x);
}

void orc_add(const orc_ctx* c, const u64* x, const u64* y, u64* out, int npoly) {
    u64 n = c->n;
    for (int p = 0; p < npoly; p++)
        for (size_t i = 0; i < (size_t)c->nq * n; i++) {
            size_t id = (size_t)p * c->nq * n + i;
            out[id] = addmod(x[id], y[id], c->mods[i / n]);
        }
}

/* multConstAndEqual with an encode_ntt plaintext: both halves times pt (NTT form over Q) */
void orc_mul_plain(const orc_ctx* c, const u64* ct, const u64* pt, u64* out) {
    u64 n = c->n;
    for (int p = 0; p < 2; p++)
        for (size_t i = 0; i < (size_t)c->nq * n; i++) {
            size_t id = (size_t)p * c->nq * n + i;
            out[id] = mulmod(ct[id], pt[i], c->mods[i / n]);
        }
}

/* compute_t_QInv_c0c1c2 without the secret-key shortcut (KeySwitch_23.cuh:703-926):
 * INTT over Q, Q->R, NTT over Q|R, tensor, INTT, scale-round to R, R->Q, NTT over Q. */
void orc_mul_tensor(const orc_ctx* c, const u64* ct1, const u64* ct2, u64* d) {
    u64 n = c->n;
    int nq = c->nq, nr = c->nr, nqr = nq + nr;
    size_t lq = (size_t)nq * n, lqr = (size_t)nqr * n;
    u64* x1 = malloc(2 * lqr * 8);
    u64* x2 = malloc(2 * lqr * 8);
    u64* tp = malloc(3 * lqr * 8);
    u64* rr = malloc((size_t)nr * n * 8);
    const u64* src[4] = {ct1, ct1 + lq, ct2, ct2 + lq};
    u64* dst[4] = {x1, x1 + lqr, x2, x2 + lqr};
    for (int p = 0; p < 4; p++) {
        memcpy(dst[p], src[p], lq * 8);
        ntt_inv_limbs(c, 0, dst[p], nq);
        orc_bconv_q_to_r(c, dst[p], dst[p] + lq);
        ntt_fwd_limbs(c, 0, dst[p], nq);
        ntt_fwd_limbs(c, nq + c->np, dst[p] + lq, nr);
    }
    orc_tensor_qr(c, x1, x2, tp);
    /* tensor order [a1a2 | a1b2+b1a2 | b1b2] since ct = [a | b] */
    for (int k = 0; k < 3; k++) {
        u64* y = tp + (size_t)k * lqr;
        ntt_inv_limbs(c, 0, y, nq);
        ntt_inv_limbs(c, nq + c->np, y + lq, nr);
        scale_round_impl(c, y, rr, c->ref_compat);
        orc_bconv_r_to_q(c, rr, d + (size_t)k * lq);
        ntt_fwd_limbs(c, 0, d + (size_t)k * lq, nq);
    }
    free(x1); free(x2); free(tp); free(rr);
}

/* relinearize [a1a2 | cross | b1b2] (NTT form) into [a | b] (NTT form):
 * digit lift of a1a2, inner product with the relin key over PQ, mod down. */
void orc_relinearize(const orc_ctx* c, const u64* d, const u64* rlk, u64* ct) {
    u64 n = c->n;
    int nq = c->nq, np = c->np, npq = nq + np;
    size_t lq = (size_t)nq * n, lpq = (size_t)npq * n;
    u64* d2 = malloc(lq * 8);
    u64* up = malloc((size_t)c->dnum * lpq * 8);
    u64* acc = calloc(2 * lpq, 8);
    u64* dn = malloc(2 * lq * 8);
    memcpy(d2, d, lq * 8);
    ntt_inv_limbs(c, 0, d2, nq);
    orc_modup(c, d2, up);
    for (int dg = 0; dg < c->dnum; dg++) {
        u64* u = up + (size_t)dg * lpq;
        ntt_fwd_limbs(c, 0, u, npq);
        const u64* ka = rlk + (size_t)dg * 2 * lpq;
        const u64* kb = ka + lpq;
        for (size_t i = 0; i < lpq; i++) {
            u64 q = c->mods[i / n];
            acc[i] = addmod(acc[i], mulmod(u[i], ka[i], q), q);
            acc[lpq + i] = addmod(acc[lpq + i], mulmod(u[i], kb[i], q), q);
        }
    }
    ntt_inv_limbs(c, 0, acc, npq);
    ntt_inv_limbs(c, 0, acc + lpq, npq);
    orc_moddown(c, acc, dn, 2);
    ntt_fwd_limbs(c, 0, dn, nq);
    ntt_fwd_limbs(c, 0, dn + lq, nq);
    for (size_t i = 0; i < lq; i++) {
        u64 q = c->mods[i / n];
        ct[i] = addmod(d[lq + i], dn[i], q);              /* a = cross + a' */
        ct[lq + i] = addmod(d[2 * lq + i], dn[lq + i], q); /* b = b1b2 + b' */
    }
    free(d2); free(up); free(acc); free(dn);
}

/* ---- key switching over a gadget decomposition of base 2^w --------------
 * d2 = sum_i [d2]_{q_i} * g_i (mod Q) with g_i = Q/q_i * [(Q/q_i)^-1]_{q_i};
 * each residue [d2]_{q_i} < 2^60 is cut into J = ceil(60 / w) pieces of w bits,
 * z_{ij} < 2^w, the same small integer in every prime. Key component (i, j):
 * a uniform, b = e - a*s + 2^{wj} * P * [l == i] * s^2 mod p_l over Q|P. The
 * product sum_{ij} NTT(z_ij) * key_ij is reduced by P (mod-down) as in the
 * hybrid method. No counterpart in the reference. */
int orc_gadget_pieces(int w) { return (60 + w - 1) / w; }

void orc_keygen_relin_gadget(const orc_ctx* c, const uint8_t key[32], const u64* sk, int w, u64* gk) {
    u64 n = c->n;
    int nq = c->nq, np = c->np, npq = nq + np, J = orc_gadget_pieces(w);
    int idx[128];
    for (int i = 0; i < npq; i++) idx[i] = i;
    int64_t* e = malloc(n * sizeof(int64_t));
    for (int i = 0; i < nq; i++)
        for (int j = 0; j < J; j++) {
            uint32_t sub = (uint32_t)(i * J + j);
            u64* a = gk + (size_t)sub * 2 * npq * n;
            u64* b = a + (size_t)npq * n;
            orc_sample_uniform(c, key, DOM_GK_A, 0, sub, idx, npq, a);
            orc_sample_gaussian(c, key, DOM_GK_E, 0, sub, e);
            small_to_rns(c, e, 0, npq, b);
            ntt_fwd_limbs(c, 0, b, npq);
            for (int l = 0; l < npq; l++) {
                u64 q = c->mods[l];
                u64 g = l == i ? mulmod(c->p_mod_q[l], powmod(2, (u64)w * j, q), q) : 0;
                for (u64 k = 0; k < n; k++) {
                    size_t id = (size_t)l * n + k;
                    u64 v = submod(b[id], mulmod(a[id], sk[id], q), q);
                    if (g) v = addmod(v, mulmod(mulmod(sk[id], sk[id], q), g, q), q);
                    b[id] = v;
                }
            }
        }
    free(e);
}

void orc_relinearize_gadget(const orc_ctx* c, const u64* d, const u64* gk, int w, u64* ct) {
    u64 n = c->n;
    int nq = c->nq, np = c->np, npq = nq + np, J = orc_gadget_pieces(w);
    size_t lq = (size_t)nq * n, lpq = (size_t)npq * n;
    u64 mask = (w >= 64) ? ~0ULL : (((u64)1 << w) - 1);
    u64* d2 = malloc(lq * 8);
    u64* z = malloc(lpq * 8);
    u64* acc = calloc(2 * lpq, 8);
    u64* dn = malloc(2 * lq * 8);
    memcpy(d2, d, lq * 8);
    ntt_inv_limbs(c, 0, d2, nq);
    for (int i = 0; i < nq; i++)
        for (int j = 0; j < J; j++) {
            for (int m = 0; m < npq; m++)
                for (u64 k = 0; k < n; k++) z[(size_t)m * n + k] = (d2[(size_t)i * n + k] >> (w * j)) & mask;
            ntt_fwd_limbs(c, 0, z, npq);
            const u64* ka = gk + (size_t)(i * J + j) * 2 * lpq;
            const u64* kb = ka + lpq;
            for (size_t x = 0; x < lpq; x++) {
                u64 q = c->mods[x / n];
                acc[x] = addmod(acc[x], mulmod(z[x], ka[x], q), q);
                acc[lpq + x] = addmod(acc[lpq + x], mulmod(z[x], kb[x], q), q);
            }
        }
    ntt_inv_limbs(c, 0, acc, npq);
    ntt_inv_limbs(c, 0, acc + lpq, npq);
    orc_moddown(c, acc, dn, 2);
    ntt_fwd_limbs(c, 0, dn, nq);
    ntt_fwd_limbs(c, 0, dn + lq, nq);
    for (size_t x = 0; x < lq; x++) {
        u64 q = c->mods[x / n];
        ct[x] = addmod(d[lq + x], dn[x], q);
        ct[lq + x] = addmod(d[2 * lq + x], dn[lq + x], q);
    }
    free(d2); free(z); free(acc); free(dn);
}

/* ---- Galois automorphisms X -> X^g (g odd mod 2N) -------------------------
 * In NTT form an automorphism permutes the evaluation points: index i holds
 * A(psi^e_i), e_i = 2 brv(i) + 1, and (A o X^g)(psi^e) = A(psi^(e g)), so
 * out[i] = in[j] with e_j = e_i * g mod 2N, the same for every prime.
 * Rotations use g = 5^r mod 2N (the reference's rotGroups, BFVcontext.cuh:788-799),
 * conjugation g = 2N - 1. */
static u64 brv_bits(u64 x, int bits) {
    u64 r = 0;
    for (int b = 0; b < bits; b++) { r = (r << 1) | (x & 1); x >>= 1; }
    return r;
}
void orc_galois_ntt(const orc_ctx* c, u64 g, const u64* in, u64* out, int nlimbs) {
    u64 n = c->n, m = 2 * n;
    int logn = (int)c->logn;
    u64* perm = malloc(n * 8);
    for (u64 i = 0; i < n; i++) {
        u64 e = (2 * brv_bits(i, logn) + 1) * (g % m) % m;
        perm[i] = brv_bits((e - 1) / 2, logn);
    }
    for (int l = 0; l < nlimbs; l++)
        for (u64 i = 0; i < n; i++) out[(size_t)l * n + i] = in[(size_t)l * n + perm[i]];
    free(perm);
}

/* key switching key from s(X^g) to s: digit d: a uniform, b = e - a s + P * [l in digit d] * s(X^g),
 * layout as the relinearisation key; randomness keyed by (DOM_GAL_*, id = g, sub = d) */
void orc_keygen_galois(const orc_ctx* c, const uint8_t key[32], const u64* sk, u64 g, u64* gk) {
    u64 n = c->n;
    int nq = c->nq, np = c->np, npq = nq + np;
    int idx[128];
    for (int i = 0; i < npq; i++) idx[i] = i;
    u64* sg = malloc((size_t)npq * n * 8);
    orc_galois_ntt(c, g, sk, sg, npq);
    int64_t* e = malloc(n * sizeof(int64_t));
    for (int d = 0; d < c->dnum; d++) {
        int lo = d * c->alpha, hi = lo + c->alpha; if (hi > nq) hi = nq;
        u64* a = gk + (size_t)d * 2 * npq * n;
        u64* b = a + (size_t)npq * n;
        orc_sample_uniform(c, key, DOM_GAL_A, g, (uint32_t)d, idx, npq, a);
        orc_sample_gaussian(c, key, DOM_GAL_E, g, (uint32_t)d, e);
        small_to_rns(c, e, 0, npq, b);
        ntt_fwd_limbs(c, 0, b, npq);
        for (int l = 0; l < npq; l++) {
            u64 q = c->mods[l];
            for (u64 k = 0; k < n; k++) {
                size_t id = (size_t)l * n + k;
                u64 v = submod(b[id], mulmod(a[id], sk[id], q), q);
                if (l >= lo && l < hi) v = addmod(v, mulmod(sg[id], c->p_mod_q[l], q), q);
                b[id] = v;
            }
        }
    }
    free(e); free(sg);
}

/* ct (2 x nq, NTT) -> automorphism then key switch back to s: key switch of
 * [g(a) | 0 | g(b)] as a tensor (leftRotateAndEqual_23, KeySwitch_23.cuh:544-578,
 * restated with the automorphism applied before the key switch) */
void orc_apply_galois(const orc_ctx* c, const u64* gk, u64 g, const u64* ct, u64* out) {
    size_t lq = (size_t)c->nq * c->n;
    u64* t = calloc(3 * lq, 8);
    orc_galois_ntt(c, g, ct, t, c->nq);
    orc_galois_ntt(c, g, ct + lq, t + 2 * lq, c->nq);
    orc_relinearize(c, t, gk, out);
    free(t);
}

void orc_mul_relin(const orc_ctx* c, const u64* ct1, const u64* ct2, const u64* rlk, u64* ct) {
    u64* d = malloc((size_t)3 * c->nq * c->n * 8);
    orc_mul_tensor(c, ct1, ct2, d);
    orc_relinearize(c, d, rlk, ct);
    free(d);
}

/* invariant noise budget: log2(Q) - log2(max |[t * (b + a*s)]_Q|) - 1 */
double orc_noise_budget(const orc_ctx* c, const u64* sk, const u64* ct) {
    u64 n = c->n;
    int nq = c->nq;
    u64* x = malloc((size_t)nq * n * 8);
    for (size_t i = 0; i < (size_t)nq * n; i++) {
        u64 q = c->mods[i / n];
        x[i] = addmod(mulmod(ct[i], sk[i], q), ct[(size_t)nq * n + i], q);
    }
    ntt_inv_limbs(c, 0, x, nq);
    big Q; big_set(&Q, 1);
    for (int i = 0; i < nq; i++) big_mul_word(&Q, c->mods[i]);
    big half; big_div_word(&Q, 2, &half);
    big hats[64];
    for (int i = 0; i < nq; i++) {
        big_set(&hats[i], 1);
        for (int k = 0; k < nq; k++) if (k != i) big_mul_word(&hats[i], c->mods[k]);
    }
    double worst = -INFINITY;
    for (u64 k = 0; k < n; k++) {
        big z; big_set(&z, 0);
        for (int i = 0; i < nq; i++) {
            u64 q = c->mods[i];
            u64 y = mulmod(mulmod(x[(size_t)i * n + k], c->t % q, q), c->q2r.hatinv[i], q);
            big term = hats[i];
            big_mul_word(&term, y);
            big_add(&z, &term);
        }
        while (big_cmp(&z, &Q) >= 0) big_sub(&z, &Q);
        if (big_cmp(&z, &half) > 0) { big w = Q; big_sub(&w, &z); z = w; }
        double lz = big_log2(&z);
        if (lz > worst) worst = lz;
    }
    free(x);
    return big_log2(&Q) - worst - 1.0;
}

/* The reference's relinearisation (multAndEqual_23, KeySwitch_23.cuh:277-305):
 * a1a2 to coefficients, Qj blocks lifted into T, NTT over T, external product
 * with the KLSS key (NTT over T, [ax|bx][digit][Ri][T]), INTT over T, exact
 * T -> P|Q, mod down, NTT over Q, add [cross | b1b2]. d is [a1a2|cross|b1b2] in
 * NTT form over Q. */
void orc_klss_relinearize(const orc_ctx* c, const u64* d, const u64* key_t, u64* ct) {
    u64 n = c->n;
    int nq = c->nq, nt = c->nt;
    int nri = orc_klss_ri_blocks(c), nqj = orc_klss_qj_blocks(c);
    int t0 = c->nq + c->np + c->nr;
    size_t lq = (size_t)nq * n;
    u64* d2 = malloc(lq * 8);
    u64* dig = malloc((size_t)nqj * nt * n * 8);
    u64* ext = malloc((size_t)2 * nri * nt * n * 8);
    u64* pq = calloc((size_t)2 * nri * nt * n, 8);
    u64* dn = malloc(2 * lq * 8);
    memcpy(d2, d, lq * 8);
    ntt_inv_limbs(c, 0, d2, nq);
    orc_klss_modup_qj_to_t(c, d2, dig);
    for (int b = 0; b < nqj; b++) ntt_fwd_limbs(c, t0, dig + (size_t)b * nt * n, nt);
    orc_klss_external_product(c, dig, key_t, ext);
    for (int b = 0; b < 2 * nri; b++) ntt_inv_limbs(c, t0, ext + (size_t)b * nt * n, nt);
    orc_klss_modup_t_to_pq(c, ext, pq, 2);
    orc_klss_moddown(c, pq, dn, 2);
    ntt_fwd_limbs(c, 0, dn, nq);
    ntt_fwd_limbs(c, 0, dn + lq, nq);
    for (size_t i = 0; i < lq; i++) {
        u64 q = c->mods[i / n];
        ct[i] = addmod(d[lq + i], dn[i], q);
        ct[lq + i] = addmod(d[2 * lq + i], dn[lq + i], q);
    }
    free(d2); free(dig); free(ext); free(pq); free(dn);
}
