// libkbfv: context construction, launch plumbing, the fused batched
// multiply + relinearize pipeline, and the C ABI declared in include/kbfv.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/kbfv.h"
#include "context.cuh"
#include "host_math.hpp"
#include "kernels.cuh"
#include "ntt.cuh"
#include "klss.cuh"

using namespace kbfv;
namespace H = kbfv::host;

// ===========================================================================
// errors
// ===========================================================================
static thread_local std::string g_last_error;

struct KbfvError : std::runtime_error {
    int code;
    KbfvError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define KB_CHECK_CUDA(call)                                                                        \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw KbfvError(e_ == cudaErrorMemoryAllocation ? KBFV_ERR_NOMEM : KBFV_ERR_CUDA,      \
                            std::string(#call) + ": " + cudaGetErrorString(e_));                   \
    } while (0)

#define KB_REQUIRE(cond, code, msg) \
    do {                            \
        if (!(cond)) throw KbfvError((code), (msg)); \
    } while (0)

template <class F>
static int guarded(F&& f) {
    try {
        f();
        return KBFV_OK;
    } catch (const KbfvError& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return KBFV_ERR_INVALID;
    }
}

static void check_launch(const char* what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw KbfvError(KBFV_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ===========================================================================
// context construction (BFVContext::BFVContext / preComputeOnCPU / copyMemoryToGPU,
// include/BFVcontext.cuh:13-1395, restated without NTL and without __constant__)
// ===========================================================================
namespace {

struct Blob {
    std::vector<uint8_t> bytes;
    size_t add(const void* p, size_t n) {
        size_t off = (bytes.size() + 255) & ~(size_t)255;
        bytes.resize(off + n);
        std::memcpy(bytes.data() + off, p, n);
        return off;
    }
    template <class T>
    size_t add(const std::vector<T>& v) { return add(v.data(), v.size() * sizeof(T)); }
};

std::vector<uint64_t> bitrev_powers(uint64_t root, uint64_t q, int logn) {
    const uint64_t n = (uint64_t)1 << logn;
    std::vector<uint64_t> out(n);
    uint64_t cur = 1;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t r = 0, x = i;
        for (int b = 0; b < logn; b++) { r = (r << 1) | (x & 1); x >>= 1; }
        out[r] = cur;  // out[brv(i)] = root^i
        cur = H::mulmod(cur, root, q);
    }
    return out;
}

struct HostBconv {
    std::vector<uint64_t> hatinv, hatinvs, hat, alpha;
    std::vector<double> inv;
};

// BaseConverter::init (include/BasisConv_QR.cuh:53-189)
HostBconv make_bconv(const std::vector<uint64_t>& in, const std::vector<uint64_t>& out) {
    HostBconv b;
    const size_t nin = in.size(), nout = out.size();
    b.hatinv.resize(nin); b.hatinvs.resize(nin); b.inv.resize(nin);
    b.hat.resize(nin * nout); b.alpha.resize((nin + 1) * nout);
    for (size_t i = 0; i < nin; i++) {
        uint64_t h = 1;
        for (size_t k = 0; k < nin; k++) if (k != i) h = H::mulmod(h, in[k] % in[i], in[i]);
        b.hatinv[i] = nin > 1 ? H::invmod(h, in[i]) : 1;
        b.hatinvs[i] = H::shoup(b.hatinv[i], in[i]);
        b.inv[i] = 1.0 / (double)in[i];
    }
    for (size_t j = 0; j < nout; j++) {
        const uint64_t o = out[j];
        uint64_t bm = 1;
        for (size_t i = 0; i < nin; i++) {
            uint64_t h = 1;
            for (size_t k = 0; k < nin; k++) if (k != i) h = H::mulmod(h, in[k] % o, o);
            b.hat[j * nin + i] = h;
            bm = H::mulmod(bm, in[i] % o, o);
        }
        for (size_t a = 0; a <= nin; a++) b.alpha[a * nout + j] = H::mulmod(a, bm, o);
    }
    return b;
}

void gaussian_cdt(double sigma, int bound, std::vector<uint64_t>& table) {
    std::vector<long double> w(2 * bound + 1);
    long double z = 0;
    for (int x = -bound; x <= bound; x++) {
        w[x + bound] = expl(-(long double)x * x / (2.0L * (long double)sigma * sigma));
        z += w[x + bound];
    }
    table.assign(2 * bound + 1, 0);
    long double acc = 0;
    for (int k = 0; k < 2 * bound; k++) {
        acc += w[k];
        long double v = acc / z * 18446744073709551616.0L;
        table[k] = v >= 18446744073709551615.0L ? UINT64_MAX : (uint64_t)v;
    }
    table[2 * bound] = UINT64_MAX;
}

}  // namespace

static void build_context(Context& c, const kbfv_params& prm) {
    KB_REQUIRE(prm.log_n >= 10 && prm.log_n <= 16, KBFV_ERR_INVALID, "log_n must be in [10, 16]");
    KB_REQUIRE(prm.q_count >= 1 && prm.q_count <= (uint32_t)kMaxQ, KBFV_ERR_INVALID, "q_count out of range");
    KB_REQUIRE(prm.p_count >= 1 && prm.p_count <= (uint32_t)kMaxP, KBFV_ERR_INVALID, "p_count out of range");
    c.logn = (int)prm.log_n;
    c.n = (uint64_t)1 << c.logn;
    c.t = prm.plain_modulus;
    c.nq = (int)prm.q_count;
    c.np = (int)prm.p_count;
    c.nr = c.nq + 1;
    c.nt = (int)prm.t_count;
    c.gamma = prm.gamma ? (int)prm.gamma : 1;
    if (prm.digit_primes) {  // explicit digit size (levels keep the top level's digits)
        c.alpha = (int)prm.digit_primes;
        c.dnum = (c.nq + c.alpha - 1) / c.alpha;
    } else {
        c.dnum = prm.dnum ? (int)prm.dnum : 1;
        KB_REQUIRE(c.dnum <= c.nq, KBFV_ERR_INVALID, "dnum exceeds q_count");
        c.alpha = (c.nq + c.dnum - 1) / c.dnum;
    }
    KB_REQUIRE(H::is_prime(c.t) && (c.t - 1) % (2 * c.n) == 0, KBFV_ERR_PARAMS,
               "plain modulus must be a prime congruent to 1 mod 2N");

    std::vector<uint64_t> P, Q;
    if (prm.p) P.assign(prm.p, prm.p + c.np);
    else P = H::primes_bits(c.n, (int)prm.p_bits, c.np, {});
    KB_REQUIRE((int)P.size() == c.np, KBFV_ERR_PARAMS, "not enough special primes of the requested size");
    if (prm.q) Q.assign(prm.q, prm.q + c.nq);
    else Q = H::primes_bits(c.n, (int)prm.q_bits, c.nq, P);
    KB_REQUIRE((int)Q.size() == c.nq, KBFV_ERR_PARAMS, "not enough ciphertext primes of the requested size");
    uint64_t qmin = *std::min_element(Q.begin(), Q.end());
    // R base: r_num = q_num + 1 primes below min q (include/BFVcontext.cuh:56-58)
    std::vector<uint64_t> R = H::primes_below(c.n, qmin, c.nr);
    KB_REQUIRE((int)R.size() == c.nr, KBFV_ERR_PARAMS, "not enough R primes below min q");

    c.mods.clear();
    c.mods.insert(c.mods.end(), Q.begin(), Q.end());
    c.mods.insert(c.mods.end(), P.begin(), P.end());
    c.mods.insert(c.mods.end(), R.begin(), R.end());
    for (int i = 0; i < c.nt; i++) c.mods.push_back(prm.t_primes[i]);
    c.mods.push_back(c.t);
    const int nall = (int)c.mods.size();
    KB_REQUIRE(nall <= kMaxPrimes, KBFV_ERR_INVALID, "too many primes");
    for (int i = 0; i < nall; i++) {
        const uint64_t q = c.mods[i];
        KB_REQUIRE(H::is_prime(q) && q < ((uint64_t)1 << 60) && (q - 1) % (2 * c.n) == 0, KBFV_ERR_PARAMS,
                   "every modulus must be a prime below 2^60 congruent to 1 mod 2N");
        for (int j = 0; j < i; j++)
            KB_REQUIRE(c.mods[j] != q || (i == nall - 1), KBFV_ERR_PARAMS, "moduli must be distinct");
    }

    DevConsts& dc = c.dc;
    dc.logn = c.logn; dc.nq = c.nq; dc.np = c.np; dc.nr = c.nr; dc.nt = c.nt;
    dc.dnum = c.dnum; dc.alpha = c.alpha; dc.npq = c.nq + c.np; dc.nqr = c.nq + c.nr;
    dc.idx_p = c.nq; dc.idx_r = c.nq + c.np; dc.idx_t = c.nq + c.np + c.nr; dc.idx_pt = nall - 1;
    dc.t = c.t;
    dc.key_nq = c.nq;
    dc.key_npq = c.nq + c.np;

    Blob blob;
    std::vector<uint64_t> mu_hi(nall), mu_lo(nall);
    for (int i = 0; i < nall; i++) H::barrett_mu(c.mods[i], mu_hi[i], mu_lo[i]);
    std::vector<uint64_t> mu_prod(nall);
    for (int i = 0; i < nall; i++) {
        const int k = 64 - __builtin_clzll(c.mods[i]);
        mu_prod[i] = (uint64_t)(((unsigned __int128)1 << (62 + k)) / c.mods[i]);
    }
    size_t o_mods = blob.add(c.mods), o_muh = blob.add(mu_hi), o_mul = blob.add(mu_lo);
    size_t o_mup = blob.add(mu_prod);

    // twiddles: fwd[i] = psi^brv(i); inv[i] = psi^-brv(i), inv[0] = n^-1, inv[1] *= n^-1
    std::vector<tw_t> twf((size_t)nall << c.logn), twi((size_t)nall << c.logn);
    for (int p = 0; p < nall; p++) {
        const uint64_t q = c.mods[p];
        const uint64_t psi = H::root_2n(q, c.n);
        KB_REQUIRE(H::root_ok(psi, q, c.n), KBFV_ERR_PARAMS, "no primitive 2N-th root for a modulus");
        const uint64_t ipsi = H::invmod(psi, q);
        std::vector<uint64_t> f = bitrev_powers(psi, q, c.logn), g = bitrev_powers(ipsi, q, c.logn);
        const uint64_t ninv = H::invmod(c.n % q, q);
        g[0] = ninv;
        g[1] = H::mulmod(g[1], ninv, q);
        tw_t* tf = twf.data() + ((size_t)p << c.logn);
        tw_t* ti = twi.data() + ((size_t)p << c.logn);
        for (uint64_t i = 0; i < c.n; i++) {
            tf[i].x = f[i]; tf[i].y = H::shoup(f[i], q);
            ti[i].x = g[i]; ti[i].y = H::shoup(g[i], q);
        }
    }
    size_t o_twf = blob.add(twf), o_twi = blob.add(twi);

    HostBconv q2r = make_bconv(Q, R), r2q = make_bconv(R, Q);
    c.h_q2r_hatinv = q2r.hatinv;
    size_t o_q2r[5] = {blob.add(q2r.hatinv), blob.add(q2r.hatinvs), blob.add(q2r.hat), blob.add(q2r.alpha),
                       blob.add(q2r.inv)};
    size_t o_r2q[5] = {blob.add(r2q.hatinv), blob.add(r2q.hatinvs), blob.add(r2q.hat), blob.add(r2q.alpha),
                       blob.add(r2q.inv)};

    // t/Q scale-and-round constants (include/BFVcontext.cuh:1267-1389)
    std::vector<double> sr_frac(c.nq);
    std::vector<uint64_t> sr_c((size_t)c.nr * (c.nq + 1));
    {
        std::vector<uint64_t> qr(Q);
        qr.insert(qr.end(), R.begin(), R.end());
        const int nqr = (int)qr.size();
        H::Big tR(c.t);
        for (uint64_t r : R) tR.mul_word(r);
        std::vector<H::Big> divs(nqr);
        for (int i = 0; i < nqr; i++) {
            const uint64_t si = qr[i];
            uint64_t h = 1;
            for (int k = 0; k < nqr; k++) if (k != i) h = H::mulmod(h, qr[k] % si, si);
            H::Big v = tR;
            v.mul_word(H::invmod(h, si));
            if (i < c.nq) sr_frac[i] = (double)v.mod_word(si) / (double)si;
            divs[i] = v.div_word(si);
        }
        for (int j = 0; j < c.nr; j++) {
            for (int i = 0; i < c.nq; i++) sr_c[(size_t)j * (c.nq + 1) + i] = divs[i].mod_word(R[j]);
            sr_c[(size_t)j * (c.nq + 1) + c.nq] = divs[c.nq + j].mod_word(R[j]);
        }
    }
    size_t o_srf = blob.add(sr_frac), o_src = blob.add(sr_c);

    // decrypt rounding constants (include/BFVcontext.cuh:1030-1156) and variant (1680-1717)
    const uint64_t qmax = *std::max_element(Q.begin(), Q.end());
    const int qmsb = H::bit_count(qmax), sizeqmsb = H::bit_count((uint64_t)c.nq), tmsb = H::bit_count(c.t);
    const int hf = qmsb >> 1;
    std::vector<uint64_t> dmt(c.nq, 0), dmts(c.nq, 0), dmbt(c.nq, 0), dmbts(c.nq, 0);
    std::vector<double> dfr(c.nq, 0.0), dfrb(c.nq, 0.0);
    for (int i = 0; i < c.nq; i++) {
        const uint64_t qi = Q[i], hinv = q2r.hatinv[i];
        const H::u128 big_t = (H::u128)c.t * hinv;
        dmt[i] = (uint64_t)((big_t / qi) % c.t);
        dmts[i] = H::shoup(dmt[i], c.t);
        dfr[i] = (double)(uint64_t)(big_t % qi) / (double)qi;
        if (qmsb + sizeqmsb >= 52) {
            const uint64_t hb = (uint64_t)(((H::u128)hinv << hf) % qi);
            const H::u128 bigb = (H::u128)c.t * hb;
            dmbt[i] = (uint64_t)((bigb / qi) % c.t);
            dmbts[i] = H::shoup(dmbt[i], c.t);
            dfrb[i] = (double)(uint64_t)(bigb % qi) / (double)qi;
        }
    }
    if (qmsb + sizeqmsb < 52) c.dec_variant = (qmsb + tmsb + sizeqmsb) < 52 ? 1 : 0;
    else c.dec_variant = (hf + tmsb + sizeqmsb) < 52 ? 3 : 2;
    dc.dec_variant = c.dec_variant;
    dc.qmsbhf = hf;
    size_t o_dec[6] = {blob.add(dmt), blob.add(dmts), blob.add(dmbt), blob.add(dmbts), blob.add(dfr), blob.add(dfrb)};

    // delta * m (include/BFVcontext.cuh:881-926)
    {
        uint64_t qmt = 1;
        for (uint64_t q : Q) qmt = H::mulmod(qmt, q % c.t, c.t);
        dc.negq_mod_t = c.t - qmt;
        dc.negq_mod_t_s = H::shoup(dc.negq_mod_t, c.t);
    }
    std::vector<uint64_t> tinv(c.nq), tinvs(c.nq);
    for (int i = 0; i < c.nq; i++) {
        tinv[i] = H::invmod(c.t % Q[i], Q[i]);
        tinvs[i] = H::shoup(tinv[i], Q[i]);
    }
    size_t o_tinv = blob.add(tinv), o_tinvs = blob.add(tinvs);

    // key switching: P mod q, P^-1 mod q, (P/p_k)^-1 mod p_k, (P/p_k) mod q
    std::vector<uint64_t> pmq(c.nq), pinv(c.nq), pinvs(c.nq), phm((size_t)c.nq * c.np), phi(c.np), phis(c.np);
    for (int i = 0; i < c.nq; i++) {
        uint64_t pm = 1;
        for (uint64_t p : P) pm = H::mulmod(pm, p % Q[i], Q[i]);
        pmq[i] = pm;
        pinv[i] = H::invmod(pm, Q[i]);
        pinvs[i] = H::shoup(pinv[i], Q[i]);
        for (int k = 0; k < c.np; k++) {
            uint64_t h = 1;
            for (int m = 0; m < c.np; m++) if (m != k) h = H::mulmod(h, P[m] % Q[i], Q[i]);
            phm[(size_t)i * c.np + k] = h;
        }
    }
    for (int k = 0; k < c.np; k++) {
        uint64_t h = 1;
        for (int m = 0; m < c.np; m++) if (m != k) h = H::mulmod(h, P[m] % P[k], P[k]);
        phi[k] = H::invmod(h, P[k]);
        phis[k] = H::shoup(phi[k], P[k]);
    }
    // digit lift constants: digit d covers primes [d*alpha, min((d+1)*alpha, nq))
    const int npq = c.nq + c.np;
    std::vector<uint64_t> dhi(c.nq), dhis(c.nq), dhm((size_t)c.dnum * npq * c.alpha, 0), dqm((size_t)c.dnum * npq, 0);
    for (int d = 0; d < c.dnum; d++) {
        const int lo = d * c.alpha, hi = std::min(lo + c.alpha, c.nq);
        for (int j = lo; j < hi; j++) {
            uint64_t h = 1;
            for (int k = lo; k < hi; k++) if (k != j) h = H::mulmod(h, Q[k] % Q[j], Q[j]);
            dhi[j] = H::invmod(h, Q[j]);
            dhis[j] = H::shoup(dhi[j], Q[j]);
        }
        for (int m = 0; m < npq; m++) {
            const uint64_t mod = c.mods[m];
            uint64_t qm = 1;
            for (int j = lo; j < hi; j++) {
                uint64_t h = 1;
                for (int k = lo; k < hi; k++) if (k != j) h = H::mulmod(h, Q[k] % mod, mod);
                dhm[((size_t)d * npq + m) * c.alpha + (j - lo)] = h;
                qm = H::mulmod(qm, Q[j] % mod, mod);
            }
            dqm[(size_t)d * npq + m] = qm;
        }
    }
    // v * Q_d mod p_m for the lift's quotient estimate v = 0..alpha
    std::vector<uint64_t> dvq((size_t)c.dnum * (c.alpha + 1) * npq);
    for (int d = 0; d < c.dnum; d++)
        for (int v = 0; v <= c.alpha; v++)
            for (int m = 0; m < npq; m++)
                dvq[((size_t)d * (c.alpha + 1) + v) * npq + m] =
                    H::mulmod((uint64_t)v, dqm[(size_t)d * npq + m], c.mods[m]);
    size_t o_ks[11] = {blob.add(pmq), blob.add(pinv), blob.add(pinvs), blob.add(phi), blob.add(phis),
                       blob.add(phm), blob.add(dhi), blob.add(dhis), blob.add(dhm), blob.add(dqm), blob.add(dvq)};
    // T-base key switch constants (include/BasisConv.cuh:11-226; the reference's
    // precompute is in include/BFVcontext.cuh). Blocks lift by approximate CRT:
    // (B/b_j)^-1 mod b_j, B/b_j mod t_k and B mod t_k per block B.
    c.klss_ok = c.nt > 0 && c.nt <= kMaxT && c.np <= kMaxBlk && c.gamma >= 1 && c.gamma <= kMaxBlk &&
                c.nq % c.np == 0 && c.alpha == c.np && c.dnum == c.nq / c.np;
    size_t o_kl[14] = {};
    if (c.klss_ok) {
        const int nt = c.nt, g = c.gamma, nqj = c.nq / c.np, nri = (npq + g - 1) / g;
        const std::vector<uint64_t> Tm(c.mods.begin() + c.nq + c.np + c.nr, c.mods.begin() + c.nq + c.np + c.nr + nt);
        std::vector<uint64_t> PQr;  // reference order: P then Q
        PQr.insert(PQr.end(), P.begin(), P.end());
        PQr.insert(PQr.end(), Q.begin(), Q.end());
        auto lift = [&](const uint64_t* blk, int w, int stride, uint64_t* hinv, uint64_t* hinvs, uint64_t* hat_t,
                        uint64_t* mod_t) {
            for (int j = 0; j < w; j++) {
                uint64_t h = 1;
                for (int k = 0; k < w; k++) if (k != j) h = H::mulmod(h, blk[k] % blk[j], blk[j]);
                hinv[j] = H::invmod(h, blk[j]);
                hinvs[j] = H::shoup(hinv[j], blk[j]);
            }
            for (int t = 0; t < nt; t++) {
                uint64_t bm = 1;
                for (int j = 0; j < w; j++) {
                    uint64_t h = 1;
                    for (int k = 0; k < w; k++) if (k != j) h = H::mulmod(h, blk[k] % Tm[t], Tm[t]);
                    hat_t[(size_t)t * stride + j] = h;
                    bm = H::mulmod(bm, blk[j] % Tm[t], Tm[t]);
                }
                mod_t[t] = bm;
            }
        };
        std::vector<uint64_t> qhi((size_t)nqj * c.np), qhis(qhi.size()), qht((size_t)nqj * nt * c.np), qmt((size_t)nqj * nt);
        for (int b = 0; b < nqj; b++)
            lift(Q.data() + (size_t)b * c.np, c.np, c.np, &qhi[(size_t)b * c.np], &qhis[(size_t)b * c.np],
                 &qht[(size_t)b * nt * c.np], &qmt[(size_t)b * nt]);
        std::vector<uint64_t> rhi((size_t)nri * g, 0), rhis(rhi.size(), 0), rht((size_t)nri * nt * g, 0), rmt((size_t)nri * nt);
        for (int b = 0; b < nri; b++)
            lift(PQr.data() + (size_t)b * g, std::min(g, npq - b * g), g, &rhi[(size_t)b * g], &rhis[(size_t)b * g],
                 &rht[(size_t)b * nt * g], &rmt[(size_t)b * nt]);
        std::vector<uint64_t> thi(nt), this_(nt), thpq((size_t)npq * nt), tpq(npq), htt(nt), htpq(npq);
        H::Big Tb(1);
        for (uint64_t tk : Tm) Tb.mul_word(tk);
        const H::Big half = Tb.div_word(2);
        for (int i = 0; i < nt; i++) {
            uint64_t h = 1;
            for (int k = 0; k < nt; k++) if (k != i) h = H::mulmod(h, Tm[k] % Tm[i], Tm[i]);
            thi[i] = H::invmod(h, Tm[i]);
            this_[i] = H::shoup(thi[i], Tm[i]);
            htt[i] = half.mod_word(Tm[i]);
        }
        for (int m = 0; m < npq; m++) {
            const uint64_t r = PQr[m];
            for (int i = 0; i < nt; i++) {
                uint64_t h = 1;
                for (int k = 0; k < nt; k++) if (k != i) h = H::mulmod(h, Tm[k] % r, r);
                thpq[(size_t)m * nt + i] = h;
            }
            tpq[m] = Tb.mod_word(r);
            htpq[m] = half.mod_word(r);
        }
        const std::vector<uint64_t>* tabs[14] = {&qhi, &qhis, &qht, &qmt, &rhi, &rhis, &rht, &rmt,
                                                 &thi, &this_, &thpq, &tpq, &htt, &htpq};
        for (int i = 0; i < 14; i++) o_kl[i] = blob.add(*tabs[i]);
        c.kc.nt = nt; c.kc.gamma = g; c.kc.nri = nri; c.kc.nqj = nqj;
    }
    // modulus switch by the last prime
    std::vector<uint64_t> msi(c.nq, 0), msis(c.nq, 0), msh(c.nq, 0);
    {
        const uint64_t ql = Q[c.nq - 1];
        dc.ms_half = ql >> 1;
        for (int i = 0; i + 1 < c.nq; i++) {
            msi[i] = H::invmod(ql % Q[i], Q[i]);
            msis[i] = H::shoup(msi[i], Q[i]);
            msh[i] = dc.ms_half % Q[i];
        }
    }
    size_t o_ms[3] = {blob.add(msi), blob.add(msis), blob.add(msh)};
    std::vector<uint64_t> cdt;
    gaussian_cdt(3.2, 19, cdt);
    dc.gauss_bound = 19;
    size_t o_cdt = blob.add(cdt);

    KB_CHECK_CUDA(cudaGetDevice(&c.device));
    KB_CHECK_CUDA(cudaMalloc(&c.pool, blob.bytes.size()));
    KB_CHECK_CUDA(cudaMemcpy(c.pool, blob.bytes.data(), blob.bytes.size(), cudaMemcpyHostToDevice));
    uint8_t* base = (uint8_t*)c.pool;
    auto U = [&](size_t o) { return (const uint64_t*)(base + o); };
    auto D = [&](size_t o) { return (const double*)(base + o); };
    dc.mods = U(o_mods); dc.mu_hi = U(o_muh); dc.mu_lo = U(o_mul); dc.mu_prod = U(o_mup);
    dc.tw_fwd = (const tw_t*)(base + o_twf); dc.tw_inv = (const tw_t*)(base + o_twi);
    dc.q2r_hatinv = U(o_q2r[0]); dc.q2r_hatinvs = U(o_q2r[1]); dc.q2r_hat = U(o_q2r[2]);
    dc.q2r_alpha = U(o_q2r[3]); dc.q2r_inv = D(o_q2r[4]);
    dc.r2q_hatinv = U(o_r2q[0]); dc.r2q_hatinvs = U(o_r2q[1]); dc.r2q_hat = U(o_r2q[2]);
    dc.r2q_alpha = U(o_r2q[3]); dc.r2q_inv = D(o_r2q[4]);
    dc.sr_frac = D(o_srf); dc.sr_c = U(o_src);
    dc.dec_mod_t = U(o_dec[0]); dc.dec_mod_t_s = U(o_dec[1]); dc.dec_modB_t = U(o_dec[2]);
    dc.dec_modB_t_s = U(o_dec[3]); dc.dec_frac = D(o_dec[4]); dc.dec_fracB = D(o_dec[5]);
    dc.tinv_q = U(o_tinv); dc.tinv_qs = U(o_tinvs);
    dc.p_mod_q = U(o_ks[0]); dc.pinv_q = U(o_ks[1]); dc.pinv_qs = U(o_ks[2]); dc.phatinv_p = U(o_ks[3]);
    dc.phatinv_ps = U(o_ks[4]); dc.phat_mod_q = U(o_ks[5]); dc.dig_hatinv = U(o_ks[6]);
    dc.dig_hatinvs = U(o_ks[7]); dc.dig_hat_mod = U(o_ks[8]); dc.dig_q_mod = U(o_ks[9]);
    dc.dig_vq_mod = U(o_ks[10]);
    dc.ms_qlinv = U(o_ms[0]); dc.ms_qlinvs = U(o_ms[1]); dc.ms_half_mod = U(o_ms[2]);
    dc.gauss_cdt = U(o_cdt);
    if (c.klss_ok) {
        KlssConsts& k = c.kc;
        k.qj_hatinv = U(o_kl[0]); k.qj_hatinvs = U(o_kl[1]); k.qj_hat_t = U(o_kl[2]); k.qj_mod_t = U(o_kl[3]);
        k.ri_hatinv = U(o_kl[4]); k.ri_hatinvs = U(o_kl[5]); k.ri_hat_t = U(o_kl[6]); k.ri_mod_t = U(o_kl[7]);
        k.thatinv = U(o_kl[8]); k.thatinvs = U(o_kl[9]); k.that_pq = U(o_kl[10]); k.t_pq = U(o_kl[11]);
        k.halft_t = U(o_kl[12]); k.halft_pq = U(o_kl[13]);
    }
    KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.ptrs_event, cudaEventDisableTiming));
}

// ===========================================================================
// launch helpers
// ===========================================================================
static inline cudaStream_t S(kbfv_stream s) { return (cudaStream_t)s; }
static inline unsigned blocks_for(size_t total, unsigned threads) { return (unsigned)((total + threads - 1) / threads); }
// grid of a grid-stride kernel: enough blocks to cover `total`, at most 2^20
static inline unsigned stride_blocks(size_t total, unsigned threads) {
    return (unsigned)std::min<size_t>((total + threads - 1) / threads, (size_t)1 << 20);
}

template <int LOGB, class Src, class Dst, bool FULL = true>
static void launch_fwd_block(const DevConsts& dc, Src s, Dst d, int rows, int logn, cudaStream_t st) {
    constexpr int SMEM = BlockShape<LOGB>::SMEM_BYTES;
    static bool configured = false;
    if (!configured) {
        KB_CHECK_CUDA(cudaFuncSetAttribute(ntt_fwd_block_kernel<LOGB, Src, Dst, FULL>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
        configured = true;
    }
    const int nblk = 1 << (logn - LOGB);
    ntt_fwd_block_kernel<LOGB, Src, Dst, FULL><<<rows * nblk, BlockShape<LOGB>::THREADS, SMEM, st>>>(
        s, d, dc.tw_fwd, dc.mods, logn);
}

template <int LOGB, class Src, class Dst, bool WHOLE>
static void launch_inv_block(const DevConsts& dc, Src s, Dst d, int rows, int logn, cudaStream_t st) {
    constexpr int SMEM = BlockShape<LOGB>::SMEM_BYTES;
    static bool configured = false;
    if (!configured) {
        KB_CHECK_CUDA(cudaFuncSetAttribute(ntt_inv_block_kernel<LOGB, Src, Dst, WHOLE>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM));
        configured = true;
    }
    const int nblk = 1 << (logn - LOGB);
    ntt_inv_block_kernel<LOGB, Src, Dst, WHOLE><<<rows * nblk, BlockShape<LOGB>::THREADS, SMEM, st>>>(
        s, d, dc.tw_inv, dc.mods, logn);
}

// The view of a store target that the column pass of a split transform writes
// and the block kernel reads back: the target itself, unless its store adds an
// epilogue (an overload for that target returns its plain rows).
template <class Dst>
static inline Dst plain_of(const Dst& d) { return d; }

// At N = 2^14, launches of at most this many rows (fewer 1024-thread CTAs
// than SMs, e.g. one ciphertext pair per call: 2-45 rows) run as a radix-4
// column pass and 2^12-point blocks: four times the CTAs cover the SMs, 15-23 us
// instead of 29-31 us per launch of 8-45 rows on the B200. At 64 rows the
// split alone is still faster, but beside a concurrent sub-batch it cost the
// batched multiply ~1%, so 64-row launches keep the whole-ring blocks.
constexpr int kSplitRows14 = 48;

// Forward NTT of `rows` rows read through `s` and written through `d`.
// For logn <= 14 one block kernel (N = 2^14 with at most kSplitRows14 rows:
// as for 15/16 with a radix-4 column pass); for 15/16 a radix-8/16 column pass
// (s -> plain_of(d)) then 2^12-point block kernels from plain_of(d) to d in
// place (d must also be readable): several 256-thread CTAs per SM run faster
// than one 1024-thread CTA per 2^14-point block. FULL = false leaves outputs in [0, 8q) for consumers that reduce
// anyway (pipeline stages only).
template <class Src, class Dst, bool FULL = true>
static void ntt_fwd(const DevConsts& dc, Src s, Dst d, int rows, cudaStream_t st) {
    if (rows <= 0) return;
    switch (dc.logn) {
        case 10: launch_fwd_block<10, Src, Dst, FULL>(dc, s, d, rows, 10, st); break;
        case 11: launch_fwd_block<11, Src, Dst, FULL>(dc, s, d, rows, 11, st); break;
        case 12: launch_fwd_block<12, Src, Dst, FULL>(dc, s, d, rows, 12, st); break;
        case 13: launch_fwd_block<13, Src, Dst, FULL>(dc, s, d, rows, 13, st); break;
        case 14: {
            if (rows > kSplitRows14) {
                launch_fwd_block<14, Src, Dst, FULL>(dc, s, d, rows, 14, st);
                break;
            }
            const size_t total = (size_t)rows << 12;
            using DP = decltype(plain_of(d));
            const DP dp = plain_of(d);
            ntt_fwd_col_kernel<2, Src, DP><<<stride_blocks(total, 256), 256, 0, st>>>(s, dp, dc.tw_fwd, dc.mods, 14, total);
            launch_fwd_block<12, DP, Dst, FULL>(dc, dp, d, rows, 14, st);
            break;
        }
        case 15: {
            const size_t total = (size_t)rows << 12;
            using DP = decltype(plain_of(d));
            const DP dp = plain_of(d);
            ntt_fwd_col_kernel<3, Src, DP><<<stride_blocks(total, 256), 256, 0, st>>>(s, dp, dc.tw_fwd, dc.mods, 15, total);
            launch_fwd_block<12, DP, Dst, FULL>(dc, dp, d, rows, 15, st);
            break;
        }
        case 16: {
            const size_t total = (size_t)rows << 12;
            using DP = decltype(plain_of(d));
            const DP dp = plain_of(d);
            ntt_fwd_col_kernel<4, Src, DP><<<stride_blocks(total, 256), 256, 0, st>>>(s, dp, dc.tw_fwd, dc.mods, 16, total);
            launch_fwd_block<12, DP, Dst, FULL>(dc, dp, d, rows, 16, st);
            break;
        }
        default: throw KbfvError(KBFV_ERR_INVALID, "unsupported ring degree");
    }
    check_launch("ntt_fwd");
}

template <class Src, class Dst>
static void ntt_inv(const DevConsts& dc, Src s, Dst d, int rows, cudaStream_t st) {
    if (rows <= 0) return;
    switch (dc.logn) {
        case 10: launch_inv_block<10, Src, Dst, true>(dc, s, d, rows, 10, st); break;
        case 11: launch_inv_block<11, Src, Dst, true>(dc, s, d, rows, 11, st); break;
        case 12: launch_inv_block<12, Src, Dst, true>(dc, s, d, rows, 12, st); break;
        case 13: launch_inv_block<13, Src, Dst, true>(dc, s, d, rows, 13, st); break;
        case 14: {
            if (rows > kSplitRows14) {
                launch_inv_block<14, Src, Dst, true>(dc, s, d, rows, 14, st);
                break;
            }
            launch_inv_block<12, Src, Dst, false>(dc, s, d, rows, 14, st);
            const size_t total = (size_t)rows << 12;
            ntt_inv_col_kernel<2, Dst, Dst><<<stride_blocks(total, 256), 256, 0, st>>>(d, d, dc.tw_inv, dc.mods, 14, total);
            break;
        }
        case 15: {
            launch_inv_block<12, Src, Dst, false>(dc, s, d, rows, 15, st);
            const size_t total = (size_t)rows << 12;
            ntt_inv_col_kernel<3, Dst, Dst><<<stride_blocks(total, 256), 256, 0, st>>>(d, d, dc.tw_inv, dc.mods, 15, total);
            break;
        }
        case 16: {
            launch_inv_block<12, Src, Dst, false>(dc, s, d, rows, 16, st);
            const size_t total = (size_t)rows << 12;
            ntt_inv_col_kernel<4, Dst, Dst><<<stride_blocks(total, 256), 256, 0, st>>>(d, d, dc.tw_inv, dc.mods, 16, total);
            break;
        }
        default: throw KbfvError(KBFV_ERR_INVALID, "unsupported ring degree");
    }
    check_launch("ntt_inv");
}

static inline RowsIO rows_io(const DevConsts& dc, uint64_t* base, int p0, int period) {
    return RowsIO{base, dc.logn, p0, period};
}

// Standalone NTT of plain rows with a chosen radix split for rings above 2^lb:
// a column pass of logn - lb stages (forward: first; inverse: last) and block
// kernels of 2^lb points, lb in 12..14 (0: the built-in shapes of ntt_fwd/inv).
template <int RC, int LB>
static void ntt_rows_split(const DevConsts& dc, RowsIO io, int rows, bool fwd, cudaStream_t st) {
    const size_t total = (size_t)rows << LB;
    if (fwd) {
        ntt_fwd_col_kernel<RC, RowsIO, RowsIO><<<stride_blocks(total, 256), 256, 0, st>>>(io, io, dc.tw_fwd, dc.mods,
                                                                                      dc.logn, total);
        launch_fwd_block<LB, RowsIO, RowsIO, true>(dc, io, io, rows, dc.logn, st);
    } else {
        launch_inv_block<LB, RowsIO, RowsIO, false>(dc, io, io, rows, dc.logn, st);
        ntt_inv_col_kernel<RC, RowsIO, RowsIO><<<stride_blocks(total, 256), 256, 0, st>>>(io, io, dc.tw_inv, dc.mods,
                                                                                      dc.logn, total);
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

// bucketed MAX template dispatch for per-coefficient kernels
#define DISPATCH_MAXQ(nq, MACRO) \
    do {                         \
        if ((nq) <= 8) { MACRO(8); }       \
        else if ((nq) <= 16) { MACRO(16); } \
        else if ((nq) <= 24) { MACRO(24); } \
        else { MACRO(33); }                 \
    } while (0)

static void launch_bconv(const DevConsts& dc, const BconvTables& tb, const uint64_t* in, uint64_t* out, int polys,
                         size_t in_stride, size_t out_stride, cudaStream_t st) {
    if (polys <= 0) return;
    const int threads = 256;
    dim3 grid((unsigned)((1u << dc.logn) / threads), (unsigned)polys);
    const size_t sh = (size_t)tb.nin * tb.nout * 8;
#define L_BC(M) bconv_kernel<M><<<grid, threads, sh, st>>>(tb, in, out, dc.logn, in_stride, out_stride)
    DISPATCH_MAXQ(tb.nin, L_BC);
#undef L_BC
    check_launch("bconv");
}

// ===========================================================================
// scratch
// ===========================================================================
static uint8_t* ensure_scratch(Context& c, size_t bytes) {
    if (bytes > c.scratch_bytes) {
        if (c.scratch) {
            KB_CHECK_CUDA(cudaDeviceSynchronize());
            KB_CHECK_CUDA(cudaFree(c.scratch));
            c.scratch = nullptr;
            c.scratch_bytes = 0;
        }
        size_t want = std::max(bytes, (size_t)64 << 20);
        KB_CHECK_CUDA(cudaMalloc(&c.scratch, want));
        c.scratch_bytes = want;
    }
    return (uint8_t*)c.scratch;
}

// ===========================================================================
// multiply pipeline (HPS tensor + hybrid key switch), batched
// ===========================================================================
constexpr int kMaxBatch = 128;  // pointer tables ride in kernel parameters
struct PtrBatch {
    const uint64_t* a[kMaxBatch];
    const uint64_t* b[kMaxBatch];
    uint64_t* o[kMaxBatch];
};

struct MulScratch {
    uint64_t *sa, *sb, *sc, *sd, *sd2, *se;
    uint64_t *st1, *st2;  // T-base key switch: digits [item][nqj][nt], products [item][2][nri][nt]
    size_t bytes;
};

static MulScratch mul_scratch_layout(const Context& c, int count, uint8_t* base) {
    const size_t limb = c.n * 8;
    const int npq = c.nq + c.np, nqr = c.nq + c.nr;
    size_t off = 0;
    MulScratch m{};
    auto take = [&](size_t limbs) {
        uint64_t* p = (uint64_t*)(base ? base + off : nullptr);
        off += limbs * limb;
        return p;
    };
    m.sa = take((size_t)count * 4 * c.nq);
    m.sb = take((size_t)count * 4 * c.nr);
    m.sc = take((size_t)count * 3 * nqr);
    m.sd = take((size_t)count * 2 * c.nq);
    m.sd2 = take((size_t)count * c.dnum * npq);
    m.se = take((size_t)count * 2 * npq);
    if (c.klss_ok) {
        m.st1 = take((size_t)count * c.kc.nqj * c.nt);
        m.st2 = take((size_t)count * 2 * c.kc.nri * c.nt);
    }
    m.bytes = off;
    return m;
}

// Pointer arrays must be device-readable: the batched entry points pass
// PtrBatch by value as a kernel parameter, so functors point into it through
// this wrapper kernel-parameter view.
struct PairQRowsP {
    PtrBatch pb;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const int item = row / (4 * nq), w = row % (4 * nq), p = w / nq, l = w % nq;
        const uint64_t* base = p < 2 ? pb.a[item] : pb.b[item];
        return PtrRow{const_cast<uint64_t*>(base) + (((size_t)(p & 1) * nq + l) << logn)};
    }
};

// rows of consecutive Q|R polynomials; limb l of Q|R uses prime l (Q) or idx_r + l - nq (R)
struct QRRowsIO {
    uint64_t* base;
    int logn, nq, nqr, idx_r;
    __device__ __forceinline__ int prime(int row) const {
        const int l = row % nqr;
        return l < nq ? l : idx_r + (l - nq);
    }
    __device__ __forceinline__ PtrRow bind(int row) const { return PtrRow{base + ((size_t)row << logn)}; }
};

// K4 source: tensor product of the pair at limb l of Q|R, one of three outputs
struct TensorRow {
    const uint64_t *a1, *b1, *a2, *b2;
    int k;
    uint64_t q, mh, ml;  // mh: barrett_prod constant (inputs are fully reduced)
    __device__ __forceinline__ uint64_t load(int j) const {
        if (k == 0) return mul_mod_prod(a1[j], a2[j], q, mh);
        if (k == 2) return mul_mod_prod(b1[j], b2[j], q, mh);
        u128 acc = mul_wide(a1[j], b2[j]);
        mac(acc, b1[j], a2[j]);  // < 2 q^2
        return barrett_prod(acc, q, mh);
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct TensorSrc {
    PtrBatch pb;
    const uint64_t* sb;  // NTT-form R limbs: [item][4][nr]
    DevConsts dc;
    __device__ __forceinline__ int prime(int row) const {
        const int l = row % dc.nqr;
        return l < dc.nq ? l : dc.idx_r + (l - dc.nq);
    }
    __device__ __forceinline__ TensorRow bind(int row) const {
        const int nqr = dc.nqr, nq = dc.nq, nr = dc.nr, logn = dc.logn;
        const int item = row / (3 * nqr), w = row % (3 * nqr), k = w / nqr, l = w % nqr;
        TensorRow t;
        t.k = k;
        const int pi = l < nq ? l : dc.idx_r + (l - nq);
        t.q = dc.mods[pi]; t.mh = dc.mu_prod[pi]; t.ml = 0;
        if (l < nq) {
            const uint64_t* A = pb.a[item];
            const uint64_t* B = pb.b[item];
            t.a1 = A + ((size_t)l << logn); t.b1 = A + ((size_t)(nq + l) << logn);
            t.a2 = B + ((size_t)l << logn); t.b2 = B + ((size_t)(nq + l) << logn);
        } else {
            const int r = l - nq;
            const uint64_t* base = sb + (((size_t)item * 4 * nr) << logn);
            t.a1 = base + ((size_t)(0 * nr + r) << logn); t.b1 = base + ((size_t)(1 * nr + r) << logn);
            t.a2 = base + ((size_t)(2 * nr + r) << logn); t.b2 = base + ((size_t)(3 * nr + r) << logn);
        }
        return t;
    }
};

// K6b source: inner product with the relinearisation key over Q|P
struct KeyIPRow {
    const uint64_t* dig;  // limb m of digit 0 (digit stride ds)
    const uint64_t* key;  // limb m, half h of digit 0 (digit stride ks)
    size_t ds, ks;
    int dnum;
    uint64_t q, mh, ml, mp;
    __device__ __forceinline__ uint64_t load(int j) const {
        if (dnum == 1) return mul_mod_prod(dig[j], key[j], q, mp);  // digits fully reduced
        u128 acc{0, 0};
        for (int d = 0; d < dnum; d++) mac(acc, dig[d * ds + j], key[d * ks + j]);
        return barrett128(acc, q, mh, ml);
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct KeyIPSrc {
    const uint64_t* sd2;  // [item][ndig][npq]
    const uint64_t* rlk;  // [ndig][2][npq]
    DevConsts dc;
    int ndig;             // digits: dnum (hybrid) or q_count * pieces (gadget)
    int m0 = 0, nm = 0;   // rows cover limbs m0 .. m0+nm-1 of Q|P (nm = 0: all of Q|P)
    __device__ __forceinline__ int prime(int row) const { return m0 + row % (nm ? nm : dc.npq); }
    __device__ __forceinline__ KeyIPRow bind(int row) const {
        const int npq = dc.npq, logn = dc.logn, per = nm ? nm : npq;
        const int item = row / (2 * per), w = row % (2 * per), h = w / per, m = m0 + w % per;
        KeyIPRow r;
        r.dig = sd2 + (((size_t)item * ndig * npq + m) << logn);
        // key limbs: [digit][a|b][Q|P] of the top level; a level reads its live Q limbs and P
        const int km = m < dc.nq ? m : dc.key_nq + (m - dc.nq);
        r.key = rlk + (((size_t)h * dc.key_npq + km) << logn);
        r.ds = (size_t)npq << logn;
        r.ks = (size_t)2 * dc.key_npq << logn;
        r.dnum = ndig;
        r.q = dc.mods[m]; r.mh = dc.mu_hi[m]; r.ml = dc.mu_lo[m]; r.mp = dc.mu_prod[m];
        return r;
    }
};

// Gadget decomposition source: rows (item, digit g = i*J + j, m) -> the j-th
// w-bit piece of limb i of a1*a2 (coefficient form), the same small integer in
// every prime m of Q|P.
struct GadgetRow {
    const uint64_t* x;
    int shift;
    uint64_t mask;
    __device__ __forceinline__ uint64_t load(int j) const { return (x[j] >> shift) & mask; }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct GadgetDigitSrc {
    const uint64_t* sd2;  // [item][nq]
    DevConsts dc;
    int pieces, w;
    __device__ __forceinline__ int prime(int row) const { return row % dc.npq; }
    __device__ __forceinline__ GadgetRow bind(int row) const {
        const int ndig = dc.nq * pieces;
        const int item = row / (ndig * dc.npq), g = (row / dc.npq) % ndig;
        GadgetRow r;
        r.x = sd2 + (((size_t)item * dc.nq + g / pieces) << dc.logn);
        r.shift = w * (g % pieces);
        r.mask = (w >= 64) ? ~0ULL : (((uint64_t)1 << w) - 1);
        return r;
    }
};

// K7 source: mod down P|Q -> q_l and add the tensor term (coefficient form)
struct ModDownAddRow {
    const uint64_t* x;    // limb l of the Q|P polynomial, or null (Q part added in the NTT domain)
    const uint64_t* xp;   // limb 0 of its P part
    const uint64_t* add;  // limb l of the term to add, or null
    const uint64_t* pmods;
    const uint64_t* phatinv;
    const uint64_t* phatinvs;
    const uint64_t* phat;  // row l of (P/p_k) mod q_l
    size_t limb;
    int np;
    uint64_t q, mh, ml, pinv, pinvs;
    __device__ __forceinline__ uint64_t load(int j) const {
        uint64_t conv;
        if (np == 1) {
            conv = barrett64(xp[j], q, mh);
        } else {
            u128 acc{0, 0};
            for (int kk = 0; kk < np; kk++) {
                uint64_t rb = shoup(xp[kk * limb + j], phatinv[kk], phatinvs[kk], pmods[kk]);
                mac(acc, rb, phat[kk]);
            }
            conv = barrett128(acc, q, mh, ml);
        }
        uint64_t v = shoup(q - conv + (x ? x[j] : 0), pinv, pinvs, q);
        if (add) v = add_mod(v, add[j], q);
        return v;
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct ModDownAddSrc {
    const uint64_t* se;   // [item][2][npq]
    const uint64_t* sd;   // [item][2][nq] or null
    DevConsts dc;
    bool p_only = false;  // se holds only the P limbs (OutCtKeyDst adds the Q part)
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ ModDownAddRow bind(int row) const {
        const int nq = dc.nq, npq = dc.npq, logn = dc.logn;
        const int item = row / (2 * nq), w = row % (2 * nq), h = w / nq, l = w % nq;
        ModDownAddRow r;
        const uint64_t* poly = se + (((size_t)item * 2 + h) * npq << logn);
        r.x = p_only ? nullptr : poly + ((size_t)l << logn);
        r.xp = poly + ((size_t)nq << logn);
        r.add = sd ? sd + (((size_t)(item * 2 + h) * nq + l) << logn) : nullptr;
        r.pmods = dc.mods + dc.idx_p;
        r.phatinv = dc.phatinv_p;
        r.phatinvs = dc.phatinv_ps;
        r.phat = dc.phat_mod_q + (size_t)l * dc.np;
        r.limb = (size_t)1 << logn;
        r.np = dc.np;
        r.q = dc.mods[l]; r.mh = dc.mu_hi[l]; r.ml = dc.mu_lo[l];
        r.pinv = dc.pinv_q[l]; r.pinvs = dc.pinv_qs[l];
        return r;
    }
};

// ModDownAddSrc for one special prime: [x_P]_q is x_P mod q, so the row needs
// no conversion tables (fewer live registers in the transform's first pass)
struct ModDownAdd1Row {
    const uint64_t* x;    // limb l of the Q|P polynomial, or null
    const uint64_t* xp;   // its P limb
    const uint64_t* add;  // limb l of the term to add, or null
    uint64_t q, mh, pinv, pinvs;
    __device__ __forceinline__ uint64_t load(int j) const {
        const uint64_t conv = barrett64(xp[j], q, mh);
        uint64_t v = shoup(q - conv + (x ? x[j] : 0), pinv, pinvs, q);
        if (add) v = add_mod(v, add[j], q);
        return v;
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct ModDownAdd1Src {
    const uint64_t* se;   // [item][2][npq]
    const uint64_t* sd;   // [item][2][nq] or null
    DevConsts dc;
    bool p_only = false;
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ ModDownAdd1Row bind(int row) const {
        const int nq = dc.nq, npq = dc.npq, logn = dc.logn;
        const int item = row / (2 * nq), w = row % (2 * nq), h = w / nq, l = w % nq;
        const uint64_t* poly = se + (((size_t)item * 2 + h) * npq << logn);
        ModDownAdd1Row r;
        r.x = p_only ? nullptr : poly + ((size_t)l << logn);
        r.xp = poly + ((size_t)nq << logn);
        r.add = sd ? sd + (((size_t)(item * 2 + h) * nq + l) << logn) : nullptr;
        r.q = dc.mods[l]; r.mh = dc.mu_hi[l];
        r.pinv = dc.pinv_q[l]; r.pinvs = dc.pinv_qs[l];
        return r;
    }
};

struct OutCtDst {  // rows: (item, h, l) -> out[item] + (h*nq + l)*N
    PtrBatch pb;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const int item = row / (2 * nq), w = row % (2 * nq);
        return PtrRow{pb.o[item] + ((size_t)w << logn)};
    }
};

// rows (item, h, k) -> limb nq + k (P part) of se ([item][2][npq])
struct SeRowsP {
    uint64_t* se;
    int logn, nq, np, npq;
    __device__ __forceinline__ int prime(int row) const { return nq + row % np; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const int item = row / (2 * np), w = row % (2 * np), h = w / np, k = w % np;
        return PtrRow{se + (((size_t)(item * 2 + h) * npq + nq + k) << logn)};
    }
};

// Output store of the key-switch tail: adds P^-1 * sum_d digit_d * key_d[h] at
// limb l of Q (all NTT form, fully reduced) to the transformed value.
struct OutKeyRow {
    uint64_t* p;
    const uint64_t* dig;  // limb l of digit 0, digit stride ds
    const uint64_t* key;  // limb l of half h of digit 0, digit stride ks
    size_t ds, ks;
    int ndig;
    uint64_t q, mh, ml, mp, pinv, pinvs;
    __device__ __forceinline__ uint64_t load(int j) const { return p[j]; }
    __device__ __forceinline__ void store(int j, uint64_t v) const {
        uint64_t ip;
        if (ndig == 1) {
            ip = mul_mod_prod(dig[j], key[j], q, mp);
        } else {
            u128 acc{0, 0};
            for (int d = 0; d < ndig; d++) mac(acc, dig[d * ds + j], key[d * ks + j]);
            ip = barrett128(acc, q, mh, ml);
        }
        p[j] = add_mod(v, shoup(ip, pinv, pinvs, q), q);
    }
};
struct OutCtKeyDst {  // rows: (item, h, l) -> out[item] + (h*nq + l)*N
    PtrBatch pb;
    const uint64_t* sd2;  // NTT-form digits [item][ndig][npq]
    const uint64_t* rlk;  // [ndig][2][Q|P] of the top level
    DevConsts dc;
    int ndig;
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ OutKeyRow bind(int row) const {
        const int nq = dc.nq, logn = dc.logn;
        const int item = row / (2 * nq), w = row % (2 * nq), h = w / nq, l = w % nq;
        OutKeyRow r;
        r.p = pb.o[item] + ((size_t)w << logn);
        r.dig = sd2 + (((size_t)item * ndig * dc.npq + l) << logn);
        r.key = rlk + (((size_t)h * dc.key_npq + l) << logn);
        r.ds = (size_t)dc.npq << logn;
        r.ks = (size_t)2 * dc.key_npq << logn;
        r.ndig = ndig;
        r.q = dc.mods[l]; r.mh = dc.mu_hi[l]; r.ml = dc.mu_lo[l]; r.mp = dc.mu_prod[l];
        r.pinv = dc.pinv_q[l]; r.pinvs = dc.pinv_qs[l];
        return r;
    }
};
// the column pass of a split transform writes plain values; only the block
// kernel's final store runs the epilogue
static inline OutCtDst plain_of(const OutCtKeyDst& d) { return OutCtDst{d.pb, d.dc.logn, d.dc.nq}; }

// K5 in one kernel, for launches of one or two pairs (one launch less on the
// per-call path): scale-and-round to R, R -> Q, and (mode 1) the key-switch
// lift of a1*a2.
// mode 0: all three outputs over Q to out0 ([item][3][nq]).
// mode 1: a1*a2 lifted into sd2 ([item][dnum][npq]); cross, b1*b2 to sd ([item][2][nq]).
// mode 2: a1*a2 over Q into sd2 ([item][nq]); cross, b1*b2 to sd (T-base key switch).
template <int MAXQ>
__global__ void k5_round_kernel(DevConsts c, const uint64_t* __restrict__ sc, uint64_t* __restrict__ out0,
                                uint64_t* __restrict__ sd, uint64_t* __restrict__ sd2, int mode) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int poly = blockIdx.y, item = poly / 3, which = poly % 3;
    const uint64_t* src = sc + ((size_t)poly * c.nqr << c.logn);
    uint64_t xq[MAXQ], xr[MAXQ + 1], rr[MAXQ + 1];
#pragma unroll
    for (int i = 0; i < MAXQ; i++)
        if (i < c.nq) xq[i] = src[((size_t)i << c.logn) + k];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) xr[j] = src[((size_t)(c.nq + j) << c.logn) + k];
    scale_round_coeff<MAXQ>(c, xq, xr, rr);
    // R -> Q
    const BconvTables tb = r2q_tables(c);
    uint64_t y[MAXQ + 1];
    const long long v = bconv_prep<MAXQ + 1>(y, rr, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
#pragma unroll
    for (int i = 0; i < MAXQ; i++) {
        if (i < c.nq)
            xq[i] = bconv_out<MAXQ + 1>(y, tb.nin, tb.hat + (size_t)i * tb.nin, tb.alpha[v * tb.nout + i],
                                        c.mods[i], c.mu_hi[i], c.mu_lo[i]);
    }
    if (mode == 0) {
        uint64_t* dst = out0 + ((size_t)poly * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    } else if (which == 0 && mode == 2) {  // a1*a2 over Q, coefficient form, to sd2 ([item][nq])
        uint64_t* dst = sd2 + ((size_t)item * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    } else if (which == 0) {
        modup_coeff<MAXQ>(c, xq, sd2 + ((size_t)item * c.dnum * c.npq << c.logn), k);
    } else {
        uint64_t* dst = sd + (((size_t)item * 2 + (which - 1)) * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    }
}

// K5, in two kernels so that each holds fewer registers (more warps per SM):
// K5a: t/Q scale-and-round Q|R -> R of each tensor polynomial into rr ([poly][nr]).
template <int MAXQ>
__global__ void k5_scale_kernel(DevConsts c, const uint64_t* __restrict__ sc, uint64_t* __restrict__ rr_out) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int poly = blockIdx.y;
    const uint64_t* src = sc + ((size_t)poly * c.nqr << c.logn);
    uint64_t xq[MAXQ], xr[MAXQ + 1], rr[MAXQ + 1];
#pragma unroll
    for (int i = 0; i < MAXQ; i++)
        if (i < c.nq) xq[i] = src[((size_t)i << c.logn) + k];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) xr[j] = src[((size_t)(c.nq + j) << c.logn) + k];
    scale_round_coeff<MAXQ>(c, xq, xr, rr);
    uint64_t* dst = rr_out + ((size_t)poly * c.nr << c.logn);
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) dst[((size_t)j << c.logn) + k] = rr[j];
}

// K5b: R -> Q, and (mode 1) the key-switch lift of a1*a2.
// mode 0: all three outputs over Q to out0 ([item][3][nq]).
// mode 1: a1*a2 lifted into sd2 ([item][dnum][npq]); cross, b1*b2 to sd ([item][2][nq]).
// mode 2: a1*a2 over Q into sd2 ([item][nq]); cross, b1*b2 to sd (T-base key switch).
template <int MAXQ>
__global__ void k5_lift_kernel(DevConsts c, const uint64_t* __restrict__ rr_in, uint64_t* __restrict__ out0,
                               uint64_t* __restrict__ sd, uint64_t* __restrict__ sd2, int mode) {
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int poly = blockIdx.y, item = poly / 3, which = poly % 3;
    const uint64_t* src = rr_in + ((size_t)poly * c.nr << c.logn);
    uint64_t rr[MAXQ + 1], xq[MAXQ];
#pragma unroll
    for (int j = 0; j < MAXQ + 1; j++)
        if (j < c.nr) rr[j] = src[((size_t)j << c.logn) + k];
    const BconvTables tb = r2q_tables(c);
    uint64_t y[MAXQ + 1];
    const long long v = bconv_prep<MAXQ + 1>(y, rr, tb.nin, tb.in_mods, tb.hatinv, tb.hatinvs, tb.binv);
#pragma unroll
    for (int i = 0; i < MAXQ; i++) {
        if (i < c.nq)
            xq[i] = bconv_out<MAXQ + 1>(y, tb.nin, tb.hat + (size_t)i * tb.nin, tb.alpha[v * tb.nout + i],
                                        c.mods[i], c.mu_hi[i], c.mu_lo[i]);
    }
    if (mode == 0) {
        uint64_t* dst = out0 + ((size_t)poly * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    } else if (which == 0 && mode == 2) {  // a1*a2 over Q, coefficient form, to sd2 ([item][nq])
        uint64_t* dst = sd2 + ((size_t)item * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    } else if (which == 0) {
        modup_coeff<MAXQ>(c, xq, sd2 + ((size_t)item * c.dnum * c.npq << c.logn), k);
    } else {
        uint64_t* dst = sd + (((size_t)item * 2 + (which - 1)) * c.nq << c.logn);
#pragma unroll
        for (int i = 0; i < MAXQ; i++)
            if (i < c.nq) dst[((size_t)i << c.logn) + k] = xq[i];
    }
}

// Key-switch tail over NTT-form digits (sd2, [item][ndig][npq]) and a key
// ([ndig][2][Q|P] of the top level), written to the outputs of pb:
//   out_h = add_h + P^-1 (x_h,Q - [x_h,P]_Q),  x_h = sum_d digit_d * key_d[h].
// Only the P limbs of x are brought back to coefficient form (inverse NTT over
// P, the key product fused into its loads) for the conversion to Q. The Q limbs
// stay in the NTT domain, where the forward NTT's store adds them:
//   NTT(add - P^-1 [x_P]_Q) + P^-1 x_Q,  with x_Q computed at the store.
static void ks_tail(const DevConsts& dc, const uint64_t* sd2, const uint64_t* key, int ndig, uint64_t* se,
                    const uint64_t* add, const PtrBatch& pb, int count, cudaStream_t st) {
    ntt_inv(dc, KeyIPSrc{sd2, key, dc, ndig, dc.nq, dc.np}, SeRowsP{se, dc.logn, dc.nq, dc.np, dc.npq},
            count * 2 * dc.np, st);
    const OutCtKeyDst dst{pb, sd2, key, dc, ndig};
    if (dc.np == 1)
        ntt_fwd(dc, ModDownAdd1Src{se, add, dc, true}, dst, count * 2 * dc.nq, st);
    else
        ntt_fwd(dc, ModDownAddSrc{se, add, dc, true}, dst, count * 2 * dc.nq, st);
}

// INTT over Q of the four input polynomials, Q -> R, NTT over R, fused tensor +
// INTT over Q|R: steps shared by kbfv_mul and the fused multiply-relinearise.
static void mul_front(Context& c, const PtrBatch& pb, int count, const MulScratch& m, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    // K1: INTT over Q of [a1, b1, a2, b2]
    ntt_inv(dc, PairQRowsP{pb, dc.logn, dc.nq}, rows_io(dc, m.sa, 0, dc.nq), count * 4 * dc.nq, st);
    // K2: Q -> R (centred)
    launch_bconv(dc, q2r_tables(dc), m.sa, m.sb, count * 4, (size_t)dc.nq << dc.logn, (size_t)dc.nr << dc.logn, st);
    // K3: NTT over R in place, fully reduced (the tensor's products use barrett_prod)
    ntt_fwd<RowsIO, RowsIO, true>(dc, rows_io(dc, m.sb, dc.idx_r, dc.nr), rows_io(dc, m.sb, dc.idx_r, dc.nr),
                                   count * 4 * dc.nr, st);
    // K4: tensor (Q part from the NTT-form inputs, R part from K3) fused into INTT over Q|R
    TensorSrc ts{pb, m.sb, dc};
    ntt_inv(dc, ts, QRRowsIO{m.sc, dc.logn, dc.nq, dc.nqr, dc.idx_r}, count * 3 * dc.nqr, st);
}

static void k5_launch(Context& c, int count, const MulScratch& m, uint64_t* out0, int mode, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    const int threads = 128;
    dim3 grid((unsigned)(c.n / threads), (unsigned)(count * 3));
    // the R limbs of the inputs (m.sb, 4 x nr limbs per pair) are dead after K4:
    // they hold the scale-and-round results (3 x nr limbs per pair)
#define L_K5(M)                                                                            \
    do {                                                                                   \
        if (count <= 2) {                                                                  \
            k5_round_kernel<M><<<grid, threads, 0, st>>>(dc, m.sc, out0, m.sd, m.sd2, mode); \
        } else {                                                                           \
            k5_scale_kernel<M><<<grid, threads, 0, st>>>(dc, m.sc, m.sb);                  \
            k5_lift_kernel<M><<<grid, threads, 0, st>>>(dc, m.sb, out0, m.sd, m.sd2, mode); \
        }                                                                                  \
    } while (0)
    DISPATCH_MAXQ(dc.nq + 1, L_K5);
#undef L_K5
    check_launch("k5_round");
}

static void mul_relin_chunk(Context& c, const uint64_t* rlk, const PtrBatch& pb, int count, const MulScratch& m,
                            cudaStream_t st) {
    const DevConsts& dc = c.dc;
    mul_front(c, pb, count, m, st);
    k5_launch(c, count, m, nullptr, 1, st);
    // K6a: NTT over Q|P of the lifted digits, in place, fully reduced (key product uses barrett_prod)
    ntt_fwd<RowsIO, RowsIO, true>(dc, rows_io(dc, m.sd2, 0, dc.npq), rows_io(dc, m.sd2, 0, dc.npq),
                                   count * dc.dnum * dc.npq, st);
    // K6b: key product over P fused into INTT over P; K7: mod down + add (cross |
    // b1b2) fused into NTT over Q, the key product over Q added at its store
    ks_tail(dc, m.sd2, rlk, dc.dnum, m.se, m.sd, pb, count, st);
}

// rows (item, limb) of the first polynomial of consecutive 3-polynomial tensors
struct TensorA2 {
    const uint64_t* tz;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        const int item = row / nq, l = row % nq;
        return PtrRow{const_cast<uint64_t*>(tz) + (((size_t)item * 3 * nq + l) << logn)};
    }
};

// Fused stages run as one block kernel for N <= 2^14; for split transforms
// (N = 2^15, 2^16, and launches of few rows at 2^14) the fused loader feeds
// the column pass and the store target is read back by the block kernel, which
// every functor here supports.
static void require_batchable(const Context& c) {
    KB_REQUIRE(c.logn >= 10 && c.logn <= 16, KBFV_ERR_UNSUPPORTED, "ring degree outside 2^10..2^16");
}

// T-base key switch (the reference's KLSS, include/KeySwitch_23.cuh:244-330) of
// a1*a2 given in coefficient form over Q (sd2, [item][nq]); writes the P|Q
// results into se ([item][2][npq]).
static void klss_keyswitch(Context& c, const uint64_t* rlk_t, int count, const MulScratch& m, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    const KlssConsts& kc = c.kc;
    // Qj blocks -> T (modUpQjtoT_23)
    klss_block_to_t_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)kc.nqj, (unsigned)count), 128, 0, st>>>(
        dc, kc, m.sd2, m.st1, 0, (size_t)c.nq << c.logn, (size_t)kc.nqj * c.nt << c.logn);
    check_launch("klss_qj_to_t");
    // NTT over T
    ntt_fwd<RowsIO, RowsIO, true>(dc, rows_io(dc, m.st1, dc.idx_t, c.nt), rows_io(dc, m.st1, dc.idx_t, c.nt),
                                   count * kc.nqj * c.nt, st);
    // external product over T fused into INTT over T (external_product_T)
    ntt_inv(dc, ExtProdSrc{m.st1, rlk_t, dc, c.nt, kc.nri, kc.nqj, kc.nqj}, rows_io(dc, m.st2, dc.idx_t, c.nt),
            count * 2 * kc.nri * c.nt, st);
    // centred T -> P|Q (modUpTtoPQl_23)
    klss_t_to_pq_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)kc.nri, (unsigned)(count * 2)), 128, 0, st>>>(
        dc, kc, m.st2, m.se);
    check_launch("klss_t_to_pq");
}

static void mul_relin_klss_chunk(Context& c, const uint64_t* rlk_t, const PtrBatch& pb, int count,
                                 const MulScratch& m, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    mul_front(c, pb, count, m, st);
    k5_launch(c, count, m, nullptr, 2, st);
    klss_keyswitch(c, rlk_t, count, m, st);
    ntt_fwd(dc, ModDownAddSrc{m.se, m.sd, dc}, OutCtDst{pb, dc.logn, dc.nq}, count * 2 * dc.nq, st);
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

static void require_top(const Context& c) {
    KB_REQUIRE(!c.parent, KBFV_ERR_LEVEL, "keys and encryptions are made on the top-level context");
}

// ---- modulus switch (divide by the last prime and round) ---------------------
struct LastLimbSrc {  // row = polynomial: its last limb
    const uint64_t* ct;
    int logn, nq;
    __device__ __forceinline__ int prime(int) const { return nq - 1; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        return PtrRow{const_cast<uint64_t*>(ct) + (((size_t)row * nq + nq - 1) << logn)};
    }
};
struct ModSwitchRow {
    const uint64_t* last;
    uint64_t ql, half, q, mh, half_i;
    // [x + floor(ql/2)]_ql - floor(ql/2), taken mod q_i: the rounding correction
    __device__ __forceinline__ uint64_t load(int j) const {
        const uint64_t x = csub(last[j] + half, ql);
        return sub_mod(barrett64(x, q, mh), half_i, q);
    }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct ModSwitchSrc {  // rows (poly, i < nq-1)
    const uint64_t* last;  // [poly][N], coefficient form, < q_last
    DevConsts dc;
    __device__ __forceinline__ int prime(int row) const { return row % (dc.nq - 1); }
    __device__ __forceinline__ ModSwitchRow bind(int row) const {
        const int nout = dc.nq - 1, poly = row / nout, i = row % nout;
        ModSwitchRow r;
        r.last = last + ((size_t)poly << dc.logn);
        r.ql = dc.mods[dc.nq - 1];
        r.half = dc.ms_half;
        r.q = dc.mods[i]; r.mh = dc.mu_hi[i];
        r.half_i = dc.ms_half_mod[i];
        return r;
    }
};
// out[poly][i] = (ct[poly][i] - corr[poly][i]) * q_last^-1 mod q_i
__global__ void mod_switch_combine_kernel(DevConsts c, const uint64_t* __restrict__ ct,
                                          const uint64_t* __restrict__ corr, uint64_t* __restrict__ out,
                                          size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int nout = c.nq - 1;
    const size_t row = i >> c.logn, j = i & (((size_t)1 << c.logn) - 1);
    const size_t poly = row / nout;
    const int l = (int)(row % nout);
    const uint64_t q = c.mods[l];
    const uint64_t x = ct[((poly * c.nq + l) << c.logn) + j];
    out[i] = shoup(x + q - corr[i], c.ms_qlinv[l], c.ms_qlinvs[l], q);
}

// rows (item, l) of the a-part of ciphertexts, read through the Galois permutation
struct GaloisRow {
    const uint64_t* p;
    uint64_t g;
    int logn;
    __device__ __forceinline__ uint64_t load(int j) const { return p[galois_perm((uint32_t)j, g, logn)]; }
    __device__ __forceinline__ void store(int, uint64_t) const {}
};
struct GaloisASrc {
    const uint64_t* ct;  // [item][a|b][nq]
    uint64_t g;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ GaloisRow bind(int row) const {
        const int item = row / nq, l = row % nq;
        return GaloisRow{ct + (((size_t)item * 2 * nq + l) << logn), g, logn};
    }
};

// ---- pointer-table variants of encryption, decryption and addition ----------
// delta * m of item i (plaintext pb.a[i]) into its work slot
__global__ void delta_m_ptr_kernel(DevConsts c, PtrBatch pb, uint64_t* __restrict__ work, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const size_t lq = (size_t)c.nq << c.logn;
    const size_t item = i / lq, w = i % lq;
    const int l = (int)(w >> c.logn);
    const uint64_t mv = pb.a[item][w & (((size_t)1 << c.logn) - 1)];
    const uint64_t mq = shoup(mv, c.negq_mod_t, c.negq_mod_t_s, c.t);
    work[item * 4 * lq + 3 * lq + w] = shoup(mq, c.tinv_q[l], c.tinv_qs[l], c.mods[l]);
}
__global__ void enc_combine_ptr_kernel(DevConsts c, const uint64_t* __restrict__ pk, const uint64_t* __restrict__ work,
                                       PtrBatch pb, size_t total) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const size_t lq = (size_t)c.nq << c.logn;
    const size_t item = i / lq, w = i % lq;
    const int l = (int)(w >> c.logn);
    const uint64_t q = c.mods[l], mh = c.mu_hi[l], ml = c.mu_lo[l];
    const uint64_t* wk = work + item * 4 * lq;
    const uint64_t v = wk[w], e0 = wk[lq + w], e1 = wk[2 * lq + w], dm = wk[3 * lq + w];
    uint64_t* ct = pb.o[item];
    ct[w] = add_mod(mul_mod(v, pk[w], q, mh, ml), e0, q);
    ct[lq + w] = add_mod(add_mod(mul_mod(v, pk[lq + w], q, mh, ml), e1, q), dm, q);
}
// x = pb.a[item], y = pb.b[item], out = pb.o[item]: 2 x nq limbs each; grid.y = item
__global__ void add_ptr_kernel(DevConsts c, PtrBatch pb, size_t per_item) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= per_item) return;
    const int item = blockIdx.y;
    const int l = (int)((i >> c.logn) % c.nq);
    pb.o[item][i] = add_mod(pb.a[item][i], pb.b[item][i], c.mods[l]);
}
// decryption source with ciphertexts at pb.a[item]
struct DecSrcP {
    PtrBatch pb;
    const uint64_t* sk;
    DevConsts dc;
    struct Row {
        const uint64_t *a, *b, *s;
        uint64_t q, mp;
        __device__ __forceinline__ uint64_t load(int j) const { return add_mod(mul_mod_prod(a[j], s[j], q, mp), b[j], q); }
        __device__ __forceinline__ void store(int, uint64_t) const {}
    };
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ Row bind(int row) const {
        const int item = row / dc.nq, l = row % dc.nq;
        Row r;
        r.a = pb.a[item] + ((size_t)l << dc.logn);
        r.b = r.a + ((size_t)dc.nq << dc.logn);
        r.s = sk + ((size_t)l << dc.logn);
        r.q = dc.mods[l];
        r.mp = dc.mu_prod[l];
        return r;
    }
};
template <int MAXQ>
__global__ void decrypt_round_ptr_kernel(DevConsts c, const uint64_t* __restrict__ in, PtrBatch pb) {
    // the rounding of decrypt_round_kernel, written to pb.o[item]
    const size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t* src = in + ((size_t)blockIdx.y * c.nq << c.logn);
    pb.o[blockIdx.y][k] = decrypt_round_coeff<MAXQ>(c, src, k);
}

// sub-batches of a batched multiply: one per `branches`, at least 8 pairs each
constexpr int kMinBranchPairs = 8;
static int branch_count(const Context& c, int cnt) {
    return std::max(1, std::min(c.branches, cnt / kMinBranchPairs));
}
static size_t branch_region_bytes(const Context& c, int per) {
    return (mul_scratch_layout(c, per, nullptr).bytes + 255) & ~(size_t)255;
}
static size_t mul_scratch_need(const Context& c, int cnt) {
    const int nb = branch_count(c, cnt);
    const size_t whole = mul_scratch_layout(c, cnt, nullptr).bytes;
    return nb == 1 ? whole : std::max(whole, branch_region_bytes(c, (cnt + nb - 1) / nb) * nb);
}
static void ensure_branch_streams(Context& c) {
    if (c.fork_ev) return;
    for (int i = 0; i < 3; i++) {
        KB_CHECK_CUDA(cudaStreamCreateWithFlags(&c.aux[i], cudaStreamNonBlocking));
        KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.join_ev[i], cudaEventDisableTiming));
    }
    KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.fork_ev, cudaEventDisableTiming));
}

static void require_klss(const Context& c) {
    KB_REQUIRE(c.klss_ok, KBFV_ERR_INVALID,
               "context has no T-base key switch (needs T primes, q_count divisible by p_count, dnum = q_count / p_count)");
}

// ---- arithmetic-rate probe: independent register chains of one primitive -------
// kind 0: 64x64->128 multiply-accumulate, 1: mul.lo.u64, 2: mul.hi.u64,
// 3: forward butterfly with the approximate-quotient Shoup product from 64-bit
// multiplies (shoup4_64), 4: fully reduced Shoup,
// 5: 128-bit Barrett, 6: one-high-product Barrett, 7: 32x32->64 multiply-add,
// 8: 32x32 high product, 9: 32-bit multiply-add, 10: mac32 (64x64->128
// multiply-accumulate from 32-bit partial products), 11: forward butterfly
// with shoup4_32 (the NTT kernels' butterfly).
constexpr int kProbeChains = 8;
template <int KIND>
__global__ void probe_arith_kernel(uint64_t* out, int iters, uint64_t q, uint64_t mh, uint64_t ml, uint64_t mp) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t a[kProbeChains], b[kProbeChains];
    u128 acc[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) {
        a[c] = (0x9E3779B97F4A7C15ULL * (uint64_t)(t * kProbeChains + c + 1)) % q;
        b[c] = (0xC2B2AE3D27D4EB4FULL * (uint64_t)(t * kProbeChains + c + 7)) % q;
        acc[c] = u128{0, 0};
    }
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int c = 0; c < kProbeChains; c++) {
            if (KIND == 0) mac64(acc[c], a[c], b[c]);
            if (KIND == 1) acc[c].lo += a[c] * b[c];
            if (KIND == 2) acc[c].lo += __umul64hi(a[c], b[c]);
            if (KIND == 3) {  // the butterfly with the Shoup product from 64-bit multiplies
                uint64_t x = a[c], y = b[c];
                const uint64_t v = shoup4_64(y, b[c], a[c], q);
                x = csub63(x, q << 2);
                y = x + (q << 2) - v;
                x = x + v;
                acc[c].lo += x ^ y;
            }
            if (KIND == 4) acc[c].lo += shoup(a[c], b[c], a[c] ^ b[c], q);
            if (KIND == 5) acc[c].lo += barrett128(u128{a[c], b[c] >> 4}, q, mh, ml);
            if (KIND == 6) acc[c].lo += barrett_prod(mul_wide(a[c], b[c]), q, mp);
            if (KIND == 7) acc[c].lo += (uint64_t)(uint32_t)a[c] * (uint32_t)b[c];
            if (KIND == 8) acc[c].lo += __umulhi((uint32_t)a[c], (uint32_t)b[c]);
            if (KIND == 9) acc[c].lo = (uint32_t)a[c] * (uint32_t)b[c] + (uint32_t)acc[c].lo;
            if (KIND == 10) mac32(acc[c], a[c], b[c]);
            if (KIND == 11) {  // the NTT kernels' butterfly (Shoup product from 32-bit multiplies)
                uint64_t x = a[c], y = b[c];
                ct_bfly(x, y, tw_t{b[c], a[c]}, q, q << 2);
                acc[c].lo += x ^ y;
            }
            a[c] = (a[c] + (acc[c].lo & 15)) & 0x0fffffffffffffffULL;
        }
    }
    uint64_t r = 0;
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) r ^= acc[c].lo ^ acc[c].hi ^ a[c];
    out[t] = r;
}

// ===========================================================================
// C ABI
// ===========================================================================
struct kbfv_context {
    Context c;
};

static Context& CX(kbfv_context* h) {
    if (!h) throw KbfvError(KBFV_ERR_INVALID, "null context");
    return h->c;
}

extern "C" {

const char* kbfv_last_error(void) { return g_last_error.c_str(); }
const char* kbfv_version(void) { return "kbfv-b200 0.1 (sm_100a)"; }

int kbfv_context_create(const kbfv_params* params, kbfv_context** out) {
    return guarded([&] {
        KB_REQUIRE(params && out, KBFV_ERR_INVALID, "null argument");
        auto* h = new kbfv_context();
        try {
            build_context(h->c, *params);
        } catch (...) {
            if (h->c.pool) cudaFree(h->c.pool);
            delete h;
            throw;
        }
        *out = h;
    });
}

int kbfv_context_create_reference(uint32_t log_n, kbfv_context** out) {
    return guarded([&] {
        // include/Params.cuh:31-145
        static const uint64_t q14[] = {0x7FFE28001ULL, 0x7FFF18001ULL, 0x7FFF80001ULL, 0x7FFFB0001ULL};
        static const uint64_t p14[] = {0xFFFFCA8001ULL, 0xFFFFE80001ULL};
        static const uint64_t t4[] = {0xffffffffffc0001ULL, 0xfffffffff840001ULL, 0xfffffffff6a0001ULL,
                                      0xfffffffff5a0001ULL};
        static const uint64_t q15[] = {36028797001138177ULL, 36028797003563009ULL, 36028797003694081ULL,
                                       36028797005135873ULL, 36028797005529089ULL, 36028797005856769ULL,
                                       36028797009985537ULL, 36028797010444289ULL, 36028797012606977ULL,
                                       36028797013000193ULL, 36028797013327873ULL, 36028797014376449ULL,
                                       36028797014573057ULL, 36028797014704129ULL, 36028797017456641ULL};
        static const uint64_t p15[] = {72057594037338113ULL};
        kbfv_params p{};
        p.log_n = log_n;
        if (log_n == 14) {
            p.plain_modulus = 23068673; p.q_count = 4; p.q = q14; p.p_count = 2; p.p = p14;
            p.dnum = 2; p.t_count = 4; p.t_primes = t4; p.gamma = 2;
        } else if (log_n == 15) {
            p.plain_modulus = 0xC0001; p.q_count = 15; p.q = q15; p.p_count = 1; p.p = p15;
            p.dnum = 15; p.t_count = 4; p.t_primes = t4; p.gamma = 4;
        } else {
            throw KbfvError(KBFV_ERR_PARAMS, "the reference defines parameter sets for logN 14 and 15 only");
        }
        int rc = kbfv_context_create(&p, out);
        if (rc != KBFV_OK) throw KbfvError(rc, g_last_error);
    });
}

int kbfv_context_destroy(kbfv_context* ctx) {
    return guarded([&] {
        if (!ctx) return;
        Context& c = ctx->c;
        cudaDeviceSynchronize();
        for (void* lv : c.levels)
            if (lv) kbfv_context_destroy((kbfv_context*)lv);
        if (c.pool) cudaFree(c.pool);
        if (c.scratch) cudaFree(c.scratch);
        if (c.ptrs_event) cudaEventDestroy(c.ptrs_event);
        for (int i = 0; i < 3; i++) {
            if (c.aux[i]) cudaStreamDestroy(c.aux[i]);
            if (c.join_ev[i]) cudaEventDestroy(c.join_ev[i]);
        }
        if (c.fork_ev) cudaEventDestroy(c.fork_ev);
        for (int i = 0; i < 4; i++) {
            if (c.hs[i]) cudaStreamDestroy(c.hs[i]);
            for (cudaEvent_t e : {c.hjoin[i], c.hin[i], c.hcomp[i], c.hout[i]})
                if (e) cudaEventDestroy(e);
        }
        if (c.hfork) cudaEventDestroy(c.hfork);
        for (int i = 0; i < 3; i++) {
            if (c.lane[i]) cudaStreamDestroy(c.lane[i]);
            if (c.lane_join[i]) cudaEventDestroy(c.lane_join[i]);
        }
        if (c.lane_fork) cudaEventDestroy(c.lane_fork);
        delete ctx;
    });
}

int kbfv_context_info(const kbfv_context* ctx, uint64_t* n, uint32_t* q_count, uint32_t* p_count, uint32_t* r_count,
                      uint32_t* t_count, uint32_t* dnum, uint32_t* alpha) {
    return guarded([&] {
        KB_REQUIRE(ctx, KBFV_ERR_INVALID, "null context");
        const Context& c = ctx->c;
        if (n) *n = c.n;
        if (q_count) *q_count = c.nq;
        if (p_count) *p_count = c.np;
        if (r_count) *r_count = c.nr;
        if (t_count) *t_count = c.nt;
        if (dnum) *dnum = c.dnum;
        if (alpha) *alpha = c.alpha;
    });
}

int kbfv_context_primes(const kbfv_context* ctx, uint64_t* primes, uint32_t* count) {
    return guarded([&] {
        KB_REQUIRE(ctx && count, KBFV_ERR_INVALID, "null argument");
        *count = (uint32_t)ctx->c.mods.size();
        if (primes) std::memcpy(primes, ctx->c.mods.data(), ctx->c.mods.size() * 8);
    });
}

uint64_t kbfv_context_plain_modulus(const kbfv_context* ctx) { return ctx ? ctx->c.t : 0; }
int kbfv_context_decrypt_variant(const kbfv_context* ctx) { return ctx ? ctx->c.dec_variant : -1; }

size_t kbfv_mul_relin_scratch_bytes(const kbfv_context* ctx, uint32_t count) {
    if (!ctx) return 0;
    return mul_scratch_need(ctx->c, (int)std::min<uint32_t>(count, kMaxBatch));
}

int kbfv_reserve(kbfv_context* ctx, uint32_t pairs) {
    return guarded([&] {
        Context& c = CX(ctx);
        std::lock_guard<std::mutex> lk(c.mu);
        const int chunk = (int)std::min<uint32_t>(std::max<uint32_t>(pairs, 1), kMaxBatch);
        size_t need = mul_scratch_need(c, chunk);
        // encryption work area: 4 polys x nq per item; secret/relin keygen: 2*(nq+np)
        need = std::max(need, (size_t)chunk * 4 * c.nq * c.n * 8);
        ensure_scratch(c, need);
    });
}

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

// ---- randomness helpers ----
static void hsalsa_host(const uint8_t key[32], const uint8_t nonce16[16], uint32_t out[8]);
static SalsaKey subkey_for(const uint8_t seed[32], uint32_t domain, uint32_t sub) {
    uint8_t n16[16] = {0};
    for (int i = 0; i < 4; i++) { n16[i] = (uint8_t)(domain >> (8 * i)); n16[4 + i] = (uint8_t)(sub >> (8 * i)); }
    SalsaKey k;
    hsalsa_host(seed, n16, k.k);
    static const char* sig = "expand 32-byte k";
    for (int i = 0; i < 4; i++) std::memcpy(&k.sigma[i], sig + 4 * i, 4);
    return k;
}

static inline uint32_t rl(uint32_t u, int c) { return (u << c) | (u >> (32 - c)); }
static inline uint32_t ld32(const uint8_t* x) {
    return (uint32_t)x[0] | ((uint32_t)x[1] << 8) | ((uint32_t)x[2] << 16) | ((uint32_t)x[3] << 24);
}
static void hsalsa_host(const uint8_t key[32], const uint8_t nonce16[16], uint32_t out[8]) {
    static const char* sig = "expand 32-byte k";
    uint32_t x[16];
    x[0] = ld32((const uint8_t*)sig); x[5] = ld32((const uint8_t*)sig + 4);
    x[10] = ld32((const uint8_t*)sig + 8); x[15] = ld32((const uint8_t*)sig + 12);
    for (int i = 0; i < 4; i++) { x[1 + i] = ld32(key + 4 * i); x[11 + i] = ld32(key + 16 + 4 * i); }
    for (int i = 0; i < 4; i++) x[6 + i] = ld32(nonce16 + 4 * i);
    for (int r = 0; r < 10; r++) {
        x[4] ^= rl(x[0] + x[12], 7);   x[8] ^= rl(x[4] + x[0], 9);
        x[12] ^= rl(x[8] + x[4], 13);  x[0] ^= rl(x[12] + x[8], 18);
        x[9] ^= rl(x[5] + x[1], 7);    x[13] ^= rl(x[9] + x[5], 9);
        x[1] ^= rl(x[13] + x[9], 13);  x[5] ^= rl(x[1] + x[13], 18);
        x[14] ^= rl(x[10] + x[6], 7);  x[2] ^= rl(x[14] + x[10], 9);
        x[6] ^= rl(x[2] + x[14], 13);  x[10] ^= rl(x[6] + x[2], 18);
        x[3] ^= rl(x[15] + x[11], 7);  x[7] ^= rl(x[3] + x[15], 9);
        x[11] ^= rl(x[7] + x[3], 13);  x[15] ^= rl(x[11] + x[7], 18);
        x[1] ^= rl(x[0] + x[3], 7);    x[2] ^= rl(x[1] + x[0], 9);
        x[3] ^= rl(x[2] + x[1], 13);   x[0] ^= rl(x[3] + x[2], 18);
        x[6] ^= rl(x[5] + x[4], 7);    x[7] ^= rl(x[6] + x[5], 9);
        x[4] ^= rl(x[7] + x[6], 13);   x[5] ^= rl(x[4] + x[7], 18);
        x[11] ^= rl(x[10] + x[9], 7);  x[8] ^= rl(x[11] + x[10], 9);
        x[9] ^= rl(x[8] + x[11], 13);  x[10] ^= rl(x[9] + x[8], 18);
        x[12] ^= rl(x[15] + x[14], 7); x[13] ^= rl(x[12] + x[15], 9);
        x[14] ^= rl(x[13] + x[12], 13); x[15] ^= rl(x[14] + x[13], 18);
    }
    out[0] = x[0]; out[1] = x[5]; out[2] = x[10]; out[3] = x[15];
    out[4] = x[6]; out[5] = x[7]; out[6] = x[8]; out[7] = x[9];
}

enum { DOM_SK = 1, DOM_PK_A = 2, DOM_PK_E = 3, DOM_RLK_A = 4, DOM_RLK_E = 5, DOM_ENC_V = 6, DOM_ENC_E0 = 7,
       DOM_ENC_E1 = 8, DOM_GK_A = 9, DOM_GK_E = 10, DOM_GAL_A = 11, DOM_GAL_E = 12 };

static void sample_small(Context& c, const uint8_t seed[32], uint32_t domain, uint64_t id0, int kind, int prime0,
                         int limbs, uint64_t* out, size_t item_stride, int items, cudaStream_t st) {
    SalsaKey k = subkey_for(seed, domain, 0);
    const int per = kind == 0 ? 16 : 8;
    const size_t total = (size_t)items * (c.n / per);
    if (kind == 0)
        sample_small_kernel<0><<<blocks_for(total, 128), 128, 0, st>>>(c.dc, k, id0, prime0, limbs, out, item_stride, items);
    else
        sample_small_kernel<1><<<blocks_for(total, 128), 128, 0, st>>>(c.dc, k, id0, prime0, limbs, out, item_stride, items);
    check_launch("sample_small");
}

static void sample_uniform(Context& c, const uint8_t seed[32], uint32_t domain, uint32_t sub, uint64_t id0, int prime0,
                           int limbs, uint64_t* out, size_t item_stride, int items, cudaStream_t st) {
    SalsaKey k = subkey_for(seed, domain, sub);
    const size_t total = (size_t)items * limbs * c.n / 4;
    sample_uniform_kernel<<<blocks_for(total, 128), 128, 0, st>>>(c.dc, k, id0, prime0, limbs, out, item_stride, items);
    check_launch("sample_uniform");
}

int kbfv_keygen_secret(kbfv_context* ctx, const uint8_t seed[32], int secret_kind, uint32_t h, uint64_t* d_sk,
                       kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk, KBFV_ERR_INVALID, "null argument");
        const int npq = c.nq + c.np;
        cudaStream_t st = S(stream);
        if (secret_kind == 1) {
            KB_CHECK_CUDA(cudaMemsetAsync(d_sk, 0, (size_t)npq * c.n * 8, st));
            SalsaKey k = subkey_for(seed, DOM_SK, 0);
            sample_hwt_kernel<<<1, 32, 0, st>>>(c.dc, k, 0, (int)h, 0, npq, d_sk, 0, 1);
            check_launch("sample_hwt");
        } else {
            sample_small(c, seed, DOM_SK, 0, 0, 0, npq, d_sk, 0, 1, st);
        }
        RowsIO io = rows_io(c.dc, d_sk, 0, npq);
        ntt_fwd(c.dc, io, io, npq, st);
    });
}

int kbfv_keygen_public(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t* d_pk,
                       kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk && d_pk, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        uint64_t* a = d_pk;
        uint64_t* b = d_pk + lq;
        sample_uniform(c, seed, DOM_PK_A, 0, 0, 0, c.nq, a, 0, 1, st);
        sample_small(c, seed, DOM_PK_E, 0, 1, 0, c.nq, b, 0, 1, st);
        RowsIO io = rows_io(c.dc, b, 0, c.nq);
        ntt_fwd(c.dc, io, io, c.nq, st);
        pk_combine_kernel<<<blocks_for(lq, 256), 256, 0, st>>>(c.dc, a, d_sk, b, lq);
        check_launch("pk_combine");
    });
}

int kbfv_keygen_relin(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t* d_rlk,
                      kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk && d_rlk, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const int npq = c.nq + c.np;
        const size_t lpq = (size_t)npq * c.n;
        for (int d = 0; d < c.dnum; d++) {
            uint64_t* a = d_rlk + (size_t)d * 2 * lpq;
            uint64_t* b = a + lpq;
            sample_uniform(c, seed, DOM_RLK_A, (uint32_t)d, 0, 0, npq, a, 0, 1, st);
            SalsaKey k = subkey_for(seed, DOM_RLK_E, (uint32_t)d);
            const size_t total = c.n / 8;
            sample_small_kernel<1><<<blocks_for(total, 128), 128, 0, st>>>(c.dc, k, 0, 0, npq, b, 0, 1);
            check_launch("sample_gauss");
            RowsIO io = rows_io(c.dc, b, 0, npq);
            ntt_fwd(c.dc, io, io, npq, st);
            rlk_combine_kernel<<<blocks_for(lpq, 256), 256, 0, st>>>(c.dc, a, d_sk, b, d, lpq);
            check_launch("rlk_combine");
        }
    });
}

static int gadget_pieces(int w) { return (60 + w - 1) / w; }

int kbfv_keygen_relin_gadget(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint32_t log_base,
                             uint64_t* d_gk, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk && d_gk, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(log_base >= 4 && log_base <= 30, KBFV_ERR_INVALID, "gadget base 2^w needs 4 <= w <= 30");
        const int w = (int)log_base, J = gadget_pieces(w);
        cudaStream_t st = S(stream);
        const int npq = c.nq + c.np;
        const size_t lpq = (size_t)npq * c.n;
        for (int i = 0; i < c.nq; i++) {
            uint64_t pm = 1;  // P mod q_i
            for (int k = 0; k < c.np; k++) pm = H::mulmod(pm, c.mods[c.nq + k] % c.mods[i], c.mods[i]);
            for (int j = 0; j < J; j++) {
                const uint32_t sub = (uint32_t)(i * J + j);
                uint64_t* a = d_gk + (size_t)sub * 2 * lpq;
                uint64_t* b = a + lpq;
                sample_uniform(c, seed, DOM_GK_A, sub, 0, 0, npq, a, 0, 1, st);
                SalsaKey k = subkey_for(seed, DOM_GK_E, sub);
                sample_small_kernel<1><<<blocks_for(c.n / 8, 128), 128, 0, st>>>(c.dc, k, 0, 0, npq, b, 0, 1);
                check_launch("sample_gauss");
                RowsIO io = rows_io(c.dc, b, 0, npq);
                ntt_fwd(c.dc, io, io, npq, st);
                const uint64_t g = H::mulmod(pm, H::powmod(2, (uint64_t)w * j, c.mods[i]), c.mods[i]);
                gk_combine_kernel<<<blocks_for(lpq, 256), 256, 0, st>>>(c.dc, a, d_sk, b, i, g, lpq);
                check_launch("gk_combine");
            }
        }
    });
}

int kbfv_encode(kbfv_context* ctx, const uint64_t* d_slots, uint64_t* d_m, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!count) return;
        if (d_m != d_slots)
            KB_CHECK_CUDA(cudaMemcpyAsync(d_m, d_slots, (size_t)count * c.n * 8, cudaMemcpyDeviceToDevice, S(stream)));
        RowsIO io = rows_io(c.dc, d_m, c.dc.idx_pt, 1);
        ntt_inv(c.dc, io, io, (int)count, S(stream));
    });
}

int kbfv_decode(kbfv_context* ctx, const uint64_t* d_m, uint64_t* d_slots, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!count) return;
        if (d_m != d_slots)
            KB_CHECK_CUDA(cudaMemcpyAsync(d_slots, d_m, (size_t)count * c.n * 8, cudaMemcpyDeviceToDevice, S(stream)));
        RowsIO io = rows_io(c.dc, d_slots, c.dc.idx_pt, 1);
        ntt_fwd(c.dc, io, io, (int)count, S(stream));
    });
}

// values (< t) as polynomial coefficients, replicated over Q and transformed
struct ReplicateSrc {
    const uint64_t* vals;
    int logn, nq;
    __device__ __forceinline__ int prime(int row) const { return row % nq; }
    __device__ __forceinline__ PtrRow bind(int row) const {
        return PtrRow{const_cast<uint64_t*>(vals) + ((size_t)(row / nq) << logn)};
    }
};

int kbfv_encode_ntt(kbfv_context* ctx, const uint64_t* d_vals, uint64_t* d_pt_ntt, uint32_t count,
                    kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        if (!count) return;
        require_batchable(c);
        ntt_fwd(c.dc, ReplicateSrc{d_vals, c.logn, c.nq}, rows_io(c.dc, d_pt_ntt, 0, c.nq), (int)(count * c.nq),
                S(stream));
    });
}

int kbfv_encrypt(kbfv_context* ctx, const uint8_t seed[32], uint64_t enc_id, const uint64_t* d_pk, const uint64_t* d_m,
                 uint64_t* d_ct, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_pk && d_m && d_ct, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint64_t* work = (uint64_t*)ensure_scratch(c, (size_t)cnt * 4 * lq * 8);
            const uint64_t id0 = enc_id + off;
            // [v | e0 | e1 | dm] per item
            sample_small(c, seed, DOM_ENC_V, id0, 0, 0, c.nq, work, 4 * lq, cnt, st);
            sample_small(c, seed, DOM_ENC_E0, id0, 1, 0, c.nq, work + lq, 4 * lq, cnt, st);
            sample_small(c, seed, DOM_ENC_E1, id0, 1, 0, c.nq, work + 2 * lq, 4 * lq, cnt, st);
            for (int i = 0; i < cnt; i++) {
                const size_t tot = lq;
                delta_m_kernel<<<blocks_for(tot, 256), 256, 0, st>>>(c.dc, d_m + (size_t)(off + i) * c.n,
                                                                      work + (size_t)i * 4 * lq + 3 * lq, tot);
            }
            check_launch("delta_m");
            RowsIO io = rows_io(c.dc, work, 0, c.nq);
            ntt_fwd(c.dc, io, io, cnt * 4 * c.nq, st);
            const size_t total = (size_t)cnt * lq;
            enc_combine_kernel<<<stride_blocks(total, 256), 256, 0, st>>>(c.dc, d_pk, work, d_ct + (size_t)off * 2 * lq, total);
            check_launch("enc_combine");
        }
    });
}

// decrypt: INTT over Q of (a*s + b), then the rounding
struct DecSrc {
    const uint64_t* ct;
    const uint64_t* sk;
    DevConsts dc;
    struct Row {
        const uint64_t *a, *b, *s;
        uint64_t q, mh, ml;
        // a and s fully reduced: one-high-product Barrett (mh holds its constant)
        __device__ __forceinline__ uint64_t load(int j) const { return add_mod(mul_mod_prod(a[j], s[j], q, mh), b[j], q); }
        __device__ __forceinline__ void store(int, uint64_t) const {}
    };
    __device__ __forceinline__ int prime(int row) const { return row % dc.nq; }
    __device__ __forceinline__ Row bind(int row) const {
        const int item = row / dc.nq, l = row % dc.nq;
        const size_t lq = (size_t)dc.nq << dc.logn;
        Row r;
        r.a = ct + item * 2 * lq + ((size_t)l << dc.logn);
        r.b = r.a + lq;
        r.s = sk + ((size_t)l << dc.logn);
        r.q = dc.mods[l]; r.mh = dc.mu_prod[l]; r.ml = 0;
        return r;
    }
};

int kbfv_decrypt(kbfv_context* ctx, const uint64_t* d_sk, const uint64_t* d_ct, uint64_t* d_m, uint32_t count,
                 kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_sk && d_ct && d_m, KBFV_ERR_INVALID, "null argument");
        require_batchable(c);
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint64_t* work = (uint64_t*)ensure_scratch(c, (size_t)cnt * lq * 8);
            ntt_inv(c.dc, DecSrc{d_ct + (size_t)off * 2 * lq, d_sk, c.dc}, rows_io(c.dc, work, 0, c.nq), cnt * c.nq, st);
            dim3 grid((unsigned)(c.n / 128), (unsigned)cnt);
#define L_DR(M) decrypt_round_kernel<M><<<grid, 128, 0, st>>>(c.dc, work, d_m + (size_t)off * c.n)
            DISPATCH_MAXQ(c.nq, L_DR);
#undef L_DR
            check_launch("decrypt_round");
        }
    });
}

int kbfv_add(kbfv_context* ctx, const uint64_t* d_x, const uint64_t* d_y, uint64_t* d_out, uint32_t count,
             kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        const size_t total = (size_t)count * 2 * c.nq * c.n;
        if (!total) return;
        add_kernel<<<blocks_for(total, 256), 256, 0, S(stream)>>>(c.dc, d_x, d_y, d_out, total, c.nq);
        check_launch("add");
    });
}

int kbfv_mul_plain(kbfv_context* ctx, const uint64_t* d_ct, const uint64_t* d_pt_ntt, uint64_t* d_out, uint32_t count,
                   kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        const size_t total = (size_t)count * 2 * c.nq * c.n;
        if (!total) return;
        mul_plain_kernel<<<blocks_for(total, 256), 256, 0, S(stream)>>>(c.dc, d_ct, d_pt_ntt, d_out, total);
        check_launch("mul_plain");
    });
}

static PtrBatch make_batch(const uint64_t* const* a, const uint64_t* const* b, uint64_t* const* o, int cnt) {
    PtrBatch pb;
    std::memset(&pb, 0, sizeof pb);
    for (int i = 0; i < cnt; i++) {
        pb.a[i] = a[i];
        pb.b[i] = b[i];
        pb.o[i] = o ? o[i] : nullptr;
    }
    return pb;
}

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
            mul_front(c, pb, cnt, m, st);
            k5_launch(c, cnt, m, out, 0, st);
            RowsIO io = rows_io(c.dc, out, 0, c.nq);
            ntt_fwd(c.dc, io, io, cnt * 3 * c.nq, st);
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
                mul_relin_chunk(c, d_rlk, pb, cnt, m, st);
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
                mul_relin_chunk(c, d_rlk, pb, n, m, b == 0 ? st : c.aux[b - 1]);
            }
            for (int b = 1; b < nb; b++) {
                KB_CHECK_CUDA(cudaEventRecord(c.join_ev[b - 1], c.aux[b - 1]));
                KB_CHECK_CUDA(cudaStreamWaitEvent(st, c.join_ev[b - 1], 0));
            }
        }
    });
}

int kbfv_tune_set(kbfv_context* ctx, int knob, int64_t value) {
    return guarded([&] {
        Context& c = CX(ctx);
        switch (knob) {
            case KBFV_TUNE_NTT_BLOCK_LOG:
                KB_REQUIRE(value == 0 || (value >= 12 && value <= 14), KBFV_ERR_INVALID,
                           "NTT block log must be 0 (built-in) or 12..14");
                c.ntt_block_log = (int)value;
                break;
            case KBFV_TUNE_BRANCHES:
                KB_REQUIRE(value >= 1 && value <= 4, KBFV_ERR_INVALID, "branches must be 1..4");
                c.branches = (int)value;
                break;
            case KBFV_TUNE_HOST_CHUNK:
                KB_REQUIRE(value >= 0 && value <= kMaxBatch, KBFV_ERR_INVALID, "host chunk must be 0..128");
                c.host_chunk = (int)value;
                break;
            default: throw KbfvError(KBFV_ERR_INVALID, "unknown tuning knob");
        }
    });
}

int kbfv_tune_get(const kbfv_context* ctx, int knob, int64_t* value) {
    return guarded([&] {
        const Context& c = CX(const_cast<kbfv_context*>(ctx));
        KB_REQUIRE(value, KBFV_ERR_INVALID, "null argument");
        switch (knob) {
            case KBFV_TUNE_NTT_BLOCK_LOG: *value = c.ntt_block_log; break;
            case KBFV_TUNE_BRANCHES: *value = c.branches; break;
            case KBFV_TUNE_HOST_CHUNK: *value = c.host_chunk; break;
            default: throw KbfvError(KBFV_ERR_INVALID, "unknown tuning knob");
        }
    });
}

int kbfv_set_branches(kbfv_context* ctx, uint32_t branches) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(branches >= 1 && branches <= 4, KBFV_ERR_INVALID, "branches must be 1..4");
        c.branches = (int)branches;
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
            mul_relin_chunk(c, d_rlk, pb, n, m, comp);
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


// ---- T-base key switch (the reference's KLSS) ------------------------------
int kbfv_context_klss(const kbfv_context* ctx, uint32_t* ri_blocks, uint32_t* qj_blocks, uint64_t* key_words) {
    return guarded([&] {
        const Context& c = CX(const_cast<kbfv_context*>(ctx));
        require_klss(c);
        if (ri_blocks) *ri_blocks = (uint32_t)c.kc.nri;
        if (qj_blocks) *qj_blocks = (uint32_t)c.kc.nqj;
        if (key_words) *key_words = (uint64_t)2 * c.kc.nqj * c.kc.nri * c.nt * c.n;
    });
}

int kbfv_rlk_to_klss(kbfv_context* ctx, const uint64_t* d_rlk, uint64_t* d_rlk_t, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(d_rlk && d_rlk_t, KBFV_ERR_INVALID, "null key pointer");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const KlssConsts& kc = c.kc;
        const int npq = dc.npq;
        uint64_t* coef = (uint64_t*)ensure_scratch(c, (size_t)c.dnum * 2 * npq * c.n * 8);
        // key [digit][a|b][Q|P] in NTT form -> coefficient form
        ntt_inv(dc, rows_io(dc, const_cast<uint64_t*>(d_rlk), 0, npq), rows_io(dc, coef, 0, npq),
                c.dnum * 2 * npq, st);
        // Ri blocks -> T (modUpPQtoT_23), written as [a|b][digit][Ri][T]
        for (int h = 0; h < 2; h++) {
            klss_block_to_t_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)kc.nri, (unsigned)c.dnum), 128, 0, st>>>(
                dc, kc, coef + ((size_t)h * npq << c.logn), d_rlk_t + ((size_t)h * c.dnum * kc.nri * c.nt << c.logn), 1,
                (size_t)2 * npq << c.logn, (size_t)kc.nri * c.nt << c.logn);
            check_launch("klss_pq_to_t");
        }
        RowsIO io = rows_io(dc, d_rlk_t, dc.idx_t, c.nt);
        ntt_fwd(dc, io, io, 2 * c.dnum * kc.nri * c.nt, st);
    });
}

int kbfv_klss_modup_qj_to_t(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                            kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(polys <= 65535, KBFV_ERR_INVALID, "at most 65535 polynomials per call");
        if (!polys) return;
        klss_block_to_t_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)c.kc.nqj, polys), 128, 0, S(stream)>>>(
            c.dc, c.kc, d_in, d_out, 0, (size_t)c.nq << c.logn, (size_t)c.kc.nqj * c.nt << c.logn);
        check_launch("klss_qj_to_t");
    });
}

int kbfv_klss_modup_pq_to_t(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys,
                            kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(polys <= 65535, KBFV_ERR_INVALID, "at most 65535 polynomials per call");
        if (!polys) return;
        klss_block_to_t_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)c.kc.nri, polys), 128, 0, S(stream)>>>(
            c.dc, c.kc, d_in, d_out, 1, (size_t)c.dc.npq << c.logn, (size_t)c.kc.nri * c.nt << c.logn);
        check_launch("klss_pq_to_t");
    });
}

int kbfv_klss_external_product(kbfv_context* ctx, const uint64_t* d_digits, const uint64_t* d_rlk_t,
                               uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(d_rlk_t, KBFV_ERR_NO_KEY, "T-base relinearisation key missing");
        const KlssConsts& kc = c.kc;
        ntt_inv(c.dc, ExtProdSrc{d_digits, d_rlk_t, c.dc, c.nt, kc.nri, kc.nqj, kc.nqj},
                rows_io(c.dc, d_out, c.dc.idx_t, c.nt), (int)count * 2 * kc.nri * c.nt, S(stream));
    });
}

int kbfv_klss_t_to_pq(kbfv_context* ctx, const uint64_t* d_in, uint64_t* d_out, uint32_t polys, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(polys <= 65535, KBFV_ERR_INVALID, "at most 65535 polynomials per call");
        if (!polys) return;
        klss_t_to_pq_kernel<<<dim3((unsigned)(c.n / 128), (unsigned)c.kc.nri, polys), 128, 0, S(stream)>>>(
            c.dc, c.kc, d_in, d_out);
        check_launch("klss_t_to_pq");
    });
}

int kbfv_relinearize_klss(kbfv_context* ctx, const uint64_t* d_rlk_t, const uint64_t* d_tensor, uint64_t* d_ct,
                          uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(d_rlk_t, KBFV_ERR_NO_KEY, "T-base relinearisation key missing");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
            MulScratch m = mul_scratch_layout(c, cnt, base);
            const uint64_t* tz = d_tensor + (size_t)off * 3 * lq;
            uint64_t* out = d_ct + (size_t)off * 2 * lq;
            ntt_inv(dc, TensorA2{tz, dc.logn, dc.nq}, rows_io(dc, m.sd2, 0, dc.nq), cnt * dc.nq, st);
            klss_keyswitch(c, d_rlk_t, cnt, m, st);
            std::vector<uint64_t*> O(cnt);
            std::vector<const uint64_t*> Z(cnt);
            for (int i = 0; i < cnt; i++) { O[i] = out + (size_t)i * 2 * lq; Z[i] = nullptr; }
            PtrBatch pb = make_batch(Z.data(), Z.data(), O.data(), cnt);
            ntt_fwd(dc, ModDownAddSrc{m.se, nullptr, dc}, OutCtDst{pb, dc.logn, dc.nq}, cnt * 2 * dc.nq, st);
            for (int i = 0; i < cnt; i++) {
                const size_t tot = 2 * lq;
                add_kernel<<<blocks_for(tot, 256), 256, 0, st>>>(dc, out + (size_t)i * 2 * lq, tz + (size_t)i * 3 * lq + lq,
                                                                 out + (size_t)i * 2 * lq, tot, dc.nq);
            }
            check_launch("relin_add");
        }
    });
}

int kbfv_mul_relin_klss(kbfv_context* ctx, const uint64_t* d_rlk_t, const uint64_t* d_ct_a, const uint64_t* d_ct_b,
                        uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        require_klss(c);
        KB_REQUIRE(d_rlk_t, KBFV_ERR_NO_KEY, "T-base relinearisation key missing");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            std::vector<const uint64_t*> A(cnt), B(cnt);
            std::vector<uint64_t*> O(cnt);
            for (int i = 0; i < cnt; i++) {
                A[i] = d_ct_a + (size_t)(off + i) * 2 * lq;
                B[i] = d_ct_b + (size_t)(off + i) * 2 * lq;
                O[i] = d_out + (size_t)(off + i) * 2 * lq;
            }
            PtrBatch pb = make_batch(A.data(), B.data(), O.data(), cnt);
            uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
            MulScratch m = mul_scratch_layout(c, cnt, base);
            mul_relin_klss_chunk(c, d_rlk_t, pb, cnt, m, st);
        }
    });
}


// ---- parameter sets, seeds, batched NTT over pointer arrays, plaintext add -----
struct kbfv_params_owned {
    kbfv_params p;
    std::vector<uint64_t> q, pp;
};

int kbfv_params_create(uint32_t log_n, const uint32_t* q_bits, uint32_t q_count, const uint32_t* p_bits,
                       uint32_t p_count, uint64_t plain_modulus, uint32_t dnum, kbfv_params** out) {
    return guarded([&] {
        KB_REQUIRE(out && q_bits && p_bits, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(log_n >= 10 && log_n <= 16, KBFV_ERR_INVALID, "log_n out of range");
        KB_REQUIRE(q_count >= 1 && q_count <= (uint32_t)kMaxQ && p_count >= 1 && p_count <= (uint32_t)kMaxP,
                   KBFV_ERR_INVALID, "prime counts out of range");
        auto* o = new kbfv_params_owned();
        const uint64_t n = (uint64_t)1 << log_n;
        std::vector<uint64_t> used;
        auto pick = [&](uint32_t bits, std::vector<uint64_t>& dst) {
            if (bits < 20 || bits > 60) {
                delete o;
                throw KbfvError(KBFV_ERR_INVALID, "prime sizes must be 20..60 bits");
            }
            auto v = H::primes_bits(n, (int)bits, 1, used);
            if (v.empty()) {
                delete o;
                throw KbfvError(KBFV_ERR_PARAMS, "not enough NTT-friendly primes of the requested size");
            }
            dst.push_back(v[0]);
            used.push_back(v[0]);
        };
        for (uint32_t i = 0; i < p_count; i++) pick(p_bits[i], o->pp);
        for (uint32_t i = 0; i < q_count; i++) pick(q_bits[i], o->q);
        std::memset(&o->p, 0, sizeof o->p);
        o->p.log_n = log_n;
        o->p.plain_modulus = plain_modulus;
        o->p.q_count = q_count;
        o->p.q = o->q.data();
        o->p.p_count = p_count;
        o->p.p = o->pp.data();
        o->p.dnum = dnum ? dnum : 1;
        *out = &o->p;
    });
}

int kbfv_params_destroy(kbfv_params* params) {
    if (params) delete reinterpret_cast<kbfv_params_owned*>(params);  // p is the first member
    return KBFV_OK;
}

int kbfv_set_seed(kbfv_context* ctx, const uint8_t seed[32]) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(seed, KBFV_ERR_INVALID, "null seed");
        std::memcpy(c.seed, seed, 32);
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

int kbfv_add_plain(kbfv_context* ctx, const uint64_t* d_ct, const uint64_t* d_m, uint64_t* d_out, uint32_t count,
                   kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_ct && d_m && d_out, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint64_t* dm = (uint64_t*)ensure_scratch(c, (size_t)cnt * lq * 8);
            delta_m_kernel<<<blocks_for((size_t)cnt * lq, 256), 256, 0, st>>>(c.dc, d_m + (size_t)off * c.n, dm,
                                                                             (size_t)cnt * lq);
            check_launch("delta_m");
            RowsIO io = rows_io(c.dc, dm, 0, c.nq);
            ntt_fwd(c.dc, io, io, cnt * c.nq, st);
            for (int i = 0; i < cnt; i++) {
                const uint64_t* src = d_ct + (size_t)(off + i) * 2 * lq;
                uint64_t* dst = d_out + (size_t)(off + i) * 2 * lq;
                if (dst != src) KB_CHECK_CUDA(cudaMemcpyAsync(dst, src, lq * 8, cudaMemcpyDeviceToDevice, st));
                add_kernel<<<blocks_for(lq, 256), 256, 0, st>>>(c.dc, src + lq, dm + (size_t)i * lq, dst + lq, lq,
                                                                c.nq);
            }
            check_launch("add_plain");
        }
    });
}


// ---- levels ---------------------------------------------------------------
int kbfv_context_at_level(kbfv_context* ctx, uint32_t live_q, kbfv_context** out) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(out, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(!c.parent, KBFV_ERR_INVALID, "levels are taken from the top-level context");
        KB_REQUIRE(live_q >= 1 && live_q <= (uint32_t)c.nq, KBFV_ERR_LEVEL, "live prime count out of range");
        if (live_q == (uint32_t)c.nq) {
            *out = ctx;
            return;
        }
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.levels.size() < (size_t)c.nq) c.levels.resize(c.nq, nullptr);
        if (!c.levels[live_q]) {
            kbfv_params prm;
            std::memset(&prm, 0, sizeof prm);
            prm.log_n = (uint32_t)c.logn;
            prm.plain_modulus = c.t;
            prm.q_count = live_q;
            prm.q = c.mods.data();
            prm.p_count = (uint32_t)c.np;
            prm.p = c.mods.data() + c.nq;
            prm.digit_primes = (uint32_t)c.alpha;
            auto* h = new kbfv_context();
            try {
                build_context(h->c, prm);
            } catch (...) {
                if (h->c.pool) cudaFree(h->c.pool);
                delete h;
                throw;
            }
            h->c.parent = &c;
            h->c.dc.key_nq = c.nq;
            h->c.dc.key_npq = c.nq + c.np;
            std::memcpy(h->c.seed, c.seed, 32);
            c.levels[live_q] = h;
        }
        *out = (kbfv_context*)c.levels[live_q];
    });
}

int kbfv_mod_switch(kbfv_context* ctx, const uint64_t* d_ct, uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(c.nq >= 2, KBFV_ERR_LEVEL, "a ciphertext with one live prime cannot be switched down");
        KB_REQUIRE(d_ct && d_out, KBFV_ERR_INVALID, "null argument");
        const size_t in_words = (size_t)count * 2 * c.nq * c.n, out_words = (size_t)count * 2 * (c.nq - 1) * c.n;
        KB_REQUIRE(d_out + out_words <= d_ct || d_ct + in_words <= d_out, KBFV_ERR_INVALID,
                   "output must not overlap the input");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const int nout = c.nq - 1;
        const uint32_t chunk = 32;
        for (uint32_t off = 0; off < count; off += chunk) {
            const int cnt = (int)std::min<uint32_t>(chunk, count - off);
            const int polys = cnt * 2;
            uint64_t* last = (uint64_t*)ensure_scratch(c, (size_t)polys * (1 + nout) * c.n * 8);
            uint64_t* corr = last + ((size_t)polys << c.logn);
            const uint64_t* in = d_ct + (size_t)off * 2 * c.nq * c.n;
            uint64_t* o = d_out + (size_t)off * 2 * nout * c.n;
            ntt_inv(dc, LastLimbSrc{in, c.logn, c.nq}, rows_io(dc, last, c.nq - 1, 1), polys, st);
            ntt_fwd(dc, ModSwitchSrc{last, dc}, rows_io(dc, corr, 0, nout), polys * nout, st);
            const size_t total = (size_t)polys * nout * c.n;
            mod_switch_combine_kernel<<<stride_blocks(total, 256), 256, 0, st>>>(dc, in, corr, o, total);
            check_launch("mod_switch");
        }
    });
}

int kbfv_mul_relin_levels(kbfv_context* ctx, const uint64_t* d_rlk, const uint32_t* live_q,
                          const uint64_t* const* ct_a, const uint64_t* const* ct_b, uint64_t* const* out,
                          uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(!c.parent, KBFV_ERR_INVALID, "call on the top-level context");
        KB_REQUIRE(live_q && ct_a && ct_b && out, KBFV_ERR_INVALID, "null pointer array");
        std::map<uint32_t, std::vector<uint32_t>> groups;
        for (uint32_t i = 0; i < count; i++) {
            KB_REQUIRE(live_q[i] >= 1 && live_q[i] <= (uint32_t)c.nq, KBFV_ERR_LEVEL, "live prime count out of range");
            groups[live_q[i]].push_back(i);
        }
        // the level groups run concurrently: the first on the caller's stream, the
        // next ones on the context's lane streams (forked from and joined back into
        // the caller's stream); each level context has its own scratch arena
        cudaStream_t st = S(stream);
        const int ng = (int)groups.size();
        const int lanes = std::min(ng, 4);
        if (lanes > 1) {
            if (!c.lane_fork) {
                for (int k = 0; k < 3; k++) {
                    KB_CHECK_CUDA(cudaStreamCreateWithFlags(&c.lane[k], cudaStreamNonBlocking));
                    KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.lane_join[k], cudaEventDisableTiming));
                }
                KB_CHECK_CUDA(cudaEventCreateWithFlags(&c.lane_fork, cudaEventDisableTiming));
            }
            KB_CHECK_CUDA(cudaEventRecord(c.lane_fork, st));
            for (int k = 1; k < lanes; k++) KB_CHECK_CUDA(cudaStreamWaitEvent(c.lane[k - 1], c.lane_fork, 0));
        }
        int g = 0;
        for (auto it = groups.rbegin(); it != groups.rend(); ++it, ++g) {  // highest level first
            kbfv_context* lv = nullptr;
            int rc = kbfv_context_at_level(ctx, it->first, &lv);
            if (rc != KBFV_OK) throw KbfvError(rc, g_last_error);
            std::vector<const uint64_t*> A, B;
            std::vector<uint64_t*> O;
            for (uint32_t i : it->second) {
                A.push_back(ct_a[i]);
                B.push_back(ct_b[i]);
                O.push_back(out[i]);
            }
            const int lane = g % lanes;
            cudaStream_t ls = lane == 0 ? st : c.lane[lane - 1];
            rc = kbfv_mul_relin_batch(lv, d_rlk, A.data(), B.data(), O.data(), (uint32_t)A.size(), (kbfv_stream)ls);
            if (rc != KBFV_OK) throw KbfvError(rc, g_last_error);
        }
        for (int k = 1; k < lanes; k++) {
            KB_CHECK_CUDA(cudaEventRecord(c.lane_join[k - 1], c.lane[k - 1]));
            KB_CHECK_CUDA(cudaStreamWaitEvent(st, c.lane_join[k - 1], 0));
        }
    });
}


// ---- key switching over a gadget decomposition ------------------------------
// G1: pieces of a1*a2 (coefficient form, sd2) fused into the forward NTT over Q|P;
// G2/G3: the key-switch tail (ks_tail) with the gadget key, written to the outputs.
static size_t gadget_sg_bytes(const Context& c, int count, int w) {
    return (size_t)count * c.nq * gadget_pieces(w) * (c.nq + c.np) * c.n * 8;
}
static int gadget_chunk(const Context& c, int w) {
    const size_t per = gadget_sg_bytes(c, 1, w);
    return (int)std::max<size_t>(1, std::min<size_t>(kMaxBatch, ((size_t)4 << 30) / per));
}

static void gadget_keyswitch(Context& c, const uint64_t* gk, int w, int count, const MulScratch& m, uint64_t* sg,
                             const uint64_t* add, const PtrBatch& pb, cudaStream_t st) {
    const DevConsts& dc = c.dc;
    const int J = gadget_pieces(w), ndig = c.nq * J;
    // fully reduced NTT outputs: the key product sums ndig terms below q^2
    ntt_fwd<GadgetDigitSrc, RowsIO, true>(dc, GadgetDigitSrc{m.sd2, dc, J, w}, rows_io(dc, sg, 0, dc.npq),
                                         count * ndig * dc.npq, st);
    ks_tail(dc, sg, gk, ndig, m.se, add, pb, count, st);
}

int kbfv_relinearize_gadget(kbfv_context* ctx, const uint64_t* d_gk, uint32_t log_base, const uint64_t* d_tensor,
                            uint64_t* d_ct, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_gk, KBFV_ERR_NO_KEY, "gadget key missing");
        KB_REQUIRE(log_base >= 4 && log_base <= 30, KBFV_ERR_INVALID, "gadget base 2^w needs 4 <= w <= 30");
        KB_REQUIRE(c.nq * gadget_pieces((int)log_base) < 256, KBFV_ERR_INVALID, "too many gadget digits");
        const int w = (int)log_base;
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const size_t lq = (size_t)c.nq * c.n;
        const int chunk = gadget_chunk(c, w);
        for (uint32_t off = 0; off < count; off += chunk) {
            const int cnt = (int)std::min<uint32_t>(chunk, count - off);
            const size_t mb = mul_scratch_layout(c, cnt, nullptr).bytes;
            uint8_t* base = ensure_scratch(c, mb + gadget_sg_bytes(c, cnt, w));
            MulScratch m = mul_scratch_layout(c, cnt, base);
            uint64_t* sg = (uint64_t*)(base + mb);
            const uint64_t* tz = d_tensor + (size_t)off * 3 * lq;
            uint64_t* out = d_ct + (size_t)off * 2 * lq;
            ntt_inv(dc, TensorA2{tz, dc.logn, dc.nq}, rows_io(dc, m.sd2, 0, dc.nq), cnt * dc.nq, st);
            std::vector<uint64_t*> O(cnt);
            std::vector<const uint64_t*> Z(cnt);
            for (int i = 0; i < cnt; i++) { O[i] = out + (size_t)i * 2 * lq; Z[i] = nullptr; }
            PtrBatch pb = make_batch(Z.data(), Z.data(), O.data(), cnt);
            gadget_keyswitch(c, d_gk, w, cnt, m, sg, nullptr, pb, st);
            for (int i = 0; i < cnt; i++) {
                const size_t tot = 2 * lq;
                add_kernel<<<blocks_for(tot, 256), 256, 0, st>>>(dc, out + (size_t)i * 2 * lq, tz + (size_t)i * 3 * lq + lq,
                                                                 out + (size_t)i * 2 * lq, tot, dc.nq);
            }
            check_launch("relin_add");
        }
    });
}

int kbfv_mul_relin_gadget(kbfv_context* ctx, const uint64_t* d_gk, uint32_t log_base, const uint64_t* d_ct_a,
                          const uint64_t* d_ct_b, uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_gk, KBFV_ERR_NO_KEY, "gadget key missing");
        KB_REQUIRE(log_base >= 4 && log_base <= 30, KBFV_ERR_INVALID, "gadget base 2^w needs 4 <= w <= 30");
        KB_REQUIRE(c.nq * gadget_pieces((int)log_base) < 256, KBFV_ERR_INVALID, "too many gadget digits");
        const int w = (int)log_base;
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        const int chunk = gadget_chunk(c, w);
        for (uint32_t off = 0; off < count; off += chunk) {
            const int cnt = (int)std::min<uint32_t>(chunk, count - off);
            std::vector<const uint64_t*> A(cnt), B(cnt);
            std::vector<uint64_t*> O(cnt);
            for (int i = 0; i < cnt; i++) {
                A[i] = d_ct_a + (size_t)(off + i) * 2 * lq;
                B[i] = d_ct_b + (size_t)(off + i) * 2 * lq;
                O[i] = d_out + (size_t)(off + i) * 2 * lq;
            }
            PtrBatch pb = make_batch(A.data(), B.data(), O.data(), cnt);
            const size_t mb = mul_scratch_layout(c, cnt, nullptr).bytes;
            uint8_t* base = ensure_scratch(c, mb + gadget_sg_bytes(c, cnt, w));
            MulScratch m = mul_scratch_layout(c, cnt, base);
            uint64_t* sg = (uint64_t*)(base + mb);
            mul_front(c, pb, cnt, m, st);
            k5_launch(c, cnt, m, nullptr, 2, st);
            gadget_keyswitch(c, d_gk, w, cnt, m, sg, m.sd, pb, st);
        }
    });
}


int kbfv_probe_arith(int kind, uint32_t iters, double* gops) {
    return guarded([&] {
        KB_REQUIRE(kind >= 0 && kind <= 11 && gops && iters >= 1, KBFV_ERR_INVALID, "bad probe arguments");
        int dev = 0, sms = 0;
        KB_CHECK_CUDA(cudaGetDevice(&dev));
        KB_CHECK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const unsigned blocks = (unsigned)sms * 8, threads = 256;
        uint64_t* out = nullptr;
        KB_CHECK_CUDA(cudaMalloc(&out, (size_t)blocks * threads * 8));
        const uint64_t q = 1152921504606584833ULL;  // 60-bit
        uint64_t mh, ml;
        H::barrett_mu(q, mh, ml);
        const uint64_t mp = (uint64_t)(((unsigned __int128)1 << 122) / q);
        cudaEvent_t e0, e1;
        KB_CHECK_CUDA(cudaEventCreate(&e0));
        KB_CHECK_CUDA(cudaEventCreate(&e1));
        float ms = 0.f;
        for (int rep = 0; rep < 2; rep++) {  // the first launch warms up
            KB_CHECK_CUDA(cudaEventRecord(e0));
            switch (kind) {
#define P_K(K) case K: probe_arith_kernel<K><<<blocks, threads>>>(out, (int)iters, q, mh, ml, mp); break;
                P_K(0) P_K(1) P_K(2) P_K(3) P_K(4) P_K(5) P_K(6) P_K(7) P_K(8) P_K(9) P_K(10) P_K(11)
#undef P_K
            }
            KB_CHECK_CUDA(cudaEventRecord(e1));
            KB_CHECK_CUDA(cudaEventSynchronize(e1));
        }
        KB_CHECK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(out);
        check_launch("probe_arith");
        *gops = (double)blocks * threads * iters * kProbeChains / (ms * 1e6);
    });
}


// ---- Galois automorphisms (rotations, conjugation) ---------------------------
uint64_t kbfv_galois_element(const kbfv_context* ctx, int64_t rot_slots) {
    if (!ctx) return 0;
    const Context& c = const_cast<kbfv_context*>(ctx)->c;
    const uint64_t m = 2 * c.n;
    if (rot_slots < 0) return m - 1;  // conjugation
    uint64_t g = 1;
    for (int64_t i = 0; i < rot_slots; i++) g = g * 5 % m;
    return g;
}

int kbfv_keygen_galois(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* d_sk, uint64_t galois_elt,
                       uint64_t* d_gk, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(d_sk && d_gk, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE((galois_elt & 1) && galois_elt < 2 * c.n, KBFV_ERR_INVALID, "Galois element must be odd and below 2N");
        cudaStream_t st = S(stream);
        const int npq = c.nq + c.np;
        const size_t lpq = (size_t)npq * c.n;
        uint64_t* sg = (uint64_t*)ensure_scratch(c, lpq * 8);
        galois_ntt_kernel<<<blocks_for(lpq, 256), 256, 0, st>>>(c.dc, d_sk, sg, galois_elt, lpq);
        check_launch("galois_sk");
        for (int d = 0; d < c.dnum; d++) {
            uint64_t* a = d_gk + (size_t)d * 2 * lpq;
            uint64_t* b = a + lpq;
            sample_uniform(c, seed, DOM_GAL_A, (uint32_t)d, galois_elt, 0, npq, a, 0, 1, st);
            SalsaKey k = subkey_for(seed, DOM_GAL_E, (uint32_t)d);
            sample_small_kernel<1><<<blocks_for(c.n / 8, 128), 128, 0, st>>>(c.dc, k, galois_elt, 0, npq, b, 0, 1);
            check_launch("sample_gauss");
            RowsIO io = rows_io(c.dc, b, 0, npq);
            ntt_fwd(c.dc, io, io, npq, st);
            ksk_combine_kernel<<<blocks_for(lpq, 256), 256, 0, st>>>(c.dc, a, d_sk, sg, b, d, lpq);
            check_launch("ksk_combine");
        }
    });
}

int kbfv_apply_galois(kbfv_context* ctx, const uint64_t* d_gk, uint64_t galois_elt, const uint64_t* d_ct,
                      uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_gk, KBFV_ERR_NO_KEY, "Galois key missing");
        KB_REQUIRE(d_ct && d_out, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE((galois_elt & 1) && galois_elt < 2 * c.n, KBFV_ERR_INVALID, "Galois element must be odd and below 2N");
        cudaStream_t st = S(stream);
        const DevConsts& dc = c.dc;
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            uint8_t* base = ensure_scratch(c, mul_scratch_layout(c, cnt, nullptr).bytes);
            MulScratch m = mul_scratch_layout(c, cnt, base);
            const uint64_t* in = d_ct + (size_t)off * 2 * lq;
            uint64_t* out = d_out + (size_t)off * 2 * lq;
            // g(b) first (the output may overwrite the input): sb holds [item][nq]
            for (int i = 0; i < cnt; i++)
                galois_ntt_kernel<<<blocks_for(lq, 256), 256, 0, st>>>(dc, in + (size_t)i * 2 * lq + lq,
                                                                        m.sb + (size_t)i * lq, galois_elt, lq);
            check_launch("galois_b");
            // g(a) read through the permutation by the inverse NTT, then the hybrid key switch
            ntt_inv(dc, GaloisASrc{in, galois_elt, dc.logn, dc.nq}, rows_io(dc, m.sa, 0, dc.nq), cnt * dc.nq, st);
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
            ks_tail(dc, m.sd2, d_gk, dc.dnum, m.se, nullptr, pb, cnt, st);
            for (int i = 0; i < cnt; i++)
                add_kernel<<<blocks_for(lq, 256), 256, 0, st>>>(dc, out + (size_t)i * 2 * lq + lq, m.sb + (size_t)i * lq,
                                                                out + (size_t)i * 2 * lq + lq, lq, dc.nq);
            check_launch("galois_add");
        }
    });
}


// ---- scalar and linear ops (BFVScheme.cuh:246-330: multConstAndEqual(uint64),
// multConstAndAddCipherEqual, sub / subAndEqual, negateAndEqual) -------------
static int linear_op(kbfv_context* ctx, const uint64_t* x, const uint64_t* y, uint64_t* out, uint64_t cnst,
                     int op, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(x && out && (op == 1 || op == 2 || y), KBFV_ERR_INVALID, "null argument");
        const size_t total = (size_t)count * 2 * c.nq * c.n;
        if (!total) return;
        ScalarTab tab{};
        for (int l = 0; op >= 2 && l < c.nq; l++) {
            tab.c[l] = cnst % c.mods[l];
            tab.cs[l] = H::shoup(tab.c[l], c.mods[l]);
        }
        linear_kernel<<<blocks_for(total, 256), 256, 0, S(stream)>>>(c.dc, x, y, out, total, c.nq, op, tab);
        check_launch("linear");
    });
}
int kbfv_sub(kbfv_context* ctx, const uint64_t* d_x, const uint64_t* d_y, uint64_t* d_out, uint32_t count,
             kbfv_stream stream) {
    return linear_op(ctx, d_x, d_y, d_out, 0, 0, count, stream);
}
int kbfv_negate(kbfv_context* ctx, const uint64_t* d_x, uint64_t* d_out, uint32_t count, kbfv_stream stream) {
    return linear_op(ctx, d_x, nullptr, d_out, 0, 1, count, stream);
}
int kbfv_mul_scalar(kbfv_context* ctx, const uint64_t* d_x, uint64_t cnst, uint64_t* d_out, uint32_t count,
                    kbfv_stream stream) {
    return linear_op(ctx, d_x, nullptr, d_out, cnst, 2, count, stream);
}
int kbfv_mul_scalar_add(kbfv_context* ctx, const uint64_t* d_x, uint64_t cnst, uint64_t* d_acc, uint32_t count,
                        kbfv_stream stream) {
    return linear_op(ctx, d_x, d_acc, d_acc, cnst, 3, count, stream);
}


// ---- wire format: versioned little-endian container for ciphertexts and keys ----
namespace {
struct WireHeader {
    char magic[8];         // "KBFVWIRE"
    uint32_t version;      // 1
    uint32_t kind;         // kbfv_wire_kind
    uint32_t log_n, q_count, p_count, count;
    uint64_t aux;          // Galois element (kind 6) or gadget log base (kind 7)
    uint64_t prime_digest; // FNV-1a over Q (live primes), P and t
    uint64_t words;        // payload words per object
};
static_assert(sizeof(WireHeader) == 56, "wire header layout");

uint64_t prime_digest(const Context& c) {
    uint64_t h = 1469598103934665603ULL;
    auto mix = [&](uint64_t v) {
        for (int b = 0; b < 8; b++) {
            h ^= (v >> (8 * b)) & 0xff;
            h *= 1099511628211ULL;
        }
    };
    for (int i = 0; i < c.nq + c.np; i++) mix(c.mods[i]);
    mix(c.t);
    return h;
}

// payload words per object, 0 for an unknown kind
uint64_t wire_words(const Context& c, int kind, uint64_t aux) {
    const uint64_t n = c.n, lq = (uint64_t)c.nq * n, lpq = (uint64_t)(c.nq + c.np) * n;
    switch (kind) {
        case 1: return 2 * lq;                                // ciphertext [a|b] over Q, NTT
        case 2: return n;                                     // plaintext coefficients mod t
        case 3: return lpq;                                   // secret key over Q|P, NTT
        case 4: return 2 * lq;                                // public key
        case 5: return (uint64_t)c.dnum * 2 * lpq;            // relinearisation key
        case 6: return (uint64_t)c.dnum * 2 * lpq;            // Galois key
        case 7: return aux >= 4 && aux <= 30 ? (uint64_t)c.nq * ((60 + aux - 1) / aux) * 2 * lpq : 0;  // gadget key
        case 8: return c.klss_ok ? (uint64_t)2 * c.kc.nqj * c.kc.nri * c.nt * n : 0;  // T-base key
        default: return 0;
    }
}
}  // namespace

size_t kbfv_wire_bytes(const kbfv_context* ctx, int kind, uint64_t aux, uint32_t count) {
    if (!ctx) return 0;
    const Context& c = const_cast<kbfv_context*>(ctx)->c;
    const uint64_t w = wire_words(c, kind, aux);
    return w ? sizeof(WireHeader) + (size_t)w * count * 8 : 0;
}

int kbfv_wire_save(kbfv_context* ctx, int kind, uint64_t aux, const uint64_t* d_obj, uint32_t count, void* h_buf,
                   size_t h_bytes, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        const uint64_t w = wire_words(c, kind, aux);
        KB_REQUIRE(w, KBFV_ERR_INVALID, "unknown object kind for this context");
        KB_REQUIRE(d_obj && h_buf, KBFV_ERR_INVALID, "null argument");
        const size_t need = sizeof(WireHeader) + (size_t)w * count * 8;
        KB_REQUIRE(h_bytes >= need, KBFV_ERR_INVALID, "buffer too small");
        WireHeader hd{};
        std::memcpy(hd.magic, "KBFVWIRE", 8);
        hd.version = 1;
        hd.kind = (uint32_t)kind;
        hd.log_n = (uint32_t)c.logn;
        hd.q_count = (uint32_t)c.nq;
        hd.p_count = (uint32_t)c.np;
        hd.count = count;
        hd.aux = aux;
        hd.prime_digest = prime_digest(c);
        hd.words = w;
        std::memcpy(h_buf, &hd, sizeof hd);
        KB_CHECK_CUDA(cudaMemcpyAsync((uint8_t*)h_buf + sizeof hd, d_obj, (size_t)w * count * 8, cudaMemcpyDeviceToHost,
                                      S(stream)));
        KB_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
    });
}

int kbfv_wire_load(kbfv_context* ctx, int kind, const void* h_buf, size_t h_bytes, uint64_t* d_obj, uint32_t max_count,
                   uint32_t* count, uint64_t* aux, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(h_buf && d_obj, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(h_bytes >= sizeof(WireHeader), KBFV_ERR_INVALID, "truncated header");
        WireHeader hd;
        std::memcpy(&hd, h_buf, sizeof hd);
        KB_REQUIRE(std::memcmp(hd.magic, "KBFVWIRE", 8) == 0 && hd.version == 1, KBFV_ERR_INVALID,
                   "not a version-1 kbfv wire object");
        KB_REQUIRE((int)hd.kind == kind, KBFV_ERR_INVALID, "object kind differs from the requested one");
        KB_REQUIRE(hd.log_n == (uint32_t)c.logn && hd.q_count == (uint32_t)c.nq && hd.p_count == (uint32_t)c.np &&
                       hd.prime_digest == prime_digest(c),
                   KBFV_ERR_INVALID, "object was written for another parameter set or level");
        const uint64_t w = wire_words(c, kind, hd.aux);
        KB_REQUIRE(w && hd.words == w, KBFV_ERR_INVALID, "payload size does not match the parameter set");
        KB_REQUIRE(hd.count <= max_count, KBFV_ERR_INVALID, "more objects than the destination holds");
        KB_REQUIRE(h_bytes >= sizeof hd + (size_t)w * hd.count * 8, KBFV_ERR_INVALID, "truncated payload");
        KB_CHECK_CUDA(cudaMemcpyAsync(d_obj, (const uint8_t*)h_buf + sizeof hd, (size_t)w * hd.count * 8,
                                      cudaMemcpyHostToDevice, S(stream)));
        KB_CHECK_CUDA(cudaStreamSynchronize(S(stream)));
        if (count) *count = hd.count;
        if (aux) *aux = hd.aux;
    });
}


int kbfv_sample_compat(kbfv_context* ctx, int kind, const void* d_rand, uint64_t* d_out, uint32_t prime0,
                       uint32_t limbs, uint32_t h, double probability, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_rand && d_out, KBFV_ERR_INVALID, "null argument");
        KB_REQUIRE(limbs >= 1 && prime0 + limbs <= c.mods.size(), KBFV_ERR_INVALID, "prime range out of table");
        cudaStream_t st = S(stream);
        const size_t n = c.n;
        switch (kind) {
            case 0:
                compat_uniform_kernel<<<blocks_for(limbs * n, 256), 256, 0, st>>>(
                    c.dc, (const uint64_t*)d_rand, d_out, (int)prime0, limbs * n);
                break;
            case 1:
                compat_gauss_kernel<<<blocks_for(n, 256), 256, 0, st>>>(c.dc, (const uint32_t*)d_rand, d_out,
                                                                       (int)prime0, (int)limbs);
                break;
            case 2:
                compat_zo_kernel<<<blocks_for(n, 256), 256, 0, st>>>(c.dc, (const uint8_t*)d_rand, d_out, (int)prime0,
                                                                    (int)limbs, probability);
                break;
            case 3:
                KB_REQUIRE(h >= 1 && h <= 1024 && h <= n, KBFV_ERR_INVALID, "Hamming weight out of range");
                KB_CHECK_CUDA(cudaMemsetAsync(d_out, 0, limbs * n * 8, st));
                compat_hwt_kernel<<<limbs, h, 0, st>>>(c.dc, (const uint8_t*)d_rand, d_out, (int)prime0, (int)h);
                break;
            default:
                throw KbfvError(KBFV_ERR_INVALID, "unknown sampler kind");
        }
        check_launch("sample_compat");
    });
}


// ---- batches at arbitrary addresses (HOST arrays of device pointers) ---------
int kbfv_encrypt_batch(kbfv_context* ctx, const uint8_t seed[32], const uint64_t* enc_ids, const uint64_t* d_pk,
                       const uint64_t* const* d_m, uint64_t* const* d_ct, uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_top(c);
        if (!seed) seed = c.seed;
        KB_REQUIRE(enc_ids && d_pk && d_m && d_ct, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            PtrBatch pb = make_batch(d_m + off, d_m + off, d_ct + off, cnt);
            IdTable ids{};
            for (int i = 0; i < cnt; i++) ids.v[i] = enc_ids[off + i];
            uint64_t* work = (uint64_t*)ensure_scratch(c, (size_t)cnt * 4 * lq * 8);
            const size_t per = c.n / 16, per8 = c.n / 8;
            const SalsaKey kv = subkey_for(seed, DOM_ENC_V, 0), k0 = subkey_for(seed, DOM_ENC_E0, 0),
                           k1 = subkey_for(seed, DOM_ENC_E1, 0);
            sample_small_ids_kernel<0><<<blocks_for(per * cnt, 128), 128, 0, st>>>(c.dc, kv, ids, 0, c.nq, work, 4 * lq, cnt);
            sample_small_ids_kernel<1><<<blocks_for(per8 * cnt, 128), 128, 0, st>>>(c.dc, k0, ids, 0, c.nq, work + lq, 4 * lq, cnt);
            sample_small_ids_kernel<1><<<blocks_for(per8 * cnt, 128), 128, 0, st>>>(c.dc, k1, ids, 0, c.nq, work + 2 * lq, 4 * lq, cnt);
            check_launch("sample_small");
            const size_t total = (size_t)cnt * lq;
            delta_m_ptr_kernel<<<stride_blocks(total, 256), 256, 0, st>>>(c.dc, pb, work, total);
            check_launch("delta_m");
            RowsIO io = rows_io(c.dc, work, 0, c.nq);
            ntt_fwd(c.dc, io, io, cnt * 4 * c.nq, st);
            enc_combine_ptr_kernel<<<stride_blocks(total, 256), 256, 0, st>>>(c.dc, d_pk, work, pb, total);
            check_launch("enc_combine");
        }
    });
}

int kbfv_decrypt_batch(kbfv_context* ctx, const uint64_t* d_sk, const uint64_t* const* d_ct, uint64_t* const* d_m,
                       uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        require_batchable(c);
        KB_REQUIRE(d_sk && d_ct && d_m, KBFV_ERR_INVALID, "null argument");
        cudaStream_t st = S(stream);
        const size_t lq = (size_t)c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            PtrBatch pb = make_batch(d_ct + off, d_ct + off, d_m + off, cnt);
            uint64_t* work = (uint64_t*)ensure_scratch(c, (size_t)cnt * lq * 8);
            ntt_inv(c.dc, DecSrcP{pb, d_sk, c.dc}, rows_io(c.dc, work, 0, c.nq), cnt * c.nq, st);
            dim3 grid((unsigned)(c.n / 128), (unsigned)cnt);
#define L_DR(M) decrypt_round_ptr_kernel<M><<<grid, 128, 0, st>>>(c.dc, work, pb)
            DISPATCH_MAXQ(c.nq, L_DR);
#undef L_DR
            check_launch("decrypt_round");
        }
    });
}

int kbfv_add_batch(kbfv_context* ctx, const uint64_t* const* d_x, const uint64_t* const* d_y, uint64_t* const* d_out,
                   uint32_t count, kbfv_stream stream) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_x && d_y && d_out, KBFV_ERR_INVALID, "null argument");
        const size_t per = (size_t)2 * c.nq * c.n;
        for (uint32_t off = 0; off < count; off += kMaxBatch) {
            const int cnt = (int)std::min<uint32_t>(kMaxBatch, count - off);
            PtrBatch pb = make_batch(d_x + off, d_y + off, d_out + off, cnt);
            add_ptr_kernel<<<dim3(blocks_for(per, 256), (unsigned)cnt), 256, 0, S(stream)>>>(c.dc, pb, per);
            check_launch("add_batch");
        }
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// allocation-free multiply: scratch in a static device array
// ---------------------------------------------------------------------------
static __device__ __align__(256) uint8_t g_noalloc_scratch[KBFV_NOALLOC_SCRATCH_BYTES];
static std::mutex g_noalloc_mu;
constexpr int kMaxDevices = 64;
static void* g_noalloc_addr[kMaxDevices];

// Device address of the static scratch on the current device, resolved once per
// device (the host-side symbol is only a handle, never a device address).
static uint8_t* noalloc_scratch(int device) {
    KB_REQUIRE(device >= 0 && device < kMaxDevices, KBFV_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            throw KbfvError(KBFV_ERR_CUDA, std::string("cudaGetSymbolAddress(static scratch): ") + cudaGetErrorString(e));
        g_noalloc_addr[device] = p;
    }
    return (uint8_t*)g_noalloc_addr[device];
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
        MulScratch m = mul_scratch_layout(c, (int)count, noalloc_scratch(dev));
        // every scratch word is written before it is read: nothing to clear
        PtrBatch pb;
        std::memset(&pb, 0, sizeof pb);
        const size_t stride = (size_t)2 * c.nq * c.n;
        for (uint32_t i = 0; i < count; i++) {
            pb.a[i] = d_ct_a + i * stride;
            pb.b[i] = d_ct_b + i * stride;
            pb.o[i] = d_out + i * stride;
        }
        mul_relin_chunk(c, d_rlk, pb, (int)count, m, S(stream));
    });
}

int kbfv_noise_budget(kbfv_context* ctx, const uint64_t* d_sk, const uint64_t* d_ct, double* bits) {
    return guarded([&] {
        Context& c = CX(ctx);
        KB_REQUIRE(d_sk && d_ct && bits, KBFV_ERR_INVALID, "null argument");
        const size_t lq = (size_t)c.nq * c.n;
        uint64_t* work = (uint64_t*)ensure_scratch(c, lq * 8);
        ntt_inv(c.dc, DecSrc{d_ct, d_sk, c.dc}, rows_io(c.dc, work, 0, c.nq), c.nq, 0);
        std::vector<uint64_t> x(lq);
        KB_CHECK_CUDA(cudaMemcpy(x.data(), work, lq * 8, cudaMemcpyDeviceToHost));
        // CRT reconstruction of t * x, centred; budget = log2 Q - log2 max - 1
        H::Big Q(1);
        for (int i = 0; i < c.nq; i++) Q.mul_word(c.mods[i]);
        H::Big half = Q.div_word(2);
        std::vector<H::Big> hats(c.nq);
        for (int i = 0; i < c.nq; i++) {
            hats[i] = H::Big(1);
            for (int k = 0; k < c.nq; k++) if (k != i) hats[i].mul_word(c.mods[k]);
        }
        double worst = -INFINITY;
        for (uint64_t k = 0; k < c.n; k++) {
            H::Big z(0);
            for (int i = 0; i < c.nq; i++) {
                const uint64_t q = c.mods[i];
                uint64_t y = H::mulmod(H::mulmod(x[(size_t)i * c.n + k], c.t % q, q), c.h_q2r_hatinv[i], q);
                H::Big term = hats[i];
                term.mul_word(y);
                z.add(term);
            }
            while (z.cmp(Q) >= 0) z.sub(Q);
            if (z.cmp(half) > 0) { H::Big w = Q; w.sub(z); z = w; }
            worst = std::max(worst, z.log2v());
        }
        *bits = Q.log2v() - worst - 1.0;
    });
}

int kbfv_salsa20_stream(const uint8_t key[32], const uint8_t nonce[24], uint64_t block0, uint8_t* d_out, size_t nbytes,
                        int compat, kbfv_stream stream) {
    return guarded([&] {
        KB_REQUIRE(key && nonce && d_out, KBFV_ERR_INVALID, "null argument");
        SalsaKey k;
        uint32_t n0, n1;
        size_t len = nbytes;
        if (compat) {
            // the reference's VecCrypt: zero constants, raw key, nonce word 1 always 0,
            // partial tail block left zero (include/RNG.cuh:18-51, include/RNG_impl.cuh:70-176)
            for (int i = 0; i < 8; i++) k.k[i] = ld32(key + 4 * i);
            for (int i = 0; i < 4; i++) k.sigma[i] = 0;
            n0 = ld32(nonce);
            n1 = 0;
            KB_CHECK_CUDA(cudaMemsetAsync(d_out, 0, nbytes, S(stream)));
            len = nbytes / 64 * 64;
        } else {
            hsalsa_host(key, nonce, k.k);
            static const char* sig = "expand 32-byte k";
            for (int i = 0; i < 4; i++) std::memcpy(&k.sigma[i], sig + 4 * i, 4);
            n0 = ld32(nonce + 16);
            n1 = ld32(nonce + 20);
        }
        if (!len) return;
        const size_t blocks = (len + 63) / 64;
        salsa_stream_kernel<<<blocks_for(blocks, 128), 128, 0, S(stream)>>>(k, n0, n1, block0, d_out, len);
        check_launch("salsa20");
    });
}

}  // extern "C"
