// libkbfv: context construction (parameter tables in one device pool), the
// scratch arena, parameter sets, tuning knobs, the arithmetic-rate probe, the
// noise budget and the wire format.
#include "pipeline.cuh"

thread_local std::string g_last_error;

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

void build_context(Context& c, const kbfv_params& prm) {
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
    // two coefficients per base-conversion thread: 16% fewer IMAD instructions,
    // 8% faster than one at N=16384, 7 + 1 primes, 32-pair sub-batches (B200)
    dc.shape = LaunchShape{kSplitRows14Default, 256, 2, 128, 2, 1, 1, kSplitRowsAloneDefault};
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
    // last-stage constants of the inverse NTT over Q scaled by (Q/q_i)^-1: the
    // transform then stores the base extension's y_i = [x_i (Q/q_i)^-1]_{q_i}
    std::vector<tw_t> q2r_fold((size_t)2 * c.nq);
    for (int i = 0; i < c.nq; i++) {
        const uint64_t q = c.mods[i];
        for (int k = 0; k < 2; k++) {
            const uint64_t v = H::mulmod(twi[((size_t)i << c.logn) + k].x, q2r.hatinv[i], q);
            q2r_fold[2 * i + k].x = v;
            q2r_fold[2 * i + k].y = H::shoup(v, q);
        }
    }
    size_t o_q2rf = blob.add(q2r_fold);
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
    dc.q2r_fold = (const tw_t*)(base + o_q2rf);
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
// scratch
// ===========================================================================
uint8_t* ensure_scratch(Context& c, size_t bytes) {
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

// ---- arithmetic-rate probe: independent register chains of one primitive -------
// kind 0: 64x64->128 multiply-accumulate, 1: mul.lo.u64, 2: mul.hi.u64,
// 3: forward butterfly with the approximate-quotient Shoup product from 64-bit
// multiplies (shoup4_64), 4: fully reduced Shoup,
// 5: 128-bit Barrett, 6: one-high-product Barrett, 7: 32x32->64 multiply-add,
// 8: 32x32 high product, 9: 32-bit multiply-add, 10: mac32 (64x64->128
// multiply-accumulate from 32-bit partial products), 11: forward butterfly
// with shoup4_32 (the NTT kernels' butterfly), 12: 32-bit multiply-add issue
// rate (16 dependent mad.lo.u32 per chain step, the IMAD pipe's peak),
// 13: 32x32->64 multiply-add issue rate (16 dependent mad.wide.u32 per step),
// 14: 60x60-bit multiply-accumulate from 30-bit halves (mac30: four
// mad.wide.u32 into three 64-bit column sums), 15: 32-bit high multiply-add
// issue rate (16 dependent mad.hi.u32 per step).
constexpr int kProbeChains = 8;
constexpr int kImadPerStep = 16;
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
            if (KIND == 12) {  // IMAD issue: 16 multiply-adds per chain step, one bookkeeping update
                uint32_t x = (uint32_t)acc[c].lo;
                const uint32_t m = (uint32_t)b[c] | 1u, k = (uint32_t)a[c];
#pragma unroll
                for (int u = 0; u < kImadPerStep; u++) x = x * m + k;
                acc[c].lo = x;
            }
            if (KIND == 13) {  // wide multiply-add issue: x = lo32(x) * m + x (64-bit)
                uint64_t x = acc[c].lo;
                const uint32_t m = (uint32_t)b[c] | 1u;
#pragma unroll
                for (int u = 0; u < kImadPerStep; u++)
                    asm("mad.wide.u32 %0, %1, %2, %0;" : "+l"(x) : "r"((uint32_t)x), "r"(m));
                acc[c].lo = x;
            }
            if (KIND == 14) {  // mac30: columns lo (a0 b0), mid (a0 b1 + a1 b0), hi (a1 b1)
                constexpr uint64_t M30 = (1ULL << 30) - 1;
                const uint32_t a0 = (uint32_t)(a[c] & M30), a1 = (uint32_t)(a[c] >> 30);
                const uint32_t b0 = (uint32_t)(b[c] & M30), b1 = (uint32_t)(b[c] >> 30);
                uint64_t lo = acc[c].lo, hi = acc[c].hi, mid = lo ^ hi;
                asm("mad.wide.u32 %0, %3, %5, %0;\n\t"
                    "mad.wide.u32 %1, %3, %6, %1;\n\t"
                    "mad.wide.u32 %1, %4, %5, %1;\n\t"
                    "mad.wide.u32 %2, %4, %6, %2;"
                    : "+l"(lo), "+l"(mid), "+l"(hi)
                    : "r"(a0), "r"(a1), "r"(b0), "r"(b1));
                acc[c].lo = lo + (mid << 30);
                acc[c].hi = hi + (mid >> 34);
            }
            if (KIND == 15) {  // high multiply-add issue: x = hi32(x * m) + k
                uint32_t x = (uint32_t)acc[c].lo;
                const uint32_t m = (uint32_t)b[c] | 0x80000001u, k = (uint32_t)a[c];
#pragma unroll
                for (int u = 0; u < kImadPerStep; u++) asm("mad.hi.u32 %0, %0, %1, %2;" : "+r"(x) : "r"(m), "r"(k));
                acc[c].lo = x;
            }
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
        if (c.d_level_consts) cudaFree(c.d_level_consts);
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

size_t kbfv_context_arena_bytes(const kbfv_context* ctx) { return ctx ? ctx->c.scratch_bytes : 0; }

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
            case KBFV_TUNE_SPLIT_ROWS:
                KB_REQUIRE(value >= 0 && value <= (1 << 20), KBFV_ERR_INVALID, "split rows must be 0..2^20");
                c.dc.shape.split_rows14 = (int)value;
                break;
            case KBFV_TUNE_BCONV_THREADS:
                KB_REQUIRE(value == 64 || value == 128 || value == 256 || value == 512, KBFV_ERR_INVALID,
                           "base-conversion CTA size must be 64, 128, 256 or 512");
                c.dc.shape.bconv_threads = (int)value;
                break;
            case KBFV_TUNE_K5_THREADS:
                KB_REQUIRE(value == 64 || value == 128 || value == 256, KBFV_ERR_INVALID,
                           "K5 CTA size must be 64, 128 or 256");
                c.dc.shape.k5_threads = (int)value;
                break;
            case KBFV_TUNE_K5_FUSED_PAIRS:
                KB_REQUIRE(value >= 0 && value <= kMaxBatch, KBFV_ERR_INVALID, "K5 fused pairs must be 0..128");
                c.dc.shape.k5_fused_pairs = (int)value;
                break;
            case KBFV_TUNE_BCONV_CPT:
                KB_REQUIRE(value == 1 || value == 2, KBFV_ERR_INVALID, "base-conversion coefficients per thread: 1 or 2");
                c.dc.shape.bconv_cpt = (int)value;
                break;
            case KBFV_TUNE_FUSE_Q2R_PAIRS:
                KB_REQUIRE(value >= 0 && value <= kMaxBatch, KBFV_ERR_INVALID, "fused Q -> R pairs must be 0..128");
                c.dc.shape.fuse_q2r_pairs = (int)value;
                break;
            case KBFV_TUNE_L2_PREFETCH:
                KB_REQUIRE(value == 0 || value == 1, KBFV_ERR_INVALID, "L2 prefetch: 0 or 1");
                c.dc.shape.l2_prefetch = (int)value;
                break;
            case KBFV_TUNE_SPLIT_ROWS_ALONE:
                KB_REQUIRE(value >= 0 && value <= (1 << 20), KBFV_ERR_INVALID, "split rows (one stream) must be 0..2^20");
                c.dc.shape.split_rows_alone = (int)value;
                break;
            case KBFV_TUNE_MIN_BRANCH_PAIRS:
                KB_REQUIRE(value >= 1 && value <= 64, KBFV_ERR_INVALID, "pairs per sub-batch must be 1..64");
                c.min_branch_pairs = (int)value;
                break;
            default: throw KbfvError(KBFV_ERR_INVALID, "unknown tuning knob");
        }
        // the levels of a top context run with the top level's knobs
        for (void* lv : c.levels) {
            if (!lv) continue;
            Context& l = reinterpret_cast<kbfv_context*>(lv)->c;
            l.dc.shape = c.dc.shape;
            l.branches = c.branches;
            l.min_branch_pairs = c.min_branch_pairs;
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
            case KBFV_TUNE_SPLIT_ROWS: *value = c.dc.shape.split_rows14; break;
            case KBFV_TUNE_BCONV_THREADS: *value = c.dc.shape.bconv_threads; break;
            case KBFV_TUNE_K5_THREADS: *value = c.dc.shape.k5_threads; break;
            case KBFV_TUNE_K5_FUSED_PAIRS: *value = c.dc.shape.k5_fused_pairs; break;
            case KBFV_TUNE_BCONV_CPT: *value = c.dc.shape.bconv_cpt; break;
            case KBFV_TUNE_FUSE_Q2R_PAIRS: *value = c.dc.shape.fuse_q2r_pairs; break;
            case KBFV_TUNE_L2_PREFETCH: *value = c.dc.shape.l2_prefetch; break;
            case KBFV_TUNE_SPLIT_ROWS_ALONE: *value = c.dc.shape.split_rows_alone; break;
            case KBFV_TUNE_MIN_BRANCH_PAIRS: *value = c.min_branch_pairs; break;
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

int kbfv_probe_arith(int kind, uint32_t iters, double* gops) {
    return guarded([&] {
        KB_REQUIRE(kind >= 0 && kind <= 15 && gops && iters >= 1, KBFV_ERR_INVALID, "bad probe arguments");
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
                P_K(0) P_K(1) P_K(2) P_K(3) P_K(4) P_K(5) P_K(6) P_K(7) P_K(8) P_K(9) P_K(10) P_K(11) P_K(12)
                P_K(13) P_K(14) P_K(15)
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
        const bool issue = kind == 12 || kind == 13 || kind == 15;
        *gops = (double)blocks * threads * iters * kProbeChains * (issue ? kImadPerStep : 1) / (ms * 1e6);
    });
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

}  // extern "C"
