"""The CUDA product against the reference's own kernel outputs (digests in
tests/golden/ref_logn*.json), at the reference's parameter sets."""
import glob
import json
import os

import numpy as np
import pytest

from tests.golden.refgen import digest, gen
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module", params=[14, 15], ids=["logn14", "logn15"])
def ref(request):
    import kunpbfv_b200 as kb
    path = os.path.join(HERE, f"ref_logn{request.param}.json")
    with open(path) as f:
        fx = json.load(f)
    ctx = kb.reference_context(request.param)
    assert ctx.q == fx["qVec"] and ctx.p == fx["pVec"] and ctx.r == fx["rVec"] and ctx.tk == fx["tVec"]
    return ctx, fx


def check(fx, name, arr):
    w = fx["arrays"][name]
    a = np.ascontiguousarray(arr, dtype=np.uint64).reshape(-1)
    assert a.size == w["count"]
    assert digest(a) == w["digest"], f"{name}: GPU head {a[:4].tolist()} vs reference {w['head'][:4]}"


def test_ntt_vs_reference(ref):
    ctx, fx = ref
    n, nq, K, nt = ctx.N, ctx.q_count, ctx.p_count, ctx.t_count
    # reference order [P | Q | T] -> product prime indices
    idx = [ctx.idx_p + i for i in range(K)] + list(range(nq)) + [ctx.idx_t + i for i in range(nt)]
    mods = [ctx.primes[i] for i in idx]
    for seed, name, fwd in ((1, "ntt_pqt_out", True), (2, "intt_pqt_out", False)):
        x = gen(seed, mods, n)
        out = np.empty_like(x)
        for l, i in enumerate(idx):
            d = dev(x[l])
            (ctx.ntt_fwd if fwd else ctx.ntt_inv)(d, i, 1)
            out[l] = host(d)
        check(fx, name, out)
    qr = list(range(nq)) + [ctx.idx_r + j for j in range(ctx.r_count)]
    x = gen(3, [ctx.primes[i] for i in qr], n)
    d = dev(np.concatenate([x[:nq], x[nq:]]))
    # Q rows then R rows: two calls with their own prime offsets
    dq, dr = d.view(-1, n)[:nq], d.view(-1, n)[nq:]
    ctx.ntt_fwd(dq, 0, nq)
    ctx.ntt_fwd(dr, ctx.idx_r, ctx.r_count)
    check(fx, "ntt_qr_out", host(d))


def test_hps_vs_reference(ref):
    ctx, fx = ref
    n = ctx.N
    check(fx, "bconv_qr_out", host(ctx.bconv_q_to_r(dev(gen(7, ctx.q, n)))))
    check(fx, "bconv_rq_out", host(ctx.bconv_r_to_q(dev(gen(8, ctx.r, n)))))
    check(fx, "decr_out", host(ctx.decrypt_round(dev(gen(10, ctx.q, n)))))
    qr = list(ctx.q) + list(ctx.r)
    check(fx, "tensor_out", host(ctx.tensor_qr(dev(gen(11, qr * 2, n)), dev(gen(12, qr * 2, n)))))
    check(fx, "delta_out", host(ctx.delta_m(dev(gen(13, [ctx.plain_modulus], n)))))
    enc = host(ctx.encode(dev(gen(5, [ctx.plain_modulus], n))))
    check(fx, "bfv_enc_out", enc)
    check(fx, "bfv_dec_out", host(ctx.decode(dev(gen(6, [ctx.plain_modulus], n)))))


def test_multiply_vs_reference(ref):
    """At logN=14 the product's HPS tensor and hybrid relinearisation reproduce
    the reference's genuine multiply (compute_t_QInv_c0c1c2 + KLSS key switch)
    bit for bit. At logN=15 the reference's own path is wrong (its scale-round
    reduces alpha in place across R primes and its T base is too small), so
    the product is checked for exact decryption instead (test_gpu_scheme)."""
    import kunpbfv_b200 as kb
    ctx, fx = ref
    if ctx.log_n != 14:
        pytest.skip("the reference's genuine multiply is incorrect at logN=15")
    n, nq, K, dnum = ctx.N, ctx.q_count, ctx.p_count, ctx.dnum
    PQ = list(ctx.p) + list(ctx.q)
    c1 = gen(23, list(ctx.q) * 2, n)
    c2 = gen(24, list(ctx.q) * 2, n)
    sch = kb.BFVScheme(ctx)
    t3 = sch.mult(kb.Ciphertext(ctx, dev(c1)), kb.Ciphertext(ctx, dev(c2)))
    d = host(t3.data).reshape(3, nq, n)
    check(fx, "mult_axax", d[0])
    check(fx, "mult_axbx", d[1])
    check(fx, "mult_bxbx", d[2])
    ka = gen(21, PQ * dnum, n).reshape(dnum, len(PQ), n)
    kb_ = gen(22, PQ * dnum, n).reshape(dnum, len(PQ), n)
    mine = lambda k: np.concatenate([k[:, K:], k[:, :K]], axis=1)
    rlk = np.stack([np.stack([mine(ka)[g], mine(kb_)[g]]) for g in range(dnum)])
    sch.rlk = dev(rlk)
    out = sch.relinearize(t3)
    check(fx, "mult_out", host(out.cipher_device))


def test_sampler_conversions_vs_reference(ref):
    """The reference's sampler conversions restated on the GPU reproduce its
    outputs on the same random words (uniform, Gaussian, ternary, HWT)."""
    ctx, fx = ref
    n, K, nq = ctx.N, ctx.p_count, ctx.q_count
    M = 2**64 - 1

    def both(kind, words, **kw):  # reference order P|Q
        d = dev(words)
        p = host(ctx.sample_compat(kind, d, ctx.idx_p, K, **kw)).reshape(K, n)
        q = host(ctx.sample_compat(kind, d, 0, nq, **kw)).reshape(nq, n)
        return np.concatenate([p, q])

    ru = gen(26, [M] * (K + nq), n)
    check(fx, "samp_uniform_in", ru)
    d = dev(ru)
    p = host(ctx.sample_compat(0, d[:K], ctx.idx_p, K)).reshape(K, n)
    q = host(ctx.sample_compat(0, d[K:], 0, nq)).reshape(nq, n)
    check(fx, "samp_uniform_out", np.concatenate([p, q]))
    check(fx, "samp_gauss_out", both(1, gen(27, [M], n // 2)))
    check(fx, "samp_zo_out", both(2, gen(28, [M], n // 8), probability=0.5))
    check(fx, "samp_hwt_out", both(3, gen(29, [M], 40), h=64))
