"""Keys, encryption, decryption and the multiply path on the B200 vs the oracle.

Bit-exact ciphertext parity (same seed -> same keys and ciphertexts), exact
decryption of m1*m2 mod t, and batch-vs-alone determinism."""
import numpy as np
import pytest

from tests.gpu_util import c3_pair, dev, host, small_pair

pytestmark = pytest.mark.gpu

T = 65537
SEED = bytes(range(32))


def setup(ctx, orc, kind=0):
    import kunpbfv_b200 as kb
    sk = kb.SecretKey(ctx, SEED, kind=kind)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    osk = orc.keygen_secret(SEED, kind)
    return sk, sch, osk


@pytest.mark.parametrize("which", ["c3", "small", "dnum2"])
def test_keys_bit_exact(which):
    ctx, orc = {"c3": c3_pair, "small": lambda: small_pair(12, 3, 1, 50),
                "dnum2": lambda: small_pair(12, 4, 2, 45, 2)}[which]()
    sk, sch, osk = setup(ctx, orc)
    assert np.array_equal(host(sk.sx_device).reshape(osk.shape), osk)
    opk = orc.keygen_public(SEED, osk)
    assert np.array_equal(host(sch.publicKey).reshape(opk.shape), opk)
    orlk = orc.keygen_relin(SEED, osk)
    assert np.array_equal(host(sch.rlk).reshape(orlk.shape), orlk)


def test_hwt_secret_bit_exact():
    import kunpbfv_b200 as kb
    ctx, orc = small_pair(12, 3, 1, 50)
    sk = kb.SecretKey(ctx, SEED, kind=1, h=64)
    assert np.array_equal(host(sk.sx_device).reshape(-1, ctx.N), orc.keygen_secret(SEED, 1, 64))


def test_encrypt_decrypt_bit_exact():
    import kunpbfv_b200 as kb
    ctx, orc = c3_pair()
    sk, sch, osk = setup(ctx, orc)
    opk = orc.keygen_public(SEED, osk)
    rng = np.random.default_rng(2)
    v = rng.integers(0, T, size=(3, ctx.N), dtype=np.uint64)
    m = host(ctx.encode(dev(v))).reshape(v.shape)
    ct = sch.encryptMsg(kb.Plaintext(ctx, dev(m)), enc_id=100)
    got = host(ct.cipher_device).reshape(3, 2, ctx.q_count, ctx.N)
    for i in range(3):
        assert np.array_equal(got[i], orc.encrypt(SEED, 100 + i, opk, m[i]))
    pt = sch.decryptMsg(sk, ct)
    dm = host(pt.mx_device).reshape(3, ctx.N)
    for i in range(3):
        assert np.array_equal(dm[i], orc.decrypt(osk, got[i]))
    assert np.array_equal(host(ctx.decode(pt.mx_device)).reshape(v.shape), v)


@pytest.mark.parametrize("which", ["c3", "small", "dnum2"])
def test_mul_relin_bit_exact_and_decrypts(which):
    import kunpbfv_b200 as kb
    ctx, orc = {"c3": c3_pair, "small": lambda: small_pair(12, 3, 1, 50),
                "dnum2": lambda: small_pair(12, 4, 2, 45, 2)}[which]()
    sk, sch, osk = setup(ctx, orc)
    orlk = orc.keygen_relin(SEED, osk)
    rng = np.random.default_rng(3)
    k = 3
    v1 = rng.integers(0, T, size=(k, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, T, size=(k, ctx.N), dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=0)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=k)
    out = sch.mult_relin(c1, c2)
    h1 = host(c1.cipher_device).reshape(k, 2, ctx.q_count, ctx.N)
    h2 = host(c2.cipher_device).reshape(k, 2, ctx.q_count, ctx.N)
    ho = host(out.cipher_device).reshape(k, 2, ctx.q_count, ctx.N)
    for i in range(k):
        assert np.array_equal(ho[i], orc.mul_relin(h1[i], h2[i], orlk)), f"pair {i}"
    dec = host(ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(k, ctx.N)
    assert np.array_equal(dec, (v1 * v2) % T)
    # split form: tensor then relinearise
    t3 = sch.mult(c1, c2)
    ht = host(t3.data).reshape(k, 3, ctx.q_count, ctx.N)
    for i in range(k):
        assert np.array_equal(ht[i], orc.mul_tensor(h1[i], h2[i]))
    assert np.array_equal(host(sch.relinearize(t3).cipher_device).reshape(ho.shape), ho)


def test_batch_equals_alone_and_64_pairs_decrypt():
    """64 pairs in one launch sequence: each result equals the pair run alone,
    and every decryption equals the slot-wise product mod t."""
    import kunpbfv_b200 as kb
    ctx, orc = c3_pair()
    sk, sch, osk = setup(ctx, orc)
    rng = np.random.default_rng(4)
    B = 64
    v1 = rng.integers(0, T, size=(B, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, T, size=(B, ctx.N), dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=1000)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=2000)
    out = sch.mult_relin(c1, c2)
    dec = host(ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(B, ctx.N)
    assert np.array_equal(dec, (v1 * v2) % T)
    ho = host(out.cipher_device).reshape(B, 2, ctx.q_count, ctx.N)
    lq = 2 * ctx.q_count * ctx.N
    for i in (0, 31, 63):
        a = kb.Ciphertext(ctx, c1.cipher_device.view(-1)[i * lq:(i + 1) * lq].clone())
        b = kb.Ciphertext(ctx, c2.cipher_device.view(-1)[i * lq:(i + 1) * lq].clone())
        alone = host(sch.mult_relin(a, b).cipher_device).reshape(2, ctx.q_count, ctx.N)
        assert np.array_equal(alone, ho[i])
    assert sch.noise_budget(sk, kb.Ciphertext(ctx, out.cipher_device.view(-1)[:lq].clone())) > 10


def test_mul_plain_and_add():
    import kunpbfv_b200 as kb
    ctx, orc = c3_pair()
    sk, sch, osk = setup(ctx, orc)
    rng = np.random.default_rng(5)
    v1 = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
    v2 = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))))
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))))
    s = sch.add(c1, c2)
    assert np.array_equal(host(ctx.decode(sch.decryptMsg(sk, s).mx_device)).reshape(-1), (v1 + v2) % T)
    # encode_ntt takes plaintext coefficients (the reference's encode mutates its input into them)
    pt = ctx.encode_ntt(ctx.encode(dev(v2)))
    sch.multConstAndEqual(c1, pt)
    assert np.array_equal(host(ctx.decode(sch.decryptMsg(sk, c1).mx_device)).reshape(-1), (v1 * v2) % T)


def test_errors_are_reported():
    import kunpbfv_b200 as kb
    ctx, orc = small_pair(12, 3, 1, 50)
    sch = kb.BFVScheme(ctx, SEED)
    c = kb.Ciphertext(ctx)
    with pytest.raises(kb.KbfvError):
        sch.mult_relin(c, c)   # no relinearisation key
    with pytest.raises(ValueError):
        kb.BFVContext(log_n=12, plain_modulus=65537, q_count=0)


def test_c1_end_to_end():
    """N=4096 with 36+36-bit ciphertext primes and a 37-bit special prime,
    t=65537, ternary secret, Gaussian error, dnum=2; batch size 1. The context
    is built from bit sizes (kbfv_params_create) and must pick the oracle's
    primes; keys, encryptions and the product are bit-exact, decryption exact."""
    import kunpbfv_b200 as kb
    import oracle
    from tests.params import c1_primes
    qs, ps = c1_primes()
    ctx = kb.BFVContext.from_bits(12, [36, 36], [37], T, dnum=2)
    assert ctx.q == qs and ctx.p == ps
    orc = oracle.Oracle(12, T, qs, ps, dnum=2)
    sk, sch, osk = setup(ctx, orc)
    opk, orlk = orc.keygen_public(SEED, osk), orc.keygen_relin(SEED, osk)
    assert np.array_equal(host(sch.rlk).reshape(orlk.shape), orlk)
    rng = np.random.default_rng(41)
    v1 = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
    v2 = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=0)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=1)
    h1 = host(c1.cipher_device).reshape(2, 2, ctx.N)
    assert np.array_equal(h1, orc.encrypt(SEED, 0, opk, orc.encode(v1)))
    h2 = host(c2.cipher_device).reshape(2, 2, ctx.N)
    out = sch.mult_relin(c1, c2)
    assert np.array_equal(host(out.cipher_device).reshape(2, 2, ctx.N), orc.mul_relin(h1, h2, orlk))
    dec = host(ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(-1)
    assert np.array_equal(dec, (v1 * v2) % T)
    assert sch.noise_budget(sk, out) > 10


def test_add_plain_bit_exact():
    """addConstAndEqual: b += NTT(Delta * m)."""
    import kunpbfv_b200 as kb
    ctx, orc = c3_pair()
    sk, sch, osk = setup(ctx, orc)
    rng = np.random.default_rng(6)
    v1 = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
    c = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=500)
    before = host(c.cipher_device).reshape(2, 2, ctx.q_count, ctx.N)
    m2 = ctx.encode(dev(v2))
    sch.addConstAndEqual(c, kb.Plaintext(ctx, m2))
    after = host(c.cipher_device).reshape(2, 2, ctx.q_count, ctx.N)
    hm = host(m2).reshape(2, ctx.N)
    for i in range(2):
        dm = orc.delta_m(hm[i])
        add = np.stack([orc.ntt_fwd(l, dm[l]) for l in range(ctx.q_count)])
        want = orc.add(before[i], np.stack([np.zeros_like(add), add]))
        assert np.array_equal(after[i], want)
    dec = host(ctx.decode(sch.decryptMsg(sk, c).mx_device)).reshape(2, ctx.N)
    assert np.array_equal(dec, (v1 + v2) % T)


def test_ntt_batch_pointer_arrays():
    """kbfv_ntt_fwd_batch / inv_batch over polynomials at separate addresses."""
    from tests.gpu_util import rand_rows
    ctx, orc = c3_pair()
    polys = [rand_rows(orc, range(ctx.q_count), ctx.N, 60 + i) for i in range(3)]
    d = [dev(p) for p in polys]
    ctx.ntt_fwd_batch(d, ctx.q_count, 0)
    for p, x in zip(polys, d):
        want = np.stack([orc.ntt_fwd(l, p[l]) for l in range(ctx.q_count)])
        assert np.array_equal(host(x).reshape(want.shape), want)
    ctx.ntt_inv_batch(d, ctx.q_count, 0)
    for p, x in zip(polys, d):
        assert np.array_equal(host(x).reshape(p.shape), p)


def test_linear_ops_and_square():
    """sub, negate, scalar multiply (+add), square: decryptions exact, and the
    limb-wise ops equal the oracle's arithmetic on the same ciphertexts."""
    import kunpbfv_b200 as kb
    ctx, orc = c3_pair()
    sk, sch, osk = setup(ctx, orc)
    rng = np.random.default_rng(8)
    v1 = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
    v2 = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=31)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=32)
    dec = lambda c: host(ctx.decode(sch.decryptMsg(sk, c).mx_device)).reshape(-1)
    vo = lambda x: x.astype(object)
    d = sch.sub(c1, c2)
    assert np.array_equal(dec(d), ((vo(v1) - vo(v2)) % T).astype(np.uint64))
    h1 = host(c1.cipher_device).reshape(2, ctx.q_count, ctx.N)
    h2 = host(c2.cipher_device).reshape(2, ctx.q_count, ctx.N)
    qs = np.array(ctx.q, dtype=object).reshape(1, -1, 1)
    assert np.array_equal(host(d.cipher_device).reshape(h1.shape), ((vo(h1) - vo(h2)) % qs).astype(np.uint64))
    n = kb.Ciphertext(ctx, c1.cipher_device.clone())
    sch.negateAndEqual(n)
    assert np.array_equal(dec(n), ((-vo(v1)) % T).astype(np.uint64))
    s = kb.Ciphertext(ctx, c1.cipher_device.clone())
    sch.multScalarAndEqual(s, 12345)
    assert np.array_equal(dec(s), (vo(v1) * 12345 % T).astype(np.uint64))
    assert np.array_equal(host(s.cipher_device).reshape(h1.shape), (vo(h1) * 12345 % qs).astype(np.uint64))
    a = kb.Ciphertext(ctx, c1.cipher_device.clone())
    sch.multConstAndAddCipherEqual(a, c2, 7)
    assert np.array_equal(dec(a), ((vo(v1) + 7 * vo(v2)) % T).astype(np.uint64))
    q = kb.Ciphertext(ctx, c1.cipher_device.clone())
    sch.squareAndEqual(q)
    assert np.array_equal(dec(q), (vo(v1) * vo(v1) % T).astype(np.uint64))
    assert np.array_equal(host(q.cipher_device), host(sch.mult_relin(c1, c1).cipher_device))


def test_pointer_batches_equal_contiguous_calls():
    """kbfv_encrypt_batch / decrypt_batch / add_batch over scattered buffers equal
    the contiguous calls item by item."""
    import ctypes as C

    import kunpbfv_b200 as kb
    from kunpbfv_b200.api import _ptr, _u8, lib
    ctx, orc = c3_pair()
    sk, sch, osk = setup(ctx, orc)
    rng = np.random.default_rng(12)
    v = rng.integers(0, T, size=(3, ctx.N), dtype=np.uint64)
    m = [ctx.encode(dev(v[i])) for i in range(3)]
    ids = [77, 5, 1234]
    outs = [kb.Ciphertext(ctx) for _ in range(3)]
    VP = C.c_void_p
    rc = lib().kbfv_encrypt_batch(ctx.handle, _u8(SEED), (C.c_uint64 * 3)(*ids), _ptr(sch.publicKey),
                                  (VP * 3)(*[_ptr(x) for x in m]), (VP * 3)(*[_ptr(o.cipher_device) for o in outs]),
                                  3, None)
    assert rc == 0
    for i in range(3):
        alone = sch.encryptMsg(kb.Plaintext(ctx, m[i]), enc_id=ids[i])
        assert np.array_equal(host(outs[i].cipher_device), host(alone.cipher_device)), i
    sums = [kb.Ciphertext(ctx) for _ in range(2)]
    rc = lib().kbfv_add_batch(ctx.handle, (VP * 2)(_ptr(outs[0].cipher_device), _ptr(outs[1].cipher_device)),
                              (VP * 2)(_ptr(outs[2].cipher_device), _ptr(outs[0].cipher_device)),
                              (VP * 2)(*[_ptr(s.cipher_device) for s in sums]), 2, None)
    assert rc == 0
    assert np.array_equal(host(sums[0].cipher_device), host(sch.add(outs[0], outs[2]).cipher_device))
    res = [ctx.zeros(ctx.N) for _ in range(2)]
    rc = lib().kbfv_decrypt_batch(ctx.handle, _ptr(sk.sx_device), (VP * 2)(*[_ptr(s.cipher_device) for s in sums]),
                                  (VP * 2)(*[_ptr(r) for r in res]), 2, None)
    assert rc == 0
    assert np.array_equal(host(ctx.decode(res[0])).reshape(-1), (v[0] + v[2]) % T)
    assert np.array_equal(host(ctx.decode(res[1])).reshape(-1), (v[1] + v[0]) % T)


def test_sub_batches_on_streams_identical():
    """A 40-pair batch run as 1, 2, 3 or 4 sub-batches on forked streams gives
    identical ciphertexts, also when captured into a CUDA graph."""
    import torch

    import kunpbfv_b200 as kb
    ctx, orc = c3_pair()
    sk, sch, osk = setup(ctx, orc)
    rng = np.random.default_rng(21)
    B = 40
    v1 = rng.integers(0, T, size=(B, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, T, size=(B, ctx.N), dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=3000)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=4000)
    outs = []
    try:
        for nb in (1, 2, 3, 4):
            ctx.set_branches(nb)
            outs.append(host(sch.mult_relin(c1, c2).cipher_device))
        for o in outs[1:]:
            assert np.array_equal(o, outs[0])
        ctx.set_branches(2)
        st = torch.cuda.Stream()
        out = kb.Ciphertext(ctx, count=B)
        with torch.cuda.stream(st):
            sch.mult_relin(c1, c2, out=out, stream=st)  # warm-up outside the capture
        torch.cuda.synchronize()
        out.cipher_device.zero_()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=st):
            sch.mult_relin(c1, c2, out=out, stream=st)
        g.replay()
        torch.cuda.synchronize()
        assert np.array_equal(host(out.cipher_device), outs[0])
        dec = host(ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(B, ctx.N)
        assert np.array_equal(dec, (v1 * v2) % T)
    finally:
        ctx.set_branches(2)
    with pytest.raises(kb.KbfvError):
        ctx.set_branches(5)
