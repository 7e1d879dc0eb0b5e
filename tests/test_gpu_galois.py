"""Rotations and conjugation (Galois automorphisms X -> X^g plus key switch)
on the B200 vs the oracle, and the decryption property: the result decrypts to
the plaintext polynomial m(X^g)."""
import numpy as np
import pytest

from tests.gpu_util import c3_pair, dev, host, small_pair

pytestmark = pytest.mark.gpu

T = 65537
SEED = bytes(range(32))


def plain_automorphism(m, g, n, t):
    out = np.zeros(n, dtype=object)
    for i in range(n):
        e = (i * g) % (2 * n)
        if e < n:
            out[e] = (out[e] + int(m[i])) % t
        else:
            out[e - n] = (out[e - n] - int(m[i])) % t
    return out.astype(np.uint64)


@pytest.mark.parametrize("which", ["small", "c3"])
def test_rotation_and_conjugation(which):
    import kunpbfv_b200 as kb
    ctx, orc = {"small": lambda: small_pair(12, 3, 1, 50), "c3": c3_pair}[which]()
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    osk = orc.keygen_secret(SEED)
    rng = np.random.default_rng(3)
    v = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
    ct = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v))), enc_id=900)
    m = host(ctx.encode(dev(v))).reshape(2, ctx.N)
    hct = host(ct.cipher_device).reshape(2, 2, ctx.q_count, ctx.N)
    for rot in (1, 3, -1):
        g = sch.galois_element(rot)
        assert g == (pow(5, rot, 2 * ctx.N) if rot >= 0 else 2 * ctx.N - 1)
        if rot >= 0:
            sch.addLeftRotKey_23(sk, rot)
        else:
            sch.addConjKey_23(sk)
        ogk = orc.keygen_galois(SEED, osk, g)
        assert np.array_equal(host(sch.galois_keys[g]).reshape(ogk.shape), ogk), rot
        out = sch.apply_galois(ct, g)
        got = host(out.cipher_device).reshape(2, 2, ctx.q_count, ctx.N)
        for i in range(2):
            assert np.array_equal(got[i], orc.apply_galois(ogk, g, hct[i])), (rot, i)
        dec = host(ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(2, ctx.N)
        for i in range(2):
            want = orc.decode(plain_automorphism(m[i], g, ctx.N, T))
            assert np.array_equal(dec[i], want), (rot, i)


def test_rotate_in_place_and_compose():
    """leftRotateAndEqual_23 in place; rotating by 1 twice equals rotating by 2."""
    import kunpbfv_b200 as kb
    ctx, orc = small_pair(12, 3, 1, 50)
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addLeftRotKey_23(sk, 1)
    sch.addLeftRotKey_23(sk, 2)
    rng = np.random.default_rng(4)
    v = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
    a = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v))), enc_id=1)
    b = kb.Ciphertext(ctx, a.cipher_device.clone())
    sch.leftRotateAndEqual_23(a, 1)
    sch.leftRotateAndEqual_23(a, 1)
    sch.leftRotateAndEqual_23(b, 2)
    da = host(ctx.decode(sch.decryptMsg(sk, a).mx_device))
    db = host(ctx.decode(sch.decryptMsg(sk, b).mx_device))
    assert np.array_equal(da, db)
    with pytest.raises(kb.KbfvError):
        sch.leftRotateAndEqual_23(a, 7)  # no key
