"""Wire format: ciphertexts and keys round-trip through bytes, loaded objects
work (decrypt, multiply, rotate), and mismatched or damaged input is refused."""
import numpy as np
import pytest

from tests.gpu_util import dev, host, small_pair

pytestmark = pytest.mark.gpu
T = 65537
SEED = bytes(range(32))


def test_round_trip_and_use():
    import kunpbfv_b200 as kb
    from kunpbfv_b200.api import wire_load, wire_save
    ctx, orc = small_pair(12, 3, 1, 50)
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    sch.addLeftRotKey_23(sk, 1)
    g = sch.galois_element(1)
    rng = np.random.default_rng(1)
    v = rng.integers(0, T, size=(3, ctx.N), dtype=np.uint64)
    ct = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v))), enc_id=5)
    blob = wire_save(ctx, "ciphertext", ct.cipher_device, count=3)
    assert len(blob) == 56 + 3 * 2 * ctx.q_count * ctx.N * 8
    back = kb.Ciphertext(ctx, count=3)
    assert wire_load(ctx, "ciphertext", blob, back.cipher_device, max_count=3) == (3, 0)
    assert np.array_equal(host(back.cipher_device), host(ct.cipher_device))
    # keys: secret, relinearisation, Galois
    sk2 = kb.SecretKey(ctx, b"\x99" * 32)
    wire_load(ctx, "secret_key", wire_save(ctx, "secret_key", sk.sx_device), sk2.sx_device)
    sch2 = kb.BFVScheme(ctx, SEED)
    sch2.rlk = ctx.zeros(*sch.rlk.shape)
    wire_load(ctx, "relin_key", wire_save(ctx, "relin_key", sch.rlk), sch2.rlk)
    gk = ctx.zeros(*sch.galois_keys[g].shape)
    assert wire_load(ctx, "galois_key", wire_save(ctx, "galois_key", sch.galois_keys[g], aux=g), gk)[1] == g
    sch2.galois_keys[g] = gk
    prod = sch2.mult_relin(back, back)
    dec = host(ctx.decode(sch.decryptMsg(sk2, prod).mx_device)).reshape(3, ctx.N)
    assert np.array_equal(dec, (v * v) % T)
    rot = sch2.apply_galois(back, g)
    assert np.array_equal(host(rot.cipher_device), host(sch.apply_galois(ct, g).cipher_device))


def test_refuses_mismatch_and_damage():
    import kunpbfv_b200 as kb
    from kunpbfv_b200.api import wire_load, wire_save
    ctx, _ = small_pair(12, 3, 1, 50)
    other, _ = small_pair(12, 4, 2, 45, 2)
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    ct = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(np.zeros(ctx.N, dtype=np.uint64)))), enc_id=1)
    blob = wire_save(ctx, "ciphertext", ct.cipher_device)
    out = kb.Ciphertext(other)
    with pytest.raises(kb.KbfvError):
        wire_load(other, "ciphertext", blob, out.cipher_device)  # other parameter set
    dst = kb.Ciphertext(ctx)
    with pytest.raises(kb.KbfvError):
        wire_load(ctx, "public_key", blob, dst.cipher_device)  # wrong kind
    with pytest.raises(kb.KbfvError):
        wire_load(ctx, "ciphertext", blob[:-8], dst.cipher_device)  # truncated
    bad = bytearray(blob)
    bad[0] ^= 1
    with pytest.raises(kb.KbfvError):
        wire_load(ctx, "ciphertext", bytes(bad), dst.cipher_device)  # magic
    # a ciphertext switched down one level loads into that level's context only
    low = sch.mod_switch(ct)
    lb = wire_save(low.ctx, "ciphertext", low.cipher_device)
    with pytest.raises(kb.KbfvError):
        wire_load(ctx, "ciphertext", lb, dst.cipher_device)
    back = kb.Ciphertext(low.ctx)
    wire_load(low.ctx, "ciphertext", lb, back.cipher_device)
    assert np.array_equal(host(back.cipher_device), host(low.cipher_device))
