"""Levels on the B200: the modulus switch, multiplies at lower levels with the
top-level key, and the uneven batch of config C4 (N=32768, 14 x 60-bit q +
2 x 60-bit special primes, digits of 5 primes, pairs at depths 0-3 in one call)."""
import functools

import numpy as np
import pytest

from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

T = 65537
SEED = b"\x33" * 32


@functools.lru_cache(maxsize=None)
def small():
    """N=4096, 6 x 50-bit q, 2 x 52-bit p, digits of 2 primes; product and oracle."""
    import kunpbfv_b200 as kb
    import oracle
    p = oracle.primes_bits(4096, 52, 2)
    q = oracle.primes_bits(4096, 50, 6, skip=p)
    ctx = kb.BFVContext(log_n=12, plain_modulus=T, q_count=6, q=q, p_count=2, p=p, dnum=3)
    assert ctx.alpha == 2
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    top = oracle.Oracle(12, T, q, p, alpha=2)
    osk = top.keygen_secret(SEED)
    return ctx, sk, sch, top, osk, q, p


def test_mod_switch_bit_exact():
    import kunpbfv_b200 as kb
    import oracle
    ctx, sk, sch, top, osk, q, p = small()
    rng = np.random.default_rng(1)
    v = rng.integers(0, T, size=(3, ctx.N), dtype=np.uint64)
    ct = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v))), enc_id=40)
    cur = ct
    want = host(ct.cipher_device).reshape(3, 2, 6, ctx.N)
    for live in (5, 4, 3, 2, 1):
        cur = sch.mod_switch(cur)
        assert cur.ctx.q_count == live
        o = oracle.Oracle(12, T, q[:live + 1], p, alpha=2)
        want = np.stack([o.mod_switch(want[i]) for i in range(3)])
        assert np.array_equal(host(cur.cipher_device).reshape(want.shape), want), live
        dec = host(cur.ctx.decode(sch.decryptMsg(sk, cur).mx_device)).reshape(3, ctx.N)
        assert np.array_equal(dec, v), live
    with pytest.raises(kb.KbfvError):
        sch.mod_switch(cur)  # one live prime left


def test_level_multiply_bit_exact():
    """At every level the product equals the oracle's multiply with the top-level
    key restricted to the live primes, and decrypts exactly."""
    import kunpbfv_b200 as kb
    import oracle
    ctx, sk, sch, top, osk, q, p = small()
    orlk = top.keygen_relin(SEED, osk)
    assert np.array_equal(host(sch.rlk).reshape(orlk.shape), orlk)
    rng = np.random.default_rng(2)
    v1 = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=50)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=60)
    for live in (6, 5, 4, 3):
        o = oracle.Oracle(12, T, q[:live], p, alpha=2)
        rl = np.stack([np.stack([np.concatenate([orlk[d][h][:live], orlk[d][h][6:]]) for h in range(2)])
                       for d in range(o.dnum)])
        out = sch.mult_relin(c1, c2)
        got = host(out.cipher_device).reshape(2, 2, live, ctx.N)
        h1 = host(c1.cipher_device).reshape(2, 2, live, ctx.N)
        h2 = host(c2.cipher_device).reshape(2, 2, live, ctx.N)
        for i in range(2):
            assert np.array_equal(got[i], o.mul_relin(h1[i], h2[i], rl)), (live, i)
        dec = host(out.ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(2, ctx.N)
        assert np.array_equal(dec, (v1 * v2) % T), live
        if live > 3:
            c1, c2 = sch.mod_switch(c1), sch.mod_switch(c2)


def test_level_context_rules():
    import kunpbfv_b200 as kb
    ctx, sk, sch, *_ = small()
    lv = ctx.at_level(4)
    assert lv.q_count == 4 and lv.q == ctx.q[:4] and lv.p == ctx.p and lv.alpha == 2 and lv.dnum == 2
    assert ctx.at_level(4) is lv and ctx.at_level(6) is ctx
    with pytest.raises(kb.KbfvError):
        ctx.at_level(7)
    with pytest.raises(kb.KbfvError):  # keys are made on the top level
        kb.BFVScheme(lv, SEED).addMultKey_23(sk)


def test_c4_uneven_batch():
    """16 pairs at depths 0-3 (14, 13, 12, 11 live primes) in one call; every
    product equals the oracle's multiply at its level (all 16 pairs), equals
    the pair multiplied alone at its level (the first 8) and decrypts exactly."""
    from concurrent.futures import ThreadPoolExecutor

    import kunpbfv_b200 as kb
    import oracle
    ctx = kb.BFVContext.from_bits(15, [60] * 14, [60, 60], T, dnum=3)
    assert ctx.alpha == 5
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    rng = np.random.default_rng(4)
    pairs, vals = [], []
    for j in range(16):
        depth = j % 4
        v1 = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
        v2 = rng.integers(0, T, size=ctx.N, dtype=np.uint64)
        a = sch.mod_switch_to(sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=100 + 2 * j), 14 - depth)
        b = sch.mod_switch_to(sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=101 + 2 * j), 14 - depth)
        pairs.append((a, b))
        vals.append((v1 * v2) % T)
    outs = sch.mult_relin_levels(pairs)
    for j, ((a, b), o) in enumerate(zip(pairs, outs)):
        assert o.ctx.q_count == 14 - j % 4
        dec = host(o.ctx.decode(sch.decryptMsg(sk, o).mx_device)).reshape(-1)
        assert np.array_equal(dec, vals[j]), j
        if j < 8:
            alone = sch.mult_relin(a, b)
            assert np.array_equal(host(alone.cipher_device), host(o.cipher_device)), j
    # the oracle on every pair: one oracle per level (the level's live primes,
    # the top level's digits and special primes, the top-level key restricted
    # to the live limbs), each level's four pairs in a thread of their own
    top = oracle.Oracle(15, T, ctx.q, ctx.p, alpha=5)
    osk = top.keygen_secret(SEED)
    assert np.array_equal(host(sk.sx_device).reshape(osk.shape), osk)
    orlk = top.keygen_relin(SEED, osk)
    ins = [tuple(host(x.cipher_device).reshape(2, 14 - j % 4, ctx.N) for x in pairs[j]) for j in range(16)]
    got = [host(outs[j].cipher_device).reshape(2, 14 - j % 4, ctx.N) for j in range(16)]

    def level(depth):
        live = 14 - depth
        o = oracle.Oracle(15, T, ctx.q[:live], ctx.p, alpha=5)
        rl = np.stack([np.stack([np.concatenate([orlk[d][h][:live], orlk[d][h][14:]]) for h in range(2)])
                       for d in range(o.dnum)])
        return {j: o.mul_relin(*ins[j], rl) for j in range(depth, 16, 4)}

    with ThreadPoolExecutor(max_workers=4) as ex:
        want = {}
        for part in ex.map(level, range(4)):
            want.update(part)
    assert sorted(want) == list(range(16))
    for j in range(16):
        assert np.array_equal(got[j], want[j]), f"pair {j} at {14 - j % 4} live primes differs from the oracle"


def test_gadget_key_switch_bit_exact():
    """Key switching over a base-2^20 gadget decomposition: the key equals the
    oracle's, the multiply equals the oracle's at the top level and at level 4
    (top-level key, first 4 x 3 components), decryptions exact."""
    import kunpbfv_b200 as kb
    import oracle
    ctx, sk, sch, top, osk, q, p = small()
    gs = kb.BFVScheme(ctx, SEED, relin="gadget", gadget_log_base=20)
    gs.addEncKey(sk)
    gs.addMultKey_23(sk)
    ogk = top.keygen_relin_gadget(SEED, osk, 20)
    assert np.array_equal(host(gs.gk).reshape(ogk.shape), ogk)
    rng = np.random.default_rng(7)
    v1 = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
    c1 = gs.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=70)
    c2 = gs.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=80)
    for live in (6, 4):
        o = oracle.Oracle(12, T, q[:live], p, alpha=2)
        gl = np.stack([np.stack([np.concatenate([ogk[g][h][:live], ogk[g][h][6:]]) for h in range(2)])
                       for g in range(live * 3)])
        out = gs.mult_relin(c1, c2)
        h1 = host(c1.cipher_device).reshape(2, 2, live, ctx.N)
        h2 = host(c2.cipher_device).reshape(2, 2, live, ctx.N)
        got = host(out.cipher_device).reshape(2, 2, live, ctx.N)
        for i in range(2):
            assert np.array_equal(got[i], o.relinearize_gadget(o.mul_tensor(h1[i], h2[i]), gl, 20)), (live, i)
        # split form: tensor then gadget relinearisation
        t3 = gs.mult(c1, c2)
        assert np.array_equal(host(gs.relinearize(t3).cipher_device).reshape(got.shape), got)
        dec = host(out.ctx.decode(gs.decryptMsg(sk, out).mx_device)).reshape(2, ctx.N)
        assert np.array_equal(dec, (v1 * v2) % T), live
        c1, c2 = gs.mod_switch_to(c1, 4), gs.mod_switch_to(c2, 4)


def test_c4_gadget_at_each_depth():
    """Config C4's external product over a base-2^20 gadget decomposition at
    N=32768, 14 x 60-bit q + 2 x 60-bit p: pairs at depths 0-3 decrypt exactly;
    the top pair equals the oracle."""
    import kunpbfv_b200 as kb
    import oracle
    ctx = kb.BFVContext.from_bits(15, [60] * 14, [60, 60], T, dnum=3)
    sk = kb.SecretKey(ctx, SEED)
    gs = kb.BFVScheme(ctx, SEED, relin="gadget", gadget_log_base=20)
    gs.addEncKey(sk)
    gs.addMultKey_23(sk)
    rng = np.random.default_rng(5)
    outs = []
    for depth in range(4):
        v1 = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
        v2 = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
        a = gs.mod_switch_to(gs.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=300 + 4 * depth), 14 - depth)
        b = gs.mod_switch_to(gs.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=302 + 4 * depth), 14 - depth)
        out = gs.mult_relin(a, b)
        dec = host(out.ctx.decode(gs.decryptMsg(sk, out).mx_device)).reshape(2, ctx.N)
        assert np.array_equal(dec, (v1 * v2) % T), depth
        outs.append((a, b, out))
    top = oracle.Oracle(15, T, ctx.q, ctx.p, alpha=5)
    osk = top.keygen_secret(SEED)
    ogk = top.keygen_relin_gadget(SEED, osk, 20)
    a, b, out = outs[0]
    ha = host(a.cipher_device).reshape(2, 2, 14, ctx.N)[0]
    hb = host(b.cipher_device).reshape(2, 2, 14, ctx.N)[0]
    want = top.relinearize_gadget(top.mul_tensor(ha, hb), ogk, 20)
    assert np.array_equal(host(out.cipher_device).reshape(2, 2, 14, ctx.N)[0], want)


def test_mixed_levels_span_several_launch_sequences():
    """Pairs at 10 different levels in shuffled order (more levels than one
    launch sequence groups): every product equals the pair multiplied alone at
    its level."""
    import kunpbfv_b200 as kb
    ctx = kb.BFVContext.from_bits(12, [40] * 10, [50], T, dnum=5)
    assert ctx.alpha == 2
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    rng = np.random.default_rng(9)
    levels = [10, 3, 7, 1, 9, 4, 2, 8, 6, 5, 10, 1, 5, 7]
    pairs = []
    for j, live in enumerate(levels):
        v = rng.integers(0, T, size=(2, ctx.N), dtype=np.uint64)
        a = sch.mod_switch_to(sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v[0]))), enc_id=900 + 2 * j), live)
        b = sch.mod_switch_to(sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v[1]))), enc_id=901 + 2 * j), live)
        pairs.append((a, b))
    outs = sch.mult_relin_levels(pairs)
    for j, ((a, b), o) in enumerate(zip(pairs, outs)):
        assert o.ctx.q_count == levels[j]
        alone = sch.mult_relin(a, b)
        assert np.array_equal(host(alone.cipher_device), host(o.cipher_device)), (j, levels[j])


@pytest.mark.parametrize("log_n,q_bits,p_bits,dnum,t,levels", [
    (14, [60] * 7, [60], 1, 65537, [7, 6, 5, 4, 7, 6, 5, 4]),   # 2^14 whole-row block kernels (rows > 48)
    (14, [60] * 7, [60], 1, 65537, [7, 4]),                     # 2^14 column pass + 2^12-point blocks
    (13, [50] * 5, [52], 5, 65537, [5, 3, 4, 2, 1, 5]),         # 2^13 blocks, one-prime digits
    (16, [60] * 6, [60], 2, 786433, [6, 4, 5, 3]),              # 2^16 column pass + 2^12-point blocks
])
def test_mixed_levels_on_other_rings(log_n, q_bits, p_bits, dnum, t, levels):
    """One launch sequence over pairs at mixed levels on the block shapes the
    other level tests do not reach: every product equals the pair multiplied
    alone at its level (itself pinned to the oracle per level)."""
    import kunpbfv_b200 as kb
    ctx = kb.BFVContext.from_bits(log_n, q_bits, p_bits, t, dnum=dnum)
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    rng = np.random.default_rng(log_n + len(levels))
    pairs = []
    for j, live in enumerate(levels):
        v = rng.integers(0, t, size=(2, ctx.N), dtype=np.uint64)
        a = sch.mod_switch_to(sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v[0]))), enc_id=700 + 2 * j), live)
        b = sch.mod_switch_to(sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v[1]))), enc_id=701 + 2 * j), live)
        pairs.append((a, b))
    outs = sch.mult_relin_levels(pairs)
    for j, ((a, b), o) in enumerate(zip(pairs, outs)):
        assert o.ctx.q_count == levels[j]
        alone = sch.mult_relin(a, b)
        assert np.array_equal(host(alone.cipher_device), host(o.cipher_device)), (j, levels[j])
