"""Parity sweep over parameter shapes: for each ring degree, prime counts,
special-prime count and digit count below, the batched multiply-relinearise on
the GPU equals the oracle's product bit for bit and decrypts to m1*m2 mod t.
The shapes reach every launch form of the pipeline: one pair per call at
N=2^13/2^14 (the split small-launch NTT), two special primes (the general
mod down), several digits (the multi-digit key product at the output store),
odd limb counts, and N=2^15/2^16 (column pass + 2^12-point blocks)."""
import numpy as np
import pytest

import oracle
from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

# (log_n, q bits, p bits, dnum, pairs)
CASES = [
    (13, [50] * 3, [52], 3, 1),
    (14, [60] * 7, [60], 1, 1),
    (14, [55] * 6, [58, 58], 3, 1),
    (14, [60] * 5, [60, 60], 2, 3),
    (14, [50] * 4, [55], 4, 2),
    (15, [60] * 6, [60, 60], 3, 1),
    (15, [55] * 9, [58, 58, 58], 3, 2),
    (16, [60] * 4, [60, 60], 2, 1),
]


def _t(log_n):
    return 65537 if (2 << log_n) <= 65536 else 786433


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"logn{c[0]}_q{len(c[1])}_p{len(c[2])}_d{c[3]}_x{c[4]}")
def test_multiply_matches_oracle(case):
    import kunpbfv_b200 as kb
    log_n, qb, pb, dnum, pairs = case
    t = _t(log_n)
    ctx = kb.BFVContext.from_bits(log_n, qb, pb, t, dnum=dnum)
    seed = bytes([log_n, len(qb), len(pb), dnum]) * 8
    sk = kb.SecretKey(ctx, seed)
    sch = kb.BFVScheme(ctx, seed)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    rng = np.random.default_rng(log_n * 100 + len(qb))
    v1 = rng.integers(0, t, size=(pairs, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, t, size=(pairs, ctx.N), dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=1)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=1 + pairs)
    out = sch.mult_relin(c1, c2)
    dec = host(ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(pairs, ctx.N)
    assert np.array_equal(dec, (v1 * v2) % t), "decryption is not m1*m2 mod t"
    orc = oracle.Oracle(log_n, t, list(ctx.q), list(ctx.p), alpha=ctx.alpha)
    osk = orc.keygen_secret(seed)
    assert np.array_equal(host(sk.sx_device).reshape(osk.shape), osk)
    orlk = orc.keygen_relin(seed, osk)
    assert np.array_equal(host(sch.rlk).reshape(orlk.shape), orlk)
    nq = ctx.q_count
    h1 = host(c1.cipher_device).reshape(pairs, 2, nq, ctx.N)
    h2 = host(c2.cipher_device).reshape(pairs, 2, nq, ctx.N)
    got = host(out.cipher_device).reshape(pairs, 2, nq, ctx.N)
    i = pairs - 1  # one pair against the oracle (the others are checked by decryption)
    assert np.array_equal(got[i], orc.mul_relin(h1[i], h2[i], orlk))
