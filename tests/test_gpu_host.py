"""The multiply of ciphertexts held in host memory (kbfv_mul_relin_host):
chunked copy-in / multiply / copy-out on the context's streams gives products
bit-identical to kbfv_mul_relin on device copies of the same ciphertexts, for
every chunk size (slot reuse included), page-locked or pageable buffers."""
import functools

import numpy as np
import pytest

from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

SEED = b"\x5a" * 32


@functools.lru_cache(maxsize=None)
def setup(count):
    """N=16384, 7 x 60-bit q + 1 special prime: `count` encrypted pairs and the
    device product."""
    import torch

    import kunpbfv_b200 as kb
    from tests.gpu_util import c3_pair
    ctx, _ = c3_pair()
    t = ctx.plain_modulus
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    rng = np.random.default_rng(21)
    v1 = rng.integers(0, t, size=(count, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, t, size=(count, ctx.N), dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=900)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=1900)
    want = sch.mult_relin(c1, c2)
    torch.cuda.synchronize()
    ha = c1.cipher_device.cpu().pin_memory()
    hb = c2.cipher_device.cpu().pin_memory()
    return kb, ctx, sk, sch, ha, hb, want, (v1 * v2) % t


@pytest.mark.parametrize("chunk", [0, 1, 4, 7, 128])
def test_host_multiply_equals_device_multiply(chunk):
    """37 pairs: chunks of 1 and 4 reuse every staging slot several times, 7
    leaves a partial last chunk, 0 is the default size, 128 one chunk."""
    kb, ctx, sk, sch, ha, hb, want, vals = setup(37)
    out = sch.mult_relin_host(ha, hb, chunk_pairs=chunk)
    assert out.is_pinned()
    assert np.array_equal(out.numpy().reshape(-1), host(want.cipher_device).view(np.int64).reshape(-1)), chunk


def test_host_multiply_decrypts_and_pageable_buffers():
    import torch
    kb, ctx, sk, sch, ha, hb, want, vals = setup(37)
    pa, pb = ha.numpy().view(np.uint64).copy(), hb.numpy().view(np.uint64).copy()  # ordinary (pageable) memory
    out = sch.mult_relin_host(pa, pb, chunk_pairs=5)
    assert np.array_equal(out.numpy().reshape(-1), want.cipher_device.cpu().numpy().reshape(-1))
    ct = kb.Ciphertext(ctx, out.cuda())
    dec = host(ctx.decode(sch.decryptMsg(sk, ct).mx_device)).reshape(37, ctx.N)
    assert np.array_equal(dec, vals)
    # queued only, then ordered after other work on a side stream
    side = torch.cuda.Stream()
    o2 = torch.empty_like(out).pin_memory()
    sch.mult_relin_host(ha, hb, out=o2, chunk_pairs=6, stream=side, synchronize=False)
    side.synchronize()
    assert torch.equal(o2, out)


def test_host_multiply_rejects_bad_arguments():
    import torch
    kb, ctx, sk, sch, ha, hb, want, vals = setup(37)
    with pytest.raises(kb.KbfvError):
        sch.mult_relin_host(ha, hb, chunk_pairs=129)
    with pytest.raises(kb.KbfvError):
        sch.mult_relin_host(ha, hb[:36])
    with pytest.raises(kb.KbfvError):
        sch.mult_relin_host(ha.cuda(), hb.cuda())
    with pytest.raises(kb.KbfvError):
        sch.mult_relin_host(ha, hb, out=torch.empty(3, dtype=torch.int64))
