"""The allocation-free multiply (kbfv_mul_relin_noalloc) against the
allocating entry point (kbfv_mul_relin).

Some callers cannot allocate device memory while they run (a service that
fixed its memory budget at start-up and must not fail with out-of-memory in the
middle of a request, code inside another framework's allocator hook);
kbfv_mul_relin_noalloc serves them from a static device array in
libkbfv.so. This file runs last so that a failure here leaves every other
result in place; it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

T = 65537
SEED = bytes(range(32))


def _setup(count):
    import kunpbfv_b200 as kb
    from kunpbfv_b200.api import to_device
    from tests.gpu_util import c3_pair
    ctx, _ = c3_pair()
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    rng = np.random.default_rng(11)
    v1 = rng.integers(0, T, size=(count, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, T, size=(count, ctx.N), dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(to_device(v1))), enc_id=500)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(to_device(v2))), enc_id=600)
    return kb, ctx, sk, sch, c1, c2, v1, v2


def _noalloc(kb, ctx, sch, c1, c2, out, count):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    return kb.lib().kbfv_mul_relin_noalloc(ctx.handle, sch.rlk.data_ptr(), c1.cipher_device.data_ptr(),
                                           c2.cipher_device.data_ptr(), out.cipher_device.data_ptr(), count,
                                           ctypes.c_void_p(stream))


def test_noalloc_matches_allocating_entry_point_twice():
    import torch
    count = 2
    kb, ctx, sk, sch, c1, c2, v1, v2 = _setup(count)
    assert ctx.scratch_bytes(count) <= (40 << 20)
    want = sch.mult_relin(c1, c2)
    torch.cuda.synchronize()
    for call in range(2):  # two calls in a row share (and reuse) the static array
        out = kb.Ciphertext(ctx, count=count)
        assert _noalloc(kb, ctx, sch, c1, c2, out, count) == 0, kb.lib().kbfv_last_error()
        torch.cuda.synchronize()
        assert torch.equal(out.cipher_device, want.cipher_device), f"call {call} differs"
    dec = kb.api.to_host(ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(count, ctx.N)
    assert np.array_equal(dec, (v1 * v2) % T)


def test_noalloc_rejects_oversized_batches():
    kb, ctx, sk, sch, c1, c2, v1, v2 = _setup(1)
    out = kb.Ciphertext(ctx, count=3)
    rc = _noalloc(kb, ctx, sch, c1, c2, out, 3)  # 3 pairs need ~55 MB > 40 MiB
    assert rc == -1
    assert b"static array holds" in kb.lib().kbfv_last_error()
