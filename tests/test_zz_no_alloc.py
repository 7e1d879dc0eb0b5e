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


def test_noalloc_first_call_on_a_fresh_context_allocates_nothing():
    """A context that never ran an allocating call multiplies through the
    allocation-free entry point: its scratch arena stays empty and the device's
    free memory is the same before and after each of two calls, whose results
    equal the allocating entry point's on another context of the same
    parameters (keys and ciphertexts are shared: same primes)."""
    import torch

    import kunpbfv_b200 as kb
    count = 2
    _, ctx, sk, sch, c1, c2, v1, v2 = _setup(count)
    # the expected products on the setup context (this also loads every
    # multiply kernel into the CUDA context, so no lazy kernel load can land
    # inside the measured calls)
    want = sch.mult_relin(c1, c2)
    fresh = kb.BFVContext(log_n=14, plain_modulus=T, q_count=ctx.q_count, q=ctx.q, p_count=ctx.p_count, p=ctx.p,
                          dnum=1)
    assert fresh.primes == ctx.primes
    assert fresh.arena_bytes() == 0
    outs = [kb.Ciphertext(fresh, count=count) for _ in range(2)]
    torch.cuda.synchronize()
    for call, out in enumerate(outs):
        free_before, _ = torch.cuda.mem_get_info()
        assert _noalloc(kb, fresh, sch, c1, c2, out, count) == 0, kb.lib().kbfv_last_error()
        torch.cuda.synchronize()
        free_after, _ = torch.cuda.mem_get_info()
        assert free_after == free_before, f"call {call}: device free memory moved by {free_before - free_after} B"
        assert fresh.arena_bytes() == 0, f"call {call} allocated the context's scratch arena"
        assert torch.equal(out.cipher_device, want.cipher_device), f"call {call} differs"
    dec = kb.api.to_host(ctx.decode(sch.decryptMsg(sk, outs[1]).mx_device)).reshape(count, ctx.N)
    assert np.array_equal(dec, (v1 * v2) % T)


def test_noalloc_rejects_oversized_batches():
    import torch
    count = 3  # 3 pairs need 3 x 143 limbs of 128 KiB = 53.6 MiB > 40 MiB
    kb, ctx, sk, sch, c1, c2, v1, v2 = _setup(count)
    assert ctx.scratch_bytes(count) > (40 << 20)
    out = kb.Ciphertext(ctx, count=count)
    before = out.cipher_device.clone()
    rc = _noalloc(kb, ctx, sch, c1, c2, out, count)
    torch.cuda.synchronize()
    assert rc == -1
    assert b"static array holds" in kb.lib().kbfv_last_error()
    assert torch.equal(out.cipher_device, before), "a rejected call must launch nothing"
