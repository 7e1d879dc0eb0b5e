"""Captured multiplies (kbfv_plan_*) on the B200: the graph replay gives the
eager multiply's product for whatever the bound buffers hold at launch time,
and records itself again when the scratch arena moves or a knob changes."""
import numpy as np
import pytest

from tests.gpu_util import c3_pair, dev, host

pytestmark = pytest.mark.gpu


def _setup(pairs, seed):
    import kunpbfv_b200 as kb
    ctx, orc = c3_pair()
    sk = kb.SecretKey(ctx, b"\x61" * 32)
    sch = kb.BFVScheme(ctx, b"\x62" * 32)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    rng = np.random.default_rng(seed)

    def fresh(enc_id):
        v = rng.integers(0, 65537, size=(pairs, ctx.N), dtype=np.uint64)
        return sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v))), enc_id=enc_id)
    return kb, ctx, sk, sch, fresh


@pytest.mark.parametrize("pairs", [1, 3, 20])
def test_plan_replays_the_multiply(pairs):
    """First launch (eager + record), then replays over new buffer contents;
    every product equals kbfv_mul_relin's (pinned to the oracle by the
    multiply tests), and the replays record nothing."""
    import torch
    kb, ctx, sk, sch, fresh = _setup(pairs, 5)
    a, b = fresh(100), fresh(200)
    out = kb.Ciphertext(ctx, count=pairs)
    plan = sch.mult_relin_plan(a, b, out)
    try:
        for rnd in range(4):
            if rnd:  # new operands in the same buffers
                na, nb = fresh(100 + 7 * rnd), fresh(200 + 7 * rnd)
                a.cipher_device.copy_(na.cipher_device)
                b.cipher_device.copy_(nb.cipher_device)
            plan.launch()
            torch.cuda.synchronize()
            want = sch.mult_relin(a, b).cipher_device
            torch.cuda.synchronize()
            assert torch.equal(out.cipher_device, want), rnd
        assert plan.info() == (4, 1)
    finally:
        plan.close()


def test_plan_records_again_after_arena_move_and_knob_change():
    import torch
    kb, ctx, sk, sch, fresh = _setup(2, 9)
    a, b = fresh(300), fresh(400)
    out = kb.Ciphertext(ctx, count=2)
    plan = sch.mult_relin_plan(a, b, out)
    keep = ctx.tune_get("split_rows")
    try:
        plan.launch()
        plan.launch()
        assert plan.info() == (2, 1)
        want = sch.mult_relin(a, b).cipher_device.clone()
        before = ctx.arena_bytes()
        ctx.reserve(128)  # the arena grows: a new allocation
        assert ctx.arena_bytes() > before
        out.cipher_device.zero_()
        plan.launch()
        torch.cuda.synchronize()
        assert plan.info() == (3, 2) and torch.equal(out.cipher_device, want)
        ctx.tune_set("split_rows", 0)
        out.cipher_device.zero_()
        plan.launch()
        plan.launch()
        torch.cuda.synchronize()
        assert plan.info() == (5, 3) and torch.equal(out.cipher_device, want)
    finally:
        ctx.tune_set("split_rows", keep)
        plan.close()


def test_plan_rejects_bad_arguments():
    import kunpbfv_b200 as kb
    from kunpbfv_b200.api import lib, _ptr
    import ctypes as C
    _, ctx, sk, sch, fresh = _setup(1, 3)
    a = fresh(1)
    h = C.c_void_p()
    assert lib().kbfv_plan_mul_relin(ctx.handle, _ptr(sch.rlk), _ptr(a.cipher_device), _ptr(a.cipher_device),
                                    _ptr(a.cipher_device), 0, C.byref(h)) != 0
    assert lib().kbfv_plan_mul_relin(ctx.handle, None, _ptr(a.cipher_device), _ptr(a.cipher_device),
                                    _ptr(a.cipher_device), 1, C.byref(h)) != 0
    assert lib().kbfv_plan_launch(None, None) != 0
    assert lib().kbfv_plan_destroy(None) == 0


def test_levels_plan_replays_the_mixed_batch():
    """A plan over pairs at four levels (kbfv_plan_mul_relin_levels): every
    launch equals kbfv_mul_relin_levels on the buffers' current contents."""
    import torch

    import kunpbfv_b200 as kb
    from kunpbfv_b200 import tune
    ctx = kb.BFVContext.from_bits(14, [60] * 7, [60], 65537, dnum=1)
    sk = kb.SecretKey(ctx, b"\x63" * 32)
    sch = kb.BFVScheme(ctx, b"\x64" * 32)
    sch.addMultKey_23(sk)
    pairs, outs = [], []
    for j in range(10):
        lv = ctx.at_level(7 - j % 4)
        pairs.append((kb.Ciphertext(lv, tune._random_pairs(lv, 1, 30 + j)),
                      kb.Ciphertext(lv, tune._random_pairs(lv, 1, 60 + j))))
        outs.append(kb.Ciphertext(lv, count=1))
    plan = sch.mult_relin_levels_plan(pairs, outs)
    try:
        for rnd in range(3):
            if rnd:
                for j, (a, b) in enumerate(pairs):
                    a.cipher_device.copy_(tune._random_pairs(a.ctx, 1, 100 * rnd + j).view_as(a.cipher_device))
            plan.launch()
            torch.cuda.synchronize()
            got = [o.cipher_device.clone() for o in outs]
            want = sch.mult_relin_levels(pairs)
            torch.cuda.synchronize()
            for j, (g, w) in enumerate(zip(got, want)):
                assert torch.equal(g, w.cipher_device), (rnd, j)
        assert plan.info() == (3, 1)
    finally:
        plan.close()
