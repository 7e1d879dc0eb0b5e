"""The request server (kbfv_server_*): continuous batching across rings of
N = 4096, 8192, 16384, admission by a device budget, exact decryptions, and
each request's ciphertext bit-identical whether it ran alone or in the mix."""
import functools

import numpy as np
import pytest

from tests.gpu_util import dev, host

pytestmark = pytest.mark.gpu

T = 65537


@functools.lru_cache(maxsize=None)
def rings():
    import kunpbfv_b200 as kb
    from kunpbfv_b200.serve import Ring
    # one key-switch digit per ciphertext prime (digits no larger than the
    # special prime) so chains of several multiplies keep their noise budget
    ctxs = [kb.BFVContext.from_bits(12, [36, 36], [37], T, dnum=2),
            kb.BFVContext.from_bits(13, [50, 50, 50], [52], T, dnum=3),
            kb.BFVContext.from_bits(14, [60] * 7, [60], T, dnum=7)]
    return [Ring.make(c, bytes([7 + i]) * 32) for i, c in enumerate(ctxs)]


MAX_MUL = [1, 3, 4]  # multiplies a chain may hold on each ring (noise budget)


def test_mixed_stream_exact_and_identical_alone():
    from kunpbfv_b200.serve import Server, make_workload
    rs = rings()
    w = make_workload(rs, 36, MAX_MUL, seed=3)
    mix = {}
    with Server(rs, hbm_budget_bytes=1 << 30, max_batch=32) as srv:
        ids = [srv.submit(w.ring[i], w.slots[i], w.ops[i], 1000 + 16 * i, return_ct=True) for i in range(36)]
        for i, rid in enumerate(ids):
            res, ct, ms = srv.wait(rid, timeout_ms=120000, ring=w.ring[i], want_ct=True)
            assert np.array_equal(res, w.want[i]), f"request {i}: wrong decryption"
            assert ms > 0
            mix[i] = ct
        st = srv.stats()
        assert st["completed"] == 36 and st["failed"] == 0
        # multiplies of different requests shared launches
        assert st["mul_ops"] > st["mul_launches"]
        # the same requests one at a time on the same server
        for i in range(0, 36, 3):
            rid = srv.submit(w.ring[i], w.slots[i], w.ops[i], 1000 + 16 * i, return_ct=True)
            res, ct, _ = srv.wait(rid, timeout_ms=120000, ring=w.ring[i], want_ct=True)
            assert np.array_equal(res, w.want[i])
            assert np.array_equal(ct, mix[i]), f"request {i}: ciphertext differs alone vs in the mix"


def test_server_matches_direct_api():
    """A served chain equals the same chain through BFVScheme calls."""
    import kunpbfv_b200 as kb
    from kunpbfv_b200.serve import OP_MUL, Server
    rs = rings()
    r = rs[2]
    ctx, sch = r.ctx, r.scheme
    rng = np.random.default_rng(9)
    slots = rng.integers(0, T, size=(4, ctx.N), dtype=np.uint64)
    ops = [OP_MUL, 1, OP_MUL]
    cts = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(slots))), enc_id=777)
    lq = 2 * ctx.q_count * ctx.N
    flat = cts.cipher_device.view(-1)
    acc = kb.Ciphertext(ctx, flat[:lq].clone())
    for i, op in enumerate(ops):
        nxt = kb.Ciphertext(ctx, flat[(i + 1) * lq:(i + 2) * lq].clone())
        acc = sch.mult_relin(acc, nxt) if op == OP_MUL else sch.add(acc, nxt)
    want_ct = host(acc.cipher_device).reshape(-1)
    with Server(rs, hbm_budget_bytes=1 << 30, max_batch=8) as srv:
        rid = srv.submit(2, slots, ops, 777, return_ct=True)
        res, ct, _ = srv.wait(rid, timeout_ms=120000, ring=2, want_ct=True)
    assert np.array_equal(ct, want_ct)
    want = (slots[0] * slots[1]) % T
    want = ((want + slots[2]) % T * slots[3]) % T
    assert np.array_equal(res, want)


def test_budget_limits_admission():
    """A budget that holds two N=16384 requests at a time still completes a
    burst of twelve, never exceeding the budget."""
    from kunpbfv_b200.serve import OP_MUL, Server
    rs = rings()
    r = rs[2]
    n, nq = r.ctx.N, r.ctx.q_count
    per = ((3 * n + 3 * 2 * nq * n + n) * 8 + 255) // 256 * 256
    budget = 2 * per + per // 2
    rng = np.random.default_rng(11)
    with Server(rs, hbm_budget_bytes=budget, max_batch=8) as srv:
        subs = []
        for j in range(12):
            s = rng.integers(0, T, size=(3, n), dtype=np.uint64)
            subs.append((srv.submit(2, s, [OP_MUL, OP_MUL], 5000 + 16 * j), s))
        for rid, s in subs:
            res, _, _ = srv.wait(rid, timeout_ms=120000, ring=2)
            assert np.array_equal(res, (s[0] * s[1] % T) * s[2] % T)
        st = srv.stats()
    assert st["bytes_peak"] <= budget
    assert st["completed"] == 12


def test_rejects_bad_requests():
    import kunpbfv_b200 as kb
    from kunpbfv_b200.serve import Server
    rs = rings()
    with Server(rs[:1], hbm_budget_bytes=64 << 20, max_batch=4) as srv:
        bad = np.full((2, rs[0].ctx.N), T, dtype=np.uint64)  # values must be < t
        with pytest.raises(kb.KbfvError):
            srv.submit(0, bad, [0], 1)
        with pytest.raises(kb.KbfvError):
            srv.submit(3, bad * 0, [0], 1)  # no such ring
        with pytest.raises(kb.KbfvError):
            srv.submit(0, np.zeros((10, rs[0].ctx.N), dtype=np.uint64), [0] * 9, 1)  # more than 8 ops


def test_open_loop_poisson_small():
    """A short Poisson stream across the rings: every decryption exact, p50/p99 reported."""
    from kunpbfv_b200.serve import Server, make_workload, run_open_loop
    rs = rings()
    w = make_workload(rs, 24, MAX_MUL, seed=5)
    with Server(rs, hbm_budget_bytes=1 << 30, max_batch=32) as srv:
        out = run_open_loop(srv, w, rate=200.0, duration_s=1.0, seed=2)
    assert out["completed"] == out["offered"] > 0
    assert out["wrong"] == 0 and out["errors"] == 0
    assert out["p99_ms"] >= out["p50_ms"] > 0
