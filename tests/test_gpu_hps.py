"""HPS and key-switch building blocks on the B200 vs the oracle (bit-exact)."""
import numpy as np
import pytest

from tests.gpu_util import c3_pair, dev, host, rand_rows, small_pair

pytestmark = pytest.mark.gpu

PAIRS = [("c3", lambda: c3_pair()), ("small", lambda: small_pair(12, 3, 1, 50)),
         ("dnum2", lambda: small_pair(12, 4, 2, 45, 2)), ("onedigit", lambda: small_pair(12, 3, 1, 50, 3))]


@pytest.fixture(params=PAIRS, ids=[p[0] for p in PAIRS])
def pair(request):
    return request.param[1]()


def test_bconv_q_to_r_and_back(pair):
    ctx, orc = pair
    n = ctx.N
    x = rand_rows(orc, range(ctx.q_count), n, 1)
    y = host(ctx.bconv_q_to_r(dev(x))).reshape(ctx.r_count, n)
    assert np.array_equal(y, orc.bconv_q_to_r(x))
    r = rand_rows(orc, [ctx.idx_r + j for j in range(ctx.r_count)], n, 2)
    z = host(ctx.bconv_r_to_q(dev(r))).reshape(ctx.q_count, n)
    assert np.array_equal(z, orc.bconv_r_to_q(r))


def test_tensor_qr(pair):
    ctx, orc = pair
    idx = list(range(ctx.q_count)) + [ctx.idx_r + j for j in range(ctx.r_count)]
    c1 = np.stack([rand_rows(orc, idx, ctx.N, 3), rand_rows(orc, idx, ctx.N, 4)])
    c2 = np.stack([rand_rows(orc, idx, ctx.N, 5), rand_rows(orc, idx, ctx.N, 6)])
    got = host(ctx.tensor_qr(dev(c1), dev(c2))).reshape(3, len(idx), ctx.N)
    assert np.array_equal(got, orc.tensor_qr(c1, c2))


def test_scale_round(pair):
    ctx, orc = pair
    idx = list(range(ctx.q_count)) + [ctx.idx_r + j for j in range(ctx.r_count)]
    x = rand_rows(orc, idx, ctx.N, 7)
    got = host(ctx.scale_round_qr_r(dev(x))).reshape(ctx.r_count, ctx.N)
    assert np.array_equal(got, orc.scale_round_qr_r(x))


def test_decrypt_round(pair):
    ctx, orc = pair
    x = rand_rows(orc, range(ctx.q_count), ctx.N, 8)
    got = host(ctx.decrypt_round(dev(x))).reshape(ctx.N)
    assert np.array_equal(got, orc.decrypt_round(x))


def test_delta_m(pair):
    ctx, orc = pair
    m = np.random.default_rng(9).integers(0, ctx.plain_modulus, size=ctx.N, dtype=np.uint64)
    got = host(ctx.delta_m(dev(m))).reshape(ctx.q_count, ctx.N)
    assert np.array_equal(got, orc.delta_m(m))


def test_modup_moddown(pair):
    ctx, orc = pair
    x = rand_rows(orc, range(ctx.q_count), ctx.N, 10)
    got = host(ctx.modup(dev(x))).reshape(ctx.dnum, ctx.q_count + ctx.p_count, ctx.N)
    assert np.array_equal(got, orc.modup(x))
    y = np.stack([rand_rows(orc, range(ctx.q_count + ctx.p_count), ctx.N, 11 + i) for i in range(2)])
    got = host(ctx.moddown(dev(y))).reshape(2, ctx.q_count, ctx.N)
    assert np.array_equal(got, orc.moddown(y))


def test_edge_values(pair):
    """All-zero and all-(q-1) inputs through the per-coefficient kernels."""
    ctx, orc = pair
    n = ctx.N
    for fill in ("zero", "max"):
        x = np.stack([np.full(n, 0 if fill == "zero" else q - 1, dtype=np.uint64) for q in ctx.q])
        assert np.array_equal(host(ctx.bconv_q_to_r(dev(x))).reshape(ctx.r_count, n), orc.bconv_q_to_r(x))
        assert np.array_equal(host(ctx.decrypt_round(dev(x))).reshape(n), orc.decrypt_round(x))
        assert np.array_equal(host(ctx.modup(dev(x))).reshape(ctx.dnum, -1, n), orc.modup(x))
