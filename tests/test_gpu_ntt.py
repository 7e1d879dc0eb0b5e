"""NTT / INTT on the B200 through the C ABI vs the oracle (bit-exact)."""
import numpy as np
import pytest

import oracle
from tests.gpu_util import dev, host, make_pair, rand_rows
from tests.params import chain

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_n", [10, 11, 12, 13, 14, 15, 16])
def test_ntt_fwd_inv_vs_oracle(log_n):
    n = 1 << log_n
    ps = list(chain(log_n, 60, 4))
    ctx, orc = make_pair(log_n, ps[1:4], ps[:1])
    # rows over all primes of the table [Q|P|R], 2 polys each
    idxs = list(range(len(orc.primes) - 1))
    x = np.concatenate([rand_rows(orc, idxs, n, log_n), rand_rows(orc, idxs, n, log_n + 100)])
    d = dev(x)
    ctx.ntt_fwd(d, 0, len(idxs))
    got = host(d).reshape(x.shape)
    want = np.stack([orc.ntt_fwd(idxs[r % len(idxs)], x[r]) for r in range(x.shape[0])])
    assert np.array_equal(got, want)
    ctx.ntt_inv(d, 0, len(idxs))
    assert np.array_equal(host(d).reshape(x.shape), x)


def test_ntt_inverse_of_oracle_output():
    log_n = 14
    ps = list(chain(log_n, 60, 8))
    ctx, orc = make_pair(log_n, ps[1:8], ps[:1])
    x = rand_rows(orc, range(7), 1 << log_n, 3)
    X = np.stack([orc.ntt_fwd(i, x[i]) for i in range(7)])
    d = dev(X)
    ctx.ntt_inv(d, 0, 7)
    assert np.array_equal(host(d).reshape(x.shape), x)


def test_ntt_plain_modulus_rows():
    """encode/decode transforms (mod t = 65537)."""
    ctx, orc = make_pair(14, *[list(chain(14, 60, 8))[1:8], list(chain(14, 60, 8))[:1]])
    rng = np.random.default_rng(1)
    v = rng.integers(0, 65537, size=(3, 1 << 14), dtype=np.uint64)
    m = host(ctx.encode(dev(v))).reshape(v.shape)
    assert np.array_equal(m, np.stack([orc.encode(r) for r in v]))
    back = host(ctx.decode(dev(m))).reshape(v.shape)
    assert np.array_equal(back, v)


# C2 rows checked against the oracle: two polynomials per prime, all 64
# polynomials distinct, so every prime's twiddle table and every polynomial
# slot of the batch is covered by at least one full row
C2_FWD_ROWS = [(p, (2 * p) % 64) for p in range(32)] + [(p, (2 * p + 37) % 64) for p in range(32)]


def test_ntt_c2_shape_vs_oracle_and_round_trip():
    """N=65536, 32 primes x 64 polys (1 GiB): 64 full forward rows (two per
    prime, every polynomial once) equal the oracle's transform, 32 full
    inverse rows (one per prime) equal the oracle's inverse of the GPU's
    forward output, and the whole batch round-trips bit-exactly."""
    import torch
    log_n = 16
    n = 1 << log_n
    ps = list(chain(log_n, 60, 34))
    ctx, orc = make_pair(log_n, ps[2:34], ps[:1])
    nprime, npoly = 32, 64
    assert sorted({poly for _, poly in C2_FWD_ROWS}) == list(range(npoly))
    g = torch.Generator(device="cuda").manual_seed(0)
    mods = torch.tensor([orc.primes[i] for i in range(nprime)], dtype=torch.int64, device="cuda")
    x = torch.randint(0, 1 << 62, (npoly, nprime, n), generator=g, device="cuda", dtype=torch.int64)
    x = torch.remainder(x, mods.view(1, nprime, 1))
    x0 = x.clone()
    ctx.ntt_fwd(x, 0, nprime)
    fwd = x.clone()
    for prime, poly in C2_FWD_ROWS:
        want = orc.ntt_fwd(prime, host(x0[poly, prime]))
        assert np.array_equal(host(x[poly, prime]), want), f"forward row (poly {poly}, prime {prime})"
    ctx.ntt_inv(x, 0, nprime)
    for prime in range(nprime):
        poly = (5 * prime + 1) % npoly
        want = orc.ntt_inv(prime, host(fwd[poly, prime]))
        assert np.array_equal(host(x[poly, prime]), want), f"inverse row (poly {poly}, prime {prime})"
    assert torch.equal(x, x0)
