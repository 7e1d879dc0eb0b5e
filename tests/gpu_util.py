"""Helpers pairing a product context with an oracle context on the same primes."""
import functools

import numpy as np

import oracle
from tests.params import T65537, c3_primes, plain_modulus_for, small_primes


def dev(a):
    from kunpbfv_b200.api import to_device
    return to_device(np.ascontiguousarray(a, dtype=np.uint64))


def host(t):
    from kunpbfv_b200.api import to_host
    return to_host(t)


def make_pair(log_n, qs, ps, dnum=1, t=None):
    t = t or plain_modulus_for(log_n)
    import kunpbfv_b200 as kb
    ctx = kb.BFVContext(log_n=log_n, plain_modulus=t, q_count=len(qs), q=qs, p_count=len(ps), p=ps, dnum=dnum)
    orc = oracle.Oracle(log_n, t, qs, ps, dnum=dnum)
    assert ctx.primes == orc.primes, "product and oracle derive different prime tables"
    return ctx, orc


@functools.lru_cache(maxsize=None)
def c3_pair():
    qs, ps = c3_primes()
    return make_pair(14, qs, ps, 1)


@functools.lru_cache(maxsize=None)
def small_pair(log_n=12, nq=3, np_=1, bits=50, dnum=1):
    qs, ps = small_primes(log_n, nq, np_, bits)
    return make_pair(log_n, qs, ps, dnum)


def rand_rows(orc, idxs, n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.integers(0, orc.primes[i], size=n, dtype=np.uint64) for i in idxs])
