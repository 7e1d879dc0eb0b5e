"""Parameter sets shared by the tests (prime lists come from the oracle's generator)."""
import functools

import oracle

T65537 = 65537


@functools.lru_cache(maxsize=None)
def chain(log_n: int, bits: int, count: int):
    return tuple(oracle.primes_bits(1 << log_n, bits, count))


@functools.lru_cache(maxsize=None)
def c3_primes():
    """N=16384, 7 x 60-bit ciphertext primes + 1 special prime (largest first)."""
    ps = chain(14, 60, 8)
    return list(ps[1:8]), [ps[0]]


@functools.lru_cache(maxsize=None)
def small_primes(log_n: int = 12, nq: int = 3, np_: int = 1, bits: int = 50):
    ps = chain(log_n, bits, nq + np_)
    return list(ps[np_:np_ + nq]), list(ps[:np_])


def plain_modulus_for(log_n: int) -> int:
    """65537 while 2N divides 65536, else 786433 (= 3 * 2^18 + 1)."""
    return 65537 if (2 << log_n) <= 65536 else 786433


@functools.lru_cache(maxsize=None)
def c1_primes():
    """N=4096: ciphertext primes of 36 and 36 bits, special prime of 37 bits
    (SEAL's default coeff_modulus sizes for N=4096), all 1 mod 8192."""
    p = oracle.primes_bits(4096, 37, 1)
    q = oracle.primes_bits(4096, 36, 2, skip=p)
    return q, p
