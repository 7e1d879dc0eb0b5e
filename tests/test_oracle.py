"""CPU tests of the oracle itself: definitions, round trips, and pins.

The reference ships no golden vectors (its correctness programs only print
slots), so the oracle is pinned by (a) independent restatements of the
definitions it claims (naive NTT evaluation, schoolbook negacyclic product,
big-integer CRT), (b) libsodium's XSalsa20 through PyNaCl, and (c) the
committed fixtures in tests/golden/ produced by the reference's own kernels
(the recipe is in the docstring of tests/golden/make_ref_fixtures.py).
"""
import numpy as np
import pytest

from tests.params import T65537, c3_primes, small_primes

pytestmark = []


def brv(x, bits):
    r = 0
    for _ in range(bits):
        r = (r << 1) | (x & 1)
        x >>= 1
    return r


def test_primes_and_roots(oracle_mod):
    O = oracle_mod
    ps = O.primes_bits(1 << 14, 60, 8)
    assert len(ps) == 8
    for q in ps:
        assert O.is_prime(q) and (q - 1) % (1 << 15) == 0 and q < (1 << 60)
        psi = O.root_2n(q, 1 << 14)
        assert pow(psi, 1 << 14, q) == q - 1
    assert ps == sorted(ps, reverse=True)


def test_reference_r_base_rule(oracle_mod):
    """R = r_num primes 1 mod 2N below min q, descending (uintarith_bfv.h:983-1016)."""
    O = oracle_mod
    q = [0x7FFE28001, 0x7FFF18001, 0x7FFF80001, 0x7FFFB0001]
    r = O.primes_below(1 << 14, min(q), 5)
    assert len(r) == 5 and all(x < min(q) for x in r)
    step = 1 << 15
    # every skipped candidate between consecutive R primes is composite
    v = min(q) - step
    got = []
    while len(got) < 5:
        if O.is_prime(v):
            got.append(v)
        v -= step
    assert got == r


def _ref_primitive_root(q):
    """Python restatement of findPrimeFactors/findPrimitiveRoot (Utils.cuh:54-88)."""
    import math
    s, number = set(), q - 1
    while number % 2 == 0:
        s.add(2)
        number //= 2
    i = 3
    while i < math.sqrt(number):
        while number % i == 0:
            s.add(i)
            number //= i
        i += 1
    if number > 2:
        s.add(number)
    phi = q - 1
    for r in range(2, phi + 1):
        if all(pow(r, phi // f, q) != 1 for f in s):
            return r
    return None


def test_primitive_root_quirk(oracle_mod):
    """The reference's factor loop stops at sqrt of the shrinking cofactor; a
    cofactor 9 is kept as the 'prime' 9. The oracle restates that search."""
    O = oracle_mod
    primes = [65537, 786433, 23068673, 0x7FFE28001, 0xFFFFCA8001]
    # primes q = 1 + 2^k * 9 (cofactor 9 after removing 2s)
    k, found = 10, 0
    while found < 3 and k < 40:
        q = 1 + (1 << k) * 9
        if O.is_prime(q):
            primes.append(q)
            found += 1
        k += 1
    for q in primes:
        assert O.primitive_root(q) == _ref_primitive_root(q), q


@pytest.mark.parametrize("log_n", [4, 5, 6])
def test_ntt_matches_definition(oracle_mod, log_n):
    """Output index k holds A(psi^(2*brv(k)+1)) (ntt_60bit.cuh:289-601 convention)."""
    O = oracle_mod
    n = 1 << log_n
    q = O.primes_bits(n, 30, 2)
    o = O.Oracle(log_n, 65537, q[:1], q[1:], dnum=1)
    rng = np.random.default_rng(log_n)
    a = rng.integers(0, q[0], size=n, dtype=np.uint64)
    A = o.ntt_fwd(0, a)
    psi = o.psi(0)
    for k in range(n):
        x = pow(psi, 2 * brv(k, log_n) + 1, q[0])
        v = 0
        for j in reversed(range(n)):
            v = (v * x + int(a[j])) % q[0]
        assert int(A[k]) == v
    assert np.array_equal(o.ntt_inv(0, A), a)


def test_ntt_convolution(oracle_mod):
    O = oracle_mod
    qs, ps = small_primes(10, 2, 1, 40)
    o = O.Oracle(10, 65537, qs, ps)
    n = o.n
    rng = np.random.default_rng(3)
    q = qs[0]
    a = rng.integers(0, q, size=n, dtype=np.uint64)
    b = rng.integers(0, q, size=n, dtype=np.uint64)
    A, B = o.ntt_fwd(0, a), o.ntt_fwd(0, b)
    prod = np.array([(int(x) * int(y)) % q for x, y in zip(A, B)], dtype=np.uint64)
    c = o.ntt_inv(0, prod)
    assert np.array_equal(c, O.negacyclic_mul(a, b, q))


def _crt(vals, mods):
    Q = 1
    for m in mods:
        Q *= m
    x = 0
    for v, m in zip(vals, mods):
        Mi = Q // m
        x += int(v) * Mi * pow(Mi, -1, m)
    return x % Q, Q


def test_bconv_is_centred_lift(oracle_mod):
    O = oracle_mod
    qs, ps = small_primes(10, 3, 1, 50)
    o = O.Oracle(10, 65537, qs, ps)
    rng = np.random.default_rng(5)
    x = np.stack([rng.integers(0, q, size=o.n, dtype=np.uint64) for q in qs])
    y = o.bconv_q_to_r(x)
    for k in range(0, o.n, 37):
        v, Q = _crt(x[:, k], qs)
        if v > Q // 2:
            v -= Q
        for j, r in enumerate(o.r):
            assert int(y[j, k]) == v % r


@pytest.mark.parametrize("bits,tol", [(30, 0), (60, 1 << 10)])
def test_scale_round_matches_bigint(oracle_mod, bits, tol):
    """round(t/Q * x) mod R for x given over Q|R (poly_arithmetic.cuh:1263-1307).

    The reference accumulates sum x_i * frac_i in one double; with 30-bit
    primes that sum is exact enough for exact rounding, with 60-bit primes
    its integer part (up to 2^62) leaves no fractional bits, so the rounding
    is off by a bounded amount (extra noise of the product, not a failure).
    """
    O = oracle_mod
    qs, ps = small_primes(10, 3, 1, bits)
    o = O.Oracle(10, 65537, qs, ps)
    rng = np.random.default_rng(9)
    mods = list(qs) + list(o.r)
    QR = 1
    for m in mods:
        QR *= m
    Q = 1
    for m in qs:
        Q *= m
    lim = QR // (4 * o.n)
    vals = []
    for k in range(o.n):
        v = 0
        for _ in range(len(mods)):
            v = (v << 62) | int(rng.integers(0, 1 << 62))
        vals.append((v % lim) * (1 if k % 2 else -1))
    x = np.array([[v % m for v in vals] for m in mods], dtype=np.uint64)
    y = o.scale_round_qr_r(x)
    R = QR // Q
    worst = 0
    for k in range(o.n):
        want = (2 * 65537 * vals[k] + Q) // (2 * Q)  # round half up
        got, _ = _crt(y[:, k], o.r)
        d = (got - want) % R
        d = min(d, R - d)
        worst = max(worst, d)
    assert worst <= tol


def test_scheme_roundtrip_small(oracle_mod):
    O = oracle_mod
    qs, ps = small_primes(12, 3, 1, 50)
    o = O.Oracle(12, T65537, qs, ps)
    key = bytes(range(32))
    sk = o.keygen_secret(key)
    pk = o.keygen_public(key, sk)
    rlk = o.keygen_relin(key, sk)
    rng = np.random.default_rng(1)
    v1 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
    v2 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
    m1, m2 = o.encode(v1), o.encode(v2)
    assert np.array_equal(o.decode(m1), v1)
    c1, c2 = o.encrypt(key, 1, pk, m1), o.encrypt(key, 2, pk, m2)
    assert np.array_equal(o.decode(o.decrypt(sk, c1)), v1)
    assert np.array_equal(o.decode(o.decrypt(sk, o.add(c1, c2))), (v1 + v2) % T65537)
    c3 = o.mul_relin(c1, c2, rlk)
    assert np.array_equal(o.decode(o.decrypt(sk, c3)), (v1 * v2) % T65537)
    assert o.noise_budget(sk, c3) > 0
    # tensor + separate relinearisation == fused
    assert np.array_equal(o.relinearize(o.mul_tensor(c1, c2), rlk), c3)


def test_scheme_c3_params(oracle_mod):
    """N=16384, 7x60-bit q + 1 special prime, t=65537, dnum=1 (the benchmark parameters)."""
    O = oracle_mod
    qs, ps = c3_primes()
    o = O.Oracle(14, T65537, qs, ps, dnum=1)
    assert o.decrypt_variant() == 3
    key = b"\x11" * 32
    sk = o.keygen_secret(key)
    pk = o.keygen_public(key, sk)
    rlk = o.keygen_relin(key, sk)
    rng = np.random.default_rng(7)
    v1 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
    v2 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
    c1 = o.encrypt(key, 10, pk, o.encode(v1))
    c2 = o.encrypt(key, 11, pk, o.encode(v2))
    c3 = o.mul_relin(c1, c2, rlk)
    assert np.array_equal(o.decode(o.decrypt(sk, c3)), (v1 * v2) % T65537)
    assert o.noise_budget(sk, c3) > 10


def test_scheme_c1_params(oracle_mod):
    """N=4096, q = 36+36 bits, special prime 37 bits, t=65537, ternary secret,
    Gaussian error sigma 3.2, one digit per ciphertext prime (dnum=2): batch-encode
    two vectors of 4096 values mod t, encrypt, multiply, relinearise, decrypt."""
    from tests.params import c1_primes
    O = oracle_mod
    qs, ps = c1_primes()
    o = O.Oracle(12, T65537, qs, ps, dnum=2)
    key = b"\x01" * 32
    sk = o.keygen_secret(key)
    pk = o.keygen_public(key, sk)
    rlk = o.keygen_relin(key, sk)
    rng = np.random.default_rng(41)
    v1 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
    v2 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
    c1 = o.encrypt(key, 0, pk, o.encode(v1))
    c2 = o.encrypt(key, 1, pk, o.encode(v2))
    c3 = o.mul_relin(c1, c2, rlk)
    assert np.array_equal(o.decode(o.decrypt(sk, c3)), (v1 * v2) % T65537)
    assert o.noise_budget(sk, c3) > 0


def test_hybrid_dnum(oracle_mod):
    O = oracle_mod
    qs, ps = small_primes(12, 4, 2, 45)
    for dnum in (1, 2, 4):
        o = O.Oracle(12, T65537, qs, ps, dnum=dnum)
        key = bytes([dnum]) * 32
        sk = o.keygen_secret(key)
        pk = o.keygen_public(key, sk)
        rlk = o.keygen_relin(key, sk)
        rng = np.random.default_rng(dnum)
        v1 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
        v2 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
        c3 = o.mul_relin(o.encrypt(key, 1, pk, o.encode(v1)), o.encrypt(key, 2, pk, o.encode(v2)), rlk)
        assert np.array_equal(o.decode(o.decrypt(sk, c3)), (v1 * v2) % T65537)


def test_modup_one_prime_digits_consistent(oracle_mod):
    """With one prime per digit the lift's float estimate of x / q_j rounds to
    1 for x close to q_j; the lifted residues must still represent one integer
    (x or x - q_j) in every prime of Q|P."""
    qs, ps = small_primes(12, 3, 1, 50)
    o = oracle_mod.Oracle(12, T65537, qs, ps, dnum=3)
    n = o.n
    rng = np.random.default_rng(3)
    x = np.stack([rng.integers(0, q, size=n, dtype=np.uint64) for q in qs])
    for j, q in enumerate(qs):  # values whose float ratio to q rounds to 1.0
        x[j, :64] = q - 1 - np.arange(64, dtype=np.uint64)
    lift = o.modup(x)
    PQ = list(qs) + list(ps)
    for d, qd in enumerate(qs):
        for k in list(range(64)) + [100, 2000]:
            v = int(x[d, k])
            got = [int(lift[d, m, k]) for m in range(len(PQ))]
            assert got in ([v % m for m in PQ], [(v - qd) % m for m in PQ]), (d, k)


def _levels_setup(oracle_mod):
    """6 x 50-bit q, 2 x 52-bit special primes, digits of 2 primes (dnum 3), N=4096."""
    p = oracle_mod.primes_bits(4096, 52, 2)
    q = oracle_mod.primes_bits(4096, 50, 6, skip=p)
    top = oracle_mod.Oracle(12, T65537, q, p, alpha=2)
    key = b"\x33" * 32
    sk = top.keygen_secret(key)
    return top, q, p, key, sk, top.keygen_public(key, sk), top.keygen_relin(key, sk)


def _crt_rows(rows, mods):
    Q = 1
    for m in mods:
        Q *= m
    acc = [0] * rows.shape[1]
    for i, m in enumerate(mods):
        f = (Q // m) * pow(Q // m, -1, m)
        for k, v in enumerate(rows[i]):
            acc[k] += int(v) * f
    return [a % Q for a in acc], Q


def test_mod_switch_is_divide_and_round(oracle_mod):
    """c' = (c - r) / q_l with r = c mod q_l centred: checked with big integers."""
    top, q, p, key, sk, pk, rlk = _levels_setup(oracle_mod)
    rng = np.random.default_rng(8)
    ct = top.encrypt(key, 5, pk, top.encode(rng.integers(0, T65537, size=top.n, dtype=np.uint64)))
    out = top.mod_switch(ct)
    lower = oracle_mod.Oracle(12, T65537, q[:5], p, alpha=2)
    ql, h = q[5], q[5] >> 1
    for poly in range(2):
        coef = np.stack([top.ntt_inv(i, ct[poly][i]) for i in range(6)])
        big, _ = _crt_rows(coef, q)
        got = np.stack([lower.ntt_inv(i, out[poly][i]) for i in range(5)])
        gbig, Q5 = _crt_rows(got, q[:5])
        for k in range(0, top.n, 97):
            r = (big[k] + h) % ql - h
            assert (big[k] - r) % ql == 0
            assert gbig[k] == ((big[k] - r) // ql) % Q5, k


def test_levels_decrypt_and_multiply(oracle_mod):
    """Encrypt at the top level, switch down, multiply at each level with the
    top-level key restricted to the live primes (digits keep their top-level
    primes; the last digit may be partial), decrypt exactly."""
    top, q, p, key, sk, pk, rlk = _levels_setup(oracle_mod)
    rng = np.random.default_rng(9)
    v1 = rng.integers(0, T65537, size=top.n, dtype=np.uint64)
    v2 = rng.integers(0, T65537, size=top.n, dtype=np.uint64)
    c1 = top.encrypt(key, 1, pk, top.encode(v1))
    c2 = top.encrypt(key, 2, pk, top.encode(v2))
    nq = len(q)
    for live in (6, 5, 4, 3):
        o = oracle_mod.Oracle(12, T65537, q[:live], p, alpha=2)
        skl = np.concatenate([sk[:live], sk[nq:]])
        assert np.array_equal(o.decode(o.decrypt(skl, c1)), v1)
        dl = o.dnum
        rl = np.stack([np.stack([np.concatenate([rlk[d][h][:live], rlk[d][h][nq:]]) for h in range(2)])
                       for d in range(dl)])
        prod = o.mul_relin(c1, c2, rl)
        assert np.array_equal(o.decode(o.decrypt(skl, prod)), (v1 * v2) % T65537), live
        if live > 3:
            c1, c2 = o.mod_switch(c1), o.mod_switch(c2)


def test_gadget_key_switch(oracle_mod):
    """Key switching over a base-2^20 gadget decomposition (3 pieces per 60-bit
    prime) decrypts exactly, at the top level and at a lower level with the
    key restricted to the live primes, with far less noise than the hybrid
    method's one-digit key switch."""
    top, q, p, key, sk, pk, rlk = _levels_setup(oracle_mod)
    w = 20
    gk = top.keygen_relin_gadget(key, sk, w)
    J = 3
    assert gk.shape == (6 * J, 2, 8, top.n)
    rng = np.random.default_rng(12)
    v1 = rng.integers(0, T65537, size=top.n, dtype=np.uint64)
    v2 = rng.integers(0, T65537, size=top.n, dtype=np.uint64)
    c1 = top.encrypt(key, 1, pk, top.encode(v1))
    c2 = top.encrypt(key, 2, pk, top.encode(v2))
    d = top.mul_tensor(c1, c2)
    out = top.relinearize_gadget(d, gk, w)
    assert np.array_equal(top.decode(top.decrypt(sk, out)), (v1 * v2) % T65537)
    hyb = top.relinearize(d, rlk)
    assert top.noise_budget(sk, out) >= top.noise_budget(sk, hyb) - 1
    # level 4 (two primes switched away) with the first 4 * J key components
    o = oracle_mod.Oracle(12, T65537, q[:4], p, alpha=2)
    a, b = top.mod_switch(c1), top.mod_switch(c2)
    o5 = oracle_mod.Oracle(12, T65537, q[:5], p, alpha=2)
    a, b = o5.mod_switch(a), o5.mod_switch(b)
    gl = np.stack([np.stack([np.concatenate([gk[g][h][:4], gk[g][h][6:]]) for h in range(2)]) for g in range(4 * J)])
    skl = np.concatenate([sk[:4], sk[6:]])
    res = o.relinearize_gadget(o.mul_tensor(a, b), gl, w)
    assert np.array_equal(o.decode(o.decrypt(skl, res)), (v1 * v2) % T65537)


def test_galois_automorphisms(oracle_mod):
    """Automorphism X -> X^g in NTT form + key switch decrypts to m(X^g) for
    rotations (g = 5^r) and conjugation (g = 2N - 1); the NTT-form permutation
    equals the coefficient-form automorphism."""
    qs, ps = small_primes(12, 3, 1, 50)
    o = oracle_mod.Oracle(12, T65537, qs, ps)
    n = o.n
    key = b"\x05" * 32
    sk = o.keygen_secret(key)
    pk = o.keygen_public(key, sk)
    rng = np.random.default_rng(0)
    m = o.encode(rng.integers(0, T65537, size=n, dtype=np.uint64))
    ct = o.encrypt(key, 1, pk, m)

    def auto(poly, g, mod):
        out = np.zeros(n, dtype=object)
        for i in range(n):
            e = (i * g) % (2 * n)
            if e < n:
                out[e] = (out[e] + int(poly[i])) % mod
            else:
                out[e - n] = (out[e - n] - int(poly[i])) % mod
        return out.astype(np.uint64)

    x = rng.integers(0, qs[0], size=n, dtype=np.uint64)
    for g in (5, 25, 2 * n - 1):
        # permutation in NTT form == automorphism in coefficient form
        got = o.ntt_inv(0, o.galois_ntt(g, o.ntt_fwd(0, x)))
        assert np.array_equal(got, auto(x, g, qs[0]))
        gk = o.keygen_galois(key, sk, g)
        r = o.apply_galois(gk, g, ct)
        assert np.array_equal(o.decode(o.decrypt(sk, r)), o.decode(auto(m, g, T65537)))
        assert o.noise_budget(sk, r) > 10


def test_xsalsa20_against_libsodium(oracle_mod):
    """Pin the XSalsa20 keystream to libsodium's crypto_secretbox (PyNaCl):
    secretbox XORs the message with keystream bytes from offset 32."""
    nacl = pytest.importorskip("nacl.bindings")
    O = oracle_mod
    rng = np.random.default_rng(0)
    for trial in range(4):
        key = bytes(rng.integers(0, 256, 32, dtype=np.uint8))
        nonce = bytes(rng.integers(0, 256, 24, dtype=np.uint8))
        n = 64 * 5 + trial * 7
        box = nacl.crypto_secretbox(b"\x00" * n, nonce, key)
        ks = box[-n:]
        ours = O.xsalsa20(key, nonce, 32 + n)[32:]
        assert ours == ks


def test_gaussian_sampler_statistics(oracle_mod):
    O = oracle_mod
    qs, ps = small_primes(14, 1, 1, 50)
    o = O.Oracle(14, T65537, qs, ps)
    xs = np.concatenate([o.sample_gaussian(b"\x05" * 32, 3, i, 0) for i in range(8)])
    assert abs(xs.mean()) < 0.05
    assert abs(xs.std() - 3.2) < 0.05
    assert xs.min() >= -19 and xs.max() <= 19
    t = o.sample_ternary(b"\x05" * 32, 6, 0, 0)
    counts = [(t == v).sum() for v in (-1, 0, 1)]
    assert min(counts) > 0.3 * len(t)


def test_hwt_sampler(oracle_mod):
    O = oracle_mod
    qs, ps = small_primes(14, 1, 1, 50)
    o = O.Oracle(14, T65537, qs, ps)
    s = o.sample_hwt(b"\x01" * 32, 1, 0, 0, 64)
    assert 0 < np.count_nonzero(s) <= 64
    assert set(np.unique(s)) <= {-1, 0, 1}
