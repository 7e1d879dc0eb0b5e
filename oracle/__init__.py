"""CPU oracle for the BFV multiply path (test infrastructure only).

This package is the checker for the CUDA product: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import it.
It wraps ``liboracle.so`` (built from ``kbfv_oracle.c`` by ``make -C oracle``),
a C restatement of the reference's algorithms; see ``kbfv_oracle.c`` for the
reference file:line each function follows.

Arrays are numpy ``uint64`` in limb-major order ``poly[limb][coeff]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

U64P = C.POINTER(C.c_uint64)
I64P = C.POINTER(C.c_int64)
U8P = C.POINTER(C.c_uint8)


def build(force: bool = False) -> str:
    """Compile the oracle with make (gcc); returns the library path."""
    src = os.path.join(_HERE, "kbfv_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", _HERE, "-s"], check=True)
    return _LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L: C.CDLL) -> None:
    V = None
    sig = {
        "orc_is_prime": (C.c_int, [C.c_uint64]),
        "orc_primes_below": (C.c_size_t, [C.c_uint64, C.c_uint64, C.c_size_t, U64P, C.c_int]),
        "orc_primes_bits": (C.c_size_t, [C.c_uint64, C.c_int, C.c_size_t, U64P, C.c_size_t, U64P]),
        "orc_primitive_root": (C.c_uint64, [C.c_uint64]),
        "orc_root_2n": (C.c_uint64, [C.c_uint64, C.c_uint64]),
        "orc_root_is_primitive": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint64]),
        "orc_create": (C.c_void_p, [C.c_uint32, C.c_uint64, U64P, C.c_int, U64P, C.c_int, C.c_int,
                                    U64P, C.c_int, C.c_int]),
        "orc_destroy": (V, [C.c_void_p]),
        "orc_set_ref_compat": (V, [C.c_void_p, C.c_int]),
        "orc_klss_relinearize": (V, [C.c_void_p, U64P, U64P, U64P]),
        "orc_mod_switch": (V, [C.c_void_p, U64P, U64P, C.c_int]),
        "orc_gadget_pieces": (C.c_int, [C.c_int]),
        "orc_galois_ntt": (V, [C.c_void_p, C.c_uint64, U64P, U64P, C.c_int]),
        "orc_keygen_galois": (V, [C.c_void_p, U8P, U64P, C.c_uint64, U64P]),
        "orc_apply_galois": (V, [C.c_void_p, U64P, C.c_uint64, U64P, U64P]),
        "orc_keygen_relin_gadget": (V, [C.c_void_p, U8P, U64P, C.c_int, U64P]),
        "orc_relinearize_gadget": (V, [C.c_void_p, U64P, U64P, C.c_int, U64P]),
        "orc_prime_count": (C.c_int, [C.c_void_p]),
        "orc_primes": (V, [C.c_void_p, U64P]),
        "orc_psi": (C.c_uint64, [C.c_void_p, C.c_int]),
        "orc_ntt_fwd": (V, [C.c_void_p, C.c_int, U64P, C.c_int]),
        "orc_ntt_inv": (V, [C.c_void_p, C.c_int, U64P, C.c_int]),
        "orc_bconv_q_to_r": (V, [C.c_void_p, U64P, U64P]),
        "orc_bconv_r_to_q": (V, [C.c_void_p, U64P, U64P]),
        "orc_tensor_qr": (V, [C.c_void_p, U64P, U64P, U64P]),
        "orc_scale_round_qr_r": (V, [C.c_void_p, U64P, U64P]),
        "orc_scale_round_qr_r_ref": (V, [C.c_void_p, U64P, U64P]),
        "orc_decrypt_round": (V, [C.c_void_p, U64P, U64P, C.c_int]),
        "orc_decrypt_variant": (C.c_int, [C.c_void_p]),
        "orc_delta_m": (V, [C.c_void_p, U64P, U64P]),
        "orc_modup": (V, [C.c_void_p, U64P, U64P]),
        "orc_moddown": (V, [C.c_void_p, U64P, U64P, C.c_int]),
        "orc_klss_ri_blocks": (C.c_int, [C.c_void_p]),
        "orc_klss_qj_blocks": (C.c_int, [C.c_void_p]),
        "orc_klss_modup_qj_to_t": (V, [C.c_void_p, U64P, U64P]),
        "orc_klss_modup_pq_to_t": (V, [C.c_void_p, U64P, U64P]),
        "orc_klss_external_product": (V, [C.c_void_p, U64P, U64P, U64P]),
        "orc_klss_modup_t_to_pq": (V, [C.c_void_p, U64P, U64P, C.c_int]),
        "orc_klss_moddown": (V, [C.c_void_p, U64P, U64P, C.c_int]),
        "orc_hsalsa20": (V, [U8P, U8P, U8P]),
        "orc_xsalsa20_stream": (V, [U8P, U8P, C.c_uint64, U8P, C.c_size_t]),
        "orc_salsa20_compat_stream": (V, [U8P, C.c_uint64, U8P, C.c_size_t]),
        "orc_gaussian_cdt": (V, [C.c_double, C.c_int, U64P]),
        "orc_sample_uniform": (V, [C.c_void_p, U8P, C.c_uint32, C.c_uint64, C.c_uint32,
                                   C.POINTER(C.c_int), C.c_int, U64P]),
        "orc_sample_ternary": (V, [C.c_void_p, U8P, C.c_uint32, C.c_uint64, C.c_uint32, I64P]),
        "orc_sample_gaussian": (V, [C.c_void_p, U8P, C.c_uint32, C.c_uint64, C.c_uint32, I64P]),
        "orc_sample_hwt": (V, [C.c_void_p, U8P, C.c_uint32, C.c_uint64, C.c_uint32, C.c_int, I64P]),
        "orc_keygen_secret": (V, [C.c_void_p, U8P, C.c_int, C.c_int, U64P]),
        "orc_keygen_public": (V, [C.c_void_p, U8P, U64P, U64P]),
        "orc_keygen_relin": (V, [C.c_void_p, U8P, U64P, U64P]),
        "orc_encode": (V, [C.c_void_p, U64P, U64P]),
        "orc_decode": (V, [C.c_void_p, U64P, U64P]),
        "orc_encrypt": (V, [C.c_void_p, U8P, C.c_uint64, U64P, U64P, U64P]),
        "orc_decrypt": (V, [C.c_void_p, U64P, U64P, U64P]),
        "orc_add": (V, [C.c_void_p, U64P, U64P, U64P, C.c_int]),
        "orc_mul_plain": (V, [C.c_void_p, U64P, U64P, U64P]),
        "orc_mul_tensor": (V, [C.c_void_p, U64P, U64P, U64P]),
        "orc_relinearize": (V, [C.c_void_p, U64P, U64P, U64P]),
        "orc_mul_relin": (V, [C.c_void_p, U64P, U64P, U64P, U64P]),
        "orc_noise_budget": (C.c_double, [C.c_void_p, U64P, U64P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    if a.dtype == np.uint64:
        return a.ctypes.data_as(U64P)
    if a.dtype == np.int64:
        return a.ctypes.data_as(I64P)
    if a.dtype == np.uint8:
        return a.ctypes.data_as(U8P)
    raise TypeError(a.dtype)


def _key(key: bytes) -> np.ndarray:
    assert len(key) == 32
    return np.frombuffer(bytes(key), dtype=np.uint8).copy()


def is_prime(n: int) -> bool:
    return bool(lib().orc_is_prime(n))


def primes_below(n: int, upper: int, count: int, require_root: bool = True) -> list:
    out = np.zeros(count, dtype=np.uint64)
    got = lib().orc_primes_below(n, upper, count, _p(out), int(require_root))
    return [int(x) for x in out[:got]]


def primes_bits(n: int, bits: int, count: int, skip=()) -> list:
    out = np.zeros(count, dtype=np.uint64)
    sk = np.array(list(skip) or [0], dtype=np.uint64)
    got = lib().orc_primes_bits(n, bits, count, _p(sk), len(skip), _p(out))
    return [int(x) for x in out[:got]]


def primitive_root(q: int) -> int:
    return int(lib().orc_primitive_root(q))


def root_2n(q: int, n: int) -> int:
    return int(lib().orc_root_2n(q, n))


def xsalsa20(key: bytes, nonce: bytes, nbytes: int, block0: int = 0) -> bytes:
    out = np.zeros(nbytes, dtype=np.uint8)
    nn = np.frombuffer(bytes(nonce), dtype=np.uint8).copy()
    lib().orc_xsalsa20_stream(_p(_key(key)), _p(nn), block0, _p(out), nbytes)
    return out.tobytes()


def salsa20_compat(key: bytes, nonce: int, nbytes: int) -> bytes:
    out = np.zeros(nbytes, dtype=np.uint8)
    lib().orc_salsa20_compat_stream(_p(_key(key)), nonce, _p(out), nbytes)
    return out.tobytes()


def gaussian_cdt(sigma: float = 3.2, bound: int = 19) -> np.ndarray:
    out = np.zeros(2 * bound + 1, dtype=np.uint64)
    lib().orc_gaussian_cdt(sigma, bound, _p(out))
    return out


class Oracle:
    """An oracle context for one parameter set (see ``orc_create``)."""

    def __init__(self, log_n: int, t: int, q, p, dnum: int = 1, tk=(), gamma: int = 1, alpha: int = 0):
        """alpha > 0 fixes the key-switch digit size (digits = ceil(nq / alpha))."""
        L = lib()
        self.log_n = log_n
        self.n = 1 << log_n
        self.t = t
        self.nq, self.np_ = len(q), len(p)
        self.nr = self.nq + 1
        self.nt = len(tk)
        self.dnum = -(-len(q) // alpha) if alpha else dnum
        qa = np.array(q, dtype=np.uint64)
        pa = np.array(p if len(p) else [0], dtype=np.uint64)
        ta = np.array(tk if len(tk) else [0], dtype=np.uint64)
        self._h = L.orc_create(log_n, t, _p(qa), len(q), _p(pa), len(p), -alpha if alpha else dnum, _p(ta), len(tk),
                               gamma)
        if not self._h:
            raise ValueError("oracle context creation failed (not enough R primes)")
        cnt = L.orc_prime_count(self._h)
        pr = np.zeros(cnt, dtype=np.uint64)
        L.orc_primes(self._h, _p(pr))
        self.primes = [int(x) for x in pr]
        self.q = self.primes[: self.nq]
        self.p = self.primes[self.nq: self.nq + self.np_]
        self.r = self.primes[self.nq + self.np_: self.nq + self.np_ + self.nr]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.orc_destroy(h)
            self._h = None

    # ---- index helpers
    def q_index(self, i):
        return i

    def p_index(self, i):
        return self.nq + i

    def r_index(self, j):
        return self.nq + self.np_ + j

    def t_index(self):
        return len(self.primes) - 1

    def psi(self, idx: int) -> int:
        return int(lib().orc_psi(self._h, idx))

    # ---- NTT
    def ntt_fwd(self, idx: int, rows: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(rows, dtype=np.uint64).copy()
        lib().orc_ntt_fwd(self._h, idx, _p(a), a.size // self.n)
        return a

    def ntt_inv(self, idx: int, rows: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(rows, dtype=np.uint64).copy()
        lib().orc_ntt_inv(self._h, idx, _p(a), a.size // self.n)
        return a

    def ntt_fwd_limbs(self, idxs, poly: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(poly, dtype=np.uint64).reshape(len(idxs), self.n).copy()
        for l, i in enumerate(idxs):
            row = np.ascontiguousarray(a[l])
            lib().orc_ntt_fwd(self._h, i, _p(row), 1)
            a[l] = row
        return a

    # ---- HPS
    def _call(self, fn, *ins, out_shape, extra=()):
        ins = [np.ascontiguousarray(x, dtype=np.uint64) for x in ins]
        out = np.zeros(out_shape, dtype=np.uint64)
        getattr(lib(), fn)(self._h, *[_p(x) for x in ins], _p(out), *extra)
        return out

    def bconv_q_to_r(self, x):
        return self._call("orc_bconv_q_to_r", x, out_shape=(self.nr, self.n))

    def bconv_r_to_q(self, x):
        return self._call("orc_bconv_r_to_q", x, out_shape=(self.nq, self.n))

    def tensor_qr(self, c1, c2):
        return self._call("orc_tensor_qr", c1, c2, out_shape=(3, self.nq + self.nr, self.n))

    def scale_round_qr_r(self, x):
        return self._call("orc_scale_round_qr_r", x, out_shape=(self.nr, self.n))

    def scale_round_qr_r_ref(self, x):
        """The reference's variant (alpha reduced in place across R primes)."""
        return self._call("orc_scale_round_qr_r_ref", x, out_shape=(self.nr, self.n))

    def decrypt_round(self, x, variant: int = -1):
        return self._call("orc_decrypt_round", x, out_shape=(self.n,), extra=(variant,))

    def decrypt_variant(self) -> int:
        return int(lib().orc_decrypt_variant(self._h))

    def delta_m(self, m):
        return self._call("orc_delta_m", m, out_shape=(self.nq, self.n))

    def modup(self, d2):
        return self._call("orc_modup", d2, out_shape=(self.dnum, self.nq + self.np_, self.n))

    def moddown(self, x, npoly: int = 2):
        return self._call("orc_moddown", x, out_shape=(npoly, self.nq, self.n), extra=(npoly,))

    def keygen_relin_gadget(self, key, sk, w: int):
        J = int(lib().orc_gadget_pieces(w))
        out = np.zeros((self.nq * J, 2, self.nq + self.np_, self.n), dtype=np.uint64)
        sk = np.ascontiguousarray(sk, dtype=np.uint64)
        lib().orc_keygen_relin_gadget(self._h, _p(_key(key)), _p(sk), w, _p(out))
        return out

    def relinearize_gadget(self, d, gk, w: int):
        d = np.ascontiguousarray(d, dtype=np.uint64)
        gk = np.ascontiguousarray(gk, dtype=np.uint64)
        out = np.zeros((2, self.nq, self.n), dtype=np.uint64)
        lib().orc_relinearize_gadget(self._h, _p(d), _p(gk), w, _p(out))
        return out

    def galois_ntt(self, g: int, x):
        x = np.ascontiguousarray(x, dtype=np.uint64)
        out = np.zeros_like(x)
        lib().orc_galois_ntt(self._h, g, _p(x), _p(out), x.size // self.n)
        return out

    def keygen_galois(self, key, sk, g: int):
        out = np.zeros((self.dnum, 2, self.nq + self.np_, self.n), dtype=np.uint64)
        sk = np.ascontiguousarray(sk, dtype=np.uint64)
        lib().orc_keygen_galois(self._h, _p(_key(key)), _p(sk), g, _p(out))
        return out

    def apply_galois(self, gk, g: int, ct):
        gk = np.ascontiguousarray(gk, dtype=np.uint64)
        ct = np.ascontiguousarray(ct, dtype=np.uint64)
        out = np.zeros((2, self.nq, self.n), dtype=np.uint64)
        lib().orc_apply_galois(self._h, _p(gk), g, _p(ct), _p(out))
        return out

    def mod_switch(self, ct, npoly: int = 2):
        return self._call("orc_mod_switch", ct, out_shape=(npoly, self.nq - 1, self.n), extra=(npoly,))

    # ---- KLSS
    def klss_blocks(self):
        return int(lib().orc_klss_ri_blocks(self._h)), int(lib().orc_klss_qj_blocks(self._h))

    def klss_modup_qj_to_t(self, d2):
        _, nqj = self.klss_blocks()
        return self._call("orc_klss_modup_qj_to_t", d2, out_shape=(nqj, self.nt, self.n))

    def klss_modup_pq_to_t(self, x_ref_order):
        nri, _ = self.klss_blocks()
        return self._call("orc_klss_modup_pq_to_t", x_ref_order, out_shape=(nri, self.nt, self.n))

    def klss_external_product(self, digits_t, key_t):
        nri, _ = self.klss_blocks()
        return self._call("orc_klss_external_product", digits_t, key_t, out_shape=(2, nri, self.nt, self.n))

    def klss_modup_t_to_pq(self, x_t, npoly: int = 2):
        nri, _ = self.klss_blocks()
        return self._call("orc_klss_modup_t_to_pq", x_t, out_shape=(npoly, nri * self.nt, self.n),
                          extra=(npoly,))

    def set_ref_compat(self, on: bool):
        lib().orc_set_ref_compat(self._h, int(on))

    def klss_relinearize(self, d, key_t):
        return self._call("orc_klss_relinearize", d, key_t, out_shape=(2, self.nq, self.n))

    def klss_moddown(self, x, npoly: int = 2):
        return self._call("orc_klss_moddown", x, out_shape=(npoly, self.nq, self.n), extra=(npoly,))

    # ---- samplers
    def sample_uniform(self, key, domain, ident, sub, idxs):
        ia = (C.c_int * len(idxs))(*idxs)
        out = np.zeros((len(idxs), self.n), dtype=np.uint64)
        lib().orc_sample_uniform(self._h, _p(_key(key)), domain, ident, sub, ia, len(idxs), _p(out))
        return out

    def _sample_small(self, fn, key, domain, ident, sub, *extra):
        out = np.zeros(self.n, dtype=np.int64)
        getattr(lib(), fn)(self._h, _p(_key(key)), domain, ident, sub, *extra, _p(out))
        return out

    def sample_ternary(self, key, domain, ident, sub):
        return self._sample_small("orc_sample_ternary", key, domain, ident, sub)

    def sample_gaussian(self, key, domain, ident, sub):
        return self._sample_small("orc_sample_gaussian", key, domain, ident, sub)

    def sample_hwt(self, key, domain, ident, sub, h=64):
        return self._sample_small("orc_sample_hwt", key, domain, ident, sub, h)

    # ---- scheme
    def keygen_secret(self, key, kind: int = 0, h: int = 64):
        out = np.zeros((self.nq + self.np_, self.n), dtype=np.uint64)
        lib().orc_keygen_secret(self._h, _p(_key(key)), kind, h, _p(out))
        return out

    def keygen_public(self, key, sk):
        out = np.zeros((2, self.nq, self.n), dtype=np.uint64)
        lib().orc_keygen_public(self._h, _p(_key(key)), _p(np.ascontiguousarray(sk)), _p(out))
        return out

    def keygen_relin(self, key, sk):
        out = np.zeros((self.dnum, 2, self.nq + self.np_, self.n), dtype=np.uint64)
        lib().orc_keygen_relin(self._h, _p(_key(key)), _p(np.ascontiguousarray(sk)), _p(out))
        return out

    def encode(self, slots):
        return self._call("orc_encode", slots, out_shape=(self.n,))

    def decode(self, m):
        return self._call("orc_decode", m, out_shape=(self.n,))

    def encrypt(self, key, enc_id, pk, m):
        out = np.zeros((2, self.nq, self.n), dtype=np.uint64)
        lib().orc_encrypt(self._h, _p(_key(key)), enc_id, _p(np.ascontiguousarray(pk)),
                          _p(np.ascontiguousarray(m, dtype=np.uint64)), _p(out))
        return out

    def decrypt(self, sk, ct):
        return self._call("orc_decrypt", sk, ct, out_shape=(self.n,))

    def add(self, x, y, npoly: int = 2):
        return self._call("orc_add", x, y, out_shape=(npoly, self.nq, self.n), extra=(npoly,))

    def mul_plain(self, ct, pt_ntt):
        return self._call("orc_mul_plain", ct, pt_ntt, out_shape=(2, self.nq, self.n))

    def mul_tensor(self, c1, c2):
        return self._call("orc_mul_tensor", c1, c2, out_shape=(3, self.nq, self.n))

    def relinearize(self, d, rlk):
        return self._call("orc_relinearize", d, rlk, out_shape=(2, self.nq, self.n))

    def mul_relin(self, c1, c2, rlk):
        return self._call("orc_mul_relin", c1, c2, rlk, out_shape=(2, self.nq, self.n))

    def noise_budget(self, sk, ct) -> float:
        return float(lib().orc_noise_budget(self._h, _p(np.ascontiguousarray(sk)), _p(np.ascontiguousarray(ct))))


def negacyclic_mul(a, b, q: int) -> np.ndarray:
    """Schoolbook product in Z_q[x]/(x^n+1) with Python ints (small n only)."""
    n = len(a)
    out = [0] * n
    for i in range(n):
        ai = int(a[i])
        if ai == 0:
            continue
        for j in range(n):
            k = i + j
            v = ai * int(b[j])
            if k < n:
                out[k] += v
            else:
                out[k - n] -= v
    return np.array([x % q for x in out], dtype=np.uint64)
