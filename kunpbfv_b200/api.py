"""ctypes bindings of libkbfv.so and the reference-shaped Python classes.

Class and method names follow kunpBFV (include/BFVScheme.h:12-178,
include/BFVcontext.h:17-391): ``BFVContext``, ``BFVScheme.encryptMsg``,
``decryptMsg``, ``addAndEqual``, ``multAndEqual_23``, ``multConstAndEqual``,
``BFVContext.encode`` / ``decode`` / ``encode_ntt``. Errors surface as
``KbfvError`` subclasses of the exception types the reference throws
(``ValueError`` for std::invalid_argument, ``RuntimeError`` otherwise).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libkbfv.so")
_lib: Optional[C.CDLL] = None

U64P = C.POINTER(C.c_uint64)
U8P = C.POINTER(C.c_uint8)
VP = C.c_void_p

KBFV_OK = 0
_ERR_NAMES = {
    -1: "invalid argument",
    -2: "parameter set",
    -3: "CUDA",
    -4: "out of device memory",
    -5: "missing key",
    -6: "level",
    -7: "unsupported",
}


# kbfv_tune_knob (include/kbfv.h)
TUNE_KNOBS = {"ntt_block_log": 0, "branches": 1, "host_chunk": 2, "split_rows": 3, "bconv_threads": 4,
              "k5_threads": 5, "k5_fused_pairs": 6, "bconv_cpt": 7,
              "fuse_q2r_pairs": 8, "l2_prefetch": 9,
              "split_rows_alone": 10, "min_branch_pairs": 11}


class KbfvError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"kbfv error {code} ({_ERR_NAMES.get(code, '?')}): {msg}")
        self.code = code


class KbfvInvalidArgument(KbfvError, ValueError):
    pass


class _Params(C.Structure):
    _fields_ = [
        ("log_n", C.c_uint32),
        ("plain_modulus", C.c_uint64),
        ("q_count", C.c_uint32),
        ("q", U64P),
        ("q_bits", C.c_uint32),
        ("p_count", C.c_uint32),
        ("p", U64P),
        ("p_bits", C.c_uint32),
        ("dnum", C.c_uint32),
        ("t_count", C.c_uint32),
        ("t_primes", U64P),
        ("gamma", C.c_uint32),
        ("digit_primes", C.c_uint32),
    ]


def library_path() -> str:
    return _LIB_PATH


def lib() -> C.CDLL:
    """Load libkbfv.so; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError(
                f"{_LIB_PATH} is missing; build it with `python -m kunpbfv_b200.build` "
                "(there is no CPU fallback)")
        L = C.CDLL(_LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L: C.CDLL) -> None:
    I = C.c_int
    u32, u64 = C.c_uint32, C.c_uint64
    sig = {
        "kbfv_last_error": (C.c_char_p, []),
        "kbfv_version": (C.c_char_p, []),
        "kbfv_context_create": (I, [C.POINTER(_Params), C.POINTER(VP)]),
        "kbfv_context_create_reference": (I, [u32, C.POINTER(VP)]),
        "kbfv_context_destroy": (I, [VP]),
        "kbfv_context_info": (I, [VP, U64P, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), C.POINTER(u32),
                                  C.POINTER(u32), C.POINTER(u32)]),
        "kbfv_context_primes": (I, [VP, U64P, C.POINTER(u32)]),
        "kbfv_context_plain_modulus": (u64, [VP]),
        "kbfv_context_decrypt_variant": (I, [VP]),
        "kbfv_mul_relin_scratch_bytes": (C.c_size_t, [VP, u32]),
        "kbfv_context_arena_bytes": (C.c_size_t, [VP]),
        "kbfv_reserve": (I, [VP, u32]),
        "kbfv_ntt_fwd": (I, [VP, VP, u32, u32, u32, VP]),
        "kbfv_ntt_inv": (I, [VP, VP, u32, u32, u32, VP]),
        "kbfv_bconv_q_to_r": (I, [VP, VP, VP, u32, VP]),
        "kbfv_bconv_r_to_q": (I, [VP, VP, VP, u32, VP]),
        "kbfv_tensor_qr": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_scale_round_qr_r": (I, [VP, VP, VP, u32, VP]),
        "kbfv_decrypt_round": (I, [VP, VP, VP, u32, VP]),
        "kbfv_delta_m": (I, [VP, VP, VP, u32, VP]),
        "kbfv_modup": (I, [VP, VP, VP, u32, VP]),
        "kbfv_moddown": (I, [VP, VP, VP, u32, VP]),
        "kbfv_keygen_secret": (I, [VP, U8P, I, u32, VP, VP]),
        "kbfv_keygen_public": (I, [VP, U8P, VP, VP, VP]),
        "kbfv_keygen_relin": (I, [VP, U8P, VP, VP, VP]),
        "kbfv_encode": (I, [VP, VP, VP, u32, VP]),
        "kbfv_decode": (I, [VP, VP, VP, u32, VP]),
        "kbfv_encode_ntt": (I, [VP, VP, VP, u32, VP]),
        "kbfv_encrypt": (I, [VP, U8P, u64, VP, VP, VP, u32, VP]),
        "kbfv_decrypt": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_add": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_mul_plain": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_mul": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_relinearize": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_mul_relin_batch": (I, [VP, VP, C.POINTER(VP), C.POINTER(VP), C.POINTER(VP), u32, VP]),
        "kbfv_set_branches": (I, [VP, u32]),
        "kbfv_tune_set": (I, [VP, I, C.c_int64]),
        "kbfv_tune_get": (I, [VP, I, C.POINTER(C.c_int64)]),
        "kbfv_mul_relin": (I, [VP, VP, VP, VP, VP, u32, VP]),
        "kbfv_mul_relin_noalloc": (I, [VP, VP, VP, VP, VP, u32, VP]),
        "kbfv_plan_mul_relin": (I, [VP, VP, VP, VP, VP, u32, C.POINTER(VP)]),
        "kbfv_plan_mul_relin_levels": (I, [VP, VP, C.POINTER(u32), C.POINTER(VP), C.POINTER(VP), C.POINTER(VP), u32,
                                           C.POINTER(VP)]),
        "kbfv_plan_launch": (I, [VP, VP]),
        "kbfv_plan_info": (I, [VP, C.POINTER(u64), C.POINTER(u64)]),
        "kbfv_plan_destroy": (I, [VP]),
        "kbfv_mul_relin_host": (I, [VP, VP, VP, VP, VP, u32, u32, VP]),
        "kbfv_context_klss": (I, [VP, C.POINTER(u32), C.POINTER(u32), U64P]),
        "kbfv_params_create": (I, [u32, C.POINTER(u32), u32, C.POINTER(u32), u32, u64, u32,
                                   C.POINTER(C.POINTER(_Params))]),
        "kbfv_params_destroy": (I, [C.POINTER(_Params)]),
        "kbfv_set_seed": (I, [VP, U8P]),
        "kbfv_ntt_fwd_batch": (I, [VP, C.POINTER(VP), u32, u32, u32, VP]),
        "kbfv_ntt_inv_batch": (I, [VP, C.POINTER(VP), u32, u32, u32, VP]),
        "kbfv_add_plain": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_context_at_level": (I, [VP, u32, C.POINTER(VP)]),
        "kbfv_probe_arith": (I, [I, u32, C.POINTER(C.c_double)]),
        "kbfv_galois_element": (u64, [VP, C.c_int64]),
        "kbfv_sub": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_sample_compat": (I, [VP, I, VP, VP, u32, u32, u32, C.c_double, VP]),
        "kbfv_encrypt_batch": (I, [VP, U8P, U64P, VP, C.POINTER(VP), C.POINTER(VP), u32, VP]),
        "kbfv_decrypt_batch": (I, [VP, VP, C.POINTER(VP), C.POINTER(VP), u32, VP]),
        "kbfv_add_batch": (I, [VP, C.POINTER(VP), C.POINTER(VP), C.POINTER(VP), u32, VP]),
        "kbfv_wire_bytes": (C.c_size_t, [VP, I, u64, u32]),
        "kbfv_wire_save": (I, [VP, I, u64, VP, u32, VP, C.c_size_t, VP]),
        "kbfv_wire_load": (I, [VP, I, VP, C.c_size_t, VP, u32, C.POINTER(u32), C.POINTER(u64), VP]),
        "kbfv_negate": (I, [VP, VP, VP, u32, VP]),
        "kbfv_mul_scalar": (I, [VP, VP, u64, VP, u32, VP]),
        "kbfv_mul_scalar_add": (I, [VP, VP, u64, VP, u32, VP]),
        "kbfv_keygen_galois": (I, [VP, U8P, VP, u64, VP, VP]),
        "kbfv_apply_galois": (I, [VP, VP, u64, VP, VP, u32, VP]),
        "kbfv_keygen_relin_gadget": (I, [VP, U8P, VP, u32, VP, VP]),
        "kbfv_relinearize_gadget": (I, [VP, VP, u32, VP, VP, u32, VP]),
        "kbfv_mul_relin_gadget": (I, [VP, VP, u32, VP, VP, VP, u32, VP]),
        "kbfv_mod_switch": (I, [VP, VP, VP, u32, VP]),
        "kbfv_mul_relin_levels": (I, [VP, VP, C.POINTER(u32), C.POINTER(VP), C.POINTER(VP), C.POINTER(VP), u32, VP]),
        "kbfv_rlk_to_klss": (I, [VP, VP, VP, VP]),
        "kbfv_klss_modup_qj_to_t": (I, [VP, VP, VP, u32, VP]),
        "kbfv_klss_modup_pq_to_t": (I, [VP, VP, VP, u32, VP]),
        "kbfv_klss_external_product": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_klss_t_to_pq": (I, [VP, VP, VP, u32, VP]),
        "kbfv_relinearize_klss": (I, [VP, VP, VP, VP, u32, VP]),
        "kbfv_mul_relin_klss": (I, [VP, VP, VP, VP, VP, u32, VP]),
        "kbfv_noise_budget": (I, [VP, VP, VP, C.POINTER(C.c_double)]),
        "kbfv_salsa20_stream": (I, [U8P, U8P, u64, VP, C.c_size_t, I, VP]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args


def _check(rc: int) -> None:
    if rc != KBFV_OK:
        msg = lib().kbfv_last_error().decode(errors="replace")
        if rc == -1:
            raise KbfvInvalidArgument(rc, msg)
        raise KbfvError(rc, msg)


def _u8(b: bytes):
    a = (C.c_uint8 * len(b)).from_buffer_copy(bytes(b))
    return a


def _torch():
    import torch  # deferred: importing the bindings does not need a GPU

    return torch


def _stream_ptr(stream) -> int:
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


def _ptr(t) -> int:
    return t.data_ptr()


def to_device(a: np.ndarray, device="cuda"):
    """numpy uint64 -> torch int64 device tensor (same bits)."""
    torch = _torch()
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return torch.from_numpy(a.view(np.int64)).to(device)


def to_host(t) -> np.ndarray:
    return t.detach().cpu().numpy().view(np.uint64)


@dataclass
class Params:
    log_n: int
    plain_modulus: int
    q_count: int
    q_bits: int = 60
    p_count: int = 1
    p_bits: int = 60
    dnum: int = 1
    q: Optional[Sequence[int]] = None
    p: Optional[Sequence[int]] = None
    t_primes: Sequence[int] = ()
    gamma: int = 1
    digit_primes: int = 0


class BFVContext:
    """A parameter set (BFVContext, include/BFVcontext.h:17-391).

    Public fields mirror the reference: ``N``, ``L`` (= q_count - 1),
    ``K`` (= p_count), ``slots`` (= N), ``plain_modulus``.
    """

    def __init__(self, params: Optional[Params] = None, *, _handle=None, _owner=None, **kw):
        L = lib()
        self._owner = _owner  # level contexts belong to their top-level context
        if _handle is not None:
            self._h = _handle
        else:
            if params is None:
                params = Params(**kw)
            self.params = params
            keep = []

            def arr(v):
                if not v:
                    return None
                a = (C.c_uint64 * len(v))(*[int(x) for x in v])
                keep.append(a)
                return C.cast(a, U64P)

            pr = _Params(params.log_n, params.plain_modulus, params.q_count, arr(params.q), params.q_bits,
                         params.p_count, arr(params.p), params.p_bits, params.dnum, len(params.t_primes),
                         arr(list(params.t_primes)), params.gamma, params.digit_primes)
            h = VP()
            _check(L.kbfv_context_create(C.byref(pr), C.byref(h)))
            self._h = h
        n = C.c_uint64()
        nq, np_, nr, nt, dnum, alpha = (C.c_uint32() for _ in range(6))
        _check(L.kbfv_context_info(self._h, C.byref(n), C.byref(nq), C.byref(np_), C.byref(nr), C.byref(nt),
                                   C.byref(dnum), C.byref(alpha)))
        self.N = int(n.value)
        self.log_n = self.N.bit_length() - 1
        self.q_count, self.p_count, self.r_count, self.t_count = nq.value, np_.value, nr.value, nt.value
        self.dnum, self.alpha = dnum.value, alpha.value
        self.L = self.q_count - 1
        self.K = self.p_count
        self.slots = self.N
        self.plain_modulus = int(L.kbfv_context_plain_modulus(self._h))
        cnt = C.c_uint32()
        _check(L.kbfv_context_primes(self._h, None, C.byref(cnt)))
        buf = (C.c_uint64 * cnt.value)()
        _check(L.kbfv_context_primes(self._h, buf, C.byref(cnt)))
        self.primes = [int(x) for x in buf]
        self.q = self.primes[: self.q_count]
        self.p = self.primes[self.q_count: self.q_count + self.p_count]
        self.r = self.primes[self.q_count + self.p_count: self.q_count + self.p_count + self.r_count]
        self.tk = self.primes[self.q_count + self.p_count + self.r_count: -1]
        self.decrypt_variant = int(L.kbfv_context_decrypt_variant(self._h))

    # prime-table offsets
    @property
    def idx_p(self):
        return self.q_count

    @property
    def idx_r(self):
        return self.q_count + self.p_count

    @property
    def idx_t(self):
        return self.q_count + self.p_count + self.r_count

    @property
    def idx_plain(self):
        return len(self.primes) - 1

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and _lib is not None and getattr(self, "_owner", None) is None:
            _lib.kbfv_context_destroy(h)
        self._h = None

    def at_level(self, live_q: int) -> "BFVContext":
        """the context for ciphertexts with the first live_q primes of Q (owned by this one)"""
        if live_q == self.q_count and self._owner is None:
            return self
        cache = self.__dict__.setdefault("_levels", {})
        if live_q not in cache:
            h = VP()
            _check(lib().kbfv_context_at_level(self._h, live_q, C.byref(h)))
            cache[live_q] = BFVContext(_handle=h, _owner=self)
        return cache[live_q]

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_branches(self, branches: int):
        """sub-batches (and streams) a batched multiply of two or more pairs uses, 1..4"""
        _check(lib().kbfv_set_branches(self._h, branches))

    def tune_set(self, knob: str, value: int):
        """set a speed-only knob: ntt_block_log (12..14), branches (1..4), host_chunk (0..128)"""
        _check(lib().kbfv_tune_set(self._h, TUNE_KNOBS[knob], int(value)))

    def tune_get(self, knob: str) -> int:
        v = C.c_int64()
        _check(lib().kbfv_tune_get(self._h, TUNE_KNOBS[knob], C.byref(v)))
        return int(v.value)

    def reserve(self, pairs: int):
        _check(lib().kbfv_reserve(self._h, pairs))

    def scratch_bytes(self, pairs: int) -> int:
        return int(lib().kbfv_mul_relin_scratch_bytes(self._h, pairs))

    def arena_bytes(self) -> int:
        """Bytes of device memory the context's scratch arena holds now."""
        return int(lib().kbfv_context_arena_bytes(self._h))

    # ---- device buffers
    def zeros(self, *shape):
        torch = _torch()
        return torch.zeros(shape, dtype=torch.int64, device="cuda")

    @classmethod
    def from_bits(cls, log_n: int, q_bits, p_bits, plain_modulus: int, dnum: int = 1) -> "BFVContext":
        """Parameter set from per-prime bit sizes (kbfv_params_create), e.g.
        from_bits(12, [36, 36], [37], 65537, dnum=2)."""
        qb = (C.c_uint32 * len(q_bits))(*q_bits)
        pb = (C.c_uint32 * len(p_bits))(*p_bits)
        out = C.POINTER(_Params)()
        _check(lib().kbfv_params_create(log_n, qb, len(q_bits), pb, len(p_bits), plain_modulus, dnum, C.byref(out)))
        try:
            h = VP()
            _check(lib().kbfv_context_create(out, C.byref(h)))
        finally:
            lib().kbfv_params_destroy(out)
        return cls(_handle=h)

    def sample_compat(self, kind: int, rand, prime0: int, limbs: int, h: int = 64, probability: float = 0.5,
                      stream=None):
        """the reference's sampler conversions on random words (kbfv_sample_compat)"""
        out = self.zeros(limbs, self.N)
        _check(lib().kbfv_sample_compat(self._h, kind, _ptr(rand), _ptr(out), prime0, limbs, h, probability,
                                        _stream_ptr(stream)))
        return out

    def set_seed(self, seed: bytes):
        _check(lib().kbfv_set_seed(self._h, _u8(seed)))

    def ntt_fwd_batch(self, polys, limbs: int, prime0: int = 0, stream=None):
        """forward NTT of polynomials at arbitrary addresses (a list of device tensors)"""
        arr = (VP * len(polys))(*[_ptr(p) for p in polys])
        _check(lib().kbfv_ntt_fwd_batch(self._h, arr, len(polys), limbs, prime0, _stream_ptr(stream)))

    def ntt_inv_batch(self, polys, limbs: int, prime0: int = 0, stream=None):
        arr = (VP * len(polys))(*[_ptr(p) for p in polys])
        _check(lib().kbfv_ntt_inv_batch(self._h, arr, len(polys), limbs, prime0, _stream_ptr(stream)))

    # ---- NTT (ToNTTInplace / FromNTTInplace)
    def ntt_fwd(self, rows, prime0: int, period: int, stream=None):
        nrows = rows.numel() // self.N
        _check(lib().kbfv_ntt_fwd(self._h, _ptr(rows), nrows, prime0, period, _stream_ptr(stream)))

    def ntt_inv(self, rows, prime0: int, period: int, stream=None):
        nrows = rows.numel() // self.N
        _check(lib().kbfv_ntt_inv(self._h, _ptr(rows), nrows, prime0, period, _stream_ptr(stream)))

    # ---- encoder (include/Encoder.cuh)
    def encode(self, slots, out=None, stream=None):
        count = slots.numel() // self.N
        out = out if out is not None else self.zeros(count, self.N)
        _check(lib().kbfv_encode(self._h, _ptr(slots), _ptr(out), count, _stream_ptr(stream)))
        return out

    def decode(self, m, out=None, stream=None):
        count = m.numel() // self.N
        out = out if out is not None else self.zeros(count, self.N)
        _check(lib().kbfv_decode(self._h, _ptr(m), _ptr(out), count, _stream_ptr(stream)))
        return out

    def encode_ntt(self, vals, out=None, stream=None):
        count = vals.numel() // self.N
        out = out if out is not None else self.zeros(count, self.q_count, self.N)
        _check(lib().kbfv_encode_ntt(self._h, _ptr(vals), _ptr(out), count, _stream_ptr(stream)))
        return out

    # ---- building blocks
    def _op(self, name, ins, out, polys, stream=None):
        args = [self._h] + [_ptr(x) for x in ins] + [_ptr(out), polys, _stream_ptr(stream)]
        _check(getattr(lib(), name)(*args))
        return out

    def bconv_q_to_r(self, x, stream=None):
        polys = x.numel() // (self.q_count * self.N)
        return self._op("kbfv_bconv_q_to_r", [x], self.zeros(polys, self.r_count, self.N), polys, stream)

    def bconv_r_to_q(self, x, stream=None):
        polys = x.numel() // (self.r_count * self.N)
        return self._op("kbfv_bconv_r_to_q", [x], self.zeros(polys, self.q_count, self.N), polys, stream)

    def tensor_qr(self, c1, c2, stream=None):
        nqr = self.q_count + self.r_count
        pairs = c1.numel() // (2 * nqr * self.N)
        return self._op("kbfv_tensor_qr", [c1, c2], self.zeros(pairs, 3, nqr, self.N), pairs, stream)

    def scale_round_qr_r(self, x, stream=None):
        polys = x.numel() // ((self.q_count + self.r_count) * self.N)
        return self._op("kbfv_scale_round_qr_r", [x], self.zeros(polys, self.r_count, self.N), polys, stream)

    def decrypt_round(self, x, stream=None):
        polys = x.numel() // (self.q_count * self.N)
        return self._op("kbfv_decrypt_round", [x], self.zeros(polys, self.N), polys, stream)

    def delta_m(self, m, stream=None):
        polys = m.numel() // self.N
        return self._op("kbfv_delta_m", [m], self.zeros(polys, self.q_count, self.N), polys, stream)

    def modup(self, x, stream=None):
        polys = x.numel() // (self.q_count * self.N)
        npq = self.q_count + self.p_count
        return self._op("kbfv_modup", [x], self.zeros(polys, self.dnum, npq, self.N), polys, stream)

    def moddown(self, x, stream=None):
        npq = self.q_count + self.p_count
        polys = x.numel() // (npq * self.N)
        return self._op("kbfv_moddown", [x], self.zeros(polys, self.q_count, self.N), polys, stream)

    # ---- key switch over the T base (the reference's KLSS)
    def klss_info(self):
        """(Ri blocks, Qj blocks, T-form key words); raises if the context has no T base."""
        nri, nqj, kw = C.c_uint32(), C.c_uint32(), C.c_uint64()
        _check(lib().kbfv_context_klss(self._h, C.byref(nri), C.byref(nqj), C.byref(kw)))
        return nri.value, nqj.value, kw.value

    def klss_modup_qj_to_t(self, x, stream=None):
        _, nqj, _ = self.klss_info()
        polys = x.numel() // (self.q_count * self.N)
        return self._op("kbfv_klss_modup_qj_to_t", [x], self.zeros(polys, nqj, self.t_count, self.N), polys, stream)

    def klss_modup_pq_to_t(self, x, stream=None):
        nri, _, _ = self.klss_info()
        polys = x.numel() // ((self.q_count + self.p_count) * self.N)
        return self._op("kbfv_klss_modup_pq_to_t", [x], self.zeros(polys, nri, self.t_count, self.N), polys, stream)

    def klss_external_product(self, digits, key_t, stream=None):
        nri, nqj, _ = self.klss_info()
        count = digits.numel() // (nqj * self.t_count * self.N)
        out = self.zeros(count, 2, nri, self.t_count, self.N)
        _check(lib().kbfv_klss_external_product(self._h, _ptr(digits), _ptr(key_t), _ptr(out), count,
                                                _stream_ptr(stream)))
        return out

    def klss_t_to_pq(self, x, stream=None):
        nri, _, _ = self.klss_info()
        polys = x.numel() // (nri * self.t_count * self.N)
        npq = self.q_count + self.p_count
        return self._op("kbfv_klss_t_to_pq", [x], self.zeros(polys, npq, self.N), polys, stream)


def reference_context(log_n: int) -> BFVContext:
    """The reference's own parameter set for logN 14 or 15 (include/Params.cuh:31-145)."""
    h = VP()
    _check(lib().kbfv_context_create_reference(log_n, C.byref(h)))
    return BFVContext(_handle=h)


class SecretKey:
    """SecretKey (include/SecretKey.cuh:10-62): NTT form over Q|P."""

    def __init__(self, ctx: BFVContext, seed: bytes = b"\x00" * 32, kind: int = 0, h: int = 64, stream=None):
        self.ctx = ctx
        self.sx_device = ctx.zeros(ctx.q_count + ctx.p_count, ctx.N)
        _check(lib().kbfv_keygen_secret(ctx.handle, _u8(seed), kind, h, _ptr(self.sx_device), _stream_ptr(stream)))


class Plaintext:
    """Plaintext coefficients mod t (N words per plaintext)."""

    def __init__(self, ctx: BFVContext, data=None, count: int = 1):
        self.ctx = ctx
        self.mx_device = data if data is not None else ctx.zeros(count, ctx.N)

    @property
    def count(self):
        return self.mx_device.numel() // self.ctx.N


class Ciphertext:
    """Ciphertext [a | b] over Q in NTT form (include/Ciphertext.cuh:5-89); may hold a batch."""

    def __init__(self, ctx: BFVContext, data=None, count: int = 1):
        self.ctx = ctx
        self.cipher_device = data if data is not None else ctx.zeros(count, 2, ctx.q_count, ctx.N)
        self.l = ctx.L

    @property
    def count(self):
        return self.cipher_device.numel() // (2 * self.ctx.q_count * self.ctx.N)

    @property
    def ax_device(self):
        return self.cipher_device.view(self.count, 2, self.ctx.q_count, self.ctx.N)[:, 0]

    @property
    def bx_device(self):
        return self.cipher_device.view(self.count, 2, self.ctx.q_count, self.ctx.N)[:, 1]


class Tensor3:
    """Unrelinearised product [a1a2 | cross | b1b2] over Q in NTT form."""

    def __init__(self, ctx: BFVContext, data=None, count: int = 1):
        self.ctx = ctx
        self.data = data if data is not None else ctx.zeros(count, 3, ctx.q_count, ctx.N)


class MulPlan:
    """kbfv_plan_*: a hybrid mult+relin bound to fixed device buffers, replayed
    as one CUDA graph after its first launch. Keeps its buffers and key alive.
    With `pairs` (a list of (ct_a, ct_b) at possibly different levels) and
    `outs`, the plan is the mixed-level multiply (kbfv_plan_mul_relin_levels)."""

    def __init__(self, scheme: "BFVScheme", c1: Ciphertext = None, c2: Ciphertext = None, out=None, pairs=None):
        self._keep = (scheme, c1, c2, out, pairs)
        self._ctx = scheme.context
        h = VP()
        if pairs is None:
            _check(lib().kbfv_plan_mul_relin(c1.ctx.handle, _ptr(scheme.rlk), _ptr(c1.cipher_device),
                                             _ptr(c2.cipher_device), _ptr(out.cipher_device), c1.count, C.byref(h)))
        else:
            n = len(pairs)
            lv = (C.c_uint32 * n)(*[a.ctx.q_count for a, _ in pairs])
            A = (VP * n)(*[_ptr(a.cipher_device) for a, _ in pairs])
            B = (VP * n)(*[_ptr(b.cipher_device) for _, b in pairs])
            O = (VP * n)(*[_ptr(o.cipher_device) for o in out])
            _check(lib().kbfv_plan_mul_relin_levels(scheme.context.handle, _ptr(scheme.rlk), lv, A, B, O, n,
                                                    C.byref(h)))
        self._h = h
        self.out = out

    def launch(self, stream=None) -> Ciphertext:
        _check(lib().kbfv_plan_launch(self._h, _stream_ptr(stream)))
        return self.out

    def info(self):
        """(launches, captures) so far."""
        n, k = C.c_uint64(), C.c_uint64()
        _check(lib().kbfv_plan_info(self._h, C.byref(n), C.byref(k)))
        return n.value, k.value

    def close(self):
        if getattr(self, "_h", None):
            lib().kbfv_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BFVScheme:
    """BFVScheme (include/BFVScheme.h:12-178) over one context."""

    def __init__(self, ctx: BFVContext, seed: bytes = b"\x00" * 32, relin: str = "hybrid", gadget_log_base: int = 20):
        """relin: "hybrid" (digit lift over Q|P, the default), "klss" (the
        reference's key switch over the T base; needs a context with T primes)
        or "gadget" (base-2^gadget_log_base decomposition of every residue)."""
        if relin not in ("hybrid", "klss", "gadget"):
            raise ValueError("relin must be 'hybrid', 'klss' or 'gadget'")
        self.gadget_log_base = gadget_log_base
        self.gk = None
        self.galois_keys = {}  # Galois element -> key (rotKey_vec_23 / ConjKey_23)
        self.context = ctx
        self.seed = bytes(seed)
        self.relin = relin
        self.publicKey = None
        self.rlk = None
        self.rlk_t = None
        self._enc_counter = 0
        if relin == "klss":
            ctx.klss_info()

    def mallocMemory(self, pairs: int = 1):
        self.context.reserve(pairs)

    def addEncKey(self, sk: SecretKey, stream=None):
        ctx = self.context
        self.publicKey = ctx.zeros(2, ctx.q_count, ctx.N)
        _check(lib().kbfv_keygen_public(ctx.handle, _u8(self.seed), _ptr(sk.sx_device), _ptr(self.publicKey),
                                        _stream_ptr(stream)))

    def addMultKey_23(self, sk: SecretKey, stream=None):
        ctx = self.context
        self.rlk = ctx.zeros(ctx.dnum, 2, ctx.q_count + ctx.p_count, ctx.N)
        _check(lib().kbfv_keygen_relin(ctx.handle, _u8(self.seed), _ptr(sk.sx_device), _ptr(self.rlk),
                                       _stream_ptr(stream)))
        if self.relin == "klss":
            self.convert_rlk_klss(stream)
        if self.relin == "gadget":
            self.addGadgetKey(sk, self.gadget_log_base, stream)

    def addGadgetKey(self, sk: SecretKey, log_base: int = 20, stream=None):
        ctx = self.context
        pieces = -(-60 // log_base)
        self.gadget_log_base = log_base
        self.gk = ctx.zeros(ctx.q_count * pieces, 2, ctx.q_count + ctx.p_count, ctx.N)
        _check(lib().kbfv_keygen_relin_gadget(ctx.handle, _u8(self.seed), _ptr(sk.sx_device), log_base,
                                              _ptr(self.gk), _stream_ptr(stream)))

    def convert_rlk_klss(self, stream=None):
        """The T-form copy of self.rlk (addMultKey_23's conversion, KeySwitch_23.cuh:55-65)."""
        ctx = self.context
        nri, nqj, _ = ctx.klss_info()
        self.rlk_t = ctx.zeros(2, nqj, nri, ctx.t_count, ctx.N)
        _check(lib().kbfv_rlk_to_klss(ctx.handle, _ptr(self.rlk), _ptr(self.rlk_t), _stream_ptr(stream)))

    def encryptMsg(self, pt: Plaintext, enc_id: Optional[int] = None, stream=None) -> Ciphertext:
        if self.publicKey is None:
            raise KbfvError(-5, "public key not generated (call addEncKey)")
        ctx = self.context
        cnt = pt.count
        if enc_id is None:
            enc_id = self._enc_counter
            self._enc_counter += cnt
        ct = Ciphertext(ctx, count=cnt)
        _check(lib().kbfv_encrypt(ctx.handle, _u8(self.seed), enc_id, _ptr(self.publicKey), _ptr(pt.mx_device),
                                  _ptr(ct.cipher_device), cnt, _stream_ptr(stream)))
        return ct

    def decryptMsg(self, sk: SecretKey, ct: Ciphertext, stream=None) -> Plaintext:
        ctx = ct.ctx  # the ciphertext's level
        pt = Plaintext(ctx, count=ct.count)
        _check(lib().kbfv_decrypt(ctx.handle, _ptr(sk.sx_device), _ptr(ct.cipher_device), _ptr(pt.mx_device),
                                  ct.count, _stream_ptr(stream)))
        return pt

    def add(self, c1: Ciphertext, c2: Ciphertext, stream=None) -> Ciphertext:
        out = Ciphertext(c1.ctx, count=c1.count)
        _check(lib().kbfv_add(c1.ctx.handle, _ptr(c1.cipher_device), _ptr(c2.cipher_device),
                              _ptr(out.cipher_device), c1.count, _stream_ptr(stream)))
        return out

    def addAndEqual(self, c1: Ciphertext, c2: Ciphertext, stream=None):
        _check(lib().kbfv_add(self.context.handle, _ptr(c1.cipher_device), _ptr(c2.cipher_device),
                              _ptr(c1.cipher_device), c1.count, _stream_ptr(stream)))

    def sub(self, c1: Ciphertext, c2: Ciphertext, stream=None) -> Ciphertext:
        out = Ciphertext(c1.ctx, count=c1.count)
        _check(lib().kbfv_sub(c1.ctx.handle, _ptr(c1.cipher_device), _ptr(c2.cipher_device), _ptr(out.cipher_device),
                              c1.count, _stream_ptr(stream)))
        return out

    def subAndEqual(self, c1: Ciphertext, c2: Ciphertext, stream=None):
        _check(lib().kbfv_sub(c1.ctx.handle, _ptr(c1.cipher_device), _ptr(c2.cipher_device), _ptr(c1.cipher_device),
                              c1.count, _stream_ptr(stream)))

    def negateAndEqual(self, ct: Ciphertext, stream=None):
        _check(lib().kbfv_negate(ct.ctx.handle, _ptr(ct.cipher_device), _ptr(ct.cipher_device), ct.count,
                                 _stream_ptr(stream)))

    def multScalarAndEqual(self, ct: Ciphertext, cnst: int, stream=None):
        """multConstAndEqual(Ciphertext&, uint64_tt) (BFVScheme.cuh:247-268)"""
        _check(lib().kbfv_mul_scalar(ct.ctx.handle, _ptr(ct.cipher_device), cnst, _ptr(ct.cipher_device), ct.count,
                                     _stream_ptr(stream)))

    def multConstAndAddCipherEqual(self, c1: Ciphertext, c2: Ciphertext, cnst: int, stream=None):
        """c1 += c2 * cnst (BFVScheme.cuh:272-288)"""
        _check(lib().kbfv_mul_scalar_add(c1.ctx.handle, _ptr(c2.cipher_device), cnst, _ptr(c1.cipher_device),
                                         c1.count, _stream_ptr(stream)))

    def squareAndEqual(self, ct: Ciphertext, stream=None):
        """squareAndEqual (KeySwitch_23.cuh:422-466): ct * ct, relinearised"""
        self.mult_relin(ct, ct, out=ct, stream=stream)

    def addConstAndEqual(self, ct: Ciphertext, pt: Plaintext, stream=None):
        """ct.b += NTT(Delta * m) (BFVScheme.cuh:192-217)"""
        _check(lib().kbfv_add_plain(self.context.handle, _ptr(ct.cipher_device), _ptr(pt.mx_device),
                                    _ptr(ct.cipher_device), ct.count, _stream_ptr(stream)))

    def multConstAndEqual(self, ct: Ciphertext, pt_ntt, stream=None):
        _check(lib().kbfv_mul_plain(self.context.handle, _ptr(ct.cipher_device), _ptr(pt_ntt),
                                    _ptr(ct.cipher_device), ct.count, _stream_ptr(stream)))

    def mult(self, c1: Ciphertext, c2: Ciphertext, stream=None) -> Tensor3:
        out = Tensor3(c1.ctx, count=c1.count)
        _check(lib().kbfv_mul(c1.ctx.handle, _ptr(c1.cipher_device), _ptr(c2.cipher_device), _ptr(out.data),
                              c1.count, _stream_ptr(stream)))
        return out

    def relinearize(self, t3: Tensor3, stream=None) -> Ciphertext:
        if self.rlk is None:
            raise KbfvError(-5, "rotKey_23 not exists")
        cnt = t3.data.numel() // (3 * t3.ctx.q_count * t3.ctx.N)
        out = Ciphertext(t3.ctx, count=cnt)
        if self.relin == "gadget":
            _check(lib().kbfv_relinearize_gadget(t3.ctx.handle, _ptr(self.gk), self.gadget_log_base, _ptr(t3.data),
                                                 _ptr(out.cipher_device), cnt, _stream_ptr(stream)))
        elif self.relin == "klss":
            _check(lib().kbfv_relinearize_klss(self.context.handle, _ptr(self.rlk_t), _ptr(t3.data),
                                               _ptr(out.cipher_device), cnt, _stream_ptr(stream)))
        else:
            _check(lib().kbfv_relinearize(t3.ctx.handle, _ptr(self.rlk), _ptr(t3.data),
                                          _ptr(out.cipher_device), cnt, _stream_ptr(stream)))
        return out

    def mult_relin(self, c1: Ciphertext, c2: Ciphertext, out: Optional[Ciphertext] = None, stream=None) -> Ciphertext:
        """Batched ct1[i] * ct2[i] with relinearisation (multAndEqual_23 without the shortcut)."""
        if self.rlk is None:
            raise KbfvError(-5, "rotKey_23 not exists")
        out = out if out is not None else Ciphertext(c1.ctx, count=c1.count)
        if self.relin == "gadget":
            _check(lib().kbfv_mul_relin_gadget(c1.ctx.handle, _ptr(self.gk), self.gadget_log_base,
                                               _ptr(c1.cipher_device), _ptr(c2.cipher_device), _ptr(out.cipher_device),
                                               c1.count, _stream_ptr(stream)))
        elif self.relin == "klss":
            _check(lib().kbfv_mul_relin_klss(self.context.handle, _ptr(self.rlk_t), _ptr(c1.cipher_device),
                                             _ptr(c2.cipher_device), _ptr(out.cipher_device), c1.count,
                                             _stream_ptr(stream)))
        else:  # at the ciphertexts' level, with the top-level key
            _check(lib().kbfv_mul_relin(c1.ctx.handle, _ptr(self.rlk), _ptr(c1.cipher_device),
                                        _ptr(c2.cipher_device), _ptr(out.cipher_device), c1.count,
                                        _stream_ptr(stream)))
        return out

    def mult_relin_host(self, h_a, h_b, out=None, chunk_pairs: int = 0, stream=None, synchronize: bool = True):
        """Hybrid mult+relin of ciphertext pairs held in host memory (torch CPU
        int64 tensors, page-locked for overlapped copies, or numpy uint64 arrays)
        of the context's top level: [count, 2, q_count, N] each. Copies in,
        multiplies and copies out chunk by chunk on the context's streams; the
        products land in `out` (allocated page-locked when not given). With
        synchronize=False the call only queues the work on `stream`."""
        torch = _torch()
        if self.rlk is None:
            raise KbfvError(-5, "rotKey_23 not exists")
        if self.relin != "hybrid":
            raise KbfvInvalidArgument(-1, "host-memory multiply runs the hybrid key switch only")
        ctx = self.context

        def as_host(x):
            if isinstance(x, np.ndarray):
                return torch.from_numpy(np.ascontiguousarray(x, dtype=np.uint64).view(np.int64))
            if x.device.type != "cpu" or x.dtype != torch.int64 or not x.is_contiguous():
                raise KbfvInvalidArgument(-1, "host ciphertexts must be contiguous CPU int64 tensors")
            return x

        a, b = as_host(h_a), as_host(h_b)
        words = 2 * ctx.q_count * ctx.N
        if a.numel() != b.numel() or a.numel() % words:
            raise KbfvInvalidArgument(-1, "host ciphertexts must hold whole ciphertexts, as many in each")
        count = a.numel() // words
        if out is None:
            out = torch.empty(count, 2, ctx.q_count, ctx.N, dtype=torch.int64, pin_memory=True)
        elif isinstance(out, np.ndarray):
            raise KbfvInvalidArgument(-1, "out must be a CPU int64 tensor")
        if out.numel() != a.numel() or out.device.type != "cpu" or out.dtype != torch.int64:
            raise KbfvInvalidArgument(-1, "out must be a CPU int64 tensor as large as the inputs")
        sp = _stream_ptr(stream)
        _check(lib().kbfv_mul_relin_host(ctx.handle, _ptr(self.rlk), a.data_ptr(), b.data_ptr(), out.data_ptr(),
                                         count, chunk_pairs, sp))
        if synchronize:
            if stream is None:
                torch.cuda.current_stream().synchronize()
            elif hasattr(stream, "synchronize"):
                stream.synchronize()
            else:
                torch.cuda.synchronize()
        return out

    def mult_relin_plan(self, c1: Ciphertext, c2: Ciphertext, out: Ciphertext) -> "MulPlan":
        """A captured multiply bound to these three buffers (kbfv_plan_mul_relin):
        each ``launch()`` multiplies whatever c1 and c2 hold at that time into
        ``out``; launches after the first replay one CUDA graph."""
        if self.rlk is None:
            raise KbfvError(-5, "rotKey_23 not exists")
        if self.relin != "hybrid":
            raise KbfvInvalidArgument(-1, "captured multiplies run the hybrid key switch only")
        if not (c1.count == c2.count == out.count):
            raise KbfvInvalidArgument(-1, "c1, c2 and out must hold as many ciphertexts")
        return MulPlan(self, c1, c2, out)

    def mult_relin_levels_plan(self, pairs, outs) -> "MulPlan":
        """A captured mixed-level multiply (kbfv_plan_mul_relin_levels): each
        ``launch()`` multiplies the pairs' current contents into ``outs`` (each
        at its pair's level) with one CUDA graph launch after the first."""
        if self.rlk is None:
            raise KbfvError(-5, "rotKey_23 not exists")
        if len(outs) != len(pairs):
            raise KbfvInvalidArgument(-1, "one output per pair")
        return MulPlan(self, out=outs, pairs=pairs)

    def mult_relin_ptrs(self, a_ptrs, b_ptrs, out_ptrs, stream=None):
        n = len(a_ptrs)
        A = (VP * n)(*a_ptrs)
        B = (VP * n)(*b_ptrs)
        O = (VP * n)(*out_ptrs)
        _check(lib().kbfv_mul_relin_batch(self.context.handle, _ptr(self.rlk), A, B, O, n, _stream_ptr(stream)))

    # ---- rotations and conjugation (Galois automorphisms)
    def galois_element(self, rot_slots: int) -> int:
        return int(lib().kbfv_galois_element(self.context.handle, rot_slots))

    def addGaloisKey(self, sk: SecretKey, g: int, stream=None):
        if g in self.galois_keys:
            return
        ctx = self.context
        key = ctx.zeros(ctx.dnum, 2, ctx.q_count + ctx.p_count, ctx.N)
        _check(lib().kbfv_keygen_galois(ctx.handle, _u8(self.seed), _ptr(sk.sx_device), g, _ptr(key),
                                        _stream_ptr(stream)))
        self.galois_keys[g] = key

    def addLeftRotKey_23(self, sk: SecretKey, rot_num: int, stream=None):
        self.addGaloisKey(sk, self.galois_element(rot_num), stream)

    def addConjKey_23(self, sk: SecretKey, stream=None):
        self.addGaloisKey(sk, 2 * self.context.N - 1, stream)

    def apply_galois(self, ct: Ciphertext, g: int, out: Optional[Ciphertext] = None, stream=None) -> Ciphertext:
        if g not in self.galois_keys:
            raise KbfvError(-5, "rotKey_23 not exists")
        out = out if out is not None else Ciphertext(ct.ctx, count=ct.count)
        _check(lib().kbfv_apply_galois(ct.ctx.handle, _ptr(self.galois_keys[g]), g, _ptr(ct.cipher_device),
                                       _ptr(out.cipher_device), ct.count, _stream_ptr(stream)))
        return out

    def leftRotateAndEqual_23(self, ct: Ciphertext, rot_slots: int, stream=None):
        self.apply_galois(ct, self.galois_element(rot_slots), out=ct, stream=stream)

    def rightRotateAndEqual_23(self, ct: Ciphertext, rot_slots: int, stream=None):
        """the reference's conversion: a left rotation by N/2 - 2^rot_slots (KeySwitch_23.cuh:580-584)"""
        self.leftRotateAndEqual_23(ct, self.context.N // 2 - (1 << rot_slots), stream)

    def conjugate_23(self, ct: Ciphertext, stream=None):
        self.apply_galois(ct, 2 * self.context.N - 1, out=ct, stream=stream)

    def mod_switch(self, ct: Ciphertext, stream=None) -> Ciphertext:
        """drop the last live prime (divide and round); the result lives at ct.ctx's level - 1"""
        top = ct.ctx._owner or ct.ctx
        lower = top.at_level(ct.ctx.q_count - 1)
        out = Ciphertext(lower, count=ct.count)
        _check(lib().kbfv_mod_switch(ct.ctx.handle, _ptr(ct.cipher_device), _ptr(out.cipher_device), ct.count,
                                     _stream_ptr(stream)))
        return out

    def mod_switch_to(self, ct: Ciphertext, live_q: int, stream=None) -> Ciphertext:
        while ct.ctx.q_count > live_q:
            ct = self.mod_switch(ct, stream)
        return ct

    def mult_relin_levels(self, pairs, outs=None, stream=None):
        """[(ct_a, ct_b)] at possibly different levels -> products, one call (one
        launch sequence for up to 128 pairs in up to 8 levels); `outs` may give
        the output ciphertexts (each at its pair's level)"""
        n = len(pairs)
        if outs is None:
            outs = [Ciphertext(a.ctx, count=1) for a, _ in pairs]
        lv = (C.c_uint32 * n)(*[a.ctx.q_count for a, _ in pairs])
        A = (VP * n)(*[_ptr(a.cipher_device) for a, _ in pairs])
        B = (VP * n)(*[_ptr(b.cipher_device) for _, b in pairs])
        O = (VP * n)(*[_ptr(o.cipher_device) for o in outs])
        _check(lib().kbfv_mul_relin_levels(self.context.handle, _ptr(self.rlk), lv, A, B, O, n, _stream_ptr(stream)))
        return outs

    def multAndEqual_23(self, c1: Ciphertext, c2: Ciphertext, stream=None):
        self.mult_relin(c1, c2, out=c1, stream=stream)

    def noise_budget(self, sk: SecretKey, ct: Ciphertext) -> float:
        v = C.c_double()
        _check(lib().kbfv_noise_budget(ct.ctx.handle, _ptr(sk.sx_device), _ptr(ct.cipher_device), C.byref(v)))
        return float(v.value)


WIRE_KINDS = {"ciphertext": 1, "plaintext": 2, "secret_key": 3, "public_key": 4, "relin_key": 5, "galois_key": 6,
              "gadget_key": 7, "klss_key": 8}


def wire_save(ctx: BFVContext, kind: str, tensor, count: int = 1, aux: int = 0) -> bytes:
    """serialize device objects (kbfv_wire_save) -> bytes"""
    k = WIRE_KINDS[kind]
    nbytes = lib().kbfv_wire_bytes(ctx.handle, k, aux, count)
    if not nbytes:
        raise KbfvError(-1, f"{kind} is not available for this context")
    buf = (C.c_uint8 * nbytes)()
    _check(lib().kbfv_wire_save(ctx.handle, k, aux, _ptr(tensor), count, buf, nbytes, None))
    return bytes(buf)


def wire_load(ctx: BFVContext, kind: str, data: bytes, out, max_count: int = 1):
    """deserialize into the device tensor `out`; returns (count, aux)"""
    k = WIRE_KINDS[kind]
    buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
    cnt, aux = C.c_uint32(), C.c_uint64()
    _check(lib().kbfv_wire_load(ctx.handle, k, buf, len(data), _ptr(out), max_count, C.byref(cnt), C.byref(aux), None))
    return cnt.value, aux.value


PROBE_KINDS = ["64x64->128 multiply-accumulate", "mul.lo.u64", "mul.hi.u64",
               "forward NTT butterfly from 64-bit multiplies",
               "Shoup product", "128-bit Barrett", "one-high-product Barrett", "32x32->64 multiply-add",
               "32x32 high product", "32-bit multiply-add", "64x64->128 multiply-accumulate from 32-bit parts",
               "forward NTT butterfly from 32-bit parts (the kernels')",
               "32-bit multiply-add issue rate (IMAD pipe)", "32x32->64 multiply-add issue rate",
               "60x60-bit multiply-accumulate from 30-bit halves", "32-bit high multiply-add issue rate"]


def probe_arith(kind: int, iters: int = 4096) -> float:
    """Gop/s of one modular primitive on the current GPU (kbfv_probe_arith)."""
    v = C.c_double()
    _check(lib().kbfv_probe_arith(kind, iters, C.byref(v)))
    return float(v.value)


def salsa20_stream(key: bytes, nonce: bytes, nbytes: int, block0: int = 0, compat: bool = False, stream=None):
    torch = _torch()
    out = torch.zeros(nbytes, dtype=torch.uint8, device="cuda")
    _check(lib().kbfv_salsa20_stream(_u8(key), _u8(nonce), block0, out.data_ptr(), nbytes, int(compat),
                                     _stream_ptr(stream)))
    return out
