"""Python binding of the request server (include/kbfv_serve.h) and an
open-loop Poisson load generator over it."""
from __future__ import annotations

import ctypes as C
import threading
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from .api import BFVContext, BFVScheme, KbfvError, SecretKey, _ptr, _u8, lib

OP_MUL, OP_ADD = 0, 1
RETURN_CT = 1


class _Config(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("pinned_bytes", C.c_uint64), ("max_batch", C.c_uint32),
                ("max_active", C.c_uint32), ("inflight_iterations", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("iterations", C.c_uint64), ("mul_launches", C.c_uint64), ("mul_ops", C.c_uint64),
                ("add_ops", C.c_uint64), ("bytes_in_use", C.c_uint64), ("bytes_peak", C.c_uint64),
                ("pending", C.c_uint32), ("active", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_declared = False


def _declare():
    global _declared
    if _declared:
        return
    L = lib()
    VP, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
    U64P = C.POINTER(C.c_uint64)
    sig = {
        "kbfv_server_create": (C.c_int, [C.POINTER(_Config), C.POINTER(VP)]),
        "kbfv_server_add_ring": (C.c_int, [VP, VP, C.POINTER(C.c_uint8), VP, VP, VP, C.POINTER(u32)]),
        "kbfv_server_start": (C.c_int, [VP]),
        "kbfv_server_submit": (C.c_int, [VP, u32, VP, u32, C.POINTER(C.c_uint8), u64, u32, U64P]),
        "kbfv_server_wait": (C.c_int, [VP, u64, C.c_int64, VP, VP, C.POINTER(C.c_double)]),
        "kbfv_server_get_stats": (C.c_int, [VP, C.POINTER(ServerStats)]),
        "kbfv_server_last_error": (C.c_char_p, []),
        "kbfv_server_destroy": (C.c_int, [VP]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype, f.argtypes = res, args
    _declared = True


def _chk(rc, what):
    if rc != 0:
        msg = lib().kbfv_server_last_error() or lib().kbfv_last_error()
        raise KbfvError(rc, f"{what}: {msg.decode() if msg else ''}")


@dataclass
class Ring:
    """One served ring degree: a context with its scheme (public and
    relinearisation keys on the device) and the secret key used to decrypt."""
    ctx: BFVContext
    scheme: BFVScheme
    sk: SecretKey

    @classmethod
    def make(cls, ctx: BFVContext, seed: bytes) -> "Ring":
        sk = SecretKey(ctx, seed)
        sch = BFVScheme(ctx, seed)
        sch.addEncKey(sk)
        sch.addMultKey_23(sk)
        return cls(ctx, sch, sk)


class Server:
    """Continuous-batching server over several rings (kbfv_server_*)."""

    def __init__(self, rings: Sequence[Ring], hbm_budget_bytes: int = 2 << 30, max_batch: int = 64,
                 max_active: int = 0, inflight_iterations: int = 2, pinned_bytes: int = 256 << 20):
        _declare()
        self.rings = list(rings)
        cfg = _Config(hbm_budget_bytes, pinned_bytes, max_batch, max_active, inflight_iterations)
        self._h = C.c_void_p()
        _chk(lib().kbfv_server_create(C.byref(cfg), C.byref(self._h)), "create")
        try:
            for r in self.rings:
                rid = C.c_uint32()
                seed = (C.c_uint8 * 32).from_buffer_copy(r.scheme.seed)
                _chk(lib().kbfv_server_add_ring(self._h, r.ctx.handle, seed, _ptr(r.scheme.publicKey),
                                                _ptr(r.scheme.rlk), _ptr(r.sk.sx_device), C.byref(rid)), "add_ring")
            _chk(lib().kbfv_server_start(self._h), "start")
        except Exception:
            lib().kbfv_server_destroy(self._h)
            self._h = None
            raise

    def submit(self, ring: int, slots: np.ndarray, ops: Sequence[int], enc_id: int, return_ct: bool = False) -> int:
        """slots: (len(ops)+1, N) uint64 values mod t; returns the request id."""
        a = np.ascontiguousarray(slots, dtype=np.uint64)
        o = (C.c_uint8 * len(ops))(*ops)
        rid = C.c_uint64()
        _chk(lib().kbfv_server_submit(self._h, ring, a.ctypes.data, len(ops), o, enc_id,
                                      RETURN_CT if return_ct else 0, C.byref(rid)), "submit")
        return rid.value

    def wait(self, request_id: int, timeout_ms: int = -1, ring: Optional[int] = None, want_ct: bool = False):
        """-> (result slots, final ciphertext or None, latency in ms)"""
        n = self.rings[ring].ctx.N if ring is not None else max(r.ctx.N for r in self.rings)
        out = np.empty(n, dtype=np.uint64)
        ct = None
        if want_ct:
            nq = self.rings[ring].ctx.q_count if ring is not None else max(r.ctx.q_count for r in self.rings)
            ct = np.empty(2 * nq * n, dtype=np.uint64)
        lat = C.c_double()
        _chk(lib().kbfv_server_wait(self._h, request_id, timeout_ms, out.ctypes.data,
                                    ct.ctypes.data if ct is not None else None, C.byref(lat)), "wait")
        return out, ct, lat.value

    def stats(self) -> dict:
        st = ServerStats()
        _chk(lib().kbfv_server_get_stats(self._h, C.byref(st)), "stats")
        return st.as_dict()

    def close(self):
        if self._h:
            lib().kbfv_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def chain_result(slots: np.ndarray, ops: Sequence[int], t: int) -> np.ndarray:
    """the plaintext chain: acc = x0; acc = acc (op) x_{i+1} mod t"""
    acc = slots[0].astype(np.uint64)
    for i, op in enumerate(ops):
        x = slots[i + 1].astype(np.uint64)
        acc = (acc * x) % t if op == OP_MUL else (acc + x) % t
    return acc


@dataclass
class Workload:
    """Pre-generated request templates: per template a ring, an op chain, its
    input slots and the expected plaintext result."""
    ring: List[int] = field(default_factory=list)
    ops: List[List[int]] = field(default_factory=list)
    slots: List[np.ndarray] = field(default_factory=list)
    want: List[np.ndarray] = field(default_factory=list)


def make_workload(rings: Sequence[Ring], templates: int, max_mul: Sequence[int], seed: int = 0,
                  max_ops: int = 4) -> Workload:
    """Chains of 1..max_ops operations; at most max_mul[r] multiplies on ring r
    (its noise budget); the ring of each template is uniform over rings."""
    rng = np.random.default_rng(seed)
    w = Workload()
    for _ in range(templates):
        r = int(rng.integers(0, len(rings)))
        k = int(rng.integers(1, max_ops + 1))
        muls = 0
        ops = []
        for _ in range(k):
            op = OP_MUL if (rng.random() < 0.6 and muls < max_mul[r]) else OP_ADD
            muls += op == OP_MUL
            ops.append(op)
        t = rings[r].ctx.plain_modulus
        slots = rng.integers(0, t, size=(k + 1, rings[r].ctx.N), dtype=np.uint64)
        w.ring.append(r)
        w.ops.append(ops)
        w.slots.append(slots)
        w.want.append(chain_result(slots, ops, t))
    return w


def run_open_loop(server: Server, w: Workload, rate: float, duration_s: float, seed: int = 1,
                  enc_base: int = 1 << 32, return_ct: bool = False) -> dict:
    """Poisson arrivals at `rate` requests/s for `duration_s`, requests cycling
    through the workload templates with fresh encryption ids. Latency is
    submit-to-decrypted-result as the server measures it. Every result is
    checked against the plaintext chain."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=int(rate * duration_s * 1.5) + 16)
    arrivals = np.cumsum(gaps)
    arrivals = arrivals[arrivals < duration_s]
    ids = []
    lock = threading.Lock()
    lat, wrong, errors, bad = [], [0], [], []
    done = threading.Event()

    def collector():
        i = 0
        while True:
            with lock:
                have = len(ids)
            if i >= have:
                if done.is_set():
                    with lock:
                        if i >= len(ids):
                            return
                    continue
                time.sleep(0.0002)
                continue
            rid, tmpl = ids[i]
            try:
                res, _, ms = server.wait(rid, ring=w.ring[tmpl])
                lat.append(ms)
                if not np.array_equal(res, w.want[tmpl]):
                    wrong[0] += 1
                    if len(bad) < 8:
                        bad.append({"request": rid, "ring": w.ring[tmpl], "ops": w.ops[tmpl],
                                    "slots_wrong": int(np.count_nonzero(res != w.want[tmpl]))})
            except KbfvError as e:
                errors.append(str(e))
            i += 1

    th = threading.Thread(target=collector, daemon=True)
    th.start()
    t0 = time.perf_counter()
    for j, at in enumerate(arrivals):
        now = time.perf_counter() - t0
        if at > now:
            time.sleep(at - now)
        tmpl = j % len(w.ring)
        rid = server.submit(w.ring[tmpl], w.slots[tmpl], w.ops[tmpl], enc_base + 16 * j, return_ct)
        with lock:
            ids.append((rid, tmpl))
    t_sub = time.perf_counter() - t0
    done.set()
    th.join()
    t_all = time.perf_counter() - t0
    lat_a = np.array(lat) if lat else np.array([float("nan")])
    return {
        "rate": rate, "offered": len(arrivals), "completed": len(lat), "wrong": wrong[0], "errors": len(errors),
        "duration_s": round(t_all, 3), "submit_span_s": round(t_sub, 3),
        "throughput": round(len(lat) / t_all, 1),
        "p50_ms": round(float(np.percentile(lat_a, 50)), 3), "p99_ms": round(float(np.percentile(lat_a, 99)), 3),
        "mean_ms": round(float(lat_a.mean()), 3),
        **({"wrong_detail": bad} if bad else {}),
    }
