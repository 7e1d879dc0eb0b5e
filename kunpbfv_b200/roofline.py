"""Arithmetic roofline of the fused multiply + relinearise pipeline.

At 60-bit moduli every kernel of the multiply is bound by the issue rate of
64-bit integer multiplies on the IMAD ("fmaheavy") pipe, not by HBM. This
module counts the modular arithmetic one ciphertext pair costs in the 9-kernel
pipeline (kunpbfv_b200/csrc/mul.cu, k5_kernels.cuh, pipeline.cuh), by class of
primitive:

  bfly   NTT butterfly (one Shoup product with a three-partial-product quotient
         plus lazy add/sub: ct_bfly / gs_bfly, csrc/ntt.cuh)
  mac    60x60 -> 128-bit multiply-accumulate (mac32, csrc/arith.cuh)
  prod   product of two residues reduced by the one-high-product Barrett
         (mul_mod_prod)
  b128   128-bit Barrett reduction (barrett128)
  shoup  one high and one low 64-bit product: a Shoup product with a
         precomputed quotient, a 64-bit Barrett, or a one-high-product Barrett
         of a ready 128-bit sum

and turns the counts into the time the step would take if every primitive ran
at the rate `kbfv_probe_arith` measures for it in register chains on the same
GPU (no memory traffic, no synchronisation): the arithmetic floor of the step.
The step's roofline fraction is that floor divided by the measured step time.

It also reads the IMAD-pipe instruction counts of the same pipeline from a
committed ncu summary (profiles/mult_relin_imad_n16384.md) when that summary was
taken from the current kernel sources (it records the csrc/ files it covers
and a hash of them).
"""
from __future__ import annotations

import hashlib
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

# probe kinds of kbfv_probe_arith measuring each class
PROBE_KIND = {"bfly": 11, "mac": 10, "prod": 6, "b128": 5, "shoup": 4}


def pipeline_counts(n: int, log_n: int, nq: int, np_: int, dnum: int) -> dict:
    """Per-pair primitive counts of the hybrid multiply + relinearise
    (kbfv_mul_relin_batch) for ring degree n, nq ciphertext primes, np_ special
    primes and dnum key-switch digits (R base of nq + 1 primes)."""
    nr, npq = nq + 1, nq + np_
    nqr = nq + nr
    alpha = -(-nq // dnum)
    digits = [min(alpha, nq - d * alpha) for d in range(dnum)]
    # limb NTTs: K1 INTT of 4 polys over Q, K3 NTT of 4 over R, K4 INTT of 3
    # over Q|R, K6a NTT of the dnum digits over Q|P, K6b INTT of 2 over P,
    # K7 NTT of 2 over Q
    ntt_rows = 4 * nq + 4 * nr + 3 * nqr + dnum * npq + 2 * np_ + 2 * nq
    c = {k: 0 for k in PROBE_KIND}
    c["bfly"] = ntt_rows * (n // 2) * log_n
    per_coeff = {k: 0 for k in PROBE_KIND}

    def add(**kw):
        for k, v in kw.items():
            per_coeff[k] += v

    # K2 Q -> R (4 polys): y_i = Shoup(x_i), nq x nr sums, nr reductions
    add(shoup=4 * nq, mac=4 * nq * nr, b128=4 * nr)
    # K4 tensor in the INTT's loader, per limb of Q|R: a1a2 and b1b2 (prod),
    # a1b2 + b1a2 (2 mac + one-high-product Barrett)
    add(prod=2 * nqr, mac=2 * nqr, shoup=nqr)
    # K5a scale-and-round (3 polys): per R prime nq + 1 sums, a reduction and
    # the rounding term mod r_j
    add(mac=3 * nr * (nq + 1), b128=3 * nr, shoup=3 * nr)
    # K5b R -> Q (3 polys)
    add(shoup=3 * nr, mac=3 * nr * nq, b128=3 * nq)
    # K5b digit lift of a1a2: per digit its Shoup products, and per prime of
    # Q|P outside the digit a sum over the digit and a reduction
    for a in digits:
        add(shoup=a, mac=(npq - a) * a, b128=(npq - a))
    # K6b key product over P in the INTT's loader (2 halves)
    if dnum == 1:
        add(prod=2 * np_)
    else:
        add(mac=2 * np_ * dnum, b128=2 * np_)
    # K7: mod down in the NTT's loader, key product over Q and P^-1 at its store
    if np_ == 1:
        add(shoup=2 * nq * 2)
    else:
        add(shoup=2 * nq * (np_ + 1), mac=2 * nq * np_, b128=2 * nq)
    if dnum == 1:
        add(prod=2 * nq, shoup=2 * nq)
    else:
        add(mac=2 * nq * dnum, b128=2 * nq, shoup=2 * nq)
    for k, v in per_coeff.items():
        c[k] += v * n
    formula = (
        f"bfly = limb-NTTs x (N/2) log2 N = (4q + 4r + 3(q+r) + dnum(q+p) + 2p + 2q) x {n // 2} x {log_n}"
        f" = {ntt_rows} x {n // 2 * log_n}; per coefficient: K2 4q shoup + 4qr mac + 4r b128;"
        f" K4 2(q+r) prod + 2(q+r) mac + (q+r) shoup; K5a 3r(q+1) mac + 3r b128 + 3r shoup;"
        f" K5b 3r shoup + 3rq mac + 3q b128, lift sum_d [a_d shoup + (q+p-a_d)(a_d mac + b128)];"
        f" K6b 2p prod (dnum 1); K7 4q shoup + 2q prod + 2q shoup (p = 1, dnum 1);"
        f" q={nq} r={nr} p={np_} dnum={dnum} N={n}"
    )
    products = c["bfly"] + c["mac"] + c["prod"] + c["shoup"]
    return {"counts": c, "ntt_rows": ntt_rows, "products": products, "formula": formula}


def arithmetic_floor_s(counts: dict, rates: dict) -> float:
    """Seconds per pair if every primitive ran at its measured rate (rates in op/s)."""
    return sum(counts[k] / rates[k] for k in counts if counts[k])


def source_sha16(files) -> str:
    """Hash of the named CUDA sources of libkbfv (file names under csrc/): ties
    a committed profile to the kernels it was taken from."""
    h = hashlib.sha256()
    d = os.path.join(HERE, "csrc")
    for f in sorted(files):
        with open(os.path.join(d, f), "rb") as fh:
            h.update(f.encode() + b"\0" + fh.read())
    return h.hexdigest()[:16]


def profile_matches(prof: dict | None) -> bool:
    """True when a profile summary names its source files and their hash
    equals the current sources' hash."""
    if not prof or "source_files" not in prof or "source_sha16" not in prof:
        return False
    try:
        return source_sha16(prof["source_files"].split()) == prof["source_sha16"]
    except OSError:
        return False


def read_profile(name: str) -> dict | None:
    """`key: value` lines of a committed profile summary (profiles/<name>);
    None when absent."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    out = {}
    with open(path) as f:
        for line in f:
            m = re.match(r"^- `([a-z0-9_]+)`: `([^`]*)`", line.strip())
            if m:
                out[m.group(1)] = m.group(2)
    return out
