"""The multiply step's arithmetic count (kunpbfv_b200.roofline) on the
benchmark's parameter set, cross-checked by hand against the pipeline's
kernels, and the profile-to-source tie (CPU only)."""
import os

from kunpbfv_b200 import roofline as rl


def test_c3_counts_per_pair():
    n, log_n, q, p = 16384, 14, 7, 1
    r = q + 1
    pc = rl.pipeline_counts(n, log_n, q, p, 1)
    # K1 4q + K3 4r + K4 3(q+r) + K6a (q+p) + K6b 2p + K7 2q limb transforms
    assert pc["ntt_rows"] == 4 * q + 4 * r + 3 * (q + r) + (q + p) + 2 * p + 2 * q == 129
    c = pc["counts"]
    assert c["bfly"] == 129 * (n // 2) * log_n
    # per coefficient: K2 4qr + K4 2(q+r) + K5a 3r(q+1) + K5b 3rq + lift p*q sums
    assert c["mac"] == n * (4 * q * r + 2 * (q + r) + 3 * r * (q + 1) + 3 * r * q + p * q)
    # K2 4r + K5a 3r + K5b 3q + lift p reductions of 128-bit sums
    assert c["b128"] == n * (4 * r + 3 * r + 3 * q + p)
    # K4 2(q+r) + K6b 2p + K7 2q one-high-product Barrett products
    assert c["prod"] == n * (2 * (q + r) + 2 * p + 2 * q)
    # K2 4q + K4 (q+r) + K5a 3r + K5b 3r + lift q + K7 4q + 2q
    assert c["shoup"] == n * (4 * q + (q + r) + 3 * r + 3 * r + q + 4 * q + 2 * q)
    assert pc["products"] == c["bfly"] + c["mac"] + c["prod"] + c["shoup"] == 28016640
    assert "129" in pc["formula"]


def test_floor_is_the_sum_of_class_times():
    pc = rl.pipeline_counts(16384, 14, 7, 1, 1)
    rates = {k: 1e12 for k in rl.PROBE_KIND}
    assert abs(rl.arithmetic_floor_s(pc["counts"], rates) - (pc["products"] + pc["counts"]["b128"]) / 1e12) < 1e-15


def test_dnum_and_special_primes_change_the_count():
    a = rl.pipeline_counts(32768, 15, 14, 2, 3)
    assert a["ntt_rows"] == 4 * 14 + 4 * 15 + 3 * 29 + 3 * 16 + 2 * 2 + 2 * 14
    b = rl.pipeline_counts(32768, 15, 14, 2, 1)
    assert a["counts"]["mac"] != b["counts"]["mac"]


def test_profile_tie_follows_the_sources(tmp_path):
    files = ["ntt.cuh", "arith.cuh"]
    sha = rl.source_sha16(files)
    assert rl.profile_matches({"source_files": " ".join(files), "source_sha16": sha})
    assert not rl.profile_matches({"source_files": " ".join(files), "source_sha16": "0" * 16})
    assert not rl.profile_matches(None)
    assert not rl.profile_matches({"source_files": "no_such_file.cuh", "source_sha16": sha})
