"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute calls: this runs without a GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    inc = os.path.join(ROOT, "include")
    for fn in sorted(os.listdir(inc)):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(inc, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(kbfv_[A-Za-z0-9_]+)\s*\(", src, re.M):
            names.append(m.group(1))
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_symbols()
    # the entry points a kunpBFV caller binds (context, keys, encoder, scheme ops, NTT, seed)
    for must in ("kbfv_params_create", "kbfv_context_create", "kbfv_context_destroy", "kbfv_keygen_secret",
                 "kbfv_keygen_public", "kbfv_keygen_relin", "kbfv_encode", "kbfv_decode", "kbfv_encrypt",
                 "kbfv_decrypt", "kbfv_add", "kbfv_add_plain", "kbfv_mul_plain", "kbfv_mul", "kbfv_relinearize",
                 "kbfv_mul_relin_batch", "kbfv_ntt_fwd", "kbfv_ntt_inv", "kbfv_ntt_fwd_batch", "kbfv_ntt_inv_batch",
                 "kbfv_noise_budget", "kbfv_set_seed"):
        assert must in names, must


def test_library_exports_all_declared_symbols():
    from kunpbfv_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_reports_version_without_gpu():
    import kunpbfv_b200 as kb
    assert b"sm_100a" in kb.lib().kbfv_version()


def test_params_create_without_gpu(oracle_mod):
    """Per-prime bit sizes (36, 36 | 37 at N=4096) give distinct NTT-friendly
    primes equal to the oracle's generator; no device is touched."""
    import kunpbfv_b200 as kb
    from kunpbfv_b200.api import _Params
    L = kb.lib()
    qb = (ctypes.c_uint32 * 2)(36, 36)
    pb = (ctypes.c_uint32 * 1)(37)
    out = ctypes.POINTER(_Params)()
    assert L.kbfv_params_create(12, qb, 2, pb, 1, 65537, 2, ctypes.byref(out)) == 0
    prm = out.contents
    q = [prm.q[i] for i in range(prm.q_count)]
    p = [prm.p[i] for i in range(prm.p_count)]
    assert prm.log_n == 12 and prm.plain_modulus == 65537 and prm.dnum == 2
    assert [x.bit_length() for x in q] == [36, 36] and [x.bit_length() for x in p] == [37]
    assert len(set(q + p)) == 3 and all(x % 8192 == 1 for x in q + p)
    want_p = oracle_mod.primes_bits(4096, 37, 1)
    want_q = oracle_mod.primes_bits(4096, 36, 2, skip=want_p)
    assert p == want_p and q == want_q
    assert L.kbfv_params_destroy(out) == 0
    # out-of-range sizes are rejected with a status, not a crash
    bad = (ctypes.c_uint32 * 1)(61)
    out2 = ctypes.POINTER(_Params)()
    assert L.kbfv_params_create(12, bad, 1, pb, 1, 65537, 1, ctypes.byref(out2)) == -1


def test_compat_header_compiles_and_links(tmp_path):
    """include/kbfv_compat.hpp (the reference's class API over the C ABI) and the
    reference-style driver compile and link against libkbfv.so without a GPU."""
    import shutil
    import subprocess
    from kunpbfv_b200 import build
    nvcc = "/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else shutil.which("nvcc")
    if not nvcc:
        pytest.skip("nvcc not available")
    lib = build.build()
    out = tmp_path / "compat_mult"
    r = subprocess.run([nvcc, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                        os.path.join(ROOT, "tests", "cpp", "compat_mult.cpp"), "-L", os.path.dirname(lib), "-lkbfv",
                        "-Xlinker", "-rpath", "-Xlinker", os.path.dirname(lib), "-o", str(out)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert out.exists()


def _reference_dir():
    """Where the oracle recipe finds the reference sources (oracle/Makefile's REF)."""
    import re as _re
    with open(os.path.join(ROOT, "oracle", "Makefile")) as f:
        m = _re.search(r"^REF\s*\?=\s*(\S+)", f.read(), _re.M)
    return os.environ.get("REF") or (m.group(1) if m else "")


REF = _reference_dir()
DRIVERS = ["correct_mult", "correct_add", "correct_encrypt", "perf_mult", "perf_add", "perf_encrypt", "bfv_demo"]


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF, "include")), reason="reference sources absent")
def test_reference_drivers_compile_unmodified(tmp_path):
    """The reference's seven driver programs compile, byte for byte as they
    are, against the drop-in headers include/kunpbfv/ and link to libkbfv.so
    (the recipe is oracle/Makefile's `drivers` target)."""
    import subprocess
    from kunpbfv_b200 import build
    build.build()
    out = tmp_path / "drivers"
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-s", "drivers", f"DRIVER_OUT={out}"],
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    for d in DRIVERS:
        assert (out / d).exists(), d
