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
    for must in ("kbfv_context_create", "kbfv_ntt_fwd", "kbfv_mul_relin_batch", "kbfv_encrypt", "kbfv_decrypt",
                 "kbfv_relinearize", "kbfv_keygen_relin", "kbfv_noise_budget"):
        assert must in names


def test_library_exports_all_declared_symbols():
    from kunpbfv_b200 import build
    path = build.build()
    lib = ctypes.CDLL(path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_library_reports_version_without_gpu():
    import kunpbfv_b200 as kb
    assert b"sm_100a" in kb.lib().kbfv_version()
