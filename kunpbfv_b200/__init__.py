"""kunpbfv_b200 -- B200-native BFV multiply path behind kunpBFV's API.

The compute path is ``libkbfv.so`` (hand-written sm_100a CUDA, C ABI in
``include/kbfv.h``). This module binds it with ctypes and mirrors the
reference's classes (``BFVContext``, ``BFVScheme``, ``SecretKey``,
``Plaintext``, ``Ciphertext``) for Python callers, tests and the benchmark.
Device memory is held in torch tensors (int64 storage, uint64 bit patterns);
torch is only the allocator and stream provider here.

There is no CPU fallback: if the extension is missing, importing the
bindings raises.
"""
from __future__ import annotations

import ctypes as C
import os

from .api import (  # noqa: F401
    BFVContext,
    BFVScheme,
    Ciphertext,
    KbfvError,
    MulPlan,
    Plaintext,
    SecretKey,
    Tensor3,
    lib,
    library_path,
    reference_context,
)

__all__ = [
    "BFVContext",
    "BFVScheme",
    "Ciphertext",
    "KbfvError",
    "MulPlan",
    "Plaintext",
    "SecretKey",
    "Tensor3",
    "lib",
    "library_path",
    "reference_context",
]
