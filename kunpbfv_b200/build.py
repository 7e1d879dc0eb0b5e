"""Build libkbfv.so (sm_100a) in-tree with nvcc: each translation unit is
compiled to an object under _build/ (in parallel, only when it or a header
changed), then linked into the shared library."""
from __future__ import annotations

import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libkbfv.so")
# native timing program of the per-call forms (bench.py runs it), linked to LIB
PEROP_SRC = os.path.join(HERE, "csrc", "perop_bench.cpp")
PEROP_BIN = os.path.join(HERE, "perop_bench")
OBJDIR = os.path.join(HERE, "_build")
# translation units of libkbfv.so (compiled in parallel)
SOURCES = [os.path.join(HERE, "csrc", f) for f in
           ("k5_m8.cu", "k5_m16.cu", "k5_m24.cu", "k5_m33.cu", "mul.cu", "levels.cu", "scheme.cu", "ntt_ops.cu", "klss_api.cu", "context.cu", "plan.cu", "serve.cpp")]
HEADERS = [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))
           if f.endswith((".cuh", ".hpp", ".h"))] + [
    os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]
DEPS = SOURCES + HEADERS

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(d) > t for d in DEPS if os.path.exists(d))


def _obj(src: str) -> str:
    return os.path.join(OBJDIR, os.path.basename(src) + ".o")


def _stale_obj(src: str) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return any(os.path.getmtime(d) > t for d in [src] + HEADERS if os.path.exists(d))


def build_perop(force: bool = False) -> str:
    """The per-call timing program (host code over the C ABI)."""
    if force or not os.path.exists(PEROP_BIN) or any(
            os.path.getmtime(d) > os.path.getmtime(PEROP_BIN) for d in (PEROP_SRC, LIB)):
        subprocess.run([nvcc(), "-std=c++17", "-O2", PEROP_SRC, "-L", HERE, "-lkbfv", "-Xlinker", "-rpath",
                        "-Xlinker", "$ORIGIN", "-o", PEROP_BIN + ".tmp"], check=True)
        os.replace(PEROP_BIN + ".tmp", PEROP_BIN)
    return PEROP_BIN


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not stale():
        build_perop()
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    todo = [s for s in SOURCES if force or _stale_obj(s)]

    def compile_one(src):
        cmd = [nvcc(), *NVCC_FLAGS, "-c", "-o", _obj(src) + ".tmp", src]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        os.replace(_obj(src) + ".tmp", _obj(src))

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        for f in [ex.submit(compile_one, s) for s in todo]:
            f.result()
    link = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp",
            *[_obj(s) for s in SOURCES], "-lpthread"]
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    build_perop(force=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
