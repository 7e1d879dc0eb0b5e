"""Autotuner for the speed-only knobs of a context (``kbfv_tune_set``).

Knobs (include/kbfv.h, ``kbfv_tune_knob``):

* ``ntt_block_log`` - the radix split of the standalone NTT on rings above
  2^v points: a column pass of ``log_n - v`` stages and block kernels of 2^v
  points, v in 12..14, or 0 for the built-in shapes;
* ``branches`` - sub-batches (one stream each) of a batched multiply, 1..4;
* ``host_chunk`` - pairs per chunk of the host-memory multiply, 0..128;
* the launch shapes inside the multiply pipeline: ``split_rows`` (at N=2^14,
  transforms of at most this many rows run as a radix-4 column pass and
  2^12-point blocks instead of one 1024-thread block per row), ``bconv_threads``
  (CTA size of the Q -> R base conversion), ``k5_threads`` (CTA size of the
  scale-and-round / R -> Q / digit-lift kernels) and ``k5_fused_pairs``
  (batches of at most this many pairs run those as one kernel), ``bconv_cpt``
  (coefficients per thread of the base conversion) and ``fuse_q2r_pairs``
  (batches of at most this many pairs run the Q -> R base extension in the
  loader of the forward NTT over R, no separate base-conversion launch),
  ``l2_prefetch`` (NTT block kernels ask L2 for the block one wave ahead)
  ``split_rows_alone`` (``split_rows`` for multiplies that run as one
  stream, where no sibling sub-batch fills idle SMs) and ``min_branch_pairs``
  (pairs per sub-batch at least).

Each candidate is timed on the device with CUDA events (two warm-up calls,
then the median of three timed trials of ``reps`` calls). Knobs never change
results: every candidate's output is compared with the default's, and a
mismatch raises. The winners are applied to the context and stored in a JSON
cache keyed by device and parameter set, so a later process applies them with
``apply_cached`` instead of timing again. The reference has no tuner (its
kernel shapes are fixed at compile time).
"""
from __future__ import annotations

import json
import os
import statistics
from typing import Callable, Dict, Optional

DEFAULT_CACHE = os.environ.get("KBFV_TUNE_CACHE",
                               os.path.join(os.path.expanduser("~"), ".cache", "kunpbfv_b200", "tune.json"))

NTT_BLOCK_LOGS = (0, 12, 13, 14)  # 0: built-in shapes
BRANCHES = (1, 2, 3, 4)
HOST_CHUNKS = (4, 8, 12, 16, 24)
# the multiply pipeline's launch shapes, tuned one after another on the batch
# (coordinate descent from the defaults, first candidate of each list)
PIPELINE_KNOBS = {
    "branches": (2, 1, 3, 4),
    "bconv_threads": (256, 128, 512, 64),
    "bconv_cpt": (2, 1),
    "k5_threads": (128, 64, 256),
    "split_rows": (48, 0, 256, 1 << 20),
    "l2_prefetch": (1, 0),
}
# tuned on a two-pair multiply (the per-call size it governs)
K5_FUSED_PAIRS = (2, 0, 4)
# tuned on one-pair and two-pair multiplies together
FUSE_Q2R_PAIRS = (1, 0, 2)
# tuned on four-pair and eight-pair multiplies (1 and 2 tie there; 1 is 3.5%
# faster at three pairs)
MIN_BRANCH_PAIRS = (1, 2, 4, 8)
# tuned on two-pair and eight-pair multiplies
SPLIT_ROWS_ALONE = (148, 48, 96, 256, 512)


def cache_key(device: str, log_n: int, q_count: int, p_count: int, dnum: int, pairs: int) -> str:
    return f"{device}|logn={log_n}|q={q_count}|p={p_count}|dnum={dnum}|pairs={pairs}"


def context_key(ctx, pairs: int) -> str:
    import torch
    dev = torch.cuda.get_device_name()
    return cache_key(dev, ctx.log_n, ctx.q_count, ctx.p_count, ctx.dnum, pairs)


def load_cache(path: str = DEFAULT_CACHE) -> Dict[str, dict]:
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def save_cache(entries: Dict[str, dict], path: str = DEFAULT_CACHE) -> None:
    """Merge `entries` into the cache file (written atomically)."""
    data = load_cache(path)
    data.update(entries)
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def time_ms(fn: Callable[[], None], reps: int = 5, trials: int = 3) -> float:
    """Median over `trials` of the CUDA-event time of `reps` calls, per call."""
    import torch
    stream = torch.cuda.current_stream()
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(trials):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        out.append(a.elapsed_time(b) / reps)
    return statistics.median(out)


def _random_rows(ctx, rows: int, prime0: int, period: int, seed: int = 1):
    import torch
    g = torch.Generator(device="cuda").manual_seed(seed)
    x = torch.randint(0, 1 << 62, (rows, ctx.N), dtype=torch.int64, device="cuda", generator=g)
    mods = torch.tensor([ctx.primes[prime0 + r % period] for r in range(rows)], dtype=torch.int64, device="cuda")
    return torch.remainder(x, mods[:, None])


def tune_ntt(ctx, rows: int = 512, reps: int = 5) -> Dict[str, object]:
    """Radix split of the standalone forward + inverse NTT over `rows` rows."""
    import torch
    if ctx.log_n <= 12:
        return {"ntt_block_log": 0, "ms": {}}
    keep = ctx.tune_get("ntt_block_log")
    x0 = _random_rows(ctx, rows, 0, ctx.q_count)
    ms, want = {}, None
    try:
        for v in [v for v in NTT_BLOCK_LOGS if v < ctx.log_n]:
            ctx.tune_set("ntt_block_log", v)
            y = x0.clone()
            ctx.ntt_fwd(y, 0, ctx.q_count)
            torch.cuda.synchronize()
            if want is None:
                want = y.clone()
            elif not torch.equal(y, want):
                raise RuntimeError(f"NTT split {v} changed the transform")
            ctx.ntt_inv(y, 0, ctx.q_count)
            torch.cuda.synchronize()
            if not torch.equal(y, x0):
                raise RuntimeError(f"NTT split {v} broke the round trip")

            def step():
                ctx.ntt_fwd(y, 0, ctx.q_count)
                ctx.ntt_inv(y, 0, ctx.q_count)
            ms[v] = round(time_ms(step, reps), 4)
    finally:
        ctx.tune_set("ntt_block_log", keep)
    best = min(ms, key=ms.get)
    return {"ntt_block_log": best, "ms": {str(k): v for k, v in ms.items()}}


def _random_pairs(ctx, pairs: int, seed: int):
    import torch
    rows = pairs * 2 * ctx.q_count
    return _random_rows(ctx, rows, 0, ctx.q_count, seed).view(pairs, 2, ctx.q_count, ctx.N)


def tune_host_chunk(scheme, pairs: int = 64, reps: int = 3) -> Dict[str, object]:
    """Pairs per chunk of the host-memory multiply (page-locked buffers)."""
    import torch
    ctx = scheme.context
    h_a = _random_pairs(ctx, pairs, 4).cpu().pin_memory()
    h_b = _random_pairs(ctx, pairs, 5).cpu().pin_memory()
    h_o = torch.empty_like(h_a).pin_memory()
    ms, want = {}, None
    for ch in HOST_CHUNKS:
        if ch > pairs:
            continue
        scheme.mult_relin_host(h_a, h_b, out=h_o, chunk_pairs=ch)
        if want is None:
            want = h_o.clone()
        elif not torch.equal(h_o, want):
            raise RuntimeError(f"host chunk {ch} changed the product")
        ms[ch] = round(time_ms(lambda: scheme.mult_relin_host(h_a, h_b, out=h_o, chunk_pairs=ch,
                                                              synchronize=False), reps), 4)
    if not ms:
        return {"host_chunk": 0, "ms": {}}
    best = min(ms, key=ms.get)
    return {"host_chunk": best, "ms": {str(k): v for k, v in ms.items()}}


def _sweep(ctx, knob, values, run, out, want, reps):
    """Time `run` for every value of `knob` (others as set); every output must
    equal `want` (a ciphertext and its expected tensor, or tuples of both).
    Leaves the fastest value applied; returns {value: ms}."""
    import torch
    outs, wants = (out, want) if isinstance(out, tuple) else ((out,), (want,))
    ms = {}
    for v in values:
        ctx.tune_set(knob, v)
        run()
        torch.cuda.synchronize()
        if not all(torch.equal(o.cipher_device, w) for o, w in zip(outs, wants)):
            raise RuntimeError(f"{knob}={v} changed the product")
        ms[v] = round(time_ms(run, reps), 4)
    ctx.tune_set(knob, min(ms, key=ms.get))
    return ms


def tune_pipeline(scheme, pairs: int = 64, reps: int = 5) -> Dict[str, object]:
    """The multiply pipeline's knobs (PIPELINE_KNOBS on a batch of `pairs`,
    K5_FUSED_PAIRS on two pairs, FUSE_Q2R_PAIRS on one and two pairs), one at
    a time from the defaults; every candidate's product is compared with the
    default shapes' product."""
    import torch

    from .api import Ciphertext
    ctx = scheme.context
    keep = {k: ctx.tune_get(k) for k in list(PIPELINE_KNOBS) + ["k5_fused_pairs", "fuse_q2r_pairs",
                                                                  "split_rows_alone", "min_branch_pairs"]}
    c1 = Ciphertext(ctx, _random_pairs(ctx, pairs, 2))
    c2 = Ciphertext(ctx, _random_pairs(ctx, pairs, 3))
    out = Ciphertext(ctx, count=pairs)
    two = min(2, pairs)
    d1 = Ciphertext(ctx, c1.cipher_device[:two].clone())
    d2 = Ciphertext(ctx, c2.cipher_device[:two].clone())
    out2 = Ciphertext(ctx, count=two)
    e1 = Ciphertext(ctx, c1.cipher_device[:1].clone())
    e2 = Ciphertext(ctx, c2.cipher_device[:1].clone())
    out1 = Ciphertext(ctx, count=1)
    eight = min(8, pairs)
    f1 = Ciphertext(ctx, c1.cipher_device[:eight].clone())
    f2 = Ciphertext(ctx, c2.cipher_device[:eight].clone())
    out8 = Ciphertext(ctx, count=eight)
    four = min(4, pairs)
    g1 = Ciphertext(ctx, c1.cipher_device[:four].clone())
    g2 = Ciphertext(ctx, c2.cipher_device[:four].clone())
    out4 = Ciphertext(ctx, count=four)
    result: Dict[str, object] = {}
    try:
        for k, vals in PIPELINE_KNOBS.items():  # defaults first: the reference products
            ctx.tune_set(k, vals[0])
        ctx.tune_set("k5_fused_pairs", K5_FUSED_PAIRS[0])
        ctx.tune_set("fuse_q2r_pairs", FUSE_Q2R_PAIRS[0])
        ctx.tune_set("split_rows_alone", SPLIT_ROWS_ALONE[0])
        ctx.tune_set("min_branch_pairs", MIN_BRANCH_PAIRS[0])
        scheme.mult_relin(c1, c2, out=out)
        scheme.mult_relin(d1, d2, out=out2)
        scheme.mult_relin(e1, e2, out=out1)
        scheme.mult_relin(f1, f2, out=out8)
        scheme.mult_relin(g1, g2, out=out4)
        torch.cuda.synchronize()
        want, want2, want1 = out.cipher_device.clone(), out2.cipher_device.clone(), out1.cipher_device.clone()
        want8 = out8.cipher_device.clone()
        want4 = out4.cipher_device.clone()
        for k, vals in PIPELINE_KNOBS.items():
            ms = _sweep(ctx, k, vals, lambda: scheme.mult_relin(c1, c2, out=out), out, want, reps)
            result[k], result[k + "_ms"] = min(ms, key=ms.get), {str(v): t for v, t in ms.items()}
        ms = _sweep(ctx, "k5_fused_pairs", K5_FUSED_PAIRS, lambda: scheme.mult_relin(d1, d2, out=out2), out2,
                    want2, reps)
        result["k5_fused_pairs"], result["k5_fused_pairs_ms"] = min(ms, key=ms.get), {
            str(v): t for v, t in ms.items()}

        def per_call():
            scheme.mult_relin(e1, e2, out=out1)
            scheme.mult_relin(d1, d2, out=out2)
        ms = _sweep(ctx, "fuse_q2r_pairs", FUSE_Q2R_PAIRS, per_call, (out1, out2), (want1, want2), reps)
        result["fuse_q2r_pairs"], result["fuse_q2r_pairs_ms"] = min(ms, key=ms.get), {
            str(v): t for v, t in ms.items()}

        def small():
            scheme.mult_relin(g1, g2, out=out4)
            scheme.mult_relin(f1, f2, out=out8)
        ms = _sweep(ctx, "min_branch_pairs", MIN_BRANCH_PAIRS, small, (out4, out8), (want4, want8), reps)
        result["min_branch_pairs"], result["min_branch_pairs_ms"] = min(ms, key=ms.get), {
            str(v): t for v, t in ms.items()}

        def one_stream():
            scheme.mult_relin(d1, d2, out=out2)
            scheme.mult_relin(f1, f2, out=out8)
        ms = _sweep(ctx, "split_rows_alone", SPLIT_ROWS_ALONE, one_stream, (out2, out8), (want2, want8), reps)
        result["split_rows_alone"], result["split_rows_alone_ms"] = min(ms, key=ms.get), {
            str(v): t for v, t in ms.items()}
    except Exception:
        for k, v in keep.items():
            ctx.tune_set(k, v)
        raise
    return result


PIPELINE_CHOICES = ("branches", "bconv_threads", "bconv_cpt", "k5_threads", "split_rows", "l2_prefetch",
                    "k5_fused_pairs", "fuse_q2r_pairs", "min_branch_pairs", "split_rows_alone")


def apply_choice(ctx, choice: dict) -> None:
    for knob in ("ntt_block_log", "host_chunk") + PIPELINE_CHOICES:
        if knob in choice:
            ctx.tune_set(knob, int(choice[knob]))


def autotune(ctx, scheme=None, pairs: int = 64, cache_path: Optional[str] = DEFAULT_CACHE, force: bool = False,
             ntt_rows: int = 512, host: bool = True) -> dict:
    """Pick every knob for `ctx` (the multiply knobs need `scheme` with a
    relinearisation key), apply the choice and store it in the cache. A cached
    choice for the same device and parameter set is applied without timing
    unless `force`."""
    key = context_key(ctx, pairs)
    if cache_path and not force:
        hit = load_cache(cache_path).get(key)
        if hit is not None:
            apply_choice(ctx, hit)
            return dict(hit, cached=True)
    choice: Dict[str, object] = {}
    r = tune_ntt(ctx, ntt_rows)
    choice["ntt_block_log"], choice["ntt_ms"] = r["ntt_block_log"], r["ms"]
    if scheme is not None and scheme.rlk is not None and scheme.relin == "hybrid":
        choice.update(tune_pipeline(scheme, pairs))
        if host:
            r = tune_host_chunk(scheme, pairs)
            choice["host_chunk"], choice["host_chunk_ms"] = r["host_chunk"], r["ms"]
    apply_choice(ctx, choice)
    if cache_path:
        save_cache({key: choice}, cache_path)
    return dict(choice, cached=False)


def apply_cached(ctx, pairs: int = 64, cache_path: str = DEFAULT_CACHE) -> Optional[dict]:
    """Apply a stored choice for this device and parameter set, if any."""
    hit = load_cache(cache_path).get(context_key(ctx, pairs))
    if hit is not None:
        apply_choice(ctx, hit)
    return hit
