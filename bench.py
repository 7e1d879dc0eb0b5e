"""Benchmark: batched BFV multiply + relinearise at N=16384 on B200.

Workload (one "step"): 64 independent ciphertext pairs, N=16384, 7 x 60-bit
ciphertext primes + 1 special prime, t=65537, dnum=1, multiplied and
relinearised by one fused launch sequence (captured in a CUDA graph).
Inputs are resident in HBM (235 MB, larger than the 126 MB L2, so no flush
is needed between steps).

The end-to-end rate (`e2e`) goes through the C ABI with page-locked host
buffers (kbfv_mul_relin_host: copies inside the timed region, overlapped with
the multiply), on every rank, timed as the maximum over ranks. At one GPU the
line also carries the side measurements: the one-pair-per-call ("per-op")
forms, the standalone NTT at N=65536 x 2048 rows (32 primes x 64 polynomials),
the uneven-level batch, the serving sweep and the CPU baseline; with more GPUs
they are skipped, since every GPU of the job would wait for rank 0. The default
300 timed steps take about a second, so the SM clock is sampled (every 20 ms)
many times inside the timed region; only those samples are reported.

`--impl reference` times the reference path on the host cores instead: the
reference (kunpBFV) has no CPU implementation, so this is the CPU oracle's
restatement of it, run with all host threads.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "BFV mult+relin ct/s @N=16384 batched vs per-op on 1 B200; NTT HBM GB/s; p50/p99"
T = 65537
LOG_N = 14
NQ, NP = 7, 1
BATCH = 64
SEED = bytes(range(32))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--skip-extras", action="store_true", help="only the headline workload")
    ap.add_argument("--kernel", default=None, choices=["ntt16k", "ntt16k_inv", "pipeline1", "arith"],
                    help="run one kernel on a profiling-sized case and exit (for ncu)")
    ap.add_argument("--rows", type=int, default=1024, help="rows for the ntt16k profiling cases")
    ap.add_argument("--pairs", type=int, default=16, help="pairs for the pipeline1 profiling case")
    ap.add_argument("--set", default="", help="tuning knobs for the profiling cases, e.g. bconv_cpt=1,k5_threads=256")
    ap.add_argument("--serve-rates", default="500,1000,2000,3000,4000,6000,8000",
                    help="Poisson arrival rates (requests/s) of the serving sweep")
    ap.add_argument("--serve-seconds", type=float, default=2.5,
                    help="shortest arrival window per rate (longer where needed for --serve-requests)")
    ap.add_argument("--serve-requests", type=int, default=10000,
                    help="requests offered per rate point at least (window = max(seconds, requests / rate))")
    ap.add_argument("--serving-only", action="store_true", help="run only the serving sweep and print it")
    return ap.parse_args()


def run_kernel_case(args):
    """Profiling cases: the forward / inverse NTT block kernel on --rows rows of
    N=16384 (1024 rows = 128 MiB, above L2), batched multiplies of --pairs pairs,
    or the arithmetic-rate probe of the 64-bit modular primitives."""
    import torch

    import kunpbfv_b200 as kb
    if args.kernel == "arith":
        from kunpbfv_b200.api import PROBE_KINDS, probe_arith
        print(json.dumps({name: round(probe_arith(k), 1) for k, name in enumerate(PROBE_KINDS)}))
        return
    ctx = c3_context(kb)
    for kv in filter(None, args.set.split(",")):
        knob, value = kv.split("=")
        ctx.tune_set(knob.strip(), int(value))
    if args.kernel.startswith("ntt16k"):
        rows = args.rows
        x = torch.randint(0, 1 << 59, (rows, ctx.N), dtype=torch.int64, device="cuda")
        fn = ctx.ntt_inv if args.kernel.endswith("inv") else ctx.ntt_fwd
        torch.cuda.synchronize()
        torch.cuda.profiler.start()  # ncu --profile-from-start off captures only these launches
        for _ in range(args.steps):
            fn(x, 0, NQ)
    else:
        from kunpbfv_b200.api import to_device
        import numpy as np
        sk = kb.SecretKey(ctx, SEED)
        sch = kb.BFVScheme(ctx, SEED)
        sch.addEncKey(sk)
        sch.addMultKey_23(sk)
        rng = np.random.default_rng(0)
        v = rng.integers(0, T, size=(args.pairs, ctx.N), dtype=np.uint64)
        c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(to_device(v))), enc_id=0)
        out = kb.Ciphertext(ctx, count=args.pairs)
        ctx.reserve(args.pairs)
        sch.mult_relin(c1, c1, out=out)  # loads the kernels and sizes the scratch
        torch.cuda.synchronize()
        torch.cuda.profiler.start()  # ncu --profile-from-start off captures only these launches
        for _ in range(args.steps):
            sch.mult_relin(c1, c1, out=out)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    print(json.dumps({"kernel_case": args.kernel, "steps": args.steps, "branches": ctx.tune_get("branches")}))


def c3_context(kb):
    """C3's parameter set from the library's own prime generator
    (kbfv_params_create: the largest 60-bit primes = 1 mod 2N, P first)."""
    return kb.BFVContext.from_bits(LOG_N, [60] * NQ, [60] * NP, T, dnum=1)


def c3_primes_oracle():
    """The same primes from the oracle's generator (CPU legs only)."""
    import oracle
    ps = oracle.primes_bits(1 << LOG_N, 60, NQ + NP)
    return ps[NP:NP + NQ], ps[:NP]


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples (every 20 ms) kept only while the timed region runs:
    mark() at its start and end."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.rows = []  # (arrival time, fields)
        self.window = [None, None]

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            if line.strip():
                self.rows.append((time.monotonic(), line.strip().split(",")))

    def mark(self):
        self.window[0 if self.window[0] is None else 1] = time.monotonic()

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.reader.join(timeout=5)

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        t0, t1 = self.window
        rows = [r for t, r in self.rows if t0 is None or t1 is None or t0 <= t <= t1]
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                for nm, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                pass
        if sm:
            out["sm_mhz"] = statistics.median(sm)
            out["sm_max_mhz"] = max(mx)
        out["reasons"] = sorted(reasons)
        out["samples"] = len(sm)
        return out


def dist_init(args):
    from kunpbfv_b200.replicas import init
    return init("nccl")


def barrier(world):
    from kunpbfv_b200.replicas import barrier as b
    b(world)


def max_over_ranks(world, v):
    from kunpbfv_b200.replicas import max_over_ranks as m
    return m(world, v)


# ---------------------------------------------------------------------------
# CPU legs: the oracle's restatement of the reference's multiply on the host
# cores. One method for the reference arm and for the cpu_baseline leg of our
# arm: a persistent pool of one thread per core; a step is every thread
# multiplying its own PAIRS_PER_THREAD pairs (the C oracle runs with the GIL
# released), the step ends when the last thread is done.
# ---------------------------------------------------------------------------
PAIRS_PER_THREAD = 2
CPU_STEP_BUDGET_S = 240.0  # the reference arm's timed steps stop here (stated in its line)


class CpuOracle:
    def __init__(self, seed_rng: int):
        import numpy as np

        import oracle
        qs, ps = c3_primes_oracle()
        self.o = o = oracle.Oracle(LOG_N, T, qs, ps, dnum=1)
        sk = o.keygen_secret(SEED)
        pk = o.keygen_public(SEED, sk)
        self.rlk = o.keygen_relin(SEED, sk)
        self.cores = os.cpu_count() or 1
        rng = np.random.default_rng(seed_rng)
        self.work = []  # per thread: its pairs
        for t in range(self.cores):
            pairs = []
            for k in range(PAIRS_PER_THREAD):
                i = t * PAIRS_PER_THREAD + k
                v1 = rng.integers(0, T, size=o.n, dtype=np.uint64)
                v2 = rng.integers(0, T, size=o.n, dtype=np.uint64)
                pairs.append((o.encrypt(SEED, 2 * i, pk, o.encode(v1)), o.encrypt(SEED, 2 * i + 1, pk, o.encode(v2))))
            self.work.append(pairs)
        from concurrent.futures import ThreadPoolExecutor
        self.pool = ThreadPoolExecutor(max_workers=self.cores)
        self.pairs_per_step = self.cores * PAIRS_PER_THREAD

    def _thread(self, t):
        for a, b in self.work[t]:
            self.o.mul_relin(a, b, self.rlk)

    def step(self) -> float:
        t0 = time.perf_counter()
        list(self.pool.map(self._thread, range(self.cores)))
        return time.perf_counter() - t0

    def run(self, steps: int, warmup: int, budget_s: float | None = None):
        """(median seconds per step, steps timed): at most `steps`, stopping
        early once the timed steps exceed budget_s."""
        for _ in range(max(1, warmup)):
            self.step()
        times = []
        for _ in range(max(1, steps)):
            times.append(self.step())
            if budget_s is not None and sum(times) >= budget_s:
                break
        return statistics.median(times), len(times)

    def close(self):
        self.pool.shutdown()

    def describe(self, per_step: float, steps: int) -> str:
        return (f"{self.pairs_per_step} pairs per step ({PAIRS_PER_THREAD} per thread on {self.cores} threads), "
                f"{steps} steps, median {per_step * 1e3:.1f} ms per step; C oracle restatement of the "
                f"reference's multiply (kunpBFV has no CPU path)")


def run_reference(args, world, rank):
    """The reference arm: the CPU oracle restatement on all host cores, on our
    arm's config, metric and unit; --steps steps after --warmup warm-up steps
    (stopping early only if the timed steps pass CPU_STEP_BUDGET_S)."""
    if rank != 0:
        return
    cpu = CpuOracle(seed_rng=0)
    per_step, steps = cpu.run(args.steps, args.warmup, budget_s=CPU_STEP_BUDGET_S)
    cpu.close()
    v = cpu.pairs_per_step / per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "ct/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": round(per_step * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": "mult+relin N=16384 7x60q+1p t=65537 dnum=1 (HPS tensor + hybrid key switch)",
                   "batch_pairs_per_step": cpu.pairs_per_step, "parallelism": f"{cpu.cores} host threads"},
        "steps_requested": args.steps,
        "cpu_baseline": {"value": round(v, 3), "unit": "ct/s", "cores": cpu.cores, "kind": "port",
                         "sample": cpu.describe(per_step, steps), "seal": seal_on_host()},
        "e2e": {"value": round(v, 3), "unit": "ct/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if steps < args.steps:
        line["steps_note"] = f"timed steps stopped at {CPU_STEP_BUDGET_S:.0f} s of CPU time"
    ref_gpu = reference_gpu_timing()
    if ref_gpu is not None:
        line["reference_gpu"] = ref_gpu
    print(json.dumps(line), flush=True)


def reference_gpu_timing(reps: int = 20):
    """kunpBFV's own GPU multiply, timed by the reference-kernel harness built
    from its sources (oracle/_ref/ref_harness), at its own parameter sets
    (logN 14 and 15): the genuine product as multAndEqual_23 runs it, one pair
    per call. None when the harness or a GPU is absent."""
    import subprocess
    import tempfile
    exe = os.path.join(os.path.dirname(os.path.abspath(__file__)), "oracle", "_ref", "ref_harness")
    try:
        import torch
        if not (os.path.exists(exe) and torch.cuda.is_available()):
            return None
    except Exception:
        return None
    out = {"form": "tensor (compute_t_QInv_c0c1c2) then the T-base key switch and add-back, one pair per call, "
                   "CUDA events over " + str(reps) + " calls",
           "caveat": "the reference's tensor step allocates device memory on every call and also computes its "
                     "secret-key shortcut product, which this sequence then discards"}
    for log_n in (14, 15):
        with tempfile.TemporaryDirectory() as d:
            try:
                r = subprocess.run([exe, str(log_n), d, "0", str(reps)], capture_output=True, text=True, timeout=300)
                lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
                if r.returncode != 0 or not lines:
                    out[f"logn{log_n}"] = {"error": (r.stderr or r.stdout)[-200:]}
                    continue
                t = json.loads(lines[-1])
                out[f"logn{log_n}"] = {"ms_per_mult": round(t["ms_per_mult"], 4),
                                       "ct_per_s": round(1e3 / t["ms_per_mult"], 1)}
            except Exception as e:  # report, keep the CPU line
                out[f"logn{log_n}"] = {"error": repr(e)[-200:]}
    return out


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
SEAL_GLOBS = ("/usr/local/include/SEAL-4.*", "/usr/include/SEAL-4.*", "/usr/local/lib/libseal*",
              "/usr/local/lib64/libseal*", "/usr/lib/libseal*", "/usr/lib/x86_64-linux-gnu/libseal*")


def seal_on_host():
    """Microsoft SEAL 4.x, the CPU BFV library the baseline would use if this
    host had it: the paths found (none on these hosts, so the C oracle on all
    host cores is the CPU baseline)."""
    import glob
    found = sorted(p for g in SEAL_GLOBS for p in glob.glob(g))
    return {"installed": bool(found), "checked": list(SEAL_GLOBS), "found": found[:4]}


def cpu_baseline_sample(seconds=12.0):
    """The CPU oracle on the host cores, by the reference arm's method, over a
    bounded sample (about `seconds` of timed steps)."""
    cpu = CpuOracle(seed_rng=1)
    est = cpu.step()  # warm-up step, also the estimate of one step
    per_step, steps = cpu.run(max(3, int(seconds / max(est, 1e-3))), 0, budget_s=seconds)
    cpu.close()
    return {"value": round(cpu.pairs_per_step / per_step, 3), "unit": "ct/s", "cores": cpu.cores, "kind": "port",
            "sample": cpu.describe(per_step, steps), "seal": seal_on_host()}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import kunpbfv_b200 as kb
    from kunpbfv_b200.api import to_device

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    ctx = c3_context(kb)
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    ctx.reserve(BATCH)
    # the autotuner's choice of the speed-only knobs for this parameter set and
    # batch (sub-batches and launch shapes of the multiply pipeline, host chunk,
    # NTT split); every choice gives identical results, and the tuner checks
    # that while it times them
    from kunpbfv_b200 import tune
    tuned = tune.autotune(ctx, sch, pairs=BATCH, cache_path=None)
    tuned = {k: tuned[k] for k in ("ntt_block_log", "host_chunk") + tune.PIPELINE_CHOICES if k in tuned}
    rng = np.random.default_rng(rank)
    v1 = rng.integers(0, T, size=(BATCH, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, T, size=(BATCH, ctx.N), dtype=np.uint64)
    from kunpbfv_b200.replicas import enc_id_base, job_rate
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(to_device(v1))), enc_id=enc_id_base(rank))
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(to_device(v2))), enc_id=enc_id_base(rank) + BATCH)
    out = kb.Ciphertext(ctx, count=BATCH)
    torch.cuda.synchronize()

    def step():
        sch.mult_relin(c1, c2, out=out, stream=stream)

    # correctness gate on the benchmark data itself
    with torch.cuda.stream(stream):
        step()
    torch.cuda.synchronize()
    dec = kb.api.to_host(ctx.decode(sch.decryptMsg(sk, out).mx_device)).reshape(BATCH, ctx.N)
    ok = bool(np.array_equal(dec, (v1 * v2) % T))
    budget = sch.noise_budget(sk, kb.Ciphertext(ctx, out.cipher_device.view(-1)[: 2 * NQ * ctx.N].clone()))

    graph = None
    if not args.no_graph:
        for _ in range(2):
            with torch.cuda.stream(stream):
                step()
        torch.cuda.synchronize()
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=stream):
            step()
        torch.cuda.synchronize()

    def run_step():
        if graph is not None:
            with torch.cuda.stream(stream):
                graph.replay()
        else:
            with torch.cuda.stream(stream):
                step()

    for _ in range(args.warmup):
        run_step()
    torch.cuda.synchronize()
    barrier(world)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier(world)
        clk.mark()
        ev0.record(stream)
        for _ in range(args.steps):
            run_step()
        ev1.record(stream)
        torch.cuda.synchronize()
        clk.mark()
    barrier(world)
    ms = ev0.elapsed_time(ev1) / args.steps
    ms = max_over_ranks(world, ms)
    value = job_rate(world, BATCH, ms)
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": "ct/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u64", "data": "synthetic (seeded XSalsa20 encryptions of uniform slots)",
        "config": {"workload": "mult+relin N=16384 7x60q+1p t=65537 dnum=1 (HPS tensor + hybrid key switch)",
                   "batch_pairs_per_gpu": BATCH, "cuda_graph": graph is not None,
                   "l2": "inputs 235 MB > 126 MB L2, no flush", "parallelism": f"replicas x{world}",
                   "tuned": tuned},
        "decrypt_exact": ok, "noise_budget_bits": round(budget, 2),
        # 9 kernels per sub-batch; batches of 2 x min_branch_pairs pairs and more run as `branches` sub-batches
        # (at least min_branch_pairs pairs each) on forked streams
        "gpu_launches": 9 * max(1, min(ctx.tune_get("branches"), BATCH // ctx.tune_get("min_branch_pairs")))
        * args.steps,
        "clocks": clk.summary(),
    }
    line["e2e"] = e2e_all_ranks(world, sch, c1, c2, out, stream)
    # the side measurements run on one GPU only (at N > 1 they would hold every
    # GPU of the job while rank 0 alone works)
    if rank == 0 and world == 1 and not args.skip_extras:
        try:
            line.update(extras(args, ctx, sch, c1, c2, out, stream, dev, ms))
        except Exception as e:  # report, keep the headline line
            line["extras_error"] = repr(e)
        try:
            sv = serving(args)
            line["serving"] = sv
            line["p50_ms"], line["p99_ms"] = sv["p50_ms"], sv["p99_ms"]
        except Exception as e:
            line["serving_error"] = repr(e)
        try:
            line["cpu_baseline"] = cpu_baseline_sample()
        except Exception as e:
            line["cpu_baseline_error"] = repr(e)
    if rank == 0:
        print(json.dumps(line), flush=True)


def per_op_native():
    """The per-call forms timed from native code over the C ABI
    (kunpbfv_b200/perop_bench: no interpreter between calls): the fused one-pair
    call, the same call replayed from a captured plan, the plain
    one-kernel-per-building-block form and the batched call, 64 pairs, same
    parameters as the headline."""
    from kunpbfv_b200 import build as kb_build
    exe = kb_build.PEROP_BIN
    if not os.path.exists(exe):
        return {"error": "perop_bench not built"}
    r = subprocess.run([exe, str(BATCH), "3"], capture_output=True, text=True, timeout=300)
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": (r.stderr or r.stdout)[-300:]}
    d = json.loads(lines[-1])
    d["form"] = ("C++ loop over the C ABI: fused = kbfv_mul_relin with count 1 per pair; plan = kbfv_plan_launch "
                 "of a one-pair plan (fixed buffers, one CUDA graph launch per call); plain = one kernel per "
                 "building block (about 25 launches and 10 device copies per pair) then kbfv_relinearize; "
                 "batched = one kbfv_mul_relin of all pairs (no CUDA graph)")
    return d


def c4_uneven(stream):
    """Config C4: N=32768, 14 x 60-bit q + 2 x 60-bit special primes, digits of
    5 primes (dnum 3); 16 pairs at 14, 13, 12 and 11 live primes (4 each) in one
    kbfv_mul_relin_levels call (one launch sequence over the mixed levels),
    against the same pairs as four batched calls, one per level."""
    import torch

    import kunpbfv_b200 as kb
    from kunpbfv_b200 import tune
    from kunpbfv_b200.api import VP, _ptr, lib
    ctx = kb.BFVContext.from_bits(15, [60] * 14, [60, 60], T, dnum=3)
    sk = kb.SecretKey(ctx, SEED)
    sch = kb.BFVScheme(ctx, SEED)
    sch.addMultKey_23(sk)
    pairs, outs = [], []
    for j in range(16):
        lv = ctx.at_level(14 - j % 4)
        pairs.append((kb.Ciphertext(lv, tune._random_pairs(lv, 1, 10 + j)),
                      kb.Ciphertext(lv, tune._random_pairs(lv, 1, 50 + j))))
        outs.append(kb.Ciphertext(lv, count=1))
    ms_one = time_cuda(lambda: sch.mult_relin_levels(pairs, outs=outs, stream=stream), stream, 10)
    one = [o.cipher_device.clone() for o in outs]
    groups = {}
    for j, (a, b) in enumerate(pairs):
        groups.setdefault(a.ctx.q_count, []).append(j)

    def per_level():
        for live, js in groups.items():
            n = len(js)
            A = (VP * n)(*[_ptr(pairs[j][0].cipher_device) for j in js])
            B = (VP * n)(*[_ptr(pairs[j][1].cipher_device) for j in js])
            O = (VP * n)(*[_ptr(outs[j].cipher_device) for j in js])
            lib().kbfv_mul_relin_batch(ctx.at_level(live).handle, _ptr(sch.rlk), A, B, O, n, stream.cuda_stream)

    ms_lv = time_cuda(per_level, stream, 10)
    same = all(torch.equal(x, o.cipher_device) for x, o in zip(one, outs))
    # the same mixed batch captured once and replayed as one CUDA graph launch
    plan = sch.mult_relin_levels_plan(pairs, outs)
    ms_graph = time_cuda(lambda: plan.launch(stream=stream), stream, 10)
    same = same and all(torch.equal(x, o.cipher_device) for x, o in zip(one, outs))
    plan.close()
    ctx.close()
    return {"pairs": 16, "levels": [14, 13, 12, 11], "one_call_ms": round(ms_one, 4),
            "one_call_ct_per_s": round(16 / ms_one * 1e3, 1), "one_graph_launch_ms": round(ms_graph, 4),
            "per_level_calls_ms": round(ms_lv, 4), "bit_identical": bool(same),
            "form": "kbfv_mul_relin_levels: one launch sequence over the mixed levels (9 pipeline stages, "
                    "each NTT a column pass + 2^12-point blocks at N=32768); one_graph_launch: the same "
                    "batch recorded by kbfv_plan_mul_relin_levels and replayed with one cudaGraphLaunch; "
                    "per_level_calls: four kbfv_mul_relin_batch calls on the level contexts, one after another"}


def step_roofline(ms_step, hbm_peak, peak_kind):
    """The headline step against the IMAD bound: every primitive of the 9-kernel
    pipeline counted per pair (kunpbfv_b200.roofline.pipeline_counts), each at
    the rate kbfv_probe_arith measures for it live on this GPU; and, from the
    committed ncu summary of the same kernel sources, the IMAD-pipe instructions
    per pair against the measured IMAD issue rate. Beside them the step's HBM
    rate (inputs, outputs and the key read once per launch)."""
    from kunpbfv_b200 import roofline as rl
    from kunpbfv_b200.api import probe_arith
    pc = rl.pipeline_counts(1 << LOG_N, LOG_N, NQ, NP, 1)
    rates = {k: probe_arith(kind) * 1e9 for k, kind in rl.PROBE_KIND.items()}
    floor_s = rl.arithmetic_floor_s(pc["counts"], rates)
    step_s = ms_step / 1e3
    n = 1 << LOG_N
    bytes_pair = 4 * NQ * n * 8 + 2 * NQ * n * 8 + 2 * (NQ + NP) * n * 8 // BATCH
    out = {"bound": "imad", "unit": "modmul/s",
           "modmuls_per_pair": pc["products"],
           "reductions_per_pair": pc["counts"]["b128"],
           "counts_per_pair": pc["counts"], "ntt_rows_per_pair": pc["ntt_rows"], "formula": pc["formula"],
           "achieved": round(pc["products"] * BATCH / step_s, 0),
           "peak": round(pc["products"] / floor_s, 0),
           "frac": round(floor_s * BATCH / step_s, 4),
           "floor_ms_per_step": round(floor_s * BATCH * 1e3, 4), "ms_per_step": round(ms_step, 4),
           "peak_source": "each class at its kbfv_probe_arith rate (register chains, no memory traffic): " +
                          ", ".join(f"{k} kind {v}" for k, v in rl.PROBE_KIND.items()),
           "rates_gops": {k: round(v / 1e9, 1) for k, v in rates.items()},
           "hbm": {"bytes_per_pair": bytes_pair, "achieved_gbs": round(bytes_pair * BATCH / step_s / 1e9, 1),
                   "frac": round(bytes_pair * BATCH / step_s / 1e9 / hbm_peak, 4), "peak_kind": peak_kind}}
    imad_peak = probe_arith(12) * 1e9 / 32  # warp-level IMAD instructions per second
    prof = rl.read_profile("mult_relin_imad_n16384.md")
    imad = {"unit": "warp inst/s", "peak": round(imad_peak, 0),
            "peak_source": "kbfv_probe_arith(12): dependent 32-bit multiply-adds, 8 chains per thread"}
    if rl.profile_matches(prof):
        ipp = float(prof["fmaheavy_warp_inst_per_pair"])
        imad.update({"inst_per_pair": ipp, "achieved": round(ipp * BATCH / step_s, 0),
                     "frac": round(ipp * BATCH / step_s / imad_peak, 4),
                     "source": "profiles/mult_relin_imad_n16384.md (sm__inst_executed_pipe_fmaheavy.sum)"})
    else:
        imad["note"] = "no ncu summary of the current kernel sources"
    out["imad"] = imad
    return out


def time_cuda(fn, stream, iters, warm=2):
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(iters):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / iters


def e2e_all_ranks(world, sch, c1, c2, out, stream, iters=10):
    """The headline metric end to end through the C ABI on every rank: each
    step copies that rank's 64 pairs in from page-locked host memory, multiplies
    them and copies the products back (kbfv_mul_relin_host: chunked copy-in /
    multiply / copy-out, the copies of one chunk overlapping the multiply of its
    neighbours). Timed with CUDA events on the calling stream between barriers;
    the job's time is the maximum over ranks."""
    import torch

    from kunpbfv_b200.replicas import job_rate
    h_a = c1.cipher_device.cpu().pin_memory()
    h_b = c2.cipher_device.cpu().pin_memory()
    h_o = torch.empty(out.cipher_device.shape, dtype=torch.int64, pin_memory=True)

    def e2e():
        sch.mult_relin_host(h_a, h_b, out=h_o, stream=stream, synchronize=False)

    for _ in range(2):
        e2e()
    torch.cuda.synchronize()
    barrier(world)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(iters):
        e2e()
    b.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(world, a.elapsed_time(b) / iters)
    if not torch.equal(h_o.view(-1), out.cipher_device.cpu().view(-1)):
        raise RuntimeError("host-memory multiply differs from the device multiply")
    return {"value": round(job_rate(world, BATCH, ms), 2), "unit": "ct/s",
            "h2d_bytes_per_step": 2 * h_a.numel() * 8 * world, "d2h_bytes_per_step": h_o.numel() * 8 * world,
            "ms_per_step": round(ms, 4),
            "form": "kbfv_mul_relin_host on every rank, chunked copy-in / multiply / copy-out"}


def extras(args, ctx, sch, c1, c2, out, stream, dev, ms_step):
    import torch

    import kunpbfv_b200 as kb
    res = {}
    N = ctx.N
    lq = 2 * NQ * N
    peak, peak_kind = load_peaks()

    # per-op form: one pair per call, eager launches
    a1 = [c1.cipher_device.view(-1)[i * lq:(i + 1) * lq] for i in range(BATCH)]
    b1 = [c2.cipher_device.view(-1)[i * lq:(i + 1) * lq] for i in range(BATCH)]
    o1 = [out.cipher_device.view(-1)[i * lq:(i + 1) * lq] for i in range(BATCH)]

    def per_op():
        with torch.cuda.stream(stream):
            for i in range(BATCH):
                sch.mult_relin_ptrs([a1[i].data_ptr()], [b1[i].data_ptr()], [o1[i].data_ptr()], stream=stream)

    ms_op = time_cuda(per_op, stream, 3)
    res["per_op"] = {"value": round(BATCH / (ms_op / 1e3), 2), "unit": "ct/s",
                     "form": "one pair per call through the Python binding (ctypes pointer arrays built per "
                             "call), 9-14 eager launches each (small launches split), no graph"}
    # the operation-by-operation form: tensor (kbfv_mul) then relinearisation
    # (kbfv_relinearize) as separate calls, one pair each (13 launches per pair)
    t3 = kb.Tensor3(ctx, count=1)
    one = kb.Ciphertext(ctx, count=1)
    ca = [kb.Ciphertext(ctx, a1[i]) for i in range(BATCH)]
    cb = [kb.Ciphertext(ctx, b1[i]) for i in range(BATCH)]

    def per_op_split():
        with torch.cuda.stream(stream):
            for i in range(BATCH):
                from kunpbfv_b200.api import _ptr, lib
                lib().kbfv_mul(ctx.handle, _ptr(ca[i].cipher_device), _ptr(cb[i].cipher_device), _ptr(t3.data), 1,
                               stream.cuda_stream)
                lib().kbfv_relinearize(ctx.handle, _ptr(sch.rlk), _ptr(t3.data), _ptr(one.cipher_device), 1,
                                       stream.cuda_stream)

    ms_split = time_cuda(per_op_split, stream, 3)
    res["per_op_split"] = {"value": round(BATCH / (ms_split / 1e3), 2), "unit": "ct/s",
                           "form": "one pair per call through the Python binding, multiply then relinearise as "
                                   "separate calls, no graph"}

    # the plain one-op-per-launch form: the HPS tensor composed from the
    # building-block entry points (INTT, base conversion, NTT, tensor, INTT,
    # scale-and-round, base conversion, NTT; one kernel each, about 20 launches
    # and 6 device copies per pair), then kbfv_relinearize; one pair per call
    from kunpbfv_b200.api import _ptr, lib
    NR, NQR = ctx.r_count, NQ + ctx.r_count
    L = lib()
    sp = stream.cuda_stream
    x4 = torch.empty(4, NQ, N, dtype=torch.int64, device=dev)
    r4 = torch.empty(4, NR, N, dtype=torch.int64, device=dev)
    qr = torch.empty(2, 2, NQR, N, dtype=torch.int64, device=dev)
    tz = torch.empty(3, NQR, N, dtype=torch.int64, device=dev)
    sr = torch.empty(3, NR, N, dtype=torch.int64, device=dev)
    d3 = torch.empty(3, NQ, N, dtype=torch.int64, device=dev)
    po = torch.empty(2, NQ, N, dtype=torch.int64, device=dev)

    def plain_pair(i):
        A, B = a1[i].view(2, NQ, N), b1[i].view(2, NQ, N)
        x4[:2].copy_(A)
        x4[2:].copy_(B)
        L.kbfv_ntt_inv(ctx.handle, _ptr(x4), 4 * NQ, 0, NQ, sp)
        L.kbfv_bconv_q_to_r(ctx.handle, _ptr(x4), _ptr(r4), 4, sp)
        L.kbfv_ntt_fwd(ctx.handle, _ptr(r4), 4 * NR, ctx.idx_r, NR, sp)
        qr[0, :, :NQ].copy_(A)
        qr[1, :, :NQ].copy_(B)
        qr[:, :, NQ:].copy_(r4.view(2, 2, NR, N))
        L.kbfv_tensor_qr(ctx.handle, _ptr(qr[0]), _ptr(qr[1]), _ptr(tz), 1, sp)
        for k in range(3):
            L.kbfv_ntt_inv(ctx.handle, _ptr(tz[k]), NQ, 0, NQ, sp)
            L.kbfv_ntt_inv(ctx.handle, _ptr(tz[k, NQ:]), NR, ctx.idx_r, NR, sp)
        L.kbfv_scale_round_qr_r(ctx.handle, _ptr(tz), _ptr(sr), 3, sp)
        L.kbfv_bconv_r_to_q(ctx.handle, _ptr(sr), _ptr(d3), 3, sp)
        L.kbfv_ntt_fwd(ctx.handle, _ptr(d3), 3 * NQ, 0, NQ, sp)
        L.kbfv_relinearize(ctx.handle, _ptr(sch.rlk), _ptr(d3), _ptr(po), 1, sp)

    def per_op_plain():
        with torch.cuda.stream(stream):
            for i in range(BATCH):
                plain_pair(i)

    with torch.cuda.stream(stream):
        plain_pair(0)
    torch.cuda.synchronize()
    if not torch.equal(po.view(-1), o1[0]):
        raise RuntimeError("the building-block multiply differs from the fused one")
    ms_plain = time_cuda(per_op_plain, stream, 3)
    res["per_op_plain"] = {"value": round(BATCH / (ms_plain / 1e3), 2), "unit": "ct/s",
                           "form": "one pair per call through the Python binding, one kernel per building block "
                                   "(about 25 launches and 6 device copies per pair), no graph"}

    # this engine at the reference's own parameter sets (logN 14, 15) with the
    # reference's key switch over the T base: one pair per call (the form the
    # reference runs) and a 64-pair batch
    from kunpbfv_b200 import tune
    refp = {}
    for log_n in (14, 15):
        rctx = kb.reference_context(log_n)
        rsk = kb.SecretKey(rctx, SEED)
        rs = kb.BFVScheme(rctx, SEED, relin="klss")
        rs.addMultKey_23(rsk)
        ra = kb.Ciphertext(rctx, tune._random_pairs(rctx, 64, 7))
        rb = kb.Ciphertext(rctx, tune._random_pairs(rctx, 64, 8))
        ro = kb.Ciphertext(rctx, count=64)
        lq_r = 2 * rctx.q_count * rctx.N
        a1r = [kb.Ciphertext(rctx, ra.cipher_device.view(-1)[i * lq_r:(i + 1) * lq_r]) for i in range(8)]
        b1r = [kb.Ciphertext(rctx, rb.cipher_device.view(-1)[i * lq_r:(i + 1) * lq_r]) for i in range(8)]
        o1r = [kb.Ciphertext(rctx, ro.cipher_device.view(-1)[i * lq_r:(i + 1) * lq_r]) for i in range(8)]

        def one_by_one():
            for i in range(8):
                rs.mult_relin(a1r[i], b1r[i], out=o1r[i], stream=stream)

        ms1 = time_cuda(one_by_one, stream, 3) / 8
        msb = time_cuda(lambda: rs.mult_relin(ra, rb, out=ro, stream=stream), stream, 3) / 64
        refp[f"logn{log_n}"] = {"q": rctx.q_count, "p": rctx.p_count, "t_primes": rctx.t_count,
                                "per_op_ms_per_mult": round(ms1, 4), "per_op_ct_per_s": round(1e3 / ms1, 1),
                                "batched_ms_per_mult": round(msb, 4), "batched_ct_per_s": round(1e3 / msb, 1)}
        del ra, rb, ro, a1r, b1r, o1r, rs, rsk
        rctx.close()
    res["reference_params"] = dict(refp, form="T-base key switch (bit-exact with the reference's genuine "
                                              "multiply); per-op: one pair per call; batched: 64 pairs per call")

    res["per_op_native"] = per_op_native()
    res["c4_uneven"] = c4_uneven(stream)

    # dominant kernel (forward NTT block kernel, N=16384) timed alone on the
    # same row count as the pipeline's largest forward-NTT launch
    # (the built-in one-block-per-row shape whatever split the tuner chose)
    rows = BATCH * 4 * (NQ + 1)
    x = torch.randint(0, 1 << 59, (rows, N), dtype=torch.int64, device=dev)
    keep_split = ctx.tune_get("ntt_block_log")
    ctx.tune_set("ntt_block_log", 0)
    ms_ntt = time_cuda(lambda: ctx.ntt_fwd(x, ctx.idx_r, NQ + 1, stream=stream), stream, 10)
    ctx.tune_set("ntt_block_log", keep_split)
    alg = 16 * N * rows + 16 * N * (NQ + 1)
    ach = alg / (ms_ntt / 1e3) / 1e9
    bfly = rows * (N // 2) * LOG_N
    # DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of this launch at
    # 2048 rows, from the committed ncu summary of the same kernel sources
    from kunpbfv_b200 import roofline as rl
    prof = rl.read_profile("ntt_fwd_block_n16384.md")
    traffic = None
    if rl.profile_matches(prof) and rows == int(prof.get("traffic_rows", 0)):
        traffic = int(prof["traffic_bytes"])
    res["roofline"] = {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                       "frac": round(ach / peak, 4), "traffic": traffic,
                       "traffic_source": ("profiles/ntt_fwd_block_n16384.md (ncu capture of these kernel sources)"
                                          if traffic is not None else "no ncu summary of the current kernel sources"),
                       "kernel": f"ntt_fwd_block_kernel<14> on {rows} rows ({peak_kind} peak)",
                       "ms_per_launch": round(ms_ntt, 4),
                       "algorithmic_bytes": alg,
                       "note": "60-bit Shoup butterflies are bound by the IMAD pipe, not HBM: ncu shows "
                               "fmaheavy busy ~66% of elapsed with math-pipe throttling the top stall",
                       "butterflies_per_s": round(bfly / (ms_ntt / 1e3), 0)}
    # the bound that does apply: the butterfly issue rate of this GPU, measured
    # live by the register-chain probe (kbfv_probe_arith kind 11: the kernels'
    # butterfly, no memory traffic)
    from kunpbfv_b200.api import probe_arith
    bfly_peak = probe_arith(11) * 1e9
    res["roofline"]["arith"] = {"bound": "imad", "unit": "butterflies/s",
                                "achieved": round(bfly / (ms_ntt / 1e3), 0), "peak": round(bfly_peak, 0),
                                "frac": round(bfly / (ms_ntt / 1e3) / bfly_peak, 4),
                                "peak_source": "kbfv_probe_arith(11): the kernels' 60-bit forward butterfly in register chains"}
    del x
    res["roofline"]["step"] = step_roofline(ms_step, peak, peak_kind)

    # standalone NTT, N=65536, 32 primes x 64 polynomials (1 GiB)
    ctx2 = kb.BFVContext.from_bits(16, [60] * 32, [60], 786433, dnum=1)
    mods = torch.tensor(ctx2.q, dtype=torch.int64, device=dev)
    y = torch.randint(0, 1 << 62, (64, 32, 1 << 16), dtype=torch.int64, device=dev)
    y = torch.remainder(y, mods.view(1, 32, 1))
    # the autotuner's radix split for this ring (column pass + 2^v-point blocks)
    from kunpbfv_b200 import tune
    split = tune.tune_ntt(ctx2, rows=2048)
    ctx2.tune_set("ntt_block_log", split["ntt_block_log"])
    ms_f = time_cuda(lambda: ctx2.ntt_fwd(y, 0, 32, stream=stream), stream, 5)
    ms_i = time_cuda(lambda: ctx2.ntt_inv(y, 0, 32, stream=stream), stream, 5)
    alg2 = 16 * 65536 * 2048 + 16 * 65536 * 32
    res["ntt_n65536"] = {"fwd_gbs": round(alg2 / (ms_f / 1e3) / 1e9, 1),
                         "inv_gbs": round(alg2 / (ms_i / 1e3) / 1e9, 1),
                         "fwd_ms": round(ms_f, 4), "inv_ms": round(ms_i, 4),
                         "frac_of_peak_fwd": round(alg2 / (ms_f / 1e3) / 1e9 / peak, 4),
                         "rows": 2048, "algorithmic_bytes": alg2,
                         "split": {"block_log": split["ntt_block_log"], "tuner_ms_fwd_inv": split["ms"]}}
    del y
    ctx2.close()
    return res


# Serving rings: one per ring degree, one key-switch digit per ciphertext
# prime where the special prime is a single prime (noise stays small over
# chains), and the most multiplies per chain each ring's noise budget allows.
SERVE_RINGS = [  # (log_n, q bits, p bits, dnum, max multiplies per chain)
    (12, [36, 36], [37], 2, 1),
    (13, [50, 50, 50], [52], 3, 3),
    (14, [60] * 7, [60], 7, 4),
    (15, [60] * 14, [60, 60], 3, 4),
]


def serving(args):
    """Open-loop Poisson streams of 1-4 op chains (mult+relin / add) over
    N = 4096, 8192, 16384, 32768 through the request server; every result is
    decrypted and checked exactly. Latency is submit-to-decrypted-result."""
    import kunpbfv_b200 as kb
    from kunpbfv_b200.serve import Ring, Server, make_workload, run_open_loop
    rings = [Ring.make(kb.BFVContext.from_bits(ln, qb, pb, T, dnum=d), bytes([40 + i]) * 32)
             for i, (ln, qb, pb, d, _) in enumerate(SERVE_RINGS)]
    w = make_workload(rings, 64, [m for *_, m in SERVE_RINGS], seed=11)
    points = []
    with Server(rings, hbm_budget_bytes=24 << 30, max_batch=64, pinned_bytes=2 << 30) as srv:
        run_open_loop(srv, w, rate=200.0, duration_s=0.5, seed=99)  # warm-up
        for i, rate in enumerate(float(r) for r in args.serve_rates.split(",")):
            window = max(args.serve_seconds, args.serve_requests / rate)
            pt = run_open_loop(srv, w, rate=rate, duration_s=window, seed=100 + i,
                               enc_base=(i + 1) << 36)
            points.append(pt)
        st = srv.stats()
    ok = [p for p in points if p["throughput"] >= 0.9 * p["offered"] / p["submit_span_s"]]
    head = ok[-1] if ok else points[0]
    return {
        "rings": [{"N": 1 << ln, "q_bits": qb, "p_bits": pb, "dnum": d, "max_mul": m}
                  for ln, qb, pb, d, m in SERVE_RINGS],
        "chains": "1-4 ops, 60% multiply (capped per ring), fresh seeded encryptions",
        "points": points,
        "all_decryptions_exact": all(p["wrong"] == 0 and p["errors"] == 0 for p in points),
        "headline_rate": head["rate"], "p50_ms": head["p50_ms"], "p99_ms": head["p99_ms"],
        "throughput": head["throughput"],
        "server": {"iterations": st["iterations"], "mul_launches": st["mul_launches"], "mul_ops": st["mul_ops"],
                   "add_ops": st["add_ops"], "device_bytes_peak": st["bytes_peak"]},
    }


def main():
    args = parse()
    if args.kernel:
        run_kernel_case(args)
        return
    if args.serving_only:
        print(json.dumps(serving(args)), flush=True)
        return
    world, rank, local = dist_init(args)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        from kunpbfv_b200.replicas import finish
        finish(world)


if __name__ == "__main__":
    main()
