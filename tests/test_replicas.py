"""The multi-GPU path's host logic on CPU: two gloo ranks, each a replica over
its own pairs (oracle multiplies), timed as the maximum over ranks. The union
of the ranks' results equals one process doing all the pairs."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from tests.params import T65537, small_primes

PAIRS_PER_RANK = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _inputs(o, key, pk, rank):
    from kunpbfv_b200.replicas import enc_id_base
    rng = np.random.default_rng(100 + rank)
    out = []
    for i in range(PAIRS_PER_RANK):
        v1 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
        v2 = rng.integers(0, T65537, size=o.n, dtype=np.uint64)
        base = enc_id_base(rank) + 2 * i
        out.append((v1, v2, o.encrypt(key, base, pk, o.encode(v1)), o.encrypt(key, base + 1, pk, o.encode(v2))))
    return out


def _rank_main(rank, world, port, results):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import oracle
    from kunpbfv_b200 import replicas
    w, r, _ = replicas.init("gloo", timeout_s=60)
    assert (w, r) == (world, rank)
    qs, ps = small_primes(10, 2, 1, 40)
    o = oracle.Oracle(10, T65537, qs, ps)
    key = b"\x0b" * 32
    sk = o.keygen_secret(key)
    pk, rlk = o.keygen_public(key, sk), o.keygen_relin(key, sk)
    replicas.barrier(w)
    outs = []
    for v1, v2, c1, c2 in _inputs(o, key, pk, rank):
        c3 = o.mul_relin(c1, c2, rlk)
        assert np.array_equal(o.decode(o.decrypt(sk, c3)), (v1 * v2) % T65537)
        outs.append(c3)
    ms = 10.0 * (rank + 1)  # a rank-dependent step time
    ms_max = replicas.max_over_ranks(w, ms)
    results[rank] = (ms_max, replicas.job_rate(w, PAIRS_PER_RANK, ms_max), [x.tobytes() for x in outs])
    replicas.finish(w)


def test_two_gloo_ranks_replicas():
    world = 2
    port = _free_port()
    with mp.Manager() as man:
        results = man.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, results)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=240)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        res = dict(results)
    assert res[0][0] == res[1][0] == 20.0  # the slowest rank
    assert res[0][1] == pytest.approx(world * PAIRS_PER_RANK / 0.020)
    # one process doing both ranks' pairs gives the same ciphertexts
    import oracle
    qs, ps = small_primes(10, 2, 1, 40)
    o = oracle.Oracle(10, T65537, qs, ps)
    key = b"\x0b" * 32
    sk = o.keygen_secret(key)
    pk, rlk = o.keygen_public(key, sk), o.keygen_relin(key, sk)
    for rank in range(world):
        for i, (v1, v2, c1, c2) in enumerate(_inputs(o, key, pk, rank)):
            assert o.mul_relin(c1, c2, rlk).tobytes() == res[rank][2][i]


def test_single_process_defaults():
    from kunpbfv_b200 import replicas
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        os.environ.pop(k, None)
    assert replicas.world_from_env() == (1, 0, 0)
    assert replicas.max_over_ranks(1, 3.5) == 3.5
    assert replicas.enc_id_base(3) == 3 * replicas.ENC_ID_STRIDE
