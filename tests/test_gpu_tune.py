"""The tuning knobs and the autotuner (kunpbfv_b200.tune): every radix split of
the standalone NTT on rings of 2^13-2^16 points gives the oracle's transform, every
sub-batch count and host chunk gives the same product, and the tuner applies
and caches its choice."""
import numpy as np
import pytest

from tests.gpu_util import dev, host, rand_rows, small_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_n", [13, 14, 15, 16])
def test_ntt_splits_match_oracle(log_n):
    ctx, orc = small_pair(log_n=log_n, nq=2, np_=1, bits=60)
    rows = 6
    x = np.concatenate([rand_rows(orc, [0, 1], ctx.N, seed=s) for s in range(rows // 2)])
    want = np.concatenate([orc.ntt_fwd(r % 2, x[r:r + 1]) for r in range(rows)])
    try:
        for v in (0, 12, 13, 14):
            ctx.tune_set("ntt_block_log", v)
            assert ctx.tune_get("ntt_block_log") == v
            y = dev(x)
            ctx.ntt_fwd(y, 0, 2)
            assert np.array_equal(host(y), want), v
            ctx.ntt_inv(y, 0, 2)
            assert np.array_equal(host(y), x), v
    finally:
        ctx.tune_set("ntt_block_log", 0)


def test_knob_bounds():
    import kunpbfv_b200 as kb
    ctx, _ = small_pair()
    for knob, bad in (("ntt_block_log", 11), ("ntt_block_log", 15), ("ntt_block_log", 1), ("branches", 0),
                      ("branches", 5), ("host_chunk", -1), ("host_chunk", 129)):
        with pytest.raises(kb.KbfvError):
            ctx.tune_set(knob, bad)
    assert ctx.tune_get("branches") == 2 and ctx.tune_get("host_chunk") == 0
    assert ctx.tune_get("ntt_block_log") == 0


def test_autotune_applies_and_caches(tmp_path):
    import kunpbfv_b200 as kb
    from kunpbfv_b200 import tune
    ctx = kb.BFVContext.from_bits(13, [50, 50, 50], [52], 65537, dnum=3)
    sk = kb.SecretKey(ctx, b"\x21" * 32)
    sch = kb.BFVScheme(ctx, b"\x22" * 32)
    sch.addMultKey_23(sk)
    cache = str(tmp_path / "tune.json")
    got = tune.autotune(ctx, sch, pairs=32, cache_path=cache)
    assert not got["cached"]
    assert got["branches"] in tune.BRANCHES and got["host_chunk"] in tune.HOST_CHUNKS
    assert ctx.tune_get("branches") == got["branches"]
    assert ctx.tune_get("host_chunk") == got["host_chunk"]
    assert set(got["branches_ms"]) == {str(b) for b in tune.BRANCHES}
    for k in ("bconv_threads", "bconv_cpt", "k5_threads", "split_rows", "k5_fused_pairs", "fuse_q2r_pairs",
              "split_rows_alone", "min_branch_pairs"):
        assert ctx.tune_get(k) == got[k], k
    assert set(got["fuse_q2r_pairs_ms"]) == {str(v) for v in tune.FUSE_Q2R_PAIRS}
    # a fresh context of the same parameters takes the cached choice without timing
    ctx2 = kb.BFVContext.from_bits(13, [50, 50, 50], [52], 65537, dnum=3)
    hit = tune.autotune(ctx2, None, pairs=32, cache_path=cache)
    assert hit["cached"] and ctx2.tune_get("branches") == got["branches"]
    assert ctx2.tune_get("fuse_q2r_pairs") == got["fuse_q2r_pairs"]
    assert tune.apply_cached(ctx2, pairs=32, cache_path=cache)["host_chunk"] == got["host_chunk"]


def test_autotune_ntt_split_large_ring(tmp_path):
    import kunpbfv_b200 as kb
    from kunpbfv_b200 import tune
    ctx, _ = small_pair(log_n=16, nq=2, np_=1, bits=60)
    got = tune.autotune(ctx, None, cache_path=str(tmp_path / "t.json"), ntt_rows=64)
    assert got["ntt_block_log"] in tune.NTT_BLOCK_LOGS
    assert ctx.tune_get("ntt_block_log") == got["ntt_block_log"]
    assert set(got["ntt_ms"]) == {"0", "12", "13", "14"}
    ctx.tune_set("ntt_block_log", 0)


def test_host_chunk_knob_drives_the_default_chunk():
    """chunk_pairs = 0 takes the context's host_chunk knob; every chunk gives
    the product of the device multiply."""
    import torch

    import kunpbfv_b200 as kb
    from kunpbfv_b200 import tune
    ctx = kb.BFVContext.from_bits(13, [50, 50, 50], [52], 65537, dnum=3)
    sk = kb.SecretKey(ctx, b"\x31" * 32)
    sch = kb.BFVScheme(ctx, b"\x32" * 32)
    sch.addMultKey_23(sk)
    a = tune._random_pairs(ctx, 11, 5)
    b = tune._random_pairs(ctx, 11, 6)
    want = sch.mult_relin(kb.Ciphertext(ctx, a), kb.Ciphertext(ctx, b)).cipher_device.cpu()
    ha, hb = a.cpu().pin_memory(), b.cpu().pin_memory()
    try:
        for knob in (0, 1, 3, 128):
            ctx.tune_set("host_chunk", knob)
            out = sch.mult_relin_host(ha, hb, chunk_pairs=0)
            assert torch.equal(out.view(-1), want.view(-1)), knob
    finally:
        ctx.tune_set("host_chunk", 0)


@pytest.mark.parametrize("knob,values", [("bconv_threads", (64, 128, 256, 512)), ("k5_threads", (64, 128, 256)),
                                         ("split_rows", (0, 48, 1 << 20)), ("k5_fused_pairs", (0, 2, 4)),
                                         ("bconv_cpt", (1, 2)), ("fuse_q2r_pairs", (128, 0, 1)),
                                         ("l2_prefetch", (0, 1)), ("split_rows_alone", (0, 48, 148, 1 << 20)),
                                         ("min_branch_pairs", (1, 2, 8))])
def test_pipeline_shapes_keep_the_product(knob, values):
    """Every launch shape of the multiply pipeline gives the oracle's product
    (N=16384, 7 + 1 primes; 3 pairs: K5 fused or split by k5_fused_pairs,
    112-row transforms split or not by split_rows)."""
    import kunpbfv_b200 as kb
    import oracle
    from tests.gpu_util import c3_pair
    ctx, orc = c3_pair()
    seed = b"\x44" * 32
    sk = kb.SecretKey(ctx, seed)
    sch = kb.BFVScheme(ctx, seed)
    sch.addEncKey(sk)
    sch.addMultKey_23(sk)
    rng = np.random.default_rng(12)
    v1 = rng.integers(0, 65537, size=(3, ctx.N), dtype=np.uint64)
    v2 = rng.integers(0, 65537, size=(3, ctx.N), dtype=np.uint64)
    c1 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v1))), enc_id=5)
    c2 = sch.encryptMsg(kb.Plaintext(ctx, ctx.encode(dev(v2))), enc_id=9)
    osk = orc.keygen_secret(seed)
    orlk = orc.keygen_relin(seed, osk)
    h1 = host(c1.cipher_device).reshape(3, 2, 7, ctx.N)
    h2 = host(c2.cipher_device).reshape(3, 2, 7, ctx.N)
    want = np.stack([orc.mul_relin(h1[i], h2[i], orlk) for i in range(3)])
    keep = ctx.tune_get(knob)
    try:
        for v in values:
            ctx.tune_set(knob, v)
            assert ctx.tune_get(knob) == v
            got = host(sch.mult_relin(c1, c2).cipher_device).reshape(want.shape)
            assert np.array_equal(got, want), (knob, v)
    finally:
        ctx.tune_set(knob, keep)


def test_pipeline_knob_bounds_and_levels():
    import kunpbfv_b200 as kb
    ctx = kb.BFVContext.from_bits(13, [50, 50, 50], [52], 65537, dnum=3)
    for knob, bad in (("bconv_threads", 100), ("bconv_threads", 1024), ("k5_threads", 512), ("k5_threads", 32),
                      ("split_rows", -1), ("k5_fused_pairs", 129), ("fuse_q2r_pairs", 129), ("bconv_cpt", 3),
                      ("l2_prefetch", 2), ("split_rows_alone", -1), ("min_branch_pairs", 0),
                      ("min_branch_pairs", 65)):
        with pytest.raises(kb.KbfvError):
            ctx.tune_set(knob, bad)
    assert (ctx.tune_get("split_rows"), ctx.tune_get("bconv_threads"), ctx.tune_get("k5_threads"),
            ctx.tune_get("k5_fused_pairs"), ctx.tune_get("bconv_cpt"), ctx.tune_get("fuse_q2r_pairs"),
            ctx.tune_get("l2_prefetch"), ctx.tune_get("split_rows_alone"),
            ctx.tune_get("min_branch_pairs")) == (48, 256, 128, 2, 2, 1, 1, 148, 1)
    lv = ctx.at_level(2)
    ctx.tune_set("k5_threads", 64)
    assert lv.tune_get("k5_threads") == 64  # levels follow the top level's knobs
    assert ctx.at_level(1).tune_get("k5_threads") == 64  # and so do levels made later


@pytest.mark.parametrize("log_n,q_bits,p_bits,dnum,pairs,split_rows", [
    (14, [60] * 7, [60], 1, 5, 48),        # whole-ring blocks (140- and 160-row transforms)
    (14, [60] * 7, [60], 1, 1, 48),        # per-call size: column pass + 2^12 blocks, scale folded in the column pass
    (14, [60] * 7, [60], 1, 3, 1 << 20),   # every transform split
    (13, [50] * 3, [52], 3, 4, 48),        # 2^13 blocks, three digits
    (15, [55] * 10, [58] * 2, 5, 2, 48),   # 2^15 column pass + blocks; 10 primes (the 16-prime bucket)
    (16, [58] * 18, [60] * 2, 3, 1, 48),   # 2^16; 18 primes (the 24-prime bucket)
])
def test_fused_q2r_keeps_the_product(log_n, q_bits, p_bits, dnum, pairs, split_rows):
    """The Q -> R base extension inside the NTT over R gives the products of
    the separate base-conversion launch (itself pinned to the oracle by the
    multiply tests), for mult_relin and for the tensor alone, on every
    transform shape: whole-ring blocks, the split at N=2^14, the 2^15/2^16
    column passes (the scaled last inverse stage then runs in the column
    kernel) and the prime-count buckets."""
    import torch

    import kunpbfv_b200 as kb
    from kunpbfv_b200 import tune
    ctx = kb.BFVContext.from_bits(log_n, q_bits, p_bits, 786433 if log_n == 16 else 65537, dnum=dnum)
    sk = kb.SecretKey(ctx, b"\x51" * 32)
    sch = kb.BFVScheme(ctx, b"\x52" * 32)
    sch.addMultKey_23(sk)
    c1 = kb.Ciphertext(ctx, tune._random_pairs(ctx, pairs, 21))
    c2 = kb.Ciphertext(ctx, tune._random_pairs(ctx, pairs, 22))
    keep = (ctx.tune_get("fuse_q2r_pairs"), ctx.tune_get("split_rows"))
    try:
        ctx.tune_set("split_rows", split_rows)
        got = {}
        for fuse in (0, 1):
            ctx.tune_set("fuse_q2r_pairs", 128 * fuse)
            got[fuse] = (sch.mult_relin(c1, c2).cipher_device.clone(), sch.mult(c1, c2).data.clone())
        torch.cuda.synchronize()
        assert torch.equal(got[0][0], got[1][0]), "mult_relin"
        assert torch.equal(got[0][1], got[1][1]), "mult (tensor)"
    finally:
        ctx.tune_set("fuse_q2r_pairs", keep[0])
        ctx.tune_set("split_rows", keep[1])
