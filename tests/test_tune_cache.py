"""Host side of the autotuner: cache keys and the JSON cache file (no GPU)."""
import json

from kunpbfv_b200 import tune


def test_cache_key_names_device_and_parameters():
    k = tune.cache_key("NVIDIA B200", 14, 7, 1, 1, 64)
    assert k == "NVIDIA B200|logn=14|q=7|p=1|dnum=1|pairs=64"
    assert k != tune.cache_key("NVIDIA B200", 14, 7, 1, 1, 32)


def test_cache_roundtrip_and_merge(tmp_path):
    path = str(tmp_path / "sub" / "tune.json")
    assert tune.load_cache(path) == {}
    tune.save_cache({"a": {"branches": 2}}, path)
    tune.save_cache({"b": {"ntt_block_log": 13}}, path)
    data = tune.load_cache(path)
    assert data == {"a": {"branches": 2}, "b": {"ntt_block_log": 13}}
    with open(path) as f:
        assert json.load(f) == data


def test_corrupt_cache_reads_as_empty(tmp_path):
    path = tmp_path / "tune.json"
    path.write_text("{not json")
    assert tune.load_cache(str(path)) == {}


class _FakeCtx:
    def __init__(self):
        self.set = {}

    def tune_set(self, knob, value):
        self.set[knob] = value


def test_apply_choice_sets_known_knobs_only():
    ctx = _FakeCtx()
    tune.apply_choice(ctx, {"branches": 3, "host_chunk": 8, "ntt_ms": {"12": 1.0}, "cached": True})
    assert ctx.set == {"branches": 3, "host_chunk": 8}
