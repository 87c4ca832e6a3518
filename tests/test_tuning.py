"""Autotuner: the tuning cache on the host (CPU), and on the GPU the tuner's
choice applied to the context, bit-exact output under every tuning it
leaves, and the cache round trip."""
import ctypes
import os

import pytest
import torch

from tests.cases import sorted_lines


def test_tuning_cache_roundtrip(tmp_path):
    from unitigcoarsening_b200 import api
    path = str(tmp_path / "tune.json")
    assert api.load_tuning(path, "x") is None
    t = {"tile_capacity": 2048, "tile_threads": 256, "bucket_bits": 0, "load_factor_pct": 300,
         "contract_method": 0, "warp_capacity": 128, "bucket_fill": 4}
    api.store_tuning(path, "B200|k31|2^24", t, 1.5)
    api.store_tuning(path, "B200|k63|2^24", dict(t, warp_capacity=64), 2.5)
    assert api.load_tuning(path, "B200|k31|2^24") == t
    assert api.load_tuning(path, "B200|k63|2^24")["warp_capacity"] == 64
    assert api.load_tuning(path, "B200|k31|2^25") is None


def test_tuning_struct_matches_header():
    """The ctypes mirror of uc_tuning has the header's fields in order."""
    import re
    from unitigcoarsening_b200 import api
    src = open(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "uc.h")).read()
    body = re.search(r"typedef struct uc_tuning \{(.*?)\} uc_tuning;", src, re.S).group(1)
    names = re.findall(r"uint32_t (\w+);", body)
    assert names == [n for n, _ in api.Tuning._fields_]
    assert ctypes.sizeof(api.Tuning) == 4 * len(names)


@pytest.mark.gpu
def test_autotune_applies_choice_and_stays_exact(comp, oracle, tmp_path):
    from unitigcoarsening_b200 import synth
    text = synth.make_text(synth.scale_plain(length=2_000_000, seed=21), 31).numpy().tobytes()
    d = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
    want = sorted_lines(oracle.compact(text, 31)[0])
    cache = str(tmp_path / "tune.json")
    try:
        res = comp.autotune(d, 31, 8, reps=2, max_ms=4000, cache=cache)
        assert not res["cached"] and res["trials"] >= 2 and res["ms"] > 0
        cur = comp.get_tuning()
        for f in cur:
            assert cur[f] == res[f]
        got = sorted_lines(comp.compact(d, 31, 8).cpu().numpy().tobytes())
        assert got == want
        # second call: from the cache, nothing timed
        comp.set_tuning(tile_capacity=0, tile_threads=0, load_factor_pct=0, warp_capacity=0, bucket_fill=0,
                        contract_method=0)
        again = comp.autotune(d, 31, 8, cache=cache)
        assert again["cached"]
        assert {f: again[f] for f in cur} == cur
    finally:
        comp.set_tuning(tile_capacity=0, tile_threads=0, bucket_bits=0, load_factor_pct=0, contract_method=0,
                        warp_capacity=0, bucket_fill=0)


@pytest.mark.gpu
@pytest.mark.parametrize("fill", [1, 2, 32, 64])
def test_bucket_fill_keeps_output(comp, oracle, fill):
    from unitigcoarsening_b200 import synth
    text = synth.make_text(synth.scale_plain(length=500_000, seed=22), 31).numpy().tobytes()
    want = sorted_lines(oracle.compact(text, 31)[0])
    comp.set_tuning(bucket_fill=fill)
    try:
        d = torch.frombuffer(bytearray(text), dtype=torch.uint8).cuda()
        got = sorted_lines(comp.compact(d, 31, 8).cpu().numpy().tobytes())
    finally:
        comp.set_tuning(bucket_fill=0)
    assert got == want


@pytest.mark.gpu
@pytest.mark.parametrize("field,value", [("tile_threads", 1024), ("tile_capacity", 128), ("load_factor_pct", 100),
                                         ("warp_capacity", 48), ("bucket_fill", 65), ("bucket_bits", 26)])
def test_set_tuning_rejects_out_of_range(comp, field, value):
    from unitigcoarsening_b200 import UCError
    before = comp.get_tuning()
    with pytest.raises(UCError):
        comp.set_tuning(**{field: value})
    assert comp.get_tuning() == before
