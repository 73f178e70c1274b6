"""The autotuner's cache (warpjq_b200/tune.py), without a GPU: keys group
inputs by device, query and line-length class; the cache file round-trips
and a damaged one reads as empty."""

import os

from warpjq_b200 import tune


def test_shape_key_groups_line_lengths_by_power_of_two():
    a = tune.shape_key("B200", "count", b"x" * 199 + b"\n")
    b = tune.shape_key("B200", "count", b"y" * 239 + b"\n")
    c = tune.shape_key("B200", "count", b"z" * 99 + b"\n")
    assert a == b != c
    assert tune.shape_key("B200", "sum(.a)", b"x\n") != tune.shape_key("B200", "count", b"x\n")
    assert tune.shape_key("B200", "count", b"x\n", "1-2") != tune.shape_key("B200", "count", b"x\n", "1-3")
    assert tune.library_id() != "unbuilt"  # the tests run against a built library


def test_cache_round_trip_and_damage(tmp_path):
    p = os.path.join(tmp_path, "sub", "tune.json")
    assert tune.load_cache(p) == {}
    tune.save_cache(p, {"k": {"tile": 6400, "halo": 512, "group_keys": None}})
    assert tune.load_cache(p)["k"]["tile"] == 6400
    with open(p, "w") as f:
        f.write("{not json")
    assert tune.load_cache(p) == {}
