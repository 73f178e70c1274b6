"""Multi-GPU merge fed by real device runs: the input is cut into byte
ranges as for several ranks, each range is scanned on the device
(shard.device_partial), and the rank-order merge must render the oracle's
output for the whole input.  One process, one GPU, the ranges run one after
another (no process group is needed to test the partials and the merge)."""

import pytest

import warpjq_b200 as wjq
from warpjq_b200 import shard
from oracle import pyoracle as orc
from tests import corpus

pytestmark = pytest.mark.gpu

QUERIES = ["select(.status == 500) | count", "sum(.bytes)", "min(.latency_ms)", "max(.bytes)",
           "group_by(.host) | sum(.bytes)", "group_by(.path) | count", "group_by(.status) | avg(.bytes)",
           "select(.status >= 500) | {p: .path, b: .bytes}", "select(.status == 500)"]


@pytest.mark.parametrize("world", [1, 2, 3])
def test_device_partials_merge_to_the_whole_input_result(world):
    buf, used, _ = wjq.gen_nginx(6 << 20, seed=4)
    data = bytes(buf[:used]) + b'{oops\n\n{"status":500,"host":"h\\u00e9","bytes":1}\n'
    bounds = shard.shard_bounds(data, world)
    for q in QUERIES:
        parts = [shard.device_partial(q, data[lo:hi]) for lo, hi in bounds]
        got = shard.render(q, shard.merge(parts))
        assert got == orc.run(q, data).out, q


def test_hostile_corpus_groups_merge_by_decoded_key(golden):
    data = corpus.corpus(31, 1200, 0.05)
    bounds = shard.shard_bounds(data, 3)
    for q in ["group_by(.host) | count", "group_by(.msg) | count", "count"]:
        parts = [shard.device_partial(q, data[lo:hi]) for lo, hi in bounds]
        assert shard.render(q, shard.merge(parts)) == orc.run(q, data).out, q


@pytest.mark.parametrize("world", [1, 3])
def test_csv_device_partials_merge_to_the_whole_input_result(world):
    """CSV cut for several ranks (shard.csv_shard_bounds): each range runs
    behind a copy of the header, converted and scanned on the device, and the
    merge renders what the oracle prints for the whole input's NDJSON."""
    from oracle import csv_map
    from tests.test_shard_gloo import make_csv
    data = make_csv()
    nd = csv_map.csv_to_ndjson(data)
    h_end, bounds = shard.csv_shard_bounds(data, world)
    for q in ["select(.status == 500) | count", "sum(.bytes)", "group_by(.host) | sum(.bytes)",
              "group_by(.path) | count", "select(.status >= 500) | {p: .path, b: .bytes}", ".ua"]:
        parts = [shard.csv_device_partial(q, data[:h_end], data[lo:hi]) for lo, hi in bounds]
        assert shard.render(q, shard.merge(parts)) == orc.run(q, nd).out, q
