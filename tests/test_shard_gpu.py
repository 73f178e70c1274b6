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
