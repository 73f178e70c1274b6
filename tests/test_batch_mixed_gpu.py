"""Mixed batches (warpjq_batch_launch_mixed): inputs with different queries
in one launch sequence, one specialised scan launch per distinct query over
its inputs' tiles; aggregate queries, and row queries (projection,
passthrough, a single path) whose rows come out in input order.  Every
input's output must equal the oracle's for that input alone, whichever
query drives the launch (an aggregate, a grouped aggregate or a row query),
on a second launch over the same buffers too, and when the row launches'
records overflow the per-CTA arena they share (the batch is rerun with more
room)."""

import random

import numpy as np
import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc
from tests.test_batch_gpu import inputs, pack

pytestmark = pytest.mark.gpu

AGG = ["count", "select(.status == 500) | count", "sum(.bytes)", "avg(.bytes)", "min(.latency_ms)",
       "max(.bytes)", "group_by(.host) | sum(.bytes)", "group_by(.a) | count", "group_by(.path) | count",
       "select(.status >= 500) | group_by(.host) | count"]


def test_mixed_batch_matches_each_input_alone():
    import torch
    ins = inputs()
    data, offs, lens = pack(ins)
    host = np.frombuffer(data, dtype=np.uint8)
    dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
    dev[:len(data)].copy_(torch.from_numpy(host.copy()))
    qs = {q: wjq.Query(q) for q in AGG}
    rng = random.Random(5)
    pick = [rng.choice(AGG) for _ in ins]
    stream = torch.cuda.current_stream().cuda_stream
    for driver in ("count", "group_by(.host) | sum(.bytes)"):
        D = wjq.Query(driver)
        for rep in range(2):
            D.batch_launch_mixed([qs[q] for q in pick], dev.data_ptr(), offs, lens, stream)
            items, all_ = D.batch_collect()
            outs = wjq.batch_outputs_mixed([qs[q] for q in pick], items, all_, host)
            for i, (q, x) in enumerate(zip(pick, ins)):
                assert outs[i] == orc.run(q, x).out, (driver, rep, i, q, outs[i][:200])
        D.close()
    for Q in qs.values():
        Q.close()


ROWS = ["select(.status >= 500) | {p: .path, b: .bytes}", "select(.status == 500)", ".path",
        "select(.a == 1) | {a: .a, b: .b}", "select(.host == \"api-01\") | .latency_ms"]


def test_mixed_batch_with_row_queries_matches_each_input_alone():
    import torch
    ins = inputs()
    data, offs, lens = pack(ins)
    host = np.frombuffer(data, dtype=np.uint8)
    dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
    dev[:len(data)].copy_(torch.from_numpy(host.copy()))
    qs = {q: wjq.Query(q) for q in AGG + ROWS}
    rng = random.Random(11)
    pick = [rng.choice(AGG + ROWS) for _ in ins]
    stream = torch.cuda.current_stream().cuda_stream
    for driver in ("count", "select(.status == 500)"):
        D = wjq.Query(driver)
        for rep in range(2):
            D.batch_launch_mixed([qs[q] for q in pick], dev.data_ptr(), offs, lens, stream)
            items, all_ = D.batch_collect()
            assert all_.n_selected == sum(it.n_selected for it in items)
            outs = wjq.batch_outputs_mixed([qs[q] for q in pick], items, all_, host)
            for i, (q, x) in enumerate(zip(pick, ins)):
                assert outs[i] == orc.run(q, x).out, (driver, rep, i, q, outs[i][:200])
        D.close()
    for Q in qs.values():
        Q.close()


def test_mixed_row_launches_overflowing_the_shared_record_arena():
    # Lines of ~10 bytes: a 6 KB tile holds ~600 rows, and a CTA's records
    # from the two row queries' launches (every line selected) accumulate in
    # one arena sized for about one row per KiB plus 1024, so CTAs that take
    # a tile in both launches (~7,000 tiles against a few thousand CTAs)
    # overflow it and the batch is rerun with a larger arena.
    import torch
    rng = random.Random(3)
    ins = []
    for k in range(7):
        n = 700_000 + rng.randrange(50_000)
        ins.append(b"".join(b'{"a":%d}\n' % rng.randrange(1000) for _ in range(n)))
    data, offs, lens = pack(ins)
    host = np.frombuffer(data, dtype=np.uint8)
    dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
    dev[:len(data)].copy_(torch.from_numpy(host.copy()))
    pick = [".a", "select(.a >= 0)", "sum(.a)", ".a", "select(.a >= 0)", ".a", "group_by(.a) | count"]
    qs = {q: wjq.Query(q) for q in set(pick)}
    stream = torch.cuda.current_stream().cuda_stream
    D = wjq.Query("count")
    for rep in range(2):
        D.batch_launch_mixed([qs[q] for q in pick], dev.data_ptr(), offs, lens, stream)
        items, all_ = D.batch_collect()
        assert all_.n_selected == sum(it.n_selected for it in items)
        outs = wjq.batch_outputs_mixed([qs[q] for q in pick], items, all_, host)
        for i, (q, x) in enumerate(zip(pick, ins)):
            want = orc.run(q, x).out
            assert outs[i] == want, (rep, i, q, len(outs[i]), len(want))
    D.close()
    for Q in qs.values():
        Q.close()
