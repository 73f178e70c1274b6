"""Mixed batches (warpjq_batch_launch_mixed): inputs with different queries
in one launch of the scan kernel, each tile taking its input's plan from
device memory; aggregate queries, and row queries (projection, passthrough,
a single path) whose rows come out in input order.  Every input's output
must equal the oracle's for that input alone, whichever query drives the
launch (an aggregate, a grouped aggregate or a row query), on a second
launch over the same buffers too."""

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
