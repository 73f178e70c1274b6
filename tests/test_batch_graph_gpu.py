"""Batched runs replayed from one CUDA graph (warpjq_batch_graph_*): one
batch per query, captured once on forked streams, replayed with one launch.
Every input's output must equal the oracle's for that input, on the first
replay, on later replays, and after the inputs' bytes change in place; a
plain batch on one of the graph's contexts, or a buffer grown by an
overflow, must make the next replay refuse instead of writing through stale
addresses."""

import numpy as np
import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc
from tests.test_batch_gpu import inputs, pack

pytestmark = pytest.mark.gpu

QUERIES = ["count", "sum(.bytes)", "min(.latency_ms)", "group_by(.host) | count",
           "select(.status >= 500) | {p: .path, b: .bytes}", "select(.status == 500)"]


def _device(data: bytes):
    import torch
    dev = torch.zeros(len(data) + 16, dtype=torch.uint8, device="cuda")
    dev[:len(data)].copy_(torch.from_numpy(np.frombuffer(data, dtype=np.uint8).copy()))
    return dev


def _check(qs, parts, host, ins_per_query):
    for Q, ins in zip(qs, ins_per_query):
        items, all_ = Q.batch_collect()
        outs = Q.batch_outputs(items, all_, host)
        for i, x in enumerate(ins):
            assert outs[i] == orc.run(Q.query, x).out, (Q.query, i)


def test_graph_replays_match_the_oracle():
    import torch
    ins = inputs()
    data, offs, lens = pack(ins)
    dev = _device(data)
    host = np.frombuffer(data, dtype=np.uint8)
    # each query takes every third input, starting at its own offset
    picks = [list(range(k % 3, len(ins), 3)) for k in range(len(QUERIES))]
    qs = [wjq.Query(q) for q in QUERIES]
    g = wjq.BatchGraph([(Q, dev.data_ptr(), [offs[i] for i in p], [lens[i] for i in p])
                        for Q, p in zip(qs, picks)])
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(3):
        g.launch(stream)
        _check(qs, None, host, [[ins[i] for i in p] for p in picks])
    g.close()
    for Q in qs:
        Q.close()


def test_replay_after_the_bytes_change_in_place():
    import torch
    buf, used, _ = wjq.gen_nginx(2 << 20, seed=21)
    lines = bytes(buf[:used]).split(b"\n")[:-1]
    ins = [b"\n".join(lines[i:i + 50]) + b"\n" for i in range(0, 4000, 50)]
    data, offs, lens = pack(ins)
    dev = _device(data)
    qs = [wjq.Query(q) for q in ["select(.status == 500) | count", "group_by(.path) | count",
                                 "select(.status == 500)"]]
    g = wjq.BatchGraph([(Q, dev.data_ptr(), offs, lens) for Q in qs])
    stream = torch.cuda.current_stream().cuda_stream
    g.launch(stream)
    _check(qs, None, np.frombuffer(data, dtype=np.uint8), [ins] * len(qs))
    # same layout, other bytes: every 200 becomes 500 (same length)
    data2 = data.replace(b'"status":200', b'"status":500').replace(b"/api/v1/users", b"/api/v1/uxers")
    ins2 = [data2[o:o + n] for o, n in zip(offs, lens)]
    dev[:len(data2)].copy_(torch.from_numpy(np.frombuffer(data2, dtype=np.uint8).copy()))
    torch.cuda.synchronize()
    g.launch(stream)
    _check(qs, None, np.frombuffer(data2, dtype=np.uint8), [ins2] * len(qs))
    g.close()
    for Q in qs:
        Q.close()


def test_a_plain_batch_invalidates_the_graph():
    import torch
    ins = inputs()[:20]
    data, offs, lens = pack(ins)
    dev = _device(data)
    Q = wjq.Query("count")
    g = wjq.BatchGraph([(Q, dev.data_ptr(), offs, lens)])
    stream = torch.cuda.current_stream().cuda_stream
    g.launch(stream)
    Q.batch_collect()
    Q.batch_launch(dev.data_ptr(), offs[:5], lens[:5], stream)
    Q.batch_collect()
    with pytest.raises(RuntimeError, match="create the graph again"):
        g.launch(stream)
    g.close()
    g2 = wjq.BatchGraph([(Q, dev.data_ptr(), offs, lens)])
    g2.launch(stream)
    _check([Q], None, np.frombuffer(data, dtype=np.uint8), [ins])
    g2.close()
    Q.close()


def test_an_overflow_in_a_replay_stays_complete_and_retires_the_graph():
    import torch
    q = "select(.k == 1) | {a: .k, b: .k, c: .k, d: .k}"
    cold = b'{"k":2}\n' * 300_000   # nothing selected when the graph is made
    hot = b'{"k":1}\n' * 300_000    # rows 3.25x the input when it is replayed
    data, offs, lens = pack([cold])
    dev = _device(data)
    Q = wjq.Query(q)
    g = wjq.BatchGraph([(Q, dev.data_ptr(), offs, lens)])
    stream = torch.cuda.current_stream().cuda_stream
    data2 = data.replace(cold, hot)
    dev[:len(data2)].copy_(torch.from_numpy(np.frombuffer(data2, dtype=np.uint8).copy()))
    torch.cuda.synchronize()
    g.launch(stream)
    _check([Q], None, np.frombuffer(data2, dtype=np.uint8), [[hot]])
    with pytest.raises(RuntimeError, match="create the graph again"):
        g.launch(stream)
    g.close()
    Q.close()
