"""Batched device-resident runs (warpjq_batch_launch / warpjq_batch_collect):
many inputs of one query in one launch sequence.  Every input's output must
be byte-identical to the oracle's output for that input alone, and its line
counts to a run over it alone; the bytes between inputs in the batch buffer
are junk lines that must never be read as part of an input."""

import numpy as np
import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc
from tests import corpus

pytestmark = pytest.mark.gpu

QUERIES = ["count", "select(.status == 500) | count", "sum(.bytes)", "avg(.bytes)", "min(.latency_ms)",
           "group_by(.host) | sum(.bytes)", "group_by(.a) | count",
           "select(.status >= 500) | {p: .path, b: .bytes}", "select(.status == 500)", ".a", "."]
JUNK = b'\n{"status":500,"host":"junk","bytes":7,"a":1}\n'


def inputs():
    buf, used, _ = wjq.gen_nginx(3 << 20, seed=8)
    nginx = bytes(buf[:used])
    lines = nginx.split(b"\n")
    ins = [b"", b"\n", b"5", b'{"a":1}', b'{"a":2}\n{"a":', b'\n\n   \n', b'{"a":1}\r\n{"a":2}\r\n',
           b'{"a":"' + b"x" * 20000 + b'","status":500}\n', b'{"a":' + b"[" * 100 + b"]" * 100 + b"}\n",
           corpus.corpus(5, 300, 0.1), corpus.corpus(6, 50, 0.0, crlf=True), corpus.edge_corpus()]
    pos = 0
    for k in range(40):  # nginx pieces of assorted sizes, some cut mid-line
        n = [1, 37, 1000, 6400, 6401, 12800, 50000, 200000][k % 8]
        ins.append(nginx[pos:pos + n])
        pos += n
    ins.append(b"\n".join(lines[:20000]) + b"\n")
    return ins


def pack(ins):
    offs, parts, pos = [], [], 0
    for x in ins:
        pad = (-pos) % 16
        parts.append(JUNK[:pad] if pad <= len(JUNK) else b"\n" * pad)
        pos += pad
        offs.append(pos)
        parts.append(x)
        pos += len(x)
        parts.append(JUNK)
        pos += len(JUNK)
    return b"".join(parts), offs, [len(x) for x in ins]


def test_every_batch_input_matches_its_own_run():
    import torch
    ins = inputs()
    data, offs, lens = pack(ins)
    host = np.frombuffer(data, dtype=np.uint8)
    dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
    dev[:len(data)].copy_(torch.from_numpy(host.copy()))
    for q in QUERIES:
        Q = wjq.Query(q)
        alone = wjq.Query(q)
        for rep in range(2):  # the second batch reuses the first one's buffers
            Q.batch_launch(dev.data_ptr(), offs, lens, torch.cuda.current_stream().cuda_stream)
            items, all_ = Q.batch_collect()
            outs = Q.batch_outputs(items, all_, host)
            for i, x in enumerate(ins):
                want = orc.run(q, x)
                assert outs[i] == want.out, (q, rep, i, outs[i][:200], want.out[:200])
                if rep:
                    continue
                alone.launch_device(dev.data_ptr() + offs[i], lens[i],
                                    torch.cuda.current_stream().cuda_stream)
                r = alone.collect_device()
                it = items[i]
                assert (it.n_lines, it.n_blank, it.n_invalid, it.n_type_error) == \
                       (r.n_lines, r.n_blank, r.n_invalid, r.n_type_error), (q, i)
                assert it.first_invalid == r.first_invalid, (q, i)
        alone.close()
        Q.close()


def test_batch_with_many_small_inputs_and_one_empty_batch():
    import torch
    buf, used, _ = wjq.gen_nginx(2 << 20, seed=3)
    lines = bytes(buf[:used]).split(b"\n")[:-1]
    ins = [b"\n".join(lines[i:i + (i % 7) + 1]) + b"\n" for i in range(0, 3000, 4)]
    data, offs, lens = pack(ins)
    host = np.frombuffer(data, dtype=np.uint8)
    dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
    dev[:len(data)].copy_(torch.from_numpy(host.copy()))
    for q in ["group_by(.host) | count", "select(.status == 500)", "max(.bytes)"]:
        Q = wjq.Query(q)
        Q.batch_launch(dev.data_ptr(), offs, lens)
        items, all_ = Q.batch_collect()
        outs = Q.batch_outputs(items, all_, host)
        for i, x in enumerate(ins):
            assert outs[i] == orc.run(q, x).out, (q, i)
        Q.batch_launch(dev.data_ptr(), [], [])
        items, all_ = Q.batch_collect()
        assert items == [] and all_.n_lines == 0
        Q.close()
