"""The native serving loop (include/warpjq_serve.h, warpjq_b200.serve.
NativeServer) on the device: NDJSON and CSV requests over many queries, from
host memory and from device memory (aligned, used in place, and unaligned,
copied), submitted while earlier ones run; every output must equal the
oracle's for that input alone and what the same server prints for the
request served alone.  A request larger than the budget is refused."""

import numpy as np
import pytest
import torch

from tests.test_serve_gpu import QUERIES, matches, workload
from warpjq_b200.serve import NativeServer

pytestmark = pytest.mark.gpu


def _device(data: bytes, misalign: int = 0):
    t = torch.zeros(len(data) + 32, dtype=torch.uint8, device="cuda")
    if data:
        t[misalign:misalign + len(data)] = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
    return t[misalign:misalign + len(data)]


def test_native_server_matches_the_oracle_for_every_request():
    reqs = workload(seed=5, n=160)
    srv = NativeServer(QUERIES, n_slots=3, mixed_min=4)
    srv.warm(8 << 20)
    ids = {}
    for i, (q, data, fmt) in enumerate(reqs):
        src = data
        if i % 3 == 1:
            src = _device(data)             # in place
        elif i % 3 == 2:
            src = _device(data, misalign=3)  # copied into the slot's arena
        ids[srv.submit(q, src, fmt)] = i
    done = srv.drain()
    srv.close()
    assert len(done) == len(reqs)
    bad = []
    for r in done:
        q, data, fmt = reqs[ids[r.id]]
        assert r.rc == 0, r.error
        if not matches(r.out, q, data, fmt):
            bad.append((ids[r.id], q, fmt))
    assert not bad, bad[:5]


def test_native_server_alone_equals_in_the_mix():
    reqs = workload(seed=9, n=60)
    mix = NativeServer(QUERIES, n_slots=3, mixed_min=2)
    ids = {mix.submit(q, d, f): i for i, (q, d, f) in enumerate(reqs)}
    in_mix = {ids[r.id]: r.out for r in mix.drain()}
    mix.close()
    alone = NativeServer(QUERIES, n_slots=1, max_batch=1, mixed_min=0)
    for i, (q, d, f) in enumerate(reqs):
        alone.submit(q, d, f)
        (r,) = alone.drain()
        assert r.rc == 0, r.error
        assert r.out == in_mix[i], (i, q, f)
    alone.close()


def test_native_server_budget():
    nb = b'{"status":500,"bytes":1}\n' * 4000
    srv = NativeServer(["select(.status == 500) | count"], n_slots=2, budget_bytes=(1 << 20) + 3 * len(nb))
    big = np.zeros(8 << 20, dtype=np.uint8)
    big[::100] = 10
    rid_big = srv.submit("select(.status == 500) | count", big)
    rids = [srv.submit("select(.status == 500) | count", nb) for _ in range(8)]
    done = {r.id: r for r in srv.drain()}
    srv.close()
    assert done[rid_big].rc == 1 and "over the budget" in done[rid_big].error
    for rid in rids:
        assert done[rid].rc == 0 and done[rid].out == b"4000\n"
