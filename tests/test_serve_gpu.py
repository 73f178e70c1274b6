"""The continuous-batching server (warpjq_b200/serve.py) on the device: a mix
of NDJSON and CSV requests over many queries, arriving while earlier ones
are on the GPU, each output identical to the oracle's for its input alone
and to the same request served alone; the memory budget splits admission
into several rounds and refuses a request larger than itself."""

import random

import pytest

import warpjq_b200 as wjq
from oracle import csv_map
from oracle import pyoracle as orc
from tests.test_gpu_parity import close_enough
from warpjq_b200.serve import Server

pytestmark = pytest.mark.gpu

QUERIES = ["count", "select(.status == 500) | count", "sum(.bytes)", "max(.latency_ms)",
           "avg(.latency_ms)", "group_by(.host) | count", "group_by(.path) | max(.latency_ms)",
           "select(.status >= 500) | {p: .path, b: .bytes}", "select(.status == 503)",
           'select(.req.user.tier == "gold" and .resp.code != 200) | {u: .req.user.id, l: .resp.latency}',
           "group_by(.req.user.tier) | count"]


def workload(seed=3, n=120):
    rng = random.Random(seed)
    nb, nu, _ = wjq.gen_nginx(6 << 20, seed=seed)
    nginx = bytes(nb[:nu]).split(b"\n")[:-1]
    sb, su, _ = wjq.gen_nested(3 << 20, seed=seed, n_users=1000)
    nested = bytes(sb[:su]).split(b"\n")[:-1]
    cb, cu, _ = wjq.gen_nginx_csv(4 << 20, seed=seed)
    crow = bytes(cb[:cu]).split(b"\n")
    head, crow = crow[0], crow[1:-1]
    reqs = []
    for i in range(n):
        k = rng.randrange(1, 3000)
        kind = rng.random()
        if kind < 0.2:  # CSV: a header and a run of rows
            a = rng.randrange(0, len(crow) - k)
            data, fmt = head + b"\n" + b"\n".join(crow[a:a + k]) + b"\n", "csv"
            q = rng.choice(QUERIES[:9])
        elif kind < 0.35:
            a = rng.randrange(0, len(nested) - k)
            data, fmt = b"\n".join(nested[a:a + k]) + b"\n", "ndjson"
            q = rng.choice(QUERIES[9:] + QUERIES[:1])
        else:
            a = rng.randrange(0, len(nginx) - k)
            data, fmt = b"\n".join(nginx[a:a + k]) + b"\n", "ndjson"
            q = rng.choice(QUERIES[:9])
        reqs.append((q, data, fmt))
    return reqs


def expected(q, data, fmt):
    return orc.run(q, csv_map.csv_to_ndjson(data) if fmt == "csv" else data).out


def matches(got, q, data, fmt):
    """Byte-identical to the oracle, except fractional FP averages: within
    1e-9 relative (the oracle adds in line order, the device in a fixed
    tree; each is deterministic)."""
    want = expected(q, data, fmt)
    return got == want or ("avg(" in q and close_enough(got, want))


def test_each_result_is_the_same_alone_and_in_the_mix(monkeypatch):
    import warpjq_b200.serve as serve
    monkeypatch.setattr(serve, "MIXED_MIN", 2)  # exercise the mixed batches on these small slots too
    reqs = workload()
    srv = Server(QUERIES, n_slots=3)
    handles = []
    for i, (q, data, fmt) in enumerate(reqs):
        handles.append(srv.submit(q, data, fmt))
        if i % 7 == 0:  # later requests arrive while earlier ones run
            srv.poll()
    srv.drain()
    assert all(not h.error for h in handles)
    for h, (q, data, fmt) in zip(handles, reqs):
        assert matches(h.out, q, data, fmt), (h.id, q, fmt, h.out[:200])
    # the same requests, one at a time
    alone = Server(QUERIES, n_slots=1)
    for h, (q, data, fmt) in list(zip(handles, reqs))[:40]:
        r = alone.submit(q, data, fmt)
        alone.drain()
        assert r.out == h.out, (h.id, q)  # exact: an input's tiles and order do not depend on the mix
    alone.close()
    srv.close()


def test_device_resident_requests():
    import torch
    reqs = workload(seed=9, n=40)
    srv = Server(QUERIES, n_slots=2)
    srv.warm(1 << 20)
    hs = []
    for q, data, fmt in reqs:
        t = torch.frombuffer(bytearray(data), dtype=torch.uint8).cuda()
        hs.append(srv.submit(q, t, fmt))
    srv.drain()
    for h, (q, data, fmt) in zip(hs, reqs):
        assert matches(h.out, q, data, fmt), (h.id, q)
    srv.close()


def test_budget_splits_admission_and_refuses_oversized_requests():
    reqs = workload(seed=5, n=30)
    biggest = max(len(d) for _, d, _ in reqs)
    budget = 3 * wjq.serve.footprint(biggest * 2, "csv")
    srv = Server(QUERIES, n_slots=3, budget_bytes=budget)
    hs = [srv.submit(q, d, f) for q, d, f in reqs]
    rounds = 0
    while srv.pending():
        assert srv.in_flight_bytes <= budget
        if srv.poll():
            rounds += 1
    assert rounds > 1
    for h, (q, d, f) in zip(hs, reqs):
        assert matches(h.out, q, d, f)
    big = srv.submit("count", b'{"a":1}\n' * (budget // 8), "ndjson")
    assert big.error and "over the budget" in big.error
    srv.close()
