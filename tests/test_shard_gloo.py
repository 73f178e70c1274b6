"""Multi-GPU host logic on CPU: two `gloo` ranks split one input by newline-
aligned byte ranges (warpjq_b200.shard), each builds its partial result,
rank 0 gathers, merges and renders them with the host library's formatter,
and the bytes must equal the oracle's output for the whole input.

The ranks' partials are made here on the CPU (no GPU on this machine): rows
from the oracle over the rank's range, aggregate states by a small
evaluator for the nginx-schema queries below.  On a GPU box
`shard.partial_from_device` makes them from a device-resident run instead.
"""

import json
import math
import os
import socket
import tempfile

import pytest
import torch.multiprocessing as mp

import warpjq_b200 as wjq
from warpjq_b200 import shard
from oracle import pyoracle as orc

ROW_QUERIES = ["select(.status >= 500) | {p: .path, b: .bytes}", "select(.status == 500)"]
AGG_QUERIES = {
    "select(.status == 500) | count": (("status", "==", 500), None, None),
    "sum(.bytes)": (None, "bytes", None),
    "min(.latency_ms)": (None, "latency_ms", None),
    "max(.bytes)": (None, "bytes", None),
    "select(.status >= 500) | sum(.bytes)": (("status", ">=", 500), "bytes", None),
    "group_by(.host) | sum(.bytes)": (None, "bytes", "host"),
    "group_by(.status) | count": (None, None, "status"),
}


def make_data() -> bytes:
    buf, used, _ = wjq.gen_nginx(1 << 20, seed=9)
    lines = bytes(buf[:used]).split(b"\n")[:-1]
    out = []
    for i, ln in enumerate(lines):
        if i % 41 == 7:
            out.append(b"{oops")
        if i % 53 == 3:
            out.append(b"   ")
        out.append(ln)
    return b"\n".join(out) + b"\n"


def cpu_partial(query: str, data: bytes) -> shard.Partial:
    if query in ROW_QUERIES:
        r = orc.run(query, data)
        return shard.Partial(rows=r.out)
    flt, agg, grp = AGG_QUERIES[query]
    p = shard.Partial()
    groups = {}
    for ln in data.split(b"\n"):
        if not ln.strip():
            continue
        try:
            o = json.loads(ln)
        except ValueError:
            continue
        if flt:
            k, op, lit = flt
            v = o.get(k)
            if not isinstance(v, (int, float)) or not (v == lit if op == "==" else v >= lit):
                continue
        tgt = p
        if grp:
            gv = o.get(grp)
            kind, raw = (4, gv.encode()) if isinstance(gv, str) else (3, str(gv).encode())
            tgt = groups.get((kind, raw))
            if tgt is None:
                tgt = groups[(kind, raw)] = shard.GroupPart(kind=kind, raw=raw)
        tgt.count += 1
        if agg:
            v = o.get(agg)
            if isinstance(v, (int, float)) and not isinstance(v, bool):
                tgt.numeric += 1
                tgt.min, tgt.max = min(tgt.min, float(v)), max(tgt.max, float(v))
                if isinstance(v, int):
                    tgt.isum += v
                    tgt.n_int += 1
                else:
                    tgt.fsum += v
    p.groups = list(groups.values())
    return p


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        data = make_data()
        lo, hi = shard.shard_bounds(data, world)[rank]
        for i, q in enumerate(ROW_QUERIES + list(AGG_QUERIES)):
            parts = shard.gather(cpu_partial(q, data[lo:hi]), rank, world)
            if rank == 0:
                with open(os.path.join(out_dir, f"{i}.out"), "wb") as f:
                    f.write(shard.render(q, shard.merge(parts)))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_bounds_cut_after_newlines():
    data = make_data()
    for world in (1, 2, 3, 8):
        b = shard.shard_bounds(data, world)
        assert b[0][0] == 0 and b[-1][1] == len(data) and len(b) == world
        for (a0, a1), (b0, _) in zip(b, b[1:]):
            assert a1 == b0 and data[a1 - 1:a1] == b"\n"
    one_line = b'{"a":' + b"1" * 1000 + b"}\n"
    assert shard.shard_bounds(one_line, 4) == [(0, len(one_line)), (len(one_line),) * 2,
                                               (len(one_line),) * 2, (len(one_line),) * 2]


def test_decoded_string_keys_merge_across_ranks():
    a = shard.Partial(groups=[shard.GroupPart(kind=4, raw=b"caf\\u00e9", count=1)])
    b = shard.Partial(groups=[shard.GroupPart(kind=4, raw="café".encode(), count=2)])
    m = shard.merge([a, b])
    assert len(m.groups) == 1 and m.groups[0].count == 3
    assert shard.decode_key(4, b"\\ud83d\\ude00\\ud800x") == "😀�x".encode()


def test_two_gloo_ranks_merge_to_the_single_input_result():
    world = 2
    with tempfile.TemporaryDirectory() as out_dir:
        mp.start_processes(_rank_main, args=(world, _free_port(), out_dir), nprocs=world,
                           start_method="spawn", join=True)
        data = make_data()
        for i, q in enumerate(ROW_QUERIES + list(AGG_QUERIES)):
            with open(os.path.join(out_dir, f"{i}.out"), "rb") as f:
                got = f.read()
            want = orc.run(q, data).out
            assert got == want, (q, got[:200], want[:200])
