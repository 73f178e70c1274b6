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


def first_invalid(data: bytes):
    """Index of the first physical line that is neither blank nor valid JSON
    (the nginx-schema test data has no other kind of bad line)."""
    for i, ln in enumerate(data.split(b"\n")[:-1]):
        if ln.strip():
            try:
                json.loads(ln)
            except ValueError:
                return i
    return None


def cpu_partial(query: str, data: bytes) -> shard.Partial:
    base = dict(n_lines=data.count(b"\n"), first_invalid=first_invalid(data))
    if query in ROW_QUERIES:
        r = orc.run(query, data)
        return shard.Partial(rows=r.out, **base)
    flt, agg, grp = AGG_QUERIES[query]
    p = shard.Partial(**base)
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


def make_data_late_bad() -> bytes:
    """Valid lines, blank lines, and malformed lines only in the second half,
    so with two ranks the first bad line lies in rank 1's range."""
    buf, used, _ = wjq.gen_nginx(1 << 19, seed=5)
    lines = bytes(buf[:used]).split(b"\n")[:-1]
    out = []
    for i, ln in enumerate(lines):
        if i % 17 == 4:
            out.append(b"")
        if i > len(lines) * 3 // 4 and i % 29 == 11:
            out.append(b'{"status":500,')
        out.append(ln)
    return b"\n".join(out) + b"\n"


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        for tag, data in (("a", make_data()), ("b", make_data_late_bad())):
            lo, hi = shard.shard_bounds(data, world)[rank]
            for i, q in enumerate(ROW_QUERIES + list(AGG_QUERIES)):
                part = cpu_partial(q, data[lo:hi])
                if q in ROW_QUERIES and rank % 2:
                    # rows handed over as a tensor, as a device-resident run does
                    import torch
                    part.rows = torch.frombuffer(bytearray(part.rows), dtype=torch.uint8) if part.rows \
                        else torch.empty(0, dtype=torch.uint8)
                parts = shard.gather(part, rank, world)
                if rank == 0:
                    m = shard.merge(parts)
                    with open(os.path.join(out_dir, f"{tag}{i}.out"), "wb") as f:
                        f.write(shard.render(q, m))
                    with open(os.path.join(out_dir, f"{tag}{i}.json"), "w") as f:
                        json.dump({"first_invalid": m.first_invalid, "n_lines": m.n_lines}, f)
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


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_merge_to_the_single_input_result(world):
    with tempfile.TemporaryDirectory() as out_dir:
        mp.start_processes(_rank_main, args=(world, _free_port(), out_dir), nprocs=world,
                           start_method="spawn", join=True)
        for tag, data in (("a", make_data()), ("b", make_data_late_bad())):
            fi = first_invalid(data)
            assert fi is not None
            if tag == "b":  # the first bad line is past rank 0's range
                assert fi >= data[:shard.shard_bounds(data, world)[0][1]].count(b"\n")
            for i, q in enumerate(ROW_QUERIES + list(AGG_QUERIES)):
                with open(os.path.join(out_dir, f"{tag}{i}.out"), "rb") as f:
                    got = f.read()
                want = orc.run(q, data).out
                assert got == want, (tag, q, got[:200], want[:200])
                with open(os.path.join(out_dir, f"{tag}{i}.json")) as f:
                    st = json.load(f)
                assert st["first_invalid"] == fi and st["n_lines"] == data.count(b"\n"), (tag, q, st, fi)


def make_csv() -> bytes:
    """The nginx records as CSV, with quoted newlines and doubled quotes put
    into some ua fields, so cuts must find row ends outside quotes."""
    buf, used, _ = wjq.gen_nginx_csv(1 << 20, seed=9)
    rows = bytes(buf[:used]).split(b"\n")[:-1]
    out = [rows[0]]
    for i, r in enumerate(rows[1:]):
        if i % 7 == 3:
            r = r.replace(b',"', b',"line one\nline "" two\n', 1)
        out.append(r)
    return b"\n".join(out) + b"\n"


def test_csv_shard_bounds_cut_at_row_ends():
    from oracle import csv_map
    from tests.test_csv_gpu import fuzz_csv
    for data in [make_csv(), fuzz_csv(3, 2000, crlf=True, bom=True), fuzz_csv(4, 500),
                 b"k\n" + b'"' + b"x\n" * 5000 + b'"\n1\n']:
        whole = csv_map.csv_to_ndjson(data).split(b"\n")[:-1]
        for world in (1, 2, 3, 5):
            h_end, b = shard.csv_shard_bounds(data, world)
            assert b[0][0] == h_end and b[-1][1] == len(data) and len(b) == world
            parts = []
            for (a0, a1), nxt in zip(b, b[1:] + [(len(data), len(data))]):
                assert a1 == nxt[0]
                assert data[:a1].count(b'"') % 2 == 0  # each cut is outside quotes
                parts += csv_map.csv_to_ndjson(data[:h_end] + data[a0:a1]).split(b"\n")[:-1]
            assert parts == whole, world


def _rank_main_csv(rank, world, port, out_dir):
    import torch.distributed as dist
    from oracle import csv_map
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        data = make_csv()
        h_end, bounds = shard.csv_shard_bounds(data, world)
        lo, hi = bounds[rank]
        mine = csv_map.csv_to_ndjson(data[:h_end] + data[lo:hi])
        for i, q in enumerate(ROW_QUERIES + list(AGG_QUERIES)):
            parts = shard.gather(cpu_partial(q, mine), rank, world)
            if rank == 0:
                with open(os.path.join(out_dir, f"{i}.out"), "wb") as f:
                    f.write(shard.render(q, shard.merge(parts)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_merge_csv_shards_to_the_single_input_result():
    from oracle import csv_map
    world = 2
    with tempfile.TemporaryDirectory() as out_dir:
        mp.start_processes(_rank_main_csv, args=(world, _free_port(), out_dir), nprocs=world,
                           start_method="spawn", join=True)
        nd = csv_map.csv_to_ndjson(make_csv())
        for i, q in enumerate(ROW_QUERIES + list(AGG_QUERIES)):
            with open(os.path.join(out_dir, f"{i}.out"), "rb") as f:
                got = f.read()
            want = orc.run(q, nd).out
            assert got == want, (q, got[:200], want[:200])
