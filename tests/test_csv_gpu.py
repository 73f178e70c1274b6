"""CSV input on the device: warpjq_csv_convert must produce byte for byte the
NDJSON of the mapping in oracle/csv_map.py, whole or in chunks, from device
or host memory, at any alignment; and a query over CSV (warpjq_query_run_csv)
must print what the oracle prints for the mapped NDJSON."""

import random

import numpy as np
import pytest

import warpjq_b200 as wjq
from oracle import csv_map
from oracle import pyoracle as orc
from tests.test_csv_map import HAND

pytestmark = pytest.mark.gpu


def _dev(data: bytes, shift: int = 0):
    import torch
    buf = torch.zeros(len(data) + 32 + shift, dtype=torch.uint8, device="cuda")
    if data:
        buf[shift:shift + len(data)].copy_(torch.frombuffer(bytearray(data), dtype=torch.uint8))
    return buf, buf.data_ptr() + shift


def _read(ptr: int, n: int) -> bytes:
    import torch
    from warpjq_b200.shard import _DeviceBytes
    if n == 0:
        return b""
    return torch.as_tensor(_DeviceBytes(ptr, n), device="cuda").cpu().numpy().tobytes()


def fuzz_csv(seed: int, rows: int, cols: int = 5, crlf: bool = False, bom: bool = False) -> bytes:
    rng = random.Random(seed)
    pieces = ['a', 'b', ' ', ',', '"', '""', '\n', '\r', '\t', '\\', '\x01', 'é', '12', '-3.5e2', '0', '01']
    out = [("﻿" if bom else "") + ",".join(f"col{j}" if j % 3 else f'"c,{j}"' for j in range(cols))]
    for _ in range(rows):
        fields = []
        for _ in range(rng.randrange(0, cols + 2)):
            body = "".join(rng.choice(pieces) for _ in range(rng.randrange(0, 6)))
            if rng.random() < 0.5:
                fields.append('"' + body.replace('"', '""') + '"')
            else:
                fields.append(body.replace('"', "").replace(",", "").replace("\n", "").replace("\r", ""))
        out.append(",".join(fields))
    text = ("\r\n" if crlf else "\n").join(out) + ("\r\n" if crlf else "\n")
    return text.encode()


def cases():
    cs = [src for src, _ in HAND]
    cs += [fuzz_csv(s, r, crlf=s % 2 == 1, bom=s % 3 == 0) for s, r in enumerate([1, 5, 50, 400, 3000, 20000])]
    cs.append(fuzz_csv(99, 2000)[:-1])                    # no final newline
    cs.append(b"k\n" + b'"' + b"x" * 200_000 + b'"\n1\n')  # one row across many tiles
    cs.append(b"k\n" + b'"' + b"\n" * 70_000 + b'"\n2\n')  # newlines inside quotes across tiles
    cs.append(b"k\n" + b'"open quote never closes\n' * 3000)
    buf, used, _ = wjq.gen_nginx_csv(3 << 20, seed=4)
    cs.append(bytes(buf[:used]))
    return cs


def test_converter_matches_the_mapping_at_any_alignment():
    conv = wjq.CsvConverter()
    for i, src in enumerate(cases()):
        want = csv_map.csv_to_ndjson(src)
        for shift in (0, 3, 13):
            conv.reset()
            keep, ptr = _dev(src, shift)
            d, n, used, recs = conv.convert(ptr, len(src))
            got = _read(d, n)
            assert got == want, (i, shift, got[:300], want[:300])
            assert used == len(src)
            assert recs == want.count(b"\n")
            del keep
    conv.close()


def test_host_input_matches_device_input():
    conv = wjq.CsvConverter()
    for src in cases()[-6:]:
        conv.reset()
        host = np.frombuffer(bytearray(src) + b"\0", dtype=np.uint8)
        d, n, used, _ = conv.convert(host.ctypes.data, len(src), host=True)
        assert _read(d, n) == csv_map.csv_to_ndjson(src)
    conv.close()


def test_chunked_conversion_equals_the_whole():
    conv = wjq.CsvConverter()
    rng = random.Random(3)
    for src in [fuzz_csv(7, 3000), fuzz_csv(8, 3000, crlf=True), cases()[-1][:400_000]]:
        want = csv_map.csv_to_ndjson(src)
        for _ in range(3):
            conv.reset()
            pos, parts = 0, []
            while True:
                n = min(len(src) - pos, rng.randrange(1, 60_000))
                final = pos + n == len(src)
                keep, ptr = _dev(src[pos:pos + n])
                d, nd, used, _ = conv.convert(ptr, n, final=final)
                parts.append(_read(d, nd))
                if final:
                    assert used == n
                    break
                pos += used  # bytes after the last whole row come again
            assert b"".join(parts) == want
    conv.close()


QUERIES = ["count", "select(.status == 500) | count", "group_by(.path) | max(.latency_ms)",
           "group_by(.host) | sum(.bytes)", "select(.status >= 500) | {p: .path, b: .bytes}",
           "select(.status == 503)", "max(.bytes)", "min(.latency_ms)", ".ua"]


def test_queries_over_csv_match_the_oracle():
    buf, used, rows = wjq.gen_nginx_csv(5 << 20, seed=12)
    src = bytes(buf[:used])
    nd = csv_map.csv_to_ndjson(src)
    for q in QUERIES:
        want = orc.run(q, nd)
        for chunk in (0, 1 << 20):  # one chunk, and chunks of 1 MiB (rows carried over)
            Q = wjq.Query(q, chunk_bytes=chunk)
            r = Q.run_csv(src)
            assert r.rc == 0, r.err
            assert r.out == want.out, (q, chunk, r.out[:300], want.out[:300])
            assert r.stats["lines_in"] == rows
            Q.close()


def test_dirty_csv_queries_match_the_oracle():
    src = fuzz_csv(21, 5000, crlf=True, bom=True)
    nd = csv_map.csv_to_ndjson(src)
    for q in ["count", 'group_by(.col1) | count', "select(.col1 != null) | {a: .col1, b: .col2}", ".col4",
              '."c,0"']:
        want = orc.run(q, nd)
        Q = wjq.Query(q)
        r = Q.run_csv(src)
        assert r.rc == 0, r.err
        assert r.out == want.out, (q, r.out[:300], want.out[:300])
        Q.close()


def test_empty_and_header_only_csv():
    for src in [b"", b"a,b\n", b"a,b"]:
        Q = wjq.Query("count")
        r = Q.run_csv(src)
        assert r.rc == 0 and r.out == orc.run("count", b"").out
        Q.close()


def test_pipelined_chunks_carry_long_rows():
    """warpjq_query_run_csv copies chunk k + 1 while chunk k is converted;
    rows longer than the room kept for a carried row (64 KiB), and a row
    longer than a whole 1 MiB chunk, must come out the same as in one piece,
    from page-locked and from ordinary host memory."""
    import torch
    rng = random.Random(17)
    rows = [b"k,v"]
    for i in range(400):
        n = rng.choice([10, 100, 1000, 90_000, 300_000]) if i != 200 else 2_500_000
        rows.append(b'"' + (b"x" * n).replace(b"xxxxxxxxxx", b'x""x,x\nxxx', 1) + b'",' + str(i).encode())
    src = b"\n".join(rows) + b"\n"
    nd = csv_map.csv_to_ndjson(src)
    pinned = torch.empty(len(src), dtype=torch.uint8).pin_memory()
    pinned.numpy()[:] = np.frombuffer(src, dtype=np.uint8)
    for q in ["count", "sum(.v)", "select(.v > 390) | {v: .v, k: .k}"]:
        want = orc.run(q, nd).out
        for data in (src, pinned.numpy()):
            Q = wjq.Query(q, chunk_bytes=1 << 20)
            r = Q.run_csv(data)
            assert r.rc == 0, r.err
            assert r.out == want, (q, r.out[:200], want[:200])
            Q.close()
