"""Running over a file (warpjq_query_run_file): chunks read with parallel
preads into page-locked buffers, cut after the last newline with the partial
line carried into the next chunk.  Output must equal the oracle's over the
file's bytes: with a byte-order mark, without a final newline, with a line
longer than a chunk (the buffers and the device context grow), and on an
empty file."""

import os
import tempfile

import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc
from tests import corpus

pytestmark = pytest.mark.gpu

QUERIES = ["select(.status == 500) | count", "group_by(.host) | sum(.bytes)",
           "select(.status >= 500) | {p: .path, b: .bytes}", ".a", "count"]


def check(data: bytes, chunk_bytes: int):
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "in.ndjson")
        with open(path, "wb") as f:
            f.write(data)
        for q in QUERIES:
            Q = wjq.Query(q, chunk_bytes=chunk_bytes)
            got = Q.run_file(path)
            want = orc.run(q, data)
            assert got.rc == 0, got.err
            assert got.out == want.out, (q, got.out[:200], want.out[:200])
            assert got.stats["malformed"] == want.stats["malformed"], q
            assert got.stats["lines_in"] == want.stats["lines_in"], q
            Q.close()


def test_file_input_matches_the_oracle():
    buf, used, _ = wjq.gen_nginx(6 << 20, seed=13)
    nginx = bytes(buf[:used])
    check(nginx, 1 << 20)                                    # many chunks, carried lines
    check(b"\xef\xbb\xbf" + nginx[:200000] + b'{"a":1}', 1 << 20)  # BOM, no final newline
    check(corpus.corpus(7, 2000, 0.1) + b"\n\n", 1 << 20)
    long_line = b'{"a":"' + b"y" * (3 << 20) + b'","status":500}\n'
    check(nginx[:100000] + long_line + nginx[100000:300000], 1 << 20)  # a 3 MB line


def test_file_input_strict_mode_names_the_file_and_empty_file():
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "bad.ndjson")
        with open(path, "wb") as f:
            f.write(b'{"a":1}\n{oops\n')
        r = wjq.Query(".a").run_file(path, on_invalid="abort")
        assert r.rc == 1 and "line 2" in r.err and "bad.ndjson" in r.err, r.err
        empty = os.path.join(d, "empty.ndjson")
        open(empty, "wb").close()
        r = wjq.Query("count").run_file(empty)
        assert r.rc == 0 and r.out == orc.run("count", b"").out
        r = wjq.Query("count").run_file(os.path.join(d, "missing"))
        assert r.rc == 1 and "cannot open" in r.err
