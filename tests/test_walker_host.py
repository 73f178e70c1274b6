"""The device line walkers (the bounded walk_line and the window walker
walk_masked, with its object fast path walk_objects) and evaluator (warpjq_b200/csrc/walker.cuh), compiled for the
host, against the oracle's per-line semantics
(exec/cpu.rs:299-371): same verdict per line -- blank, invalid, type error,
filtered, selected -- and, for selected lines, the same resolved value of
every needed path (kind, raw bytes, and the correctly rounded number)."""

import ctypes
import os
import subprocess

import pytest

from oracle import pyoracle as orc
from tests import corpus

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "native", "walker_host.cc")
OUT = os.path.join(HERE, "native", "_build", "libwalker_host.so")


@pytest.fixture(scope="module")
def harness():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    deps = [SRC] + [os.path.join(ROOT, "warpjq_b200", "csrc", f)
                    for f in ("walker.cuh", "devutil.cuh", "plan.h", "plan_build.h")]
    if not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in deps):
        subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-o", OUT, SRC,
                        os.path.join(ROOT, "warpjq_b200", "csrc", "host", "query.cc")], check=True)
    L = ctypes.CDLL(OUT)
    L.wh_eval.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_int,
                          ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]
    L.wh_free.argtypes = [ctypes.c_void_p]
    o = orc.lib()
    o.oracle_eval_lines.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t,
                                    ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t)]
    return L, o


def _run(fn, free, query, data, *mode):
    p = ctypes.c_void_p()
    n = ctypes.c_size_t()
    rc = fn(query.encode(), data, len(data), *mode, ctypes.byref(p), ctypes.byref(n))
    assert rc == 0, (query, rc)
    out = ctypes.string_at(p.value, n.value) if p.value else b""
    free(p)
    return out.split(b"\n")


def check(harness, data, queries, label):
    L, o = harness
    for q in queries:
        ref = _run(o.oracle_eval_lines, o.oracle_free, q, data)
        for mode, name in ((0, "walk_line"), (1, "walk_masked"), (2, "walk_objects")):
            dev = _run(L.wh_eval, L.wh_free, q, data, mode)
            assert len(dev) == len(ref), (label, q, name)
            for i, (a, b) in enumerate(zip(dev, ref)):
                assert a == b, f"{label}: `{q}` line {i} ({name}):\n walker: {a[:300]!r}\n oracle: {b[:300]!r}"


def test_walker_on_hostile_corpora(harness, golden):
    check(harness, corpus.corpus(1, 1500), golden["diff_queries"], "clean")
    check(harness, corpus.corpus(2, 1500, 0.15), golden["diff_queries"], "malformed")
    check(harness, corpus.corpus(3, 600, 0.05, crlf=True), golden["diff_queries"], "crlf")
    check(harness, corpus.corpus(4, 300, 1.0), golden["diff_queries"], "all malformed")
    check(harness, corpus.edge_corpus(), golden["diff_queries"], "edge")


def test_walker_on_conformance_documents(harness, golden):
    docs = [c["doc"] for c in golden["must_accept"] + golden["must_reject"] + golden["implementation_defined"]]
    docs += golden["json_reject"] + golden["json_accept"] + golden["json_truncated"] + golden["json_mismatched"]
    data = ("\n".join(d for d in docs if "\n" not in d) + "\n").encode()
    check(harness, data, [".", ".a", ".a[0]", "select(.a)", '{x: .a, y: .b}'], "conformance")


def test_walker_on_lookup_vectors(harness, golden):
    for c in golden["lookup"]:
        check(harness, (c["line"] + "\n").encode(), [c["path"]], "lookup")
    for c in golden["select"]:
        check(harness, (c["line"] + "\n").encode(), [c["query"]], "select")


def test_walker_on_deep_and_odd_structure(harness):
    lines = [
        b"[" * 70 + b"]" * 70, b"[" * 70 + b"]" * 69, b'{"a":' * 80 + b"1" + b"}" * 80,
        b'{"a":[1,{"b":[2,3,{"c":4}]}],"a":{"b":5}}', b'{"a":{"b":1},"a":5}', b'{"a":5,"a":{"b":1}}',
        b'{"a":[10,20,30]}', b'{"a":[]}', b'{"a":[[1,2],[3,4]]}', b'[{"a":1}]', b'"str"', b"5",
        b'{"a":null}', b'{"a":{"b":null}}', b'{"\\u0061":1}', b'{"a":"\\u00e9","b":"\\ud83d\\ude00"}',
        b' \x0c ', b'\x0c{}', b'{"a":1}\r', b'{"a":1} \t\r', b'{"a": 1 , "b" : [ 1 , 2 ] }',
        b'{"a":1e400,"b":-1e-400,"c":123456789012345678901234567890}', b'{"a":-0.0}',
        b'{"a":0.1e1}', b'{"a":1E+2}', b'{"a":2.2250738585072011e-308}', b'{"a":9007199254740993}',
    ]
    data = b"\n".join(lines) + b"\n"
    check(harness, data, [".", ".a", ".a.b", ".a[1]", ".a[1].b[2].c", ".a[0][1]", "select(.a > 1)",
                          "select(.a == 100)", '{a: .a, b: .b, c: .c}', "select(.a.b)", ".a.b.c"], "deep/odd")


def test_walker_number_parsing_is_correctly_rounded(harness):
    import random
    rng = random.Random(5)
    vals = []
    for _ in range(3000):
        k = rng.randrange(6)
        if k == 0:
            vals.append(str(rng.randrange(-10**18, 10**18)))
        elif k == 1:
            vals.append(f"{rng.random() * 10 ** rng.randrange(-30, 30):.{rng.randrange(1, 20)}e}")
        elif k == 2:
            vals.append("0." + "".join(rng.choice("0123456789") for _ in range(rng.randrange(1, 40))))
        elif k == 3:
            vals.append(str(rng.randrange(1, 10)) + "e" + str(rng.randrange(-330, 310)))
        elif k == 4:
            d = "".join(rng.choice("0123456789") for _ in range(rng.randrange(16, 60)))
            vals.append(d.lstrip("0") or "0")
        else:
            # halfway-style cases: 2^k +- tiny
            vals.append(repr(2.0 ** rng.randrange(-1000, 1000)) + "1")
    data = "".join('{"a":%s}\n' % v for v in vals).encode()
    check(harness, data, [".a", "select(.a > 0)"], "numbers")


def test_walker_on_mutated_lines(harness):
    """Random byte edits of valid lines: backslash runs of every length at
    every alignment, truncated literals and numbers, stray structure, raw
    control bytes inside strings."""
    import random
    rng = random.Random(17)
    base = corpus.corpus(9, 400).split(b"\n")[:-1]
    base += [b'{"a":"' + b"\\" * k + b'","b":"x' + b"\\\\" * k + b'"}' for k in range(1, 12)]
    base += [b'{"a":"' + b"y" * k + b'\\"' + b"z" * (k % 5) + b'"}' for k in range(40)]
    alphabet = list(b'"\\{}[]:,0123456789.eE+-tfnrulsa \t\r\x0c\x01\x1f\x7f') + [0xC3, 0xA9]
    lines = []
    for _ in range(4000):
        b = bytearray(rng.choice(base))
        for _ in range(rng.randrange(1, 4)):
            k = rng.randrange(3)
            at = rng.randrange(len(b) + 1)
            if k == 0:
                b[at:at] = bytes([rng.choice(alphabet)])
            elif k == 1 and at < len(b):
                del b[at]
            elif at < len(b):
                b[at] = rng.choice(alphabet)
        lines.append(bytes(b).replace(b"\n", b" "))
    data = b"\n".join(lines) + b"\n"
    check(harness, data, [".", ".a", ".status", "select(.a)", '{a: .a, b: .b}', ".arr[1]",
                          ".nested.deep.v"], "mutated")


def test_walker_on_the_benchmark_schemas(harness):
    """The object fast path's common shapes: nginx-style lines (escaped
    quotes and backslashes in ua) and the nested schema (objects 3-5 deep,
    \\u escapes, malformed lines), as generated and with random edits, under
    the benchmark queries."""
    import random
    import warpjq_b200 as wjq
    nb, nu, _ = wjq.gen_nginx(400_000, seed=4)
    sb, su, _ = wjq.gen_nested(400_000, seed=4, n_users=1000)
    nginx = bytes(nb[:nu]).split(b"\n")[:-1]
    nested = bytes(sb[:su]).split(b"\n")[:-1]
    rng = random.Random(23)
    mutated = []
    for _ in range(2000):
        b = bytearray(rng.choice(nginx + nested))
        at = rng.randrange(len(b))
        b[at] = rng.choice(b'"\\{}[]:, \x01ua0')
        mutated.append(bytes(b).replace(b"\n", b" "))
    check(harness, b"\n".join(nginx + mutated) + b"\n",
          ["select(.status == 500) | count", "select(.status >= 500) | {p: .path, b: .bytes}",
           "group_by(.host) | sum(.bytes)", ".ua", "select(.latency_ms > 50) | .method"], "nginx")
    check(harness, b"\n".join(nested + mutated) + b"\n",
          ['select(.req.user.tier == "gold" and .resp.code != 200) | {u: .req.user.id, l: .resp.latency}',
           "group_by(.req.user.id) | avg(.resp.latency)", ".req.path", ".meta.trace.span",
           "select(.req.user.geo.cc == \"jp\") | {c: .req.user.geo, m: .req.method}"], "nested")
