"""GPU parity: the sm_100a backend, driven through the C ABI by the host
driver, must produce exactly the oracle's bytes (the oracle restates the
reference CPU engine, which the reference's own differential tests treat as
ground truth, crates/warpjq-core/tests/differential.rs:339-371)."""

import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc
from tests import corpus

pytestmark = pytest.mark.gpu

FORMATS = ["ndjson", "csv", "count"]


def csv_ok(query):
    rc, p = orc.parse(query)
    return rc == 0 and p["output"] != "passthrough"


def close_enough(a: bytes, b: bytes, rel=1e-9) -> bool:
    """Row-by-row equality, except that numbers may differ by `rel` (FP sums
    of fractional values: the reference adds in line order, this backend in a
    fixed tree order)."""
    import re
    la, lb = a.split(b"\n"), b.split(b"\n")
    if len(la) != len(lb):
        return False
    num = re.compile(rb"-?\d+(?:\.\d+)?(?:[eE][+-]?\d+)?")
    for x, y in zip(la, lb):
        if x == y:
            continue
        if num.sub(b"#", x) != num.sub(b"#", y):
            return False
        for u, v in zip(num.findall(x), num.findall(y)):
            fu, fv = float(u), float(v)
            if abs(fu - fv) > rel * max(abs(fu), abs(fv), 1e-300):
                return False
    return True


def agree(data, queries, label, chunk_bytes=1 << 16, formats=FORMATS, on_invalid="skip",
          fractional=()):
    checked = 0
    for q in queries:
        for f in formats:
            if f == "csv" and not csv_ok(q):
                continue
            want = orc.run(q, data, fmt=f, on_invalid=on_invalid, chunk_bytes=chunk_bytes, threads=4)
            got = wjq.run_bytes(q, data, fmt=f, on_invalid=on_invalid, chunk_bytes=chunk_bytes)
            assert got.rc == want.rc, (label, q, f, got.err, want.err)
            if want.rc == 0:
                if q in fractional and close_enough(got.out, want.out):
                    pass
                elif got.out != want.out:
                    gl, wl = got.out.split(b"\n"), want.out.split(b"\n")
                    for i, (a, b) in enumerate(zip(gl, wl)):
                        if a != b:
                            break
                    raise AssertionError(f"{label}: `{q}` [{f}] differs at row {i}:\n gpu: {a[:200]!r}\n cpu: {b[:200]!r}"
                                         f"\n gpu rows {len(gl)} cpu rows {len(wl)}")
                for k in ("lines_in", "malformed", "type_errors", "lines_out"):
                    assert got.stats[k] == want.stats[k], (label, q, f, k, got.stats, want.stats)
            checked += 1
    return checked


@pytest.fixture(scope="module", autouse=True)
def device():
    why = wjq.probe()
    if why:
        pytest.fail(f"no usable B200: {why}")


def test_known_answers(golden):  # exec/cpu.rs:545-707
    log = golden["cpu_log"].encode()
    for c in golden["cpu_log_cases"]:
        r = wjq.run_bytes(c["query"], log, fmt=c["format"], chunk_bytes=64)
        assert r.rc == 0, r.err
        assert r.out == c["expected"].encode(), c["query"]
    for c in golden["cpu_empty_cases"]:
        assert wjq.run_bytes(c["query"], b"").out == c["expected"].encode(), c


def test_conformance_verdicts(golden):  # conformance.rs:300-358
    docs = golden["must_accept"] + golden["must_reject"] + golden["implementation_defined"]
    for c in docs:
        if not c["doc"].strip():
            continue
        line = (c["doc"] + "\n").encode()
        cpu = orc.run(".", line, on_invalid="abort", threads=1).rc
        gpu = wjq.run_bytes(".", line, on_invalid="abort").rc
        assert cpu == gpu, c["name"]


def test_backends_agree_on_hostile_input(golden):
    assert agree(corpus.corpus(1, 4000), golden["diff_queries"], "clean") > 0


def test_backends_agree_with_malformed_lines_mixed_in(golden):
    agree(corpus.corpus(2, 4000, 0.15), golden["diff_queries"], "15% malformed")


def test_backends_agree_on_crlf_input(golden):
    agree(corpus.corpus(3, 2000, 0.05, crlf=True), golden["diff_queries"], "crlf")


def test_backends_agree_across_many_seeds(golden):
    for seed in range(10, 16):
        agree(corpus.corpus(seed, 800, 0.08), golden["diff_queries"], f"seed {seed}")


def test_backends_agree_on_edge_case_corpus(golden):
    agree(corpus.edge_corpus(), golden["diff_queries"], "edge cases")


def test_backends_agree_when_every_line_is_malformed(golden):
    agree(corpus.corpus(4, 500, 1.0), golden["diff_queries"], "all malformed")


def test_projection_expanding_past_the_output_buffer():  # differential.rs:442-479
    data = "".join(f'{{"a":{1_000_000_000 + i}}}\n' for i in range(40_000)).encode()
    q = "{alpha: .a, bravo: .a, charlie: .a, delta: .a, echo: .a, foxtrot: .a}"
    agree(data, [q], "expansion", formats=["ndjson"])


def test_deeply_nested_lines(golden):  # differential.rs:520-533
    data = b'{"a":1}\n' + b'{"a":' + b"[" * 5000 + b"]" * 5000 + b'}\n{"a":2}\n'
    agree(data, golden["diff_queries"], "deep")
    deeper = b'{"a":' + b"[" * 100_000 + b"]" * 100_000 + b'}\n' + b"[" * 70 + b"]" * 69 + b"\n"
    agree(deeper, [".", "count", ".a", "select(.a)"], "deeper", formats=["ndjson"])


def test_empty_and_tiny_input(golden):  # differential.rs:535-546
    for data in [b"", b"\n", b"{}\n", b"{}", b"\n\n\n"]:
        agree(data, golden["diff_queries"], repr(data))


def test_lines_longer_than_a_tile():
    long = "x" * 200_000
    data = ('{"a":1}\n{"a":"' + long + '","b":2}\n{"b":3}\n' + '{"a":"' + long[:40000] + '"}\n').encode()
    agree(data, [".", ".b", "count", "select(.b >= 2)", "{b: .b}", "group_by(.b) | count"], "long")


def test_invariant_queries_independent_of_chunk_size(golden):  # invariants.rs:97-138
    data = corpus.corpus(21, 1500, 0.05)
    for cb in (1, 7, 997, 1 << 20):
        agree(data, golden["invariant_queries"], f"chunk {cb}", chunk_bytes=cb, formats=["ndjson"])


def test_strict_mode_names_the_first_bad_line():
    data = b'{"a":1}\n\n{"a":{"b":1}}\n{oops\n'
    for q in (".a", ".a.b"):
        g = wjq.run_bytes(q, data, on_invalid="abort")
        c = orc.run(q, data, on_invalid="abort")
        assert g.rc == c.rc == 1
        line = c.err.split("on line ")[1].split(" ")[0]
        assert f"on line {line} " in g.err, (g.err, c.err)


def test_nginx_benchmark_queries():
    buf, used, _ = wjq.gen_nginx(8 << 20, seed=3)
    data = bytes(buf[:used])
    qs = ["select(.status == 500) | count", "select(.status >= 500) | {p: .path, b: .bytes}",
          "group_by(.host) | sum(.bytes)", "select(.status == 500)", "sum(.bytes)", "avg(.latency_ms)",
          "max(.latency_ms)", "min(.bytes)", "group_by(.path) | count", "group_by(.status) | avg(.bytes)"]
    agree(data, qs, "nginx", chunk_bytes=1 << 22, fractional={"avg(.latency_ms)"})


def test_contexts_with_different_tilings_interleave():
    """Several live queries with different tile sizes and shared-memory needs
    (a grouped aggregate keeps a per-CTA key cache) launched in turn: each
    context's launches must stay valid after the others are configured."""
    import numpy as np
    buf, used, _ = wjq.gen_nginx(4 << 20, seed=5)
    data = bytes(buf[:used])
    qs = [wjq.Query("group_by(.host) | sum(.bytes)"), wjq.Query("select(.status == 500) | count"),
          wjq.Query("select(.status == 500)")]
    qs[0].autotile(np.frombuffer(data[: 1 << 20], dtype=np.uint8))
    qs[1].set_tiling(4096, 1024)
    qs[2].set_tiling(12288, 2048)
    for _ in range(2):
        for q in qs:
            r = q.run(data)
            assert r.rc == 0, r.err
            c = orc.run(q.query, data)
            assert r.out == c.out, q.query


NESTED_QUERIES = [
    'select(.req.user.tier == "gold" and .resp.code != 200) | {u: .req.user.id, l: .resp.latency}',
    "group_by(.req.user.id) | avg(.resp.latency)", "group_by(.req.user.tier) | count",
    "select(.meta.trace.span.depth > 5) | .req.path", "max(.resp.latency)", "sum(.resp.size)",
    "select(.req.user.geo.cc == \"jp\") | {c: .req.user.geo, m: .req.method}",
]


def test_nested_dirty_schema_queries():
    """The nested, dirty workload (objects 3-5 levels deep, shuffled keys,
    escapes, mixed number forms, ~2% malformed lines): host path with small
    chunks, in all output formats."""
    buf, used, _ = wjq.gen_nested(6 << 20, seed=21, n_users=50_000)
    agree(bytes(buf[:used]), NESTED_QUERIES, "nested",
          fractional={"group_by(.req.user.id) | avg(.resp.latency)"})


def test_group_table_grows_past_its_first_size():
    """group_by over ~77k distinct ids in one chunk: more keys than the
    table's first size, so the run grows the table and repeats on the device;
    the host and device-resident paths both match the oracle."""
    import torch
    buf, used, _ = wjq.gen_nested(40 << 20, seed=22, n_users=1_000_000)
    data = bytes(buf[:used])
    q = "group_by(.req.user.id) | avg(.resp.latency)"
    want = orc.run(q, data)
    got = wjq.run_bytes(q, data, chunk_bytes=64 << 20)
    assert got.rc == 0 and close_enough(got.out, want.out)
    assert want.out.count(b"\n") > 1 << 16  # more groups than the table's first 65,536 keys
    Q = wjq.Query(q)
    dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
    dev[:len(data)].copy_(torch.frombuffer(bytearray(data), dtype=torch.uint8))
    Q.launch_device(dev.data_ptr(), len(data), torch.cuda.current_stream().cuda_stream)
    r = Q.collect_device()
    assert close_enough(Q.render_device(r, data), want.out)
    Q.close()
