"""Pins the oracle (the CPU restatement of the reference engine) to the
reference project's own test vectors before anything is checked against it.

Each test names the reference test it restates.
"""

import math

import pytest

from oracle import pyoracle as orc


# conformance.rs:234-276
def test_scanner_accepts_every_valid_document(golden):
    bad = [c["name"] for c in golden["must_accept"] if not orc.validate(c["doc"].encode())[0]]
    assert not bad, bad


def test_scanner_rejects_every_invalid_document(golden):
    bad = [c["name"] for c in golden["must_reject"] if orc.validate(c["doc"].encode())[0]]
    assert not bad, bad


def test_implementation_defined_behaviour_is_pinned(golden):
    for c in golden["implementation_defined"]:
        assert orc.validate(c["doc"].encode())[0] == c["accept"], c["name"]


def test_every_error_carries_an_offset_inside_the_input(golden):  # conformance.rs:278-294
    for c in golden["must_reject"]:
        ok, off, detail = orc.validate(c["doc"].encode())
        assert not ok
        assert off <= len(c["doc"].encode()), c["name"]
        assert detail, c["name"]


# conformance.rs:300-334: through the whole pipeline under --strict
def test_pipeline_agrees_with_the_scanner(golden):
    for c in golden["must_accept"]:
        r = orc.run(".", (c["doc"] + "\n").encode(), on_invalid="abort", chunk_bytes=1 << 16, threads=1)
        assert r.rc == 0, (c["name"], r.err)
    for c in golden["must_reject"]:
        if not c["doc"].strip():
            continue
        r = orc.run(".", (c["doc"] + "\n").encode(), on_invalid="abort", chunk_bytes=1 << 16, threads=1)
        assert r.rc == 1, c["name"]


# json.rs:798-920
def test_json_unit_vectors(golden):
    for d in golden["json_reject"] + golden["json_truncated"] + golden["json_mismatched"]:
        assert not orc.validate(d.encode())[0], d
    for d in golden["json_accept"]:
        assert orc.validate(d.encode())[0], d


def test_deep_nesting_is_iterative():  # json.rs:861-884
    for n in (1000, 100_000, 1_000_000):
        assert orc.validate(b"[" * n + b"]" * n)[0]
        assert not orc.validate(b"[" * n)[0]
        assert orc.validate(b'{"a":' * n + b"1" + b"}" * n)[0]


def test_lookup_through_deep_nesting():  # json.rs:886-896
    n = 200_000
    line = b'{"a":' + b"[" * n + b"]" * n + b',"b":7}'
    assert orc.lookup(line, ".b") == ("found", "num", b"7")


def test_lookup_vectors(golden):  # json.rs:715-796
    for c in golden["lookup"]:
        outcome, kind, raw = orc.lookup(c["line"].encode(), c["path"])
        if c["outcome"] == "type_error":
            assert outcome == "type_error", c
        else:
            assert outcome == "found", c
            assert kind == c["outcome"], c
            assert raw == c["raw"].encode(), c


def test_select_vectors(golden):  # json.rs:922-958
    for c in golden["select"]:
        assert orc.eval_select(c["line"].encode(), c["query"]) == c["verdict"], c


# exec/cpu.rs:545-707
def test_cpu_engine_known_answers(golden):
    log = golden["cpu_log"].encode()
    for c in golden["cpu_log_cases"]:
        r = orc.run(c["query"], log, fmt=c["format"], chunk_bytes=64, threads=4)
        assert r.rc == 0, r
        assert r.out == c["expected"].encode(), c["query"]


def test_cpu_engine_empty_input(golden):
    for c in golden["cpu_empty_cases"]:
        r = orc.run(c["query"], b"", chunk_bytes=64, threads=4)
        assert r.out == c["expected"].encode(), c


def test_cpu_engine_misc(golden):
    for c in golden["cpu_misc_cases"]:
        r = orc.run(c["query"], c["input"].encode(), on_invalid=c["on_invalid"], chunk_bytes=64, threads=4)
        assert r.rc == 0 and r.out == c["expected"].encode(), (c, r)
        for k, v in c["stats"].items():
            assert r.stats[k] == v, (c, r.stats)


def test_strict_mode_names_the_line():  # exec/cpu.rs:651-664
    r = orc.run(".a", b'{"a":1}\n{oops\n', on_invalid="abort")
    assert r.rc == 1 and "on line 2" in r.err


def test_output_order_is_input_order_regardless_of_slicing():  # exec/cpu.rs:623-635
    data = "".join(f'{{"i":{i}}}\n' for i in range(2000)).encode()
    r = orc.run(".i", data, chunk_bytes=64, threads=4)
    assert r.out.decode().splitlines() == [str(i) for i in range(2000)]


# agg.rs:400-410
def test_format_number(golden):
    for c in golden["format_number"]:
        assert orc.format_number(c["value"]) == c["expected"], c
    for v in golden["format_number_contains_e"]:
        assert "e" in orc.format_number(v)


def test_format_number_ryu_placement():
    # The ryu crate's pretty printer: fixed notation while the decimal point
    # lands within 16 digits, scientific beyond (agg.rs:271-277).
    assert orc.format_number(2.0 ** 53) == "9007199254740992.0"
    assert orc.format_number(1e16) == "1e+16"
    assert orc.format_number(0.001234) == "0.001234"
    assert orc.format_number(1.234e-7) == "1.234e-7"
    assert orc.format_number(123.456) == "123.456"
    assert orc.format_number(-2.5) == "-2.5"
    assert orc.format_number(math.inf) == "1.7976931348623157e+308"
    assert orc.format_number(math.nan) == "null"


# query/lex.rs:370-465 and query/mod.rs:320-431
def test_lexer_numbers(golden):
    for c in golden["lex_first_token"]:
        rc, prog = orc.parse(f"select(.a == {c['query']})")
        assert rc == 0, c
        kind, val = c["token"].split(":")
        assert prog["filter"]["cmp"]["lit"]["num"] == float(val), c


def test_query_errors(golden):
    for c in golden["query_errors"]:
        rc, info = orc.parse(c["query"])
        assert rc == 2, c
        assert c["contains"] in info["error"] + info["rendered"], (c, info)


def test_parser_shapes():  # query/mod.rs:227-458
    assert orc.parse(".")[1]["output"] == "passthrough"
    p = orc.parse(".a.b[2].c")[1]
    assert p["paths"][0] == ["a", "b", 2, "c"]
    assert orc.parse('."content-type"')[1]["paths"][0] == ["content-type"]
    p = orc.parse("select(.a == 1) | select(.b == 2)")[1]
    assert "and" in p["filter"]
    p = orc.parse("select(.a == 1 or .b == 2 and .c == 3)")[1]
    assert "and" in p["filter"]["or"][1]
    p = orc.parse("{time: .ts, msg}")[1]
    assert p["output"]["project"][1][0] == "msg"
    assert orc.parse("select(.ok | not)")[1]["filter"].keys() == {"not"}
    assert len(orc.parse("select(.a == 1 or .a == 2) | {x: .a}")[1]["paths"]) == 1
    f = orc.parse("select((.a == 1 and .b == 2) or .c == 3)")[1]["flat"]
    assert len(f["cmps"]) == 3 and len(f["cond_rpn"]) == 5
    assert f["cond_rpn"][2][0] == 2 and f["cond_rpn"][4][0] == 3 and f["cond_stack_depth"] == 2
    f = orc.parse('select(.method == "POST")')[1]["flat"]
    c = f["cmps"][0]
    assert c[2] == 4 and f["blob"][c[3]:c[3] + c[4]] == "POST"
    for q in ["group_by(.host)", "group_by(.host) | {a: .b}", "count | count", "{a: .b} | {c: .d}"]:
        assert orc.parse(q)[0] == 2, q
    for depth in (100, 1000, 10000):
        assert orc.parse("select(" + "(" * depth)[0] == 2
    assert orc.parse("select(" + "(" * 500 + ".a == 1" + ")" * 500 + ")")[0] == 2
    for depth in (1, 8, 32, 64):
        assert orc.parse("select(" + "(" * depth + ".a == 1" + ")" * depth + ")")[0] == 0
    rc, e = orc.parse("select(status == 500)")
    assert rc == 2 and e["hint"] == "did you mean `.status`?"
    assert orc.parse('select(.msg == "a|b")')[0] == 0
    assert orc.parse("select(.a == 1 or (.b == 2))")[0] == 0
    for q in ["reduce", "map", "if", "def", "test", "length", "select(.a == 1) | map(.b)",
              '.a | test("x")', "select(.a == 1) | keys"]:
        rc, e = orc.parse(q)
        assert rc == 2 and ("not in the v0.1 subset" in e["error"] or "roadmap" in e["error"]), q


def test_csv_and_json_string_rendering(golden):
    for c in golden["csv_cell"]:
        # A one-field CSV projection renders exactly one cell (output.rs:45-61).
        line = ('{"a":' + __import__("json").dumps(c["input"]) + "}\n").encode()
        r = orc.run("{a: .a}", line, fmt="csv")
        assert r.out == ("a\n" + c["expected"] + "\n").encode(), c
    for c in golden["json_string"]:
        # A group key renders through write_json_string (agg.rs:164-168).
        line = ('{"k":' + __import__("json").dumps(c["input"]) + "}\n").encode()
        r = orc.run("group_by(.k) | count", line)
        assert r.out == ('{"k":' + c["expected"] + ',"count":1}\n').encode(), c


def test_group_keys_sort_in_jq_order():  # agg.rs:334-398
    data = b'{"k":"b"}\n{"k":10}\n{"k":null}\n{"k":"a"}\n{"k":true}\n{"k":2}\n{"k":false}\n{"k":-5}\n'
    r = orc.run("group_by(.k) | count", data)
    keys = [ln.split(",")[0][5:] for ln in r.out.decode().splitlines()]
    assert keys == ["null", "false", "true", "-5", "2", "10", '"a"', '"b"']


def test_chunk_size_and_threads_do_not_change_output(golden):  # invariants.rs:97-199
    data = golden["cpu_log"].encode() * 50
    for q in golden["invariant_queries"]:
        base = orc.run(q, data, chunk_bytes=1 << 20, threads=4).out
        for cb in (1, 7, 61, 997, 4096):
            assert orc.run(q, data, chunk_bytes=cb, threads=4).out == base, (q, cb)
        for t in (1, 3, 8):
            assert orc.run(q, data, threads=t).out == base, (q, t)
