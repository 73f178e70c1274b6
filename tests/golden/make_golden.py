"""Generates tests/golden/reference_vectors.json from the reference project's
own Rust test sources.

Run in a checkout that has the reference project next to it:

    python tests/golden/make_golden.py --reference /path/to/warpjq

List-shaped corpora (the JSON conformance tables, the edge-case lines, the
query matrices) are extracted mechanically by decoding the Rust string
literals in place.  Known-answer expectations that live inside test bodies
are transcribed below with their file:line, and the script refuses to write
any transcribed case whose literal text it cannot find in the cited file, so a
fixture can only ever restate what the reference's tests assert.

Only this generator reads the reference tree; the fixture it writes is
self-contained and is what the tests load.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import sys

# ---------------------------------------------------------------------------
# Rust literal decoding
# ---------------------------------------------------------------------------


def _decode_escapes(body: str) -> str:
    out = []
    i = 0
    while i < len(body):
        c = body[i]
        if c != "\\":
            out.append(c)
            i += 1
            continue
        e = body[i + 1]
        if e == "n":
            out.append("\n")
            i += 2
        elif e == "t":
            out.append("\t")
            i += 2
        elif e == "r":
            out.append("\r")
            i += 2
        elif e == "0":
            out.append("\0")
            i += 2
        elif e in "\\\"'":
            out.append(e)
            i += 2
        elif e == "x":
            out.append(chr(int(body[i + 2 : i + 4], 16)))
            i += 4
        elif e == "u":
            j = body.index("}", i)
            out.append(chr(int(body[i + 3 : j], 16)))
            i = j + 1
        elif e == "\n":
            # Line continuation: skip the newline and leading whitespace.
            i += 2
            while i < len(body) and body[i] in " \t\n":
                i += 1
        else:
            raise ValueError(f"unknown escape \\{e}")
    return "".join(out)


TOKEN_RE = re.compile(
    r"""
    (?P<raw>b?r(?P<hashes>\#*)")            # raw string start
  | (?P<str>b?")                            # normal string start
  | (?P<word>[A-Za-z_][A-Za-z0-9_]*!?)
  | (?P<num>-?\d+(?:\.\d+)?)
  | (?P<punct>[()\[\],;])
  | (?P<comment>//[^\n]*)
  | (?P<ws>\s+)
  | (?P<other>.)
    """,
    re.VERBOSE | re.DOTALL,
)


def tokenize(src: str):
    """Yields ('str', value) / ('word', w) / ('num', n) / ('p', c) tokens."""
    i = 0
    while i < len(src):
        m = TOKEN_RE.match(src, i)
        if not m:
            raise ValueError(f"cannot tokenize at {src[i:i+30]!r}")
        if m.group("raw") is not None:
            hashes = m.group("hashes")
            start = m.end()
            end = src.index('"' + hashes, start)
            yield ("str", src[start:end])
            i = end + 1 + len(hashes)
            continue
        if m.group("str") is not None:
            j = m.end()
            while src[j] != '"':
                j += 2 if src[j] == "\\" else 1
            yield ("str", _decode_escapes(src[m.end() : j]))
            i = j + 1
            continue
        if m.group("word") is not None:
            yield ("word", m.group("word"))
        elif m.group("num") is not None:
            yield ("num", m.group("num"))
        elif m.group("punct") is not None:
            yield ("p", m.group("punct"))
        elif m.group("other") is not None:
            yield ("other", m.group("other"))
        i = m.end()


def fold_concat(tokens):
    """Replaces `concat!(lit, lit, ...)` by one string token."""
    out = []
    k = 0
    while k < len(tokens):
        t = tokens[k]
        if t == ("word", "concat!") and tokens[k + 1] == ("p", "("):
            depth = 0
            parts = []
            k += 1
            while True:
                t2 = tokens[k]
                if t2 == ("p", "("):
                    depth += 1
                elif t2 == ("p", ")"):
                    depth -= 1
                    if depth == 0:
                        break
                elif t2[0] == "str":
                    parts.append(t2[1])
                k += 1
            out.append(("str", "".join(parts)))
            k += 1
            continue
        out.append(t)
        k += 1
    return out


def region(src: str, start_pat: str, end_pat: str = "\n];") -> str:
    a = src.index(start_pat) + len(start_pat)
    b = src.index(end_pat, a)
    return src[a:b]


def tuples(text: str):
    """Parses `(a, b, ...)` tuples of literals/bools out of a list body."""
    toks = fold_concat(list(tokenize(text)))
    toks = [t for t in toks if t[0] != "other" or t[1] not in "&"]
    res, cur, depth = [], None, 0
    for kind, v in toks:
        if (kind, v) == ("p", "("):
            depth += 1
            if depth == 1:
                cur = []
            continue
        if (kind, v) == ("p", ")"):
            depth -= 1
            if depth == 0:
                res.append(cur)
            continue
        if depth >= 1:
            if kind == "str":
                cur.append(v)
            elif kind == "word" and v in ("true", "false"):
                cur.append(v == "true")
    return res


def strings(text: str):
    toks = fold_concat(list(tokenize(text)))
    return [v for k, v in toks if k == "str"]


# ---------------------------------------------------------------------------
# Transcribed known-answer expectations, each checked against its source.
# ---------------------------------------------------------------------------

CPU_LOG_CASES = [
    # (query, format, expected output)   exec/cpu.rs:545-706
    (".", "ndjson", None),  # None: the LOG input itself (cpu.rs:547)
    ("select(.status == 500)", "ndjson",
     '{"status":500,"bytes":20,"host":"b","msg":"boom"}\n'
     '{"status":500,"bytes":30,"host":"a","msg":"boom again"}\n'),
    ("select(.status == 500) | count", "ndjson", "2\n"),
    ("count", "ndjson", "4\n"),
    ("select(.status==404) | {h: .host, s: .status}", "ndjson", '{"h":"c","s":404}\n'),
    ("select(.status==404) | {m: .msg}", "ndjson", '{"m":null}\n'),
    ("sum(.bytes)", "ndjson", "100\n"),
    ("min(.bytes)", "ndjson", "10\n"),
    ("max(.bytes)", "ndjson", "40\n"),
    ("avg(.bytes)", "ndjson", "25\n"),
    ("select(.status==500) | sum(.bytes)", "ndjson", "50\n"),
    ("group_by(.host) | count", "ndjson",
     '{"host":"a","count":2}\n{"host":"b","count":1}\n{"host":"c","count":1}\n'),
    ("group_by(.host) | sum(.bytes)", "ndjson",
     '{"host":"a","sum":40}\n{"host":"b","sum":20}\n{"host":"c","sum":40}\n'),
    ("{h: .host, s: .status}", "csv", "h,s\na,200\nb,500\na,500\nc,404\n"),
    ("select(.status == 500)", "count", "2\n"),
    ("select(.status == 200 or .status == 404) | count", "ndjson", "2\n"),
    ("select(.status == 500 | not) | count", "ndjson", "2\n"),
]

CPU_EMPTY_CASES = [  # exec/cpu.rs:693-701
    (".", ""), ("count", "0\n"), ("sum(.x)", "0\n"), ("min(.x)", "null\n"),
    ("avg(.x)", "null\n"), ("group_by(.h) | count", ""),
]

CPU_MISC_CASES = [
    # (input, query, on_invalid, expected, stats)   exec/cpu.rs:637-707
    ('{"a":1}\n{not json\n{"a":2}\n', ".a", "skip", "1\n2\n", {"malformed": 1, "lines_in": 3}),
    ('{"a":1}\n{"a":{"b":2}}\n', ".a.b", "skip", "2\n", {"type_errors": 1}),
    ('{"a":1}\r\n\r\n{"a":2}\r\n', ".a", "warn", "1\n2\n", {}),
]

FORMAT_NUMBER_CASES = [  # agg.rs:400-410
    (1.0, "1"), (-0.0, "0"), (1.5, "1.5"), (1e300, "1e+300"), (1e-300, "1e-300"),
    (0.1 + 0.2, "0.30000000000000004"),
]

JSON_STRING_CASES = [  # output.rs:372-379
    ("a\nb\"c\\d\x01", '"a\\nb\\"c\\\\d\\u0001"'),
]

CSV_CELL_CASES = [  # output.rs:382-392
    ("plain", "plain"), ("a,b", '"a,b"'), ('say "hi"', '"say ""hi"""'),
]

LOOKUP_CASES = [
    # (line, path, expected kind or outcome, expected raw)   json.rs:715-796, 885-896
    ('{"a":1,"b":"x"}', ".a", "num", "1"),
    ('{"a":1.0}', ".a", "num", "1.0"),
    ('{"a":1e3}', ".a", "num", "1e3"),
    ('{"a":-0.0}', ".a", "num", "-0.0"),
    ('{"a":123456789012345678901234567890}', ".a", "num", "123456789012345678901234567890"),
    ('{"r":{"p":["a","b",{"deep":7}]}}', ".r.p[2].deep", "num", "7"),
    ('{"a":1}', ".z", "missing", "null"),
    ('{"a":1}', ".z.y", "missing", "null"),
    ('{"a":[1]}', ".a[9]", "missing", "null"),
    ('{"a":1}', ".a.b", "type_error", None),
    ('{"a":{}}', ".a[0]", "type_error", None),
    ('{"a":1,"a":2}', ".a", "num", "2"),
    ('{"a\\"b":5}', '."a\\"b"', "num", "5"),
    ('{"msg":"}{[],:\\"","x":9}', ".x", "num", "9"),
    ('{"a":{"b":[1,2]},"c":0}', ".a", "obj", '{"b":[1,2]}'),
]

SELECT_CASES = [
    # (line, select query, verdict)   json.rs:922-958
    ('{"a":null}', "select(.a)", False),
    ('{"a":false}', "select(.a)", False),
    ('{"a":1}', "select(.z)", False),
    ('{"a":0}', "select(.a)", True),
    ('{"a":""}', "select(.a)", True),
    ('{"a":[]}', "select(.a)", True),
    ('{"a":5}', 'select(.a < "5")', True),
    ('{"a":"5"}', "select(.a > 5)", True),
    ('{"a":5}', "select(.a == 5)", True),
    ('{"a":null}', "select(.a < 0)", True),
    ('{"a":null}', "select(.a == null)", True),
    ('{"a":9}', "select(.a < 10)", True),
    ('{"a":1e3}', "select(.a == 1000)", True),
]

LEX_CASES = [
    # (query text, expected first-token description)   query/lex.rs:370-420
    ("42", "int:42"), ("-42", "int:-42"), ("0", "int:0"), ("4.5", "num:4.5"),
    ("1e3", "num:1000"), ("1E3", "num:1000"), ("1e+3", "num:1000"), ("1e-3", "num:0.001"),
    ("-2.5E+10", "num:-25000000000"), ("1.", "num:1"),
]

QUERY_ERROR_CASES = [
    # (query, substring of the error)   query/lex.rs:385-465, query/mod.rs:320-431
    ("-", "expected a number"), ("1e", "no digits in its exponent"),
    ("1e+", "no digits in its exponent"), ("1E-", "no digits in its exponent"),
    ('"unterminated', "unterminated"), ('"bad \\q escape"', "unknown escape"),
    ('"\\u00"', "`\\u`"), ('"\\uZZZZ"', "`\\u`"), ('"\\', "unterminated"),
    ("@", "unexpected character `@`"), ("$x", "`$`"), ("&&", "`&`"),
    (".a = 1", "did you mean `==`"), ("!", "expected `!=`"),
    ("reduce .[] as $x (0; .+$x)", "`reduce` is not"),
    ("def f: .; f", "user-defined functions"),
    ("if .a then 1 else 2 end", "`if/then/else` is not"),
    ("foreach .[] as $x (0; .+1)", "`foreach` is not"),
    ("select(.a = 1)", "did you mean `==`"),
    ("select(.a == .b)", "field-to-field"),
]


def check_cited(text: str, needle: str, where: str):
    # Accept the needle as written in a raw string or in an escaped one.
    if needle not in text and needle.replace("\\", "\\\\") not in text:
        raise SystemExit(f"transcribed case not found in {where}: {needle!r}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="root of the reference checkout")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "reference_vectors.json"))
    args = ap.parse_args()
    root = args.reference

    def read(rel):
        with open(os.path.join(root, rel), encoding="utf-8") as f:
            return f.read()

    conf = read("crates/warpjq-core/tests/conformance.rs")
    diff = read("crates/warpjq-core/tests/differential.rs")
    inv = read("crates/warpjq-core/tests/invariants.rs")
    cpu = read("crates/warpjq-core/src/exec/cpu.rs")
    jsn = read("crates/warpjq-core/src/json.rs")
    agg = read("crates/warpjq-core/src/agg.rs")
    outp = read("crates/warpjq-core/src/output.rs")
    lex = read("crates/warpjq-core/src/query/lex.rs")
    qmod = read("crates/warpjq-core/src/query/mod.rs")
    parse = read("crates/warpjq-core/src/query/parse.rs")

    g = {"_source": "reference project test files; see tests/golden/make_golden.py"}

    # conformance.rs:29-173
    g["must_accept"] = [{"name": t[0], "doc": t[1]} for t in
                        tuples(region(conf, "const MUST_ACCEPT: &[(&str, &str)] = &["))]
    g["must_reject"] = [{"name": t[0], "doc": t[1]} for t in
                        tuples(region(conf, "const MUST_REJECT: &[(&str, &str)] = &["))]
    g["implementation_defined"] = [
        {"name": t[0], "doc": t[1], "accept": t[2], "why": t[3]}
        for t in tuples(region(conf, "const IMPLEMENTATION_DEFINED: &[(&str, &str, bool, &str)] = &["))
    ]
    assert len(g["must_accept"]) == 48 and len(g["must_reject"]) == 52, (
        len(g["must_accept"]), len(g["must_reject"]))
    assert len(g["implementation_defined"]) == 5

    # json.rs:798-920
    g["json_reject"] = strings(region(jsn, "fn rejects_malformed_input() {\n        for bad in [", "] {"))
    g["json_accept"] = strings(region(jsn, "fn accepts_awkward_but_valid_input() {\n        for good in [", "] {"))
    g["json_truncated"] = strings(region(jsn, "        for doc in [", "] {"))
    g["json_mismatched"] = strings(region(jsn, "fn mismatched_brackets_are_rejected_at_every_depth() {", "\n    }"))

    # differential.rs:42-45, 191-207, 250-292, 408-431
    g["diff_keys"] = strings(region(diff, "const KEYS: &[&str] = &[", "];"))
    g["diff_hosts"] = strings(region(diff, "const HOSTS: &[&str] = &[", "];"))
    g["diff_malformed"] = strings(region(diff, "let options = [", "];"))
    g["diff_queries"] = strings(region(diff, "fn queries() -> Vec<&'static str> {\n    vec![", "]\n}"))
    g["diff_edge_lines"] = strings(region(diff, "let lines: Vec<&str> = vec![", "];"))
    g["diff_renormalised_values"] = strings(region(diff, "return [", "]["))
    assert len(g["diff_queries"]) == 40 and len(g["diff_edge_lines"]) == 20

    # invariants.rs:60-74
    g["invariant_queries"] = strings(region(inv, "const QUERIES: &[&str] = &[", "];"))

    # exec/cpu.rs:534-543
    g["cpu_log"] = strings(region(cpu, "const LOG: &str = concat!(", ");"))
    g["cpu_log"] = "".join(g["cpu_log"])
    for q, _, exp in CPU_LOG_CASES:
        check_cited(cpu, q, "exec/cpu.rs")
        if exp is not None:
            for piece in exp.split("\n"):
                if piece:
                    check_cited(cpu.replace('\\"', '"'), piece.replace("\\", ""), "exec/cpu.rs")
    g["cpu_log_cases"] = [{"query": q, "format": f, "expected": g["cpu_log"] if e is None else e}
                          for q, f, e in CPU_LOG_CASES]
    for q, _ in CPU_EMPTY_CASES:
        check_cited(cpu, q, "exec/cpu.rs")
    g["cpu_empty_cases"] = [{"query": q, "expected": e} for q, e in CPU_EMPTY_CASES]
    g["cpu_misc_cases"] = [{"input": i, "query": q, "on_invalid": o, "expected": e, "stats": s}
                           for i, q, o, e, s in CPU_MISC_CASES]

    for _, s in FORMAT_NUMBER_CASES:
        check_cited(agg, f'"{s}"', "agg.rs")
    g["format_number"] = [{"value": v, "expected": s} for v, s in FORMAT_NUMBER_CASES]
    g["format_number_contains_e"] = [1e18]  # agg.rs:409

    for s, _ in CSV_CELL_CASES:
        check_cited(outp, s.replace('"', '\\"'), "output.rs")
    g["json_string"] = [{"input": i, "expected": e} for i, e in JSON_STRING_CASES]
    g["csv_cell"] = [{"input": i, "expected": e} for i, e in CSV_CELL_CASES]

    for line, path, _, raw in LOOKUP_CASES:
        check_cited(jsn, path.lstrip(".").split(".")[0].split("[")[0].strip('"').replace('\\"', '\\"'),
                    "json.rs")
    g["lookup"] = [{"line": l, "path": p, "outcome": k, "raw": r} for l, p, k, r in LOOKUP_CASES]
    g["select"] = [{"line": l, "query": q, "verdict": v} for l, q, v in SELECT_CASES]

    for q, _ in LEX_CASES:
        check_cited(lex, f'"{q}"', "query/lex.rs")
    g["lex_first_token"] = [{"query": q, "token": t} for q, t in LEX_CASES]
    for q, m in QUERY_ERROR_CASES:
        check_cited(lex + qmod + parse, m, "query/*.rs")
    g["query_errors"] = [{"query": q, "contains": m} for q, m in QUERY_ERROR_CASES]

    with open(args.out, "w", encoding="utf-8") as f:
        json.dump(g, f, ensure_ascii=False, indent=1, sort_keys=True)
        f.write("\n")
    print(f"wrote {args.out}: " + ", ".join(f"{k}={len(v) if isinstance(v, (list, str)) else v}"
                                            for k, v in sorted(g.items()) if not k.startswith("_")))


if __name__ == "__main__":
    sys.exit(main())
