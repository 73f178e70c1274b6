"""Seeded hostile NDJSON corpora for the parity tests.

Same shape as the reference's differential corpus
(crates/warpjq-core/tests/differential.rs:87-242): a predictable outer object
with hostile values inside -- unicode, escapes, surrogate pairs, integers past
2^53, duplicate keys, empty containers, CRLF, blank lines and malformed
lines.  The value lists come from the committed fixture (extracted from that
file); the random stream is Python's own, seeded, so it is reproducible here
but not byte-identical to the reference's ChaCha8 stream.
"""

from __future__ import annotations

import json
import os
import random

_GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.json")
with open(_GOLDEN, encoding="utf-8") as _f:
    G = json.load(_f)

KEYS = G["diff_keys"]
HOSTS = G["diff_hosts"]
MALFORMED = G["diff_malformed"]
RENORMALISED = G["diff_renormalised_values"]

FIXED = [
    "null", "true", "false", "0", "-0", "9007199254740993", "123456789012345678901234567890",
    "1e3", "-2.5E+10", "1.0", "0.1", '""', '"plain"', '"with \\"escaped\\" quotes"',
    '"tab\\there\\nnewline\\\\backslash"', '"emoji \U0001F600 and é"',
    '"日本語 ☃ café"', "{}", "[]",
]


def hard_value(rng: random.Random, depth: int) -> str:
    if rng.randrange(14) == 0:
        return rng.choice(RENORMALISED)
    k = rng.randrange(20)
    if k < 19:
        return FIXED[k]
    if depth == 0:
        return str(rng.randrange(1000))
    if rng.random() < 0.5:
        n = rng.randrange(4)
        return "[" + ",".join(hard_value(rng, depth - 1) for _ in range(n)) + "]"
    n = rng.randrange(1, 4)
    return "{" + ",".join(json.dumps(KEYS[i % len(KEYS)]) + ":" + hard_value(rng, depth - 1)
                          for i in range(n)) + "}"


def good_line(rng: random.Random) -> str:
    status = rng.choice([200, 301, 404, 500, 503])
    host = rng.choice(HOSTS)
    flag = "null" if rng.random() < 0.3 else ("true" if rng.random() < 0.5 else "false")
    return ('{"status":%d,"bytes":%d,"host":%s,"msg":%s,"nested":{"deep":{"v":%d}},'
            '"arr":[%s,%d,%s],"flag":%s,"n":%s}' % (
                status, rng.randrange(100000), json.dumps(host, ensure_ascii=False),
                hard_value(rng, 1), rng.randrange(500), hard_value(rng, 0), rng.randrange(10),
                hard_value(rng, 0), flag, hard_value(rng, 2)))


def corpus(seed: int, lines: int, bad_ratio: float = 0.0, crlf: bool = False) -> bytes:
    rng = random.Random(seed)
    out = []
    for i in range(lines):
        if i > 0 and i % 37 == 0:
            out.append("\n")
        if i > 0 and i % 53 == 0:
            out.append("   \n")
        out.append(rng.choice(MALFORMED) if rng.random() < bad_ratio else good_line(rng))
        out.append("\n")
    s = "".join(out)
    if crlf:
        s = s.replace("\n", "\r\n")
    return s.encode("utf-8")


def edge_corpus() -> bytes:
    return ("\n".join(G["diff_edge_lines"]) + "\n").encode("utf-8")
