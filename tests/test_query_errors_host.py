"""The product's own query front-end (warpjq_b200/csrc/host/query.cc, through
warpjq_query_open_host) on the reference's query-error vectors, without a
GPU: every rejected query returns code 2 (the CLI's exit code for a query
error, crates/warpjq-cli/src/main.rs:169-189) with the reference's message
(query/mod.rs:320-431, query/lex.rs:370-465), rendered exactly as the oracle
renders it; accepted queries from the vectors open."""

import json
import os

import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def golden():
    with open(os.path.join(HERE, "golden", "reference_vectors.json")) as f:
        return json.load(f)


def test_rejected_queries_match_the_reference_messages(golden):
    for c in golden["query_errors"]:
        with pytest.raises(ValueError) as e:
            wjq.Query(c["query"], device=False)
        msg = str(e.value)
        assert c["contains"] in msg, (c, msg)
        rc, info = orc.parse(c["query"])
        assert rc == 2 and msg == info["rendered"], (c, msg, info["rendered"])


def test_accepted_queries_open(golden):
    qs = list(golden["diff_queries"]) + [f"select(.a == {c['query']})" for c in golden["lex_first_token"]]
    for q in qs:
        wjq.Query(q, device=False).close()
