"""The CSV-to-NDJSON mapping (oracle/csv_map.py), checked without a GPU.

The reference has no CSV reader, so the mapping is pinned two other ways:
its RFC 4180 field splitting agrees with Python's own csv module on
well-formed input, and the nginx generator's CSV rendering maps to exactly
the NDJSON lines the same generator writes for the same records.  Hand
cases cover the rules the csv module does not decide (numbers, nulls,
ragged rows, the header)."""

import csv
import io
import json
import random

import pytest

from oracle import csv_map
import warpjq_b200 as wjq

HAND = [
    (b"", b""),
    (b"a,b\n", b""),
    (b"a,b", b""),
    (b"a,b\n1,2\n", b'{"a":1,"b":2}\n'),
    (b"a,b\n1,2", b'{"a":1,"b":2}\n'),
    (b"a,b\r\n1,2\r\n", b'{"a":1,"b":2}\n'),
    (b"\xef\xbb\xbfa\n1\n", b'{"a":1}\n'),
    (b"a,b,c\n1\n", b'{"a":1}\n'),
    (b"a,b,c\n1,\n", b'{"a":1,"b":null}\n'),
    (b"a,b,c\n,,\n", b'{"a":null,"b":null,"c":null}\n'),
    (b"a\n1,2,3\n", b'{"a":1}\n'),
    (b"a\n\n\n1\n", b'\n\n{"a":1}\n'),
    (b"a\n\r\n", b"\n"),
    (b'a\n""\n', b'{"a":""}\n'),
    (b'a\n"1"\n', b'{"a":"1"}\n'),
    (b'a\n"x""y"\n', b'{"a":"x\\"y"}\n'),
    (b'a\n"x,y"\n', b'{"a":"x,y"}\n'),
    (b'a\n"x\ny"\n', b'{"a":"x\\ny"}\n'),
    (b'a\n"x"tail,2\n', b'{"a":"xtail"}\n'),
    (b'a\nab"c"d\n', b'{"a":"ab\\"c\\"d"}\n'),
    (b'a\nab"c\n1\n', b'{"a":"ab\\"c\\n1\\n"}\n'),  # an odd quote: the row runs to the end
    (b"a\n-0\n", b'{"a":-0}\n'),
    (b"a\n1.5e-3\n", b'{"a":1.5e-3}\n'),
    (b"a\n01\n", b'{"a":"01"}\n'),
    (b"a\n+1\n", b'{"a":"+1"}\n'),
    (b"a\n1.\n", b'{"a":"1."}\n'),
    (b"a\n.5\n", b'{"a":".5"}\n'),
    (b"a\n 1\n", b'{"a":" 1"}\n'),
    (b"a\nNaN\n", b'{"a":"NaN"}\n'),
    (b"a\ntrue\n", b'{"a":"true"}\n'),
    (b"a\nx\\y\n", b'{"a":"x\\\\y"}\n'),
    (b"a\nx\ty\x01\n", b'{"a":"x\\ty\\u0001"}\n'),
    (b"a\n\xc3\xa9\n", b'{"a":"\xc3\xa9"}\n'),
    (b'"k ""q"",",b\n1,2\n', b'{"k \\"q\\",":1,"b":2}\n'),
    (b"\nx\n", b"{}\n"),
    (b"a,a\n1,2\n", b'{"a":1,"a":2}\n'),
]


@pytest.mark.parametrize("src,want", HAND)
def test_hand_cases(src, want):
    assert csv_map.csv_to_ndjson(src) == want


def _random_field(rng):
    alphabet = 'ab ,"\n\r\t\\x1-.e'
    k = rng.randrange(0, 8)
    return "".join(rng.choice(alphabet) for _ in range(k))


def test_fields_agree_with_python_csv_module():
    rng = random.Random(7)
    for _ in range(300):
        n_cols = rng.randrange(1, 6)
        names = [f"c{j}" for j in range(n_cols)]
        rows = [[_random_field(rng) for _ in range(n_cols)] for _ in range(rng.randrange(1, 6))]
        buf = io.StringIO(newline="")
        w = csv.writer(buf, lineterminator="\n", quoting=csv.QUOTE_ALL)
        w.writerow(names)
        w.writerows(rows)
        data = buf.getvalue().encode()
        out = csv_map.csv_to_ndjson(data).decode().split("\n")[:-1]
        assert len(out) == len(rows)
        for line, row in zip(out, rows):
            obj = json.loads(line)  # every field quoted: all strings
            assert list(obj.keys()) == names
            assert list(obj.values()) == row


def test_minimal_quoting_agrees_with_python_csv_module():
    rng = random.Random(11)
    for _ in range(300):
        n_cols = rng.randrange(1, 6)
        rows = [[_random_field(rng) for _ in range(n_cols)] for _ in range(rng.randrange(1, 6))]
        buf = io.StringIO(newline="")
        w = csv.writer(buf, lineterminator="\r\n", quoting=csv.QUOTE_MINIMAL)
        w.writerow([f"c{j}" for j in range(n_cols)])
        w.writerows(rows)
        data = buf.getvalue().encode()
        parsed = list(csv.reader(io.StringIO(data.decode(), newline="")))[1:]
        out = csv_map.csv_to_ndjson(data).decode().split("\n")[:-1]
        assert len(out) == len(parsed)
        for line, row in zip(out, parsed):
            if line == "":  # a row the writer left empty (a single empty field)
                assert row in ([], [""])
                continue
            got = [v if isinstance(v, str) else json.dumps(v) if v is not None else "" for v in
                   json.loads(line, parse_float=str, parse_int=str).values()]
            assert got == row


def test_nginx_csv_rendering_maps_to_the_ndjson_rendering():
    import warpjq_b200 as wjq
    # within the generator's first 1 MiB block the two renderings share records
    cbuf, cused, _ = wjq.gen_nginx_csv(600_000, seed=5)
    nbuf, nused, _ = wjq.gen_nginx(1 << 20, seed=5)
    mapped = csv_map.csv_to_ndjson(bytes(cbuf[:cused])).split(b"\n")[:-1]
    lines = bytes(nbuf[:nused]).split(b"\n")
    assert len(mapped) > 2000
    assert mapped == lines[:len(mapped)]


def test_csv_records_rendered_as_ndjson_match_the_mapping():
    """warpjq_gen_nginx_csv_as_ndjson (the expected input of a query over the
    bench's CSV) is exactly the mapping of the CSV rows of the same seed and
    size, so the oracle over it checks the CSV leg at its full size."""
    for size, seed in ((1 << 20, 6), (5 << 20, 7), (200_000, 2)):
        c, cu, cl = wjq.gen_nginx_csv(size, seed=seed)
        n, nu, nl = wjq.gen_nginx_csv_as_ndjson(size, seed=seed)
        assert cl == nl
        assert csv_map.csv_to_ndjson(bytes(c[:cu])) == bytes(n[:nu])
