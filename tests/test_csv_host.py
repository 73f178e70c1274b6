"""The CSV converter's per-row device code (warpjq_b200/csrc/csv_rows.cuh)
compiled for the host, against the restated mapping (oracle/csv_map.py):
same bytes for every hand case and fuzzed input, at every input alignment,
and every row's written bytes equal to the length its first pass gave."""

import ctypes
import os
import subprocess

import pytest

from oracle import csv_map
from tests.test_csv_map import HAND

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "native", "csv_host.cc")
OUT = os.path.join(HERE, "native", "_build", "libcsv_host.so")
DEP = os.path.join(ROOT, "warpjq_b200", "csrc", "csv_rows.cuh")


@pytest.fixture(scope="module")
def harness():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if not os.path.exists(OUT) or max(os.path.getmtime(SRC), os.path.getmtime(DEP)) > os.path.getmtime(OUT):
        subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-Wl,-Bsymbolic", "-o", OUT, SRC],
                       check=True)
    L = ctypes.CDLL(OUT)
    L.ch_convert.argtypes = [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint, ctypes.POINTER(ctypes.c_void_p),
                             ctypes.POINTER(ctypes.c_size_t)]
    L.ch_free.argtypes = [ctypes.c_void_p]
    return L


def convert(L, src: bytes, shift: int) -> bytes:
    p, n = ctypes.c_void_p(), ctypes.c_size_t()
    rc = L.ch_convert(src, len(src), shift, ctypes.byref(p), ctypes.byref(n))
    out = ctypes.string_at(p.value, n.value) if p.value else b""
    L.ch_free(p)
    assert rc == 0, "a row's written bytes differ from its length pass"
    return out


def test_hand_cases_at_every_alignment(harness):
    for src, want in HAND:
        for shift in range(16):
            assert convert(harness, src, shift) == want, (src, shift)


def test_fuzzed_inputs(harness):
    from tests.test_csv_gpu import fuzz_csv
    for seed in range(40):
        src = fuzz_csv(seed, 60, cols=1 + seed % 7, crlf=seed % 2 == 1, bom=seed % 5 == 0)
        want = csv_map.csv_to_ndjson(src)
        for shift in (0, 1, 2, 3, 7):
            assert convert(harness, src, shift) == want, (seed, shift)


def test_long_fields_and_controls(harness):
    src = (b'k,v\n"' + bytes(range(1, 128)).replace(b'"', b'""') * 5 + b'",' + b"9" * 70 + b"\n" +
           b"x" * 1000 + b"," + b"-1.25E+10\n")
    for shift in range(4):
        assert convert(harness, src, shift) == csv_map.csv_to_ndjson(src)
