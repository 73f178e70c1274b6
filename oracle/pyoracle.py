"""TEST INFRASTRUCTURE -- ctypes wrapper around the oracle library.

The oracle is a CPU restatement of the reference project's Rust CPU engine.
Only the tests, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
it, always as the checker or the baseline -- never as the thing measured.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

FORMATS = {"ndjson": 0, "csv": 1, "count": 2}
ON_INVALID = {"warn": 0, "skip": 1, "abort": 2}
KINDS = ["missing", "null", "bool", "num", "str", "arr", "obj"]


def build() -> str:
    """Compiles the oracle with its Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        c_u8p = ctypes.c_char_p
        L.oracle_run.argtypes = [ctypes.c_char_p, c_u8p, ctypes.c_size_t, ctypes.c_int,
                                 ctypes.c_int, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t,
                                 ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                                 ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p, ctypes.c_size_t]
        L.oracle_run.restype = ctypes.c_int
        L.oracle_free.argtypes = [ctypes.c_void_p]
        L.oracle_validate.argtypes = [c_u8p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t),
                                      ctypes.c_char_p, ctypes.c_size_t]
        L.oracle_validate.restype = ctypes.c_int
        L.oracle_format_number.argtypes = [ctypes.c_double, ctypes.c_char_p, ctypes.c_size_t]
        L.oracle_parse.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p),
                                   ctypes.POINTER(ctypes.c_size_t)]
        L.oracle_parse.restype = ctypes.c_int
        L.oracle_lookup.argtypes = [c_u8p, ctypes.c_size_t, ctypes.c_char_p,
                                    ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_void_p),
                                    ctypes.POINTER(ctypes.c_size_t)]
        L.oracle_lookup.restype = ctypes.c_int
        L.oracle_eval_select.argtypes = [c_u8p, ctypes.c_size_t, ctypes.c_char_p]
        L.oracle_eval_select.restype = ctypes.c_int
        L.oracle_parse_f64.argtypes = [c_u8p, ctypes.c_size_t]
        L.oracle_parse_f64.restype = ctypes.c_double
        _lib = L
    return _lib


def _take(ptr, n) -> bytes:
    if not ptr.value:
        return b""
    b = ctypes.string_at(ptr.value, n.value)
    lib().oracle_free(ptr)
    return b


class OracleResult:
    def __init__(self, rc, out, stats, err):
        self.rc = rc
        self.out = out
        self.stats = stats
        self.err = err

    def __repr__(self):
        return f"OracleResult(rc={self.rc}, out={self.out[:80]!r}, stats={self.stats}, err={self.err!r})"


def _input(data):
    """(pointer argument, length, keep-alive) for bytes or a uint8 numpy array
    (the array is passed without a copy)."""
    if isinstance(data, bytes):
        return data, len(data), None
    if isinstance(data, bytearray):
        b = bytes(data)
        return b, len(b), b
    import numpy as np
    a = np.ascontiguousarray(data, dtype=np.uint8)
    return a.ctypes.data_as(ctypes.c_char_p), a.size, a


def run(query: str, data, fmt: str = "ndjson", on_invalid: str = "skip",
        chunk_bytes: int = 0, threads: int = 0, max_line_bytes: int = 0) -> OracleResult:
    """Runs a query the way the reference CPU engine's run_bytes does; `data`
    is bytes or a uint8 numpy array."""
    L = lib()
    out = ctypes.c_void_p()
    n = ctypes.c_size_t()
    stats = (ctypes.c_uint64 * 5)()
    err = ctypes.create_string_buffer(4096)
    ptr, ln, keep = _input(data)
    rc = L.oracle_run(query.encode(), ptr, ln, FORMATS[fmt], ON_INVALID[on_invalid],
                      chunk_bytes, threads, max_line_bytes, ctypes.byref(out), ctypes.byref(n),
                      stats, err, len(err))
    del keep
    body = _take(out, n)
    st = dict(zip(["bytes_in", "lines_in", "lines_out", "malformed", "type_errors"], list(stats)))
    return OracleResult(rc, body, st, err.value.decode(errors="replace"))


def validate(line: bytes):
    off = ctypes.c_size_t()
    det = ctypes.create_string_buffer(256)
    ok = lib().oracle_validate(line, len(line), ctypes.byref(off), det, len(det))
    return bool(ok), off.value, det.value.decode(errors="replace")


def format_number(v: float) -> str:
    buf = ctypes.create_string_buffer(64)
    lib().oracle_format_number(v, buf, len(buf))
    return buf.value.decode()


def parse(query: str):
    import json
    out = ctypes.c_void_p()
    n = ctypes.c_size_t()
    rc = lib().oracle_parse(query.encode(), ctypes.byref(out), ctypes.byref(n))
    return rc, json.loads(_take(out, n).decode())


def lookup(line: bytes, path: str):
    kind = ctypes.c_int()
    out = ctypes.c_void_p()
    n = ctypes.c_size_t()
    rc = lib().oracle_lookup(line, len(line), path.encode(), ctypes.byref(kind), ctypes.byref(out),
                             ctypes.byref(n))
    raw = _take(out, n)
    if rc == 0:
        return "found", KINDS[kind.value], raw
    if rc == 1:
        return "type_error", None, raw
    if rc == 2:
        return "invalid", None, raw
    raise ValueError(f"bad path {path!r}")


def eval_select(line: bytes, query: str) -> bool:
    rc = lib().oracle_eval_select(line, len(line), query.encode())
    if rc < 0:
        raise ValueError(query)
    return bool(rc)


def parse_f64(text: bytes) -> float:
    return lib().oracle_parse_f64(text, len(text))


def gen_nginx(n_bytes: int, seed: int = 1, threads: int = 0, into=None):
    """The benchmark's seeded nginx-style NDJSON, from the generator compiled
    into the oracle library (the same source as the product's generator),
    so a CPU-only measurement builds its input without the product's
    libraries.  Returns (buffer, used_bytes, n_lines)."""
    import numpy as np
    L = lib()
    L.warpjq_gen_nginx.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64,
                                   ctypes.c_uint, ctypes.POINTER(ctypes.c_uint64)]
    L.warpjq_gen_nginx.restype = ctypes.c_uint64
    buf = into if into is not None else np.empty(n_bytes, dtype=np.uint8)
    lines = ctypes.c_uint64()
    used = L.warpjq_gen_nginx(seed, buf.ctypes.data, n_bytes, 1 << 20, threads, ctypes.byref(lines))
    return buf, int(used), int(lines.value)
