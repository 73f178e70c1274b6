"""warpjq_aggregate_noalloc: the aggregate scan for callers that cannot call
cudaMalloc (an engine that owns all device memory through its own pool, or a
caller that cannot afford cudaMalloc's device synchronisation).  It keeps all
its scratch in one fixed device array, so this test checks that it gives the
same answers as the allocating entry point (warpjq_launch_device /
warpjq_collect_device) on two calls in a row, that what it returns prints
as the oracle's output for the same bytes, and where its fixed nesting
stack ends.

The file name sorts last so a run that stops at the first failure has
already run every other test; it also passes when run alone."""

import ctypes

import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc
from tests.test_gpu_parity import close_enough

pytestmark = pytest.mark.gpu

U32 = ctypes.c_uint32


class Step(ctypes.Structure):
    _fields_ = [("kind", U32), ("index", U32), ("key_off", U32), ("key_len", U32), ("key_hash", U32)]


class PathT(ctypes.Structure):
    _fields_ = [("step_off", U32), ("step_count", U32)]


class Cmp(ctypes.Structure):
    _fields_ = [("path", U32), ("op", U32), ("lit_kind", U32), ("lit_off", U32), ("lit_len", U32),
                ("_pad", U32), ("lit_num", ctypes.c_double)]


class CondOp(ctypes.Structure):
    _fields_ = [("op", U32), ("arg", U32)]


P = ctypes.POINTER


class Program(ctypes.Structure):
    _fields_ = [("steps", P(Step)), ("n_steps", U32), ("paths", P(PathT)), ("n_paths", U32),
                ("cmps", P(Cmp)), ("n_cmps", U32), ("cond_rpn", P(CondOp)), ("n_cond", U32),
                ("blob", ctypes.c_char_p), ("n_blob", U32), ("needed_paths", P(U32)), ("n_needed", U32),
                ("slot_of_path", P(U32)), ("output_kind", U32), ("output_path", U32), ("agg_kind", U32),
                ("agg_path", U32), ("group_path", U32), ("has_filter", U32), ("n_fields", U32),
                ("field_paths", P(U32)), ("prefix_off", P(U32)), ("prefix_len", P(U32)),
                ("suffix_off", U32), ("suffix_len", U32), ("csv_mode", U32)]


class NoAllocResult(ctypes.Structure):
    _fields_ = [("n_lines", ctypes.c_uint64), ("n_blank", ctypes.c_uint64),
                ("n_invalid", ctypes.c_uint64), ("n_type_error", ctypes.c_uint64),
                ("n_selected", ctypes.c_uint64), ("first_invalid", ctypes.c_uint64),
                ("count", ctypes.c_uint64), ("numeric", ctypes.c_uint64),
                ("isum_lo", ctypes.c_uint64), ("isum_hi", ctypes.c_uint64), ("n_int", ctypes.c_uint64),
                ("fsum", ctypes.c_double), ("min", ctypes.c_double), ("max", ctypes.c_double),
                ("sum", ctypes.c_double), ("saw_non_numeric", U32), ("status", U32)]


def lower(keys, agg_kind, agg_key=None, cmp=None):
    """Flat tables for `[select(.k op num) |] agg(.key)` over top-level keys."""
    blob = b"".join(k.encode() for k in keys)
    steps, off = [], 0
    for k in keys:
        h = 0x811C9DC5
        for c in k.encode():
            h = ((h ^ c) * 0x01000193) & 0xFFFFFFFF
        steps.append(Step(0, 0, off, len(k), h))
        off += len(k)
    keep = {}
    keep["steps"] = (Step * max(1, len(steps)))(*steps)
    keep["paths"] = (PathT * max(1, len(keys)))(*[PathT(i, 1) for i in range(len(keys))])
    cmps = [cmp[0]] if cmp else []
    keep["cmps"] = (Cmp * 1)(*cmps) if cmps else (Cmp * 1)()
    keep["cond"] = (CondOp * 1)(CondOp(0, 0)) if cmp else (CondOp * 1)()
    keep["needed"] = (U32 * max(1, len(keys)))(*range(len(keys)))
    keep["slot"] = (U32 * max(1, len(keys)))(*range(len(keys)))
    keep["blob"] = blob
    prog = Program(keep["steps"], len(steps), keep["paths"], len(keys), keep["cmps"], len(cmps),
                   keep["cond"], 1 if cmp else 0, blob, len(blob), keep["needed"], len(keys),
                   keep["slot"], 3, 0xFFFFFFFF, agg_kind,
                   keys.index(agg_key) if agg_key else 0xFFFFFFFF, 0xFFFFFFFF, 1 if cmp else 0,
                   0, None, None, None, 0, 0, 0)
    return prog, keep


CASES = [
    ("count", dict(keys=[], agg_kind=0)),
    ("select(.status == 500) | count", dict(keys=["status"], agg_kind=0, cmp=[Cmp(0, 0, 3, 0, 0, 0, 500.0)])),
    ("sum(.bytes)", dict(keys=["bytes"], agg_kind=1, agg_key="bytes")),
    ("min(.bytes)", dict(keys=["bytes"], agg_kind=2, agg_key="bytes")),
    ("avg(.latency_ms)", dict(keys=["latency_ms"], agg_kind=4, agg_key="latency_ms")),
    ("select(.status >= 500) | max(.latency_ms)",
     dict(keys=["status", "latency_ms"], agg_kind=3, agg_key="latency_ms", cmp=[Cmp(0, 5, 3, 0, 0, 0, 500.0)])),
]


def test_noalloc_matches_the_allocating_entry_point():
    import torch
    why = wjq.probe()
    assert not why, why
    k, _ = wjq.libraries()
    fn = k.warpjq_aggregate_noalloc
    fn.argtypes = [ctypes.POINTER(Program), ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    fn.restype = ctypes.c_int

    buf, used, _ = wjq.gen_nginx(48 << 20, seed=11)
    extra = b'{"status":500,\n{oops\n' + b"[" * 100 + b"]" * 100 + b'\n\n{"status":"x","bytes":"y"}\n'
    data = bytes(buf[:used]) + extra
    dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
    dev[: len(data)].copy_(torch.frombuffer(bytearray(data), dtype=torch.uint8))
    res = torch.zeros(ctypes.sizeof(NoAllocResult), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    err = ctypes.create_string_buffer(512)

    for query, spec in CASES:
        q = wjq.Query(query)
        q.launch_device(dev.data_ptr(), len(data), stream.cuda_stream)
        want = q.collect_device()
        prog, keep = lower(**spec)
        for call in range(2):  # two calls in a row share (and reuse) the scratch
            res.fill_(0xAB)
            rc = fn(ctypes.byref(prog), dev.data_ptr(), len(data), stream.cuda_stream, res.data_ptr(),
                    err, len(err))
            assert rc == 0, err.value
            torch.cuda.synchronize()
            got = NoAllocResult.from_buffer_copy(bytes(res.cpu().numpy()))
            ctx = f"{query} call {call}"
            assert got.status == 0, ctx
            for f in ("n_lines", "n_blank", "n_invalid", "n_type_error", "first_invalid", "count",
                      "numeric", "isum_lo", "isum_hi", "n_int", "saw_non_numeric"):
                assert getattr(got, f) == getattr(want, f), (ctx, f, getattr(got, f), getattr(want, f))
            # both sum exactly and round once: the same bits, not just close
            for f in ("min", "max", "fsum", "sum"):
                assert getattr(got, f) == getattr(want, f), (ctx, f, getattr(got, f), getattr(want, f))
            # and, on its own, what the oracle prints for the same bytes
            printed = q.render_device(as_device_result(got), data)
            oracle = orc.run(query, data)
            assert oracle.rc == 0 and close_enough(printed, oracle.out), (ctx, printed, oracle.out)
            # the oracle's line count leaves blank lines out
            assert got.n_lines - got.n_blank == oracle.stats["lines_in"], ctx
            assert got.n_invalid == oracle.stats["malformed"], ctx
        q.close()


def as_device_result(r: NoAllocResult) -> "wjq.DeviceResult":
    """The no-allocation result in the allocating path's result struct, so
    the host library's formatter prints it."""
    d = wjq.DeviceResult()
    for f in ("n_lines", "n_blank", "n_invalid", "n_type_error", "n_selected", "first_invalid", "count",
              "numeric", "isum_lo", "isum_hi", "n_int", "fsum", "min", "max", "sum", "saw_non_numeric"):
        setattr(d, f, getattr(r, f))
    return d


def test_noalloc_nesting_limit():
    """Lines nest in the fixed scratch up to 16,448 levels (64 in registers,
    16,384 in the array): such a line is counted like any other; one level
    more and the call reports status 1 instead of a wrong count."""
    import torch
    k, _ = wjq.libraries()
    fn = k.warpjq_aggregate_noalloc
    fn.argtypes = [ctypes.POINTER(Program), ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    fn.restype = ctypes.c_int
    prog, keep = lower(keys=[], agg_kind=0)
    err = ctypes.create_string_buffer(512)
    res = torch.zeros(ctypes.sizeof(NoAllocResult), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    for depth, status in ((16448, 0), (16449, 1)):
        data = b'{"a":1}\n' + b"[" * depth + b"]" * depth + b'\n{"b":2}\n'
        dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
        dev[: len(data)].copy_(torch.frombuffer(bytearray(data), dtype=torch.uint8))
        assert fn(ctypes.byref(prog), dev.data_ptr(), len(data), stream.cuda_stream, res.data_ptr(), err,
                  len(err)) == 0, err.value
        torch.cuda.synchronize()
        got = NoAllocResult.from_buffer_copy(bytes(res.cpu().numpy()))
        assert got.status == status, depth
        if status == 0:
            assert got.count == 3 and got.n_lines == 3 and got.n_invalid == 0


def test_noalloc_rejects_what_it_cannot_run():
    k, _ = wjq.libraries()
    fn = k.warpjq_aggregate_noalloc
    fn.argtypes = [ctypes.POINTER(Program), ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]
    prog, keep = lower(keys=[], agg_kind=0)
    err = ctypes.create_string_buffer(512)
    # over the 4 GiB limit: rejected before any device work
    assert fn(ctypes.byref(prog), 16, (4 << 30) + 1, None, 16, err, len(err)) == 5
    assert b"limit" in err.value
    prog.output_kind = 0  # passthrough rows need allocation
    assert fn(ctypes.byref(prog), 16, 100, None, 16, err, len(err)) == 5
