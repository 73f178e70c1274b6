"""Parity with the reference itself on the GPU: the reference's own kernels
(crates/warpjq-core/cuda/warpjq_kernels.cu, built unmodified from its source
by `make -C oracle ref` into oracle/_ref/) driven through its C ABI by this
project's host driver, against this project's backend and the oracle, on the
nginx bench workload.  The reference leaves some lines to its Rust host (its
fallback arrays); the driver refuses such chunks, so the inputs here are ones
the reference decides entirely on the device.

Skipped when oracle/_ref was not built (no reference sources where it was
built)."""

import multiprocessing as mp
import os

import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_HOST = os.path.join(ROOT, "oracle", "_ref", "libwarpjq_host.so")
QUERIES = ["select(.status == 500) | count", "select(.status >= 500) | {p: .path, b: .bytes}",
           "group_by(.host) | sum(.bytes)", "select(.status == 500)", "sum(.bytes)", "max(.latency_ms)",
           "group_by(.status) | count"]


def _run_reference(data: bytes, queries, chunk_bytes, conn):
    """In a fresh process: the reference's kernels through the C ABI."""
    import ctypes
    h = ctypes.CDLL(REF_HOST, mode=ctypes.RTLD_LOCAL)
    h.warpjq_run_bytes.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint32,
                                   ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint64,
                                   ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ctypes.c_size_t),
                                   ctypes.POINTER(ctypes.c_uint64), ctypes.c_char_p, ctypes.c_size_t]
    h.warpjq_host_free.argtypes = [ctypes.c_void_p]
    outs = []
    for q in queries:
        out, n = ctypes.c_void_p(), ctypes.c_size_t()
        st = (ctypes.c_uint64 * 5)()
        err = ctypes.create_string_buffer(4096)
        rc = h.warpjq_run_bytes(q.encode(), data, len(data), 0, 1, chunk_bytes, 0, ctypes.byref(out),
                                ctypes.byref(n), st, err, len(err))
        body = ctypes.string_at(out.value, n.value) if out.value else b""
        if out.value:
            h.warpjq_host_free(out)
        outs.append((rc, body, err.value.decode(errors="replace")))
    conn.send(outs)
    conn.close()


@pytest.mark.skipif(not os.path.exists(REF_HOST), reason="oracle/_ref not built")
def test_reference_kernels_ours_and_the_oracle_agree_on_the_nginx_workload():
    buf, used, _ = wjq.gen_nginx(64 << 20, seed=12)
    data = bytes(buf[:used])
    ctx = mp.get_context("spawn")
    parent, child = ctx.Pipe()
    p = ctx.Process(target=_run_reference, args=(data, QUERIES, 64 << 20, child))
    p.start()
    ref = parent.recv()
    p.join(timeout=600)
    assert p.exitcode == 0
    for q, (rc, ref_out, ref_err) in zip(QUERIES, ref):
        assert rc == 0, (q, ref_err)
        ours = wjq.run_bytes(q, data, chunk_bytes=64 << 20)
        assert ours.rc == 0, ours.err
        want = orc.run(q, data).out
        assert ref_out == want, ("reference kernels vs oracle", q)
        assert ours.out == want, ("this backend vs oracle", q)
