"""Results that do not depend on how the work was cut.

Sums of fractional values are accumulated exactly on the device (fixed-point
limbs, rounded once at the end), so an aggregate's bytes are the same for
any tile size, in a batch beside other inputs, and in the serving loop -- a
grouped average over a million Zipf user ids included, where the reference
adds with atomics in whatever order they land
(crates/warpjq-core/cuda/warpjq_kernels.cu:1564).  The same outputs match
the oracle within the stated tolerance (it adds in line order).

Also the plain configuration of the benchmark: 64 MB of nginx NDJSON and
`select(.status == 500) | count`, device-resident, against the oracle."""

import numpy as np
import pytest

import warpjq_b200 as wjq
from oracle import pyoracle as orc
from tests.test_gpu_parity import close_enough

pytestmark = pytest.mark.gpu

GROUP_AVG = "group_by(.req.user.id) | avg(.resp.latency)"
TILINGS = [(4096, 1024), (12288, 2048), (32768, 4096)]


def to_device(data: bytes):
    import torch
    dev = torch.empty(len(data) + 16, dtype=torch.uint8, device="cuda")
    if data:
        dev[:len(data)].copy_(torch.frombuffer(bytearray(data), dtype=torch.uint8))
    return dev


def run_device(q: str, data: bytes, dev, tiling=None) -> bytes:
    import torch
    Q = wjq.Query(q)
    if tiling:
        Q.set_tiling(*tiling)
    Q.launch_device(dev.data_ptr(), len(data), torch.cuda.current_stream().cuda_stream)
    out = Q.render_device(Q.collect_device(), data)
    Q.close()
    return out


def run_in_batch(q: str, data: bytes, others, tiling=None) -> bytes:
    """`data` as the middle input of a batch of three (the others around it)."""
    import torch
    ins = [others[0], data, others[1]]
    offs, parts, pos = [], [], 0
    for x in ins:
        pad = (-pos) % 16
        parts.append(b"\n" * pad)
        pos += pad
        offs.append(pos)
        parts.append(x)
        pos += len(x)
    buf = b"".join(parts)
    dev = to_device(buf)
    Q = wjq.Query(q)
    if tiling:
        Q.set_tiling(*tiling)
    Q.batch_launch(dev.data_ptr(), offs, [len(x) for x in ins], torch.cuda.current_stream().cuda_stream)
    items, all_ = Q.batch_collect()
    outs = Q.batch_outputs(items, all_, np.frombuffer(buf, dtype=np.uint8))
    Q.close()
    return outs[1]


def run_in_server(q: str, data: bytes, others) -> bytes:
    from warpjq_b200.serve import Server
    srv = Server([q], n_slots=2)
    hs = [srv.submit(q, x) for x in (others[0], data, others[1])]
    srv.drain()
    srv.close()
    assert all(not h.error for h in hs)
    return hs[1].out


@pytest.mark.parametrize("q,gen", [
    (GROUP_AVG, "nested"),
    ("avg(.latency_ms)", "nginx"),
    ("group_by(.path) | avg(.latency_ms)", "nginx"),
    ("sum(.resp.latency)", "nested"),
])
def test_fractional_sums_are_bit_identical_however_the_work_is_cut(q, gen):
    if gen == "nested":
        buf, used, _ = wjq.gen_nested(24 << 20, seed=31, n_users=1_000_000)
        ob, ou, _ = wjq.gen_nested(2 << 20, seed=32, n_users=1_000_000)
    else:
        buf, used, _ = wjq.gen_nginx(24 << 20, seed=31)
        ob, ou, _ = wjq.gen_nginx(2 << 20, seed=32)
    data = bytes(buf[:used])
    half = bytes(ob[:ou]).split(b"\n")
    others = [b"\n".join(half[: len(half) // 2]) + b"\n", b"\n".join(half[len(half) // 2:])]
    dev = to_device(data)
    outs = [run_device(q, data, dev, t) for t in TILINGS]
    outs.append(run_in_batch(q, data, others, TILINGS[1]))
    outs.append(run_in_server(q, data, others))
    for k, o in enumerate(outs[1:], 1):
        assert o == outs[0], (q, k)  # bit-identical bytes
    want = orc.run(q, data).out
    assert close_enough(outs[0], want), q


def test_plain_configuration_64MB_count():
    """64 MB of the nginx schema (~320k lines), select(.status == 500) |
    count, device-resident through launch_device / render_device, against
    the oracle's output and line statistics."""
    import torch
    buf, used, lines = wjq.gen_nginx(64 << 20, seed=1)
    data = bytes(buf[:used])
    q = "select(.status == 500) | count"
    dev = to_device(data)
    Q = wjq.Query(q)
    Q.autotile(np.frombuffer(data[: 1 << 20], dtype=np.uint8))
    Q.launch_device(dev.data_ptr(), len(data), torch.cuda.current_stream().cuda_stream)
    r = Q.collect_device()
    got = Q.render_device(r, data)
    Q.close()
    want = orc.run(q, data)
    assert want.rc == 0 and got == want.out
    assert r.n_lines == lines == want.stats["lines_in"]
    assert r.n_invalid == 0 and r.n_blank == 0
