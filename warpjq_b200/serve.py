"""A resident serving loop over the device backend: continuous batching.

The server keeps, per slot, a CUDA stream, one compiled query context per
query, a device arena and a CSV converter, all alive across requests (no
per-request context set-up).  Requests wait in arrival order.  Whenever a
slot is free, it takes every waiting request that fits the device-memory
budget, finds each one's NDJSON a 16-byte aligned device address (device
inputs in place, CSV converted on the device, host inputs copied into the
arena), and runs one batch per query among them (warpjq_batch_launch, by
device address; from MIXED_MIN aggregate requests of two or more queries
on, those go into one mixed batch, warpjq_batch_launch_mixed) on its
stream, then returns to the loop: requests
arriving meanwhile are admitted into the next free slot, so several slots'
work overlaps on the device.  A finished slot is collected when its event
has completed; each request's output is exactly what a run over its input
alone prints (rows cut from the batch's rows, aggregates and groups
rendered by the host formatter, group keys gathered from device memory).

There is no reference counterpart: the reference runs one query per process
invocation (crates/warpjq-cli).
"""

from __future__ import annotations

import collections
import time
from dataclasses import dataclass

import numpy as np

from . import CsvConverter, Query, batch_outputs_mixed


@dataclass
class Request:
    id: int
    query: str
    fmt: str                 # "ndjson" or "csv"
    nbytes: int
    data: object             # bytes / numpy uint8 (host) or a CUDA uint8 tensor
    t_arrive: float = 0.0
    t_admit: float = 0.0
    t_done: float = 0.0
    out: bytes = b""
    n_lines: int = 0
    error: str = ""
    footprint: int = 0

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrive


# A slot's aggregate requests go into one mixed batch from this many on
# (a few requests gain little from it, and a batch per query is the
# faster kernel).
MIXED_MIN = 16


def footprint(nbytes: int, fmt: str) -> int:
    """Device bytes a request may hold while in flight: its NDJSON in the
    arena (CSV grows about 1.5x when converted, bounded here by 2x), row
    output up to 1.25x, and a fixed part for tables."""
    nd = nbytes * 2 if fmt == "csv" else nbytes
    return nd + nd + nd // 4 + (1 << 20)


def admit_count(footprints, in_flight: int, budget: int) -> int:
    """How many of the waiting requests (in arrival order) a free slot takes:
    the longest prefix whose footprints fit beside what is in flight.  A
    request that does not fit waits, and so does everything behind it (no
    overtaking, so a large request is not starved by small ones)."""
    total, k = 0, 0
    for f in footprints:
        if in_flight + total + f > budget:
            break
        total += f
        k += 1
    return k


class _Slot:
    def __init__(self, queries, fmt_out, chunk_bytes):
        import torch
        self.stream = torch.cuda.Stream()
        self.qs = {q: Query(q, fmt=fmt_out, chunk_bytes=chunk_bytes) for q in queries}
        # runs a slot's aggregate requests of several queries as one mixed batch
        self.driver = Query("count", fmt=fmt_out, chunk_bytes=chunk_bytes)
        self.mixed: list = []  # (request, address, bytes) of the mixed batch in flight
        self.arena = torch.empty(0, dtype=torch.uint8, device="cuda")
        self.conv = CsvConverter()
        self.event = None
        self.reqs: list = []
        self.used_queries: dict = {}
        self.keep: list = []  # converted CSV inputs of the batch in flight
        self.footprint = 0

    def busy(self) -> bool:
        return bool(self.reqs)

    def close(self):
        for q in self.qs.values():
            q.close()
        self.driver.close()
        self.conv.close()


class Server:
    """Continuous-batching server for a fixed set of queries.

    submit() enqueues a request; poll() completes finished slots and admits
    waiting requests into free ones (call it in a loop); drain() polls until
    every submitted request is done.  `budget_bytes` caps the device memory
    that admitted requests may hold at once (a request alone over the budget
    is refused with an error); `max_batch` caps the requests a slot takes
    (1 with one slot serves requests one at a time); with `mixed`, a slot's
    aggregate requests of two or more queries, MIXED_MIN or more of them,
    run as one mixed batch (one launch sequence and one collect, each input
    with its own plan) instead of one batch per query."""

    def __init__(self, queries, n_slots: int = 3, budget_bytes: int = 120 << 30, fmt_out: str = "ndjson",
                 chunk_bytes: int = 1 << 20, max_batch: int = 0, mixed: bool = True):
        self.max_batch = max_batch  # requests per slot at most (0: no limit)
        self.mixed = mixed          # a slot's aggregate requests of several queries in one launch
        self.queries = list(dict.fromkeys(queries))
        self.slots = [_Slot(self.queries, fmt_out, chunk_bytes) for _ in range(n_slots)]
        self.budget = budget_bytes
        self.waiting = collections.deque()
        self.in_flight_bytes = 0
        self.done: list = []
        self._next_id = 0

    # -- requests ---------------------------------------------------------
    def submit(self, query: str, data, fmt: str = "ndjson", t_arrive: float | None = None) -> Request:
        if query not in self.slots[0].qs:
            raise KeyError(f"the server was not opened with query {query!r}")
        if fmt not in ("ndjson", "csv"):
            raise ValueError("fmt is 'ndjson' or 'csv'")
        n = int(data.numel()) if hasattr(data, "numel") else len(data)
        r = Request(self._next_id, query, fmt, n, data,
                    t_arrive=time.perf_counter() if t_arrive is None else t_arrive)
        r.footprint = footprint(n, fmt)
        self._next_id += 1
        if r.footprint > self.budget:
            r.error = f"request of {n} bytes needs {r.footprint} bytes of device memory, over the budget"
            r.t_done = time.perf_counter()
            self.done.append(r)
        else:
            self.waiting.append(r)
        return r

    def warm(self, reserve_bytes: int = 64 << 20):
        """Runs every slot's every query once over `reserve_bytes` of blank
        lines, and every slot's CSV converter over up to 64 MiB, so contexts
        and converters reach their sizes (records, nesting stack, group
        table, row buffers, CSV tables for inputs that large) and every
        kernel is loaded before requests arrive: serving then allocates
        (and synchronises the device in cudaFree) only for larger inputs."""
        import torch
        buf = torch.full((reserve_bytes + 16,), 0x20, dtype=torch.uint8, device="cuda")
        buf[4095::4096] = 0x0A
        line = b'{"a":"x","b":1}\n'
        small = torch.frombuffer(bytearray(line + bytes(16)), dtype=torch.uint8).cuda()
        rows = b"a,b\n" + b'"x",1\n' * (min(reserve_bytes, 64 << 20) // 6)
        csv = torch.frombuffer(bytearray(rows + bytes(16)), dtype=torch.uint8).cuda()
        for s in self.slots:
            with torch.cuda.stream(s.stream):
                for Q in s.qs.values():
                    Q.batch_launch(buf.data_ptr(), [0], [reserve_bytes], s.stream.cuda_stream)
                    Q.batch_collect()
                    # the render path on a line with every kind of result
                    Q.batch_launch(small.data_ptr(), [0], [len(line)], s.stream.cuda_stream)
                    items, all_ = Q.batch_collect()
                    Q.batch_outputs(items, all_, self._gather_keys(s, all_, base=small.data_ptr()))
                # the mixed path: every aggregate query over the blank lines
                aggs = [Q for Q in s.qs.values() if Q.is_aggregate]
                if self.mixed and len(aggs) > 1:
                    s.driver.batch_launch_mixed(aggs, buf.data_ptr(), [0] * len(aggs), [reserve_bytes] * len(aggs),
                                                s.stream.cuda_stream)
                    s.driver.batch_collect()
                # the CSV kernels and the converter's buffers
                s.conv.reset()
                s.conv.convert(csv.data_ptr(), len(rows), stream=s.stream.cuda_stream)
        torch.cuda.synchronize()

    def pending(self) -> int:
        return len(self.waiting) + sum(len(s.reqs) for s in self.slots)

    # -- the loop ---------------------------------------------------------
    def poll(self) -> list:
        """One turn of the loop; returns the requests completed in it."""
        finished = []
        for s in self.slots:
            if s.busy() and s.event.query():
                finished += self._complete(s)
        for s in self.slots:
            if not s.busy() and self.waiting:
                self._admit(s)
        return finished

    def drain(self) -> list:
        """Polls until every submitted request is done; when a turn neither
        completes nor admits anything, it waits on the oldest busy slot's
        event instead of spinning."""
        out = []
        while self.pending():
            waiting = len(self.waiting)
            got = self.poll()
            out += got
            if not got and len(self.waiting) == waiting:
                busy = [s for s in self.slots if s.busy()]
                if busy:
                    busy[0].event.synchronize()
        return out

    def close(self):
        for s in self.slots:
            s.close()

    # -- internals --------------------------------------------------------
    def _admit(self, s: _Slot):
        import torch
        k = admit_count([r.footprint for r in self.waiting], self.in_flight_bytes, self.budget)
        if self.max_batch:
            k = min(k, self.max_batch)
        if not k:
            return
        take = [self.waiting.popleft() for _ in range(k)]
        total = sum(r.footprint for r in take)
        now = time.perf_counter()
        with torch.cuda.stream(s.stream):
            # 1. every request's NDJSON at a 16-byte aligned device address:
            #    device inputs in place, CSV converted on the device (the
            #    converter's buffer serves one conversion at a time, so each
            #    result is copied out), host inputs copied into the arena
            addrs, keep, host = [None] * len(take), [], []
            for i, r in enumerate(take):
                r.t_admit = now
                if r.fmt == "csv":
                    src = self._device_bytes(r.data)
                    s.conv.reset()
                    d, nd, _, _ = s.conv.convert(src.data_ptr(), r.nbytes, stream=s.stream.cuda_stream)
                    t = torch.empty(nd + 16, dtype=torch.uint8, device="cuda")
                    if nd:
                        t[:nd].copy_(_device_tensor(d, nd))
                    keep.append(t)
                    addrs[i] = (t.data_ptr(), nd)
                elif hasattr(r.data, "is_cuda") and r.data.is_cuda and r.data.data_ptr() % 16 == 0:
                    addrs[i] = (r.data.data_ptr(), r.nbytes)
                else:
                    host.append(i)
            pos, offs = 0, {}
            for i in host:
                pos = (pos + 15) & ~15
                offs[i] = pos
                pos += take[i].nbytes
            if host and s.arena.numel() < pos + 16:
                s.arena = torch.empty(int((pos + 16) * 1.25), dtype=torch.uint8, device="cuda")
            for i in host:
                src, n, o = take[i].data, take[i].nbytes, offs[i]
                if n:
                    if hasattr(src, "is_cuda") and src.is_cuda:
                        s.arena[o:o + n].copy_(src.view(torch.uint8).reshape(-1)[:n])
                    else:
                        h = np.frombuffer(bytes(src), dtype=np.uint8) if isinstance(src, (bytes, bytearray)) \
                            else np.asarray(src, dtype=np.uint8).reshape(-1)
                        s.arena[o:o + n].copy_(torch.from_numpy(h[:n].copy()).pin_memory(), non_blocking=True)
                addrs[i] = (s.arena.data_ptr() + o, n)
            # 2. one batch per query among them, by device address
            by_q = {}
            for r, (addr, n) in zip(take, addrs):
                by_q.setdefault(r.query, []).append((r, addr, n))
            agg = [q for q in by_q if s.qs[q].is_aggregate]
            s.mixed = []
            if self.mixed and len(agg) > 1 and sum(len(by_q[q]) for q in agg) >= MIXED_MIN:
                s.mixed = [x for q in agg for x in by_q.pop(q)]
                s.driver.batch_launch_mixed([s.qs[r.query] for r, _, _ in s.mixed], 0,
                                            [a for _, a, _ in s.mixed], [n for _, _, n in s.mixed],
                                            s.stream.cuda_stream)
            for q, lst in by_q.items():
                s.qs[q].batch_launch(0, [a for _, a, _ in lst], [n for _, _, n in lst], s.stream.cuda_stream)
            s.event = torch.cuda.Event()
            s.event.record(s.stream)
        s.keep = keep
        s.reqs = take
        s.used_queries = by_q
        s.footprint = total
        self.in_flight_bytes += total

    @staticmethod
    def _device_bytes(data):
        import torch
        if hasattr(data, "is_cuda") and data.is_cuda:
            return data.view(torch.uint8).reshape(-1)
        host = np.frombuffer(bytes(data), dtype=np.uint8) if isinstance(data, (bytes, bytearray)) else np.asarray(data)
        t = torch.empty(host.size + 16, dtype=torch.uint8, device="cuda")
        if host.size:
            t[:host.size].copy_(torch.from_numpy(host.copy()))
        return t

    def _complete(self, s: _Slot) -> list:
        done_at = time.perf_counter()
        out = []
        if s.mixed:
            items, all_ = s.driver.batch_collect()
            keys = self._gather_keys(s, all_)
            outs = batch_outputs_mixed([s.qs[r.query] for r, _, _ in s.mixed], items, all_, keys)
            for (r, _, _), it, o in zip(s.mixed, items, outs):
                r.out = o
                r.n_lines = it.n_lines - it.n_blank
                r.t_done = done_at
                out.append(r)
            s.mixed = []
        for q, lst in s.used_queries.items():
            Q = s.qs[q]
            items, all_ = Q.batch_collect()
            keys = self._gather_keys(s, all_)
            outs = Q.batch_outputs(items, all_, keys)
            for (r, _, _), it, o in zip(lst, items, outs):
                r.out = o
                r.n_lines = it.n_lines - it.n_blank
                r.t_done = done_at
                out.append(r)
        self.in_flight_bytes -= s.footprint
        s.reqs, s.used_queries, s.footprint, s.event, s.keep = [], {}, 0, None, []
        self.done += out
        return out

    def _gather_keys(self, s: _Slot, all_, base: int = 0) -> np.ndarray:
        """Group keys of the batch, gathered from device memory into one host
        buffer; the groups' key offsets (device addresses, or offsets from
        `base`) are rewritten to point into it."""
        n = all_.n_groups
        if not n:
            return np.zeros(1, dtype=np.uint8)
        g = np.ctypeslib.as_array(all_.groups, shape=(n,))
        offs = np.ascontiguousarray(g["key_off"], dtype=np.uint64)
        lens = np.ascontiguousarray(g["key_len"], dtype=np.uint32)
        buf = np.zeros(int(lens.sum()) + 1, dtype=np.uint8)
        s.conv.gather(base, offs, lens, n, buf, s.stream.cuda_stream)
        at = np.zeros(n, dtype=np.uint64)
        np.cumsum(lens[:-1], out=at[1:])
        g["key_off"] = at
        return buf


def _device_tensor(ptr: int, n: int):
    """A uint8 tensor viewing n bytes of device memory (no copy)."""
    import torch
    from .shard import _DeviceBytes
    return torch.as_tensor(_DeviceBytes(ptr, n), device="cuda")


# ---------------------------------------------------------------------------
# The native server (include/warpjq_serve.h): the same continuous batching,
# with the loop, admission, placement and rendering in a C++ thread.
# ---------------------------------------------------------------------------

import ctypes as _ct


class _ServeConfig(_ct.Structure):
    _fields_ = [("n_slots", _ct.c_uint32), ("max_batch", _ct.c_uint32), ("budget_bytes", _ct.c_uint64),
                ("format", _ct.c_uint32), ("mixed_min", _ct.c_uint32), ("chunk_bytes", _ct.c_uint64),
                ("slot_bytes", _ct.c_uint64)]


class _ServeResult(_ct.Structure):
    _fields_ = [("id", _ct.c_uint64), ("query", _ct.c_uint32), ("rc", _ct.c_int32), ("out", _ct.c_void_p),
                ("out_len", _ct.c_uint64), ("n_lines", _ct.c_uint64), ("n_invalid", _ct.c_uint64),
                ("queue_ms", _ct.c_double), ("latency_ms", _ct.c_double), ("err", _ct.c_char * 160)]


SERVE_DEVICE = 1
SERVE_CSV = 2


@dataclass
class NativeResult:
    id: int
    query: int
    rc: int
    out: bytes
    n_lines: int
    n_invalid: int
    queue_ms: float
    latency_ms: float
    error: str


class NativeServer:
    """Binding of the native serving loop (warpjq_serve_*).  submit() queues
    a request and returns its id (the input must stay alive and unchanged
    until its result is polled: the server keeps a reference to it here);
    poll() returns finished requests; drain() waits for all of them."""

    def __init__(self, queries, n_slots: int = 3, budget_bytes: int = 120 << 30, fmt_out: str = "ndjson",
                 max_batch: int = 0, mixed_min: int = MIXED_MIN, chunk_bytes: int = 1 << 20,
                 slot_bytes: int = 1 << 30):
        from . import FORMATS, _load
        _, h = _load()
        self._h = h
        vp, u32, u64, cp = _ct.c_void_p, _ct.c_uint32, _ct.c_uint64, _ct.c_char_p
        h.warpjq_serve_open.argtypes = [_ct.POINTER(cp), u32, _ct.POINTER(_ServeConfig), _ct.POINTER(vp), cp,
                                        _ct.c_size_t]
        h.warpjq_serve_open.restype = _ct.c_int
        h.warpjq_serve_warm.argtypes = [vp, u64, cp, _ct.c_size_t]
        h.warpjq_serve_warm.restype = _ct.c_int
        h.warpjq_serve_enqueue.argtypes = [vp, u32, vp, u64, u32, _ct.POINTER(u64), cp, _ct.c_size_t]
        h.warpjq_serve_enqueue.restype = _ct.c_int
        h.warpjq_serve_poll.argtypes = [vp, _ct.POINTER(_ServeResult), u32, _ct.c_int]
        h.warpjq_serve_poll.restype = u32
        h.warpjq_serve_pending.argtypes = [vp]
        h.warpjq_serve_pending.restype = u64
        h.warpjq_serve_close.argtypes = [vp]
        h.warpjq_serve_close.restype = None
        self.queries = list(dict.fromkeys(queries))
        self._index = {q: i for i, q in enumerate(self.queries)}
        arr = (cp * len(self.queries))(*[q.encode() for q in self.queries])
        cfg = _ServeConfig(n_slots, max_batch, budget_bytes, FORMATS[fmt_out], mixed_min, chunk_bytes, slot_bytes)
        self._s = vp()
        err = _ct.create_string_buffer(1024)
        rc = h.warpjq_serve_open(arr, len(self.queries), _ct.byref(cfg), _ct.byref(self._s), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))
        self._keep = {}  # request id -> the input object (kept alive until polled)
        self._buf = (_ServeResult * 256)()

    def warm(self, reserve_bytes: int = 64 << 20):
        err = _ct.create_string_buffer(1024)
        if self._h.warpjq_serve_warm(self._s, reserve_bytes, err, len(err)):
            raise RuntimeError(err.value.decode(errors="replace"))

    def submit(self, query: str, data, fmt: str = "ndjson") -> int:
        """Queues `query` over `data`: bytes / a numpy uint8 array (host) or
        a CUDA uint8 tensor (device, used in place when 16-byte aligned)."""
        flags = SERVE_CSV if fmt == "csv" else 0
        if hasattr(data, "is_cuda") and data.is_cuda:
            flags |= SERVE_DEVICE
            ptr, n = data.data_ptr(), int(data.numel())
        elif isinstance(data, (bytes, bytearray)):
            data = np.frombuffer(data, dtype=np.uint8)
            ptr, n = data.ctypes.data, data.size
        else:
            data = np.ascontiguousarray(data, dtype=np.uint8).reshape(-1)
            ptr, n = data.ctypes.data, data.size
        rid = _ct.c_uint64()
        err = _ct.create_string_buffer(512)
        if self._h.warpjq_serve_enqueue(self._s, self._index[query], ptr, n, flags, _ct.byref(rid), err, len(err)):
            raise RuntimeError(err.value.decode(errors="replace"))
        self._keep[rid.value] = data
        return rid.value

    def poll(self, timeout_ms: int = 0) -> list:
        n = self._h.warpjq_serve_poll(self._s, self._buf, len(self._buf), timeout_ms)
        out = []
        for i in range(n):
            r = self._buf[i]
            body = _ct.string_at(r.out, r.out_len) if r.out else b""
            if r.out:
                self._h.warpjq_host_free(_ct.c_void_p(r.out))
            self._keep.pop(r.id, None)
            out.append(NativeResult(r.id, r.query, r.rc, body, r.n_lines, r.n_invalid, r.queue_ms, r.latency_ms,
                                    r.err.decode(errors="replace")))
        return out

    def pending(self) -> int:
        return int(self._h.warpjq_serve_pending(self._s))

    def drain(self) -> list:
        out = []
        while self.pending():
            out += self.poll(timeout_ms=-1)
        return out

    def close(self):
        if self._s:
            self._h.warpjq_serve_close(self._s)
            self._s = _ct.c_void_p()
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
