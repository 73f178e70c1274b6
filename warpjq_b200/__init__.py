"""warpjq_b200: a B200-native (sm_100a) backend for warpjq's NDJSON scan path.

The product is native code behind a C ABI:
  * libwarpjq_kernels.so -- the device backend with the reference's
    warpjq_kernels.h ABI (include/warpjq_kernels.h) plus the device-resident
    extension (include/warpjq_ext.h);
  * libwarpjq_host.so -- the host driver (include/warpjq_host.h) that parses
    a jq-subset query, streams input through the ABI and formats the output
    as warpjq does.

This module is the Python mirror of that interface, through ctypes.  It
never evaluates a line itself: if the native libraries are missing it raises.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "_lib")
KERNELS_SO = os.path.join(LIB_DIR, "libwarpjq_kernels.so")
HOST_SO = os.path.join(LIB_DIR, "libwarpjq_host.so")

FORMATS = {"ndjson": 0, "csv": 1, "count": 2}
ON_INVALID = {"warn": 0, "skip": 1, "abort": 2}

# Every symbol include/*.h declares, by library.
ABI_SYMBOLS = [
    "warpjq_probe", "warpjq_abi_check", "warpjq_ctx_create", "warpjq_ctx_destroy",
    "warpjq_slot_buffer", "warpjq_slot_capacity", "warpjq_max_lines", "warpjq_submit",
    "warpjq_wait", "warpjq_device_name",
]
EXT_SYMBOLS = [
    "warpjq_launch_device", "warpjq_collect_device", "warpjq_slot_first_errors",
    "warpjq_set_tiling", "warpjq_autotile", "warpjq_submit_host", "warpjq_host_is_pinned",
    "warpjq_batch_launch", "warpjq_batch_collect", "warpjq_host_alloc_pinned",
    "warpjq_host_free_pinned", "warpjq_csv_create", "warpjq_csv_destroy", "warpjq_csv_reset",
    "warpjq_csv_convert", "warpjq_csv_gather", "warpjq_device_read", "warpjq_batch_graph_create",
    "warpjq_batch_graph_launch", "warpjq_batch_graph_destroy", "warpjq_set_group_capacity",
    "warpjq_batch_launch_mixed",
]
HOST_SYMBOLS = [
    "warpjq_query_open", "warpjq_query_close", "warpjq_query_ctx", "warpjq_query_is_aggregate",
    "warpjq_query_run", "warpjq_run_bytes", "warpjq_query_render_device", "warpjq_host_free",
    "warpjq_gen_nginx", "warpjq_gen_nginx_block", "warpjq_query_open_host", "warpjq_query_is_grouped",
    "warpjq_gen_nested", "warpjq_gen_nested_block", "warpjq_query_run_file", "warpjq_query_run_csv",
    "warpjq_gen_nginx_csv", "warpjq_gen_nginx_csv_block", "warpjq_gen_nginx_csv_as_ndjson",
    "warpjq_query_render_batch", "warpjq_serve_open", "warpjq_serve_warm", "warpjq_serve_enqueue",
    "warpjq_serve_poll", "warpjq_serve_pending", "warpjq_serve_close",
]


class NativeLibraryMissing(RuntimeError):
    pass


_kern = None
_host = None


def _load():
    global _kern, _host
    if _host is not None:
        return _kern, _host
    for p in (KERNELS_SO, HOST_SO):
        if not os.path.exists(p):
            raise NativeLibraryMissing(
                f"{p} is not built; run `python -m warpjq_b200.build` (no CPU fallback exists)")
    k = ctypes.CDLL(KERNELS_SO, mode=ctypes.RTLD_GLOBAL)
    h = ctypes.CDLL(HOST_SO)
    vp, sz, u64, u32, cp = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_char_p
    k.warpjq_probe.argtypes = [cp, sz]
    k.warpjq_probe.restype = ctypes.c_int
    k.warpjq_abi_check.argtypes = [ctypes.POINTER(u64), sz]
    k.warpjq_abi_check.restype = ctypes.c_int
    k.warpjq_device_name.argtypes = [cp, sz]
    k.warpjq_device_name.restype = ctypes.c_int
    k.warpjq_launch_device.argtypes = [vp, vp, u64, vp, cp, sz]
    k.warpjq_launch_device.restype = ctypes.c_int
    k.warpjq_collect_device.argtypes = [vp, vp, cp, sz]
    k.warpjq_collect_device.restype = ctypes.c_int
    k.warpjq_set_tiling.argtypes = [vp, u32, u32]
    k.warpjq_set_tiling.restype = ctypes.c_int
    k.warpjq_set_group_capacity.argtypes = [vp, u32]
    k.warpjq_set_group_capacity.restype = ctypes.c_int
    k.warpjq_autotile.argtypes = [vp, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(u32),
                                  ctypes.POINTER(u32)]
    k.warpjq_autotile.restype = ctypes.c_int
    k.warpjq_batch_launch.argtypes = [vp, vp, ctypes.POINTER(u64), ctypes.POINTER(u64), u32, vp, cp, sz]
    k.warpjq_batch_launch.restype = ctypes.c_int
    k.warpjq_batch_launch_mixed.argtypes = [vp, ctypes.POINTER(vp), vp, ctypes.POINTER(u64), ctypes.POINTER(u64),
                                            u32, vp, cp, sz]
    k.warpjq_batch_launch_mixed.restype = ctypes.c_int
    k.warpjq_batch_collect.argtypes = [vp, vp, vp, cp, sz]
    k.warpjq_batch_collect.restype = ctypes.c_int
    h.warpjq_query_open.argtypes = [cp, u32, u64, ctypes.POINTER(vp), cp, sz]
    h.warpjq_query_open.restype = ctypes.c_int
    h.warpjq_query_close.argtypes = [vp]
    h.warpjq_query_ctx.argtypes = [vp]
    h.warpjq_query_ctx.restype = vp
    h.warpjq_query_is_aggregate.argtypes = [vp]
    h.warpjq_query_is_aggregate.restype = ctypes.c_int
    h.warpjq_query_open_host.argtypes = [cp, u32, ctypes.POINTER(vp), cp, sz]
    h.warpjq_query_open_host.restype = ctypes.c_int
    h.warpjq_query_is_grouped.argtypes = [vp]
    h.warpjq_query_is_grouped.restype = ctypes.c_int
    h.warpjq_query_run.argtypes = [vp, vp, sz, u32, u64, ctypes.POINTER(vp), ctypes.POINTER(sz),
                                   ctypes.POINTER(u64), cp, sz]
    h.warpjq_query_run.restype = ctypes.c_int
    h.warpjq_query_run_file.argtypes = [vp, cp, u32, u64, ctypes.POINTER(vp), ctypes.POINTER(sz),
                                        ctypes.POINTER(u64), cp, sz]
    h.warpjq_query_run_file.restype = ctypes.c_int
    k.warpjq_batch_graph_create.argtypes = [ctypes.POINTER(vp), u32, ctypes.POINTER(vp), ctypes.POINTER(vp),
                                            ctypes.POINTER(vp), ctypes.POINTER(u32), ctypes.POINTER(vp), cp, sz]
    k.warpjq_batch_graph_create.restype = ctypes.c_int
    k.warpjq_batch_graph_launch.argtypes = [vp, vp, cp, sz]
    k.warpjq_batch_graph_launch.restype = ctypes.c_int
    k.warpjq_batch_graph_destroy.argtypes = [vp]
    k.warpjq_csv_create.argtypes = [ctypes.POINTER(vp)]
    k.warpjq_csv_create.restype = ctypes.c_int
    k.warpjq_csv_destroy.argtypes = [vp]
    k.warpjq_csv_reset.argtypes = [vp]
    k.warpjq_csv_convert.argtypes = [vp, vp, u64, u32, vp, ctypes.POINTER(vp), ctypes.POINTER(u64),
                                     ctypes.POINTER(u64), ctypes.POINTER(u64), cp, sz]
    k.warpjq_csv_convert.restype = ctypes.c_int
    k.warpjq_csv_gather.argtypes = [vp, vp, ctypes.POINTER(u64), ctypes.POINTER(u32), u64, vp, vp, cp, sz]
    k.warpjq_csv_gather.restype = ctypes.c_int
    h.warpjq_query_run_csv.argtypes = [vp, vp, sz, u32, ctypes.POINTER(vp), ctypes.POINTER(sz),
                                       ctypes.POINTER(u64), cp, sz]
    h.warpjq_query_run_csv.restype = ctypes.c_int
    h.warpjq_gen_nginx_csv.argtypes = [u64, vp, u64, u64, ctypes.c_uint, ctypes.POINTER(u64)]
    h.warpjq_gen_nginx_csv.restype = u64
    h.warpjq_gen_nginx_csv_as_ndjson.argtypes = [u64, vp, u64, u64, ctypes.c_uint, ctypes.POINTER(u64)]
    h.warpjq_gen_nginx_csv_as_ndjson.restype = u64
    h.warpjq_run_bytes.argtypes = [cp, cp, sz, u32, u32, u64, u64, ctypes.POINTER(vp),
                                   ctypes.POINTER(sz), ctypes.POINTER(u64), cp, sz]
    h.warpjq_run_bytes.restype = ctypes.c_int
    h.warpjq_query_render_device.argtypes = [vp, vp, vp, ctypes.POINTER(vp), ctypes.POINTER(sz)]
    h.warpjq_query_render_device.restype = ctypes.c_int
    h.warpjq_query_render_batch.argtypes = [vp, vp, u32, vp, vp, vp, vp, ctypes.POINTER(vp), ctypes.POINTER(sz),
                                            ctypes.POINTER(u64)]
    h.warpjq_query_render_batch.restype = ctypes.c_int
    h.warpjq_host_free.argtypes = [vp]
    h.warpjq_gen_nginx.argtypes = [u64, vp, u64, u64, ctypes.c_uint, ctypes.POINTER(u64)]
    h.warpjq_gen_nginx.restype = u64
    h.warpjq_gen_nested.argtypes = [u64, vp, u64, u64, ctypes.c_uint, u64, ctypes.POINTER(u64)]
    h.warpjq_gen_nested.restype = u64
    _kern, _host = k, h
    return k, h


def libraries():
    """(kernels, host) ctypes handles; raises NativeLibraryMissing."""
    return _load()


@dataclass
class RunResult:
    rc: int
    out: bytes
    stats: dict
    err: str


def _take(ptr, n) -> bytes:
    if not ptr.value:
        return b""
    b = ctypes.string_at(ptr.value, n.value)
    _load()[1].warpjq_host_free(ptr)
    return b


class _HostBuffer:
    """A malloc'd result buffer of the host library, exposed to numpy
    without a copy and freed with the last array that views it."""

    def __init__(self, ptr: int, n: int):
        self.ptr, self.n = ptr, n
        self.__array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr or 0, False),
                                    "version": 3}

    def __del__(self):
        if self.ptr:
            try:
                _load()[1].warpjq_host_free(ctypes.c_void_p(self.ptr))
            except Exception:  # interpreter shutdown: the process frees it
                pass
            self.ptr = 0


def _view(ptr, n):
    import numpy as np
    if not ptr.value:
        return np.zeros(0, dtype=np.uint8)
    return np.asarray(_HostBuffer(ptr.value, n.value))


def _stats(arr):
    return dict(zip(["bytes_in", "lines_in", "lines_out", "malformed", "type_errors"], list(arr)))


def run_bytes(query: str, data: bytes, fmt: str = "ndjson", on_invalid: str = "skip",
              chunk_bytes: int = 0, max_line_bytes: int = 0) -> RunResult:
    """Runs `query` over `data` on the GPU, like warpjq's run_bytes."""
    _, h = _load()
    out = ctypes.c_void_p()
    n = ctypes.c_size_t()
    st = (ctypes.c_uint64 * 5)()
    err = ctypes.create_string_buffer(4096)
    rc = h.warpjq_run_bytes(query.encode(), data, len(data), FORMATS[fmt], ON_INVALID[on_invalid],
                            chunk_bytes, max_line_bytes, ctypes.byref(out), ctypes.byref(n), st,
                            err, len(err))
    return RunResult(rc, _take(out, n), _stats(st), err.value.decode(errors="replace"))


class _GroupExt(ctypes.Structure):
    _fields_ = [("key_off", ctypes.c_uint64), ("key_len", ctypes.c_uint32),
                ("key_kind", ctypes.c_uint32), ("count", ctypes.c_uint64),
                ("numeric", ctypes.c_uint64), ("isum_lo", ctypes.c_uint64),
                ("isum_hi", ctypes.c_uint64), ("n_int", ctypes.c_uint64),
                ("fsum", ctypes.c_double), ("min", ctypes.c_double), ("max", ctypes.c_double),
                ("sum", ctypes.c_double)]


class DeviceResult(ctypes.Structure):
    """Mirror of warpjq_device_result (include/warpjq_ext.h)."""
    _fields_ = [("n_lines", ctypes.c_uint64), ("n_blank", ctypes.c_uint64),
                ("n_invalid", ctypes.c_uint64), ("n_type_error", ctypes.c_uint64),
                ("n_selected", ctypes.c_uint64), ("first_invalid", ctypes.c_uint64),
                ("first_type_error", ctypes.c_uint64),
                ("d_out_bytes", ctypes.c_void_p), ("out_len", ctypes.c_uint64),
                ("d_out_line_idx", ctypes.c_void_p), ("d_out_row_off", ctypes.c_void_p),
                ("count", ctypes.c_uint64), ("numeric", ctypes.c_uint64),
                ("isum_lo", ctypes.c_uint64), ("isum_hi", ctypes.c_uint64),
                ("n_int", ctypes.c_uint64), ("fsum", ctypes.c_double), ("min", ctypes.c_double),
                ("max", ctypes.c_double), ("sum", ctypes.c_double),
                ("saw_non_numeric", ctypes.c_uint32), ("groups", ctypes.POINTER(_GroupExt)),
                ("n_groups", ctypes.c_uint32), ("kernels_launched", ctypes.c_uint32),
                ("scan_ms", ctypes.c_double)]

    def isum(self) -> int:
        v = (self.isum_hi << 64) | self.isum_lo
        return v - (1 << 128) if self.isum_hi >> 63 else v


class BatchItem(ctypes.Structure):
    """Mirror of warpjq_batch_item (include/warpjq_ext.h)."""
    _fields_ = [("n_lines", ctypes.c_uint64), ("n_blank", ctypes.c_uint64),
                ("n_invalid", ctypes.c_uint64), ("n_type_error", ctypes.c_uint64),
                ("n_selected", ctypes.c_uint64), ("first_invalid", ctypes.c_uint64),
                ("first_type_error", ctypes.c_uint64), ("row_begin", ctypes.c_uint64),
                ("line_begin", ctypes.c_uint64), ("count", ctypes.c_uint64),
                ("numeric", ctypes.c_uint64), ("isum_lo", ctypes.c_uint64),
                ("isum_hi", ctypes.c_uint64), ("n_int", ctypes.c_uint64), ("fsum", ctypes.c_double),
                ("min", ctypes.c_double), ("max", ctypes.c_double), ("sum", ctypes.c_double),
                ("saw_non_numeric", ctypes.c_uint32), ("group_begin", ctypes.c_uint32),
                ("n_groups", ctypes.c_uint32), ("_pad", ctypes.c_uint32)]


class Query:
    """A compiled query with its device context (warpjq_query_open)."""

    def __init__(self, query: str, fmt: str = "ndjson", chunk_bytes: int = 0, device: bool = True):
        """device=False parses and lowers only (no device context): such a
        query renders merged results (render_device) but cannot run."""
        _, h = _load()
        self._h = h
        self._q = ctypes.c_void_p()
        err = ctypes.create_string_buffer(4096)
        if device:
            rc = h.warpjq_query_open(query.encode(), FORMATS[fmt], chunk_bytes, ctypes.byref(self._q),
                                     err, len(err))
        else:
            rc = h.warpjq_query_open_host(query.encode(), FORMATS[fmt], ctypes.byref(self._q), err,
                                          len(err))
        if rc:
            raise ValueError(err.value.decode(errors="replace")) if rc == 2 else \
                RuntimeError(err.value.decode(errors="replace"))
        self.query = query
        self.fmt = fmt

    def close(self):
        if self._q:
            self._h.warpjq_query_close(self._q)
            self._q = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ctx(self):
        return self._h.warpjq_query_ctx(self._q)

    @property
    def is_aggregate(self) -> bool:
        return bool(self._h.warpjq_query_is_aggregate(self._q))

    @property
    def is_grouped(self) -> bool:
        return bool(self._h.warpjq_query_is_grouped(self._q))

    def run(self, data, on_invalid: str = "skip", max_line_bytes: int = 0,
            copy_out: bool = True) -> RunResult:
        """Runs over host memory: `data` is bytes, or a numpy uint8 array.
        With copy_out=False the output is a numpy uint8 view of the host
        library's buffer (no copy; freed with the array)."""
        if isinstance(data, (bytes, bytearray)):
            keep = ctypes.c_char_p(bytes(data))
            addr, n_bytes = ctypes.cast(keep, ctypes.c_void_p), len(data)
        else:
            addr, n_bytes = ctypes.c_void_p(data.ctypes.data), int(data.nbytes)
        out = ctypes.c_void_p()
        n = ctypes.c_size_t()
        st = (ctypes.c_uint64 * 5)()
        err = ctypes.create_string_buffer(4096)
        rc = self._h.warpjq_query_run(self._q, addr, n_bytes, ON_INVALID[on_invalid],
                                      max_line_bytes, ctypes.byref(out), ctypes.byref(n), st, err,
                                      len(err))
        body = _take(out, n) if copy_out else _view(out, n)
        return RunResult(rc, body, _stats(st), err.value.decode(errors="replace"))

    def run_file(self, path: str, on_invalid: str = "skip", max_line_bytes: int = 0,
                 copy_out: bool = True) -> RunResult:
        """Runs over a file (parallel reads into page-locked buffers,
        overlapped with the device)."""
        out = ctypes.c_void_p()
        n = ctypes.c_size_t()
        st = (ctypes.c_uint64 * 5)()
        err = ctypes.create_string_buffer(4096)
        rc = self._h.warpjq_query_run_file(self._q, path.encode(), ON_INVALID[on_invalid],
                                           max_line_bytes, ctypes.byref(out), ctypes.byref(n), st,
                                           err, len(err))
        body = _take(out, n) if copy_out else _view(out, n)
        return RunResult(rc, body, _stats(st), err.value.decode(errors="replace"))

    def run_csv(self, data, on_invalid: str = "skip", copy_out: bool = True) -> RunResult:
        """Runs over CSV in host memory (bytes or a numpy uint8 array): the
        header names the keys, each later row is one object, converted on
        the device (warpjq_query_run_csv)."""
        if isinstance(data, (bytes, bytearray)):
            keep = ctypes.c_char_p(bytes(data))
            addr, n_bytes = ctypes.cast(keep, ctypes.c_void_p), len(data)
        else:
            addr, n_bytes = ctypes.c_void_p(data.ctypes.data), int(data.nbytes)
        out = ctypes.c_void_p()
        n = ctypes.c_size_t()
        st = (ctypes.c_uint64 * 5)()
        err = ctypes.create_string_buffer(4096)
        rc = self._h.warpjq_query_run_csv(self._q, addr, n_bytes, ON_INVALID[on_invalid], ctypes.byref(out),
                                          ctypes.byref(n), st, err, len(err))
        body = _take(out, n) if copy_out else _view(out, n)
        return RunResult(rc, body, _stats(st), err.value.decode(errors="replace"))

    def set_tiling(self, tile_bytes: int = 0, halo_bytes: int = 0):
        k, _ = _load()
        if k.warpjq_set_tiling(self.ctx, tile_bytes, halo_bytes) != 0:
            raise ValueError("bad tiling")

    def set_group_capacity(self, keys: int):
        """Room for `keys` distinct keys in a fresh group table (a power of
        two, 1024 .. 2^28); the table still grows on overflow."""
        k, _ = _load()
        if k.warpjq_set_group_capacity(self.ctx, keys) != 0:
            raise ValueError("bad group capacity")

    def autotile(self, sample) -> tuple:
        """Chooses the device tiling from a host sample of the input (bytes or
        a uint8 numpy array); returns (tile_bytes, halo_bytes)."""
        k, _ = _load()
        if isinstance(sample, (bytes, bytearray)):
            buf = (ctypes.c_char * len(sample)).from_buffer_copy(sample)
            addr, n = ctypes.addressof(buf), len(sample)
        else:
            addr, n = sample.ctypes.data, sample.nbytes
        t, h = ctypes.c_uint32(), ctypes.c_uint32()
        if k.warpjq_autotile(self.ctx, ctypes.c_void_p(addr), n, ctypes.byref(t), ctypes.byref(h)) != 0:
            raise RuntimeError("autotile failed")
        return t.value, h.value

    def launch_device(self, d_ptr: int, n: int, stream: int = 0):
        """Enqueues a device-resident run (no host synchronisation)."""
        k, _ = _load()
        err = ctypes.create_string_buffer(1024)
        rc = k.warpjq_launch_device(self.ctx, ctypes.c_void_p(d_ptr), n, ctypes.c_void_p(stream),
                                    err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))

    def collect_device(self) -> DeviceResult:
        k, _ = _load()
        r = DeviceResult()
        err = ctypes.create_string_buffer(1024)
        rc = k.warpjq_collect_device(self.ctx, ctypes.byref(r), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))
        return r

    def batch_launch(self, d_ptr: int, offsets, lengths, stream: int = 0):
        """Enqueues one batched run over the device inputs
        d_ptr[offsets[i], offsets[i] + lengths[i]) (16-byte aligned starts)."""
        k, _ = _load()
        n = len(offsets)
        self._b_off = (ctypes.c_uint64 * max(1, n))(*offsets)
        self._b_len = (ctypes.c_uint64 * max(1, n))(*lengths)
        self._b_n = n
        err = ctypes.create_string_buffer(1024)
        rc = k.warpjq_batch_launch(self.ctx, ctypes.c_void_p(d_ptr), self._b_off, self._b_len, n,
                                   ctypes.c_void_p(stream), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))

    def batch_launch_mixed(self, queries, d_ptr: int, offsets, lengths, stream: int = 0):
        """Enqueues one mixed batch on this query's context: input i is
        d_ptr[offsets[i], + lengths[i]) and runs queries[i] (aggregate or row
        queries; one scan launch per distinct query over its inputs' tiles,
        each specialised for that query).  Collect with
        batch_collect() and render with batch_outputs_mixed()."""
        k, _ = _load()
        n = len(offsets)
        self._b_off = (ctypes.c_uint64 * max(1, n))(*offsets)
        self._b_len = (ctypes.c_uint64 * max(1, n))(*lengths)
        ctxs = (ctypes.c_void_p * max(1, n))(*[q.ctx for q in queries])
        self._b_n = n
        err = ctypes.create_string_buffer(1024)
        rc = k.warpjq_batch_launch_mixed(self.ctx, ctxs, ctypes.c_void_p(d_ptr), self._b_off, self._b_len, n,
                                         ctypes.c_void_p(stream), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))

    def batch_collect(self):
        """(items, all): one BatchItem per input, and the batch's
        DeviceResult (rows and groups of every input)."""
        k, _ = _load()
        items = (BatchItem * max(1, self._b_n))()
        all_ = DeviceResult()
        err = ctypes.create_string_buffer(1024)
        rc = k.warpjq_batch_collect(self.ctx, items, ctypes.byref(all_), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))
        self._b_items = items
        return list(items)[: self._b_n], all_

    def batch_outputs(self, items, all_: DeviceResult, host_data) -> list:
        """Each input's output bytes (what a run over it alone prints), from
        one native call (warpjq_query_render_batch): rows cut from one copy
        of the batch's rows, aggregates and groups rendered by the host
        formatter; `host_data` (bytes or a numpy uint8 array) holds the bytes
        the groups' key_off values index (the host copy of the batch buffer,
        or keys gathered from the device)."""
        import numpy as np
        n = len(items)
        # the collected array itself when `items` views it (the usual case),
        # else a contiguous copy
        arr = getattr(self, "_b_items", None)
        if arr is None or len(arr) < n or (n and ctypes.addressof(items[0]) != ctypes.addressof(arr[0])):
            arr = (BatchItem * max(1, n))(*items)
        rows_p = row_off_p = None
        keep = []
        if all_.n_selected and all_.d_out_bytes:  # row queries only
            import torch
            from .shard import _DeviceBytes
            nsel = all_.n_selected
            rows = torch.as_tensor(_DeviceBytes(all_.d_out_bytes, max(1, all_.out_len)), device="cuda").cpu()
            ro = torch.as_tensor(_DeviceBytes(all_.d_out_row_off, (nsel + 1) * 8), device="cuda").cpu()
            keep += [rows, ro]
            rows_p, row_off_p = ctypes.c_void_p(rows.data_ptr()), ctypes.c_void_p(ro.data_ptr())
        if isinstance(host_data, (bytes, bytearray)):
            kb = ctypes.c_char_p(bytes(host_data))
            keep.append(kb)
            kaddr = ctypes.cast(kb, ctypes.c_void_p)
        else:
            kaddr = ctypes.c_void_p(np.asarray(host_data).ctypes.data)
        out = ctypes.c_void_p()
        ln = ctypes.c_size_t()
        offs = (ctypes.c_uint64 * (n + 1))()
        rc = self._h.warpjq_query_render_batch(self._q, arr, n, ctypes.cast(all_.groups, ctypes.c_void_p), kaddr,
                                               rows_p, row_off_p, ctypes.byref(out), ctypes.byref(ln), offs)
        if rc:
            raise MemoryError("warpjq_query_render_batch")
        body = _take(out, ln)
        return [body[offs[i]:offs[i + 1]] for i in range(n)]

    def render_device(self, r: DeviceResult, host_data) -> bytes:
        """Formats a device-resident result; `host_data` (bytes or a numpy
        uint8 array) is the host copy of the input, for group keys."""
        out = ctypes.c_void_p()
        n = ctypes.c_size_t()
        if isinstance(host_data, (bytes, bytearray)):
            keep = ctypes.c_char_p(bytes(host_data))
            addr = ctypes.cast(keep, ctypes.c_void_p)
        else:
            addr = ctypes.c_void_p(host_data.ctypes.data)
        self._h.warpjq_query_render_device(self._q, ctypes.byref(r), addr, ctypes.byref(out),
                                           ctypes.byref(n))
        return _take(out, n)


def batch_outputs_mixed(queries, items, all_, host_data) -> list:
    """Each input's output of a collected mixed batch, rendered by its own
    query (queries[i] for input i); `host_data` holds the bytes the groups'
    key_off values index, as for Query.batch_outputs."""
    out = [b""] * len(items)
    by_q = {}
    for i, q in enumerate(queries):
        by_q.setdefault(id(q), (q, []))[1].append(i)
    for q, idx in by_q.values():
        sub = [items[i] for i in idx]
        q._b_items = None  # render from a contiguous copy of this query's items
        for i, o in zip(idx, q.batch_outputs(sub, all_, host_data)):
            out[i] = o
    return out


class BatchGraph:
    """One CUDA graph replaying a batch per query (warpjq_ext.h
    warpjq_batch_graph_*): batches[i] = (query, device base address,
    offsets, lengths).  Each Query must be used by one batch only; after
    launch(), collect each with query.batch_collect()."""

    def __init__(self, batches):
        k, _ = _load()
        self._k = k
        n = len(batches)
        self._queries = [b[0] for b in batches]
        self._keep = []
        ctxs = (ctypes.c_void_p * n)(*[q.ctx for q, _, _, _ in batches])
        datas = (ctypes.c_void_p * n)(*[d for _, d, _, _ in batches])
        offs = (ctypes.c_void_p * n)()
        lens = (ctypes.c_void_p * n)()
        counts = (ctypes.c_uint32 * n)()
        for i, (q, _, o, l) in enumerate(batches):
            oa = (ctypes.c_uint64 * max(1, len(o)))(*o)
            la = (ctypes.c_uint64 * max(1, len(l)))(*l)
            self._keep += [oa, la]
            offs[i] = ctypes.cast(oa, ctypes.c_void_p)
            lens[i] = ctypes.cast(la, ctypes.c_void_p)
            counts[i] = len(o)
            q._b_n = len(o)
        self._g = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        rc = k.warpjq_batch_graph_create(ctxs, n, datas, offs, lens, counts, ctypes.byref(self._g), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))

    def launch(self, stream: int = 0):
        err = ctypes.create_string_buffer(1024)
        rc = self._k.warpjq_batch_graph_launch(self._g, ctypes.c_void_p(stream), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))

    def close(self):
        if self._g:
            self._k.warpjq_batch_graph_destroy(self._g)
            self._g = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CsvConverter:
    """RFC 4180 CSV to NDJSON in device memory (warpjq_ext.h
    warpjq_csv_convert): the header row names the keys, each later row
    becomes one line."""

    def __init__(self):
        k, _ = _load()
        self._k = k
        self._c = ctypes.c_void_p()
        if k.warpjq_csv_create(ctypes.byref(self._c)):
            raise MemoryError("warpjq_csv_create")

    def reset(self):
        """The next chunk starts a new input (with a header row)."""
        self._k.warpjq_csv_reset(self._c)

    def convert(self, src: int, n: int, final: bool = True, host: bool = False, stream: int = 0):
        """Converts n bytes at address src (device memory, or host memory
        with host=True).  Returns (device address, NDJSON bytes, bytes
        consumed, data rows); the NDJSON stays valid until the next call."""
        d = ctypes.c_void_p()
        nd, used, recs = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_uint64()
        err = ctypes.create_string_buffer(1024)
        flags = (1 if final else 0) | (2 if host else 0)
        rc = self._k.warpjq_csv_convert(self._c, ctypes.c_void_p(src), n, flags, ctypes.c_void_p(stream),
                                        ctypes.byref(d), ctypes.byref(nd), ctypes.byref(used),
                                        ctypes.byref(recs), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))
        return (d.value or 0), nd.value, used.value, recs.value

    def gather(self, d_src: int, offsets, lengths, n: int, out, stream: int = 0):
        """Copies device slices d_src[offsets[i], + lengths[i]) back to back
        into `out` (a writable numpy uint8 array large enough)."""
        err = ctypes.create_string_buffer(1024)
        if hasattr(offsets, "ctypes"):  # numpy arrays
            offsets = offsets.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))
            lengths = lengths.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32))
        rc = self._k.warpjq_csv_gather(self._c, ctypes.c_void_p(d_src), offsets, lengths, n,
                                       ctypes.c_void_p(out.ctypes.data), ctypes.c_void_p(stream), err, len(err))
        if rc:
            raise RuntimeError(err.value.decode(errors="replace"))

    def close(self):
        if self._c:
            self._k.warpjq_csv_destroy(self._c)
            self._c = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def probe() -> str:
    """'' when a usable sm_100 device is present, else the reason."""
    k, _ = _load()
    err = ctypes.create_string_buffer(512)
    rc = k.warpjq_probe(err, len(err))
    return "" if rc == 0 else err.value.decode(errors="replace")


def device_name() -> str:
    k, _ = _load()
    buf = ctypes.create_string_buffer(256)
    k.warpjq_device_name(buf, len(buf))
    return buf.value.decode()


def gen_nested(n_bytes: int, seed: int = 1, n_users: int = 1_000_000, threads: int = 0, into=None):
    """About n_bytes of the nested, dirty schema (warpjq_host.h
    warpjq_gen_nested); returns (buffer, used_bytes, n_lines)."""
    import numpy as np
    _, h = _load()
    buf = into if into is not None else np.empty(n_bytes, dtype=np.uint8)
    lines = ctypes.c_uint64()
    used = h.warpjq_gen_nested(seed, buf.ctypes.data, n_bytes, 1 << 20, threads, n_users,
                               ctypes.byref(lines))
    return buf, int(used), int(lines.value)


def gen_nginx_csv(n_bytes: int, seed: int = 1, threads: int = 0, into=None):
    """About n_bytes of the nginx records as CSV (a header row, then one row
    per record, ua quoted); returns (buffer, used_bytes, n_rows)."""
    import numpy as np
    _, h = _load()
    buf = into if into is not None else np.empty(n_bytes, dtype=np.uint8)
    lines = ctypes.c_uint64()
    used = h.warpjq_gen_nginx_csv(seed, buf.ctypes.data, n_bytes, 1 << 20, threads, ctypes.byref(lines))
    return buf, int(used), int(lines.value)


def gen_nginx_csv_as_ndjson(n_bytes: int, seed: int = 1, threads: int = 0):
    """The NDJSON lines of exactly the records gen_nginx_csv(n_bytes, seed)
    writes as CSV rows; returns (buffer, used_bytes, n_lines)."""
    import numpy as np
    _, h = _load()
    buf = np.empty(2 * n_bytes + 16, dtype=np.uint8)
    lines = ctypes.c_uint64()
    used = h.warpjq_gen_nginx_csv_as_ndjson(seed, buf.ctypes.data, n_bytes, 1 << 20, threads,
                                            ctypes.byref(lines))
    return buf, int(used), int(lines.value)


def gen_nginx(n_bytes: int, seed: int = 1, threads: int = 0, into=None):
    """About n_bytes of the benchmark's nginx-style NDJSON (whole lines).

    Returns (buffer, used_bytes, n_lines).  `into` may be a writable numpy
    uint8 array of at least n_bytes (e.g. pinned host memory)."""
    import numpy as np
    _, h = _load()
    buf = into if into is not None else np.empty(n_bytes, dtype=np.uint8)
    lines = ctypes.c_uint64()
    used = h.warpjq_gen_nginx(seed, buf.ctypes.data, n_bytes, 1 << 20, threads, ctypes.byref(lines))
    return buf, int(used), int(lines.value)
