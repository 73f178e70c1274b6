"""Scans over several GPUs: one newline-aligned byte range per rank.

Lines are independent, so the input shards by byte range, cut after a
newline the way the reference cuts its chunks
(crates/warpjq-core/src/chunk.rs:234-278).  Each rank scans its range on its
own GPU with no collective on the data path; rank 0 then gathers the ranks'
partial results -- the exact aggregate state (counts, 128-bit integer sums,
the FP sum, min/max), the groups with their key bytes, or the rank's rows --
and merges them in rank order, as the reference's host merges chunk results
in input order (crates/warpjq-core/src/gpu/mod.rs:959-1221, agg.rs:73-84).
The merged state is rendered by the host library's own formatter
(warpjq_query_render_device), so output bytes are those of a one-GPU run.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

from . import DeviceResult, Query, _GroupExt

KIND_NULL, KIND_STR = 1, 4


def shard_bounds(data, world: int) -> List[Tuple[int, int]]:
    """[start, end) of each rank's range: the input cut into `world` parts
    of about equal size, each cut placed just after a newline (a part is
    empty when one line spans it)."""
    mv = memoryview(data).cast("B")
    n = len(mv)
    cuts = [0]
    for r in range(1, world):
        t = max(cuts[-1], n * r // world)
        cut = n
        pos = t
        while pos < n:
            window = bytes(mv[pos:min(n, pos + (1 << 20))])
            k = window.find(b"\n")
            if k >= 0:
                cut = pos + k + 1
                break
            pos += len(window)
        cuts.append(max(cut, cuts[-1]))
    cuts.append(n)
    return list(zip(cuts[:-1], cuts[1:]))


def csv_row_end(mv, pos: int, inside: bool) -> int:
    """Offset just past the first row end at or after `pos` (a '\n' with an
    even number of '"' before it in the input), given whether `pos` itself
    lies inside quotes; len(mv) when none follows."""
    n = len(mv)
    while pos < n:
        window = bytes(mv[pos:min(n, pos + (1 << 20))])
        k = 0
        while True:
            q = window.find(b'"', k)
            nl = window.find(b"\n", k)
            if nl < 0 and q < 0:
                break
            if nl >= 0 and (q < 0 or nl < q):
                if not inside:
                    return pos + nl + 1
                k = nl + 1
            else:
                inside = not inside
                k = q + 1
        pos += len(window)
    return n


def _count_quotes(mv, lo: int, hi: int) -> int:
    """'"' bytes in mv[lo, hi), counted a window at a time."""
    n = 0
    for a in range(lo, hi, 1 << 24):
        n += bytes(mv[a:min(hi, a + (1 << 24))]).count(b'"')
    return n


def csv_shard_bounds(data, world: int) -> Tuple[int, List[Tuple[int, int]]]:
    """CSV input cut for `world` ranks: (header end, [start, end) of each
    rank's rows).  Cuts fall just after row ends (newlines outside quotes,
    whose quote count from the input's start is even), so a quoted field's
    newlines never split; every rank runs its rows behind a copy of the
    header row [0, header end)."""
    mv = memoryview(data).cast("B")
    n = len(mv)
    h_end = csv_row_end(mv, 0, False)
    cuts = [h_end]
    for r in range(1, world):
        t = max(cuts[-1], h_end + (n - h_end) * r // world)
        # every cut lies outside quotes, so the parity at t is that of the
        # quotes between the previous cut and t
        inside = _count_quotes(mv, cuts[-1], t) % 2 == 1
        cuts.append(max(csv_row_end(mv, t, inside), cuts[-1]))
    cuts.append(n)
    return h_end, list(zip(cuts[:-1], cuts[1:]))


def decode_key(kind: int, raw: bytes) -> bytes:
    """Group-key identity: string keys compare by their decoded bytes (escapes
    resolved, a lone surrogate becomes U+FFFD; json.rs:594-654), every
    other kind by its raw bytes (agg.rs:106-212)."""
    if kind != KIND_STR or b"\\" not in raw:
        return raw
    out = bytearray()
    i, n = 0, len(raw)
    simple = {0x22: 0x22, 0x5C: 0x5C, 0x2F: 0x2F, 0x62: 0x08, 0x66: 0x0C, 0x6E: 0x0A, 0x72: 0x0D,
              0x74: 0x09}
    while i < n:
        c = raw[i]
        if c != 0x5C:
            out.append(c)
            i += 1
            continue
        e = raw[i + 1]
        i += 2
        if e != 0x75:
            out.append(simple[e])
            continue
        cp = int(raw[i:i + 4], 16)
        i += 4
        if 0xD800 <= cp < 0xDC00 and raw[i:i + 2] == b"\\u":
            lo = int(raw[i + 2:i + 6], 16)
            if 0xDC00 <= lo < 0xE000:
                cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00)
                i += 6
        if 0xD800 <= cp < 0xE000:
            cp = 0xFFFD
        out += chr(cp).encode("utf-8")
    return bytes(out)


@dataclass
class GroupPart:
    kind: int
    raw: bytes          # key bytes as in the input (string: the body)
    count: int = 0
    numeric: int = 0
    isum: int = 0       # exact sum of the integer-literal values
    n_int: int = 0
    fsum: float = 0.0   # sum of the other numbers, in order
    min: float = math.inf
    max: float = -math.inf


@dataclass
class Partial:
    """One rank's result, small and portable (torch.distributed objects)."""
    n_lines: int = 0
    n_blank: int = 0
    n_invalid: int = 0
    n_type_error: int = 0
    n_selected: int = 0
    count: int = 0
    numeric: int = 0
    isum: int = 0
    n_int: int = 0
    fsum: float = 0.0
    min: float = math.inf
    max: float = -math.inf
    saw_non_numeric: bool = False
    # lowest malformed / type-error line index within the rank's range (None:
    # none); after merge(), within the whole input
    first_invalid: Optional[int] = None
    first_type_error: Optional[int] = None
    groups: List[GroupPart] = field(default_factory=list)
    # the rank's rows: bytes, or a uint8 torch tensor (on the rank's device
    # for a device-resident run); gather() moves them without pickling
    rows: object = b""


class _DeviceBytes:
    """Device memory described for torch.as_tensor (no copy)."""

    def __init__(self, ptr: int, n: int):
        # torch accepts only writable descriptions; the view is only read
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 2}


def partial_from_device(r: DeviceResult, shard_host) -> Partial:
    """The rank's partial from a collected device-resident run; group key
    bytes are read from the rank's host copy of its shard."""
    none = (1 << 64) - 1
    p = Partial(n_lines=r.n_lines, n_blank=r.n_blank, n_invalid=r.n_invalid,
                n_type_error=r.n_type_error, n_selected=r.n_selected, count=r.count,
                numeric=r.numeric, isum=r.isum(), n_int=r.n_int, fsum=r.fsum, min=r.min, max=r.max,
                saw_non_numeric=bool(r.saw_non_numeric),
                first_invalid=None if r.first_invalid == none else int(r.first_invalid),
                first_type_error=None if r.first_type_error == none else int(r.first_type_error))
    mv = memoryview(shard_host).cast("B")
    for k in range(r.n_groups):
        g = r.groups[k]
        v = (g.isum_hi << 64) | g.isum_lo
        v = v - (1 << 128) if g.isum_hi >> 63 else v
        p.groups.append(GroupPart(kind=g.key_kind, raw=bytes(mv[g.key_off:g.key_off + g.key_len]),
                                  count=g.count, numeric=g.numeric, isum=v, n_int=g.n_int,
                                  fsum=g.fsum, min=g.min, max=g.max))
    if r.out_len and r.d_out_bytes:
        import torch
        # a device copy the rank owns (the run's buffer is reused by its next run)
        p.rows = torch.as_tensor(_DeviceBytes(r.d_out_bytes, r.out_len), device="cuda").clone()
    return p


def merge(parts: Sequence[Partial]) -> Partial:
    """Rank-order merge: counts and integer sums exactly, FP sums in rank
    order, groups by key identity (first rank's raw bytes kept)."""
    m = Partial()
    groups = {}
    rows = []
    for p in parts:
        # first bad lines: the first rank that has one, offset by the lines
        # of the ranks before it
        if m.first_invalid is None and p.first_invalid is not None:
            m.first_invalid = m.n_lines + p.first_invalid
        if m.first_type_error is None and p.first_type_error is not None:
            m.first_type_error = m.n_lines + p.first_type_error
        m.n_lines += p.n_lines
        m.n_blank += p.n_blank
        m.n_invalid += p.n_invalid
        m.n_type_error += p.n_type_error
        m.n_selected += p.n_selected
        m.count += p.count
        m.numeric += p.numeric
        m.isum += p.isum
        m.n_int += p.n_int
        m.fsum += p.fsum
        m.min = min(m.min, p.min)
        m.max = max(m.max, p.max)
        m.saw_non_numeric |= p.saw_non_numeric
        rows.append(p.rows)
        for g in p.groups:
            ident = (KIND_NULL if g.kind == 0 else g.kind, decode_key(g.kind, g.raw))
            acc = groups.get(ident)
            if acc is None:
                acc = groups[ident] = GroupPart(kind=g.kind, raw=g.raw)
            acc.count += g.count
            acc.numeric += g.numeric
            acc.isum += g.isum
            acc.n_int += g.n_int
            acc.fsum += g.fsum
            acc.min = min(acc.min, g.min)
            acc.max = max(acc.max, g.max)
    m.groups = list(groups.values())
    m.rows = b"".join(_host_bytes(r) for r in rows)
    return m


def _host_bytes(rows) -> bytes:
    if isinstance(rows, (bytes, bytearray)):
        return bytes(rows)
    return rows.cpu().numpy().tobytes()


def _sum(isum: int, n_int: int, fsum: float) -> float:
    # the device's rounding: the integer sum and the FP sum added exactly,
    # then rounded once
    from fractions import Fraction
    if not math.isfinite(fsum):
        return float(isum) + fsum
    return float(Fraction(isum) + Fraction(fsum))


def render(query: str, merged: Partial, fmt: str = "ndjson") -> bytes:
    """Output bytes of the merged result, through the host library's
    formatter (no device needed)."""
    q = Query(query, fmt, device=False)
    r = DeviceResult()
    r.n_lines, r.n_selected = merged.n_lines, merged.n_selected
    r.count, r.numeric, r.n_int = merged.count, merged.numeric, merged.n_int
    r.fsum, r.min, r.max = merged.fsum, merged.min, merged.max
    r.sum = _sum(merged.isum, merged.n_int, merged.fsum)
    r.saw_non_numeric = int(merged.saw_non_numeric)
    keys = bytearray()
    garr = (_GroupExt * max(1, len(merged.groups)))()
    for k, g in enumerate(merged.groups):
        e = garr[k]
        e.key_off, e.key_len, e.key_kind = len(keys), len(g.raw), g.kind
        keys += g.raw
        e.count, e.numeric, e.n_int = g.count, g.numeric, g.n_int
        e.isum_lo, e.isum_hi = g.isum & ((1 << 64) - 1), (g.isum >> 64) & ((1 << 64) - 1)
        e.fsum, e.min, e.max = g.fsum, g.min, g.max
        e.sum = _sum(g.isum, g.n_int, g.fsum)
    r.groups = ctypes.cast(garr, ctypes.POINTER(_GroupExt))
    r.n_groups = len(merged.groups)
    head = q.render_device(r, bytes(keys))
    q.close()
    return head + merged.rows


def gather(partial: Partial, rank: int, world: int, group=None) -> Optional[List[Partial]]:
    """Rank 0 receives every rank's partial, in rank order (others: None).

    The small part (counts, aggregate state, groups) travels as one object
    per rank.  Rows do not: the ranks' row byte counts are all-gathered, an
    exclusive scan of them gives each rank's offset in the output, and rank
    0 receives each rank's rows straight into its slice of one output tensor
    (on the ranks' devices with NCCL, in host memory with gloo).  Every rank
    takes the same collective steps in the same order."""
    if world == 1:
        return [partial]
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    rows = partial.rows
    if isinstance(rows, (bytes, bytearray)):
        rows = torch.frombuffer(bytearray(rows), dtype=torch.uint8) if rows else torch.empty(0, dtype=torch.uint8)
    rows = rows.to(dev)
    head = Partial(**{k: v for k, v in partial.__dict__.items() if k != "rows"})
    heads = [None] * world if rank == 0 else None
    dist.gather_object(head, heads, dst=0, group=group)
    sizes = torch.zeros(world, dtype=torch.int64, device=dev)
    mine = torch.tensor([rows.numel()], dtype=torch.int64, device=dev)
    dist.all_gather_into_tensor(sizes, mine, group=group)
    sz = [int(x) for x in sizes.cpu()]
    offs = [0]
    for x in sz:
        offs.append(offs[-1] + x)  # exclusive scan: rank r's rows start at offs[r]
    if rank == 0:
        out = torch.empty(offs[-1], dtype=torch.uint8, device=dev)
        out[: sz[0]].copy_(rows)
        for r in range(1, world):
            if sz[r]:
                dist.recv(out[offs[r]:offs[r + 1]], src=r, group=group)
        for r in range(world):
            heads[r].rows = out[offs[r]:offs[r + 1]]
        return heads
    if sz[rank]:
        dist.send(rows.contiguous(), dst=0, group=group)
    return None


def device_partial(query: str, shard_host, fmt: str = "ndjson") -> Partial:
    """One range's partial from a device-resident run on the current GPU."""
    import numpy as np
    import torch
    shard_np = np.frombuffer(memoryview(shard_host).cast("B"), dtype=np.uint8)
    q = Query(query, fmt)
    dev = torch.empty(max(1, len(shard_np)) + 16, dtype=torch.uint8, device="cuda")
    if len(shard_np):
        dev[:len(shard_np)].copy_(torch.from_numpy(shard_np.copy()))
        q.autotile(shard_np[: 1 << 20])
    q.launch_device(dev.data_ptr(), len(shard_np), torch.cuda.current_stream().cuda_stream)
    part = partial_from_device(q.collect_device(), shard_np)
    q.close()
    return part


def csv_device_partial(query: str, header: bytes, rows_host, fmt: str = "ndjson") -> Partial:
    """One CSV range's partial: the header and the range's rows converted to
    NDJSON on the current GPU, scanned there; group keys are gathered from
    the converted bytes on the device."""
    import numpy as np
    import torch
    from . import CsvConverter
    src = bytes(header) + bytes(memoryview(rows_host).cast("B"))
    dev = torch.zeros(len(src) + 16, dtype=torch.uint8, device="cuda")
    if src:
        dev[:len(src)].copy_(torch.frombuffer(bytearray(src), dtype=torch.uint8))
    conv = CsvConverter()
    stream = torch.cuda.current_stream().cuda_stream
    d, nd, _, _ = conv.convert(dev.data_ptr(), len(src), stream=stream)
    q = Query(query, fmt)
    q.launch_device(d, nd, stream)
    r = q.collect_device()
    keys = np.zeros(1, dtype=np.uint8)
    if r.n_groups:
        g = np.ctypeslib.as_array(r.groups, shape=(r.n_groups,))
        offs = np.ascontiguousarray(g["key_off"], dtype=np.uint64)
        lens = np.ascontiguousarray(g["key_len"], dtype=np.uint32)
        keys = np.zeros(int(lens.sum()) + 1, dtype=np.uint8)
        conv.gather(d, offs, lens, r.n_groups, keys, stream)
        at = np.zeros(r.n_groups, dtype=np.uint64)
        np.cumsum(lens[:-1], out=at[1:])
        g["key_off"] = at
    part = partial_from_device(r, keys)
    q.close()
    conv.close()
    return part


def run_sharded_csv(query: str, host_data, rank: int, world: int, fmt: str = "ndjson",
                    group=None) -> Optional[bytes]:
    """run_sharded for CSV input: every rank converts its rows, behind the
    header, on its own GPU."""
    h_end, bounds = csv_shard_bounds(host_data, world)
    mv = memoryview(host_data).cast("B")
    lo, hi = bounds[rank]
    part = csv_device_partial(query, bytes(mv[:h_end]), mv[lo:hi], fmt)
    parts = gather(part, rank, world, group)
    if rank != 0:
        return None
    return render(query, merge(parts), fmt)


def run_sharded_partial(query: str, host_data, rank: int, world: int, fmt: str = "ndjson",
                        group=None) -> Optional[Partial]:
    """run_sharded's merged result on rank 0 (None on the others): counts,
    the first malformed / type-error line of the whole input, aggregate
    state, groups and rows."""
    lo, hi = shard_bounds(host_data, world)[rank]
    part = device_partial(query, memoryview(host_data).cast("B")[lo:hi], fmt)
    parts = gather(part, rank, world, group)
    return merge(parts) if rank == 0 else None


def run_sharded(query: str, host_data, rank: int, world: int, fmt: str = "ndjson",
                group=None) -> Optional[bytes]:
    """Runs `query` over `host_data` on `world` GPUs (this process: `rank`,
    on the current CUDA device).  Returns the output bytes on rank 0."""
    m = run_sharded_partial(query, host_data, rank, world, fmt, group)
    return None if m is None else render(query, m, fmt)
