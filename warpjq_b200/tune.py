"""Autotuner: measures, instead of guessing, the scan's tunables for a query
on a sample of its input, and caches the choice.

Swept, each timed with CUDA events around the device-resident run (best of
`reps` after a warm-up):
  - lines per warp: how many lines a warp takes from the work queue at a
    time (walked 32 at a time, one per lane).  The unit of work is a tile of
    bytes, so a lines-per-warp candidate L is the tile L x the sample's mean
    line length (rounded to 256 bytes, within the tiling limits); the tile
    bytes follow from it, with the halo from warpjq_autotile's longest-line
    rule, and warpjq_autotile's own tile is a candidate too;
  - for group_by queries, the group table's starting capacity (a table
    sized for the input's cardinality avoids an overflow rerun; a small one
    is cleared and cached faster).

The cache is a JSON file keyed by device name, the device library's build,
query and the sample's mean line length (rounded to a power of two), so
inputs of the same shape reuse a choice without measuring again, and a
rebuilt library measures afresh.  warpjq_autotile's analytic choice is
always one of the candidates, so a tuned choice is never slower on the
sample than the default.
"""

from __future__ import annotations

import json
import math
import os

from . import Query, device_name

LINES_PER_WARP = (8, 16, 24, 32, 48, 64, 96, 128, 192, 256)
GROUP_KEYS = (1 << 12, 1 << 14, 1 << 16, 1 << 18, 1 << 20)


def default_cache_path() -> str:
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "warpjq_b200", "tune.json")


def library_id() -> str:
    """Identity of the built device library (size and modification time):
    a rebuilt kernel may want other tiles, so its choices are kept apart."""
    from . import KERNELS_SO
    try:
        st = os.stat(KERNELS_SO)
        return f"{st.st_size}-{int(st.st_mtime)}"
    except OSError:
        return "unbuilt"


def shape_key(device: str, query: str, sample: bytes, library: str = "") -> str:
    lines = sample.count(b"\n")
    mean = len(sample) / max(1, lines)
    return f"{device}|{library}|{query}|{2 ** round(math.log2(max(1.0, mean)))}"


def load_cache(path: str) -> dict:
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def save_cache(path: str, cache: dict):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _time(Q: Query, d_ptr: int, n: int, reps: int) -> float:
    import torch
    stream = torch.cuda.current_stream()
    Q.launch_device(d_ptr, n, stream.cuda_stream)
    Q.collect_device()
    best = None
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        Q.launch_device(d_ptr, n, stream.cuda_stream)
        e1.record(stream)
        Q.collect_device()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return best


def tune(query: str, d_ptr: int, n: int, sample: bytes, reps: int = 3, cache_path: str | None = None,
         use_cache: bool = True) -> dict:
    """Best tile (and group capacity) for `query` over n bytes at device
    address d_ptr (the sample to time on; `sample` is a host copy of its
    first bytes, for the halo rule and the cache key).  Returns
    {"tile": T, "halo": H, "group_keys": K or None, "gbs": rate, "from_cache": bool}."""
    cache_path = cache_path or default_cache_path()
    key = shape_key(device_name(), query, sample[: 1 << 20], library_id())
    cache = load_cache(cache_path) if use_cache else {}
    if use_cache and key in cache:
        return dict(cache[key], from_cache=True)
    Q = Query(query)
    t0, h = Q.autotile(sample[: 1 << 20])
    head = sample[: 1 << 20]
    mean = len(head) / max(1, head.count(b"\n"))
    per = {}
    for L in LINES_PER_WARP:
        t = max(1024, int(L * mean) // 256 * 256)
        if t + h <= 65535 - 64:
            per.setdefault(t, L)
    tiles = sorted(set(per) | {t0})
    timings = {}
    for t in tiles:
        Q.set_tiling(t, h)
        timings[t] = _time(Q, d_ptr, n, reps)
    best_t = min(timings, key=timings.get)
    Q.set_tiling(best_t, h)
    best_keys, best_ms = None, timings[best_t]
    if Q.is_grouped:
        for k in GROUP_KEYS:
            Q.set_group_capacity(k)
            ms = _time(Q, d_ptr, n, reps)
            if ms < best_ms:
                best_keys, best_ms = k, ms
    Q.close()
    res = {"lines_per_warp": round(best_t / mean, 1), "tile": best_t, "halo": h, "group_keys": best_keys,
           "gbs": round(n / (best_ms / 1e3) / 1e9, 2),
           "autotile": t0, "autotile_gbs": round(n / (timings[t0] / 1e3) / 1e9, 2),
           "swept": {str(t): round(n / (ms / 1e3) / 1e9, 2) for t, ms in timings.items()}}
    if use_cache:
        cache[key] = res
        save_cache(cache_path, cache)
    return dict(res, from_cache=False)


def apply(Q: Query, choice: dict):
    """Sets a tuned choice on a query's context."""
    Q.set_tiling(choice["tile"], choice["halo"])
    if choice.get("group_keys"):
        Q.set_group_capacity(choice["group_keys"])
