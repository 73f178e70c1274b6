"""Benchmark: GB/s scanned per query over 8 GB of device-resident nginx-style
NDJSON on B200, for the four queries of the headline workload.

One step = the four queries, each a full pass of the scan over the input:
    select(.status == 500) | count
    select(.status >= 500) | {p: .path, b: .bytes}
    group_by(.host) | sum(.bytes)
    select(.status == 500)                  (passthrough of whole lines)

value   -- input bytes scanned by all ranks / device time (CUDA events on the
           launch stream, max over ranks); inputs resident in HBM.
e2e     -- the same queries through the host C ABI (warpjq_query_run: pinned
           staging, 64 MiB chunks, H2D + kernels + D2H of results) from host
           memory, wall clock.
roofline -- the scan kernel: (input + output bytes) per launch / its
           CUDA-event duration, against the measured HBM copy bandwidth.
cpu_baseline -- the oracle (a C++ restatement of the reference CPU engine) on
           all host cores over a bounded sample of the same input.
batch   -- many small device-resident inputs, one of 8 queries each: one run
           per input with a host round trip each ("plain") against one
           batched run per query (warpjq_batch_launch), aggregate GB/s.
e2e_file -- the four queries through warpjq_query_run_file over a 2 GB file
           of the same input (page cache warm): parallel reads into
           page-locked buffers overlapped with H2D and the kernels.
nested  -- the nested, dirty schema (objects 3-5 deep, shuffled keys,
           escapes, mixed number forms, 2% malformed), device-resident, its
           two queries (one a group_by over ~1M Zipf user ids).
serve   -- open-loop Poisson arrivals of those inputs: a server that batches
           whatever has arrived, against one that serves requests one at a
           time; p50 / p99 / p999 latency and sustained GB/s.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

QUERIES = [
    "select(.status == 500) | count",
    "select(.status >= 500) | {p: .path, b: .bytes}",
    "group_by(.host) | sum(.bytes)",
    "select(.status == 500)",
]
METRIC = "GB/s scanned per query (8 GB, device-resident); batched vs plain GB/s; p99 ms"
BATCH_QUERIES = [
    "select(.status == 500) | count", "sum(.bytes)", "max(.latency_ms)", "avg(.latency_ms)",
    "group_by(.host) | sum(.bytes)", "group_by(.path) | count",
    "select(.status >= 500) | {p: .path, b: .bytes}", "select(.status == 500)",
]
WORKLOAD = ("nginx-style NDJSON (ts, host, method, path, status, bytes, latency_ms, ua), "
            "8 GB device-resident, 4 queries per step")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def scan_traffic_ratio():
    """DRAM bytes per input byte of the scan kernel, from the committed ncu
    summary (profiles/k_scan_nginx.txt), or None."""
    p = os.path.join(ROOT, "profiles", "k_scan_nginx.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            if line.startswith("dram_bytes_per_input_byte:"):
                return float(line.split(":", 1)[1])
    return None


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(data, queries, threads=0):
    """Seconds the oracle (all host threads) takes for `queries` over `data`
    (bytes or a uint8 numpy array), and each query's output bytes."""
    from oracle import pyoracle as orc
    t = time.perf_counter()
    outs = []
    for q in queries:
        r = orc.run(q, data, threads=threads)
        if r.rc != 0:
            raise RuntimeError(r.err)
        outs.append(r.out)
    return time.perf_counter() - t, outs


def same_output(got: bytes, want: bytes, rel: float = 1e-9) -> bool:
    """Byte-identical, or (aggregates of fractional values) equal line by
    line with numbers within `rel` relative: the device sums exactly and
    rounds once, the oracle adds in line order."""
    if got == want:
        return True
    a, b = got.split(b"\n"), want.split(b"\n")
    if len(a) != len(b):
        return False
    for x, y in zip(a, b):
        if x == y:
            continue
        try:
            jx, jy = json.loads(x), json.loads(y)
        except ValueError:
            return False
        if not _close(jx, jy, rel):
            return False
    return True


def _close(x, y, rel):
    if isinstance(x, dict) and isinstance(y, dict):
        return x.keys() == y.keys() and all(_close(x[k], y[k], rel) for k in x)
    if isinstance(x, list) and isinstance(y, list):
        return len(x) == len(y) and all(_close(p, q, rel) for p, q in zip(x, y))
    if isinstance(x, (int, float)) and isinstance(y, (int, float)) and not isinstance(x, bool):
        return x == y or abs(x - y) <= rel * max(abs(x), abs(y))
    return x == y


class _DevView:
    """n bytes of device memory at ptr, described for torch.as_tensor."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 2}


def _d2h(ptr: int, n: int) -> bytes:
    import torch
    return torch.as_tensor(_DevView(ptr, n), device="cuda").cpu().numpy().tobytes()


def device_output(Q, r, host_data) -> bytes:
    """A device-resident run's output bytes: aggregates rendered by the host
    library (group keys read from the host copy of the input), rows copied
    from device memory."""
    if Q.is_aggregate:
        return Q.render_device(r, host_data)
    return _d2h(r.d_out_bytes, r.out_len) if r.out_len else b""


def batch_workload(dsrc, hnp, n, n_inputs=4096, lo=4096, hi=64 << 20, seed=7):
    """Device-resident batch inputs (the batching configuration): 4096
    newline-aligned slices of the bench input with log-uniform sizes of
    4 KB - 64 MB, packed on the device at 16-byte aligned offsets, and a
    query index per input drawn uniformly from BATCH_QUERIES.  `dsrc` is the
    bench input on the device, `hnp` its host copy (for the cut points)."""
    import math
    import random
    import torch
    rng = random.Random(seed)
    spans, pos = [], 0
    for _ in range(n_inputs):
        sz = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        if pos + sz + 4096 >= n:
            pos = 0
        end = pos + sz
        k = bytes(hnp[end - 1:min(n, end + 4096)]).find(b"\n")
        end = end + k if k >= 0 else end
        spans.append((pos, end))
        pos = end
    qidx = [rng.randrange(len(BATCH_QUERIES)) for _ in range(n_inputs)]
    offs, total = [], 0
    for a, b in spans:
        total = (total + 15) & ~15
        offs.append(total)
        total += b - a
    dev = torch.empty(total + 16, dtype=torch.uint8, device="cuda")
    for (a, b), o in zip(spans, offs):
        dev[o:o + (b - a)].copy_(dsrc[a:b])
    torch.cuda.synchronize()
    return dev, offs, [b - a for a, b in spans], qidx


def measure_batch(wjq, dev, offs, lens, qidx):
    """Aggregate GB/s over all inputs: plain (one run and host round trip
    per input), batched (one batched run per query, collected at the end)
    and graph (the same batches replayed from one CUDA graph); wall clock,
    results on the host in all three."""
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    ptr = dev.data_ptr()
    from warpjq_b200 import tune
    plain_q = [wjq.Query(q, chunk_bytes=1 << 20) for q in BATCH_QUERIES]
    batch_q = [wjq.Query(q, chunk_bytes=1 << 20) for q in BATCH_QUERIES]
    groups = [[i for i in range(len(offs)) if qidx[i] == k] for k in range(len(BATCH_QUERIES))]
    total = sum(lens)
    # tile (and group capacity) per query, measured on the first 256 MB of
    # the packed inputs, applied to every arm alike
    m = min(total, 256 << 20)
    sample = dev[:1 << 20].cpu().numpy().tobytes()
    tuned = {q: tune.tune(q, ptr, m, sample, reps=2, use_cache=False) for q in BATCH_QUERIES}
    for arm in (plain_q, batch_q):
        for k, q in enumerate(BATCH_QUERIES):
            tune.apply(arm[k], tuned[q])

    def plain():
        for i in range(len(offs)):
            q = plain_q[qidx[i]]
            q.launch_device(ptr + offs[i], lens[i], stream)
            q.collect_device()

    def batched():
        for k, g in enumerate(groups):
            batch_q[k].batch_launch(ptr, [offs[i] for i in g], [lens[i] for i in g], stream)
        return [batch_q[k].batch_collect() for k in range(len(groups))]

    graph_q = [wjq.Query(q, chunk_bytes=1 << 20) for q in BATCH_QUERIES]
    for k, q in enumerate(BATCH_QUERIES):
        tune.apply(graph_q[k], tuned[q])
    graph = wjq.BatchGraph([(graph_q[k], ptr, [offs[i] for i in g], [lens[i] for i in g])
                            for k, g in enumerate(groups)])

    def replay():
        graph.launch(stream)
        return [graph_q[k].batch_collect() for k in range(len(groups))]

    # mixed: every input in one launch sequence, each with its own plan
    # (aggregate and row queries alike)
    driver = wjq.Query(BATCH_QUERIES[0], chunk_bytes=1 << 20)
    tune.apply(driver, tuned[BATCH_QUERIES[0]])
    every = list(range(len(offs)))

    def mixed():
        driver.batch_launch_mixed([batch_q[qidx[i]] for i in every], ptr, offs, lens, stream)
        return driver.batch_collect()

    out, got = {}, {}
    for name, fn in (("plain", plain), ("batched", batched), ("graph", replay), ("mixed", mixed)):
        fn()  # warm: buffers reach their sizes
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        got[name] = fn()
        torch.cuda.synchronize()
        out[name] = time.perf_counter() - t0
    graph.close()

    # every input's counts, exact sums and group count, arm against arm
    def key(it):
        return (it.n_lines, it.n_blank, it.n_invalid, it.n_selected, it.count, it.isum_lo, it.isum_hi,
                it.n_groups, it.fsum)

    def per_query_arm(res):
        per = {}
        for k, g in enumerate(groups):
            items = res[k][0]
            for j, i in enumerate(g):
                per[i] = key(items[j])
        return [per[i] for i in every]

    mixed_keys = [key(it) for it in got["mixed"][0]]
    arms_agree = per_query_arm(got["batched"]) == per_query_arm(got["graph"]) == mixed_keys
    return {"inputs": len(offs), "bytes": total,
            "sizes": "log-uniform 4 KB - 64 MB (the configuration's sizes; 4096 of them total "
                     "about 28 GB, not the configuration's approximate 8 GB)",
            "queries": len(BATCH_QUERIES), "residency": "device",
            "plain_gbs": round(total / out["plain"] / 1e9, 3),
            "batched_gbs": round(total / out["batched"] / 1e9, 3),
            "graph_gbs": round(total / out["graph"] / 1e9, 3),
            "plain_s": round(out["plain"], 4), "batched_s": round(out["batched"], 4),
            "graph_s": round(out["graph"], 4),
            "mixed_gbs": round(total / out["mixed"] / 1e9, 3),
            "arms_agree": arms_agree,
            "mixed": "all 4096 inputs in one launch sequence, each with its own plan (8 queries: "
                     "aggregates, projection and passthrough)",
            "graph": "one CUDA graph: the 8 queries' batches captured on forked streams, one launch",
            "speedup": round(out["plain"] / out["batched"], 2),
            "graph_speedup": round(out["plain"] / out["graph"], 2),
            "tuned": {q: {"lines_per_warp": c["lines_per_warp"], "tile": c["tile"], "halo": c["halo"],
                          "group_keys": c["group_keys"],
                          "gbs": c["gbs"], "autotile": c["autotile"], "autotile_gbs": c["autotile_gbs"]}
                      for q, c in tuned.items()}}


SERVE_QUERIES = BATCH_QUERIES + [
    "count", "min(.bytes)", "group_by(.method) | avg(.latency_ms)", "group_by(.status) | count",
    'select(.method == "POST") | {t: .ts, l: .latency_ms}', "select(.bytes > 5000000) | count",
    "select(.latency_ms > 100) | .path", "max(.bytes)",
]


def serve_pool(wjq, dsrc, hnp, n, n_req, seed=11, lo=1 << 10, hi=256 << 20, csv_share=0.2, host_share=0.3):
    """The serving configuration's requests: sizes log-uniform 1 KB - 256 MB,
    one of SERVE_QUERIES each, 20% CSV (32 distinct CSV inputs of such sizes,
    a header row and a run of the nginx records' rows, reused), the NDJSON
    ones newline-aligned slices of the bench input starting on a 16-byte
    aligned line start, 30% of them read from page-locked host memory and
    the rest from device memory in place.  Returns (requests, keep) with
    requests as (query, data, fmt, nbytes)."""
    import math
    import random
    import numpy as np
    import torch
    rng = random.Random(seed)
    size = lambda: int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
    buf, used, _ = wjq.gen_nginx_csv(1 << 30, seed=seed)
    raw = np.asarray(buf[:used])
    head_end = int(bytes(raw[:4096]).index(b"\n")) + 1
    csv_pool = []
    for k in range(32):
        sz = min(size(), used - head_end - 8192)
        a = rng.randrange(head_end, used - sz - 4096)
        a += bytes(raw[a:a + 8192]).index(b"\n") + 1
        e = a + sz
        e += bytes(raw[e:e + 8192]).index(b"\n") + 1
        h = torch.empty(head_end + e - a, dtype=torch.uint8).pin_memory()
        hn = h.numpy()
        hn[:head_end] = raw[:head_end]
        hn[head_end:] = raw[a:e]
        csv_pool.append(h if k % 3 == 0 else h.cuda())
    reqs = []
    for _ in range(n_req):
        q = SERVE_QUERIES[rng.randrange(len(SERVE_QUERIES))]
        if rng.random() < csv_share:
            t = csv_pool[rng.randrange(len(csv_pool))]
            reqs.append((q, t, "csv", int(t.numel())))
            continue
        sz = size()
        a = rng.randrange(0, n - sz - (1 << 20))
        while True:  # a line start on a 16-byte boundary
            j = bytes(hnp[a:a + 8192]).find(b"\n")
            a += j + 1
            if a % 16 == 0:
                break
        e = a + sz
        e += bytes(hnp[e - 1:e + 8192]).find(b"\n")
        src = hnp[a:e] if rng.random() < host_share else dsrc[a:e]
        reqs.append((q, src, "ndjson", e - a))
    return reqs, csv_pool


def measure_serving(wjq, reqs, rate, n_slots=8, max_batch=0, seed=5, mixed_min=0):
    """Open-loop Poisson arrivals at `rate` req/s through the native serving
    loop (include/warpjq_serve.h): continuous batching over `n_slots` slots
    with a 120 GB device-memory budget (with n_slots=1, max_batch=1: one
    request at a time).  Latency = completion - arrival, wall clock; every
    output rendered on the host."""
    import random
    import torch
    from warpjq_b200.serve import NativeServer
    rng = random.Random(seed)
    n_req = len(reqs)
    gaps = [rng.expovariate(rate) for _ in range(n_req)]
    total = sum(r[3] for r in reqs)
    # one batch per query in a slot (mixed batches carry every path and run
    # slower than the specialised kernels here)
    srv = NativeServer(SERVE_QUERIES, n_slots=n_slots, budget_bytes=120 << 30, max_batch=max_batch,
                       mixed_min=mixed_min)
    srv.warm(1 << 30)
    for q, x, f, _ in reqs[:32]:  # warm: every path once
        srv.submit(q, x, f)
    srv.drain()
    torch.cuda.synchronize()
    t0 = time.perf_counter() + 0.01
    arrive, t = [], t0
    for g in gaps:
        t += g
        arrive.append(t)
    nxt, done = 0, []
    while nxt < n_req:
        now = time.perf_counter()
        while nxt < n_req and arrive[nxt] <= now:
            q, x, f, _ = reqs[nxt]
            srv.submit(q, x, f)
            nxt += 1
        done += srv.poll()
        if nxt < n_req:
            time.sleep(max(0.0, min(arrive[nxt] - time.perf_counter(), 0.0005)))
    done += srv.drain()
    span = time.perf_counter() - t0
    srv.close()
    bad = [r for r in done if r.rc]
    assert not bad, bad[0].error
    lat = sorted(r.latency_ms for r in done)
    pick = lambda f: round(lat[min(n_req - 1, int(f * n_req))], 3)
    return {"p50_ms": pick(0.50), "p99_ms": pick(0.99), "p999_ms": pick(0.999),
            "sustained_gbs": round(total / span / 1e9, 3), "span_s": round(span, 3)}


def measure_serving_baselines(reqs, k=8):
    """The comparators of the serving configuration on the first k requests,
    run back to back: the plain one-process-per-query GPU path (a fresh
    process per request: interpreter, library load, CUDA context and query
    set-up, then warpjq_run_bytes over the request's bytes from a file in
    /dev/shm), and the CPU backend (the oracle, all host threads)."""
    import tempfile
    import numpy as np
    from oracle import pyoracle as orc
    from oracle import csv_map
    sample = reqs[:k]
    total = sum(r[3] for r in sample)
    datas = []
    for q, x, f, _ in sample:
        b = bytes(x.cpu().numpy()) if hasattr(x, "is_cuda") else bytes(np.asarray(x))
        datas.append(b)
    lat_p = []
    t0 = time.perf_counter()
    for (q, _, f, _), b in zip(sample, datas):
        with tempfile.NamedTemporaryFile(dir="/dev/shm" if os.path.isdir("/dev/shm") else None,
                                         delete=False) as tf:
            tf.write(b)
            path = tf.name
        code = ("import sys; sys.path.insert(0, %r); import warpjq_b200 as w; "
                "d = open(%r, 'rb').read(); " % (ROOT, path) +
                ("r = w.Query(%r).run_csv(d)" % q if f == "csv" else "r = w.run_bytes(%r, d)" % q) +
                "; sys.exit(r.rc)")
        a = time.perf_counter()
        rc = subprocess.run([sys.executable, "-c", code]).returncode
        lat_p.append((time.perf_counter() - a) * 1e3)
        os.unlink(path)
        assert rc == 0
    span_p = time.perf_counter() - t0
    t0 = time.perf_counter()
    lat_c = []
    for (q, _, f, _), b in zip(sample, datas):
        a = time.perf_counter()
        r = orc.run(q, csv_map.csv_to_ndjson(b) if f == "csv" else b)
        lat_c.append((time.perf_counter() - a) * 1e3)
        assert r.rc == 0
    span_c = time.perf_counter() - t0
    return {"requests": k, "bytes": total,
            "process_per_query": {"gbs": round(total / span_p / 1e9, 3),
                                  "mean_ms": round(sum(lat_p) / k, 1)},
            "cpu_backend": {"gbs": round(total / span_c / 1e9, 3), "mean_ms": round(sum(lat_c) / k, 1),
                            "cores": os.cpu_count(),
                            "note": "CSV requests are mapped to NDJSON on the host first (timed)"}}


def measure_plain64(wjq, hnp, reps=5):
    """The plain single-input configuration: 64 MB of the nginx schema (the
    first newline-aligned 64 MB of the bench input), `select(.status ==
    500) | count`, run the way one CLI invocation runs it: one
    warpjq_query_run from host memory (pageable, as a file's bytes would
    be), context already open; best of `reps`.  Beside it the oracle (the
    reference CPU engine's restatement) on all host threads over the same
    bytes, and the output of both."""
    from oracle import pyoracle as orc
    q = "select(.status == 500) | count"
    m = bytes(hnp[: 64 << 20]).rfind(b"\n") + 1
    data = bytes(hnp[:m])
    Q = wjq.Query(q)
    Q.run(data)  # warm: slots and result buffers
    best = None
    for _ in range(reps):
        t = time.perf_counter()
        r = Q.run(data)
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    Q.close()
    t = time.perf_counter()
    want = orc.run(q, data)
    ct = time.perf_counter() - t
    return {"query": q, "bytes": m, "gbs": round(m / best / 1e9, 3), "ms": round(best * 1e3, 3),
            "cpu_gbs": round(m / ct / 1e9, 3), "cpu_cores": os.cpu_count(),
            "residency": "host memory (pageable), one warpjq_query_run",
            "parity": r.out == want.out, "output": r.out.decode(errors="replace").strip()}


NESTED_QUERIES = [
    'select(.req.user.tier == "gold" and .resp.code != 200) | {u: .req.user.id, l: .resp.latency}',
    "group_by(.req.user.id) | avg(.resp.latency)",
]


def measure_nested(wjq, n_bytes=4_000_000_000, reps=3, check=True):
    """Device-resident GB/s of the nested workload's two queries (best of
    `reps` after a warm-up run; CUDA events around all kernels of a run)."""
    import torch
    host = torch.empty(n_bytes, dtype=torch.uint8).pin_memory()
    _, n, lines = wjq.gen_nested(n_bytes, seed=5, n_users=1_000_000, into=host.numpy())
    dev = torch.empty(n + 16, dtype=torch.uint8, device="cuda")
    dev[:n].copy_(host[:n])
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    out = {"bytes": n, "lines": lines, "residency": "device",
           "sizes": f"{n_bytes / 1e9:g} GB, 1M Zipf(0.9) user ids",
           "per_query_gbs": {}}
    outs = []
    for q in NESTED_QUERIES:
        Q = wjq.Query(q, chunk_bytes=1 << 20)
        Q.autotile(host.numpy()[: 1 << 20])
        Q.launch_device(dev.data_ptr(), n, stream.cuda_stream)
        Q.collect_device()
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            Q.launch_device(dev.data_ptr(), n, stream.cuda_stream)
            e1.record(stream)
            r = Q.collect_device()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out["per_query_gbs"][q] = round(n / (best / 1e3) / 1e9, 2)
        outs.append(device_output(Q, r, host.numpy()))
        if Q.is_grouped:
            out["groups"] = r.n_groups
        Q.close()
    del dev
    if check:  # the oracle over the same bytes (skip-invalid, as the device runs)
        _, want = cpu_baseline(host.numpy()[:n], NESTED_QUERIES)
        out["parity"] = {q: same_output(g, w) for q, g, w in zip(NESTED_QUERIES, outs, want)}
    return out


CSV_QUERY = "group_by(.path) | max(.latency_ms)"


def measure_csv(wjq, n_bytes=2_000_000_000, reps=3, e2e=True, check=True):
    """The nginx records as 2 GB of CSV (RFC 4180 quoting on ua), query
    group_by(.path) | max(.latency_ms).  Device-resident GB/s of CSV bytes
    (conversion to NDJSON on the device plus the scan; CUDA events around
    both, best of `reps` after a warm-up), and end to end from pinned host
    memory through warpjq_query_run_csv (wall clock)."""
    import torch
    host = torch.empty(n_bytes, dtype=torch.uint8).pin_memory()
    _, n, rows = wjq.gen_nginx_csv(n_bytes, seed=6, into=host.numpy())
    dev = torch.empty(n + 16, dtype=torch.uint8, device="cuda")
    dev[:n].copy_(host[:n])
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    conv = wjq.CsvConverter()
    Q = wjq.Query(CSV_QUERY)
    best = None
    for _ in range(reps + 1):
        conv.reset()
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        d, nd, used, recs = conv.convert(dev.data_ptr(), n, stream=stream.cuda_stream)
        e1.record(stream)
        Q.launch_device(d, nd, stream.cuda_stream)
        e2.record(stream)
        r = Q.collect_device()
        t = (e0.elapsed_time(e2), e0.elapsed_time(e1), e1.elapsed_time(e2))
        if best is None or t[0] < best[0]:
            best = t
    assert recs == rows and r.n_groups == 32, (recs, rows, r.n_groups)
    parity = None
    if check:
        # the oracle over the NDJSON rendering of exactly these CSV records;
        # group keys of the device result index the converted NDJSON
        conv_np = torch.as_tensor(_DevView(d, nd), device="cuda").cpu().numpy()
        got = Q.render_device(r, conv_np)
        exp, eu, _ = wjq.gen_nginx_csv_as_ndjson(n_bytes, seed=6)
        _, want = cpu_baseline(exp[:eu], [CSV_QUERY])
        parity = {CSV_QUERY: same_output(got, want[0])}
        del conv_np, exp
    Q.close()
    conv.close()
    del dev
    el = None
    if e2e:
        Qh = wjq.Query(CSV_QUERY)
        Qh.run_csv(host.numpy()[:n])
        t0 = time.perf_counter()
        rr = Qh.run_csv(host.numpy()[:n])
        el = time.perf_counter() - t0
        if rr.rc:
            raise RuntimeError(rr.err)
        Qh.close()
    return {"query": CSV_QUERY, "csv_bytes": n, "rows": rows, "ndjson_bytes": nd,
            "residency": "device (value) / pinned host (e2e)",
            "value": round(n / (best[0] / 1e3) / 1e9, 2), "unit": "GB/s of CSV",
            "convert_gbs": round(n / (best[1] / 1e3) / 1e9, 2),
            "scan_gbs_of_ndjson": round(nd / (best[2] / 1e3) / 1e9, 2),
            "ms": [round(x, 3) for x in best],
            "e2e_gbs": round(n / el / 1e9, 3) if el else None,
            "parity": parity}


def measure_file(wjq, hnp, n, n_bytes=2_000_000_000):
    """GB/s of the bench queries over a file (written once, so the page
    cache holds it), wall clock per query, one run each after a warm run."""
    import tempfile
    d = "/dev/shm" if os.path.isdir("/dev/shm") else None
    cut = min(n, n_bytes)
    cut = bytes(hnp[max(0, cut - 4096):cut]).rfind(b"\n") + max(0, cut - 4096) + 1
    fd, path = tempfile.mkstemp(suffix=".ndjson", dir=d)
    try:
        with os.fdopen(fd, "wb") as f:
            f.write(memoryview(hnp[:cut]))
        per = {}
        for q in QUERIES:
            Q = wjq.Query(q)
            Q.run_file(path, copy_out=False)
            t0 = time.perf_counter()
            r = Q.run_file(path, copy_out=False)
            el = time.perf_counter() - t0
            if r.rc:
                raise RuntimeError(r.err)
            per[q] = round(cut / el / 1e9, 3)
            Q.close()
        total = cut * len(QUERIES) / sum(cut / v / 1e9 for v in per.values()) / 1e9
        return {"value": round(total, 3), "unit": "GB/s", "file_bytes": cut,
                "where": d or tempfile.gettempdir(), "per_query_gbs": per}
    finally:
        os.unlink(path)


def run_reference(args, rank):
    """The reference arm: the reference's CPU engine, as restated by the
    oracle (the Rust crate cannot be built here), on all host cores, over
    the same input as the product's arm: the seeded 8 GB of nginx NDJSON
    (generated by the oracle library's copy of the generator, so no product
    library is loaded).  Each timed step runs one of the four queries over
    the whole input, cycling through them; warm-up steps run them over the
    input's first 256 MB.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return
    from oracle import pyoracle as orc
    cores = os.cpu_count() or 1
    buf, n, lines = orc.gen_nginx(args.bytes, seed=1)
    data = buf[:n]
    warm_n = bytes(data[: 256 << 20]).rfind(b"\n") + 1
    for k in range(args.warmup):
        cpu_baseline(data[:warm_n], [QUERIES[k % len(QUERIES)]])
    t = 0.0
    per_q = {}
    for k in range(args.steps):
        q = QUERIES[k % len(QUERIES)]
        dt, _ = cpu_baseline(data, [q])
        t += dt
        per_q.setdefault(q, []).append(dt)
    value = n * args.steps / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "GB/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
        "config": {"workload": WORKLOAD, "input_bytes": n, "lines": lines, "queries": QUERIES,
                   "same_config": True,
                   "step": "one query over the whole input, cycling through the four",
                   "per_query_gbs": {q: round(n * len(v) / sum(v) / 1e9, 4) for q, v in per_q.items()}},
        "cpu_baseline": {"value": round(value, 4), "unit": "GB/s", "cores": cores, "kind": "port",
                         "sample": f"the whole {n}-byte input per step, one query per step"},
        "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--bytes", type=int, default=8_000_000_000, help="input bytes per GPU")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch and serving legs")
    ap.add_argument("--csv-only", type=int, default=0, metavar="BYTES",
                    help="only the device-resident CSV leg, on BYTES of CSV (for profiling)")
    ap.add_argument("--nested-only", type=int, default=0, metavar="BYTES",
                    help="only the nested-schema leg, on BYTES of input (for profiling)")
    ap.add_argument("--batch-only", type=int, default=0, metavar="BYTES",
                    help="only the batching leg, its 4096 inputs cut from BYTES of nginx input")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return

    import numpy as np
    import torch
    import warpjq_b200 as wjq
    if args.csv_only:
        print(json.dumps({"csv": measure_csv(wjq, args.csv_only, reps=args.steps, e2e=False)}), flush=True)
        return
    if args.nested_only:
        print(json.dumps({"nested": measure_nested(wjq, args.nested_only, reps=args.steps)}), flush=True)
        return
    if args.batch_only:
        host = torch.empty(args.batch_only, dtype=torch.uint8).pin_memory()
        hnp = host.numpy()
        _, n, _ = wjq.gen_nginx(args.batch_only, seed=1, into=hnp)
        dsrc = torch.empty(n + 16, dtype=torch.uint8, device="cuda")
        dsrc[:n].copy_(host[:n])
        bdev, boffs, blens, bq = batch_workload(dsrc, hnp, n)
        del dsrc
        print(json.dumps({"batch": measure_batch(wjq, bdev, boffs, blens, bq)}), flush=True)
        return

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    why = wjq.probe()
    if why:
        raise SystemExit(f"no usable device: {why}")

    # Input: generated once on the host, uploaded once.
    n_target = args.bytes
    host = torch.empty(n_target, dtype=torch.uint8).pin_memory()
    hnp = host.numpy()
    _, n, lines = wjq.gen_nginx(n_target, seed=1 + rank, into=hnp)
    dev = torch.empty(n + 16, dtype=torch.uint8, device="cuda")
    dev[:n].copy_(host[:n], non_blocking=False)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    qs = [wjq.Query(q) for q in QUERIES]
    tiling = [q.autotile(hnp[: 1 << 20]) for q in qs]
    ptr = dev.data_ptr()

    def step(events=None):
        for i, q in enumerate(qs):
            if events is not None:
                events[i][0].record(stream)
            q.launch_device(ptr, n, sptr)
            if events is not None:
                events[i][1].record(stream)

    # Warm-up: grows every device buffer to its final size.
    for _ in range(args.warmup):
        step()
        results = [q.collect_device() for q in qs]
    kernels_per_step = sum(r.kernels_launched for r in results)
    first = [(r.n_selected, r.count, r.out_len, r.isum(), r.n_groups) for r in results]
    # Consistency: passthrough and count select the same lines; the host
    # groups' exact sums add up to an integer.
    assert results[0].count == results[3].n_selected, "count vs passthrough mismatch"

    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    evs = [[[torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)]
            for _ in qs] for _ in range(args.steps)]
    scan_ms = [0.0] * len(qs)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for k in range(args.steps):
        step(evs[k])
    t1.record(stream)
    torch.cuda.synchronize()
    total_ms = t0.elapsed_time(t1)
    if dist:
        dist.barrier()
    clk = clocks.stop()
    per_q_ms = [sum(evs[k][i][0].elapsed_time(evs[k][i][1]) for k in range(args.steps)) / args.steps
                for i in range(len(qs))]
    results = [q.collect_device() for q in qs]
    for i, r in enumerate(results):
        scan_ms[i] = r.scan_ms
        assert (r.n_selected, r.count, r.out_len, r.isum(), r.n_groups) == first[i], "results changed"
    # the last timed run's outputs, for the parity check against the oracle
    device_outs = [device_output(Q, r, hnp) for Q, r in zip(qs, results)] if rank == 0 else []

    t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    max_ms = float(t.item())
    scanned = n * len(qs) * args.steps * world
    value = scanned / (max_ms / 1e3) / 1e9

    # Roofline of the scan kernel: algorithmic bytes = input + output.
    hbm, which = peaks()
    alg_bytes = sum(n + r.out_len for r in results)
    scan_total_ms = sum(scan_ms)
    achieved = alg_bytes / (scan_total_ms / 1e3) / 1e9 if scan_total_ms > 0 else None
    ratio = scan_traffic_ratio()
    traffic = int(ratio * n) if ratio else None

    # End to end through the host C ABI from host memory.
    e2e_val, h2d, d2h = None, 0, 0
    if args.e2e_steps > 0:
        data_np = hnp[:n]
        host_qs = [wjq.Query(q) for q in QUERIES]
        for q in host_qs:  # warm: allocates slots and result buffers
            q.run(data_np[: 64 << 20])
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        te = time.perf_counter()
        outs = 0
        for _ in range(args.e2e_steps):
            for q in host_qs:
                r = q.run(data_np, copy_out=False)
                if r.rc != 0:
                    raise RuntimeError(r.err)
                outs += len(r.out)
        torch.cuda.synchronize()
        el = time.perf_counter() - te
        tt = torch.tensor([el], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_val = n * len(QUERIES) * args.e2e_steps * world / float(tt.item()) / 1e9
        h2d = n * len(QUERIES)
        d2h = outs // args.e2e_steps

    # The host link itself: plain pinned-to-device copies of 1 GiB (CUDA
    # events), the ceiling of any end-to-end figure from host memory.
    link_gbs = None
    if args.e2e_steps > 0:
        m = min(n, 1 << 30)
        dst = torch.empty(m, dtype=torch.uint8, device="cuda")
        dst.copy_(host[:m], non_blocking=True)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            dst.copy_(host[:m], non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        link_gbs = round(3 * m / (e0.elapsed_time(e1) / 1e3) / 1e9, 2)
        del dst

    batch = serve = nested = e2e_file = csv_leg = plain64 = None
    if rank == 0 and world == 1 and not args.no_batch:
        bdev, boffs, blens, bq = batch_workload(dev, hnp, n)
        batch = measure_batch(wjq, bdev, boffs, blens, bq)
        del bdev
        torch.cuda.empty_cache()
        # the serving configuration: 1 KB - 256 MB requests, 20% CSV, some
        # from host memory, at three arrival rates; the one-at-a-time server
        # and the per-process / CPU comparators beside it
        sreqs, keep = serve_pool(wjq, dev, hnp, n, 4000)
        serve = {"queries": len(SERVE_QUERIES), "csv_share": 0.2, "host_share_of_ndjson": 0.3,
                 "sizes": "log-uniform 1 KB - 256 MB", "budget_bytes": 120 << 30, "rates": []}
        for rate, k in ((50.0, 100), (500.0, 1000), (2000.0, 4000)):
            sub = sreqs[:k]
            span = k / rate
            entry = {"offered_req_per_s": rate, "requests": k,
                     "offered_gbs": round(sum(r[3] for r in sub) / span / 1e9, 3),
                     "batched": measure_serving(wjq, sub, rate)}
            if rate <= 500.0:
                entry["one_at_a_time"] = measure_serving(wjq, sub, rate, n_slots=1, max_batch=1)
            serve["rates"].append(entry)
        serve["baselines"] = measure_serving_baselines(sreqs)
        del sreqs, keep
        torch.cuda.empty_cache()
        plain64 = measure_plain64(wjq, hnp)
        nested = measure_nested(wjq)
        csv_leg = measure_csv(wjq)
        e2e_file = measure_file(wjq, hnp, n)

    # CPU baseline and parity: the oracle on all host cores over the whole
    # input, each query once after a warm-up pass over the first 256 MB; its
    # outputs are the expected bytes for the device runs' outputs.
    cpu = parity = None
    if rank == 0 and world == 1 and not args.no_cpu:
        warm_n = bytes(hnp[: min(256 << 20, n)]).rfind(b"\n") + 1
        cpu_baseline(hnp[:warm_n], QUERIES)
        ct, want = cpu_baseline(hnp[:n], QUERIES)
        cpu = {"value": round(n * len(QUERIES) / ct / 1e9, 4), "unit": "GB/s",
               "cores": os.cpu_count(), "kind": "port",
               "sample": f"the whole {n}-byte input, each of the 4 queries once, after a warm-up "
                         f"pass over its first {warm_n} bytes"}
        parity = {q: same_output(g, w) for q, g, w in zip(QUERIES, device_outs, want)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(max_ms / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator, BASELINE nginx schema)",
            "config": {
                "workload": WORKLOAD, "input_bytes_per_gpu": n, "lines_per_gpu": lines,
                "mean_line_bytes": round(n / lines, 1), "queries": QUERIES,
                "per_query_gbs": {q: round(n / (ms / 1e3) / 1e9, 2) for q, ms in zip(QUERIES, per_q_ms)},
                "per_query_ms": {q: round(ms, 3) for q, ms in zip(QUERIES, per_q_ms)},
                "l2": "inputs (8 GB) larger than L2 (126 MB); no flush needed",
                "tile_halo_bytes": list(tiling[0]),
                "parallelism": f"dp{world} (independent shards, no collective)",
            },
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None,
                         "peak": hbm, "unit": "GB/s",
                         "frac": round(achieved / hbm, 4) if achieved else None,
                         "traffic": traffic, "peak_source": which,
                         "kernel": "k_scan (one launch per query; algorithmic bytes = input + output)"},
            "e2e": {"value": round(e2e_val, 3) if e2e_val else None, "unit": "GB/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "host_link_h2d_gbs": link_gbs},
            "gpu_launches": kernels_per_step * args.steps,
            "clocks": clk,
            "parity": parity,
            "cpu_baseline": cpu,
            "e2e_file": e2e_file,
            "plain_64mb": plain64,
            "batch": batch,
            "nested": nested,
            "csv": csv_leg,
            "serve": serve,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
