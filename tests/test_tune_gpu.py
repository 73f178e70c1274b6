"""The autotuner on the device: it measures the lines-per-warp sweep (tiles
of that many mean lines; and, for group_by, the table capacity), never
picks something slower than the
analytic choice on its sample, reuses its cache, and a context set from the
choice still prints the oracle's bytes."""

import pytest
import torch

import warpjq_b200 as wjq
from oracle import pyoracle as orc
from warpjq_b200 import tune

pytestmark = pytest.mark.gpu


def test_tune_sweeps_caches_and_keeps_results_exact(tmp_path):
    buf, n, _ = wjq.gen_nginx(64 << 20, seed=4)
    dev = torch.empty(n + 16, dtype=torch.uint8, device="cuda")
    dev[:n].copy_(torch.from_numpy(buf[:n].copy()))
    sample = bytes(buf[: 1 << 20])
    path = str(tmp_path / "tune.json")
    for q in ["select(.status == 500) | count", "group_by(.path) | count"]:
        c = tune.tune(q, dev.data_ptr(), n, sample, reps=2, cache_path=path)
        assert not c["from_cache"]
        assert c["gbs"] >= c["autotile_gbs"]
        assert len(c["swept"]) >= 5
        assert c["lines_per_warp"] > 0 and abs(c["lines_per_warp"] * 210.5 - c["tile"]) < 0.25 * c["tile"]
        again = tune.tune(q, dev.data_ptr(), n, sample, cache_path=path)
        assert again["from_cache"] and again["tile"] == c["tile"]
        Q = wjq.Query(q)
        tune.apply(Q, c)
        small = bytes(buf[:4 << 20])
        small = small[: small.rfind(b"\n") + 1]
        d = torch.empty(len(small) + 16, dtype=torch.uint8, device="cuda")
        d[:len(small)].copy_(torch.frombuffer(bytearray(small), dtype=torch.uint8))
        Q.launch_device(d.data_ptr(), len(small), torch.cuda.current_stream().cuda_stream)
        r = Q.collect_device()
        got = Q.render_device(r, small)
        if r.d_out_bytes:  # row queries (aggregates select lines but keep no rows)
            from warpjq_b200.shard import _DeviceBytes
            got += torch.as_tensor(_DeviceBytes(r.d_out_bytes, r.out_len), device="cuda").cpu().numpy().tobytes()
        assert got == orc.run(q, small).out
        Q.close()
