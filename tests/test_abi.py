"""The drop-in boundary, checked without a GPU: the native libraries load,
export every symbol include/*.h declares, and agree on struct layouts with
the reference's Rust mirror (crates/warpjq-core/src/gpu/ffi.rs:222-242)."""

import ctypes
import os
import re
import subprocess

import pytest

import warpjq_b200 as wjq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(warpjq_[a-z_0-9]+)\s*\(", text)))


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_libraries_load():
    k, h = wjq.libraries()
    assert k and h


def test_every_declared_symbol_is_exported():
    kern = exported(wjq.KERNELS_SO)
    host = exported(wjq.HOST_SO)
    for hdr, lib in (("warpjq_kernels.h", kern), ("warpjq_ext.h", kern), ("warpjq_host.h", host),
                     ("warpjq_serve.h", host)):
        missing = [f for f in declared_functions(hdr) if f not in lib]
        assert not missing, (hdr, missing)
    assert set(wjq.ABI_SYMBOLS) <= kern and set(wjq.EXT_SYMBOLS) <= kern
    assert set(wjq.HOST_SYMBOLS) <= host


def test_abi_sizes_match_the_reference_layout():
    # step 20, path 8, cmp 32, cond_op 8, agg_partial 48, group 56 bytes.
    k, _ = wjq.libraries()
    good = (ctypes.c_uint64 * 6)(20, 8, 32, 8, 48, 56)
    assert k.warpjq_abi_check(good, 6) == 0
    bad = (ctypes.c_uint64 * 6)(20, 8, 32, 8, 48, 48)
    assert k.warpjq_abi_check(bad, 6) == 4  # WARPJQ_ERR_ABI
    assert k.warpjq_abi_check(good, 5) == 4


def test_static_library_for_the_rust_crate_exists():
    a = os.path.join(wjq.LIB_DIR, "libwarpjq_kernels.a")
    assert os.path.exists(a)
    out = subprocess.run(["nm", "--defined-only", a], capture_output=True, text=True, check=True).stdout
    for f in wjq.ABI_SYMBOLS:
        assert f in out, f


def test_no_device_is_reported_cleanly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert wjq.probe() != ""


def test_serving_open_fails_cleanly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from warpjq_b200.serve import NativeServer
    with pytest.raises(RuntimeError):
        NativeServer(["count"], n_slots=2)
