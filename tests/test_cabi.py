"""The C ABI library: it loads, exports every entry point include/gzgpu.h
declares, and fails loudly (no CPU fallback) when no CUDA device is there."""
import ctypes
import os
import re

import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "gzgpu.h")


def declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(gzgpu_[a-z_]+)\s*\(", src)) - {"gzgpu_write_fn"})


def test_header_declares_entry_points():
    names = declared()
    for n in ("gzgpu_create", "gzgpu_destroy", "gzgpu_strerror", "gzgpu_decompress",
              "gzgpu_decompress_to_writer", "gzgpu_decompress_device", "gzgpu_decompress_batch",
              "gzgpu_get_stats"):
        assert n in names


def test_library_exports_every_declared_symbol():
    from gzippy_b200 import build
    lib = ctypes.CDLL(build.build())
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing


def test_strerror_host_only():
    import gzippy_b200 as G
    assert G.strerror(0) == "ok"
    assert "CRC32" in G.strerror(G.CRC_MISMATCH)
    assert G.strerror(999) == "unknown error"


@pytest.mark.skipif(gpu_available(), reason="checks the no-device behaviour")
def test_no_device_fails_loudly():
    import gzippy_b200 as G
    with pytest.raises(G.GzippyError):
        G.Context()


def test_not_gzip_is_empty_without_device_work():
    """Non-gzip input returns immediately (src/lib.rs:50-52): checked on the
    host before any device call, so this holds on CPU-only machines too."""
    import gzippy_b200 as G
    lib = G.lib()
    n = ctypes.c_size_t(7)
    buf = (ctypes.c_uint8 * 4)()
    rc = lib.gzgpu_decompress(ctypes.c_void_p(1), b"abc", 3, buf, 4, ctypes.byref(n))
    assert rc == G.NOT_GZIP and n.value == 0
