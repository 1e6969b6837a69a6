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


def _c_layout(tmp_path, name):
    """(sizeof, [(field, offset)]) of the header's struct `name`, from the C
    compiler."""
    import subprocess
    src = open(HEADER).read()
    block = re.search(r"typedef struct \{([^{}]*?)\} " + name + ";", src, flags=re.S).group(1)
    block = re.sub(r"/\*.*?\*/", "", block, flags=re.S)
    fields = []
    for decl in block.split(";"):
        parts = [x.strip() for x in decl.split(",") if x.strip()]
        fields += [x.split()[-1].lstrip("*") for x in parts]
    prog = tmp_path / (name + ".c")
    lines = ['#include <stddef.h>', '#include <stdio.h>', f'#include "{HEADER}"', "int main(void) {",
             f'  printf("%zu\\n", sizeof({name}));']
    lines += [f'  printf("{f} %zu\\n", offsetof({name}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    prog.write_text("\n".join(lines) + "\n")
    exe = tmp_path / name
    subprocess.check_call(["gcc", "-std=c99", "-o", str(exe), str(prog)])
    out = subprocess.check_output([str(exe)], text=True).split("\n")
    return int(out[0]), [(ln.split()[0], int(ln.split()[1])) for ln in out[1:] if ln]


def test_config_layout_matches_bindings(tmp_path):
    """The Python binding's Config and the Rust shim's GzgpuConfig in
    INTEGRATION.md list gzgpu_config's fields in the header's order, and the
    Python layout has the C compiler's offsets and size."""
    import gzippy_b200 as G
    size, fields = _c_layout(tmp_path, "gzgpu_config")
    assert ctypes.sizeof(G.Config) == size
    assert [(n, getattr(G.Config, n).offset) for n, _ in G.Config._fields_] == fields
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    rust = re.search(r"pub struct GzgpuConfig \{(.*?)\}", doc, flags=re.S).group(1)
    assert re.findall(r"pub ([a-z_]+):", rust) == [n for n, _ in fields]


@pytest.mark.parametrize("c_name,py_name", [
    ("gzgpu_span", "Span"), ("gzgpu_out", "Out"), ("gzgpu_stats", "Stats"),
    ("gzgpu_server_config", "ServerConfig"), ("gzgpu_request_times", "RequestTimes"),
    ("gzgpu_server_stats", "ServerStats")])
def test_struct_layouts_match_bindings(tmp_path, c_name, py_name):
    """Every other struct of the C ABI has the Python binding's field order,
    offsets and size."""
    import gzippy_b200 as G
    cls = getattr(G, py_name)
    size, fields = _c_layout(tmp_path, c_name)
    assert ctypes.sizeof(cls) == size
    assert [(n, getattr(cls, n).offset) for n, _ in cls._fields_] == fields
