"""Golden fixtures (tests/golden, made by make_golden.py): expected status,
length and SHA-256 of the output, for the oracle (CPU) and the CUDA path."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import pyoracle as O

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MANIFEST = json.load(open(os.path.join(HERE, "manifest.json")))
IDS = [m["name"] for m in MANIFEST]


def _blob(m):
    return open(os.path.join(HERE, m["file"]), "rb").read()


@pytest.mark.parametrize("m", MANIFEST, ids=IDS)
def test_oracle_golden(m):
    st, out = O.decompress(_blob(m), cap=8 << 20)
    assert st == m["status"]
    if st == O.OK:
        assert out.size == m["out_len"] and hashlib.sha256(out.tobytes()).hexdigest() == m["sha256"]


@pytest.mark.parametrize("m", MANIFEST, ids=IDS)
def test_oracle_chunked_golden(m):
    st, out, _ = O.decompress_chunked(_blob(m), chunk_bytes=8192, threads=2, cap=8 << 20)
    assert st == m["status"]
    if st == O.OK:
        assert hashlib.sha256(out.tobytes()).hexdigest() == m["sha256"]


@pytest.fixture(scope="module")
def ctx():
    import gzippy_b200 as G
    c = G.Context(chunk_bytes=8 << 10)
    yield c
    c.close()


@pytest.mark.gpu
@pytest.mark.parametrize("m", MANIFEST, ids=IDS)
def test_gpu_golden(ctx, m):
    import gzippy_b200 as G
    blob = _blob(m)
    if m["status"] in (O.OK, O.NOT_GZIP):
        out = ctx.decompress(blob)
        assert len(out) == m["out_len"] and hashlib.sha256(out).hexdigest() == m["sha256"]
    else:
        with pytest.raises(G.GzippyError) as ei:
            ctx.decompress(blob)
        assert ei.value.code == m["status"]
