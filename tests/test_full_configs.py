"""The five decompression configurations at their full sizes, on one GPU.

Every output is compared byte for byte with the generator's plaintext
(integer work, no tolerance): by SHA-256 for the single member of 1 GiB,
the 2,048-member stream of 4 GiB and the 10,000-stream batch, and by CRC32
per request for the serving mix.  Inputs come from the same seeded
generators and on-disk cache as bench.py.
  config 1 -- one 1 GiB member (256 x 4 MiB segments of four content types,
              level 6, one serial zlib stream);
  config 2 -- 2,048 members of 2 MiB (levels 1/6/9) in one stream;
  config 3 -- 10,000 streams (log-normal sizes), batched in one job and one
              stream per call;
  config 4 -- a serving mix with both size classes (4-256 KiB and
              8-512 MiB), each request checked against its plaintext.
(config 0 is the CPU-only case; its decoders are timed by bench.py.)"""
import hashlib
import os
import sys
import threading
import zlib

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _device_decode(comp: np.ndarray, plain_bytes: int):
    import torch
    import gzippy_b200 as G
    cx = G.Context()
    try:
        d_in = torch.zeros(comp.size + 1024, dtype=torch.uint8, device="cuda")
        d_in[: comp.size] = torch.from_numpy(comp).cuda()
        d_out = torch.empty(plain_bytes + 4096, dtype=torch.uint8, device="cuda")
        n = cx.decompress_device(d_in.data_ptr(), comp.size, d_out.data_ptr(), d_out.numel())
        return n, hashlib.sha256(d_out[:n].cpu().numpy().tobytes()).hexdigest(), cx.stats()
    finally:
        cx.close()


def test_config1_single_member_1gib():
    import bench
    comp, meta = bench.load_workload("single_member_mixed", 1.0)
    assert meta["plain_bytes"] == 1 << 30 and meta["encoder"] == "zlib-serial"
    n, digest, st = _device_decode(comp, meta["plain_bytes"])
    assert n == meta["plain_bytes"] and digest == meta["sha256"]
    assert st.n_accepted > 1000        # decoded as many speculative chunks


def test_config2_multi_member_4gib():
    import bench
    comp, meta = bench.load_workload("multi_member", 1.0)
    assert meta["plain_bytes"] == 4 << 30 and len(meta["member_comp_bytes"]) == 2048
    n, digest, st = _device_decode(comp, meta["plain_bytes"])
    assert n == meta["plain_bytes"] and digest == meta["sha256"]
    assert st.n_members == 2048         # every member's CRC32 and ISIZE checked


def test_config3_batch_10000_batched_and_one_per_call():
    import torch
    import bench
    import gzippy_b200 as G
    packed, offs, lens, sizes, meta = bench.load_batch(1.0)
    assert len(offs) == 10000
    total = meta["plain_bytes"]
    d_in = torch.from_numpy(packed).cuda()
    cx = G.Context()
    try:
        d_out = torch.empty(total + 4096, dtype=torch.uint8, device="cuda")
        oo, ol, st = cx.decompress_batch_device(d_in.data_ptr(), offs, lens, d_out.data_ptr(),
                                                d_out.numel())
        assert (st == 0).all() and int(ol.sum()) == total
        assert np.array_equal(ol, sizes)
        host = d_out[:total].cpu().numpy()
        h = hashlib.sha256()
        for o, l in zip(oo, ol):
            h.update(host[int(o):int(o) + int(l)].tobytes())
        assert h.hexdigest() == meta["sha256"]
        # the plain path: one call per stream, each into its own slot
        slot = np.zeros(len(sizes), np.int64)
        at = 0
        for i, sz in enumerate(sizes):
            slot[i] = at
            at += (int(sz) + 15) & ~15
        d_out2 = torch.empty(at + 4096, dtype=torch.uint8, device="cuda")
        ib, ob = d_in.data_ptr(), d_out2.data_ptr()
        for i in range(len(offs)):
            n = cx.decompress_device(ib + int(offs[i]), int(lens[i]), ob + int(slot[i]),
                                     int(sizes[i]) + 16)
            assert n == int(sizes[i]), i
        host2 = d_out2.cpu().numpy()
        h = hashlib.sha256()
        for i, sz in enumerate(sizes):
            h.update(host2[int(slot[i]):int(slot[i]) + int(sz)].tobytes())
        assert h.hexdigest() == meta["sha256"]
    finally:
        cx.close()


def test_config4_serving_mix_with_both_size_classes():
    import gzippy_b200 as G
    from gzippy_b200 import workloads as W
    comps, sizes, crcs, specs = W.serving_pool(seed=1238, n=48)
    large = [s for s in sizes if s >= (8 << 20)]
    assert len(large) >= 1 and any(s < (256 << 10) for s in sizes)
    srv = G.Server(lanes=4)
    tickets = [None] * len(comps)

    def submit(idx):
        for i in idx:
            tickets[i] = srv.submit(comps[i])

    th = [threading.Thread(target=submit, args=(range(k, len(comps), 2),)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    try:
        for i, tk in enumerate(tickets):
            data = srv.result(tk)
            assert len(data) == sizes[i] and zlib.crc32(data) == crcs[i], (i, specs[i])
    finally:
        srv.close()
