"""Serving: the continuous-batching Server (gzgpu_server_*).

Every request decoded in the mix equals the same request decoded alone
(byte-exact; integer work, no tolerance), whatever it is batched with and
whichever lane runs it; admission respects the device-memory budget."""
import threading
import zlib

import numpy as np
import pytest

from gzippy_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _requests(seed=5, n=48):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        if rng.random() < 0.8:
            size = int(np.exp(rng.uniform(np.log(4 << 10), np.log(256 << 10))))
        else:
            size = int(np.exp(rng.uniform(np.log(2 << 20), np.log(12 << 20))))
        p = W.content(int(rng.integers(0, 4)), 300 + i, size)
        reqs.append(W.gzip_member(p, int(rng.choice([1, 6, 9]))).tobytes())
    reqs.append(reqs[0] + reqs[1])                 # two members
    reqs.append(b"plain text, not gzip")
    bad = bytearray(reqs[2])
    bad[-8] ^= 1
    reqs.append(bytes(bad))                        # CRC mismatch
    reqs.append(reqs[3][:-30])                     # truncated
    return reqs


def _alone(G, data):
    cx = G.Context()
    try:
        return G.OK, cx.decompress(data)
    except G.GzippyError as e:
        return e.code, None
    finally:
        cx.close()


def test_each_result_same_alone_and_in_mix():
    import gzippy_b200 as G
    reqs = _requests()
    want = [_alone(G, r) for r in reqs]
    srv = G.Server(lanes=3, large_bytes=4 << 20)
    tickets = [None] * len(reqs)

    def submit(idx):
        for i in idx:
            tickets[i] = srv.submit(reqs[i])

    th = [threading.Thread(target=submit, args=(range(k, len(reqs), 2),)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for i, tk in enumerate(tickets):
        rc, data, tm = srv.poll(tk, -1)
        code, ref = want[i]
        if code == G.OK:
            assert rc in (G.OK, G.NOT_GZIP) and data == ref, i
        else:
            assert rc == code, (i, rc, code)
        assert tm.total_ms >= tm.queue_ms >= 0
    s = srv.stats()
    assert s.completed == len(reqs) and s.in_flight == 0 and s.queued == 0 and s.budget_used == 0
    assert s.batches < len(reqs)           # small requests shared batches
    srv.close()


def test_budget_admission_and_over_budget():
    import gzippy_b200 as G
    reqs = [W.gzip_member(W.content(k % 4, 400 + k, 3 << 20), 6).tobytes() for k in range(8)]
    # each request is charged ~ in + 3 x out_cap + 1 MiB (~ 12 MiB): two fit at once
    srv = G.Server(lanes=3, budget_bytes=26 << 20)
    tks = [srv.submit(r, out_cap=3 << 20) for r in reqs]
    peak = 0
    while True:
        s = srv.stats()
        peak = max(peak, s.budget_used)
        if s.completed == len(reqs):
            break
    assert peak <= 26 << 20
    for r, tk in zip(reqs, tks):
        assert srv.result(tk) == zlib.decompress(r, 31)
    with pytest.raises(G.GzippyError) as ei:
        srv.submit(reqs[0], out_cap=64 << 20)
    assert ei.value.code == G.OVER_BUDGET
    srv.close()


def test_poll_pending_then_done():
    import gzippy_b200 as G
    p = W.content(W.MARKOV, 9, 24 << 20)
    c = W.gzip_member(p, 6)
    srv = G.Server(lanes=1)
    tk = srv.submit(c)
    rc, data, _ = srv.poll(tk, 0)
    if rc == G.PENDING:
        rc, data, _ = srv.poll(tk, -1)
    assert rc == G.OK and data == p.tobytes()
    with pytest.raises(Exception):
        srv.result(tk)                     # a collected ticket is released
    srv.close()


def test_small_requests_pass_large_ones():
    """With one lane reserved for small requests, small requests submitted
    behind a queue of large ones finish before the last large one (which
    waits for the large ones ahead of it on the general lane)."""
    import gzippy_b200 as G
    large = [W.gzip_member(W.content(W.MARKOV, 500 + k, 48 << 20), 1).tobytes() for k in range(3)]
    small = [W.gzip_member(W.content(k % 4, 600 + k, 64 << 10), 6).tobytes() for k in range(16)]
    srv = G.Server(lanes=2, small_lanes=1, large_bytes=4 << 20)
    assert all(len(c) >= 4 << 20 for c in large)
    wait = 120_000                         # ms; a request left queued fails, not hangs
    for c in small[:2] + large[:1]:        # first use of both lanes' buffers
        rc, _, _ = srv.poll(srv.submit(c), wait)
        assert rc == G.OK
    tl = [srv.submit(c) for c in large]
    ts = [srv.submit(c) for c in small]
    small_ms = []
    for c, tk in zip(small, ts):
        rc, data, tm = srv.poll(tk, wait)
        assert rc == G.OK and data == zlib.decompress(c, 31)
        small_ms.append(tm.total_ms)
    large_ms = []
    for c, tk in zip(large, tl):
        rc, data, tm = srv.poll(tk, wait)
        assert rc == G.OK and data == zlib.decompress(c, 31)
        large_ms.append(tm.total_ms)
    assert max(small_ms) < large_ms[-1], (small_ms, large_ms)
    s = srv.stats()
    assert s.in_flight == 0 and s.queued == 0 and s.budget_used == 0
    srv.close()
