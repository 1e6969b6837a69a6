"""Decompressed-GB/s benchmark of the B200 gzip decode path.

Workload (default): the single-member 1 GiB mixed stream -- 256 seeded 4 MiB
segments cycling Markov text / uniform random / byte runs / uint16 ramps +
noise, zlib level 6, one gzip member (generated on this machine; see
gzippy_b200/workloads).  A step decodes the whole stream.

  value : device-resident input -> device output (gzgpu_decompress_device),
          GB/s of decompressed bytes; the K steps are bracketed by
          synchronize + CUDA events on both sides, max over ranks.
  e2e   : the reference-facing host call (gzgpu_decompress) with pinned host
          buffers: H2D of the compressed stream and D2H of the output inside.
  roofline : the inflate kernel, algorithmic bytes (compressed read +
          decompressed written) per launch over its CUDA-event duration,
          against the measured HBM copy bandwidth.

`--impl reference` times the oracle's chunked speculative decoder (the C
restatement of the reference's parallel single-member path) on all host
threads, on the same workload.  Multi-GPU (torchrun): every rank decodes its
own replica (weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "byte-exact decompressed GB/s on 1 B200, batched vs plain GPU path; p50/p99 ms"
CACHE = os.path.join(tempfile.gettempdir(), "gzippy_b200_bench")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def cpus() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def load_workload(name: str, scale: float):
    """(compressed uint8 array, plain size, plain sha256, meta) -- cached on disk."""
    from gzippy_b200 import workloads as W
    os.makedirs(CACHE, exist_ok=True)
    key = f"{name}_{scale:g}_v2"
    path = os.path.join(CACHE, key + ".gz")
    meta_path = os.path.join(CACHE, key + ".json")
    if os.path.exists(path) and os.path.exists(meta_path):
        meta = json.load(open(meta_path))
        return np.fromfile(path, dtype=np.uint8), meta
    t0 = time.time()
    # single members are one serial zlib stream; the "_pigz" variants are
    # the same content in pigz-style framing (a Z_SYNC_FLUSH seam per MiB)
    enc = "pigz" if name.endswith("_pigz") else "zlib-serial"
    base = name[:-5] if name.endswith("_pigz") else name
    if base == "single_member_mixed":
        segs = max(4, int(round(256 * scale)))
        wl = W.single_member_mixed(segments=segs, keep_plain=True, encoder=enc)
    elif base == "stored_member":
        # the same 1 GiB of mixed content at level 0: a member of stored
        # blocks only (the stored-dominated case of stored_split.rs)
        segs = max(4, int(round(256 * scale)))
        wl = W.single_member_mixed(segments=segs, keep_plain=True, level=0, encoder=enc)
    elif base == "single_member_text":
        wl = W.single_member_text(size=max(1 << 20, int((64 << 20) * scale)), keep_plain=True,
                                  encoder=enc)
    elif name == "multi_member":
        wl = W.multi_member(members=max(8, int(2048 * scale)), keep_plain=True)
    else:
        raise SystemExit(f"unknown workload {name}")
    comp = wl.compressed[0]
    plain = wl.plain[0]
    meta = {"name": name, "plain_bytes": int(plain.size), "comp_bytes": int(comp.size),
            "sha256": hashlib.sha256(plain.tobytes()).hexdigest(),
            "gen_s": round(time.time() - t0, 2), "encoder": wl.meta.get("encoder", "zlib-serial"),
            "meta": {k: v for k, v in wl.meta.items() if not isinstance(v, list)}}
    if "member_comp_bytes" in wl.meta:
        meta["member_comp_bytes"] = wl.meta["member_comp_bytes"]
    comp.tofile(path)
    json.dump(meta, open(meta_path, "w"))
    return comp, meta


def load_batch(scale: float):
    """The 10,000-stream batch (log-normal sizes, median 64 KiB, sigma 1.5,
    1 KiB-64 MiB; content type uniform over the four kinds; level uniform in
    {1, 6, 9}), packed at 16-byte aligned offsets with 1 KiB of zero pad.
    Returns (packed, offsets, lengths, plain sizes, meta); cached on disk."""
    from gzippy_b200 import workloads as W
    os.makedirs(CACHE, exist_ok=True)
    n = max(16, int(round(10000 * scale)))
    base = os.path.join(CACHE, f"stream_batch_{n}")
    if os.path.exists(base + ".json"):
        meta = json.load(open(base + ".json"))
        z = np.load(base + ".npz")
        return z["packed"], z["offs"], z["lens"], z["sizes"], meta
    t0 = time.time()
    wl = W.stream_batch(streams=n, keep_plain=True)
    lens = np.array([c.size for c in wl.compressed], np.uint64)
    offs = np.zeros(n, np.uint64)
    at = 0
    for i, c in enumerate(wl.compressed):
        offs[i] = at
        at += (c.size + 15) & ~15
    packed = np.zeros(at + 1024, np.uint8)
    for o, c in zip(offs, wl.compressed):
        packed[int(o):int(o) + c.size] = c
    h = hashlib.sha256()
    for p_ in wl.plain:
        h.update(p_.tobytes())
    sizes = np.array(wl.plain_sizes, np.uint64)
    lv = np.array(wl.meta["levels"])
    meta = {"name": "stream_batch", "streams": n, "plain_bytes": int(sizes.sum()),
            "comp_bytes": int(lens.sum()), "sha256": h.hexdigest(), "gen_s": round(time.time() - t0, 2),
            "max_stream_bytes": int(sizes.max()),
            "levels": {str(k): int((lv == k).sum()) for k in (1, 6, 9)}}
    np.savez(base + ".npz", packed=packed, offs=offs, lens=lens, sizes=sizes)
    json.dump(meta, open(base + ".json", "w"))
    return packed, offs, lens, sizes, meta


def cpu_batch_baseline(packed, offs, lens, sizes, budget_s: float = 10.0, threads: int | None = None):
    """The oracle's serial decoder, one stream per task, on all host threads,
    over the first streams of the batch that fit the time budget."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import pyoracle as O
    th = threads or cpus()

    def one(i):
        o, l = int(offs[i]), int(lens[i])
        st, out = O.decompress(packed[o:o + l], cap=int(sizes[i]) + 4096)
        assert st == O.OK and out.size == int(sizes[i])
        return out.size

    done, nbytes, t0 = 0, 0, time.perf_counter()
    with ThreadPoolExecutor(th) as ex:
        while done < len(offs) and time.perf_counter() - t0 < budget_s:
            k = min(len(offs), done + 4 * th)
            nbytes += sum(ex.map(one, range(done, k)))
            done = k
    dt = time.perf_counter() - t0
    return {"value": round(nbytes / dt / 1e9, 4), "unit": "GB/s", "cores": th, "kind": "port",
            "sample": f"first {done} of {len(offs)} streams ({nbytes >> 20} MiB out), oracle serial "
                      f"decoder, one stream per task"}


def bench_batch(args, rank: int, world: int, local: int):
    """Batched path: all streams in one job per step (device-resident input and
    output) against the plain path (one stream per call) on the same GPU."""
    packed, offs, lens, sizes, meta = load_batch(args.scale)
    if world > 1 and args.impl != "reference":
        return bench_sharded(args, rank, world, local, "stream_batch", packed, offs, lens, sizes,
                             meta)
    n = len(offs)
    config = {"workload": "stream_batch", "streams": n, "levels": meta["levels"],
              "seed": 1237, "plain_bytes": meta["plain_bytes"], "comp_bytes": meta["comp_bytes"],
              "max_stream_bytes": meta["max_stream_bytes"],
              "l2": "inputs and outputs larger than the 126 MB L2; no flush",
              "parallelism": f"replicas x{world}", "autotune": not args.no_autotune}
    if args.impl == "reference":
        if rank != 0:
            return
        cb = cpu_batch_baseline(packed, offs, lens, sizes, budget_s=max(5.0, 4.0 * args.steps))
        line = {"metric": METRIC, "value": cb["value"], "unit": "GB/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
                "data": "synthetic (seeded generator + zlib levels 1/6/9)", "config": config,
                "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "GB/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    import torch
    torch.cuda.set_device(local)
    import gzippy_b200 as G
    ctx = G.Context(device=local, autotune=not args.no_autotune, decoder=args.decoder)
    d_in = torch.from_numpy(packed).cuda()
    total = meta["plain_bytes"]
    d_out = torch.empty(total + 4096, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    def step():
        return ctx.decompress_batch_device(d_in.data_ptr(), offs, lens, d_out.data_ptr(), d_out.numel())

    tune_trials = 0
    for _ in range(args.warmup):
        oo, ol, st = step()
        tune_trials += ctx.stats().tune_trials
    assert (st == 0).all() and int(ol.sum()) == total
    byte_exact = hashlib.sha256(d_out[:total].cpu().numpy().tobytes()).hexdigest() == meta["sha256"]
    assert byte_exact, "batched output differs from the plaintext"
    dec_ms, launches = [], 0
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
            s = ctx.stats()
            dec_ms.append(s.ms_decode_kernel)
            launches += s.kernel_launches
            st_last = s
        e1.record()
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    value = world * args.steps * total / (ms / 1e3) / 1e9
    clocks = clk.summary()

    # ---- plain path: one stream per call, same streams, same GPU -------------
    pctx = G.Context(device=local, decoder=args.decoder)
    aoff = np.zeros(n, np.uint64)
    at = 0
    for i in range(n):
        aoff[i] = at
        at += (int(sizes[i]) + 15) & ~15
    d_out2 = torch.empty(at + 4096, dtype=torch.uint8, device="cuda")
    ib, ob = d_in.data_ptr(), d_out2.data_ptr()
    for i in range(min(n, 32)):
        pctx.decompress_device(ib + int(offs[i]), int(lens[i]), ob + int(aoff[i]), int(sizes[i]) + 16)
    torch.cuda.synchronize()
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record()
    plain_launches = 0
    for i in range(n):
        pctx.decompress_device(ib + int(offs[i]), int(lens[i]), ob + int(aoff[i]), int(sizes[i]) + 16)
        plain_launches += pctx.stats().kernel_launches
    p1.record()
    torch.cuda.synchronize()
    plain_ms = p0.elapsed_time(p1)
    plain_gbs = total / (plain_ms / 1e3) / 1e9
    host2 = d_out2.cpu().numpy()
    h = hashlib.sha256()
    for i in range(n):
        h.update(host2[int(aoff[i]):int(aoff[i]) + int(sizes[i])].tobytes())
    plain_exact = h.hexdigest() == meta["sha256"]
    pctx.close()
    del d_out2

    # ---- e2e: the host batch call (gzgpu_decompress_batch), pinned buffers ----
    h_in = torch.from_numpy(packed).pin_memory()
    h_out = torch.empty(total + 16 * n + 4096, dtype=torch.uint8).pin_memory()
    hin, hout = h_in.numpy(), h_out.numpy()
    spans = (G.Span * n)()
    outs = (G.Out * n)()
    o2 = 0
    for i in range(n):
        spans[i] = G.Span(hin.ctypes.data + int(offs[i]), int(lens[i]))
        outs[i] = G.Out(hout.ctypes.data + o2, int(sizes[i]) + 16, 0)
        o2 += int(sizes[i]) + 16
    stv = (ctypes.c_int * n)()
    rc = ctx._lib.gzgpu_decompress_batch(ctx._h, spans, n, outs, stv)
    assert rc == 0, rc
    e2e_steps = args.e2e_steps or max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(e2e_steps):
        ctx._lib.gzgpu_decompress_batch(ctx._h, spans, n, outs, stv)
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = f0.elapsed_time(f1)
    h = hashlib.sha256()
    o2 = 0
    for i in range(n):
        h.update(hout[o2:o2 + int(sizes[i])].tobytes())
        o2 += int(sizes[i]) + 16
    e2e = {"value": round(e2e_steps * total / (e2e_ms / 1e3) / 1e9, 4), "unit": "GB/s",
           "h2d_bytes_per_step": int(lens.sum()), "d2h_bytes_per_step": int(total),
           "byte_exact": h.hexdigest() == meta["sha256"]}

    peak, peak_kind = roofline_peak()
    alg = meta["comp_bytes"] + total
    kern_ms = statistics.mean(dec_ms)
    achieved = alg / (kern_ms / 1e3) / 1e9
    line = {"metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator + zlib levels 1/6/9)", "config": config,
            "byte_exact": byte_exact, "e2e": e2e,
            "plain": {"value": round(plain_gbs, 4), "unit": "GB/s", "ms": round(plain_ms, 1),
                      "calls": n, "gpu_launches": int(plain_launches), "byte_exact": plain_exact},
            "batched_vs_plain": round(value / plain_gbs, 2),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 5),
                         "peak_kind": peak_kind, "traffic": None,
                         "kernel": "inflate_pages_kernel", "kernel_ms": round(kern_ms, 3),
                         "algorithmic_bytes": int(alg)},
            "clocks": clocks, "gpu_launches": int(launches),
            "tuned": {"chunk_bytes": int(st_last.chunk_bytes), "lut_bits": int(st_last.lut_bits),
                      "ctas_per_sm": int(st_last.ctas_per_sm), "key": int(st_last.tune_key),
                      "trials_in_warmup": int(tune_trials)},
            "stages_ms": {k: round(getattr(st_last, k), 3) for k in
                          ("ms_scan", "ms_find", "ms_decode", "ms_decode_kernel", "ms_walk",
                           "ms_resolve", "ms_crc", "ms_total")},
            "chunks": {"n": int(st_last.n_chunks), "rejected": int(st_last.n_rejected),
                       "repairs": int(st_last.n_repairs), "decode_passes": int(st_last.decode_passes)}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_batch_baseline(packed, offs, lens, sizes)
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def bench_sharded(args, rank: int, world: int, local: int, name: str, packed, offs, lens,
                  sizes, meta):
    """Independent gzip streams across `world` GPUs (the members of the
    multi-member stream, or the streams of the batch): each rank decodes a
    disjoint LPT share of them (by compressed size) as one batch job per
    step; there is no collective on the data path.  The total work is fixed
    as ranks are added (strong scaling); the job time is the slowest rank's,
    and every rank's streams must pass their CRC32/ISIZE checks."""
    import datetime
    import torch
    import torch.distributed as dist
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                            device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    import gzippy_b200 as G
    mine = lpt_shards(lens, world)[rank]
    sub_offs = np.zeros(len(mine), np.uint64)
    at = 0
    for k, i in enumerate(mine):
        sub_offs[k] = at
        at += (int(lens[i]) + 15) & ~15
    sub = np.zeros(at + 1024, np.uint8)
    for k, i in enumerate(mine):
        sub[int(sub_offs[k]):int(sub_offs[k]) + int(lens[i])] = \
            packed[int(offs[i]):int(offs[i]) + int(lens[i])]
    sub_lens = np.asarray(lens, np.uint64)[mine]
    total = int(np.asarray(sizes, np.int64)[mine].sum())
    ctx = G.Context(device=local, decoder=args.decoder)
    d_in = torch.from_numpy(sub).cuda()
    d_out = torch.empty(total + 4096, dtype=torch.uint8, device="cuda")

    def step():
        return ctx.decompress_batch_device(d_in.data_ptr(), sub_offs, sub_lens, d_out.data_ptr(),
                                           d_out.numel())

    for _ in range(args.warmup):
        oo, ol, st = step()
    ok = bool((st == 0).all()) and int(ol.sum()) == total
    launches = 0
    with ClockSampler(local) as clk:
        dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
            launches += ctx.stats().kernel_launches
        e1.record()
        torch.cuda.synchronize()
        dist.barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    agg = torch.tensor([float(total), 0.0 if ok else 1.0], dtype=torch.float64, device="cuda")
    dist.all_reduce(agg)
    value = args.steps * float(agg[0].item()) / (ms / 1e3) / 1e9
    ctx.close()
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator + zlib levels 1/6/9)",
            "config": {"workload": name, "streams": len(lens), "plain_bytes": meta["plain_bytes"],
                       "comp_bytes": meta["comp_bytes"],
                       "parallelism": f"streams sharded x{world} (LPT by compressed size)",
                       "l2": "inputs and outputs larger than the 126 MB L2; no flush"},
            "all_streams_ok": agg[1].item() == 0, "clocks": clk.summary(),
            "gpu_launches": int(launches)}), flush=True)
    dist.destroy_process_group()


def bench_members_sharded(args, rank: int, world: int, local: int):
    """The multi-member stream across GPUs: its members are independent gzip
    streams, sharded like a batch."""
    comp, meta = load_workload("multi_member", args.scale)
    mlen = np.array(meta["member_comp_bytes"], np.int64)
    moff = np.concatenate([[0], np.cumsum(mlen)[:-1]]).astype(np.uint64)
    sizes = np.full(len(mlen), meta["plain_bytes"] // len(mlen), np.int64)
    return bench_sharded(args, rank, world, local, "multi_member", comp, moff, mlen, sizes, meta)


def run_trace(srv, comps, sizes, crcs, arrivals, free, verify_every: int = 8):
    """Replay arrivals (t, pool index) against a Server; returns per-request
    (total_ms, queue_ms) in arrival order, wall seconds from the first arrival
    to the last completion, and whether the sampled outputs matched.  Results
    are collected as they complete (not in arrival order), so each output
    buffer returns to the pool as soon as its request is done."""
    import threading
    import zlib
    import gzippy_b200 as G
    lock = threading.Lock()        # free: pool index -> spare output buffers
    tickets = [None] * len(arrivals)
    t0 = time.perf_counter()

    def submitter():
        for k, (t, i) in enumerate(arrivals):
            d = t0 + t - time.perf_counter()
            if d > 0:
                time.sleep(d)
            with lock:
                lst = free.setdefault(i, [])
                out = lst.pop() if lst else np.empty(int(sizes[i]) + 64, np.uint8)
            tickets[k] = (srv.submit(comps[i], out=out), i, out)

    th = threading.Thread(target=submitter)
    th.start()
    lat, ok, n_checked = [None] * len(arrivals), True, 0
    pending, seen, n_done = {}, 0, 0
    while n_done < len(arrivals):
        while seen < len(arrivals) and tickets[seen] is not None:
            pending[seen] = tickets[seen]
            seen += 1
        progressed = False
        for k in list(pending):
            tk, i, out = pending[k]
            rc, data, tm = srv.poll(tk, 0, copy=False)
            if rc == G.PENDING:
                continue
            if rc != G.OK or len(data) != int(sizes[i]):
                ok = False
            elif k % verify_every == 0:
                n_checked += 1
                ok &= zlib.crc32(data) == crcs[i]
            lat[k] = (tm.total_ms, tm.queue_ms)
            with lock:
                free.setdefault(i, []).append(out)
            del pending[k]
            n_done += 1
            progressed = True
        if not progressed:
            time.sleep(0.0002)
    th.join()
    wall = time.perf_counter() - t0
    return lat, wall, ok, n_checked


def bench_serving(args, rank: int, world: int, local: int):
    """Serving: Poisson arrivals of mixed-size requests against the
    continuous-batching Server, and the plain path (one request per call, in
    arrival order) on the same trace."""
    from gzippy_b200 import workloads as W
    import gzippy_b200 as G
    import torch
    torch.cuda.set_device(local)
    comps, sizes, crcs, specs = W.serving_pool(n=args.pool)
    mean_req = float(np.mean(sizes))
    cfg_base = {"workload": "serving", "pool_requests": len(comps), "seed": 1238,
                "host_buffers": "page-locked inputs and outputs >= 1 MiB",
                "sizes": "4-256 KiB log-uniform (p=0.8) or 8-512 MiB log-uniform",
                "budget_bytes": 120 << 30, "lanes": args.lanes,
                "parallelism": f"replicas x{world}"}
    if args.impl == "reference":
        if rank != 0:
            return
        from concurrent.futures import ThreadPoolExecutor
        from oracle import pyoracle as O
        t0 = time.perf_counter()
        with ThreadPoolExecutor(cpus()) as ex:
            outs = list(ex.map(lambda c: O.decompress(c, cap=int(c[-4:].view("<u4")[0]) + 4096)[1].size, comps))
        dt = time.perf_counter() - t0
        v = sum(outs) / dt / 1e9
        print(json.dumps({"metric": METRIC, "value": round(v, 4), "unit": "GB/s", "n_gpus": world,
                          "steps": 1, "warmup": 0, "ms_per_step": round(dt * 1e3, 1),
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "u8", "data": "synthetic", "config": cfg_base, "impl": "reference",
                          "cpu_baseline": {"value": round(v, 4), "unit": "GB/s", "cores": cpus(),
                                           "kind": "port", "sample": "the request pool once, one "
                                           "request per task, oracle serial decoder"},
                          "e2e": {"value": round(v, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    # host buffers page-locked, as a server's caller keeps them (the large
    # ones then move by DMA without staging); small outputs stay pageable
    comps = [torch.from_numpy(c).pin_memory().numpy() for c in comps]

    def out_buf(i):
        n = int(sizes[i]) + 64
        return torch.empty(n, dtype=torch.uint8).pin_memory().numpy() if n >= (1 << 20) \
            else np.empty(n, np.uint8)

    free = {i: [out_buf(i), out_buf(i)] for i in range(len(comps))}

    # capacity: the whole pool submitted at once to a server, after a warm-up pass
    srv = G.Server(device=local, lanes=args.lanes)
    for rep in range(2):
        t0 = time.perf_counter()
        tks = [srv.submit(c, out=free[i][0]) for i, c in enumerate(comps)]
        for tk in tks:
            srv.result(tk, copy=False)
        cap_gbs = sum(sizes) / (time.perf_counter() - t0) / 1e9
    srv.close()
    rate = args.rate or 0.6 * cap_gbs * 1e9 / mean_req
    arrivals = W.poisson_arrivals(1238, rate, args.duration, len(comps))
    offered = sum(sizes[i] for _, i in arrivals)
    res = {}
    for mode in ("served", "plain"):
        if mode == "served":
            srv = G.Server(device=local, lanes=args.lanes)
        else:
            srv = G.Server(device=local, lanes=1, max_batch_requests=1, small_lanes=-1)
        # warm the lanes' buffers with one pass over the pool
        for tk in [srv.submit(c, out=free[i][0]) for i, c in enumerate(comps)]:
            srv.result(tk, copy=False)
        with ClockSampler(local) as clk:
            lat, wall, ok, n_checked = run_trace(srv, comps, sizes, crcs, arrivals, free)
        st = srv.stats()
        srv.close()
        tot = np.array([x[0] for x in lat])
        qw = np.array([x[1] for x in lat])
        # small: outputs under 1 MiB (the 4-256 KiB class of the pool)
        small = np.array([sizes[i] < (1 << 20) for _, i in arrivals[:len(lat)]])
        res[mode] = {"value": round(offered / wall / 1e9, 4), "unit": "GB/s",
                     "p50_ms": round(float(np.percentile(tot, 50)), 3),
                     "p99_ms": round(float(np.percentile(tot, 99)), 3),
                     "p50_queue_ms": round(float(np.percentile(qw, 50)), 3),
                     "p99_queue_ms": round(float(np.percentile(qw, 99)), 3),
                     "small_p50_ms": round(float(np.percentile(tot[small], 50)), 3),
                     "small_p99_ms": round(float(np.percentile(tot[small], 99)), 3),
                     "large_p50_ms": round(float(np.percentile(tot[~small], 50)), 3),
                     "large_p99_ms": round(float(np.percentile(tot[~small], 99)), 3),
                     "requests": len(lat), "batches": int(st.batches), "byte_exact_sample": ok,
                     "checked": n_checked, "wall_s": round(wall, 2), "clocks": clk.summary()}
    line = {"metric": METRIC, "value": res["served"]["value"], "unit": "GB/s", "n_gpus": world,
            "steps": 1, "warmup": 1, "ms_per_step": round(res["served"]["wall_s"] * 1e3, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator + zlib levels 1/6/9)",
            "config": dict(cfg_base, rate_hz=round(rate, 2), duration_s=args.duration,
                           batched_capacity_gbs=round(cap_gbs, 3),
                           mean_request_bytes=int(mean_req), offered_bytes=int(offered)),
            "p50_ms": res["served"]["p50_ms"], "p99_ms": res["served"]["p99_ms"],
            "served": res["served"], "plain": res["plain"],
            "e2e": {"value": res["served"]["value"], "unit": "GB/s",
                    "h2d_bytes_per_step": int(sum(len(comps[i]) for _, i in arrivals)),
                    "d2h_bytes_per_step": int(offered)},
            "clocks": res["served"]["clocks"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self) -> dict:
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def roofline_peak():
    """HBM copy bandwidth: the pool's measured figure when MEASURED_PEAKS.json
    is present, else the 6.65 TB/s fallback measured earlier on the pool."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "of measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "of fallback (MEASURED_PEAKS.json absent)"


def committed_traffic(workload: str):
    """DRAM bytes per compressed byte of the inflate kernel from the committed
    ncu summary (profiles/inflate_traffic.json), if any."""
    p = os.path.join(ROOT, "profiles", "inflate_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    return d.get("dram_bytes_per_comp_byte")


def cpu_baseline(comp: np.ndarray, meta: dict, budget_s: float = 12.0, threads: int | None = None,
                 scale: float = 1.0):
    """The oracle's chunked speculative decoder on all host threads."""
    from oracle import pyoracle as O
    th = threads or cpus()
    cap = meta["plain_bytes"] + 4096
    st, out, _ = O.decompress_chunked(comp, chunk_bytes=4 << 20, threads=th, cap=cap)
    assert st == O.OK and out.size == meta["plain_bytes"]
    times, t_end = [], time.time() + budget_s
    while time.time() < t_end or len(times) < 1:
        t0 = time.perf_counter()
        st, out, _ = O.decompress_chunked(comp, chunk_bytes=4 << 20, threads=th, cap=cap)
        times.append(time.perf_counter() - t0)
        if len(times) >= 20:
            break
    gbs = meta["plain_bytes"] / statistics.median(times) / 1e9
    return {"value": round(gbs, 3), "unit": "GB/s", "cores": th, "kind": "port",
            "sample": f"{len(times)} full decodes of the {meta['plain_bytes'] >> 20} MiB stream "
                      f"(oracle chunked decoder, 4 MiB chunks, median)",
            "cpu": cpu_model(), "config0": config0_baselines(scale=scale)}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def config0_baselines(budget_s: float = 8.0, scale: float = 1.0) -> dict:
    """The CPU figures on the 64 MiB Markov-text member (level 6, one serial
    zlib stream): the oracle's serial decoder on 1 thread (the reference's
    one-thread loop, chunk_fetcher.rs drive_thin_t1_oracle), its chunked
    speculative decoder on all host threads, and system zlib's inflate on 1
    thread (the shape of tools/bench/zng_gunzip.c).  Each is the median of
    the decodes that fit its share of the budget (at least 2)."""
    import zlib
    from oracle import pyoracle as O
    comp, meta = load_workload("single_member_text", scale)
    n = meta["plain_bytes"]
    cb = comp.tobytes()
    th = cpus()

    def timed(fn, share):
        times, t_end = [], time.time() + share
        while len(times) < 2 or (time.time() < t_end and len(times) < 10):
            t0 = time.perf_counter()
            size = fn()
            times.append(time.perf_counter() - t0)
            assert size == n
        return round(n / statistics.median(times) / 1e9, 4), len(times)

    one, k1 = timed(lambda: O.decompress(comp, cap=n + 4096)[1].size, budget_s / 3)
    allt, k2 = timed(lambda: O.decompress_chunked(comp, chunk_bytes=4 << 20, threads=th,
                                                  cap=n + 4096)[1].size, budget_s / 3)
    zl, k3 = timed(lambda: len(zlib.decompress(cb, 31)), budget_s / 3)
    return {"workload": f"single_member_text ({n >> 20} MiB Markov text, level 6, zlib-serial)",
            "unit": "GB/s", "oracle_1_thread": one, "oracle_all_threads": allt,
            "threads": th, "zlib_1_thread": zl, "zlib_version": zlib.ZLIB_RUNTIME_VERSION,
            "decodes": [k1, k2, k3], "cpu": cpu_model()}


def lpt_shards(sizes, world: int):
    """Disjoint work lists for `world` ranks: items in descending size, each
    to the rank with the least total so far (longest processing time first).
    Every item lands on exactly one rank, and no rank's total exceeds the
    mean by more than the largest item.  Returns one sorted index list per
    rank."""
    import heapq
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(x) for x in out]


def max_over_ranks(ms: float, dist, device: str = "cuda") -> float:
    """The job's time: the slowest rank's (all ranks take part; every rank
    gets the result).  `dist` is None for one process."""
    if dist is None:
        return ms
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_gbs(world: int, steps: int, bytes_per_step: int, ms: float) -> float:
    """Whole-job decompressed GB/s: every rank decodes its own replica
    (weak scaling), so the job moves world x steps x bytes in `ms`."""
    return world * steps * bytes_per_step / (ms / 1e3) / 1e9


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="single_member_mixed")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--chunk-bytes", type=int, default=0)
    ap.add_argument("--lut-bits", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=0)
    ap.add_argument("--decoder", type=int, default=0,
                    help="Huffman block decoder: 0 default, 1 lane-parallel 32-bit steps, 2 serial, 3 64-bit steps, 4 per block")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--rate", type=float, default=0.0, help="serving: arrivals/s (0 = 60%% of capacity)")
    ap.add_argument("--duration", type=float, default=60.0, help="serving: seconds of arrivals")
    ap.add_argument("--pool", type=int, default=64, help="serving: distinct requests")
    ap.add_argument("--lanes", type=int, default=4, help="serving: concurrent batches")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3:
        log("warmup raised to 3 (timing rule)")
        args.warmup = 3
    if args.workload == "stream_batch":
        return bench_batch(args, rank, world, local)
    if args.workload == "serving":
        return bench_serving(args, rank, world, local)
    if args.workload == "multi_member" and world > 1 and args.impl != "reference":
        return bench_members_sharded(args, rank, world, local)

    config = {"workload": args.workload, "streams": 1, "level": 6, "seed": 1235,
              "plain_bytes": None, "comp_bytes": None,
              "l2": "inputs (compressed) and outputs larger than the 126 MB L2; no flush",
              "parallelism": f"replicas x{world}"}

    if args.impl == "reference":
        if rank != 0:
            return
        comp, meta = load_workload(args.workload, args.scale)
        config.update(plain_bytes=meta["plain_bytes"], comp_bytes=meta["comp_bytes"],
                      encoder=meta.get("encoder", "zlib-serial"))
        th = cpus()
        from oracle import pyoracle as O
        cap = meta["plain_bytes"] + 4096
        for _ in range(args.warmup):
            st, out, _ = O.decompress_chunked(comp, chunk_bytes=4 << 20, threads=th, cap=cap)
            assert st == O.OK and out.size == meta["plain_bytes"]
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            st, out, _ = O.decompress_chunked(comp, chunk_bytes=4 << 20, threads=th, cap=cap)
            times.append(time.perf_counter() - t0)
        ok = hashlib.sha256(out.tobytes()).hexdigest() == meta["sha256"]
        sec = sum(times)
        v = args.steps * meta["plain_bytes"] / sec / 1e9
        line = {"metric": METRIC, "value": round(v, 4), "unit": "GB/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(1000 * sec / args.steps, 3), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "u8",
                "data": "synthetic (seeded generator + zlib level 6)", "config": config,
                "impl": "reference", "byte_exact": ok,
                "cpu_baseline": {"value": round(v, 4), "unit": "GB/s", "cores": th, "kind": "port",
                                 "sample": f"{args.steps} full decodes of the whole stream by the "
                                           "oracle's chunked speculative decoder (4 MiB chunks)",
                                 "cpu": cpu_model(),
                                 "config0": config0_baselines(scale=args.scale)},
                "e2e": {"value": round(v, 4), "unit": "GB/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    import gzippy_b200 as G
    comp, meta = load_workload(args.workload, args.scale)
    config.update(plain_bytes=meta["plain_bytes"], comp_bytes=meta["comp_bytes"],
                      encoder=meta.get("encoder", "zlib-serial"))
    ctx = G.Context(device=local, chunk_bytes=args.chunk_bytes, lut_bits=args.lut_bits,
                    ctas_per_sm=args.ctas_per_sm, decoder=args.decoder)

    # device-resident buffers (torch only allocates device memory here)
    pad = 1024
    d_in = torch.zeros(comp.size + pad, dtype=torch.uint8, device="cuda")
    d_in[:comp.size].copy_(torch.from_numpy(comp))
    d_out = torch.empty(meta["plain_bytes"] + 4096, dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()

    def step():
        return ctx.decompress_device(d_in.data_ptr(), comp.size, d_out.data_ptr(), d_out.numel())

    for _ in range(args.warmup):
        n = step()
    assert n == meta["plain_bytes"], (n, meta["plain_bytes"])
    digest = hashlib.sha256(d_out[:n].cpu().numpy().tobytes()).hexdigest()
    byte_exact = digest == meta["sha256"]
    assert byte_exact, "device output differs from the plaintext"

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- timed region: value --------------------------------------------------
    dec_ms, launches, st_last = [], 0, None
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
            s = ctx.stats()
            dec_ms.append(s.ms_decode_kernel)
            launches += s.kernel_launches
            st_last = s
        e1.record()
        torch.cuda.synchronize()
        barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    value = job_gbs(world, args.steps, meta["plain_bytes"], ms)
    clocks = clk.summary()

    # ---- e2e through the host C-ABI call with pinned buffers -------------------
    e2e_steps = args.e2e_steps or args.steps
    h_in = torch.from_numpy(comp).pin_memory()
    h_out = torch.empty(meta["plain_bytes"] + 4096, dtype=torch.uint8).pin_memory()
    hin_np, hout_np = h_in.numpy(), h_out.numpy()
    n = ctx.decompress_into(hin_np, hout_np)
    assert n == meta["plain_bytes"]
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(e2e_steps):
        ctx.decompress_into(hin_np, hout_np)
    f1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), dist)
    e2e_ok = hashlib.sha256(hout_np[:n].tobytes()).hexdigest() == meta["sha256"]
    # the same call with pageable buffers (a Rust Vec<u8> / numpy array that
    # was never page-locked), as the drop-in shim passes them
    p_in = np.array(comp, copy=True)
    p_out = np.empty(meta["plain_bytes"] + 4096, np.uint8)
    ctx.decompress_into(p_in, p_out)
    barrier()
    torch.cuda.synchronize()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record()
    for _ in range(e2e_steps):
        ctx.decompress_into(p_in, p_out)
    g1.record()
    torch.cuda.synchronize()
    barrier()
    pg_ms = max_over_ranks(g0.elapsed_time(g1), dist)
    pg_ok = hashlib.sha256(p_out[:n].tobytes()).hexdigest() == meta["sha256"]
    e2e = {"value": round(job_gbs(world, e2e_steps, meta["plain_bytes"], e2e_ms), 4),
           "unit": "GB/s", "h2d_bytes_per_step": int(comp.size),
           "d2h_bytes_per_step": int(meta["plain_bytes"]), "byte_exact": bool(e2e_ok),
           "host_buffers": "page-locked", "steps": e2e_steps,
           "pageable": {"value": round(job_gbs(world, e2e_steps, meta["plain_bytes"], pg_ms), 4),
                        "unit": "GB/s", "byte_exact": bool(pg_ok)}}

    # ---- roofline of the inflate kernel --------------------------------------
    peak, peak_kind = roofline_peak()
    alg = comp.size + meta["plain_bytes"]       # compressed read once + bytes written once
    kern_ms = statistics.mean(dec_ms)
    achieved = alg / (kern_ms / 1e3) / 1e9
    tpc = committed_traffic(args.workload)
    roof = {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 5), "peak_kind": peak_kind,
            "traffic": int(tpc * comp.size) if tpc else None,
            "kernel": "inflate_pages_kernel", "kernel_ms": round(kern_ms, 3),
            "algorithmic_bytes": int(alg)}

    line = {"metric": METRIC, "value": round(value, 4), "unit": "GB/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded generator + zlib level 6)", "config": config,
            "byte_exact": byte_exact, "e2e": e2e, "roofline": roof, "clocks": clocks,
            "gpu_launches": int(launches),
            "step_decode_ms": [round(x, 2) for x in dec_ms],
            "stages_ms": {k: round(getattr(st_last, k), 3) for k in
                          ("ms_scan", "ms_find", "ms_decode", "ms_decode_kernel", "ms_walk",
                           "ms_resolve", "ms_crc", "ms_total")},
            "chunks": {"n": int(st_last.n_chunks), "accepted": int(st_last.n_accepted),
                       "rejected": int(st_last.n_rejected), "repairs": int(st_last.n_repairs),
                       "tail_marker_chunks": int(st_last.n_tail_marker_chunks),
                       "chunk_bytes": int(st_last.chunk_bytes), "lut_bits": int(st_last.lut_bits)}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(comp, meta, scale=args.scale)
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
