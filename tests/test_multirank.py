"""The multi-GPU bench path on CPU: world_size-2 process groups over gloo.

Each rank of `bench.py --gpus N` decodes its own replica (weak scaling, no
collective on the data path); the job time is the slowest rank's and the
reference arm prints one line from rank 0 only.  These run without a GPU."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, device="cpu")
    q.put((rank, ms, bench.job_gbs(world, 3, 1 << 20, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_job_time_is_the_slowest_rank():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    for rank, ms, gbs in got:
        assert ms == 15.0
        assert gbs == pytest.approx(2 * 3 * (1 << 20) / 15e-3 / 1e9)


def test_reference_arm_prints_once_under_torchrun():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py",
           "--impl", "reference", "--scale", "0.02", "--steps", "1", "--warmup", "3"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    line = json.loads(lines[0])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port"


def _shard_rank(rank: int, world: int, port: int, q) -> None:
    import datetime
    import numpy as np
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    from gzippy_b200 import workloads as W
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    rng = np.random.default_rng(7)
    # compressed sizes shaped like the two sharded workloads: 2,048 members
    # of 2 MiB at ratios from 0.07 (runs) to 1.0 (random), and the 10,000
    # log-normal streams
    members = (2 << 20) * rng.choice([0.07, 0.35, 0.98, 1.0], 2048)
    streams = W.lognormal_sizes(rng, 10000) * rng.uniform(0.07, 1.0, 10000)
    mine = [bench.lpt_shards(x.astype(np.int64), world)[rank] for x in (members, streams)]
    got = [None] * world
    dist.all_gather_object(got, mine)
    q.put((rank, got, [members.astype(np.int64).tolist(), streams.astype(np.int64).tolist()]))
    dist.barrier()
    dist.destroy_process_group()


def test_lpt_shards_cover_every_stream_once_and_balance():
    """Each rank computes its own share; gathered over gloo, the shares of
    both workloads cover every member / stream exactly once, and no rank's
    compressed bytes exceed the mean by more than the largest item."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_shard_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    gathered = [r[1] for r in res]
    assert gathered[0] == gathered[1]          # every rank sees the same plan
    sizes_all = res[0][2]
    for w, sizes in enumerate(sizes_all):
        shares = [g[w] for g in gathered[0]]
        flat = sorted(i for sh in shares for i in sh)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in sh) for sh in shares]
        assert max(loads) <= sum(sizes) / world + max(sizes)
        assert max(loads) - min(loads) <= max(sizes)
