"""Multi-rank logic of bench.py on CPU ranks over gloo (world size 2): job totals take the
slowest rank's time and every rank's node updates, and batched workloads give every rank its
own deterministic shard of surfaces; two ranks advancing their shards of the batched 3D
workload through the oracle give the same combined counts and states as one process running
both shards."""
import datetime
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=ws, timeout=datetime.timedelta(seconds=60))
    try:
        t, w, nu = bench.combine_ranks(dist, 10.0 + rank, 1.0 + 2.0 * rank, 1000 * (rank + 1),
                                       "cpu")
        shard = bench.batch_surfaces("c4", bench.CONFIGS["c4"], rank)
        q.put((rank, t, w, nu, shard))
    finally:
        dist.destroy_process_group()


def test_two_ranks_combine_and_shard():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict()
    for _ in procs:
        r, t, w, nu, shard = q.get(timeout=120)
        out[r] = (t, w, nu, shard)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in range(2):
        t, w, nu, _ = out[r]
        assert (t, w, nu) == (11.0, 3.0, 3000.0)
    sys.path.insert(0, ROOT)
    import bench
    assert out[0][3] == bench.batch_surfaces("c4", bench.CONFIGS["c4"])
    assert out[1][3] != out[0][3]
    assert out[1][3] == bench.batch_surfaces("c4", bench.CONFIGS["c4"], 1)


K, STEPS = 3, 4


def _shard_main(rank, ws, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=ws, timeout=datetime.timedelta(seconds=120))
    try:
        digest = []
        _, nu, secs = bench.cpu_batch("c4", bench.CONFIGS["c4"], STEPS, K, shard=rank,
                                      digest=digest)
        t, w, total = bench.combine_ranks(dist, secs * 1e3, secs, nu, "cpu")
        q.put((rank, nu, total, digest))
    finally:
        dist.destroy_process_group()


def test_two_ranks_advance_their_shards_like_one_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict()
    for _ in procs:
        r, nu, total, digest = q.get(timeout=300)
        out[r] = (nu, total, digest)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, ROOT)
    import bench
    single = []
    for shard in range(2):
        d = []
        _, nu, _ = bench.cpu_batch("c4", bench.CONFIGS["c4"], STEPS, K, shard=shard, digest=d)
        single.append((nu, d))
    assert out[0][1] == out[1][1] == single[0][0] + single[1][0]
    for r in range(2):
        assert out[r][0] == single[r][0]
        assert out[r][2] == single[r][1]
        assert all(x is not None for x in out[r][2])
    assert out[0][2] != out[1][2]
