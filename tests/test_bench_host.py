"""Host logic of bench.py without a GPU: the timing reduction over ranks (the slowest
rank's time) on two gloo ranks, the mixed 1:1:1 team layout, and the biased action
distribution of the high-contact preset.  CPU only."""
from __future__ import annotations

import argparse
import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    q.put((rank, bench.reduce_max(10.0 + 5.0 * rank, dist, device="cpu")))
    dist.barrier()
    dist.destroy_process_group()


def test_reduce_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out == {0: 15.0, 1: 15.0}


def _args(config):
    return argparse.Namespace(config=config, arenas=None, team_size=None, tick_skip=8, cull=None, no_graph=False)


def test_presets_layout():
    import bench
    wl = bench.Workload(_args("c2"))
    ts = wl.team_sizes()
    assert len(ts) == 32768 and np.bincount(ts)[1:].tolist() == [10923, 10923, 10922]
    assert bench.Workload(_args("c3")).num_arenas == 65536 and bench.Workload(_args("c3")).team_size == 3
    assert bench.Workload(_args("c4")).reset == "high_contact"


def test_biased_actions(pkg):
    import bench
    lut = pkg.rsb.default_action_table()
    w = bench.Workload(_args("c4")).action_weights(lut)
    assert abs(w.sum() - 1) < 1e-12
    assert abs(w[lut["boost"] == 1].sum() - 0.6) < 1e-9 and abs(w[lut["jump"] == 1].sum() - 0.6) < 1e-9
    assert bench.Workload(_args("c3")).action_weights(lut) is None


def test_shard_ranges_balance_cars():
    """Strong-scaling shards: contiguous, covering every arena once, with car counts within one
    arena's cars of the even split (mixed 1:1:1 batch) or equal arena counts (uniform)."""
    import bench
    ts = np.array([1 + (a % 3) for a in range(32768)], np.int32)
    for world in (1, 2, 3, 4, 8):
        ranges = [bench.shard_range(ts, len(ts), r, world) for r in range(world)]
        assert ranges[0][0] == 0 and ranges[-1][1] == len(ts)
        assert all(ranges[r][1] == ranges[r + 1][0] for r in range(world - 1))
        cars = [int(2 * ts[lo:hi].sum()) for lo, hi in ranges]
        assert max(cars) - min(cars) <= 2 * 6, (world, cars)
        uni = [bench.shard_range(None, 1000, r, world) for r in range(world)]
        sizes = [hi - lo for lo, hi in uni]
        assert sum(sizes) == 1000 and max(sizes) - min(sizes) <= 1


def _shard_worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench
    wl = bench.Workload(_args("c2"))
    wl.shard(rank, world)
    mine = torch.tensor([wl.offset, wl.num_arenas, int(wl.team_sizes().sum())], dtype=torch.int64)
    got = [torch.zeros(3, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(got, mine)
    q.put((rank, [g.tolist() for g in got], wl.processed(world)))
    dist.barrier()
    dist.destroy_process_group()


def test_strong_shards_over_two_gloo_ranks():
    """Two ranks each take their shard of the mixed c2 preset; together they cover its 32,768
    arenas once, and each reports the whole set as the arenas processed."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict((r, (g, n)) for r, g, n in (q.get(timeout=120) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shards, processed = out[0]
    assert out[1][0] == shards and processed == 32768
    (o0, n0, t0), (o1, n1, t1) = shards
    assert o0 == 0 and o1 == n0 and n0 + n1 == 32768
    assert abs(t0 - t1) <= 3
