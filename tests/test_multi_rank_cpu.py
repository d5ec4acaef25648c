"""bench.py's N>1 logic on CPU: two `gloo` ranks (world_size 2, 127.0.0.1). By default each
rank builds its own replica; with --shard each builds one Morton range of the same diagram's
cells. Either way what runs across ranks is the timing barrier, the max over ranks, the whole-job
rate (replicas: N x sites, shards: sites, over the slowest rank) and byte sums, plus the
reference arm's rule that only rank 0 works. Each rank also checks that it generates the same workload as its peer."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    import bench
    w, r, local = bench.dist_setup("gloo")
    try:
        assert (w, r, local) == (world, rank, rank)
        # slowest rank sets the job time: ranks report 1 ms and 2 ms for 1000 sites each
        value, ms_max = bench.aggregate_rate(1000, 1.0 + rank, w, "cpu")
        # one diagram in two shards: the job rate is the diagram's sites over the slowest shard
        shard_value, _ = bench.shard_rate(1000, 1.0 + rank, w, "cpu")
        vertex_sum = bench.reduce_sum(10.0 * (rank + 1), w, "cpu")
        bench.barrier(w)
        # identical replicas: the workload generator is seeded, so every rank builds the same sites
        sites, cfg = bench.workload("uniform_small", None)
        digest = torch.tensor([float(np.float64(sites.astype(np.float64).sum()))], dtype=torch.float64)
        gathered = [torch.zeros_like(digest) for _ in range(w)]
        dist.all_gather(gathered, digest)
        # the reference arm: ranks other than 0 return without work
        class Args:
            workload, sites, cpu_sample, warmup, steps, gpus = "uniform_small", None, 10, 0, 0, w
        ref = bench.run_reference(Args, w, r) if r != 0 else None
        queue.put((rank, value, ms_max, [float(g) for g in gathered], cfg["sites"], ref, shard_value, vertex_sum))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_and_agree():
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=240) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    for rank, value, ms_max, gathered, n, ref, shard_value, vertex_sum in results:
        assert ms_max == pytest.approx(2.0)
        assert value == pytest.approx(2 * 1000 / 2e-3)
        assert shard_value == pytest.approx(1000 / 2e-3)
        assert vertex_sum == pytest.approx(30.0)
        assert gathered[0] == gathered[1]
        assert n == 10000
        assert ref is None


def test_single_rank_aggregate_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    value, ms_max = bench.aggregate_rate(500, 4.0, 1, "cpu")
    assert ms_max == 4.0 and value == pytest.approx(500 / 4e-3)


def test_spatial_sample_is_a_central_subcube():
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(3)
    sites = np.concatenate([rng.uniform(0, 100, (20000, 3)), rng.uniform(0.5, 2, (20000, 1))], axis=1).astype(np.float32)
    sub = bench.spatial_sample(sites, 2000)
    assert 2000 <= sub.shape[0] <= 2010
    c = np.median(sites[:, :3], axis=0)
    half = np.max(np.abs(sub[:, :3] - c))
    assert half < 30.0  # about (2000/20000)^(1/3) * 50 = 23 around the centre
    # a sample no smaller than the workload is the workload
    assert bench.spatial_sample(sites, 40000).shape == sites.shape


def test_batch_split_is_a_balanced_partition():
    sys.path.insert(0, ROOT)
    import bench
    rng = np.random.default_rng(5)
    sizes = np.exp(rng.uniform(np.log(200), np.log(50000), 500)).astype(np.int64)
    for world in (2, 3, 8):
        share = bench.split_sets(sizes, world)
        flat = sorted(i for part in share for i in part)
        assert flat == list(range(len(sizes)))
        loads = [int(sizes[part].sum()) for part in share]
        assert max(loads) - min(loads) <= int(sizes.max())
