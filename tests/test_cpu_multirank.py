"""The N > 1 path of bench.py on CPU: two gloo ranks, each timing its own
replica (weak scaling, no data-path collective); the job time is the max over
ranks and each rank serves a different seeded job stream."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "agent-ray_b200"), os.path.join(ROOT, "oracle")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    r, local, w = bench.dist_env()
    ms = bench.max_over_ranks(dist, 10.0 * (r + 1), "cpu")
    stream = bench.rank_stream(50, r)
    out[r] = (r, w, ms, tuple((j["scene"], j["res"], j["spp"], j["integrator"]) for j in stream))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_max_time_and_distinct_streams():
    world = 2
    port = 29500 + (os.getpid() % 2000)
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for r in range(world):
        rank, w, ms, _ = res[r]
        assert rank == r and w == world
        assert ms == 20.0  # the slowest rank's time, on every rank
    assert res[0][3] != res[1][3]  # each replica renders its own stream
