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


def _shard_worker(rank, world, port, spp, out):
    sys.path[:0] = [ROOT, os.path.join(ROOT, "agent-ray_b200"), os.path.join(ROOT, "oracle")]
    import datetime

    import torch
    from agentray import distributed as D
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))

    class FakeIntegrator:
        class config:
            pass
    FakeIntegrator.config.spp = spp

    def fake(begin, end, film):
        # stands in for the GPU render of a range: per-sample contributions
        # (index-dependent) / spp, so the reduced film checks the partition
        w = torch.arange(film.numel(), dtype=torch.float32)
        for s in range(begin, end):
            film += (w + s) / spp
    img = D.render(FakeIntegrator, None, None, 4, 3, device="cpu", render_fn=fake)
    out[rank] = img.numpy().copy()
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,spp", [(2, 16), (3, 5), (2, 1)])
def test_sample_sharding_sums_to_the_full_image(world, spp):
    import numpy as np
    from agentray import distributed as D
    ranges = [D.shard_range(spp, r, world) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == spp
    assert all(ranges[i][1] == ranges[i + 1][0] for i in range(world - 1))
    port = 30500 + (os.getpid() % 2000) + world * 7 + spp
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_shard_worker, args=(world, port, spp, out), nprocs=world, join=True)
        res = dict(out)
    w = np.arange(36, dtype=np.float64)
    expect = sum((w + s) / spp for s in range(spp)).reshape(3, 4, 3)
    for r in range(world):
        np.testing.assert_allclose(res[r], expect, rtol=1e-5)
