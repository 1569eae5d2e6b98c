"""The multi-rank plumbing (droplet_b200.ranks) as two gloo processes on CPU:
the job's time is the slowest rank's and its vertex count the sum, gradients
of views rendered on different ranks are summed, the views are split without
overlap, and each rank draws its own sample streams.  One process without a
process group gets its own values back."""
import os
import socket

import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, size, port, out):
    import torch.distributed as dist

    from droplet_b200 import ranks

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=size,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        res = {"world": ranks.world()}
        res["slowest_and_total"] = ranks.slowest_and_total(1.0 + rank, 10.0 * (rank + 1))
        res["slowest"] = ranks.slowest(0.5 + rank)
        g = torch.full((4, 512), rank + 1.0)
        a = torch.tensor([2.0 * rank], dtype=torch.float64)
        ranks.sum_gradients(g, a, None)
        res["grad"] = (float(g.min()), float(g.max()), float(a.item()))
        res["views"] = ranks.my_views(list(range(7)), rank, size)
        res["seed"] = ranks.frame_seed(1000, rank)
        dist.barrier()
        out[rank] = res
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_combine_as_the_job_does():
    size = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_worker, args=(r, size, port, out)) for r in range(size)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert [res[r]["world"] for r in range(size)] == [(0, 2), (1, 2)]
    for r in range(size):
        assert res[r]["slowest_and_total"] == (2.0, 30.0)
        assert res[r]["slowest"] == 1.5
        assert res[r]["grad"] == (3.0, 3.0, 2.0)
    views = res[0]["views"] + res[1]["views"]
    assert sorted(views) == list(range(7)) and not set(res[0]["views"]) & set(res[1]["views"])
    assert res[0]["seed"] != res[1]["seed"]


def test_one_process_keeps_its_values():
    from droplet_b200 import ranks

    import torch.distributed as dist

    if dist.is_initialized():
        pytest.skip("a process group is active")
    assert ranks.world() == (0, 1)
    assert ranks.slowest_and_total(1.25, 7.0) == (1.25, 7.0)
    g = torch.ones(3)
    ranks.sum_gradients(g)
    assert torch.equal(g, torch.ones(3))
    assert ranks.my_views([1, 2, 3], 0, 1) == [1, 2, 3]
