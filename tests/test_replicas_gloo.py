"""The N > 1 host path on CPU: two gloo ranks route disjoint shares of the
batched sweep and the request stream, and reduce timings (max) and work (sum)
as bench.py does over NCCL on GPUs."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    from shoeridingerequationsolver_b200 import replicas, scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    specs = scenes.config_c4_specs(256)
    mine = replicas.route_balanced(specs, rank, world, lambda s: s["n"] ** 3)
    pts = sum(s["n"] ** 3 for s in mine)
    total = replicas.sum_over_ranks(pts, dist)
    slowest = replicas.max_over_ranks(10.0 + rank, dist)
    reqs = replicas.route(list(range(48)), rank, world)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, [s["index"] for s in mine], total, slowest, reqs))


def test_two_gloo_ranks_route_and_reduce():
    from shoeridingerequationsolver_b200 import scenes
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, i0, t0, m0, q0), (r1, i1, t1, m1, q1) = out
    assert set(i0).isdisjoint(i1) and sorted(i0 + i1) == list(range(256))
    assert t0 == t1 == sum(s["n"] ** 3 for s in scenes.config_c4_specs(256))
    assert m0 == m1 == 11.0
    # the balanced split gives each rank the same grid points to within one instance
    byidx = {s["index"]: s["n"] ** 3 for s in scenes.config_c4_specs(256)}
    p0, p1 = sum(byidx[i] for i in i0), sum(byidx[i] for i in i1)
    assert abs(p0 - p1) <= 160 ** 3
    assert sorted(q0 + q1) == list(range(48)) and set(q0).isdisjoint(q1)


def test_route_rejects_bad_rank():
    from shoeridingerequationsolver_b200 import replicas
    with pytest.raises(ValueError):
        replicas.route([1, 2, 3], 2, 2)
