"""The multi-rank bench logic on CPU with the gloo backend (world size 2):
each rank builds its own seeded replica and the step time is the max over ranks."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        gt, init, faces, box = bench.make_workload(rank, small=True)
        ms = bench.max_over_ranks(1.0 + rank, "cpu")
        sig = torch.tensor([float(np.sum(gt))], dtype=torch.float64)
        sigs = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(sigs, sig)
        out[rank] = (ms, [float(s) for s in sigs], len(faces))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_and_max_timing():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    assert res[0][0] == res[1][0] == 2.0          # max over ranks
    assert res[0][1][0] != res[0][1][1]           # different replicas per rank
    assert res[0][2] == res[1][2] == 1280         # same topology size
