"""The multi-rank host logic of bench.py on CPU: two gloo ranks on
127.0.0.1.  Replicas share no data; the ranks only agree on the slowest
rank's timings (every rank gets the maximum), only rank 0 reports, the
reference arm's other ranks do no work, and each rank steps its own seeded
scene."""
import argparse
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        got = bench.max_over_ranks([10.0 + rank, 5.0 - rank, 3.0], world)
        ref = None
        if rank != 0:
            args = argparse.Namespace(workload="semi", steps=1, warmup=0, gpus=world, ref_sample=None)
            ref = bench.run_reference_arm(args, rank, world)
        sc = bench.make_scene("explicit", rank)
        from mps_solvers_b200 import scene
        pos, _, _ = scene.build(sc)
        q.put((rank, got, ref, float(np.asarray(pos)[:, 0].sum())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=240) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, got, ref, _ in out:
        assert got == [11.0, 5.0, 3.0], got      # the max over both ranks, on every rank
        if rank != 0:
            assert ref is None                    # the reference arm runs on rank 0 only
    assert out[0][3] != out[1][3]                 # each replica steps its own seeded scene
