"""The multi-GPU plumbing of bench.py, on CPU with the gloo backend.

The path shards without a collective on its data (every rank renders or
traverses its own replica of the workload); the only cross-rank steps are the
barrier around the timed region and the max-over-ranks time.  Two gloo ranks
check: each rank draws its own ray batches (different seeds, same scene), the
job time is the slowest rank's, and the whole-job rate counts every rank's
units.
"""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "toy-path-tracing_b200"))
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        _, batches = bench.make_workload(rank, 10)
        dist.barrier()
        slowest = bench.max_over_ranks(1.0 + rank, world, device="cpu")
        rate = bench.whole_job_rate(world, 4 * batches[0].shape[1], slowest)
        out[rank] = (float(batches[1][0:3].sum()), float(batches[0][3:6].sum()), slowest, rate)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank_main, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        res = dict(out)
    inc0, coh0, slow0, rate0 = res[0]
    inc1, coh1, slow1, rate1 = res[1]
    assert inc0 != inc1 and coh0 != coh1  # independent replicas: different ray batches per rank
    assert slow0 == slow1 == 2.0  # max over ranks
    assert rate0 == rate1 == 2 * 4 * 1024 / 2.0
