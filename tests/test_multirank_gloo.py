"""The multi-rank path of bench.py on CPU ranks (gloo, world size 2): each rank
builds its own batch of the scan (no data exchange), and the whole-job rate is
the sum of all ranks' grid-point steps over the slowest rank's time."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    from espec_b200 import workloads as W
    from oracle import oracle as O

    w = W.morse_scan(npk=3, nsteps=20, seed=bench.rank_seed(rank), sizes=(256, 384))
    c, _, _ = O.spo_batch(w["off"], w["sh"], w["sm"], w["vpot"], w["psi"],
                          np.zeros_like(w["psi"]), w["dt_fs"], w["nsteps"], nthreads=1)
    pts = float(w["off"][-1]) * w["nsteps"]
    ms = 10.0 + 5.0 * rank  # stand-in per-rank times: the slowest rank decides
    rate, ms_job, pts_job = bench.job_rate(pts, ms, world)
    out[rank] = (pts, rate, ms_job, pts_job, c.real.sum())
    dist.destroy_process_group()


def test_two_ranks_independent_batches_and_job_rate():
    world, port = 2, _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True,
                       start_method="spawn")
    (p0, r0, m0, t0, c0), (p1, r1, m1, t1, c1) = out[0], out[1]
    assert m0 == m1 == 15.0                       # max over ranks
    assert t0 == t1 == p0 + p1                    # sum over ranks
    assert r0 == r1 == (p0 + p1) / 15e-3 / 1e6    # whole-job rate
    assert c0 != c1                               # different, independent batches
