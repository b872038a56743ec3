"""Host logic of the N > 1 bench path on CPU: two gloo ranks (no GPU).

Each rank solves its own batch (replicas; no data-path collective), all ranks time the same
configuration (the tightest rtol any rank calibrated) and the job time is the max over ranks.
"""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import bench
        import __graft_entry__ as ge
        dtc = ge.load_package()
        grays, bv = bench.make_inputs(dtc, 3, 8, rank)
        tmax = bench.reduce_over_ranks([1.0 + rank, 10.0 * (rank + 1)], "max", device="cpu")
        tmin = bench.reduce_over_ranks([3e-5 if rank == 0 else 1e-5], "min", device="cpu")
        q.put((rank, float(np.abs(grays[0]).sum()), tmax, tmin))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_replicas_and_max_time():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, tmax0, tmin0), (r1, s1, tmax1, tmin1) = out
    assert s0 != s1                                   # each rank has its own domains
    assert tmax0 == tmax1 == [2.0, 20.0]              # job time = max over ranks
    assert tmin0 == tmin1 == [1e-5]                   # same rtol on every rank


def test_single_process_reduction_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.reduce_over_ranks([1.5, 2.5]) == [1.5, 2.5]
