"""Replica plumbing of bench.py on CPU: world_size 2 over gloo.

Each rank advances its own independent replica (here on the CPU oracle, the
GPU kernels being replaced by the checker since no GPU is present); the only
cross-rank traffic is the max-over-ranks timing and the summed cell count.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from nextgen_b200 import cases, dist
    from nextgen_b200.meshgen import PeriodicBoxMesh
    from oracle import Oracle
    r, w, _ = dist.init("gloo", timeout_s=60)
    m = PeriodicBoxMesh(6, jitter=0.25, seed=1234)  # same replica on every rank
    prm = cases.tgv_params()
    rho, u, p = cases.tgv_state(m.x_cv[: m.ncv], prm)
    o = Oracle(m, prm)
    o.set_state_primitive(rho, u, p)
    o.init_complete()
    dist.barrier()
    o.step(2)
    local_t = 0.5 + r  # a per-rank "duration"
    tmax = dist.max_over_ranks(local_t)
    cells = dist.sum_over_ranks(m.ncv)
    dist.barrier()
    q.put((r, tmax, cells, o.totals().tolist()))
    dist.finalize()


def test_two_replica_ranks_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert [o[1] for o in out] == [1.5, 1.5]          # max over ranks
    assert [o[2] for o in out] == [432.0, 432.0]      # whole-job cells
    assert np.array_equal(out[0][3], out[1][3])       # replicas agree bitwise
