"""Process-group plumbing for multi-GPU runs of independent replicas.

The path does not shard (one mesh per GPU; independent cases), so ranks never
exchange field data: they only agree on timings (max over ranks) and on
aggregate counts.  These helpers work with the "nccl" backend on GPUs and with
"gloo" on CPU (used by the tests).
"""
import datetime
import os

import torch
import torch.distributed as tdist


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def init(backend, timeout_s=600):
    """Initialise the default process group from torchrun's environment
    (MASTER_ADDR defaults to 127.0.0.1).  Returns (rank, world, local_rank)."""
    rank, world, local = env_rank()
    if world > 1 and not tdist.is_initialized():
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29511")
        kw = {}
        if backend == "nccl":
            kw["device_id"] = torch.device("cuda", local)
        tdist.init_process_group(backend, rank=rank, world_size=world,
                                 timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return rank, world, local


def _dev():
    if tdist.is_initialized() and tdist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def barrier():
    if tdist.is_initialized():
        t = torch.zeros(1, device=_dev())
        tdist.all_reduce(t)


def max_over_ranks(x):
    """Maximum of a float over all ranks (identity on one process)."""
    if not tdist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_dev())
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x):
    if not tdist.is_initialized():
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_dev())
    tdist.all_reduce(t, op=tdist.ReduceOp.SUM)
    return float(t.item())


def finalize():
    if tdist.is_initialized():
        tdist.destroy_process_group()
