"""Replica harness: one process per GPU, each advancing its own independent
DNS instance(s).  The path does not shard (single-GPU semantics of the
reference, no MPI decomposition), so ranks exchange no data: the process
group only lines the ranks up around the timed region and takes the maximum
of their device times.  NCCL when the ranks drive GPUs, gloo otherwise (the
multi-process logic is tested on CPU that way).

Launched by torchrun: RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR/PORT from the
environment.
"""
import os
from datetime import timedelta


def setup(backend=None, timeout_s=600):
    """(world, rank, local_rank, process group module or None)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return world, rank, local, None
    import torch
    import torch.distributed as dist
    if backend is None:
        backend = "nccl" if torch.cuda.is_available() else "gloo"
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return world, rank, local, dist


def _device(pg):
    import torch
    return torch.device("cuda") if pg.get_backend() == "nccl" else torch.device("cpu")


def barrier(pg):
    """All ranks here (and their GPU work done) before anyone goes on."""
    if pg is None:
        return
    import torch
    pg.barrier()
    if pg.get_backend() == "nccl":
        torch.cuda.synchronize()


def allmax(pg, v):
    """Maximum of v over the ranks (the timing rule for multi-GPU numbers)."""
    if pg is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=_device(pg))
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, units_per_rank, seconds_max):
    """Units processed by all ranks over the slowest rank's time (weak
    scaling: every rank does the same fixed work)."""
    return world * units_per_rank / seconds_max


def teardown(pg):
    if pg is not None:
        pg.destroy_process_group()
