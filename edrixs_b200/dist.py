"""Process-group plumbing for N-GPU replica runs (one process per GPU).

The ED/XAS/RIXS path here runs as independent replicas: every rank serves its own
requests on its own GPU.  The only cross-rank operations are a barrier around timed
regions and the maximum of the per-rank timings, so that a throughput over N GPUs is the
work of all ranks divided by the slowest rank's time.
"""
import datetime
import os

import torch
import torch.distributed as dist


def world():
    return int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))


def init_from_env(backend=None, timeout_s=600):
    """Join the process group described by torchrun's environment (no-op for one rank)."""
    ws, rank = world()
    if ws > 1 and not dist.is_initialized():
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return ws, rank


def _dev():
    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier():
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def reduce_max(x: float) -> float:
    if not (dist.is_available() and dist.is_initialized()):
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=_dev())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def finalize():
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
