"""Rank plumbing for N independent replicas, one process per GPU: a barrier and the maximum of
a per-rank duration. They are the only exchanges in a replicated measurement (no data crosses
between tunnels). The process group may be NCCL (device tensors) or gloo (CPU tensors)."""
import torch
import torch.distributed as dist


def world_size():
    return dist.get_world_size() if dist.is_available() and dist.is_initialized() else 1


def barrier():
    if world_size() > 1:
        dist.barrier()


def max_over_ranks(x, device=None):
    """The largest value of ``x`` over all ranks (every rank gets it); ``x`` itself with one
    rank. ``device`` is the rank's CUDA device when the group is NCCL."""
    if world_size() == 1:
        return float(x)
    dev = device if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank, slowest_s):
    """Units per second of the whole job: every rank processed ``units_per_rank`` units and the
    slowest took ``slowest_s`` seconds (weak scaling: per-rank work is fixed)."""
    return world_size() * units_per_rank / slowest_s
