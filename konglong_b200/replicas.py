"""Replica plumbing for multi-GPU runs: one independent shot per GPU.

RTM shots share nothing, so N GPUs run N replicas with no collective in the
data path (weak scaling).  The only cross-rank traffic is bookkeeping: a
barrier around the timed region and the max over ranks of the device time.
Ranks come from the torchrun environment (RANK / WORLD_SIZE / LOCAL_RANK);
the process group uses NCCL on GPUs and gloo in the CPU tests.
"""
import datetime
import os
from dataclasses import dataclass


@dataclass
class Ranks:
    rank: int = 0
    world: int = 1
    local_rank: int = 0

    @staticmethod
    def from_env(env=None):
        env = os.environ if env is None else env
        return Ranks(int(env.get("RANK", "0")), int(env.get("WORLD_SIZE", "1")), int(env.get("LOCAL_RANK", "0")))

    @property
    def distributed(self):
        return self.world > 1


def init(ranks, backend="nccl", timeout_s=300.0):
    """Join the process group (N > 1 only).  The timeout bounds every
    collective, so a rank that died makes the others fail instead of waiting."""
    if not ranks.distributed:
        return
    import torch.distributed as dist
    dist.init_process_group(backend, rank=ranks.rank, world_size=ranks.world,
                            timeout=datetime.timedelta(seconds=timeout_s))


def barrier(ranks):
    if ranks.distributed:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ranks, x, device=None):
    """Largest `x` over all ranks (every rank gets it)."""
    if not ranks.distributed:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_gpts(world, cells, steps, ms):
    """Whole-job throughput: every rank advanced `cells` by `steps` steps in at
    most `ms` (the max over ranks)."""
    return world * cells * steps / (ms * 1e-3) / 1e9


def runs_reference_arm(ranks):
    """The CPU reference arm is timed once, on rank 0; other ranks do no work."""
    return ranks.rank == 0


def finish(ranks):
    if ranks.distributed:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
