"""Replica coordination for multi-GPU runs.

The reference distributes ONE solve over MPI ranks (decomp.cpp subdomains
with halo exchange); on B200 one solve fits one device, so several GPUs run
independent replicas (ensemble members, repeated bench solves) and only the
host-side bookkeeping is shared: a barrier before and after a timed region
and the maximum of the per-rank device times.  No field data crosses ranks.

``ReplicaGroup`` works over any initialised ``torch.distributed`` process
group -- NCCL with CUDA tensors on a GPU node, gloo with CPU tensors in the
CPU tests -- or with no process group at all (one rank).
"""

from __future__ import annotations


class ReplicaGroup:
    def __init__(self, dist=None, device: str = "cpu"):
        self.dist = dist if (dist is not None and dist.is_available() and dist.is_initialized()) else None
        self.device = device
        self.world = self.dist.get_world_size() if self.dist else 1
        self.rank = self.dist.get_rank() if self.dist else 0

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        """Largest value of x over all ranks (every rank gets it)."""
        if self.dist is None:
            return float(x)
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def throughput(self, cells_per_rank: int, steps: int, local_ms: float) -> float:
        """Whole-job cell updates per second (Gcell-upd/s) for weak scaling:
        every rank advanced its own cells_per_rank-node domain `steps` times;
        the job took as long as the slowest rank."""
        worst = self.max_over_ranks(local_ms)
        if worst <= 0:
            raise ValueError("non-positive device time")
        return self.world * cells_per_rank * steps / (worst * 1e-3) / 1e9


def shard(items: list, rank: int, world: int) -> list:
    """Round-robin share of independent work items (ensemble members) for one
    rank; every item lands on exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    return items[rank::world]
