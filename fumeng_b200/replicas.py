"""Replicated rendering over several processes (one per GPU).

The path tracer needs no exchange between GPUs: scenes, views, pixels and samples are
independent.  Each rank renders its own batch of scenes (weak scaling); the ranks only
meet to line up the timed region and to combine two numbers, the device time (maximum
over ranks) and the paths rendered (sum over ranks).  These helpers hold that logic so
that it runs the same way with NCCL on GPUs and with gloo on CPU processes.
"""
from __future__ import annotations


def batch_indices(rank: int, per_rank: int, batch: int | None = None) -> list:
    """Scene indices rank `rank` renders: its own block of `batch` seeded scenes (the
    first `per_rank` of them), disjoint from every other rank's."""
    batch = per_rank if batch is None else batch
    return [rank * batch + s for s in range(per_rank)]


class RankGroup:
    """Barrier, max and sum over the ranks of a torch.distributed process group (or a
    single process when `dist` is None).  `device` is where the reduction tensors live:
    "cuda" for NCCL, "cpu" for gloo."""

    def __init__(self, dist=None, device: str = "cuda"):
        self.dist = dist
        self.device = device

    def _sync(self):
        if self.device == "cuda":
            import torch
            torch.cuda.synchronize()

    def barrier(self) -> None:
        self._sync()
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        if self.dist is None:
            return float(x)
        import torch
        t = torch.tensor([float(x)], device=self.device, dtype=torch.float64)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist is not None else None)

    def sum(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist is not None else None)

    def throughput(self, paths: float, elapsed_ms: float) -> float:
        """Whole-job Mpaths/s: the paths of all ranks over the slowest rank's time."""
        return self.sum(paths) / (self.max(elapsed_ms) / 1e3) / 1e6
