"""Replicas across the GPUs of one node: one process per GPU, launched by
torchrun, each solving its own copy of the job with no collective on the
data path (a single query does not shard: the reference's own 2-GPU vertex
partition ran at 0.949x of one GPU, L3_supplementary_experiments_results.md:7).

The only collectives are the timing ones: a barrier around the timed region
and the maximum (or sum) of a per-rank figure, so that a whole-job rate is
(units all ranks processed) / (slowest rank's time).  Every rank calls the
same collectives in the same order.
"""
import datetime
import os


class Replicas:
    """World/rank from the torchrun environment; a process group when the
    world has more than one rank (backend "nccl" for GPUs, "gloo" for CPU)."""

    def __init__(self, backend="nccl", timeout_s=300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self._dist = dist

    def _reduce(self, value, op):
        if self._dist is None:
            return float(value)
        import torch
        dev = "cuda" if self.backend == "nccl" else "cpu"
        t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
        self._dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, value):
        """The largest value over ranks (the slowest rank's time)."""
        if self._dist is None:
            return float(value)
        return self._reduce(value, self._dist.ReduceOp.MAX)

    def sum(self, value):
        if self._dist is None:
            return float(value)
        return self._reduce(value, self._dist.ReduceOp.SUM)

    def broadcast(self, obj):
        """Rank 0's `obj` (any picklable value) on every rank: the solver
        configuration rank 0 tuned, so that every replica runs the same one
        (tuned independently, timing noise could give the ranks different
        picks and the slowest pick would set the job's time)."""
        if self._dist is None:
            return obj
        box = [obj if self.rank == 0 else None]
        self._dist.broadcast_object_list(box, src=0)
        return box[0]

    def barrier(self):
        if self._dist is not None:
            self._dist.barrier()

    def close(self):
        if self._dist is not None:
            self._dist.barrier()
            self._dist.destroy_process_group()
            self._dist = None


def whole_job_rate(units_per_rank, world, max_seconds):
    """Weak scaling: every rank processes units_per_rank; the job ends when
    the slowest rank does."""
    return world * float(units_per_rank) / float(max_seconds)
