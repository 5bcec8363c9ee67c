"""Independent replicas across the GPUs of one node: one process per GPU, each reconstructing its
own scan, with no exchange step on the path (the reference's spatial split with halo exchange is
not this path). The process group only brackets timed regions with barriers and takes the
maximum time over ranks, so the job's throughput is the patterns of every rank over the slowest.

Launched as `torchrun --nproc-per-node N`, the ranks read RANK / LOCAL_RANK / WORLD_SIZE from the
environment; the backend is NCCL on GPUs, gloo elsewhere.
"""
import datetime
import os

import torch
import torch.distributed as dist


def env():
    """`(rank, world_size, local_rank)` from the launcher's environment (1 process: 0, 1, 0)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class Replicas:
    """The group of replica processes; a no-op for a single process."""

    def __init__(self, backend="nccl", timeout_s=120):
        self.rank, self.world, self.local = env()
        self.backend = backend
        self.active = self.world > 1
        if self.active:
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))

    def _device(self):
        return torch.device("cuda", self.local) if self.backend == "nccl" else torch.device("cpu")

    def barrier(self):
        if self.active:
            dist.barrier()

    def max(self, x):
        """The maximum of `x` over the ranks (every rank gets it)."""
        if not self.active:
            return float(x)
        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.active:
            dist.barrier()
            dist.destroy_process_group()
            self.active = False


def job_value(patterns_per_rank, world, steps, max_ms):
    """Whole-job throughput in patterns·iter/s: every rank's patterns of `steps` steps over the
    slowest rank's time."""
    return patterns_per_rank * world * steps / (max_ms / 1e3)
