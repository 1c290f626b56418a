"""Replica plumbing for runs on several GPUs of one node.

The HOS time advance does not shard: every transform of a step needs the
whole field, and the reference's MPI slab decomposition (Csource/2dpar,
fft_routines_2d_par.c) exists only to spread one field over CPU ranks.  A
field fits one B200 many times over, so N GPUs run N independent replicas,
one process per GPU, each advancing its own seeded field.  The only
collectives are the barrier around a timed region and the maximum over
ranks of its measured time; the whole-job rate is the work of all ranks
divided by that maximum.
"""
from __future__ import annotations

import datetime
import os


class Replicas:
    """Rank bookkeeping from the torchrun environment (RANK, WORLD_SIZE,
    LOCAL_RANK, MASTER_ADDR/PORT) and the two collectives of a replica run.
    With WORLD_SIZE 1 (or unset) nothing is initialised and every collective
    is the identity.  ``backend`` is "nccl" on GPUs, "gloo" on CPUs."""

    def __init__(self, backend="nccl", timeout_s=120.0):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", str(self.rank)))
        self.backend = backend
        self._pg = False
        if self.world > 1:
            import torch
            import torch.distributed as tdist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
            tdist.init_process_group(backend, rank=self.rank, world_size=self.world,
                                     timeout=datetime.timedelta(seconds=timeout_s))
            self._pg = True

    @property
    def distributed(self):
        return self._pg

    def _device(self):
        return "cuda" if self.backend == "nccl" else "cpu"

    def barrier(self):
        if self._pg:
            import torch.distributed as tdist

            tdist.barrier()

    def _reduce(self, x, op):
        import torch
        import torch.distributed as tdist

        t = torch.tensor([float(x)], dtype=torch.float64, device=self._device())
        tdist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x):
        """Maximum of x over ranks (every rank gets it)."""
        if not self._pg:
            return float(x)
        import torch.distributed as tdist

        return self._reduce(x, tdist.ReduceOp.MAX)

    def sum(self, x):
        if not self._pg:
            return float(x)
        import torch.distributed as tdist

        return self._reduce(x, tdist.ReduceOp.SUM)

    def seed(self, base):
        """Each replica advances its own field: seeds differ by rank."""
        return int(base) + self.rank

    def rate(self, units_per_rank, ms_per_rank):
        """Whole-job rate: the units all ranks processed over the slowest
        rank's time (ms), in units per second."""
        ms = self.max(ms_per_rank)
        return self.world * units_per_rank / (ms / 1e3), ms

    def close(self):
        if self._pg:
            import torch.distributed as tdist

            tdist.destroy_process_group()
            self._pg = False

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
