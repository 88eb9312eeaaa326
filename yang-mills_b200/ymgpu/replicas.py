"""Replica plumbing for multi-GPU runs: one process per GPU, each with its
own independent chains (the path shards by chain; no data-path collective).

``Replicas`` reads RANK / WORLD_SIZE / LOCAL_RANK as torchrun sets them,
opens a process group only when there is more than one rank (NCCL on GPUs,
gloo on host-only runs and tests), and offers what a replicated measurement
needs: a barrier, the maximum and the sum over ranks (every timed figure is
the slowest rank's), per-rank chain seeds, and output from rank 0 alone.
The group has a short timeout, so a rank that dies or never joins ends the
others' next collective with an error instead of a hang.
"""
from __future__ import annotations

import datetime
import json
import os
from typing import Optional


class Replicas:
    def __init__(self, backend: Optional[str] = None, timeout_s: float = 120.0, device=None):
        self.rank = int(os.environ.get("RANK", "0"))
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or "nccl"
        self._device = device
        self._dist = None
        if self.world > 1:
            import torch.distributed as dist
            kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
            if self.backend == "nccl" and device is not None:
                kw["device_id"] = device
            dist.init_process_group(self.backend, **kw)
            self._dist = dist

    def _tensor(self, x: float):
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        return torch.tensor([float(x)], dtype=torch.float64, device=dev)

    def barrier(self) -> None:
        if self._dist is not None:
            self._dist.barrier()

    def max_over_ranks(self, x: float) -> float:
        if self._dist is None:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(self, x: float) -> float:
        if self._dist is None:
            return float(x)
        t = self._tensor(x)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.SUM)
        return float(t.item())

    def chain_seed(self, master_seed: int) -> int:
        """This rank's SU(3) chain seed: the reference's derivation with the
        rank as chain id (su3_ensemble.rs:189-192)."""
        from .su3_ensemble import derive_su3_chain_seed
        return derive_su3_chain_seed(master_seed, self.rank)

    def weak_value(self, units_per_rank: float, seconds: float) -> float:
        """Whole-job throughput when every rank does the same work: the units
        of all ranks over the slowest rank's time (``seconds`` must already
        be the maximum over ranks)."""
        return self.world * units_per_rank / seconds

    def emit(self, record: dict, stream=None) -> None:
        """One JSON line, from rank 0 only."""
        if self.rank == 0:
            line = json.dumps(record)
            if stream is None:
                print(line, flush=True)
            else:
                stream.write(line + "\n")
                stream.flush()

    def close(self) -> None:
        if self._dist is not None:
            self._dist.destroy_process_group()
            self._dist = None
