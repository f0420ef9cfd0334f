"""Multi-GPU host logic: z-slab partitioning and the process-group plumbing around it.

The reconstruction shards by slices without any data-path collective: parallel-beam slices
are independent detector rows (ReconEngine already reconstructs a volume block by block of
SliceBlock rows, frameworks/tomography/Framework/ReconFramework/src/ReconEngine.cpp:923-1046),
so each rank reconstructs its own contiguous band of rows. One process per GPU, launched by
torchrun; the collectives here are timing and result assembly only (a barrier, a MAX
reduction of the step time, a gather of the slabs to rank 0).

Slab boundaries are multiples of 4 slices: the reference backprojector updates only the first
4*(nv/4) slices of a block (MultiProjBPparallel.cpp:49-110), so a plan whose inner boundaries
fall on multiples of 4 reconstructs exactly the slices a single block would, and only the
last slab can be ragged.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass(frozen=True)
class Slab:
    rank: int
    start: int  # first slice (detector row) of the slab
    stop: int   # one past the last

    @property
    def size(self) -> int:
        return self.stop - self.start


def slab_plan(nslices: int, world: int, align: int = 4) -> list[Slab]:
    """Contiguous slabs of `nslices` over `world` ranks, inner boundaries on multiples of
    `align`, sizes as even as that allows (ranks at the end may get empty slabs when there are
    fewer aligned groups than ranks)."""
    if world < 1 or nslices < 0 or align < 1:
        raise ValueError("slab_plan: world >= 1, nslices >= 0, align >= 1")
    groups = (nslices + align - 1) // align
    base, extra = divmod(groups, world)
    out, g = [], 0
    for r in range(world):
        ng = base + (1 if r < extra else 0)
        start = min(g * align, nslices)
        g += ng
        out.append(Slab(r, start, min(g * align, nslices)))
    return out


class DistContext:
    """Process group of one job (torchrun environment: RANK, WORLD_SIZE, MASTER_ADDR/PORT).
    backend "nccl" for GPUs, "gloo" for host-only runs; a short timeout so that ranks waiting
    for a lost peer end with an error instead of hanging."""

    def __init__(self, backend: str = "nccl", timeout_s: float = 300.0, device=None):
        import torch
        import torch.distributed as dist

        self.dist = dist
        self.backend = backend
        if not dist.is_initialized():
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        if device is not None:
            self.device = torch.device(device)
        elif backend == "nccl":
            self.device = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
        else:
            self.device = torch.device("cpu")

    def barrier(self) -> None:
        self.dist.barrier()

    def max(self, v: float) -> float:
        """Maximum of a per-rank value (the job's step time is the slowest rank's)."""
        import torch

        t = torch.tensor([float(v)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def gather_slabs(self, local, plan: list[Slab], axis: int):
        """Assemble per-rank slabs (torch tensors, the slab along `axis`) on rank 0; returns the
        full tensor on rank 0 and None elsewhere. Every rank calls this with its own slab."""
        import torch

        local = local.contiguous()
        shape = list(local.shape)
        sizes = [s.size for s in plan]
        maxn = max(sizes)
        shape[axis] = maxn
        pad = torch.zeros(shape, dtype=local.dtype, device=self.device)
        idx = [slice(None)] * len(shape)
        idx[axis] = slice(0, local.shape[axis])
        pad[tuple(idx)] = local.to(self.device)
        bufs = [torch.empty_like(pad) for _ in range(self.world)] if self.rank == 0 else None
        self.dist.gather(pad, gather_list=bufs, dst=0)
        if self.rank != 0:
            return None
        parts = []
        for s, b in zip(plan, bufs):
            idx[axis] = slice(0, s.size)
            parts.append(b[tuple(idx)])
        return torch.cat(parts, dim=axis)

    def close(self) -> None:
        if self.dist.is_initialized():
            self.dist.destroy_process_group()
