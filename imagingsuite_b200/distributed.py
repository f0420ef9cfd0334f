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

Cone beam (FDK) shards the same way with a detector-row window per slab (cone_slab_plan): the
rows the slab's voxels project onto, as ReconEngine's CBCT slice blocks take them
(ReconEngine.cpp:954-1008). A rank normalises, filters and backprojects only its window.
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


@dataclass(frozen=True)
class ConeSlab:
    """A slab of FDK output slices (final volume z in [start, stop)) and the detector rows
    [row_start, row_stop) its voxels project onto in every projection."""

    rank: int
    start: int
    stop: int
    row_start: int
    row_stop: int

    @property
    def size(self) -> int:
        return self.stop - self.start

    @property
    def rows(self) -> int:
        return self.row_stop - self.row_start

    def cbct_range(self, nv: int) -> tuple[int, int]:
        """The FDK kernels' slice range k in [k_begin, k_end) (final slice z = nv - 1 - k)."""
        return nv - self.stop, nv - self.start


def cone_row_window(xip, yip, zip_, nu: int, nv: int, k_begin: int, k_end: int, margin: int = 2) -> tuple[int, int]:
    """Detector rows read by the cbct slices [k_begin, k_end) of FDKbp_single's
    backprojection, from the per-projection partials of mr_fdk_partials (xip, yip [nproj][nu][3],
    zip [nproj][nv][3]; no tilt correction). The row of voxel (i, j, k) is
    (zip[k,1] + yip[j,1] + xip[i,1]) / (zip[k,2] + yip[j,2] + xip[i,2]) + 1/2, a linear-fractional
    function of (i, j) and linear in k, so over the slab's box it is extreme at the box corners;
    evaluated there in double, with `margin` rows on both sides for the kernel's float rounding
    (ReconEngine computes its CBCT row window per slice block the same way, with 8 rows of margin,
    ReconEngine.cpp:954-1008). Windows that reach the detector's first or last five rows take the
    whole edge band and the row the FDK filter copies into it (row 5, row nv - 6)."""
    import numpy as np

    if k_end <= k_begin:
        return 0, 0
    X, Y, Z = (np.asarray(a, np.float64) for a in (xip, yip, zip_))
    rows = []
    for k in (k_begin, k_end - 1):
        for j in (0, nu - 1):
            for i in (0, nu - 1):
                w = Z[:, k, 2] + Y[:, j, 2] + X[:, i, 2]
                rows.append((Z[:, k, 1] + Y[:, j, 1] + X[:, i, 1]) / w + 0.5)
    r = np.stack(rows)
    r0 = max(0, int(np.floor(r.min())) - margin)
    r1 = min(nv, int(np.floor(r.max())) + 1 + margin)
    if r0 < 5:
        r0, r1 = 0, max(r1, 6)
    if r1 > nv - 5:
        r0, r1 = min(r0, nv - 6), nv
    if nv % 2:
        # the row filter transforms rows in pairs (2m, 2m + 1) of the flattened stack; with an
        # odd row count those pairs straddle projections and no window reproduces them
        return 0, nv
    # windows on even rows keep the whole detector's row pairs (bit-identical filtered rows)
    return r0 - r0 % 2, min(nv, r1 + r1 % 2)


def cone_slab_plan(nv: int, world: int, xip, yip, zip_, nu: int, align: int = 32, margin: int = 2) -> list[ConeSlab]:
    """Contiguous slabs of the FDK volume's nv slices over `world` ranks (inner boundaries on
    multiples of `align`, the backprojector's slice tile), each with its detector-row window
    (cone_row_window). Every slab is an independent block: its voxels read only the rows of its
    window, so ranks need no data exchange."""
    out = []
    for s in slab_plan(nv, world, align):
        kb, ke = nv - s.stop, nv - s.start
        r0, r1 = cone_row_window(xip, yip, zip_, nu, nv, kb, ke, margin) if s.size else (0, 0)
        out.append(ConeSlab(s.rank, s.start, s.stop, r0, r1))
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
