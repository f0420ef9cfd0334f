"""Multi-GPU host logic on the CPU: the z-slab plan, and world-size-2 gloo jobs that
reconstruct their slabs of a parallel-beam volume with the oracle and assemble them on rank
0 (the same DistContext the benchmark drives over NCCL)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from imagingsuite_b200.distributed import Slab, slab_plan


def test_slab_plan_covers_and_aligns():
    for n in (0, 1, 7, 8, 64, 70, 1023, 1024):
        for w in (1, 2, 3, 4, 8):
            plan = slab_plan(n, w)
            assert len(plan) == w
            assert plan[0].start == 0 and plan[-1].stop == n
            for a, b in zip(plan, plan[1:]):
                assert a.stop == b.start
                assert a.stop % 4 == 0 or a.stop == n
            groups = [(s.size + 3) // 4 for s in plan]  # aligned groups per rank differ by at most one
            assert max(groups) - min(groups) <= 1


def test_slab_plan_rejects_bad_arguments():
    with pytest.raises(ValueError):
        slab_plan(10, 0)
    assert slab_plan(10, 2, align=1) == [Slab(0, 0, 5), Slab(1, 5, 10)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, proj, ang, w, centre, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch

    import oracle as O
    from imagingsuite_b200.distributed import DistContext, slab_plan

    ctx = DistContext("gloo", timeout_s=60)
    try:
        nv = proj.shape[1]
        plan = slab_plan(nv, ctx.world)
        s = plan[ctx.rank]
        # this rank's rows: an independent block of the reference backprojector
        vol = O.bp_parallel(np.ascontiguousarray(proj[:, s.start:s.stop]), ang, w, centre, buffersize=16)
        full = ctx.gather_slabs(torch.from_numpy(vol), plan, axis=2)
        t = ctx.max(0.25 + rank)
        ctx.barrier()
        q.put((rank, None if full is None else full.numpy(), t))
    finally:
        ctx.close()


def test_gloo_slabs_reassemble_single_block():
    rng = np.random.default_rng(5)
    nproj, nv, nu = 19, 12, 24
    proj = rng.standard_normal((nproj, nv, nu)).astype(np.float32)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    w = np.full(nproj, np.float32(np.pi / nproj))
    import oracle as O

    whole = O.bp_parallel(proj, ang, w, 11.3, buffersize=16)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, proj, ang, w, 11.3, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = {}
    for _ in procs:
        r, full, t = q.get(timeout=120)
        res[r] = (full, t)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1][0] is None
    assert np.array_equal(res[0][0], whole)  # slabs of 8 + 4 rows == one 12-row block
    assert res[0][1] == res[1][1] == 1.25     # every rank sees the slowest rank's time


# ------------------------------------------------------------------------- cone beam


def _fdk_case():
    import ctypes

    from imagingsuite_b200 import _lib as L

    rng = np.random.default_rng(9)
    nproj, nv, nu = 24, 96, 64
    proj = (rng.standard_normal((nproj, nv, nu)) * 0.2 + 1.0).astype(np.float32)
    ang = (np.arange(nproj) * 360.0 / nproj).astype(np.float32)
    w = np.full(nproj, np.float32(1.0 / nproj))
    g = L.FdkGeom()
    g.sod, g.sdd = 300.0, 600.0
    g.ppoint[0], g.ppoint[1] = (nu - 1) / 2 + 0.13, (nv - 1) / 2 - 0.21
    g.center = (nu - 1) / 2 + 0.07
    g.resolution[0] = g.resolution[1] = 0.8
    g.voxelsize[0] = g.voxelsize[1] = g.voxelsize[2] = 0.4
    xip = np.empty((nproj, nu, 3), np.float32)
    yip = np.empty((nproj, nu, 3), np.float32)
    zip_ = np.empty((nproj, nv, 3), np.float32)
    s2, sc, uni = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
    L.check(L.lib().mr_fdk_partials(ctypes.byref(g), nu, nv, ang.ctypes.data_as(L.P_float), nproj,
                                    xip.ctypes.data_as(L.P_float), yip.ctypes.data_as(L.P_float),
                                    zip_.ctypes.data_as(L.P_float), ctypes.byref(s2), ctypes.byref(sc),
                                    ctypes.byref(uni)))
    return proj, ang, w, (xip, yip, zip_), nu, nv


def test_cone_row_window_covers_every_voxel():
    """The corner-based row window of a slab holds every row a voxel of the slab samples
    (all voxels, double precision), with the edge bands closed."""
    from imagingsuite_b200.distributed import cone_row_window, cone_slab_plan

    proj, ang, w, (X, Y, Z), nu, nv = _fdk_case()
    for world in (2, 3):
        plan = cone_slab_plan(nv, world, X, Y, Z, nu)
        assert plan[0].start == 0 and plan[-1].stop == nv
        for s in plan:
            kb, ke = s.cbct_range(nv)
            Xd, Yd, Zd = (a.astype(np.float64) for a in (X, Y, Z))
            k = np.arange(kb, ke)
            num = Zd[:, k, 1][:, :, None, None] + Yd[:, None, :, 1][:, :, :, None] + Xd[:, None, None, :, 1]
            den = Zd[:, k, 2][:, :, None, None] + Yd[:, None, :, 2][:, :, :, None] + Xd[:, None, None, :, 2]
            r = np.floor(num / den + 0.5)
            r = r[(r >= 0) & (r < nv)]
            assert r.min() >= s.row_start and r.max() < s.row_stop, (world, s)
            if s.row_start < 5:
                assert s.row_start == 0 and s.row_stop >= 6
            if s.row_stop > nv - 5:
                assert s.row_stop == nv and s.row_start <= nv - 6
        assert cone_row_window(X, Y, Z, nu, nv, 10, 10) == (0, 0)


def _cone_rank_main(rank, world, port, filt, ang, windows, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import torch

    import oracle as O
    from imagingsuite_b200.distributed import ConeSlab, DistContext

    ctx = DistContext("gloo", timeout_s=60)
    try:
        plan = [ConeSlab(*p) for p in windows]
        s = plan[ctx.rank]
        # this rank holds only its detector-row window of the filtered projections
        held = np.zeros_like(filt)
        held[:, s.row_start:s.row_stop] = filt[:, s.row_start:s.row_stop]
        g = O.fdk_geom(300.0, 600.0, ((filt.shape[2] - 1) / 2 + 0.13, (filt.shape[1] - 1) / 2 - 0.21),
                       (filt.shape[2] - 1) / 2 + 0.07, (0.8, 0.8), (0.4, 0.4, 0.4))
        vol = O.fdk_bp(held, ang, g)[s.start:s.stop]
        full = ctx.gather_slabs(torch.from_numpy(np.ascontiguousarray(vol)), plan, axis=0)
        ctx.barrier()
        q.put((rank, None if full is None else full.numpy()))
    finally:
        ctx.close()


def test_gloo_cone_slabs_reassemble_single_block():
    """Two ranks, each holding only its slab's detector-row window of the filtered
    projections, backproject their FDK slabs; rank 0 assembles the volume, equal bit for bit to
    the single-block reconstruction."""
    import oracle as O
    from imagingsuite_b200.distributed import cone_slab_plan

    proj, ang, w, (X, Y, Z), nu, nv = _fdk_case()
    g = O.fdk_geom(300.0, 600.0, ((nu - 1) / 2 + 0.13, (nv - 1) / 2 - 0.21), (nu - 1) / 2 + 0.07, (0.8, 0.8),
                   (0.4, 0.4, 0.4))
    filt = O.fdk_prepare(proj, w, g)
    whole = O.fdk_bp(filt, ang, g)
    plan = cone_slab_plan(nv, 2, X, Y, Z, nu)
    assert all(s.rows < nv for s in plan)  # each rank holds a strict part of the detector
    windows = [(s.rank, s.start, s.stop, s.row_start, s.row_stop) for s in plan]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_cone_rank_main, args=(r, 2, port, filt, ang, windows, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[1] is None
    assert np.array_equal(res[0], whole)
