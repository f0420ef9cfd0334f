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
