"""Benchmark: FDK cone-beam reconstruction of a 1024^3 volume from 1024 projections of
1024 x 1024 pixels (uint16 counts -> FullLogNorm -> FDK ramp filter -> FDK backprojection),
FP32 and with BF16-stored filtered projections.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mr|reference] [--small]

One step = one full reconstruction of the block with the counts already in HBM. `value`
is voxel x projection updates per second (GUPS, whole job over all ranks), FP32 path.
`e2e` is the same metric through the public pipeline with pinned host buffers: the
uint16 counts go host->device and the float volume comes back every step.

Multi-GPU (torchrun): the 1024^3 volume is split into z-slabs, one per rank, each with the
detector-row window its voxels project onto (independent slabs, no data-path collective);
`scaling` is strong; the step time is the maximum over ranks.

`--impl reference` times the reference's own CPU FDK (FDKbp_single compiled from the
reference sources into oracle/_ref) on a bounded sample of the same workload with all
host threads, on rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "backprojection GUPS + projections/s, FP32 vs BF16-proj at <=1e-3 rel RMS vs FP64"
# DRAM bytes (read + write) of one k_fdk_staged<f32, exact> launch, measured with ncu on this
# workload (detector width -> bytes): 1024^3 547.23 GB + 6.27 GB, 256^3 69.9 MB + 41.8 MB
MEASURED_TRAFFIC = {1024: 553.50e9, 256: 111.7e6}


def workload(small: bool, c2: bool = False):
    if c2:
        # the plain FDK configuration: 720 projections over 360 deg on a 512 x 512 detector
        return dict(name="FDK 512^3 from 720 projections of 512x512", nu=512, nv=512, nproj=720, sod=300.0,
                    sdd=600.0, pitch=0.2, voxel=0.1, i0=50000.0)
    if small:
        return dict(name="FDK 256^3 from 256 projections of 256x256 (profiling case)", nu=256, nv=256, nproj=256,
                    sod=300.0, sdd=600.0, pitch=0.8, voxel=0.4, i0=50000.0)
    # precision form: the FDK cone-beam geometry of the 512^3 case scaled x2
    return dict(name="FDK 1024^3 from 1024 projections of 1024x1024", nu=1024, nv=1024, nproj=1024, sod=300.0,
                sdd=600.0, pitch=0.2, voxel=0.1, i0=50000.0)


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_inputs(w, seed, device):
    import torch

    from imagingsuite_b200 import phantom

    ells = phantom.ellipsoids(1000 + 4)
    fov = w["nu"] * w["voxel"]
    integ = phantom.cone_integrals_torch(ells, w["nproj"], w["nu"], w["nv"], w["sod"], w["sdd"], w["pitch"], fov,
                                         device)
    counts, flats, darks = phantom.counts_torch(integ, w["i0"], 2000 + 4 + seed, 10, 10)
    del integ
    torch.cuda.synchronize()
    return counts, flats, darks


def geometry_centres(w):
    """Piercing point and centre of rotation (pixels), off the pixel grid by fixed fractions as
    on a real scanner: with both exactly at the detector centre, voxel centres project exactly
    onto pixel boundaries at 0/90/180/270 degrees and the nearest-neighbour rule then depends
    on the last bit of the arithmetic."""
    return ((w["nu"] - 1) / 2.0 + 0.13, (w["nv"] - 1) / 2.0 - 0.21), (w["nu"] - 1) / 2.0 + 0.07


def make_config(w):
    from imagingsuite_b200 import modules as M

    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fSOD, pi.fSDD = w["sod"], w["sdd"]
    pi.fpPoint, pi.fCenter = geometry_centres(w)
    pi.fResolution = (w["pitch"], w["pitch"])
    pi.roi = pi.projection_roi = (0, 0, w["nu"], w["nv"])
    pi.nDims = (w["nu"], w["nv"], w["nproj"])
    cfg.MatrixInfo.fVoxelSize = (w["voxel"],) * 3
    cfg.MatrixInfo.nDims = (w["nu"], w["nu"], w["nv"])
    return cfg


def time_steps(fn, steps, warmup, stream, dist_ctx, events_kernel=None):
    """Warm up, then time exactly `steps` calls between barriers + synchronize; returns
    (max-over-ranks seconds, per-step kernel durations dict)."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    if dist_ctx:
        dist_ctx.barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(steps):
        fn()
    end.record(stream)
    torch.cuda.synchronize()
    # a bounded wait that expired inside a kernel leaves the device error word set (the
    # step's result would be incomplete): the run fails here instead of reporting it
    from imagingsuite_b200 import _lib as L

    L.check_device()
    if dist_ctx:
        dist_ctx.barrier()
    t = start.elapsed_time(end) / 1e3
    if dist_ctx:
        t = dist_ctx.max(t)
    return t


def kernel_time(fn, stream, reps=2):
    """Average device duration of one call of fn (CUDA events on `stream`)."""
    import torch

    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(reps):
        fn()
    e.record(stream)
    torch.cuda.synchronize()
    return s.elapsed_time(e) / 1e3 / reps


def per_kernel_ms(fn, top=20):
    """Device time per kernel name over one call of fn: the CUDA activity records of the torch
    profiler (not the timed numbers; the profiler adds overhead around launches)."""
    import torch
    from torch.profiler import ProfilerActivity, profile

    torch.cuda.synchronize()
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        fn()
        torch.cuda.synchronize()
    out = {}
    for e in prof.key_averages():
        us = getattr(e, "self_device_time_total", None)
        if us is None:
            us = getattr(e, "self_cuda_time_total", 0.0)
        if us <= 0:
            continue
        name = e.key.split("(")[0].replace("void ", "").strip()
        out[name] = out.get(name, 0.0) + us / 1e3
    return dict(sorted(out.items(), key=lambda kv: -kv[1])[:top])


def run_mr(args):
    import torch

    from imagingsuite_b200 import _lib as L
    from imagingsuite_b200 import pipeline

    world = int(os.environ.get("WORLD_SIZE", "1"))
    from imagingsuite_b200.distributed import DistContext

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    # the timing collectives (barrier, MAX of the step time) go over NCCL; MR_DIST_BACKEND=gloo
    # keeps them on the host (e.g. to exercise the slab path with several ranks per device)
    backend = os.environ.get("MR_DIST_BACKEND", "nccl")
    dctx = DistContext(backend, device=device if backend == "nccl" else None) if world > 1 else None
    rank = dctx.rank if dctx else 0
    w = workload(args.small, args.workload == "fdk-c2")
    nu, nv, nproj = w["nu"], w["nv"], w["nproj"]
    updates = float(nu) * nu * nv * nproj

    # every rank holds the same scan (one volume split across the ranks)
    counts, flats, darks = make_inputs(w, 0, device)
    cfg = make_config(w)
    angles = np.arange(nproj, dtype=np.float32) * np.float32(360.0 / nproj)
    weights = np.full(nproj, np.float32(1.0 / nproj), np.float32)
    pipe32 = pipeline.FdkPipeline(cfg, angles, weights, darks, flats, precision="fp32")
    if world > 1:
        return run_mr_slabs(args, w, dctx, pipe32, counts, local, rank, world, updates)
    pipe16 = pipeline.FdkPipeline(cfg, angles, weights, darks, flats, precision="bf16")
    pipeh = pipeline.FdkPipeline(cfg, angles, weights, darks, flats, precision="fp16")
    stream = torch.cuda.current_stream()

    sampler = ClockSampler(local)
    sampler.start()
    t32 = time_steps(lambda: pipe32.run_device(counts), args.steps, args.warmup, stream, dctx)
    clocks = sampler.stop()
    t16 = time_steps(lambda: pipe16.run_device(counts), args.steps, args.warmup, stream, dctx)
    th16 = time_steps(lambda: pipeh.run_device(counts), args.steps, args.warmup, stream, dctx)

    # dominant kernel (FDK backprojection) alone, on the launching stream
    fdk = pipe32.fdk
    filt = torch.empty((nproj, nv, nu), device=device)
    proj = pipe32._lognorm_into(counts)
    wgt, X, Y, Z, s2, sc, uni, box, _ = fdk._geo
    st = stream.cuda_stream
    L.check(L.lib().mr_fdk_filter(proj.data_ptr(), nu, nv, nproj, wgt.data_ptr(), s2, sc, L.MR_F32, filt.data_ptr(),
                                  None, st))
    vol = torch.empty((nv, nu, nu), device=device)

    def bp32():
        L.check(L.lib().mr_fdk_backproject(filt.data_ptr(), L.MR_F32, None, nu, nv, nproj, X.data_ptr(), Y.data_ptr(),
                                           Z.data_ptr(), uni, fdk._mask.data_ptr(), box[0], box[1], 0, vol.data_ptr(), st))

    tbp = kernel_time(bp32, stream)
    # slice serialisation (ReconEngine::Serialize's TIFF16 cast) of the whole volume on the device
    out16 = torch.empty((nv, nu, nu), dtype=torch.uint16, device=device)

    def ser():
        L.check(L.lib().mr_slices_u16(vol.data_ptr(), L.MR_PLANE_XY, nu, nu, nv, 0, nv, None, -0.001, 0.004,
                                      out16.data_ptr(), st))

    tser = kernel_time(ser, stream)
    del out16
    # precision form: 16-bit filtered projections through the FP64-derived maps
    *_, box16, maps = pipe16.fdk._geo
    q16 = torch.empty((nproj, nv, nu), dtype=torch.uint16, device=device)
    qs = torch.empty(nproj, device=device)
    vol16 = torch.empty((nv, nu, nu), device=device)
    tfast = {}
    for name, dt in (("bf16", L.MR_BF16), ("fp16", L.MR_F16)):
        L.check(L.lib().mr_quantize(filt.data_ptr(), nu * nv, nproj, dt, q16.data_ptr(), qs.data_ptr(), st))

        def bpf(dt=dt):
            L.check(L.lib().mr_fdk_backproject_fast(q16.data_ptr(), dt, qs.data_ptr(), nu, nv, nproj, maps.data_ptr(),
                                                    fdk._mask.data_ptr(), box16[0], box16[1], 0, vol16.data_ptr(), st))

        tfast[name] = kernel_time(bpf, stream)
    # FP64 error oracle on 16 seeded slices of the final volume
    rng = np.random.default_rng(16)
    sl_np = np.sort(rng.choice(nv, 16, replace=False)).astype(np.int32)
    sl = torch.from_numpy(sl_np).to(device)
    m64 = torch.from_numpy(pipe16.fdk.maps64(angles)).to(device)
    out64 = torch.empty((16, nu, nu), dtype=torch.float64, device=device)
    L.check(L.lib().mr_fdk_backproject_f64(filt.data_ptr(), nu, nv, nproj, m64.data_ptr(), fdk._mask.data_ptr(),
                                           sl.data_ptr(), 16, out64.data_ptr(), st))

    def errs(v):
        d = v.index_select(0, sl.long()).double() - out64
        return {"rel_rms_vs_fp64": float(torch.sqrt((d ** 2).mean() / (out64 ** 2).mean()).item()),
                "max_abs_vs_fp64": float(d.abs().max().item())}

    err32 = errs(vol)
    err16 = {}
    for name, dt in (("bf16", L.MR_BF16), ("fp16", L.MR_F16)):
        L.check(L.lib().mr_quantize(filt.data_ptr(), nu * nv, nproj, dt, q16.data_ptr(), qs.data_ptr(), st))
        L.check(L.lib().mr_fdk_backproject_fast(q16.data_ptr(), dt, qs.data_ptr(), nu, nv, nproj, maps.data_ptr(),
                                                fdk._mask.data_ptr(), box16[0], box16[1], 0, vol16.data_ptr(), st))
        err16[name] = errs(vol16)
        d = vol16.index_select(0, sl.long()).double() - vol.index_select(0, sl.long()).double()
        ref = vol.index_select(0, sl.long()).double()
        err16[name]["rel_rms_vs_fp32"] = float(torch.sqrt((d ** 2).mean() / (ref ** 2).mean()).item())
    vref_max = float(out64.abs().max().item())
    del filt, q16, vol16, vol, out64, m64

    # end to end through the pipeline with pinned host buffers
    counts_h = counts.cpu().pin_memory()
    out_h = torch.empty((nv, nu, nu), dtype=torch.float32).pin_memory()
    te2e = time_steps(lambda: pipe32.run_host(counts_h, out_h, device), max(1, min(args.steps, 3)), 1, stream, dctx)
    e2e_steps = max(1, min(args.steps, 3))

    res = None
    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except OSError:
            pass
        hbm = float(peaks.get("hbm_gbs", 6650.0))
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        # HBM: the compulsory bytes of one backprojection launch, the filtered projections read
        # once and the volume written once (4 B each)
        hbm_bytes = 4.0 * nproj * nu * nv + 4.0 * nu * nu * nv
        ach = hbm_bytes / tbp / 1e9
        # on chip: one 32-bit gather per voxel x projection update from the TMA-staged box, one
        # shared-memory wavefront per warp-update (32 updates) when conflict-free, against the
        # measured shared-memory wavefront rate of this GPU (mr_measure_smem)
        wf, smem_bytes = ctypes.c_double(), ctypes.c_double()
        L.check(L.lib().mr_measure_smem(ctypes.byref(wf), ctypes.byref(smem_bytes)))
        gather_wf = updates / 32.0 / tbp
        sm_mhz = clocks.get("sm_mhz") or float(peaks.get("sm_max_mhz", 1965.0))
        # issue: the reference-exact FP32 arithmetic takes 6 warp instructions per update (paired
        # a1 + x1 and dw * (...), two +0.5, paired floor, two address IMADs, two loads, paired
        # dw2 * v, two accumulating adds per two updates) plus the per-projection set-up (about
        # one more per update); 4 warp instructions per clock per SM
        issue_gups = 148 * 4 * sm_mhz * 1e6 * 32 / 7.0 / 1e9
        n = world
        res = {
            "metric": METRIC,
            "value": n * updates * args.steps / t32 / 1e9,
            "unit": "GUPS",
            "n_gpus": n,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": t32 / args.steps * 1e3,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded 10-ellipsoid phantom, analytic cone-beam line integrals, Poisson I0=5e4)",
            "config": {"workload": w["name"], "volume": [nu, nu, nv], "projections": nproj, "detector": [nu, nv],
                       "chain": "FullLogNorm(u16) -> FDK ramp filter -> FDK NN backprojection",
                       "l2": "inputs larger than L2 (2.1 GB counts per step)", "parallelism": f"z-slab x{n}"},
            "projections_per_s": n * nproj * args.steps / t32,
            "backprojection_gups": updates / tbp / 1e9,
            "serialize_u16": {"ms": tser * 1e3, "achieved_gbs": 6.0 * nu * nu * nv / tser / 1e9,
                              "frac_of_hbm": 6.0 * nu * nu * nv / tser / 1e9 / hbm,
                              "note": "mr_slices_u16: float volume -> uint16 slices (4 B read + 2 B written per voxel)"},
            "precision": {
                "fp64_oracle": f"FP64 geometry and accumulation on 16 seeded slices {sl_np.tolist()} of the final "
                               f"volume (max |value| {vref_max:.4g})",
                "fp32": dict(err32, backprojection_gups=updates / tbp / 1e9),
                "bf16": dict(err16["bf16"], value=n * updates * args.steps / t16 / 1e9, unit="GUPS",
                             ms_per_step=t16 / args.steps * 1e3, backprojection_gups=updates / tfast["bf16"] / 1e9),
                "fp16": dict(err16["fp16"], value=n * updates * args.steps / th16 / 1e9, unit="GUPS",
                             ms_per_step=th16 / args.steps * 1e3, backprojection_gups=updates / tfast["fp16"] / 1e9),
            },
            "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                         "traffic": MEASURED_TRAFFIC.get(nu), "kernel": "k_fdk_staged<f32, exact>",
                         "note": f"algorithmic bytes = the compulsory HBM bytes of one launch (filtered projections "
                                 f"read once + volume written once, {hbm_bytes / 1e9:.2f} GB); peak {peak_src}; "
                                 f"traffic = dram__bytes_read.sum + dram__bytes_write.sum of one launch (ncu, "
                                 f"profiles/k_fdk_staged_fdk256_fdk1024.md). The samples are gathered from shared "
                                 f"memory (TMA-staged), so HBM is not this kernel's bound: see onchip and issue"},
            "onchip": {"bound": "shared-memory wavefronts", "achieved": gather_wf / 1e9, "peak": wf.value / 1e9,
                       "unit": "G wavefronts/s", "frac": gather_wf / wf.value,
                       "gathered_gbs": 4.0 * updates / tbp / 1e9, "peak_gbs": smem_bytes.value / 1e9,
                       "note": "algorithmic: one 32-bit gather per update, one wavefront per 32 updates; peak "
                               "measured on this GPU by mr_measure_smem (conflict-free loads)"},
            "issue": {"bound": "warp-instruction issue", "achieved_gups": updates / tbp / 1e9,
                      "roofline_gups": issue_gups, "frac": updates / tbp / 1e9 / issue_gups,
                      "note": "7 warp instructions per update for the reference-exact FP32 arithmetic, 4 issued per "
                              "clock per SM, 148 SMs at the SM clock sampled during the run"},
            "e2e": {"value": n * updates * e2e_steps / te2e / 1e9, "unit": "GUPS",
                    "h2d_bytes_per_step": int(counts.numel() * 2), "d2h_bytes_per_step": int(nu * nu * nv * 4)},
            "gpu_launches": 3 * args.steps,
            "clocks": clocks,
        }
        if world == 1 and not args.no_cpu_baseline:
            res["cpu_baseline"] = cpu_baseline(w, counts, pipe32, angles, weights, cfg, device, budget_s=args.cpu_budget)
    if dctx:
        dctx.barrier()
        dctx.close()
    return res


def run_mr_slabs(args, w, dctx, pipe, counts, local, rank, world, updates):
    """N > 1: one 1024^3 volume split into z-slabs (distributed.cone_slab_plan), each rank
    normalising, filtering and backprojecting only its slab's detector-row window; no data-path
    collective. `value` is the whole volume's updates over the slowest rank's time (strong
    scaling); e2e copies each rank's row window in and its slab out."""
    import torch

    nu, nv, nproj = w["nu"], w["nv"], w["nproj"]
    device = counts.device
    plan = pipe.slab_plan(world)
    s = plan[rank]
    rows = counts[:, s.row_start:s.row_stop].contiguous()
    stream = torch.cuda.current_stream()
    sampler = ClockSampler(local)
    sampler.start()
    t = time_steps(lambda: pipe.run_slab(rows, s), args.steps, args.warmup, stream, dctx)
    clocks = sampler.stop()
    rows_h = rows.cpu().pin_memory()
    out_h = torch.empty((s.size, nu, nu), dtype=torch.float32).pin_memory()

    def e2e():
        r = rows_h.to(device, non_blocking=True)
        vol = pipe.run_slab(r, s)
        out_h.copy_(vol[s.start:s.stop], non_blocking=True)

    e2e_steps = max(1, min(args.steps, 3))
    te = time_steps(e2e, e2e_steps, 1, stream, dctx)
    h2d = dctx.max(float(rows.numel() * 2))
    d2h = dctx.max(float(s.size * nu * nu * 4))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    hbm_bytes = 2.0 * rows.numel() + 2 * 4.0 * rows.numel() + 4.0 * rows.numel() + 4.0 * s.size * nu * nu
    res = None
    if rank == 0:
        res = {"metric": METRIC, "value": updates * args.steps / t / 1e9, "unit": "GUPS", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3,
               "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic (seeded 10-ellipsoid phantom, analytic cone-beam line integrals, Poisson I0=5e4)",
               "config": {"workload": w["name"], "volume": [nu, nu, nv], "projections": nproj,
                          "chain": "FullLogNorm(u16) -> FDK ramp filter -> FDK NN backprojection, per z-slab",
                          "parallelism": f"z-slab x{world}",
                          "slabs": [[p.start, p.stop, p.row_start, p.row_stop] for p in plan],
                          "l2": "inputs larger than L2"},
               "e2e": {"value": updates * e2e_steps / te / 1e9, "unit": "GUPS",
                       "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                       "note": "per rank (largest over ranks): its row window in, its slab out"},
               "roofline": {"bound": "hbm", "achieved": hbm_bytes / (t / args.steps) / 1e9, "peak": hbm,
                            "unit": "GB/s", "frac": hbm_bytes / (t / args.steps) / 1e9 / hbm, "traffic": None,
                            "kernel": "slab step (FullLogNorm + FDK filter of the row window, k_fdk_staged)",
                            "note": "rank 0's compulsory HBM bytes per step: counts window read, filtered window "
                                    "written and read, slab written; the backprojection is bound by issue (N=1 line)"},
               "gpu_launches": 4 * args.steps, "clocks": clocks}
    dctx.barrier()
    dctx.close()
    return res


def _diff_pair(op, truth, c_true, t_true, nproj, stream, dev):
    """One projector pair on the C5 workload: forward / adjoint times, dot-product test, and the
    refinement (centroid estimate, FBP start, 50 CGLS iterations with joint centre/tilt)."""
    import torch

    from imagingsuite_b200 import joseph as J

    p = op.forward(truth, c_true, t_true)
    tf = kernel_time(lambda: op.forward(truth, c_true, t_true), stream, reps=3)
    y = p.clone()
    ta = kernel_time(lambda: op.adjoint(y, c_true, t_true), stream, reps=3)
    ta0 = kernel_time(lambda: op.adjoint(y, c_true, 0.0), stream, reps=3)
    g = torch.Generator(device=dev).manual_seed(5)
    xr = torch.randn(truth.shape, device=dev, generator=g)
    yr = torch.randn(p.shape, device=dev, generator=g)
    lhs = float(torch.dot(op.forward(xr, c_true, t_true).reshape(-1).double(), yr.reshape(-1).double()))
    rhs = float(torch.dot(xr.reshape(-1).double(), op.adjoint(yr, c_true, t_true).reshape(-1).double()))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    c0, tl0 = J.estimate_geometry(op, p)
    x0 = J.fbp(op, p, c0, tl0)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    x, c, tl, hist = J.cgls(op, p, x0, c0, tl0, iterations=50, refine_every=5)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    rel = lambda v: float(torch.linalg.vector_norm(v - truth) / torch.linalg.vector_norm(truth))
    upd = float(truth.numel()) * nproj
    return {"forward_gups": upd / tf / 1e9, "adjoint_gups": upd / ta / 1e9, "adjoint_gups_no_tilt": upd / ta0 / 1e9,
            "forward_ms": tf * 1e3, "adjoint_ms": ta * 1e3, "adjoint_ms_no_tilt": ta0 * 1e3,
            "dot_test_rel": abs(lhs - rhs) / abs(lhs),
            "estimate": {"centre": c0, "tilt_deg": tl0, "seconds": t1 - t0, "method": "sinogram centroid fit"},
            "cgls": {"iterations": len(hist), "seconds": t2 - t1, "centre": c, "tilt_deg": tl,
                     "centre_error": c - c_true, "tilt_error_deg": tl - t_true, "loss_first": hist[0],
                     "loss_last": hist[-1], "volume_rel_error_fbp": rel(x0), "volume_rel_error_cgls": rel(x)}}


def run_diff(args):
    """Differentiation form on a 512 x 512 x 128 volume, 360 projections over 180 degrees of 512
    bins; data simulated at centre offset +3.7 bins and tilt 0.4 degrees; coarse centre/tilt
    estimate, FBP start, 50 CGLS iterations with joint refinement. Two pairs: the one matched to
    the backprojector (A^T = MultiProjectionBPparallel's backprojection, A its exact transpose;
    `value`), and the Joseph pair (A = LinearForwardProjector's projector, A^T its transpose)."""
    import torch

    from imagingsuite_b200 import joseph as J
    from imagingsuite_b200 import phantom

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    n, nz, nu, nproj = (128, 32, 128, 90) if args.small else (512, 128, 512, 360)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    truth = phantom.voxelize_torch(phantom.ellipsoids(1005), n, nz, dev, fov_margin=8)  # (nz, n, n)
    c_true, t_true = nu / 2 + 3.7, 0.4
    stream = torch.cuda.current_stream()
    updates = float(n) * n * nz * nproj
    matched = _diff_pair(J.MatchedOperator(n, nz, ang), truth.permute(1, 2, 0).contiguous(), c_true, t_true, nproj,
                         stream, dev)
    joseph = _diff_pair(J.JosephOperator(n, nz, ang, nu), truth, c_true, t_true, nproj, stream, dev)
    res = {"metric": "differentiable projector pair GUPS (voxel x projection, forward) and 50-iteration CGLS with "
                     "centre/tilt refinement",
           "value": matched["forward_gups"], "unit": "GUPS", "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
           "data": "synthetic (voxelised 10-ellipsoid phantom inside the field of view, projected at the true geometry "
                   "by the same pair)",
           "config": {"workload": f"volume {n}x{n}x{nz}, {nproj} projections of {nu} bins over 180 deg",
                      "true_centre": c_true, "true_tilt_deg": t_true},
           "matched_to_backprojector": matched, "joseph": joseph}
    res.update({k: matched[k] for k in ("forward_gups", "adjoint_gups", "dot_test_rel")})
    return res


def parallel_inputs(production: bool, small: bool, dev):
    """Seeded inputs of the parallel-beam workloads (C1, or the C3 block) and their
    configuration: uint16 counts (nproj, nrows, nu), flats, darks on `dev`."""
    from imagingsuite_b200 import modules as M
    from imagingsuite_b200 import phantom

    if production:
        nu, nrows, nproj, nflat, ndark, i0 = 2048, 512, 1125, 20, 10, 3e4
        if small:
            nu, nrows, nproj = 512, 128, 282
        name = f"C3 production block: {nproj} projections of {nu} x {nu} (block of {nrows} rows), spots + rings"
    else:
        nu, nrows, nproj, nflat, ndark, i0 = 256, 64, 360, 5, 5, 3e4
        name = f"C1 parallel FBP: {nproj} projections of {nu} x {nrows} -> {nu}x{nu}x{nrows}"
    ells = phantom.ellipsoids(1000 + (3 if production else 1))
    v0 = (nu - nrows) // 2 if production else 0
    integ = phantom.parallel_integrals_torch(ells, nproj, nu, nrows, dev, box=float(nu) if production else None,
                                             v0=v0)
    counts, flats, darks = phantom.counts_torch(integ, i0, 2000 + (3 if production else 1), nflat, ndark)
    del integ
    if production:
        phantom.inject_defects_torch(counts, flats, 3003)
    cfg = M.ReconConfig()
    pi = cfg.ProjectionInfo
    pi.fCenter = (nu - 1) / 2.0
    pi.roi = pi.projection_roi = (0, 0, nu, nrows)
    pi.nDims = (nu, nrows, nproj)
    pi.nOBCount, pi.nDCCount = nflat, ndark
    return {"nu": nu, "nrows": nrows, "nproj": nproj, "name": name, "counts": counts, "flats": flats, "darks": darks,
            "cfg": cfg, "angles": (np.arange(nproj) * 180.0 / nproj).astype(np.float32),
            "weights": np.full(nproj, np.float32(np.pi / nproj))}


_SPOT_PARAMS = dict(connectivity="conn8", detectionmethod="morphdetectboth", threshold="0.1 0.1", sigma="0.01 0.01",
                    edgesmooth=5, maxarea=30, removeinfnan=False, clampdata=False, minlevel=-0.1, maxlevel=12.0)


def module_hbm(times: dict, px: float, hbm_gbs: float, production: bool) -> dict:
    """Each preprocessing module's compulsory HBM traffic over its measured time: the block read
    and written once (FullLogNorm: 2 B of uint16 counts in, 4 B out per pixel; the in-place
    cleaners and the filter: 4 B in, 4 B out), against the measured copy bandwidth."""
    bpp = {"lognorm": 6.0, "filter": 8.0}
    if production:
        bpp.update({"spotclean": 8.0, "ringclean": 8.0})
    out = {}
    for name, b in bpp.items():
        ms = times.get(name)
        if not ms:
            continue
        gbs = b * px / (ms / 1e3) / 1e9
        out[name] = {"ms": ms, "bytes_per_px": b, "achieved_gbs": gbs, "frac": gbs / hbm_gbs}
    return out


def chain_cpu(P, production: bool, updates: float, sel: int):
    """The reference's own modules (compiled from the reference sources, `oracle/_ref`) chained
    on the host cores with all threads: FullLogNorm -> [MorphSpotCleanModule ->
    WaveletRingClean] -> ProjectionFilterSingle -> MultiProjBPparallel.

    C1: the whole workload. C3: the preprocessing modules on a sample of projections of the
    block (per-projection cost), the backprojector into the full 2048 x 2048 x 512 volume with
    4 and 36 projections (per-projection cost from the difference, fixed cost apart), scaled to
    the block's projections. Returns the cpu_baseline object; value in the workload's GUPS.
    The FFT-based modules (the filter, the ring cleaner) call FFTW through the oracle's FFTW-API
    shim (FP64 radix-2), slower than FFTW itself: their share of the CPU time is an upper bound."""
    import oracle

    cores = os.cpu_count() or 1
    threads = os.environ.get("OMP_NUM_THREADS", str(cores))
    if not oracle.ref_available():
        return {"kind": "reference", "cores": 0, "value": None, "unit": "GUPS",
                "sample": "reference library oracle/_ref/libmuhrec_ref.so not built"}
    nu, nrows, nproj = P["nu"], P["nrows"], P["nproj"]
    centre = P["cfg"].ProjectionInfo.fCenter
    darks = P["darks"].cpu().numpy()
    flats = P["flats"].cpu().numpy()
    ang, wts = P["angles"], P["weights"]
    if not production:
        c = P["counts"].cpu().numpy().astype(np.float32)
        t = {}
        t0 = time.perf_counter()
        p = oracle.ref_fulllognorm(c, darks, flats, "ImageAverage", False)[0]
        t["FullLogNorm"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        p = oracle.ref_projfilter(p, "hanning", 0.5, 1.0, True, 0.1, 2)[0]
        t["ProjectionFilterSingle"] = time.perf_counter() - t0
        t0 = time.perf_counter()
        oracle.bp_parallel(p, ang, wts, centre, buffersize=16, use_ref=True)
        t["MultiProjBPparallel"] = time.perf_counter() - t0
        total = sum(t.values())
        return {"kind": "reference", "cores": cores, "value": updates / total / 1e9, "unit": "GUPS",
                "sample": f"the whole C1 workload through the reference modules (OMP_NUM_THREADS={threads})",
                "module_s": t, "total_s": total}
    k = 64  # projections through the preprocessing modules (the ring cleaner needs sinograms this tall)
    c = P["counts"][:k].cpu().numpy().astype(np.float32)
    per = {}
    t0 = time.perf_counter()
    p = oracle.ref_fulllognorm(c, darks, flats, "ImageAverage", False)[0]
    per["FullLogNorm"] = (time.perf_counter() - t0) / k
    t0 = time.perf_counter()
    p = oracle.ref_morphspotclean_module(p, **_SPOT_PARAMS, threading=True)
    per["MorphSpotCleanModule"] = (time.perf_counter() - t0) / k
    t0 = time.perf_counter()
    p = oracle.waveletringclean(p, "daub15", 2, 0.05, use_ref=True)
    per["WaveletRingClean"] = (time.perf_counter() - t0) / k
    t0 = time.perf_counter()
    p = oracle.ref_projfilter(p, "hanning", 0.5, 1.0, True, 0.1, 2)[0]
    per["ProjectionFilterSingle"] = (time.perf_counter() - t0) / k
    # the first call maps the volume's pages; the per-projection cost is the difference of two
    # later calls far enough apart that it stands clear of the fixed cost's variation
    n1, n2 = 4, 36
    oracle.bp_parallel(p[:1], ang[:1], wts[:1], centre, buffersize=16, use_ref=True)
    t0 = time.perf_counter()
    oracle.bp_parallel(p[:n1], ang[:n1], wts[:n1], centre, buffersize=16, use_ref=True)
    t1 = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.bp_parallel(p[:n2], ang[:n2], wts[:n2], centre, buffersize=16, use_ref=True)
    t2 = time.perf_counter() - t0
    per["MultiProjBPparallel"] = (t2 - t1) / (n2 - n1)
    fixed = max(t1 - n1 * per["MultiProjBPparallel"], 0.0)
    total = sum(v * nproj for k_, v in per.items() if k_ != "MultiProjBPparallel") + \
        per["MultiProjBPparallel"] * sel + fixed
    return {"kind": "reference", "cores": cores, "value": updates / total / 1e9, "unit": "GUPS",
            "sample": f"preprocessing modules on {k} projections of the block, the backprojector into the full "
                      f"{nu}x{nu}x{nrows} volume with {n1} and {n2} projections (per projection from the "
                      f"difference), scaled to {nproj} projections ({sel} backprojected); "
                      f"OMP_NUM_THREADS={threads}",
            "s_per_projection": per, "bp_fixed_s": fixed, "estimated_block_s": total}


def run_parallel(args, production: bool):
    """Parallel-beam chains. C1 (production=False): 360 projections of 256 x 64 over 180 deg,
    I0 3e4, 5 flats / 5 darks, FullLogNorm -> Hann ramp filter (cutoff 0.5) -> backprojection to
    256 x 256 x 64, centre 127.5. C3 (production=True): 1125 projections of 2048 x 2048 over 180
    deg, 20 flats / 10 darks, 0.05 % spot defects and 20 gain-error columns; one block of 512
    detector rows (the slab the reference reconstructs per SliceBlock) through FullLogNorm ->
    MorphSpotClean -> WaveletRingClean -> Hann filter -> backprojection to 2048 x 2048 x 512."""
    import torch

    from imagingsuite_b200 import modules as M
    from imagingsuite_b200 import pipeline

    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    P = parallel_inputs(production, args.small, dev)
    nu, nrows, nproj, name = P["nu"], P["nrows"], P["nproj"], P["name"]
    counts, flats, darks, cfg = P["counts"], P["flats"], P["darks"], P["cfg"]
    angles, weights = P["angles"], P["weights"]
    norm = M.FullLogNorm()
    norm.Configure(cfg, {"usenormregion": "false", "uselut": "false", "referenceaverage": "ImageAverage"})
    norm.SetReferenceImages(darks, flats)
    spot = M.MorphSpotCleanModule()
    spot.Configure(cfg, {"connectivity": "conn8", "cleanmethod": "morphcleanreplace",
                         "detectionmethod": "morphdetectboth", "threshold": "0.1 0.1", "sigma": "0.01 0.01",
                         "edgesmooth": "5", "maxarea": "30", "removeinfnan": "false", "clampdata": "false",
                         "minlevel": "-0.1", "maxlevel": "12", "threading": "false"})
    ring = M.WaveletRingClean()
    ring.Configure(cfg, {"wname": "daub15", "sigma": "0.05", "decnum": "2", "parallel": "false",
                         "method": "verticalfft"})
    filt = M.ProjectionFilterSingle()
    filt.Configure(cfg, {"filtertype": "hanning", "cutoff": "0.5", "order": "1", "usebias": "true",
                         "biasweight": "0.1", "paddingdoubler": "2"})
    bp = M.MultiProjectionBPparallel()
    bp.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1", "precision": "fp32",
                       "referencecompat": "true"})
    bp.SetROI((0, 0, nu, nrows))
    params = {"angles": " ".join("%.9g" % a for a in angles), "weights": " ".join("%.9g" % a for a in weights)}
    wdev = torch.from_numpy(weights).to(dev)
    stream = torch.cuda.current_stream()
    times = {}

    def step(record=False):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(6)] if record else None
        if record:
            ev[0].record(stream)
        bp.volume.zero_()
        proj = norm.ProcessCore(counts, {})
        if record:
            ev[1].record(stream)
        if production:
            spot.ProcessCore(proj, {})
        if record:
            ev[2].record(stream)
        if production:
            ring.ProcessCore(proj, {})
        if record:
            ev[3].record(stream)
        filt.ProcessCore(proj, {}, weights=wdev)
        if record:
            ev[4].record(stream)
        bp.Process(proj, params, prefiltered_weights=True)
        if record:
            ev[5].record(stream)
            torch.cuda.synchronize()
            for k, nm in enumerate(("lognorm", "spotclean", "ringclean", "filter", "backprojection")):
                times[nm] = ev[k].elapsed_time(ev[k + 1])
        return bp.GetVolume()

    sampler = ClockSampler(0)
    sampler.start()
    t = time_steps(step, args.steps, args.warmup, stream, None)
    clocks = sampler.stop()
    step(record=True)
    kernels = per_kernel_ms(lambda: step()) if args.kernel_times else None
    alt = None
    if production:
        # the alternative cleaners a configuration can name instead of MorphSpotClean or
        # WaveletRingClean, each timed alone on the normalised block (in place, CUDA events on
        # the launching stream)
        blk = norm.ProcessCore(counts, {})
        sample = None if args.no_cpu_baseline else blk[:16].cpu().numpy()
        basic, mix = M.BasicRingClean(), M.MedianMixRingClean()
        mix.Configure(cfg, {"threshold": "0.025", "width": "0.0025"})
        spot2 = M.SpotClean2()
        spot2.Configure(cfg, {"gamma": "0.1", "sigma": "0.001", "iterations": "1", "maxlevel": "5", "minlevel": "-0.1",
                              "maxarea": "20", "detectionmethod": "ring"})
        px = float(blk.numel())
        ts = kernel_time(lambda: spot2.ProcessCore(blk, {}), stream, reps=1)
        tb = kernel_time(lambda: basic.ProcessCore(blk, {}), stream)
        tm = kernel_time(lambda: mix.ProcessCore(blk, {}), stream)
        alt = {"block": [nproj, nrows, nu],
               "basicringclean_ms": tb * 1e3, "basicringclean_gbs": 12.0 * px / tb / 1e9,
               "medianmixringclean_ms": tm * 1e3, "medianmixringclean_gbs": 12.0 * px / tm / 1e9,
               "medianmixringclean_gpx_s": px / tm / 1e9,
               "spotclean2_ms": ts * 1e3, "spotclean2_gpx_s": px / ts / 1e9,
               "spotclean2_config": "ring detection, gamma 0.1, sigma 0.001, maxarea 20, levels [-0.1, 5]",
               "note": "algorithmic bytes 12 B/px for both: BasicRingClean reads the block for the mean, then "
                       "reads and writes it; MedianMixRingClean reads it for the mean, then reads it for the 5x5 "
                       "median and writes the mixed value"}
        if sample is not None:
            alt["cpu_baseline"] = alt_cleaners_cpu(sample)
        del blk
    sel = bp.used_projections(nproj).size
    updates = float(nu) * nu * (4 * (nrows // 4)) * sel
    # end to end: host counts in, host volume out
    counts_h = counts.cpu().pin_memory()
    out_h = torch.empty(bp.volume.shape, dtype=torch.float32).pin_memory()

    chain = pipeline.ParallelChain(norm, filt, bp, angles, weights, spot=spot if production else None,
                                   ring=ring if production else None)

    def e2e_step():
        chain.run_host(counts_h, out_h, dev)

    te = time_steps(e2e_step, max(1, min(args.steps, 3)), 1, stream, None)
    e2e_steps = max(1, min(args.steps, 3))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    tbp = times["backprojection"] / 1e3
    ach = 8.0 * updates / tbp / 1e9
    # shared-memory load wavefronts of the staged backprojector: two per warp and update (the
    # two samples of the linear interpolation, consecutive x in a warp: no bank conflicts),
    # counted for the warps that have a voxel inside the circle mask
    m = bp._mask.cpu().numpy().view(np.uint32).reshape(-1, 2).astype(np.int64)
    warps = 0
    for first, second in m:
        lo, hi = first + 1, second  # 1-based x inside: first < x <= second
        if hi >= lo:
            warps += (hi - 1) // 32 - (lo - 1) // 32 + 1
    wavefronts = 2.0 * warps * ((nrows // 4) * 4) * sel
    sm_mhz = clocks.get("sm_mhz") or float(peaks.get("sm_max_mhz", 1965.0))
    from imagingsuite_b200 import _lib as L

    wfm, _bytes = ctypes.c_double(), ctypes.c_double()
    L.check(L.lib().mr_measure_smem(ctypes.byref(wfm), ctypes.byref(_bytes)))
    wf_peak = wfm.value
    cpu = None if args.no_cpu_baseline else chain_cpu(P, production, updates, sel)
    return {"metric": "parallel-beam chain GUPS (voxel x projection updates per second)",
            "value": updates * args.steps / t / 1e9, "unit": "GUPS", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded 10-ellipsoid phantom, analytic parallel-beam "
                                                        "line integrals, Poisson counts" + (", injected spots and ring columns)" if production else ")"),
            "config": {"workload": name, "volume": [nu, nu, nrows], "projections": nproj,
                       "projections_backprojected": sel, "l2": "inputs larger than L2" if production else "inputs fit L2"},
            "projections_per_s": nproj * args.steps / t,
            "module_ms": times,
            **({"kernel_ms": kernels} if kernels else {}),
            "module_hbm": module_hbm(times, float(nu) * nrows * nproj, hbm, production),
            **({"alt_ring_cleaners": alt} if alt else {}),
            "backprojection_gups": updates / tbp / 1e9,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm,
                         "traffic": None, "kernel": "k_bp_par_staged",
                         "note": "algorithmic bytes = 8 B/update gathered (two FP32 samples) vs measured HBM copy "
                                 "bandwidth (of measured); the gathers are served from shared memory (TMA-staged), "
                                 "so the binding roofline is the on-chip one below"},
            "onchip": {"bound": "shared-memory load wavefronts", "achieved": wavefronts / tbp / 1e9,
                       "peak": wf_peak / 1e9, "unit": "G wavefronts/s", "frac": wavefronts / tbp / wf_peak,
                       "peak_source": "measured on this GPU by mr_measure_smem (conflict-free 32-bit shared loads)"},
            "e2e": {"value": updates * e2e_steps / te / 1e9, "unit": "GUPS",
                    "h2d_bytes_per_step": int(counts.numel() * 2), "d2h_bytes_per_step": int(bp.volume.numel() * 4)},
            **({"cpu_baseline": cpu} if cpu else {}),
            "clocks": clocks}


def alt_cleaners_cpu(sample):
    """The reference's BasicRingClean, MedianMixRingClean and SpotClean2 (compiled from the
    reference sources) on a sample of normalised projections, all host threads."""
    import oracle

    cores = os.cpu_count() or 1
    if not oracle.ref_available():
        return {"kind": "reference", "cores": 0, "sample": "reference library absent"}
    n, h, w = sample.shape
    t0 = time.perf_counter()
    oracle.basicringclean(sample, use_ref=True)
    tb = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.medianmixringclean(sample, use_ref=True)
    tm = time.perf_counter() - t0
    t0 = time.perf_counter()
    oracle.spotclean2(sample, "ring", 0.1, 0.001, 1, -0.1, 5.0, 20, use_ref=True)
    ts = time.perf_counter() - t0
    return {"kind": "reference", "cores": cores,
            "sample": f"{n} normalised projections of {w} x {h} (OMP_NUM_THREADS="
                      f"{os.environ.get('OMP_NUM_THREADS', cores)})",
            "basicringclean_ms_per_projection": tb / n * 1e3, "medianmixringclean_ms_per_projection": tm / n * 1e3,
            "spotclean2_ms_per_projection": ts / n * 1e3}


def _ref_geom(w):
    import oracle

    pp, centre = geometry_centres(w)
    return oracle.fdk_geom(w["sod"], w["sdd"], pp, centre, (w["pitch"],) * 2, (w["voxel"],) * 3)


def _timed(fn):
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


def _ref_rate(w, setup_s, t_small, n_small, t_big, n_big):
    """Per-projection (marginal) cost of the reference from two Process sizes, its fixed cost
    per Process call (the final mirror of the volume), and the whole workload's rate: the
    block's set-up, one Process call and nproj times the marginal cost."""
    nu, nv, nproj = w["nu"], w["nv"], w["nproj"]
    marginal = (t_big - t_small) / (n_big - n_small)
    fixed = max(t_small - n_small * marginal, 0.0)
    full = setup_s + fixed + nproj * marginal
    return {"marginal_s_per_projection": marginal, "fixed_s_per_process_call": fixed, "setup_s": setup_s,
            "full_workload_s": full, "gups": float(nu) * nu * nv * nproj / full / 1e9,
            "measured": [{"projections": n_small, "s": t_small}, {"projections": n_big, "s": t_big}]}


def cpu_baseline(w, counts, pipe, angles, weights, cfg, device, budget_s=20.0):
    """The reference FDKbp_single (compiled from the reference sources) on the box's host
    cores, all threads, configured once for the full 1024^3 block and then given 1 and 1+n of
    this workload's normalised projections by two Process calls (n sized to the budget). The
    rate comes from the difference of the two calls (per projection) plus the measured fixed
    costs, scaled to the workload's projections. The volume the reference accumulates from
    those 1+n projections is also compared with the CUDA path's FDKbp_single on the same
    projections: parity at the full detector and volume size."""
    import torch

    import oracle
    from imagingsuite_b200 import modules as M

    if not oracle.ref_available():
        return {"value": None, "unit": "GUPS", "cores": 0, "kind": "reference", "sample": "reference library absent"}
    nu, nv, nproj = w["nu"], w["nv"], w["nproj"]
    cores = os.cpu_count() or 1
    g = _ref_geom(w)
    sess = None
    sess_box = []
    setup = _timed(lambda: sess_box.append(oracle.RefFdkSession(nu, nv, nproj, g)))
    sess = sess_box[0]
    pick = np.linspace(0, nproj, 17, endpoint=False).astype(np.int64)  # spread over the arc
    sub = torch.stack([counts[int(i)] for i in pick])  # (uint16 tensors take no index lists)
    proj = pipe._lognorm_into(sub, out=torch.empty(sub.shape, dtype=torch.float32, device=device)).cpu().numpy()
    a, wt = angles[pick], weights[pick]
    t1 = _timed(lambda: sess.process(proj[:1], a[:1], wt[:1]))
    n = max(2, min(16, int((budget_s - setup - t1) / max(t1, 1e-3))))
    tn = _timed(lambda: sess.process(proj[1:1 + n], a[1:1 + n], wt[1:1 + n]))
    rate = _ref_rate(w, setup, t1, 1, tn, n)
    ref_vol = sess.volume()
    sess.close()
    # the same 1+n projections through the CUDA path's module
    fdk = M.FDKbp_single()
    fdk.Configure(cfg, {"ProjectionBufferSize": "16", "SliceBlock": "32", "SubVolume": "1 1"})
    fdk.SetROI((0, 0, nu, nv))
    text = lambda v: " ".join("%.9g" % x for x in v)
    fdk.Process(torch.from_numpy(proj[:1 + n]).to(device), {"angles": text(a[:1 + n]), "weights": text(wt[:1 + n])})
    got = fdk.GetVolume()
    ref_t = torch.from_numpy(ref_vol).to(device)
    d = got.double() - ref_t.double()
    parity = {"rel_rms": float(torch.sqrt((d ** 2).mean() / (ref_t.double() ** 2).mean()).item()),
              "max_abs": float(d.abs().max().item()), "max_ref": float(ref_t.abs().max().item()),
              "projections": 1 + n,
              "note": "CUDA FDKbp_single vs the reference FDKbp_single on the same normalised projections, whole "
                      f"{nu}x{nu}x{nv} volume (differences: FP32 FFT vs the FP64 FFT of the reference build)"}
    del got, ref_t, d, fdk
    torch.cuda.empty_cache()
    return {"value": rate["gups"], "unit": "GUPS", "cores": cores, "kind": "reference",
            "sample": f"reference FDKbp_single, {nu}x{nu}x{nv} volume set up once ({setup:.1f} s), Process of 1 "
                      f"projection ({t1:.2f} s) and of {n} ({tn:.2f} s): {rate['marginal_s_per_projection']:.3f} s per "
                      f"projection; value = {nu * nu * nv * nproj:.3g} updates / (set-up + fixed + {nproj} x "
                      f"per projection) (OMP_NUM_THREADS={os.environ.get('OMP_NUM_THREADS', cores)})",
            "rate": rate, "parity_vs_reference": parity}


def run_reference(args):
    """--impl reference: the reference's own CPU FDK on the host cores, rank 0 only. The
    reference FDKbp_single is configured once for the full block (Configure + SetROI, timed as
    set-up), warm-up steps give it 1 and 2 projections per Process call and every timed step n
    projections (n sized so a step takes about 8 s). The per-projection cost is the difference
    of the two call sizes; `value` is the whole workload's rate: set-up + one call's fixed cost
    + nproj x the per-projection cost."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and rank != 0:
        return None
    import oracle

    w = workload(args.small, args.workload == "fdk-c2")
    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "reference library oracle/_ref/libmuhrec_ref.so not built"}
    nu, nv, nproj = w["nu"], w["nv"], w["nproj"]
    rng = np.random.default_rng(0)
    g = _ref_geom(w)
    box = []
    setup = _timed(lambda: box.append(oracle.RefFdkSession(nu, nv, nproj, g)))
    sess = box[0]
    nmax = 32
    proj = (rng.standard_normal((nmax, nv, nu)) * 0.05).astype(np.float32)
    angles = np.arange(nmax, dtype=np.float32) * np.float32(360.0 / nproj)
    weights = np.full(nmax, np.float32(1.0 / nproj))
    call = lambda k: _timed(lambda: sess.process(proj[:k], angles[:k], weights[:k]))
    small = [call(1)]
    t2 = call(2)
    for _ in range(max(args.warmup - 2, 0)):
        small.append(call(1))
    t1 = float(np.median(small))
    n = int(max(3, min(nmax, round(8.0 / max(t2 - t1, 1e-3)))))
    times = [call(n) for _ in range(args.steps)]
    sess.close()
    tn = float(np.median(times))
    rate = _ref_rate(w, setup, t1, 1, tn, n)
    cores = os.cpu_count() or 1
    v = rate["gups"]
    sample = (f"reference FDKbp_single on {cores} host threads, {nu}x{nu}x{nv} volume set up once ({setup:.1f} s); "
              f"Process of 1 projection {t1:.2f} s (median of {len(small)}), of {n} projections {tn:.2f} s (median "
              f"of {args.steps} timed steps): {rate['marginal_s_per_projection']:.3f} s per projection; value = "
              f"{nu * nu * nv * nproj:.3g} updates / (set-up + fixed + {nproj} x per projection)")
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(times)) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w["name"], "projections_per_timed_step": n,
                       "step": "one FdkReconBase::Process 3D call of n projections into the configured volume"},
            "rate": rate,
            "cpu_baseline": {"value": v, "unit": "GUPS", "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_chain(args, production: bool):
    """Reference arm of the parallel-beam workloads: the reference's modules chained on the
    host cores (chain_cpu) on this workload's inputs; rank 0 only under torchrun."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and int(os.environ.get("RANK", "0")) != 0:
        return None
    import torch

    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    P = parallel_inputs(production, args.small, dev)
    nu, nrows, nproj = P["nu"], P["nrows"], P["nproj"]
    k = np.arange(nproj)
    sel = int(((k % 16) != 15).sum())  # StdBackProjectorBase drops the last entry of every full buffer of 16
    updates = float(nu) * nu * (4 * (nrows // 4)) * sel
    times = []
    cpu = None
    for _ in range(max(1, min(args.steps, 2))):
        t0 = time.perf_counter()
        cpu = chain_cpu(P, production, updates, sel)
        times.append(time.perf_counter() - t0)
    if cpu.get("value") is None:
        return {"impl": "reference", "unavailable": cpu["sample"]}
    v = cpu["value"]
    return {"impl": "reference", "metric": "parallel-beam chain GUPS (voxel x projection updates per second)",
            "value": v, "unit": "GUPS", "n_gpus": world, "steps": len(times), "warmup": 0,
            "ms_per_step": float(np.mean(times)) * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": {"workload": P["name"]},
            "cpu_baseline": cpu, "e2e": {"value": v, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_diff(args):
    """Reference arm of the differentiation workload: the reference's own forward projector
    (LinearForwardProjector, the Joseph anchor; the reference has no adjoint or gradient) on a
    few slices of the 512 x 512 x 128 volume, 360 angles, one slice per call; GUPS of the forward
    projection scaled from the slices timed."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1 and int(os.environ.get("RANK", "0")) != 0:
        return None
    import oracle

    if not oracle.ref_available():
        return {"impl": "reference", "unavailable": "reference library oracle/_ref/libmuhrec_ref.so not built"}
    n, nproj, nslices = (128, 90, 32) if args.small else (512, 360, 128)
    rng = np.random.default_rng(0)
    ang = (np.arange(nproj) * 180.0 / nproj).astype(np.float32)
    cores = os.cpu_count() or 1
    k = min(64, 2 * cores)
    sl = rng.random((k, n, n)).astype(np.float32)
    from concurrent.futures import ThreadPoolExecutor

    times = []
    with ThreadPoolExecutor(max_workers=cores) as pool:  # one slice per call; ctypes releases the GIL
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            list(pool.map(lambda j: oracle.ref_joseph_project(sl[j], ang), range(k)))
            times.append((time.perf_counter() - t0) / k)
    per_slice = float(np.median(times))
    v = float(n) * n * nproj / per_slice / 1e9
    sample = (f"reference LinearForwardProjector (one slice per call) on {k} slices of {n} x {n}, {nproj} angles, "
              f"{cores} slices at a time on {cores} host threads: {per_slice * 1e3:.2f} ms per slice (median of "
              f"{len(times)} steps); the {nslices}-slice volume would take {per_slice * nslices:.2f} s")
    return {"impl": "reference", "metric": "differentiable projector pair GUPS (voxel x projection, forward)",
            "value": v, "unit": "GUPS", "n_gpus": world, "steps": len(times), "warmup": 0,
            "ms_per_step": per_slice * k * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": {"workload": f"volume {n}x{n}x{nslices}, {nproj} projections"},
            "cpu_baseline": {"value": v, "unit": "GUPS", "cores": cores, "kind": "reference", "sample": sample},
            "e2e": {"value": v, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mr", choices=["mr", "reference"])
    ap.add_argument("--small", action="store_true", help="256^3 profiling case")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kernel-times", action="store_true",
                    help="parallel/production: per-kernel device times of one extra step (torch profiler)")
    ap.add_argument("--cpu-budget", type=float, default=20.0)
    ap.add_argument("--workload", default="fdk", choices=["fdk", "fdk-c2", "diff", "parallel", "production"],
                    help="fdk: FDK 1024^3 precision form (default); fdk-c2: FDK 512^3 from 720 projections; "
                         "diff: projector pairs + CGLS refinement; parallel: C1 parallel FBP; production: C3 "
                         "preprocessing + parallel FBP block")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if args.workload in ("parallel", "production"):
            res = run_reference_chain(args, args.workload == "production")
        elif args.workload == "diff":
            res = run_reference_diff(args)
        else:
            res = run_reference(args)
    elif args.workload == "diff":
        res = run_diff(args)
    elif args.workload in ("parallel", "production"):
        res = run_parallel(args, args.workload == "production")
    else:
        res = run_mr(args)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
