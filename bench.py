#!/usr/bin/env python
"""Cone-beam forward + backprojection throughput (GUPS) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cone512|cone256] [--storage bf16|fp16|fp32]

One step = ConeProjection3D of a 512^3 (or 256^3) volume followed by
ConeBackprojection3D of the resulting sinogram (360 views), the north-star
workload.  GUPS = 2 U / t with U = voxels x views (the update count of one
backprojection, used for both directions as the metric defines it).

* ``value``: device-resident inputs, CUDA events around exactly K steps,
  max over ranks; N ranks each run their own volume (weak scaling, no
  data-path collective).
* ``e2e``: the same step through the public API (pyronn_layers ops) with the
  volume copied from pinned host memory and the result copied back inside the
  timed region, steps pipelined over two slots as a stream of volumes runs
  (the next input's upload and the last result's download overlap a step's
  projections).
* ``roofline``: the dominant kernel's algorithmic gather bytes (8 taps per
  forward ray sample, 4 taps per backprojection update, times the storage
  element size, plus its output bytes) over its live CUDA-event time, against
  the measured HBM copy bandwidth.  Values above 1 mean the gathers are served
  on chip (L1 / texture / L2) rather than from HBM.
* ``cpu_baseline``: the FP64 CPU oracle (C, all host threads) on a bounded
  sample (some views, some z-slices), scaled to the full step.
* ``--impl reference``: the CPU oracle as the reference arm (the reference
  has no CPU implementation of these ops; its CUDA kernels are the oracle's
  parity target), same metric and config.
"""
from __future__ import annotations

import argparse
import csv
import datetime
import io
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "pyro-nn-layers_b200")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "cone-beam fwd+back GUPS, BF16 vs plain FP32 at ≤1e-3 rel err; serving p50/p99"

WORKLOADS = {
    "cone512": dict(volume=(512, 512, 512), voxel_mm=0.5, detector=(768, 1024), pixel_mm=1.0, views=360,
                    sid_mm=750.0, sdd_mm=1200.0, step_voxels=0.5),
    "cone256": dict(volume=(256, 256, 256), voxel_mm=0.5, detector=(512, 512), pixel_mm=1.0, views=360,
                    sid_mm=750.0, sdd_mm=1200.0, step_voxels=0.5),
}
PHANTOM_ELLIPSOIDS = 32
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# the dominant kernel, from a one-pass ncu capture of
#   python bench.py --steps 1 --warmup 3 --no-cpu-baseline
# keyed by (workload, volume storage, sinogram storage, hardware_interp)
NCU_DRAM_BYTES = {
    ("cone512", "fp16", "fp16", False): 37.972e9 + 0.574e9,
}
# kernels of ours launched per fwd+back step (geometry preparation, view
# classification, the two volume copies, forward; preparation, backprojection)
LAUNCHES_PER_STEP = {False: 7, True: 6}
L2_BYTES = 126 * 1024 * 1024


# ------------------------------------------------------------ helpers (CPU-testable)


def shard_seed(base_seed: int, rank: int) -> int:
    """Each rank backprojects its own volume: the phantom seed of rank r."""
    return base_seed + 1000 * rank


def aggregate(per_rank_ms, units_per_rank, steps):
    """Whole-job throughput: all ranks' units over the slowest rank's time."""
    t = max(per_rank_ms) / 1e3
    return units_per_rank * len(per_rank_ms) * steps / t


def updates(cfg) -> int:
    z, y, x = cfg["volume"]
    return z * y * x * cfg["views"]


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def decompose_np(P, spacing_zyx, origin_zyx):
    """FP64 camera centre / inverse of P in voxel-index space (same formulas as
    the device preparation kernel); used to count ray samples."""
    s = np.asarray(spacing_zyx, np.float64)[::-1]
    o = np.asarray(origin_zyx, np.float64)[::-1]
    P = np.asarray(P, np.float64)
    M = P[:, :, :3]
    Minv = np.linalg.inv(M)
    C = -np.einsum("nij,nj->ni", Minv, P[:, :, 3])
    src = (C - o) / s
    inv_ar = Minv / s[None, :, None]
    return inv_ar, src


def count_samples(cfg, device):
    """Total ray samples of one forward projection (box [0, N], first sample
    half a step in, one per step while inside), counted in FP64 on the GPU."""
    import torch
    from pyronn_layers import geometry
    g = geometry.ConeBeam3D(cfg["volume"], (cfg["voxel_mm"],) * 3, cfg["detector"], (cfg["pixel_mm"],) * 2,
                            cfg["views"], cfg["sid_mm"], cfg["sdd_mm"], step_size=cfg["step_voxels"])
    inv_ar, src = decompose_np(g.projection_matrices, g.volume_spacing, g.volume_origin)
    H, W = cfg["detector"]
    Z, Y, X = cfg["volume"]
    n_dim = torch.tensor([X, Y, Z], dtype=torch.float64, device=device)
    vv, uu = torch.meshgrid(torch.arange(H, device=device, dtype=torch.float64),
                            torch.arange(W, device=device, dtype=torch.float64), indexing="ij")
    uv1 = torch.stack([uu.flatten(), vv.flatten(), torch.ones_like(uu).flatten()], 0)
    h = cfg["step_voxels"]
    total = 0
    for p in range(cfg["views"]):
        r = torch.as_tensor(inv_ar[p], device=device) @ uv1
        r = r / torch.linalg.norm(r, dim=0, keepdim=True)
        s = torch.as_tensor(src[p], device=device)[:, None]
        with np.errstate(divide="ignore"):
            a0 = (0.0 - s) / r
            a1 = (n_dim[:, None] - s) / r
        amin = torch.minimum(a0, a1).max(dim=0).values
        amax = torch.maximum(a0, a1).min(dim=0).values
        start = amin + 0.5 * h
        n = torch.nan_to_num(torch.clamp(torch.ceil((amax - start) / h), min=0), nan=0.0, posinf=0.0)
        total += int(n.sum().item())
    return total


class ClockSampler:
    """Samples nvidia-smi clocks / throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,utilization.gpu")

    def __init__(self, gpu_index):
        self.gpu_index = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "--id=%s" % self.gpu_index, "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.rows = []
        if self.proc is None:
            return False
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for row in csv.reader(io.StringIO(out)):
            if len(row) >= 9:
                self.rows.append([c.strip() for c in row])
        return False

    def summary(self):
        if not getattr(self, "rows", None):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        # the SM clock under load: samples whose utilisation is at least 50 %
        # (the sampler also sees set-up and host-side gaps, where the clock idles)
        def num(x):
            return x.replace(".", "").isdigit()

        loaded = [r for r in self.rows if len(r) > 9 and num(r[9]) and float(r[9]) >= 50.0]
        sm = [float(r[1]) for r in (loaded or self.rows) if num(r[1])]
        smax = [float(r[2]) for r in self.rows if num(r[2])]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows), "samples_under_load": len(loaded),
                "power_w_max": max(float(r[3]) for r in self.rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in self.rows) else None}


def physical_gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return str(local_rank)


# ------------------------------------------------------------------ CPU legs


def cpu_sample(cfg, geo, vol_np, sino_np, target_s=8.0, threads=None):
    """Times the FP64 oracle on a bounded sample and returns
    (gups, sample description, threads, outputs for the accuracy check)."""
    import oracle
    threads = threads or (os.cpu_count() or 1)
    n_views, n_slices = 1, 2
    Z = cfg["volume"][0]
    t0 = time.perf_counter()
    fwd, _ = oracle.cone_projection3d_views(vol_np, geo.detector_shape, 0, n_views, geo.volume_origin,
                                            geo.volume_spacing, geo.projection_matrices, geo.step_size,
                                            nthreads=threads)
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
    z0 = Z // 2 - n_slices // 2
    back = oracle.cone_backprojection3d_slab(sino_np, geo.volume_shape, z0, z0 + n_slices, geo.volume_origin,
                                             geo.volume_spacing, geo.projection_matrices,
                                             geo.projection_multiplier, nthreads=threads)
    t_back = time.perf_counter() - t0
    t_full = t_fwd * cfg["views"] / n_views + t_back * Z / n_slices
    gups = 2 * updates(cfg) / t_full / 1e9
    desc = ("forward of %d of %d views + backprojection of %d of %d z-slices, FP64 oracle, scaled to the full step"
            % (n_views, cfg["views"], n_slices, Z))
    return gups, desc, threads, dict(fwd=fwd[:n_views], back=back[z0:z0 + n_slices], z0=z0, n_views=n_views,
                                     n_slices=n_slices, seconds=t_fwd + t_back)


def run_reference(args, cfg):
    """Reference arm: the CPU oracle on bounded samples, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from pyronn_layers import geometry, phantoms
    geo = geometry.ConeBeam3D(cfg["volume"], (cfg["voxel_mm"],) * 3, cfg["detector"], (cfg["pixel_mm"],) * 2,
                              cfg["views"], cfg["sid_mm"], cfg["sdd_mm"], step_size=cfg["step_voxels"])
    ell = phantoms.random_ellipsoids(shard_seed(2024, 0), [cfg["volume"][i] * cfg["voxel_mm"] for i in (2, 1, 0)],
                                     n=PHANTOM_ELLIPSOIDS)
    try:
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        vol = phantoms.rasterise_ellipsoids_torch(ell, cfg["volume"], geo.volume_spacing, geo.volume_origin,
                                                  dev).cpu().numpy()
    except ImportError:
        vol = phantoms.rasterise_ellipsoids(ell, cfg["volume"], geo.volume_spacing, geo.volume_origin)
    rng = np.random.Generator(np.random.PCG64(5))
    sino = rng.uniform(0, 50, geo.detector_shape).astype(np.float32)
    times = []
    for i in range(args.warmup + args.steps):
        gups, desc, threads, _ = cpu_sample(cfg, geo, vol, sino)
        if i >= args.warmup:
            times.append(2 * updates(cfg) / gups / 1e9)
    t = sum(times)
    value = 2 * updates(cfg) * args.steps / t / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(args, cfg),
        "cpu_baseline": {"value": value, "unit": "GUPS", "cores": threads, "kind": "port", "sample": desc},
        "e2e": {"value": value, "unit": "GUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def sino_storage_name(args):
    return args.storage if args.sino_storage == "same" else args.sino_storage


def config_block(args, cfg):
    z, y, x = cfg["volume"]
    return {"workload": args.workload, "volume": list(cfg["volume"]), "voxel_mm": cfg["voxel_mm"],
            "views": cfg["views"], "detector_hw": list(cfg["detector"]), "pixel_mm": cfg["pixel_mm"],
            "sid_mm": cfg["sid_mm"], "sdd_mm": cfg["sdd_mm"], "step_voxels": cfg["step_voxels"],
            "hardware_interp": bool(args.hardware_interp), "storage": args.storage,
            "sinogram_storage": sino_storage_name(args),
            "updates_per_op": updates(cfg), "phantom": "%d seeded ellipsoids" % PHANTOM_ELLIPSOIDS,
            "l2": "inputs larger than L2 (volume %d MB, sinogram %d MB at the storage dtype)"
                  % (z * y * x * (4 if args.storage == "fp32" else 2) >> 20,
                     cfg["views"] * cfg["detector"][0] * cfg["detector"][1]
                     * (4 if sino_storage_name(args) == "fp32" else 2) >> 20),
            "parallelism": "replicas (one volume per GPU)" if args.gpus > 1 else "single GPU"}


# ------------------------------------------------------------------ our arm


def run_ours(args, cfg):
    import torch
    import torch.distributed as dist

    import pyronn_layers as pl
    from pyronn_layers import geometry, ops, phantoms

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    dev = torch.device("cuda", local_rank)
    dtypes = {"bf16": torch.bfloat16, "fp16": torch.float16, "fp32": torch.float32}
    storage = dtypes[args.storage]
    sino_storage = dtypes[sino_storage_name(args)]

    geo = geometry.ConeBeam3D(cfg["volume"], (cfg["voxel_mm"],) * 3, cfg["detector"], (cfg["pixel_mm"],) * 2,
                              cfg["views"], cfg["sid_mm"], cfg["sdd_mm"], step_size=cfg["step_voxels"])
    ell = phantoms.random_ellipsoids(shard_seed(2024, rank),
                                     [cfg["volume"][i] * cfg["voxel_mm"] for i in (2, 1, 0)], n=PHANTOM_ELLIPSOIDS)
    vol32 = phantoms.rasterise_ellipsoids_torch(ell, cfg["volume"], geo.volume_spacing, geo.volume_origin, dev)
    n_proj = cfg["views"]
    H, W = cfg["detector"]
    Z, Y, X = cfg["volume"]
    hw = bool(args.hardware_interp)

    # prepared device geometry and workspaces (what a serving caller keeps resident)
    gc = ops.GeometryCone(1, dev, *geo.args(), n_proj)

    def make_step(store, out_fwd, out_back):
        x = vol32.to(store)[None].contiguous()
        sino = torch.empty((1, n_proj, H, W), dtype=out_fwd, device=dev)
        back = torch.empty((1, Z, Y, X), dtype=out_back, device=dev)
        sf0, so0 = ops.storage_code(store), ops.storage_code(out_fwd)
        ws_f = torch.empty(pl._capi.workspace_size("pyronn_cone_projection3d", 1, Z, Y, X, n_proj, H, W, sf0,
                                                   int(hw), 1), dtype=torch.uint8, device=dev)
        ws_b = torch.empty(pl._capi.workspace_size("pyronn_cone_backprojection3d", 1, n_proj, H, W, Z, Y, X, so0,
                                                   int(hw), 1), dtype=torch.uint8, device=dev)
        lib = pl._capi
        gp = gc.pointers()
        sf, so, sb = ops.storage_code(store), ops.storage_code(out_fwd), ops.storage_code(out_back)
        ev = []

        def fwd():
            lib.call("pyronn_cone_projection3d", x.data_ptr(), sino.data_ptr(), sf, so, int(hw), 1, Z, Y, X, n_proj,
                     H, W, *gp, 1, ws_f.data_ptr(), ws_f.numel(), torch.cuda.current_stream(dev).cuda_stream)

        def bwd():
            lib.call("pyronn_cone_backprojection3d", sino.data_ptr(), back.data_ptr(), so, sb, int(hw), 1, n_proj,
                     H, W, Z, Y, X, *gp, 1, ws_b.data_ptr(), ws_b.numel(), torch.cuda.current_stream(dev).cuda_stream)

        def step(record=False):
            if record:
                e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                e[0].record()
                fwd()
                e[1].record()
                bwd()
                e[2].record()
                ev.append(e)
            else:
                fwd()
                bwd()

        return step, ev, x, sino, back

    def barrier():
        if world > 1:
            dist.barrier()

    def timed(step, steps, warmup, record):
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        barrier()
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        start.record()
        for _ in range(steps):
            step(record) if record is not None else step()
        end.record()
        torch.cuda.synchronize()
        barrier()
        ms = start.elapsed_time(end)
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    # ---- the headline configuration (storage dtype in, sinogram storage
    # between the ops, FP32 volume out)
    step, ev, x, sino, back = make_step(storage, sino_storage, torch.float32)
    with ClockSampler(physical_gpu_index(local_rank)) as clk:
        ms = timed(lambda rec=False: step(rec), args.steps, args.warmup, True)
    clocks = clk.summary()
    fwd_ms = [a.elapsed_time(b) for a, b, _ in ev]
    back_ms = [b.elapsed_time(c) for _, b, c in ev]
    value = 2 * updates(cfg) * world * args.steps / (ms / 1e3) / 1e9

    # ---- the plain FP32 path on the same GPU (same kernels, FP32 storage)
    fp32_gups = None
    if storage != torch.float32:
        step32, _, _, _, _ = make_step(torch.float32, torch.float32, torch.float32)
        ms32 = timed(lambda rec=False: step32(), args.steps, args.warmup, None)
        fp32_gups = 2 * updates(cfg) * world * args.steps / (ms32 / 1e3) / 1e9
        del step32
        torch.cuda.empty_cache()

    # ---- end to end through the public API: pinned host volume in, FP32
    # volume out, every step.  Steps run as a stream of volumes does: two
    # slots, the host->device copy of step i+1 and the device->host copy of
    # step i overlap step i's projections (copy engines, own streams); the
    # timed region ends when the last result is in host memory.
    host_in = [torch.empty((1, Z, Y, X), dtype=storage, pin_memory=True) for _ in range(2)]
    for h in host_in:
        h.copy_(x.cpu())
    host_out = [torch.empty((1, Z, Y, X), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    dev_in = [torch.empty_like(x) for _ in range(2)]
    h2d, d2h = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    comp = torch.cuda.current_stream(dev)
    slot_done = [None, None]
    args_geo = geo.args()

    def e2e_run(n):
        for i in range(n):
            k = i % 2
            with torch.cuda.stream(h2d):
                if slot_done[k] is not None:
                    h2d.wait_event(slot_done[k])  # step i-2 is done reading the slot
                dev_in[k].copy_(host_in[k], non_blocking=True)
                ev_in = torch.cuda.Event()
                ev_in.record(h2d)
            comp.wait_event(ev_in)
            s = pl.cone_projection3d(dev_in[k], geo.detector_shape, *args_geo, hardware_interp=hw,
                                     out_dtype=sino_storage)
            b = pl.cone_backprojection3d(s, geo.volume_shape, *args_geo, hardware_interp=hw,
                                         out_dtype=torch.float32)
            ev_b = torch.cuda.Event()
            ev_b.record(comp)
            slot_done[k] = ev_b
            with torch.cuda.stream(d2h):
                d2h.wait_event(ev_b)
                host_out[k].copy_(b, non_blocking=True)
                b.record_stream(d2h)

    # at least 8 steps: the first upload and the last download are the only
    # copies no step's projections hide
    e2e_steps = max(8, args.steps)
    e2e_run(max(args.warmup, 3))
    torch.cuda.synchronize()
    barrier()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_start.record(comp)
    h2d.wait_stream(comp)
    e2e_run(e2e_steps)
    comp.wait_stream(h2d)
    comp.wait_stream(d2h)
    e_end.record(comp)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = e_start.elapsed_time(e_end)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = 2 * updates(cfg) * world * e2e_steps / (e2e_ms / 1e3) / 1e9

    # ---- roofline of the dominant kernel
    es = 2 if storage != torch.float32 else 4
    es_s = 2 if sino_storage != torch.float32 else 4
    S = count_samples(cfg, dev)
    f_ms, b_ms = statistics.mean(fwd_ms), statistics.mean(back_ms)
    fwd_bytes = S * 8 * es + n_proj * H * W * es_s
    back_bytes = updates(cfg) * 4 * es_s + Z * Y * X * 4
    peak, peak_kind = measured_peaks()
    if f_ms >= b_ms:
        dom, dom_bytes, dom_ms = "cone_fp_kernel (forward)", fwd_bytes, f_ms
    else:
        dom, dom_bytes, dom_ms = "cone_bp_kernel (backprojection)", back_bytes, b_ms
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": "%s HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"
                % peak_kind if peak_kind == "measured" else "fallback 6.65 TB/s",
                "traffic": args.traffic_bytes if args.traffic_bytes is not None else NCU_DRAM_BYTES.get(
                    (args.workload, args.storage, sino_storage_name(args), hw)) if f_ms >= b_ms else None,
                "algorithmic_bytes_per_launch": dom_bytes,
                "note": "algorithmic bytes = interpolation taps x element size (+ output); frac > 1 means the "
                        "gathers are served on chip, traffic (ncu dram bytes) is the HBM side"}

    line = {
        "metric": METRIC, "value": value, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "storage": args.storage,
        "sinogram_storage": sino_storage_name(args), "data": "synthetic",
        "config": config_block(args, cfg),
        "plain_fp32_value": fp32_gups,
        "storage_over_fp32": (value / fp32_gups) if fp32_gups else None,
        "kernels": {"forward_ms": f_ms, "backprojection_ms": b_ms, "ray_samples": S,
                    "forward_gsamples_per_s": S / (f_ms / 1e3) / 1e9,
                    "backprojection_gups": updates(cfg) / (b_ms / 1e3) / 1e9},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": "GUPS",
                "h2d_bytes_per_step": host_in[0].numel() * host_in[0].element_size(),
                "d2h_bytes_per_step": host_out[0].numel() * host_out[0].element_size(), "steps": e2e_steps,
                "api": "pyronn_layers.cone_projection3d + cone_backprojection3d",
                "overlap": "two slots: the H2D copy of step i+1 and the D2H copy of step i run on their own "
                           "streams during step i's projections; every step's input and result cross the host "
                           "link inside the timed region"},
        "gpu_launches": LAUNCHES_PER_STEP[hw] * args.steps,
        "clocks": clocks,
    }

    # ---- CPU baseline (rank 0, N = 1) and accuracy against the FP64 oracle
    if world == 1 and not args.no_cpu_baseline:
        vol_np = vol32.cpu().numpy()[None]
        sino_np = sino.float().cpu().numpy()
        gups, desc, threads, outs = cpu_sample(cfg, geo, vol_np, sino_np)
        line["cpu_baseline"] = {"value": gups, "unit": "GUPS", "cores": threads, "kind": "port", "sample": desc}
        nv, z0, ns = outs["n_views"], outs["z0"], outs["n_slices"]
        ours_f = sino[0, :nv].float().cpu().numpy()
        ours_b = back[0, z0:z0 + ns].float().cpu().numpy()

        def rel(a, b):
            return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))

        line["accuracy"] = {
            "forward_rel_l2_vs_fp64": rel(ours_f, outs["fwd"]),
            "backprojection_rel_l2_vs_fp64": rel(ours_b, outs["back"]),
            "note": "forward: %s storage of the FP32 phantom, %s sinogram, vs the FP64 oracle on the FP32 "
                    "phantom (%d view); backprojection: same sinogram, FP32 volume, %d z-slices"
                    % (args.storage, sino_storage_name(args), nv, ns)}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def run_serving(args):
    """Serving stream (config 5): a seeded Poisson trace of mixed jobs through
    the continuous-batching server and through the plain one-job-per-launch
    FP32 path on the same GPU; reports p50/p99 latency and aggregate GUPS."""
    import torch

    from pyronn_layers import serving
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    geos = serving.standard_geometries()
    trace = serving.poisson_trace(args.requests, args.rate, seed=7)
    jobs = serving.make_jobs(trace, geos, seed=1)
    # start-up: buffer sets and graphs of batch sizes 1 and 2 for every class
    # (a server does this before taking requests), then one job of each class
    # through both paths so lazy set-up is out of the timed traces
    classes = sorted({c for _, c in trace}, key=str)
    server = serving.ProjectorServer(geos, device=dev, keep_results=False)
    warmup_s = server.warmup(classes, batch_sizes=(1, 2))
    warm = serving.make_jobs([(0.0, c) for c in classes], geos, seed=1)
    server.run_trace(warm, realtime=False)
    server.batches, server.batch_sizes = 0, []
    serving.run_plain(serving.make_jobs([(0.0, c) for c in classes], geos, seed=1), geos, device=dev,
                      realtime=False)
    with ClockSampler(physical_gpu_index(dev.index or 0)) as clk:
        s_srv = server.run_trace(jobs, realtime=True)
    jobs_plain = serving.make_jobs(trace, geos, seed=1)
    s_plain = serving.run_plain(jobs_plain, geos, device=dev, realtime=True, keep_results=False)
    line = {
        "metric": METRIC, "value": s_srv.gups, "unit": "GUPS", "n_gpus": 1, "steps": args.requests, "warmup": 1,
        "ms_per_step": s_srv.wall_s * 1e3 / max(1, args.requests), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "storage": "fp32/bf16 mix", "data": "synthetic",
        "config": {"workload": "serving", "requests": args.requests, "rate_hz": args.rate,
                   "mix": "60% fan 512^2 (360 views, 1024 px), 30% cone 128^3 (180 views, 256^2), 10% cone 256^3 "
                          "(360 views, 512^2); forward/back 50/50; FP32/BF16 50/50",
                   "arrivals": "Poisson, seed 7"},
        "serving": s_srv.as_dict(),
        "server_startup_s": warmup_s,
        "plain_one_job_per_launch_fp32": s_plain.as_dict(),
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


FAN2D = dict(batch=64, volume=(512, 512), pixel_mm=0.5, views=360, detector=1024, det_mm=0.5, sid_mm=750.0,
             sdd_mm=1200.0)


def run_fan2d(args):
    """2D fan-beam batch (config 2): 64 independent 512^2 slices at 0.5 mm,
    360 views over 2 pi, flat 1024-px detector at 0.5 mm, SID 750 / SDD 1200;
    one step = FanProjection2D of the batch + FanBackprojection2D of its
    sinograms.  GUPS = 2 * 64 * 512^2 * 360 / t."""
    import torch

    from pyronn_layers import geometry, ops, phantoms
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    c = FAN2D
    g = geometry.FanBeam2D(c["volume"], (c["pixel_mm"],) * 2, c["detector"], c["det_mm"], c["views"], c["sid_mm"],
                           c["sdd_mm"])
    vols = np.stack([phantoms.ellipse_phantom_2d(c["volume"], (c["pixel_mm"],) * 2, seed=100 + b)[0]
                     for b in range(c["batch"])])
    storage = {"bf16": torch.bfloat16, "fp16": torch.float16, "fp32": torch.float32}[args.storage]
    units = c["batch"] * c["volume"][0] * c["volume"][1] * c["views"]

    def run(store):
        x = torch.from_numpy(vols).to(dev, store)
        geo = ops.Geometry2D(c["batch"], dev, *g.args()[:4], g.ray_vectors, c["views"], g.sid, g.sdd)
        sino = torch.empty((c["batch"], c["views"], c["detector"]), dtype=store, device=dev)
        back = torch.empty((c["batch"],) + c["volume"], dtype=torch.float32, device=dev)
        code = ops.storage_code(store)
        lib = ops._capi
        ws = torch.empty(lib.workspace_size("pyronn_projection2d", c["batch"], *c["volume"], code),
                         dtype=torch.uint8, device=dev)
        ev = []

        def step():
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            s = torch.cuda.current_stream(dev).cuda_stream
            e[0].record()
            lib.call("pyronn_fan_projection2d", x.data_ptr(), sino.data_ptr(), code, code, c["batch"],
                     *c["volume"], c["views"], c["detector"], *geo.pointers(), geo.g, ws.data_ptr(), ws.numel(), s)
            e[1].record()
            lib.call("pyronn_fan_backprojection2d", sino.data_ptr(), back.data_ptr(), code, 0, c["batch"],
                     c["views"], c["detector"], *c["volume"], *geo.pointers(), geo.g, s)
            e[2].record()
            ev.append(e)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        ev.clear()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(args.steps):
            step()
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
        f = statistics.mean(a.elapsed_time(b) for a, b, _ in ev)
        bk = statistics.mean(b.elapsed_time(c2) for _, b, c2 in ev)
        return 2 * units * args.steps / (ms / 1e3) / 1e9, ms, f, bk, sino, back

    with ClockSampler(physical_gpu_index(dev.index or 0)) as clk:
        gups, ms, f_ms, b_ms, sino, back = run(storage)
    gups32 = run(torch.float32)[0] if storage != torch.float32 else None
    line = {
        "metric": METRIC, "value": gups, "unit": "GUPS", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "storage": args.storage, "data": "synthetic",
        "config": {"workload": "fan2d", "batch": c["batch"], "slice": list(c["volume"]), "pixel_mm": c["pixel_mm"],
                   "views": c["views"], "detector_px": c["detector"], "det_mm": c["det_mm"], "sid_mm": c["sid_mm"],
                   "sdd_mm": c["sdd_mm"], "phantom": "10 seeded ellipses per slice"},
        "plain_fp32_value": gups32,
        "kernels": {"forward_ms": f_ms, "backprojection_ms": b_ms},
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


def run_fdk(args):
    """FDK of the 512^3 cone workload: cosine weighting + ramp filtering of the
    360 x 768 x 1024 projections (storage dtype in, FP32 out) and the
    backprojection of the filtered projections into an FP32 volume.  GUPS =
    512^3 * 360 / t (the backprojection's updates over filter + backprojection
    time); the filter is also reported as FP32 FLOP/s of the taps it
    multiplies (Ram-Lak: the centre and the odd offsets, 2 FLOP each)."""
    import math

    import torch

    from pyronn_layers import geometry, ops
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    cfg = WORKLOADS["cone512"]
    storage = {"bf16": torch.bfloat16, "fp16": torch.float16, "fp32": torch.float32}[args.storage]
    geo = geometry.ConeBeam3D(cfg["volume"], (cfg["voxel_mm"],) * 3, cfg["detector"], (cfg["pixel_mm"],) * 2,
                              cfg["views"], cfg["sid_mm"], cfg["sdd_mm"], step_size=cfg["step_voxels"])
    H, W = cfg["detector"]
    n = cfg["views"]
    rng = torch.Generator(device=dev).manual_seed(11)
    sino = torch.rand((1, n, H, W), generator=rng, device=dev).to(storage)
    q = torch.empty((1, n, H, W), dtype=torch.float32, device=dev)
    vol = torch.empty((1,) + tuple(cfg["volume"]), dtype=torch.float32, device=dev)
    gc = ops.GeometryCone(1, dev, geo.volume_origin, geo.volume_spacing, geo.projection_matrices, geo.step_size,
                          np.array([geo.sid * geo.sdd * math.pi / n], np.float32), n)
    ws = torch.empty(ops._capi.workspace_size("pyronn_cone_backprojection3d", 1, n, H, W, *cfg["volume"], 0, 0, 1),
                     dtype=torch.uint8, device=dev)
    code = ops.storage_code(storage)
    ev = []

    def step():
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        s = torch.cuda.current_stream(dev).cuda_stream
        e[0].record()
        ops._capi.call("pyronn_fdk_filter", sino.data_ptr(), q.data_ptr(), code, 0, 1, n, H, W, geo.sdd,
                       cfg["pixel_mm"], cfg["pixel_mm"], (H - 1) / 2.0, (W - 1) / 2.0, 0, 0, s)
        e[1].record()
        ops._capi.call("pyronn_cone_backprojection3d", q.data_ptr(), vol.data_ptr(), 0, 0, 0, 1, n, H, W,
                       *cfg["volume"], *gc.pointers(), 1, ws.data_ptr(), ws.numel(), s)
        e[2].record()
        ev.append(e)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    ev.clear()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(physical_gpu_index(dev.index or 0)) as clk:
        t0.record()
        for _ in range(args.steps):
            step()
        t1.record()
        torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    f_ms = statistics.mean(a.elapsed_time(b) for a, b, _ in ev)
    b_ms = statistics.mean(b.elapsed_time(c) for _, b, c in ev)
    wp = (W + 15) // 16 * 16
    flops = 2.0 * n * H * wp * (wp / 2 + 1)
    # the tensor-core filter's executed work: three TF32 products (hi*hi,
    # hi*lo, lo*hi) of the dense Toeplitz matrix, outputs in tiles of 128,
    # inputs in chunks of 32
    wn, wk = (W + 127) // 128 * 128, (W + 31) // 32 * 32
    tc_flops = 3 * 2.0 * n * H * wn * wk
    line = {
        "metric": "cone-beam FDK (filter + backprojection) GUPS", "value": updates(cfg) * args.steps / (ms / 1e3) / 1e9,
        "unit": "GUPS", "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "storage": args.storage, "data": "synthetic (uniform random projections)",
        "config": {"workload": "fdk", "volume": list(cfg["volume"]), "views": n, "detector_hw": [H, W],
                   "filter": "ram-lak", "filtered_storage": "fp32"},
        "kernels": {"filter_ms": f_ms, "backprojection_ms": b_ms,
                    "filter_tflops": flops / (f_ms / 1e3) / 1e12,
                    "filter_note": "useful work: the FP32 FMAs of a direct convolution over the nonzero Ram-Lak "
                                   "taps, 2 x rows x %d x (%d / 2 + 1) per launch" % (wp, wp),
                    "filter_tensor_tflops": tc_flops / (f_ms / 1e3) / 1e12,
                    "filter_tensor_note": "executed on the tensor cores (rows of up to 2048 pixels, a multiple of 4): 3 TF32 "
                                          "products x 2 x rows x %d x %d per launch" % (wn, wk)},
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["serving", "fan2d", "fdk"], default="cone512")
    ap.add_argument("--requests", type=int, default=2000, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=100.0, help="serving: Poisson arrival rate (1/s)")
    ap.add_argument("--storage", choices=["bf16", "fp16", "fp32"], default="fp16",
                    help="storage of the volume the forward projection reads (fp16: the 16-bit format that keeps "
                         "the forward within 1e-3 of the FP64 oracle; bf16 rounds piecewise-constant densities "
                         "to ~1.2e-3)")
    ap.add_argument("--sino-storage", choices=["same", "bf16", "fp16", "fp32"], default="same",
                    help="storage of the sinogram between the two ops ('same': as --storage)")
    ap.add_argument("--hardware-interp", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--traffic-bytes", type=float, default=None,
                    help="dram bytes per launch of the dominant kernel from an ncu capture")
    args = ap.parse_args(argv)
    args.warmup = max(args.warmup, 3)  # at least 3 untimed warm-up steps
    if args.workload == "fan2d":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the fan2d workload is measured on the GPU arm only"}))
            return
        run_fan2d(args)
        return
    if args.workload == "fdk":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no FDK filter"}))
            return
        run_fdk(args)
        return
    if args.workload == "serving":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the serving stream has no CPU reference arm"}))
            return
        run_serving(args)
        return
    cfg = WORKLOADS[args.workload]
    if args.impl == "reference":
        run_reference(args, cfg)
    else:
        run_ours(args, cfg)


if __name__ == "__main__":
    main()
