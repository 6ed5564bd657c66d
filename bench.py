#!/usr/bin/env python
"""Cone-beam forward + backprojection throughput (GUPS) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload cone512|cone256] [--storage bf16|fp16|fp32]

One step = ConeProjection3D of a 512^3 (or 256^3) volume followed by
ConeBackprojection3D of the resulting sinogram (360 views), 1024 x 768
detector, the headline workload.  GUPS = 2 U / t with U = voxels x views (the update count of one
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
# the dominant kernel, from a one-pass ncu capture of one forward launch of
#   python bench.py --steps 1 --warmup 3 --no-cpu-baseline
# keyed by (workload, volume storage, sinogram storage, hardware_interp)
NCU_DRAM_BYTES = {
    ("cone512", "fp16", "fp16", False): 37.231e9 + 0.571e9,
}
# ncu counters of the forward kernel from a section capture of its first
# launch at 256^3 (issue activity, lanes, instructions per ray sample; L2 ->
# SM bytes per ray sample from the same capture, scaling with the sample
# count)
NCU_FORWARD_COUNTERS = {
    ("cone512", "fp16", "fp16", False): {
        "issue_active": 0.781, "lanes_active_per_warp_instruction": 26.77,
        "thread_instructions_per_sample": 32.1, "lts2xbar_bytes_per_sample_256": 11.1,
        "source": "profiles/cone_fp_padded_kernel_cone256_fp16.md (256^3 capture; L2 -> SM bytes per sample "
                  "from its L2 read sectors of the texture unit, scaling with the samples)"},
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


def sample_spec(cfg):
    """The oracle's bounded sample of a step: (views, first z-slice, slices)."""
    n_views, n_slices = 1, 2
    return n_views, cfg["volume"][0] // 2 - n_slices // 2, n_slices


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def host_in_bytes(cfg):
    """Bytes of the FP32 host volume the e2e leg uploads per step."""
    z, y, x = cfg["volume"]
    return z * y * x * 4


L2_READ_KERNEL = r"""
extern "C" __global__ void l2_read(const uint4 *__restrict__ a, unsigned n4, unsigned passes, unsigned *out)
{
    const unsigned stride = gridDim.x * blockDim.x;
    unsigned acc = 0u;
    for (unsigned p = 0; p < passes; ++p) {
        for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += stride) {
            const uint4 v = __ldcg(a + i);  // L2, not L1
            acc ^= (v.x ^ v.y) ^ (v.z ^ v.w);
        }
    }
    if (acc == 0x9e3779b9u) out[0] = acc;  // keeps the loads
}
"""


def measure_l2_peak(dev, mib=32, passes=64, repeats=7):
    """L2 -> SM read bandwidth, measured the way the HBM peak is (a simple
    kernel, CUDA events, best of N): 16-byte ld.global.cg sweeps of a `mib`
    MiB buffer that stays L2-resident, `passes` sweeps per launch, 2048
    threads per SM, one XOR per load.  The kernel is compiled at run time with
    NVRTC for this GPU; it is a measurement probe, not part of the library."""
    import ctypes

    import torch
    from cuda.bindings import driver, nvrtc

    def ok(res):
        err = res[0]
        if int(err) != 0:
            raise RuntimeError("L2 probe: %s" % (err,))
        return res[1:] if len(res) > 2 else (res[1] if len(res) == 2 else None)

    major, minor = torch.cuda.get_device_capability(dev)
    prog = ok(nvrtc.nvrtcCreateProgram(L2_READ_KERNEL.encode(), b"l2_read.cu", 0, [], []))
    arch = ("--gpu-architecture=sm_%d%d%s" % (major, minor, "a" if major >= 9 else "")).encode()
    if int(nvrtc.nvrtcCompileProgram(prog, 1, [arch])[0]) != 0:
        raise RuntimeError("L2 probe: NVRTC compilation failed")
    size = ok(nvrtc.nvrtcGetCUBINSize(prog))
    cubin = b" " * size
    ok((nvrtc.nvrtcGetCUBIN(prog, cubin)[0], None))
    torch.cuda.init()
    with torch.cuda.device(dev):
        torch.zeros(1, device=dev)  # the primary context is current
        module = ok(driver.cuModuleLoadData(cubin))
        fn = ok(driver.cuModuleGetFunction(module, b"l2_read"))
        n4 = mib * (1 << 20) // 16
        a = torch.rand(n4 * 4, device=dev)
        out = torch.zeros(1, device=dev)
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        grid, block = 4 * sms, 512  # 2048 threads per SM
        args = (ctypes.c_void_p(a.data_ptr()), ctypes.c_uint(n4), ctypes.c_uint(passes), ctypes.c_void_p(out.data_ptr()))
        argv = (ctypes.c_void_p * 4)(*[ctypes.addressof(x) for x in args])
        stream = torch.cuda.current_stream(dev)

        def launch():
            ok((driver.cuLaunchKernel(fn, grid, 1, 1, block, 1, 1, 0, stream.cuda_stream, ctypes.addressof(argv), 0)[0],
                None))

        for _ in range(3):
            launch()
        best = 0.0
        for _ in range(repeats):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            launch()
            e.record(stream)
            torch.cuda.synchronize(dev)
            best = max(best, n4 * 16.0 * passes / (s.elapsed_time(e) / 1e3) / 1e9)
        ok((driver.cuModuleUnload(module)[0], None))
    return {"gbs": best, "how": "16-byte ld.global.cg sweeps of a %d MiB L2-resident buffer, %d sweeps per launch, "
                                "2048 threads per SM, best of %d launches (NVRTC-compiled probe)"
                                % (mib, passes, repeats)}


def oracle_slab(cfg, geo, sino_np):
    """FP64 oracle backprojection of the sample slices of one sinogram."""
    import oracle
    nv, z0, ns = sample_spec(cfg)
    out = oracle.cone_backprojection3d_slab(sino_np, geo.volume_shape, z0, z0 + ns, geo.volume_origin,
                                            geo.volume_spacing, geo.projection_matrices, geo.projection_multiplier)
    return out[z0:z0 + ns]


def reference_gpu(cfg, geo, vol32, dev, f_ms, b_ms, ours_fp32_gups, ours_gups, args):
    """The reference's own CUDA kernels (cc/kernels/*.cu.cc built unmodified
    into oracle/_ref by the oracle's recipe), run through the op-layer
    restatement oracle/ref/ref_driver.cu -- one launcher call per op with its
    per-call allocations and FP32 storage, the reference's
    Cone_Projection_Kernel_Launcher (cone_projector_3D_CudaKernel.cu.cc:225-257)
    and Cone_Backprojection3D_Kernel_Launcher
    (cone_backprojector_3D_CudaKernel.cu.cc:121-146), or their texture
    launchers (..._hardware_interp.cu.cc) for a --hardware-interp run -- on
    this workload, timed with CUDA events on the default stream; outside our
    timed regions.  Also the relative L2 distance of our FP32 results from
    theirs."""
    import ctypes

    import torch

    import oracle
    if not os.path.exists(oracle.REF_LIB):
        return {"unavailable": "oracle/_ref/libpyronn_ref.so not built (needs the reference sources)"}
    hw = 1 if args.hardware_interp else 0
    L = ctypes.CDLL(oracle.REF_LIB)
    Z, Y, X = cfg["volume"]
    H, W = cfg["detector"]
    n = cfg["views"]
    keep = []

    def dptr(a, slack=0):
        a = np.ascontiguousarray(np.asarray(a, dtype=np.float32)).reshape(-1)
        t = torch.zeros(a.size + slack, dtype=torch.float32, device=dev)
        t[: a.size] = torch.from_numpy(a).to(dev)
        keep.append(t)
        return ctypes.c_void_p(t.data_ptr())

    vo, vs, P, st, mu = (np.asarray(a, np.float32)[None] for a in geo.args())
    g = [dptr(vo), dptr(vs), dptr(P), dptr(st), dptr(mu)]
    vol = vol32[None].contiguous()
    sino = torch.zeros(n * H * W + W + 8, dtype=torch.float32, device=dev)  # slack for its x == W taps
    back = torch.zeros(Z * Y * X, dtype=torch.float32, device=dev)
    fargs = (ctypes.c_void_p(vol.data_ptr()), ctypes.c_void_p(sino.data_ptr()), hw, 1, Z, Y, X, n, H, W, g[0], g[1],
             g[2], g[3])
    bargs = (ctypes.c_void_p(sino.data_ptr()), ctypes.c_void_p(back.data_ptr()), hw, 1, n, H, W, Z, Y, X, g[0], g[1],
             g[2], g[4])

    def timed(fn, reps=2):
        rc = fn()
        if rc != 0:
            raise RuntimeError("reference launcher failed with CUDA error %d" % rc)
        times = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            times.append(s.elapsed_time(e))
        return statistics.mean(times)

    try:
        fms = timed(lambda: L.ref_cone_projection3d(*fargs))
        bms = timed(lambda: L.ref_cone_backprojection3d(*bargs))
    except RuntimeError as exc:
        return {"unavailable": str(exc)}
    # our FP32 results on the same inputs, for the parity figure at this size
    from pyronn_layers import ops
    ours_s = ops.cone_projection3d(vol, geo.detector_shape, *geo.args(), hardware_interp=bool(hw))
    e_f = rel_l2(ours_s.reshape(-1).cpu().numpy(), sino[: n * H * W].cpu().numpy())
    ours_v = ops.cone_backprojection3d(sino[: n * H * W].reshape(1, n, H, W), geo.volume_shape, *geo.args(),
                                       hardware_interp=bool(hw))
    e_b = rel_l2(ours_v.reshape(-1).cpu().numpy(), back.cpu().numpy())
    gups = 2 * updates(cfg) / ((fms + bms) / 1e3) / 1e9
    return {"value": gups, "unit": "GUPS", "forward_ms": fms, "backprojection_ms": bms,
            "storage": "fp32 (the reference's only storage type)", "hardware_interp": bool(hw),
            "ours_fp32_over_reference": ours_fp32_gups / gups, "ours_over_reference": ours_gups / gups,
            "forward_over_reference": fms / f_ms, "backprojection_over_reference": bms / b_ms,
            "ours_fp32_forward_rel_l2_vs_reference": e_f, "ours_fp32_backprojection_rel_l2_vs_reference": e_b,
            "what": "the reference's own kernels (cc/kernels/*.cu.cc built unmodified for sm_100a) through a "
                    "restatement of its TF op layer (oracle/ref/ref_driver.cu): FP32, per-call allocations and "
                    "host-side matrix decomposition as the reference's ops do, default stream, 1 warm-up + 2 timed "
                    "calls per op; forward/backprojection_over_reference compare against OUR headline kernels"}


# ------------------------------------------------------------------ CPU legs


def cpu_sample(cfg, geo, vol_np, sino_np, target_s=8.0, threads=None):
    """Times the FP64 oracle on a bounded sample and returns
    (gups, sample description, threads, outputs for the accuracy check)."""
    import oracle
    threads = threads or (os.cpu_count() or 1)
    n_views, z0, n_slices = sample_spec(cfg)
    Z = cfg["volume"][0]
    t0 = time.perf_counter()
    fwd, _ = oracle.cone_projection3d_views(vol_np, geo.detector_shape, 0, n_views, geo.volume_origin,
                                            geo.volume_spacing, geo.projection_matrices, geo.step_size,
                                            nthreads=threads)
    t_fwd = time.perf_counter() - t0
    t0 = time.perf_counter()
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

    # ---- BF16 storage (the precision the metric names), same kernels
    bf16 = None
    if storage != torch.bfloat16:
        step16, ev16, _, sino16, back16 = make_step(torch.bfloat16, torch.bfloat16, torch.float32)
        ms16 = timed(lambda rec=False: step16(rec), args.steps, args.warmup, True)
        bf16 = {"value": 2 * updates(cfg) * world * args.steps / (ms16 / 1e3) / 1e9, "unit": "GUPS",
                "storage": "bf16 volume, bf16 sinogram, FP32 sums, FP32 volume out",
                "forward_ms": statistics.mean(a.elapsed_time(b) for a, b, _ in ev16),
                "backprojection_ms": statistics.mean(b.elapsed_time(c) for _, b, c in ev16)}
        nv, z0, ns = sample_spec(cfg)
        bf16_outputs = (sino16[0, :nv].float().cpu().numpy(), sino16.float().cpu().numpy()
                        if world == 1 and not args.no_cpu_baseline else None,
                        back16[0, z0:z0 + ns].float().cpu().numpy())
        del step16, sino16, back16
        torch.cuda.empty_cache()

    # ---- end to end through the public API: pinned FP32 host volume in, FP32
    # volume out, every step.  Each step uploads the FP32 volume, converts it
    # to the storage dtype on the device, projects and backprojects, and
    # downloads the FP32 result.  Steps run as a stream of volumes does: two
    # slots, the host->device copy of step i+1 and the device->host copy of
    # step i overlap step i's projections (copy engines, own streams); the
    # timed region ends when the last result is in host memory.
    host_in = [torch.empty((1, Z, Y, X), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    for h in host_in:
        h.copy_(vol32[None].cpu())
    host_out = [torch.empty((1, Z, Y, X), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    dev_in = [torch.empty((1, Z, Y, X), dtype=torch.float32, device=dev) for _ in range(2)]
    h2d, d2h = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    comp = torch.cuda.current_stream(dev)
    slot_done = [None, None]
    # the scan's geometry as device tensors, once, as a caller streaming
    # volumes through one scan holds it (host arrays would be copied to the
    # device by every call, each copy from pageable memory waiting for the
    # stream's queued work)
    args_geo = tuple(torch.as_tensor(np.asarray(a, np.float32), device=dev) for a in geo.args())

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
            xs = dev_in[k].to(storage)
            s = pl.cone_projection3d(xs, geo.detector_shape, *args_geo, hardware_interp=hw,
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

    # at least 16 steps: the first upload and the last download are the only
    # copies no step's projections hide (about 2 % of 8 steps, 1 % of 16)
    e2e_steps = max(16, args.steps)
    e2e_run(max(args.warmup, 3))
    torch.cuda.synchronize()
    pl.check_device_errors(dev)
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
    pl.check_device_errors(dev)  # a bounded device wait that gave up would void the run
    del dev_in, host_in
    torch.cuda.empty_cache()

    # ---- roofline of the dominant kernel, against the L2 copy bandwidth
    # measured here (the taps are served on chip; HBM traffic is `traffic`)
    es = 2 if storage != torch.float32 else 4
    es_s = 2 if sino_storage != torch.float32 else 4
    S = count_samples(cfg, dev)
    f_ms, b_ms = statistics.mean(fwd_ms), statistics.mean(back_ms)
    fwd_bytes = S * 8 * es + n_proj * H * W * es_s
    back_bytes = updates(cfg) * 4 * es_s + Z * Y * X * 4
    try:
        l2 = measure_l2_peak(dev)
    except Exception as exc:  # the probe needs NVRTC; report its absence instead of a number
        l2 = {"gbs": None, "how": "L2 probe failed: %s" % exc}
    hbm_peak, peak_kind = measured_peaks()
    if f_ms >= b_ms:
        dom, dom_bytes, dom_ms = "cone_fp_padded_kernel (forward)", fwd_bytes, f_ms
    else:
        dom, dom_bytes, dom_ms = "cone_bp_tma_kernel (backprojection)", back_bytes, b_ms
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    ncu_key = (args.workload, args.storage, sino_storage_name(args), hw)
    roofline = {"bound": "issue", "kernel": dom, "achieved": achieved, "peak": l2["gbs"], "unit": "GB/s",
                "frac": achieved / l2["gbs"] if l2["gbs"] else None,
                "peak_source": "L2 read bandwidth measured in this run (%s)" % l2["how"],
                "traffic": args.traffic_bytes if args.traffic_bytes is not None else NCU_DRAM_BYTES.get(ncu_key)
                if f_ms >= b_ms else None,
                "algorithmic_bytes_per_launch": dom_bytes,
                "hbm_peak": hbm_peak, "hbm_peak_source": "%s HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs)"
                % peak_kind if peak_kind == "measured" else "fallback 6.65 TB/s",
                "ncu": NCU_FORWARD_COUNTERS.get(ncu_key) if f_ms >= b_ms else None,
                "note": "algorithmic bytes = 8 taps x element size per ray sample (+ sinogram), over the live CUDA-event "
                        "time; the limiter is instruction issue (ncu), not bytes: see ncu.issue_active"}

    line = {
        "metric": METRIC, "value": value, "unit": "GUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "storage": args.storage,
        "sinogram_storage": sino_storage_name(args), "data": "synthetic",
        "config": config_block(args, cfg),
        "plain_fp32_value": fp32_gups,
        "storage_over_fp32": (value / fp32_gups) if fp32_gups else None,
        "bf16": bf16,
        "kernels": {"forward_ms": f_ms, "backprojection_ms": b_ms, "ray_samples": S,
                    "forward_gsamples_per_s": S / (f_ms / 1e3) / 1e9,
                    "backprojection_gups": updates(cfg) / (b_ms / 1e3) / 1e9},
        "roofline": roofline,
        "e2e": {"value": e2e_value, "unit": "GUPS",
                "h2d_bytes_per_step": host_in_bytes(cfg), "d2h_bytes_per_step": Z * Y * X * 4, "steps": e2e_steps,
                "api": "pyronn_layers.cone_projection3d + cone_backprojection3d (the scan's geometry as device "
                       "tensors, made once)",
                "input": "FP32 volume in pinned host memory, converted to the storage dtype on the device inside "
                         "the timed region",
                "overlap": "two slots: the H2D copy of step i+1 and the D2H copy of step i run on their own "
                           "streams during step i's projections; every step's input and result cross the host "
                           "link inside the timed region"},
        # (+1 per step where the backprojection pairs a 16-bit sinogram: at
        # least 100 voxels per detector pixel; +1 where the forward scans a
        # 16-bit volume's range before its cell copy)
        "gpu_launches": (LAUNCHES_PER_STEP[hw] + int(not hw and sino_storage != torch.float32
                                                    and Z * Y * X >= 100 * H * W)
                         + int(not hw and args.storage != "fp32")) * args.steps,
        "clocks": clocks,
    }

    # ---- baselines (rank 0, N = 1): the CPU oracle on a bounded sample, the
    # accuracy of the GPU results against it, and the reference's own CUDA
    # kernels built from its sources -- all outside the timed regions
    if world == 1 and not args.no_cpu_baseline:
        vol_np = vol32.cpu().numpy()[None]
        sino_np = sino.float().cpu().numpy()
        gups, desc, threads, outs = cpu_sample(cfg, geo, vol_np, sino_np)
        line["cpu_baseline"] = {"value": gups, "unit": "GUPS", "cores": threads, "kind": "port", "sample": desc}
        nv, z0, ns = sample_spec(cfg)
        ours_f = sino[0, :nv].float().cpu().numpy()
        ours_b = back[0, z0:z0 + ns].float().cpu().numpy()
        line["accuracy"] = {
            "forward_rel_l2_vs_fp64": rel_l2(ours_f, outs["fwd"]),
            "backprojection_rel_l2_vs_fp64": rel_l2(ours_b, outs["back"]),
            "note": "forward: %s storage of the FP32 phantom, %s sinogram, vs the FP64 oracle on the FP32 "
                    "phantom (%d view); backprojection: same sinogram, FP32 volume, %d z-slices"
                    % (args.storage, sino_storage_name(args), nv, ns)}
        if bf16 is not None:
            f16, s16_all, b16 = bf16_outputs
            ref_b16 = oracle_slab(cfg, geo, s16_all)
            bf16["forward_rel_l2_vs_fp64"] = rel_l2(f16, outs["fwd"])
            bf16["backprojection_rel_l2_vs_fp64"] = rel_l2(b16, ref_b16)
            bf16["fwd_back_rel_l2_bound"] = 1e-3
            bf16["note"] = ("forward: BF16 storage of the FP32 phantom and a BF16 sinogram vs the FP64 oracle on the "
                            "FP32 phantom; the rounding of BF16 storage alone (2^-9 relative, RMS 1.1e-3 for "
                            "uniform rounding) exceeds the 1e-3 bound; FP16 storage meets it (accuracy above)")
        del sino_np
        line["reference_gpu"] = reference_gpu(cfg, geo, vol32, dev, f_ms, b_ms, fp32_gups or value, value, args)
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


def run_serving_sweep(args):
    """Serving capacity (config 5's mix): the same seeded trace at stepped
    Poisson rates and closed-loop (every request queued at t = 0), through the
    continuous-batching server and through the plain one-job-per-launch FP32
    path on the same GPU.  Per rate: offered and achieved GUPS, p50 / p99
    latency.  Reported: each path's saturation GUPS (closed loop), the highest
    rate whose achieved GUPS keeps up with the offered load (within 5 %), and
    the highest rate whose p99 stays under the stated bound."""
    import torch

    from pyronn_layers import serving
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    geos = serving.standard_geometries()
    rates = [float(r) for r in args.rates.split(",")]
    p99_bound_ms = args.p99_bound_ms
    classes = sorted({c for _, c in serving.poisson_trace(args.requests, 100.0, seed=7)}, key=str)
    server = serving.ProjectorServer(geos, device=dev, keep_results=False)
    warmup_s = server.warmup(classes, batch_sizes=(1, 2, 4, 8))
    warm = serving.make_jobs([(0.0, c) for c in classes], geos, seed=1)
    server.run_trace(warm, realtime=False)
    serving.run_plain(serving.make_jobs([(0.0, c) for c in classes], geos, seed=1), geos, device=dev,
                      realtime=False)
    rows = []
    with ClockSampler(physical_gpu_index(dev.index or 0)) as clk:
        for rate in rates:
            trace = serving.poisson_trace(args.requests, rate, seed=7)
            mean_updates = float(np.mean([geos[c.geometry].updates for _, c in trace]))
            offered = rate * mean_updates / 1e9 if math.isfinite(rate) else None
            server.batches, server.batch_sizes = 0, []
            jobs = serving.make_jobs(trace, geos, seed=1)
            s_srv = server.run_trace(jobs, realtime=True)
            jobs_plain = serving.make_jobs(trace, geos, seed=1)
            s_plain = serving.run_plain(jobs_plain, geos, device=dev, realtime=True, keep_results=False)
            rows.append({"rate_hz": rate if math.isfinite(rate) else "closed-loop", "offered_gups": offered,
                         "server": {"gups": s_srv.gups, "p50_ms": s_srv.p50_ms, "p99_ms": s_srv.p99_ms,
                                    "mean_batch": s_srv.mean_batch},
                         "plain": {"gups": s_plain.gups, "p50_ms": s_plain.p50_ms, "p99_ms": s_plain.p99_ms}})

    def summary(path):
        fin = [r for r in rows if r["offered_gups"] is not None]
        closed = [r[path]["gups"] for r in rows if r["offered_gups"] is None]
        keeps = [r["rate_hz"] for r in fin if r[path]["gups"] >= 0.95 * r["offered_gups"]]
        under = [r["rate_hz"] for r in fin if r[path]["p99_ms"] <= p99_bound_ms]
        return {"saturation_gups": max(closed) if closed else None,
                "max_sustained_gups": max([r[path]["gups"] for r in fin if r["rate_hz"] in keeps], default=None),
                "highest_rate_keeping_up_hz": max(keeps, default=None),
                "highest_rate_p99_under_bound_hz": max(under, default=None)}

    srv, plain = summary("server"), summary("plain")
    line = {
        "metric": METRIC, "value": srv["saturation_gups"] or srv["max_sustained_gups"], "unit": "GUPS", "n_gpus": 1,
        "steps": args.requests * len(rates), "warmup": 1, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "storage": "fp32/bf16 mix", "data": "synthetic",
        "config": {"workload": "serving-sweep", "requests_per_rate": args.requests, "rates_hz": args.rates,
                   "p99_bound_ms": p99_bound_ms,
                   "mix": "60% fan 512^2 (360 views, 1024 px), 30% cone 128^3 (180 views, 256^2), 10% cone 256^3 "
                          "(360 views, 512^2); forward/back 50/50; FP32/BF16 50/50",
                   "arrivals": "Poisson, seed 7; closed-loop: every request queued at t = 0"},
        "server": srv, "plain_one_job_per_launch_fp32": plain, "rows": rows, "server_startup_s": warmup_s,
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


FAN2D = dict(kind="fan", batch=64, volume=(512, 512), pixel_mm=0.5, views=360, detector=1024, det_mm=0.5,
             sid_mm=750.0, sdd_mm=1200.0, min_steps=1, accuracy_slices=1)
# one 256^2 slice per step; the tiny step is launch-bound, so a batch of
# slices per call is timed beside it (`batched`), and at least 200 steps are
# timed for a stable CUDA-event time
PAR2D = dict(kind="parallel", batch=1, volume=(256, 256), pixel_mm=1.0, views=180, detector=367, det_mm=1.0,
             min_steps=200, batched=256, accuracy_slices=1)
WORKLOADS_2D = {"fan2d": FAN2D, "par2d": PAR2D}


def geometry_2d(c):
    from pyronn_layers import geometry
    if c["kind"] == "fan":
        return geometry.FanBeam2D(c["volume"], (c["pixel_mm"],) * 2, c["detector"], c["det_mm"], c["views"],
                                  c["sid_mm"], c["sdd_mm"])
    return geometry.ParallelBeam2D(c["volume"], (c["pixel_mm"],) * 2, c["detector"], c["det_mm"], c["views"])


def reference_gpu_2d(c, g, vols, dev, ours, ours_fp32_gups, ours_gups):
    """The reference's own 2D kernels (cc/kernels/{par,fan}_{projector,
    backprojector}_2D_CudaKernel.cu.cc built unmodified into oracle/_ref by the
    oracle's recipe) through the op-layer restatement oracle/ref/ref_driver.cu:
    one launcher call per batch element, as the reference's ops loop
    (cc/ops/par_projector_2D_OPKernel.cc, fan_projector_2D_OPKernel.cc), FP32,
    default stream, 1 warm-up + the best of 5 timed calls per op (their
    per-call texture allocations make single calls noisy); outside our timed
    regions.  `ours` = (forward ms, backprojection ms, FP32 sinogram, FP32
    volume) of our kernels on the same FP32 inputs, for the ratios and the
    relative L2 distance of our results from theirs."""
    import ctypes

    import torch

    import oracle
    if not os.path.exists(oracle.REF_LIB):
        return {"unavailable": "oracle/_ref/libpyronn_ref.so not built (needs the reference sources)"}
    L = ctypes.CDLL(oracle.REF_LIB)
    B, (Y, X), n, W = c["batch"], c["volume"], c["views"], c["detector"]
    keep = []

    def dptr(a):
        t = torch.from_numpy(np.ascontiguousarray(np.asarray(a, dtype=np.float32)).reshape(-1)).to(dev)
        keep.append(t)
        return ctypes.c_void_p(t.data_ptr())

    def rows(a):
        return dptr(np.repeat(np.asarray(a, np.float32).reshape(1, -1), B, axis=0))

    geo = [rows(g.volume_origin), rows(g.detector_origin), rows(g.volume_spacing), rows(g.detector_spacing)]
    if c["kind"] == "fan":
        geo += [rows(g.sid), rows(g.sdd)]
    geo.append(rows(g.ray_vectors))
    vol = torch.from_numpy(np.ascontiguousarray(vols, dtype=np.float32)).to(dev)
    sino = torch.zeros(B * n * W, dtype=torch.float32, device=dev)
    back = torch.zeros(B * Y * X, dtype=torch.float32, device=dev)
    fwd = L.ref_fan_projection2d if c["kind"] == "fan" else L.ref_parallel_projection2d
    bwd = L.ref_fan_backprojection2d if c["kind"] == "fan" else L.ref_parallel_backprojection2d
    fargs = (ctypes.c_void_p(vol.data_ptr()), ctypes.c_void_p(sino.data_ptr()), B, Y, X, n, W, *geo)
    bargs = (ctypes.c_void_p(sino.data_ptr()), ctypes.c_void_p(back.data_ptr()), B, n, W, Y, X, *geo)

    def timed(fn, reps=5):
        if fn() != 0:
            raise RuntimeError("reference launcher failed")
        times = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            fn()
            e.record()
            torch.cuda.synchronize()
            times.append(s.elapsed_time(e))
        return min(times)

    try:
        fms = timed(lambda: fwd(*fargs))
        ref_sino = sino.clone()
        # their backprojection of OUR FP32 sinogram, so both backprojections
        # see the same input
        sino.copy_(ours[2].reshape(-1))
        bms = timed(lambda: bwd(*bargs))
    except RuntimeError as exc:
        return {"unavailable": str(exc)}
    gups = 2 * B * Y * X * n / ((fms + bms) / 1e3) / 1e9
    return {"value": gups, "unit": "GUPS", "forward_ms": fms, "backprojection_ms": bms,
            "storage": "fp32 (the reference's only storage type)",
            "ours_fp32_over_reference": ours_fp32_gups / gups, "ours_over_reference": ours_gups / gups,
            "ours_fp32_forward_rel_l2_vs_reference": rel_l2(ours[2].reshape(-1).cpu().numpy(),
                                                            ref_sino.cpu().numpy()),
            "ours_fp32_backprojection_rel_l2_vs_reference": rel_l2(ours[3].reshape(-1).cpu().numpy(),
                                                                   back.cpu().numpy()),
            "what": "the reference's own 2D kernels (built unmodified for sm_100a) through a restatement of its TF "
                    "op layer (oracle/ref/ref_driver.cu): one launcher call per batch element, FP32, default "
                    "stream, 1 warm-up + the best of 5 timed calls per op"}


def run_2d(args):
    """2D workloads.  fan2d (config 2): 64 independent 512^2 slices at
    0.5 mm, 360 views over 2 pi, flat 1024-px detector at 0.5 mm, SID 750 /
    SDD 1200.  par2d (config 1): one 256^2 slice at 1.0 mm, 180 views over
    pi, 367-px detector at 1.0 mm.  One step = the projection of the batch +
    the backprojection of its sinograms; GUPS = 2 * batch * slice pixels *
    views / t.  Beside it: the plain FP32 path, the relative L2 error of the
    first slice against the FP64 oracle, and the reference's own kernels."""
    import torch

    from pyronn_layers import ops, phantoms
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    c = WORKLOADS_2D[args.workload]
    fan = c["kind"] == "fan"
    g = geometry_2d(c)
    seed0 = 100 if fan else 1
    vols = np.stack([phantoms.ellipse_phantom_2d(c["volume"], (c["pixel_mm"],) * 2, seed=seed0 + b)[0]
                     for b in range(c["batch"])])
    storage = {"bf16": torch.bfloat16, "fp16": torch.float16, "fp32": torch.float32}[args.storage]
    steps = max(args.steps, c["min_steps"])
    lib = ops._capi
    fwd_name = "pyronn_fan_projection2d" if fan else "pyronn_parallel_projection2d"
    bwd_name = "pyronn_fan_backprojection2d" if fan else "pyronn_parallel_backprojection2d"
    geo_extra = (g.sid, g.sdd) if fan else ()

    def run(store, batch_vols, graph=False):
        B = batch_vols.shape[0]
        units = B * c["volume"][0] * c["volume"][1] * c["views"]
        x = torch.from_numpy(batch_vols).to(dev, store)
        geo = ops.Geometry2D(B, dev, *g.args()[:4], g.ray_vectors, c["views"], *geo_extra)
        sino = torch.empty((B, c["views"], c["detector"]), dtype=store, device=dev)
        back = torch.empty((B,) + c["volume"], dtype=torch.float32, device=dev)
        code = ops.storage_code(store)
        ws = torch.empty(lib.workspace_size("pyronn_projection2d", B, *c["volume"], code), dtype=torch.uint8,
                         device=dev)
        ev = []

        def launch_fwd(s):
            lib.call(fwd_name, x.data_ptr(), sino.data_ptr(), code, code, B, *c["volume"], c["views"],
                     c["detector"], *geo.pointers(), geo.g, ws.data_ptr(), ws.numel(), s)

        def launch_bwd(s):
            lib.call(bwd_name, sino.data_ptr(), back.data_ptr(), code, 0, B, c["views"], c["detector"],
                     *c["volume"], *geo.pointers(), geo.g, s)

        if graph:
            # one step captured as a CUDA graph and replayed: the step without
            # the host's per-call cost
            side = torch.cuda.Stream(dev)
            with torch.cuda.stream(side):
                for _ in range(args.warmup):
                    launch_fwd(side.cuda_stream)
                    launch_bwd(side.cuda_stream)
            torch.cuda.synchronize(dev)
            cg = torch.cuda.CUDAGraph()
            with torch.cuda.graph(cg, stream=side):
                launch_fwd(side.cuda_stream)
                launch_bwd(side.cuda_stream)
            for _ in range(args.warmup):
                cg.replay()
            torch.cuda.synchronize(dev)
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0.record()
            for _ in range(steps):
                cg.replay()
            t1.record()
            torch.cuda.synchronize(dev)
            ms = t0.elapsed_time(t1)
            del cg
            ops.check_device_errors(dev)
            return {"gups": 2 * units * steps / (ms / 1e3) / 1e9, "ms": ms}

        def step():
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            s = torch.cuda.current_stream(dev).cuda_stream
            e[0].record()
            launch_fwd(s)
            e[1].record()
            launch_bwd(s)
            e[2].record()
            ev.append(e)

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        ev.clear()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record()
        for _ in range(steps):
            step()
        t1.record()
        torch.cuda.synchronize()
        ms = t0.elapsed_time(t1)
        f = statistics.mean(a.elapsed_time(b) for a, b, _ in ev)
        bk = statistics.mean(b.elapsed_time(c2) for _, b, c2 in ev)
        ops.check_device_errors(dev)
        return {"gups": 2 * units * steps / (ms / 1e3) / 1e9, "ms": ms, "forward_ms": f, "backprojection_ms": bk,
                "sino": sino, "back": back}

    with ClockSampler(physical_gpu_index(dev.index or 0)) as clk:
        r = run(storage, vols)
    r32 = run(torch.float32, vols) if storage != torch.float32 else r
    batched = None
    if c.get("batched"):
        rb = run(storage, np.repeat(vols[:1], c["batched"], axis=0))
        batched = {"value": rb["gups"], "unit": "GUPS", "slices_per_call": c["batched"],
                   "forward_ms": rb["forward_ms"], "backprojection_ms": rb["backprojection_ms"],
                   "note": "the same slice repeated, %d per call: the kernels' throughput without the per-call "
                           "launch cost that bounds the one-slice step" % c["batched"]}
        del rb
        rg = run(storage, vols, graph=True)
        batched["one_slice_graph_replay"] = {"value": rg["gups"], "unit": "GUPS", "ms_per_step": rg["ms"] / steps,
                                             "note": "the one-slice step captured once as a CUDA graph and replayed "
                                                     "%d times" % steps}

    def accuracy(res):
        import oracle
        k = c["accuracy_slices"]
        v = vols[:k]
        geo_args = g.args()
        if fan:
            ref_s = oracle.fan_projection2d(v, g.detector_shape, *geo_args)
        else:
            ref_s = oracle.parallel_projection2d(v, g.detector_shape, *geo_args)
        ours_s = res["sino"][:k].float().cpu().numpy()
        # the oracle backprojects our sinogram: the backprojection's own error
        if fan:
            ref_b = oracle.fan_backprojection2d(ours_s, c["volume"], *geo_args)
        else:
            ref_b = oracle.parallel_backprojection2d(ours_s, c["volume"], *geo_args)
        return {"forward_rel_l2_vs_fp64": rel_l2(ours_s.reshape(-1), ref_s.reshape(-1)),
                "backprojection_rel_l2_vs_fp64": rel_l2(res["back"][:k].cpu().numpy().reshape(-1),
                                                        ref_b.reshape(-1)),
                "slices": k}

    acc = {args.storage: accuracy(r)}
    if r32 is not r:
        acc["fp32"] = accuracy(r32)
    acc["note"] = ("forward: our sinogram of the first slice (stored as named) against the FP64 oracle on the FP32 "
                   "phantom; backprojection: the FP64 oracle's backprojection of the same sinogram")
    ref = reference_gpu_2d(c, g, vols, dev, (r32["forward_ms"], r32["backprojection_ms"], r32["sino"], r32["back"]),
                           r32["gups"], r["gups"])
    line = {
        "metric": METRIC, "value": r["gups"], "unit": "GUPS", "n_gpus": 1, "steps": steps, "warmup": args.warmup,
        "ms_per_step": r["ms"] / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "storage": args.storage, "data": "synthetic",
        "config": {"workload": args.workload, "geometry": c["kind"], "batch": c["batch"],
                   "slice": list(c["volume"]), "pixel_mm": c["pixel_mm"], "views": c["views"],
                   "detector_px": c["detector"], "det_mm": c["det_mm"],
                   **({"sid_mm": c["sid_mm"], "sdd_mm": c["sdd_mm"]} if fan else {}),
                   "phantom": "10 seeded ellipses per slice"},
        "plain_fp32_value": r32["gups"],
        "kernels": {"forward_ms": r["forward_ms"], "backprojection_ms": r["backprojection_ms"]},
        "accuracy": acc, "batched": batched, "reference_gpu": ref,
        "clocks": clk.summary(),
    }
    print(json.dumps(line))


DIFFCONE = dict(batch=4, volume=(128, 128, 128), voxel_mm=1.0, views=180, detector=(256, 256), pixel_mm=1.5,
                sid_mm=600.0, sdd_mm=1000.0, i0=1e5, unrolled=20)


def run_diffcone(args):
    """Differentiable cone beam (config 4): a batch of 4 volumes of 128^3 at
    1.0 mm, 180 views over 2 pi, 256 x 256 detector at 1.5 mm, SID 600 / SDD
    1000; y = -log(Poisson(1e5 exp(-A x_true)) / 1e5); one training step =
    20 unrolled gradient steps x <- x - lr_k A^T (A x - y) from x = 0 (each
    wrapped in activation checkpointing), the loss 1/2 |A x_20 - y|^2, its
    backward pass through every step (checkpointed steps recomputed) and an
    Adam update of the 20 learned step lengths.  The projector's gradient is
    the exact transpose (matched adjoint) unless --unmatched.  GUPS = projector
    and backprojector calls per training step (counted) x 4 x 128^3 x 180 / t.
    Reported with and without checkpointing: time per step and peak memory."""
    import torch

    from pyronn_layers import geometry, ops, phantoms, recon
    if int(os.environ.get("RANK", "0")) != 0:
        return
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
    c = DIFFCONE
    geo = geometry.ConeBeam3D(c["volume"], (c["voxel_mm"],) * 3, c["detector"], (c["pixel_mm"],) * 2, c["views"],
                              c["sid_mm"], c["sdd_mm"])
    vols = np.stack([phantoms.ellipsoid_phantom_3d(c["volume"], geo.volume_spacing, seed=400 + b)[0]
                     for b in range(c["batch"])]) * np.float32(0.02)
    x_true = torch.from_numpy(vols).to(dev)
    y_dev = recon.poisson_sinogram(ops.cone_projection3d(x_true, geo.detector_shape, *geo.args()), c["i0"], seed=4)
    y_host = y_dev.cpu().pin_memory()
    units = c["batch"] * int(np.prod(c["volume"])) * c["views"]

    def step_length(matched):
        """1 / the largest eigenvalue of A^T A (power iteration, 12 steps):
        the step that keeps the unrolled descent stable, the learned step
        lengths' starting value."""
        x = torch.rand_like(x_true)
        lam = 1.0
        with torch.no_grad():
            for _ in range(12):
                ax = ops.cone_projection3d(x, geo.detector_shape, *geo.args())
                atax = (ops.cone_backprojection3d_matched(ax, geo.volume_shape, *geo.args()) if matched
                        else ops.cone_backprojection3d(ax, geo.volume_shape, *geo.args()))
                lam = float(atax.norm() / x.norm())
                x = atax / atax.norm()
        return 1.0 / lam

    calls = {"n": 0}
    counted = {}
    for name in ("_run_cone", "_run_matched"):
        fn = getattr(ops, name)

        def wrap(*a, _fn=fn, **k):
            calls["n"] += 1
            return _fn(*a, **k)
        counted[name] = fn
        setattr(ops, name, wrap)

    def run(ckpt, steps, warmup, matched, lr0):
        net = recon.UnrolledGradientDescent(geo, n_steps=c["unrolled"], init_lr=lr0, matched_adjoint=matched,
                                            checkpoint=ckpt).to(dev)
        opt = torch.optim.Adam(net.parameters(), lr=1e-2)
        y = torch.empty_like(y_dev)
        losses = []

        def step():
            y.copy_(y_host, non_blocking=True)  # this step's target sinogram from pinned host memory
            opt.zero_grad(set_to_none=True)
            xk = net(torch.zeros_like(x_true), y)
            r = ops.cone_projection3d(xk, geo.detector_shape, *geo.args(), matched_adjoint=matched) - y
            loss = 0.5 * (r.double() ** 2).sum()
            loss.backward()
            opt.step()
            losses.append(loss.detach().to("cpu", non_blocking=True))  # the step's result back on the host

        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        ops.check_device_errors(dev)
        torch.cuda.reset_peak_memory_stats(dev)
        calls["n"] = 0
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(steps):
            step()
        e.record()
        torch.cuda.synchronize()
        ops.check_device_errors(dev)
        return {"ms_per_step": s.elapsed_time(e) / steps, "calls_per_step": calls["n"] / steps,
                "peak_mem_gib": torch.cuda.max_memory_allocated(dev) / 2 ** 30,
                "loss_first": float(losses[0]), "loss_last": float(losses[-1])}

    try:
        lr_u, lr_m = step_length(False), step_length(True)
        with ClockSampler(physical_gpu_index(dev.index or 0)) as clk:
            ck = run(True, args.steps, args.warmup, False, lr_u)
        plain = run(False, max(1, args.steps // 2), 1, False, lr_u)
        exact = run(True, 2, 1, True, lr_m)
    finally:
        for name, fn in counted.items():
            setattr(ops, name, fn)
    gups = ck["calls_per_step"] * units / (ck["ms_per_step"] / 1e3) / 1e9
    ck["initial_step_length"], exact["initial_step_length"] = lr_u, lr_m
    exact["gups"] = exact["calls_per_step"] * units / (exact["ms_per_step"] / 1e3) / 1e9
    line = {
        "metric": "differentiable cone-beam training step (config 4) GUPS", "value": gups, "unit": "GUPS",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ck["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "storage": "fp32",
        "data": "synthetic (seeded ellipsoid phantoms, Poisson noise)",
        "config": {"workload": "diffcone", "batch": c["batch"], "volume": list(c["volume"]), "voxel_mm": c["voxel_mm"],
                   "views": c["views"], "detector_hw": list(c["detector"]), "pixel_mm": c["pixel_mm"],
                   "sid_mm": c["sid_mm"], "sdd_mm": c["sdd_mm"], "i0": c["i0"], "unrolled_steps": c["unrolled"],
                   "adjoint": "the reference's pairing: the voxel-driven backprojector as the projector's gradient "
                              "(exact transpose: see exact_adjoint)",
                   "optimizer": "Adam on the 20 learned step lengths"},
        "checkpointed": ck, "no_checkpointing": plain,
        "exact_adjoint": dict(exact, note="the same training step with the matched (exact-transpose, atomic "
                                          "scatter) backprojector as gradient and in the unrolled steps; 1 warm-up "
                                          "+ 2 timed steps"),
        "updates_per_op": units,
        "e2e": {"value": gups, "unit": "GUPS", "h2d_bytes_per_step": int(y_host.numel() * 4),
                "d2h_bytes_per_step": 8,
                "note": "the training step is timed through the public API with the target sinogram uploaded and "
                        "the loss downloaded every step"},
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
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["serving", "serving-sweep", "fan2d", "par2d", "fdk", "diffcone"],
                    default="cone512")

    ap.add_argument("--requests", type=int, default=2000, help="serving: number of requests")
    ap.add_argument("--rate", type=float, default=100.0, help="serving: Poisson arrival rate (1/s)")
    ap.add_argument("--rates", default="300,600,900,1200,1800,inf",
                    help="serving-sweep: arrival rates (1/s; inf = closed loop)")
    ap.add_argument("--p99-bound-ms", type=float, default=100.0, help="serving-sweep: the p99 latency bound")
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
    if args.workload in WORKLOADS_2D:
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the 2D workloads are measured on the GPU arm "
                                                                   "only (their reference_gpu block times the "
                                                                   "reference's kernels)"}))
            return
        run_2d(args)
        return
    if args.workload == "diffcone":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the training workload is measured on the GPU arm "
                                                                   "only"}))
            return
        run_diffcone(args)
        return
    if args.workload == "fdk":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no FDK filter"}))
            return
        run_fdk(args)
        return
    if args.workload == "serving-sweep":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the serving stream has no CPU reference arm"}))
            return
        run_serving_sweep(args)
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
