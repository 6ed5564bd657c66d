"""Filtered backprojection on top of the projector ops: FDK for circular
cone-beam scans, FBP for 2D parallel- and fan-beam scans.

The reference's ops have no filtering step (the PYRO-NN package filters in
Python); here the filtering runs in the library (``pyronn_fdk_filter``: Feldkamp
cosine weights and the Ram-Lak / Shepp-Logan ramp kernels of Kak & Slaney,
convolved along each detector row), then the reference-compatible
backprojection op does the rest with the FDK scale as its multiplier.

Full-circle cone scans (no short-scan / Parker weighting).  The 2D fan
backprojection op weights by the reference's 1 / |x - source|^2, not the
exact FBP's 1 / U^2 (depth along the central ray), so fan FBP images carry a
cos^2(fan angle) shading away from the centre -- a property of the
reference's op that is kept.
"""
from __future__ import annotations

import math

import torch

from . import _capi, ops

FILTERS = {"ram-lak": _capi.FILTER_RAM_LAK, "shepp-logan": _capi.FILTER_SHEPP_LOGAN}


def _filter_code(name: str) -> int:
    try:
        return FILTERS[name]
    except KeyError:
        raise ValueError("filter must be one of %s, got %r" % (sorted(FILTERS), name)) from None


def _run_filter(x: torch.Tensor, params, weight_output: bool, out_dtype) -> torch.Tensor:
    sdd, dv, du, cv, cu, code = params
    x4 = x if x.dim() == 4 else x.unsqueeze(2)  # 2D sinograms are rows of height 1
    x4 = x4.contiguous()
    od = x.dtype if out_dtype is None else out_dtype
    ops.storage_code(od)
    out = torch.empty(x4.shape, dtype=od, device=x.device)
    b, n, h, w = x4.shape
    with torch.cuda.device(x.device):
        _capi.call("pyronn_fdk_filter", x4.data_ptr(), out.data_ptr(), ops.storage_code(x4.dtype),
                   ops.storage_code(od), b, n, h, w, sdd, dv, du, cv, cu, code, int(weight_output),
                   ops._stream(x.device))
        if ops._sync_error_checks:  # otherwise ops.device_errors() reads the filter's word
            ops.check_device_errors(x.device)
    return out if x.dim() == 4 else out.squeeze(2)


class _FdkFilter(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, params, out_dtype):
        ctx.params = params
        ctx.in_dtype = x.dtype
        return _run_filter(x, params, False, out_dtype)

    @staticmethod
    def backward(ctx, grad):
        # the ramp kernel is symmetric: the adjoint weights after filtering
        return _run_filter(grad.contiguous(), ctx.params, True, ctx.in_dtype), None, None


def fdk_filter(projections: torch.Tensor, sdd: float, detector_spacing, principal_point=None,
               filter: str = "ram-lak", out_dtype=torch.float32) -> torch.Tensor:
    """Cosine-weight (sdd > 0) and ramp-filter every detector row.

    projections: [batch, n_proj, det_h, det_w] or [batch, n_proj, det_w] CUDA
    tensor; detector_spacing = (dv, du) mm (a single du for 2D);
    principal_point = (cv, cu) pixel indices (default: detector centre);
    sdd = 0 filters without weighting (parallel beam)."""
    if not projections.is_cuda:
        raise ValueError("projections must be a CUDA tensor")
    if projections.dim() not in (3, 4):
        raise ValueError("projections must be [batch, n_proj, (det_h,) det_w]")
    h = projections.shape[2] if projections.dim() == 4 else 1
    w = projections.shape[-1]
    if isinstance(detector_spacing, (int, float)):
        dv, du = 1.0, float(detector_spacing)
    else:
        dv, du = float(detector_spacing[0]), float(detector_spacing[-1])
    cv, cu = ((h - 1) / 2.0, (w - 1) / 2.0) if principal_point is None else principal_point
    params = (float(sdd), dv, du, float(cv), float(cu), _filter_code(filter))
    return _FdkFilter.apply(projections, params, out_dtype)


def fdk_reconstruct(sinogram: torch.Tensor, geo, filter: str = "ram-lak", hardware_interp: bool = False,
                    out_dtype=torch.float32) -> torch.Tensor:
    """FDK reconstruction of a full-circle cone-beam scan.

    geo: a geometry.ConeBeam3D (centred detector); sinogram [batch, n_proj,
    det_h, det_w].  Filters, then backprojects with projection_multiplier =
    SID * SDD * pi / n_proj (the FDK constant for the op's 1 / w^2
    weighting, w the depth along the principal ray in mm)."""
    n_proj = geo.detector_shape[0]
    q = fdk_filter(sinogram, geo.sdd, geo.detector_spacing, None, filter)
    mult = torch.tensor([geo.sid * geo.sdd * math.pi / n_proj], dtype=torch.float32)
    return ops.cone_backprojection3d(q, geo.volume_shape, geo.volume_origin, geo.volume_spacing,
                                     geo.projection_matrices, geo.step_size, mult,
                                     hardware_interp=hardware_interp, out_dtype=out_dtype)


def fbp_reconstruct_2d(sinogram: torch.Tensor, geo, filter: str = "ram-lak", out_dtype=torch.float32):
    """FBP of a 2D scan: geo a geometry.ParallelBeam2D (over pi) or FanBeam2D
    (over 2 pi); sinogram [batch, n_proj, det_w]."""
    du = float(geo.detector_spacing[0])
    cu = -float(geo.detector_origin[0]) / du
    fan = hasattr(geo, "sid")
    sdd = float(geo.sdd[0]) if fan else 0.0
    q = fdk_filter(sinogram, sdd, (1.0, du), (0.0, cu), filter)
    if fan:
        return ops.fan_backprojection2d(q, geo.volume_shape, *geo.args(), out_dtype=out_dtype)
    return ops.parallel_backprojection2d(q, geo.volume_shape, *geo.args(), out_dtype=out_dtype)
