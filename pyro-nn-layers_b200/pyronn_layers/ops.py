"""The six projector ops with the reference's op surface, on torch CUDA tensors.

Names, argument order and argument meaning follow the reference's TF op
registrations (the TF-generated snake_case wrappers), e.g.
``cone_projection3d(volume, projection_shape, volume_origin, volume_spacing,
projection_matrices, step_size, projection_multiplier, hardware_interp=False)``
mirrors ``REGISTER_OP("ConeProjection3D")`` (cc/ops/cone_projector_3D_OPKernel.cc:34-43).

* The data tensor carries the mandatory batch dimension (CHANGELOG 0.0.4) and
  lives on a CUDA device; float32, bfloat16 and float16 storage are accepted;
  the output has the input's dtype unless ``out_dtype`` says otherwise (sums
  accumulate in FP32 either way).
* Shape arguments may be tensors (any device) or sequences of ints.
* Geometry tensors may be batched (leading dim == batch, one row per batch
  element as the reference's ``flat_outer_dims(index)`` rows) or unbatched /
  leading dim 1 (shared by the whole batch).
* Every op is differentiable w.r.t. its data input; the gradient of a
  projector is the paired backprojector applied to the incoming gradient and
  vice versa (the pairing the PYRO-NN package registers for these ops); the
  geometry inputs get no gradient.
* Errors raise :class:`~pyronn_layers._capi.PyronnError` (the reference exits
  the process or ignores CUDA errors).  Kernels with bounded device-side waits
  (the TMA-staged cone backprojector, the tensor-core FDK filter) report a
  wait that gave up through a device flag after the call has returned: the
  ops fold those flags into a per-device word on the stream, without
  synchronising, and :func:`check_device_errors` (or ``device_errors``) reads
  it at a point where the caller synchronises anyway;
  ``set_sync_error_checks(True)`` or ``PYRONN_SYNC_ERROR_CHECKS=1`` makes
  every such op synchronise and raise at once instead.
"""
from __future__ import annotations

import collections
import ctypes
import hashlib
import math
import os
from typing import Sequence

import numpy as np
import torch

from . import _capi

_DTYPES = {torch.float32: _capi.FLOAT32, torch.bfloat16: _capi.BFLOAT16, torch.float16: _capi.FLOAT16}


def storage_code(dtype: torch.dtype) -> int:
    try:
        return _DTYPES[dtype]
    except KeyError:
        raise TypeError("unsupported storage dtype %s (float32, bfloat16, float16)" % dtype) from None


def _shape(shape, n: int, what: str) -> list:
    if isinstance(shape, torch.Tensor):
        vals = [int(v) for v in shape.detach().reshape(-1).cpu().tolist()]
    else:
        vals = [int(v) for v in shape]
    if len(vals) != n:
        raise ValueError("%s must have %d entries, got %d" % (what, n, len(vals)))
    if any(v <= 0 for v in vals):
        raise ValueError("%s entries must be positive: %s" % (what, vals))
    return vals


# Device copies of host geometry (numpy arrays, sequences, CPU tensors), by
# content: a copy from pageable host memory waits for the stream's queued
# work, so a loop that passes the same host geometry to every call would
# otherwise serialise host and device at each call.  Bounded, least recently
# used first out; keyed by the bytes, so a changed array is a new entry.
_HOST_GEOM_CACHE: "collections.OrderedDict" = collections.OrderedDict()
_HOST_GEOM_CACHE_SIZE = 64


def _host_geometry_on_device(t, device) -> torch.Tensor:
    a = np.ascontiguousarray(t.numpy() if isinstance(t, torch.Tensor) else np.asarray(t), dtype=np.float32)
    dev = torch.device(device)
    if dev.type == "cuda" and dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    key = (str(dev), a.shape, hashlib.blake2b(a.tobytes(), digest_size=16).digest())
    hit = _HOST_GEOM_CACHE.get(key)
    if hit is not None:
        _HOST_GEOM_CACHE.move_to_end(key)
        return hit
    d = torch.from_numpy(a.copy()).to(dev)
    if dev.type == "cuda":
        # the copy is complete before any stream uses the cached tensor
        torch.cuda.current_stream(dev).synchronize()
    _HOST_GEOM_CACHE[key] = d
    while len(_HOST_GEOM_CACHE) > _HOST_GEOM_CACHE_SIZE:
        _HOST_GEOM_CACHE.popitem(last=False)
    return d


def _geom(t, batch: int, row_shape: Sequence[int], device, what: str):
    """Returns (contiguous float32 tensor [g, *row_shape] on device, g)."""
    if not (isinstance(t, torch.Tensor) and t.device.type == "cuda"):
        t = _host_geometry_on_device(t.detach() if isinstance(t, torch.Tensor) else t, device)
    t = torch.as_tensor(t, dtype=torch.float32)
    row_numel = 1
    for s in row_shape:
        row_numel *= int(s)
    if t.numel() == row_numel:
        g = 1
    elif t.numel() == row_numel * batch and t.dim() >= 1 and t.shape[0] == batch:
        g = batch
    else:
        raise ValueError("%s: expected %s per batch element (shared, or batched with leading dim %d), got shape %s"
                         % (what, list(row_shape), batch, tuple(t.shape)))
    t = t.reshape((g,) + tuple(int(s) for s in row_shape)).to(device=device, dtype=torch.float32).contiguous()
    return t, g


def _common_g(*gs: int) -> int:
    g = max(gs)
    return g


def _expand(t: torch.Tensor, g: int) -> torch.Tensor:
    if t.shape[0] == g:
        return t
    return t.expand((g,) + tuple(t.shape[1:])).contiguous()


def _check_data(x: torch.Tensor, ndim: int, what: str):
    if not isinstance(x, torch.Tensor):
        raise TypeError("%s must be a torch.Tensor" % what)
    if not x.is_cuda:
        raise ValueError("%s must be a CUDA tensor (the projector ops have no CPU implementation)" % what)
    if x.dim() != ndim:
        raise ValueError("%s must have %d dims [batch, ...], got shape %s" % (what, ndim, tuple(x.shape)))
    storage_code(x.dtype)
    return x.contiguous()


def _stream(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


# ------------------------------------------------------------ device error flags

_sync_error_checks = os.environ.get("PYRONN_SYNC_ERROR_CHECKS", "0") not in ("", "0")
_error_words = {}  # device index -> int32 [1]: OR of the device error flags seen


def set_sync_error_checks(enabled: bool) -> None:
    """With True, every op with bounded device-side waits synchronises after
    its launch and raises PyronnDeviceError if a wait gave up (debugging);
    with False (the default) the flags accumulate on the device for
    check_device_errors."""
    global _sync_error_checks
    _sync_error_checks = bool(enabled)


def _error_word(device):
    idx = device.index if device.index is not None else torch.cuda.current_device()
    w = _error_words.get(idx)
    if w is None:
        if torch.cuda.is_current_stream_capturing():
            return None  # created outside captures only (a capture's pool may be freed with its graph)
        w = torch.zeros(1, dtype=torch.int32, device=torch.device("cuda", idx))
        _error_words[idx] = w
    return w


def note_workspace_error(workspace: torch.Tensor, device) -> None:
    """Folds the device error flag that the call just enqueued on the current
    stream leaves in its workspace header (first 32-bit word) into the
    device's error word, on that stream (no synchronisation)."""
    flag = workspace[:4].view(torch.int32)
    if _sync_error_checks and not torch.cuda.is_current_stream_capturing():
        value = int(flag.item())
        if value:
            raise _capi.PyronnDeviceError(value, "cone backprojection")
        return
    w = _error_word(device)
    if w is not None:
        w.bitwise_or_(flag)


def device_errors(device=None, clear: bool = True) -> int:
    """Synchronises the device and returns the OR of the device error flags
    raised since the last call (pyronn_layers ops' workspaces and the
    tensor-core FDK filter's word): 0 when every bounded wait completed,
    _capi.DEVICE_ERROR_WAIT_TIMEOUT when one gave up and its output was not
    written."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    torch.cuda.synchronize(dev)
    value = 0
    w = _error_words.get(dev.index)
    if w is not None:
        value = int(w.item())
        if clear:
            w.zero_()
    flag = ctypes.c_int(0)
    with torch.cuda.device(dev):
        _capi.call("pyronn_fdk_error", _stream(dev), ctypes.byref(flag))
    return value | flag.value


def check_device_errors(device=None) -> None:
    """Raises PyronnDeviceError if device_errors() reports a flag."""
    value = device_errors(device)
    if value:
        raise _capi.PyronnDeviceError(value)


# ---------------------------------------------------------------- geometry packs


class Geometry2D:
    """Prepared device geometry of a 2D op (parallel or fan)."""

    def __init__(self, batch, device, volume_origin, detector_origin, volume_spacing, detector_spacing, rays,
                 n_proj, sid=None, sdd=None):
        vo, g1 = _geom(volume_origin, batch, (2,), device, "volume_origin")
        do, g2 = _geom(detector_origin, batch, (1,), device, "detector_origin")
        vs, g3 = _geom(volume_spacing, batch, (2,), device, "volume_spacing")
        ds, g4 = _geom(detector_spacing, batch, (1,), device, "detector_spacing")
        rv, g5 = _geom(rays, batch, (n_proj, 2), device, "ray_vectors")
        gs = [g1, g2, g3, g4, g5]
        self.fan = sid is not None
        if self.fan:
            si, g6 = _geom(sid, batch, (1,), device, "source_2_isocenter_distance")
            sd, g7 = _geom(sdd, batch, (1,), device, "source_2_detector_distance")
            gs += [g6, g7]
        g = _common_g(*gs)
        self.g = g
        self.volume_origin = _expand(vo, g)
        self.detector_origin = _expand(do, g)
        self.volume_spacing = _expand(vs, g)
        self.detector_spacing = _expand(ds, g)
        self.rays = _expand(rv, g)
        if self.fan:
            self.sid = _expand(si, g)
            self.sdd = _expand(sd, g)

    def pointers(self):
        p = [self.volume_origin.data_ptr(), self.detector_origin.data_ptr(), self.volume_spacing.data_ptr(),
             self.detector_spacing.data_ptr()]
        if self.fan:
            p += [self.sid.data_ptr(), self.sdd.data_ptr()]
        p.append(self.rays.data_ptr())
        return p


class GeometryCone:
    """Prepared device geometry of a cone op."""

    def __init__(self, batch, device, volume_origin, volume_spacing, projection_matrices, step_size,
                 projection_multiplier, n_proj):
        vo, g1 = _geom(volume_origin, batch, (3,), device, "volume_origin")
        vs, g2 = _geom(volume_spacing, batch, (3,), device, "volume_spacing")
        pm, g3 = _geom(projection_matrices, batch, (n_proj, 3, 4), device, "projection_matrices")
        st, g4 = _geom(step_size, batch, (1,), device, "step_size")
        mu, g5 = _geom(projection_multiplier, batch, (1,), device, "projection_multiplier")
        g = _common_g(g1, g2, g3, g4, g5)
        self.g = g
        self.n_proj = n_proj
        self.volume_origin = _expand(vo, g)
        self.volume_spacing = _expand(vs, g)
        self.projection_matrices = _expand(pm, g)
        self.step_size = _expand(st, g)
        self.projection_multiplier = _expand(mu, g)

    def pointers(self):
        return [self.volume_origin.data_ptr(), self.volume_spacing.data_ptr(),
                self.projection_matrices.data_ptr(), self.step_size.data_ptr(),
                self.projection_multiplier.data_ptr()]


# ------------------------------------------------------------- raw launches


def _out_dtype(x: torch.Tensor, out_dtype) -> torch.dtype:
    d = x.dtype if out_dtype is None else out_dtype
    storage_code(d)
    return d


def _run_2d(forward: bool, x: torch.Tensor, out_dims, geo: Geometry2D, out_dtype=None,
            workspace=None) -> torch.Tensor:
    batch = x.shape[0]
    dev = x.device
    od = _out_dtype(x, out_dtype)
    if forward:
        vol_y, vol_x = x.shape[1], x.shape[2]
        n_proj, det_w = out_dims
        out = torch.empty((batch, n_proj, det_w), dtype=od, device=dev)
        fn = "pyronn_fan_projection2d" if geo.fan else "pyronn_parallel_projection2d"
        dims = [batch, vol_y, vol_x, n_proj, det_w]
        # workspace for the x- and y-fastest bilinear cell copies of the batch
        ws_bytes = _capi.workspace_size("pyronn_projection2d", batch, vol_y, vol_x, storage_code(x.dtype))
        if workspace is None or workspace.numel() < ws_bytes:
            workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
        ws = [workspace.data_ptr(), workspace.numel()]
    else:
        n_proj, det_w = x.shape[1], x.shape[2]
        vol_y, vol_x = out_dims
        out = torch.empty((batch, vol_y, vol_x), dtype=od, device=dev)
        fn = "pyronn_fan_backprojection2d" if geo.fan else "pyronn_parallel_backprojection2d"
        dims = [batch, n_proj, det_w, vol_y, vol_x]
        ws = []
    with torch.cuda.device(dev):
        _capi.call(fn, x.data_ptr(), out.data_ptr(), storage_code(x.dtype), storage_code(od), *dims,
                   *geo.pointers(), geo.g, *ws, _stream(dev))
    return out


def _run_cone(forward: bool, x: torch.Tensor, out_dims, geo: GeometryCone, hardware_interp: bool,
              out_dtype=None, workspace=None) -> torch.Tensor:
    batch = x.shape[0]
    dev = x.device
    od = _out_dtype(x, out_dtype)
    if forward:
        vol_z, vol_y, vol_x = x.shape[1:]
        n_proj, det_h, det_w = out_dims
        out = torch.empty((batch, n_proj, det_h, det_w), dtype=od, device=dev)
        fn = "pyronn_cone_projection3d"
        dims = [batch, vol_z, vol_y, vol_x, n_proj, det_h, det_w]
        ws_args = dims + [storage_code(x.dtype), int(bool(hardware_interp)), geo.g]
    else:
        n_proj, det_h, det_w = x.shape[1:]
        vol_z, vol_y, vol_x = out_dims
        out = torch.empty((batch, vol_z, vol_y, vol_x), dtype=od, device=dev)
        fn = "pyronn_cone_backprojection3d"
        dims = [batch, n_proj, det_h, det_w, vol_z, vol_y, vol_x]
        ws_args = dims + [storage_code(x.dtype), int(bool(hardware_interp)), geo.g]
    ws_bytes = _capi.workspace_size(fn, *ws_args)
    if workspace is None or workspace.numel() < ws_bytes:
        workspace = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        _capi.call(fn, x.data_ptr(), out.data_ptr(), storage_code(x.dtype), storage_code(od),
                   int(bool(hardware_interp)), *dims, *geo.pointers(), geo.g, workspace.data_ptr(),
                   workspace.numel(), _stream(dev))
        if not forward and not hardware_interp:
            note_workspace_error(workspace, dev)  # the TMA-staged path's bounded waits
    return out


def _run_matched(p: torch.Tensor, vol_dims, geo: GeometryCone) -> torch.Tensor:
    batch = p.shape[0]
    dev = p.device
    n_proj, det_h, det_w = p.shape[1:]
    vol_z, vol_y, vol_x = vol_dims
    out = torch.empty((batch, vol_z, vol_y, vol_x), dtype=torch.float32, device=dev)
    fn = "pyronn_cone_backprojection3d_matched"
    ws_bytes = _capi.workspace_size(fn, geo.g, n_proj)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        _capi.call(fn, p.data_ptr(), out.data_ptr(), storage_code(p.dtype), batch, n_proj, det_h, det_w, vol_z, vol_y,
                   vol_x, geo.volume_origin.data_ptr(), geo.volume_spacing.data_ptr(),
                   geo.projection_matrices.data_ptr(), geo.step_size.data_ptr(), geo.g, ws.data_ptr(), ws_bytes,
                   _stream(dev))
    return out


# ------------------------------------------------------------- autograd


class _Op2D(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, forward_op, out_dims, geo, out_dtype):
        ctx.forward_op = forward_op
        ctx.in_dims = tuple(x.shape[1:])
        ctx.in_dtype = x.dtype
        ctx.geo = geo
        return _run_2d(forward_op, x, out_dims, geo, out_dtype)

    @staticmethod
    def backward(ctx, grad):
        g = grad.contiguous()
        gx = _run_2d(not ctx.forward_op, g, ctx.in_dims, ctx.geo, ctx.in_dtype)
        return gx, None, None, None, None


class _OpCone(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, forward_op, out_dims, geo, hardware_interp, out_dtype, matched=False):
        ctx.forward_op = forward_op
        ctx.in_dims = tuple(x.shape[1:])
        ctx.in_dtype = x.dtype
        ctx.geo = geo
        ctx.hardware_interp = hardware_interp
        ctx.matched = matched
        if matched and not forward_op:
            return _run_matched(x, out_dims, geo).to(out_dtype or torch.float32)
        return _run_cone(forward_op, x, out_dims, geo, hardware_interp, out_dtype)

    @staticmethod
    def backward(ctx, grad):
        g = grad.contiguous()
        if ctx.matched and ctx.forward_op:
            gx = _run_matched(g, ctx.in_dims, ctx.geo).to(ctx.in_dtype)
        else:
            gx = _run_cone(not ctx.forward_op, g, ctx.in_dims, ctx.geo, ctx.hardware_interp, ctx.in_dtype)
        return gx, None, None, None, None, None, None


# ----------------------------------------------------------- public op surface


def parallel_projection2d(volume, projection_shape, volume_origin, detector_origin, volume_spacing,
                          detector_spacing, ray_vectors, name=None, out_dtype=None):
    """A x for 2D parallel beam: [B, Y, X] -> [B, n_proj, det_w].

    projection_shape = (n_proj, det_w) (cc/ops/par_projector_2D_OPKernel.cc:101-107)."""
    x = _check_data(volume, 3, "volume")
    n_proj, det_w = _shape(projection_shape, 2, "projection_shape")
    geo = Geometry2D(x.shape[0], x.device, volume_origin, detector_origin, volume_spacing, detector_spacing,
                     ray_vectors, n_proj)
    return _Op2D.apply(x, True, (n_proj, det_w), geo, out_dtype)


def parallel_backprojection2d(sinogram, volume_shape, volume_origin, detector_origin, volume_spacing,
                              detector_spacing, ray_vectors, name=None, out_dtype=None):
    """A^T p for 2D parallel beam: [B, n_proj, det_w] -> [B, Y, X].

    volume_shape = (Y, X) (cc/ops/par_backprojector_2D_OPKernel.cc:95-102)."""
    p = _check_data(sinogram, 3, "sinogram")
    vol_y, vol_x = _shape(volume_shape, 2, "volume_shape")
    geo = Geometry2D(p.shape[0], p.device, volume_origin, detector_origin, volume_spacing, detector_spacing,
                     ray_vectors, p.shape[1])
    return _Op2D.apply(p, False, (vol_y, vol_x), geo, out_dtype)


def fan_projection2d(volume, projection_shape, volume_origin, detector_origin, volume_spacing, detector_spacing,
                     source_2_isocenter_distance, source_2_detector_distance, central_ray_vectors, name=None,
                     out_dtype=None):
    """A x for 2D fan beam (flat detector): [B, Y, X] -> [B, n_proj, det_w]."""
    x = _check_data(volume, 3, "volume")
    n_proj, det_w = _shape(projection_shape, 2, "projection_shape")
    geo = Geometry2D(x.shape[0], x.device, volume_origin, detector_origin, volume_spacing, detector_spacing,
                     central_ray_vectors, n_proj, source_2_isocenter_distance, source_2_detector_distance)
    return _Op2D.apply(x, True, (n_proj, det_w), geo, out_dtype)


def fan_backprojection2d(sinogram, volume_shape, volume_origin, detector_origin, volume_spacing, detector_spacing,
                         source_2_isocenter_distance, source_2_detector_distance, central_ray_vectors, name=None,
                         out_dtype=None):
    """Distance-weighted fan-beam backprojection: [B, n_proj, det_w] -> [B, Y, X]."""
    p = _check_data(sinogram, 3, "sinogram")
    vol_y, vol_x = _shape(volume_shape, 2, "volume_shape")
    geo = Geometry2D(p.shape[0], p.device, volume_origin, detector_origin, volume_spacing, detector_spacing,
                     central_ray_vectors, p.shape[1], source_2_isocenter_distance, source_2_detector_distance)
    return _Op2D.apply(p, False, (vol_y, vol_x), geo, out_dtype)


def cone_projection3d(volume, projection_shape, volume_origin, volume_spacing, projection_matrices, step_size,
                      projection_multiplier, hardware_interp=False, name=None, out_dtype=None, matched_adjoint=False):
    """A x for 3D cone beam: [B, Z, Y, X] -> [B, n_proj, det_h, det_w].

    projection_shape = (n_proj, det_h, det_w) (cc/ops/cone_projector_3D_OPKernel.cc:219-226);
    step_size in voxels along the ray; projection_multiplier is unused by the
    forward op, as in the reference.  matched_adjoint=True makes the gradient
    the exact transpose (cone_backprojection3d_matched) instead of the paired
    voxel-driven backprojector (software interpolation only)."""
    x = _check_data(volume, 4, "volume")
    n_proj, det_h, det_w = _shape(projection_shape, 3, "projection_shape")
    if matched_adjoint and hardware_interp:
        raise ValueError("matched_adjoint is the transpose of the software-interpolation projector")
    geo = GeometryCone(x.shape[0], x.device, volume_origin, volume_spacing, projection_matrices, step_size,
                       projection_multiplier, n_proj)
    return _OpCone.apply(x, True, (n_proj, det_h, det_w), geo, bool(hardware_interp), out_dtype,
                         bool(matched_adjoint))


def cone_backprojection3d_matched(sinogram, volume_shape, volume_origin, volume_spacing, projection_matrices,
                                  step_size, projection_multiplier=None, name=None, out_dtype=None):
    """Exact transpose of the software-interpolation cone_projection3d:
    [B, n_proj, det_h, det_w] -> [B, Z, Y, X] (FP32 accumulation by atomics).

    No counterpart in the reference (its voxel-driven backprojector is not the
    transpose of its projector).  projection_multiplier is accepted for
    signature symmetry and not applied."""
    p = _check_data(sinogram, 4, "sinogram")
    vol_z, vol_y, vol_x = _shape(volume_shape, 3, "volume_shape")
    mult = 1.0 if projection_multiplier is None else projection_multiplier
    geo = GeometryCone(p.shape[0], p.device, volume_origin, volume_spacing, projection_matrices, step_size, mult,
                       p.shape[1])
    return _OpCone.apply(p, False, (vol_z, vol_y, vol_x), geo, False, out_dtype, True)


def cone_backprojection3d(sinogram, volume_shape, volume_origin, volume_spacing, projection_matrices, step_size,
                          projection_multiplier, hardware_interp=False, name=None, out_dtype=None):
    """Voxel-driven cone backprojection: [B, n_proj, det_h, det_w] -> [B, Z, Y, X].

    volume_shape = (Z, Y, X) (cc/ops/cone_backprojector_3D_OPKernel.cc:109-116);
    step_size is accepted and unused, as in the reference."""
    p = _check_data(sinogram, 4, "sinogram")
    vol_z, vol_y, vol_x = _shape(volume_shape, 3, "volume_shape")
    geo = GeometryCone(p.shape[0], p.device, volume_origin, volume_spacing, projection_matrices, step_size,
                       projection_multiplier, p.shape[1])
    return _OpCone.apply(p, False, (vol_z, vol_y, vol_x), geo, bool(hardware_interp), out_dtype)


def release_cached_arrays() -> None:
    """Frees the CUDA arrays the hardware_interp paths keep cached on the current device."""
    _capi.call("pyronn_release_cached_arrays")


def circular_projection_matrices(n_proj: int, sid: float, sdd: float, detector_shape, detector_spacing,
                                 angular_range: float = 2.0 * math.pi, start: float = 0.0, principal_point=None,
                                 device="cuda") -> torch.Tensor:
    """[n_proj, 3, 4] float32 projection matrices of a circular cone-beam scan,
    built on `device` in FP64 (pyronn_circular_projection_matrices); the same
    conventions and arguments as geometry.circular_projection_matrices, which
    builds them on the host."""
    H, W = int(detector_shape[0]), int(detector_shape[1])
    cv, cu = ((H - 1) / 2.0, (W - 1) / 2.0) if principal_point is None else principal_point
    dev = torch.device(device)
    out = torch.empty((int(n_proj), 3, 4), dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        _capi.call("pyronn_circular_projection_matrices", out.data_ptr(), int(n_proj), float(sid), float(sdd),
                   float(detector_spacing[0]), float(detector_spacing[1]), float(cv), float(cu),
                   float(angular_range), float(start), _stream(dev))
    return out


def circular_ray_vectors_2d(n_proj: int, angular_range: float = math.pi, start: float = 0.0,
                            device="cuda") -> torch.Tensor:
    """[n_proj, 2] float32 (cos, sin) ray vectors built on `device` in FP64
    (pyronn_circular_ray_vectors_2d); geometry.ray_vectors_2d on the host."""
    dev = torch.device(device)
    out = torch.empty((int(n_proj), 2), dtype=torch.float32, device=dev)
    with torch.cuda.device(dev):
        _capi.call("pyronn_circular_ray_vectors_2d", out.data_ptr(), int(n_proj), float(angular_range), float(start),
                   _stream(dev))
    return out
