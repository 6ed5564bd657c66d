"""pyronn_cone_backprojection3d_noalloc: the cone backprojection for callers
that cannot allocate device memory or lend a workspace (e.g. a framework whose
allocator owns the GPU, or a loop that must not call cudaMalloc).  Its scratch
is a fixed array inside the library, so these tests check, through the C ABI,
that it gives the workspace entry point's result on two calls in a row (the
second with another geometry and size, so leftovers of the first would show),
and that requests beyond the fixed size are refused.

Kept in the last-collected file so a failure here cannot stop the rest of a
-x run; it also passes on its own in a fresh process."""
import numpy as np
import pytest
import torch

from pyronn_layers import _capi, geometry, ops
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _case(dev, seed, vol_shape, det, n_proj, batch, dtype):
    geo = geometry.ConeBeam3D(vol_shape, (1.0, 0.9, 1.1), det, (1.2, 1.3), n_proj, 160.0, 260.0,
                              projection_multiplier=0.7)
    rng = np.random.Generator(np.random.PCG64(seed))
    sino = torch.as_tensor(rng.uniform(0, 1, (batch, n_proj) + tuple(det)).astype(np.float32)).to(dev, dtype)
    gc = ops.GeometryCone(batch, dev, *geo.args(), n_proj)
    return geo, sino, gc


def _with_workspace(geo, sino, gc):
    batch, n_proj, det_h, det_w = sino.shape
    out = torch.empty((batch,) + geo.volume_shape, device=sino.device)
    code = ops.storage_code(sino.dtype)
    ws_bytes = _capi.workspace_size("pyronn_cone_backprojection3d", batch, n_proj, det_h, det_w, *geo.volume_shape,
                                    code, 0, gc.g)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=sino.device)
    _capi.call("pyronn_cone_backprojection3d", sino.data_ptr(), out.data_ptr(), code, 0, 0, batch, n_proj, det_h,
               det_w, *geo.volume_shape, *gc.pointers(), gc.g, ws.data_ptr(), ws_bytes,
               torch.cuda.current_stream().cuda_stream)
    return out


def _no_alloc(geo, sino, gc):
    batch, n_proj, det_h, det_w = sino.shape
    out = torch.empty((batch,) + geo.volume_shape, device=sino.device)
    _capi.call("pyronn_cone_backprojection3d_noalloc", sino.data_ptr(), out.data_ptr(),
               ops.storage_code(sino.dtype), 0, batch, n_proj, det_h, det_w, *geo.volume_shape, *gc.pointers(),
               gc.g, torch.cuda.current_stream().cuda_stream)
    return out


def test_no_alloc_matches_workspace_entry_point_twice(cuda):
    cases = [
        (_case(cuda, 1, (20, 24, 28), (30, 36), 16, 2, torch.float32)),
        (_case(cuda, 2, (16, 20, 24), (24, 40), 11, 1, torch.bfloat16)),
    ]
    for geo, sino, gc in cases:  # two calls in a row, different sizes
        ref = _with_workspace(geo, sino, gc)
        got = _no_alloc(geo, sino, gc)
        torch.cuda.synchronize()
        assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < 1e-5


def test_no_alloc_refuses_more_views_than_its_scratch(cuda):
    lib = _capi.load()
    n_proj = _capi.NOALLOC_MAX_VIEWS + 1
    x = torch.empty(16, device=cuda)
    status = lib.pyronn_cone_backprojection3d_noalloc(x.data_ptr(), x.data_ptr(), 0, 0, 1, n_proj, 4, 4, 4, 4, 4,
                                                      x.data_ptr(), x.data_ptr(), x.data_ptr(), x.data_ptr(),
                                                      x.data_ptr(), 1, None)
    assert status == _capi.ERROR_UNSUPPORTED
    assert b"exceeds the fixed scratch" in lib.pyronn_last_error()


def test_no_alloc_reports_a_timed_out_wait(cuda):
    """The entry point's device error flag sits in its fixed scratch, which
    callers cannot address: pyronn_noalloc_error reads it.  The testing hook
    pyronn_debug_starve_tma_wait makes the backprojector's bounded wait run
    out (no copy in flight); the flag reports it, and the next call, unstarved,
    clears it and gives the workspace entry point's result."""
    import ctypes
    geo, sino, gc = _case(cuda, 3, (16, 8, 32), (64, 64), 4, 1, torch.float32)
    stream = torch.cuda.current_stream().cuda_stream
    flag = ctypes.c_int(-1)
    _capi.call("pyronn_debug_starve_tma_wait", 1)
    try:
        _no_alloc(geo, sino, gc)
    finally:
        _capi.call("pyronn_debug_starve_tma_wait", 0)
    _capi.call("pyronn_noalloc_error", stream, ctypes.byref(flag))
    assert flag.value == _capi.DEVICE_ERROR_WAIT_TIMEOUT
    got = _no_alloc(geo, sino, gc)
    _capi.call("pyronn_noalloc_error", stream, ctypes.byref(flag))
    assert flag.value == _capi.DEVICE_ERROR_NONE
    ref = _with_workspace(geo, sino, gc)
    torch.cuda.synchronize()
    assert rel_l2(got.cpu().numpy(), ref.cpu().numpy()) < 1e-5
