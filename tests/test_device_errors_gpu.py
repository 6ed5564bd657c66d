"""Device-side failure reporting of the bounded waits, on the GPU, without a
fault: the testing hook pyronn_debug_starve_tma_wait makes the TMA-staged
cone backprojector's last pass wait for bytes that no copy delivers (no copy
is in flight), with a short spin limit.  The wait runs out; the kernel
records PYRONN_DEVICE_ERROR_WAIT_TIMEOUT, uses its barriers no more, waits
(bounded) for any copy still in flight and finishes (its voxels are invalid
and the flag says so), and the host reads the flag:
  * through the workspace (pyronn_workspace_error) on the C ABI;
  * through the ops' per-device error word (device_errors /
    check_device_errors) and the synchronous mode (set_sync_error_checks).
Afterwards the same call, unstarved, reports no error and matches the oracle:
the context stayed usable.  One CTA (a 32 x 8 x 16 voxel tile, four views:
one pass) keeps the launch small."""
import ctypes

import numpy as np
import pytest
import torch

import oracle
import pyronn_layers as pl
from pyronn_layers import _capi, geometry, ops
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def _one_tile_case(dev):
    geo = geometry.ConeBeam3D((16, 8, 32), (1.0, 1.0, 1.0), (64, 64), (1.0, 1.0), 4, 200.0, 300.0)
    rng = np.random.Generator(np.random.PCG64(41))
    sino = rng.uniform(0, 1, (1,) + geo.detector_shape).astype(np.float32)
    return geo, sino, torch.as_tensor(sino).to(dev)


def _starved(enable):
    _capi.call("pyronn_debug_starve_tma_wait", int(enable))


def test_starved_wait_is_reported_through_the_workspace(cuda):
    geo, sino_np, sino = _one_tile_case(cuda)
    gc = ops.GeometryCone(1, cuda, *geo.args(), geo.detector_shape[0])
    ws_bytes = _capi.workspace_size("pyronn_cone_backprojection3d", 1, *geo.detector_shape, *geo.volume_shape, 0, 0,
                                    1)
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=cuda)
    stream = torch.cuda.current_stream().cuda_stream
    flag = ctypes.c_int(-1)
    for starve, expected in ((True, _capi.DEVICE_ERROR_WAIT_TIMEOUT), (False, _capi.DEVICE_ERROR_NONE)):
        out = torch.full((1,) + geo.volume_shape, -7.0, device=cuda)
        _starved(starve)
        try:
            _capi.call("pyronn_cone_backprojection3d", sino.data_ptr(), out.data_ptr(), 0, 0, 0, 1,
                       *geo.detector_shape, *geo.volume_shape, *gc.pointers(), 1, ws.data_ptr(), ws_bytes, stream)
        finally:
            _starved(False)
        _capi.call("pyronn_workspace_error", ws.data_ptr(), stream, ctypes.byref(flag))
        assert flag.value == expected
        if not starve:
            ref = oracle.cone_backprojection3d(sino_np, geo.volume_shape, *geo.args())
            assert rel_l2(out.cpu().numpy(), ref) < 1e-5


def test_starved_wait_is_reported_by_the_ops(cuda):
    geo, sino_np, sino = _one_tile_case(cuda)
    pl.device_errors(cuda)  # clear
    _starved(True)
    try:
        pl.cone_backprojection3d(sino, geo.volume_shape, *geo.args())
    finally:
        _starved(False)
    assert pl.device_errors(cuda) == _capi.DEVICE_ERROR_WAIT_TIMEOUT
    assert pl.device_errors(cuda) == 0  # read and cleared
    out = pl.cone_backprojection3d(sino, geo.volume_shape, *geo.args())
    pl.check_device_errors(cuda)
    ref = oracle.cone_backprojection3d(sino_np, geo.volume_shape, *geo.args())
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5
    # synchronous mode raises at the call
    pl.set_sync_error_checks(True)
    _starved(True)
    try:
        with pytest.raises(pl.PyronnDeviceError):
            pl.cone_backprojection3d(sino, geo.volume_shape, *geo.args())
    finally:
        _starved(False)
        pl.set_sync_error_checks(False)
    pl.check_device_errors(cuda)


def test_fdk_filter_error_word_is_clear(cuda):
    from pyronn_layers import fbp
    rng = np.random.Generator(np.random.PCG64(42))
    p = torch.as_tensor(rng.uniform(0, 1, (1, 3, 40, 256)).astype(np.float32)).to(cuda)
    fbp.fdk_filter(p, 1000.0, (1.0, 1.0))
    flag = ctypes.c_int(-1)
    _capi.call("pyronn_fdk_error", torch.cuda.current_stream().cuda_stream, ctypes.byref(flag))
    assert flag.value == _capi.DEVICE_ERROR_NONE
