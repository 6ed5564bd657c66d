"""GPU tests of the FDK / FBP pre-processing (pyronn_fdk_filter) and of the
reconstructions built on it, against the FP64 restatement in
oracle/filters.py.

Tolerances (relative L2): FP32 filtering vs FP64, 1e-5 (rows of up to ~100
terms with cancellation); 16-bit output storage adds its rounding (6e-4
fp16); reconstructions against the oracle's FDK, 1e-4 (filter + backprojection
in FP32)."""
import math

import numpy as np
import pytest
import torch

import oracle
import pyronn_layers as pl
from pyronn_layers import _capi, fbp, geometry, phantoms
from conftest import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("filt", ["ram-lak", "shepp-logan"])
@pytest.mark.parametrize("shape,sdd,pp", [
    ((2, 5, 7, 64), 900.0, None),          # cone rows, centred principal point
    ((1, 3, 4, 77), 450.0, (1.3, 40.2)),   # width not a multiple of 16, offset principal point
    ((2, 6, 1, 200), 0.0, None),           # parallel-beam rows: no weighting
    ((1, 2, 3, 1030), 1200.0, None),       # wide rows: several warps per row
    ((1, 3, 130, 1024), 1200.0, None),     # tensor cores: 8 output tiles, 4 accumulators, a partial row block
    ((1, 1, 5, 2048), 1000.0, (2.0, 1000.5)),  # tensor cores at their widest rows (64 chunks per accumulator set)
    ((1, 1, 2, 2052), 1000.0, None),       # just past the tensor-core width: CUDA cores
])
def test_fdk_filter_vs_oracle(cuda, filt, shape, sdd, pp):
    rng = np.random.Generator(np.random.PCG64(21))
    p = rng.uniform(0, 2, shape).astype(np.float32)
    sp = (1.1, 0.7)
    x = torch.as_tensor(p, device=cuda)
    out = fbp.fdk_filter(x, sdd, sp, pp, filt)
    h, w = shape[2], shape[3]
    cv, cu = ((h - 1) / 2, (w - 1) / 2) if pp is None else pp
    kind = oracle.filters.RAM_LAK if filt == "ram-lak" else oracle.filters.SHEPP_LOGAN
    ref = oracle.fdk_filter(p, sdd, sp[0], sp[1], cv, cu, kind)
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
def test_fdk_filter_storage_types(cuda, dtype):
    rng = np.random.Generator(np.random.PCG64(22))
    x = torch.as_tensor(rng.uniform(0, 2, (1, 4, 6, 96)), dtype=dtype, device=cuda)
    ref = oracle.fdk_filter(x.float().cpu().numpy(), 800.0, 1.0, 1.0, 2.5, 47.5)
    out = fbp.fdk_filter(x, 800.0, (1.0, 1.0))
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5
    out16 = fbp.fdk_filter(x, 800.0, (1.0, 1.0), out_dtype=torch.float16)
    assert rel_l2(out16.float().cpu().numpy(), ref) < 1e-5 + 6e-4


def test_fdk_filter_in_place_and_adjoint(cuda):
    """In-place filtering (the CUDA-core kernel, which holds whole rows in
    shared memory) agrees with out-of-place filtering (the tensor-core kernel)
    to FP32 rounding; the weight_output form is the adjoint (dot-product
    test), which is also the autograd backward."""
    rng = np.random.Generator(np.random.PCG64(23))
    x = torch.as_tensor(rng.uniform(-1, 1, (2, 3, 5, 48)), dtype=torch.float32, device=cuda)
    y = torch.as_tensor(rng.uniform(-1, 1, (2, 3, 5, 48)), dtype=torch.float32, device=cuda)
    fx = fbp.fdk_filter(x, 700.0, (0.9, 1.2))
    xi = x.clone()
    _capi.call("pyronn_fdk_filter", xi.data_ptr(), xi.data_ptr(), 0, 0, 2, 3, 5, 48, 700.0, 0.9, 1.2, 2.0, 23.5,
               0, 0, torch.cuda.current_stream().cuda_stream)
    assert rel_l2(xi.cpu().numpy(), fx.cpu().numpy()) < 3e-6
    xg = x.clone().requires_grad_(True)
    (fbp.fdk_filter(xg, 700.0, (0.9, 1.2)) * y).sum().backward()
    lhs = float((fx.double() * y.double()).sum())
    rhs = float((x.double() * xg.grad.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-6


def test_fdk_reconstruction(cuda):
    """FDK through the library (filter + cone backprojection op) equals the
    oracle's FDK and gives back the phantom's densities."""
    vs, sp = (48, 48, 48), (1.0, 1.0, 1.0)
    geo = geometry.ConeBeam3D(vs, sp, (80, 96), (1.6, 1.6), 180, 600.0, 1000.0)
    vol, _ = phantoms.ellipsoid_phantom_3d(vs, sp, seed=5, n=4)
    x = torch.as_tensor(vol[None], dtype=torch.float32, device=cuda)
    sino = pl.cone_projection3d(x, geo.detector_shape, *geo.args())
    rec = fbp.fdk_reconstruct(sino, geo)[0].cpu().numpy()
    H, W = geo.detector_shape[1:]
    q = oracle.fdk_filter(sino.cpu().numpy(), geo.sdd, 1.6, 1.6, (H - 1) / 2, (W - 1) / 2).astype(np.float32)
    args = list(geo.args())
    args[4] = np.array([geo.sid * geo.sdd * math.pi / 180], np.float32)
    ref = oracle.cone_backprojection3d(q, vs, *args)[0]
    assert rel_l2(rec, ref) < 1e-4
    c = slice(12, 36)
    assert abs(rec[c, c, c].mean() / vol[c, c, c].mean() - 1) < 0.01


def test_parallel_fbp_reconstruction(cuda):
    geo = geometry.ParallelBeam2D((128, 128), (1.0, 1.0), 183, 1.0, 360)
    img, _ = phantoms.ellipse_phantom_2d((128, 128), (1.0, 1.0), seed=8, n=6)
    x = torch.as_tensor(img[None], dtype=torch.float32, device=cuda)
    sino = pl.parallel_projection2d(x, geo.detector_shape, *geo.args())
    rec = fbp.fbp_reconstruct_2d(sino, geo)[0].cpu().numpy()
    c = slice(32, 96)
    assert abs(rec[c, c].mean() / img[c, c].mean() - 1) < 0.01
    assert np.linalg.norm(rec[c, c] - img[c, c]) / np.linalg.norm(img[c, c]) < 0.06


def test_fdk_filter_rejects_bad_arguments(cuda):
    lib = _capi.load()
    x = torch.zeros(64, device=cuda)
    s = torch.cuda.current_stream().cuda_stream
    st = lib.pyronn_fdk_filter(x.data_ptr(), x.data_ptr(), 0, 0, 1, 1, 1, _capi.FDK_MAX_WIDTH + 1, 1.0, 1.0, 1.0,
                               0.0, 0.0, 0, 0, s)
    assert st == _capi.ERROR_UNSUPPORTED
    st = lib.pyronn_fdk_filter(x.data_ptr(), x.data_ptr(), 0, 0, 1, 1, 1, 8, 1.0, 1.0, -1.0, 0.0, 0.0, 0, 0, s)
    assert st == _capi.ERROR_INVALID_ARGUMENT
    st = lib.pyronn_fdk_filter(x.data_ptr(), x.data_ptr(), 0, 0, 1, 1, 1, 8, 1.0, 1.0, 1.0, 0.0, 0.0, 5, 0, s)
    assert st == _capi.ERROR_INVALID_ARGUMENT
    with pytest.raises(ValueError):
        fbp.fdk_filter(x.view(1, 1, 1, 64), 1.0, (1.0, 1.0), filter="hann")
