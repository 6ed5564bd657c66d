"""GPU parity of the six ops (all storage dtypes, both interpolation modes)
against the FP64 oracle and against the reference's own outputs (golden
fixtures).  Every call goes through the C ABI (libpyronn_b200.so).

Tolerances (relative L2):
  * FP32 arithmetic vs the FP64 oracle on the same (storage-rounded) input:
    2e-5 for ray marches (thousands of FP32 sums), 1e-5 for backprojections;
  * hardware_interp (texture unit, 8-bit interpolation weights) vs exact
    weights: forward 5e-4 (measured 3.6e-5 to 6.7e-5), backprojection of a
    noise sinogram 2e-3 (one texture-weighted fetch per update: the reference's
    own outputs are 3.5e-4 to 6.0e-4 from the exact weights); 5e-3 on the
    one-voxel and ragged shapes, where a handful of texels dominate;
  * 16-bit OUTPUT storage adds its rounding: 4e-3 (bf16), 6e-4 (fp16);
  * against the reference's outputs (golden fixtures): 1e-5 on the software
    cone paths (measured below 6e-7); hardware_interp cone 5e-5 (the same
    texture unit on both sides: measured 4.4e-6 to 1.9e-5); 2D forward 5e-5
    (the reference's texture weights averaged over its 0.2 mm steps: measured
    1.1e-5); 2D backprojection 5e-4 (one texture-weighted tap pair per view:
    measured 1.1e-4 to 1.2e-4).
"""
import ctypes
import math

import numpy as np
import pytest
import torch

import oracle
import pyronn_layers as pl
from pyronn_layers import _capi, geometry, phantoms
from conftest import load_golden, rel_l2

pytestmark = pytest.mark.gpu

DTYPES = [torch.float32, torch.bfloat16, torch.float16]
OUT_TOL = {torch.float32: 0.0, torch.bfloat16: 4e-3, torch.float16: 6e-4}
# the 3D forward's 16-bit cells interpolate in the storage type (z lerps of
# the z0 taps and the stored half-differences, y lerp of the pair, one
# rounding each; measured on these phantoms: FP16 1.4e-5, BF16 1.1e-4)
CONE_FWD_TOL = {torch.float32: 2e-5, torch.float16: 2e-5, torch.bfloat16: 2e-4}


def t(a, dev, dtype=torch.float32):
    return torch.as_tensor(np.asarray(a)).to(device=dev, dtype=dtype)


def rounded(x):
    return x.float().cpu().numpy()


# ------------------------------------------------------------------ 2D


def _par_setup(dev, dtype):
    geo = geometry.ParallelBeam2D((48, 56), (1.0, 0.8), 91, 0.9, 36)
    vol = np.stack([phantoms.ellipse_phantom_2d((48, 56), (1.0, 0.8), seed=s, n=5)[0] for s in (1, 2)])
    return geo, t(vol, dev, dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_parallel_projection_vs_oracle(cuda, dtype):
    geo, x = _par_setup(cuda, dtype)
    out = pl.parallel_projection2d(x, geo.detector_shape, *geo.args(), out_dtype=torch.float32)
    ref = oracle.parallel_projection2d(rounded(x), geo.detector_shape, *geo.args())
    assert rel_l2(out.cpu().numpy(), ref) < 2e-5
    out16 = pl.parallel_projection2d(x, geo.detector_shape, *geo.args())
    assert out16.dtype == dtype
    assert rel_l2(out16.float().cpu().numpy(), ref) < 2e-5 + OUT_TOL[dtype]


@pytest.mark.parametrize("dtype", DTYPES)
def test_parallel_backprojection_vs_oracle(cuda, dtype):
    geo, _ = _par_setup(cuda, dtype)
    rng = np.random.Generator(np.random.PCG64(3))
    p = t(rng.uniform(0, 1, (2,) + geo.detector_shape), cuda, dtype)
    out = pl.parallel_backprojection2d(p, geo.volume_shape, *geo.args(), out_dtype=torch.float32)
    ref = oracle.parallel_backprojection2d(rounded(p), geo.volume_shape, *geo.args())
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5


def _fan_setup(dev, dtype):
    geo = geometry.FanBeam2D((40, 52), (0.5, 0.5), 100, 0.5, 45, 70.0, 110.0)
    vol = np.stack([phantoms.ellipse_phantom_2d((40, 52), (0.5, 0.5), seed=s, n=5)[0] for s in (4, 5, 6)])
    return geo, t(vol, dev, dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_fan_projection_vs_oracle(cuda, dtype):
    geo, x = _fan_setup(cuda, dtype)
    out = pl.fan_projection2d(x, geo.detector_shape, *geo.args(), out_dtype=torch.float32)
    ref = oracle.fan_projection2d(rounded(x), geo.detector_shape, *geo.args())
    assert rel_l2(out.cpu().numpy(), ref) < 2e-5


@pytest.mark.parametrize("dtype", DTYPES)
def test_fan_backprojection_vs_oracle(cuda, dtype):
    geo, _ = _fan_setup(cuda, dtype)
    rng = np.random.Generator(np.random.PCG64(9))
    p = t(rng.uniform(0, 1, (3,) + geo.detector_shape), cuda, dtype)
    out = pl.fan_backprojection2d(p, geo.volume_shape, *geo.args(), out_dtype=torch.float32)
    ref = oracle.fan_backprojection2d(rounded(p), geo.volume_shape, *geo.args())
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5


def test_axis_aligned_rays(cuda):
    """Rays with an exactly zero component skip that slab test
    (par_projector_2D_CudaKernel.cu.cc:36,48)."""
    vol, _ = phantoms.ellipse_phantom_2d((32, 32), (1.0, 1.0), seed=11, n=4)
    rays = np.array([[1, 0], [0, 1], [-1, 0], [0, -1], [0.6, 0.8]], np.float32)
    args = (geometry.centered_origin((32, 32), (1, 1)), geometry.detector_origin_1d(47, 1.0),
            np.array([1, 1], np.float32), np.array([1.0], np.float32), rays)
    out = pl.parallel_projection2d(t(vol[None], cuda), (5, 47), *args)
    ref = oracle.parallel_projection2d(vol[None], (5, 47), *args)
    assert rel_l2(out.cpu().numpy(), ref) < 2e-5


@pytest.mark.parametrize("fan", [False, True])
@pytest.mark.parametrize("dtype", DTYPES)
def test_2d_forward_layout_choice_is_bit_exact(cuda, fan, dtype):
    """Given a workspace, the forward reads bilinear cell copies (y-fastest
    for views whose rays run along x); without one, the caller's slice with a
    bounds test per tap.  The taps are combined in the same order, so a result
    is the same bits either way, for every view direction."""
    if fan:
        geo, x = _fan_setup(cuda, dtype)
        fn = "pyronn_fan_projection2d"
    else:
        geo, x = _par_setup(cuda, dtype)
        fn = "pyronn_parallel_projection2d"
    gp = pl.ops.Geometry2D(x.shape[0], cuda, *geo.args()[:4], geo.args()[-1], geo.detector_shape[0],
                           *(geo.args()[4:6] if fan else ()))
    n_proj, det_w = geo.detector_shape
    code = pl.ops.storage_code(dtype)
    outs = []
    for with_ws in (False, True):
        out = torch.full((x.shape[0], n_proj, det_w), float("nan"), device=cuda)
        ws_bytes = _capi.workspace_size("pyronn_projection2d", x.shape[0], *x.shape[1:], code)
        ws = torch.full((ws_bytes,), 255, dtype=torch.uint8, device=cuda)
        _capi.call(fn, x.data_ptr(), out.data_ptr(), code, 0, x.shape[0], *x.shape[1:], n_proj, det_w,
                   *gp.pointers(), gp.g, ws.data_ptr() if with_ws else None, ws_bytes if with_ws else 0,
                   torch.cuda.current_stream().cuda_stream)
        outs.append(out.cpu())
    assert torch.isfinite(outs[0]).all()
    assert torch.equal(outs[0], outs[1])


# ------------------------------------------------------------------ cone


def _cone_geo(vol_shape=(20, 24, 28), det=(30, 36), n_proj=16, step=0.5):
    return geometry.ConeBeam3D(vol_shape, (1.0, 0.9, 1.1), det, (1.2, 1.3), n_proj, 160.0, 260.0,
                               step_size=step, projection_multiplier=0.8)


@pytest.mark.parametrize("hw", [False, True])
@pytest.mark.parametrize("dtype", DTYPES)
def test_cone_projection_vs_oracle(cuda, dtype, hw):
    geo = _cone_geo()
    vol = np.stack([phantoms.ellipsoid_phantom_3d(geo.volume_shape, geo.volume_spacing, seed=s, n=6)[0]
                    for s in (1, 2)])
    x = t(vol, cuda, dtype)
    out = pl.cone_projection3d(x, geo.detector_shape, *geo.args(), hardware_interp=hw, out_dtype=torch.float32)
    ref = oracle.cone_projection3d(rounded(x), geo.detector_shape, *geo.args(), hardware_interp=hw)
    tol = 5e-4 if hw else CONE_FWD_TOL[dtype]
    assert rel_l2(out.cpu().numpy(), ref) < tol


@pytest.mark.parametrize("sid,step", [(160.0, 0.5), (160.0, 0.37), (128.0, 0.5)])
def test_cone_projection_alpha_sequences(cuda, sid, step):
    """The forward counts a ray's samples when its float alpha sequence is
    exact (step a multiple of ulp(alpha), alphas inside one binade: SID 160
    with step 0.5) and compares alpha against the exit otherwise (step 0.37;
    SID 128, where the march crosses alpha = 128): both match the oracle's
    float alpha march."""
    geo = geometry.ConeBeam3D((20, 24, 28), (1.0, 0.9, 1.1), (30, 36), (1.2, 1.3), 16, sid, sid + 100.0,
                              step_size=step)
    vol = phantoms.ellipsoid_phantom_3d(geo.volume_shape, geo.volume_spacing, seed=3, n=6)[0][None]
    out = pl.cone_projection3d(t(vol, cuda), geo.detector_shape, *geo.args())
    ref = oracle.cone_projection3d(vol, geo.detector_shape, *geo.args())
    assert rel_l2(out.cpu().numpy(), ref) < 2e-5


@pytest.mark.parametrize("hw", [False, True])
@pytest.mark.parametrize("dtype", DTYPES)
def test_cone_backprojection_vs_oracle(cuda, dtype, hw):
    geo = _cone_geo()
    rng = np.random.Generator(np.random.PCG64(5))
    p = t(rng.uniform(0, 1, (2,) + geo.detector_shape), cuda, dtype)
    out = pl.cone_backprojection3d(p, geo.volume_shape, *geo.args(), hardware_interp=hw, out_dtype=torch.float32)
    ref = oracle.cone_backprojection3d(rounded(p), geo.volume_shape, *geo.args(), hardware_interp=hw)
    tol = 2e-3 if hw else 1e-5  # one texture-weighted fetch per update on a noise sinogram
    assert rel_l2(out.cpu().numpy(), ref) < tol
    out16 = pl.cone_backprojection3d(p, geo.volume_shape, *geo.args(), hardware_interp=hw)
    assert rel_l2(out16.float().cpu().numpy(), ref) < tol + OUT_TOL[dtype]


def test_cone_backprojection_edge_taps(cuda):
    """Detector smaller than the shadow: the software path reads the x == W /
    y == H taps from the next row / next view (the reference's `>` bounds) and
    zero past the end of the buffer."""
    geo = geometry.ConeBeam3D((16, 20, 20), (1.0, 1.0, 1.0), (10, 12), (1.5, 1.5), 7, 150.0, 260.0)
    rng = np.random.Generator(np.random.PCG64(6))
    p = rng.uniform(0.5, 1, (1,) + geo.detector_shape).astype(np.float32)
    out = pl.cone_backprojection3d(t(p, cuda), geo.volume_shape, *geo.args())
    ref = oracle.cone_backprojection3d(p, geo.volume_shape, *geo.args())
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5
    clean = oracle.cone_backprojection3d(p, geo.volume_shape, *geo.args(), hardware_interp=True)
    assert rel_l2(ref, clean) > 1e-3  # the quirk taps really are exercised


BP_PATH_GEOMETRIES = {
    # shadow inside the detector, tiles fit the staging box: TMA-staged tiles
    "staged": dict(vol=(24, 32, 32), det=(40, 64), px=1.2, sid=400.0, sdd=600.0),
    # magnification ~3: tile footprints overflow the box, per-view global path
    "magnified": dict(vol=(24, 40, 44), det=(30, 40), px=1.0, sid=90.0, sdd=200.0),
    # 37-pixel rows are not 16-byte aligned: the direct-gather kernel
    "unaligned": dict(vol=(24, 32, 32), det=(40, 37), px=1.2, sid=400.0, sdd=600.0),
}


@pytest.mark.parametrize("case", sorted(BP_PATH_GEOMETRIES))
@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_cone_backprojection_kernel_paths(cuda, dtype, case):
    c = BP_PATH_GEOMETRIES[case]
    geo = geometry.ConeBeam3D(c["vol"], (1.0, 1.0, 1.0), c["det"], (c["px"], c["px"]), 12, c["sid"], c["sdd"])
    rng = np.random.Generator(np.random.PCG64(12))
    p = t(rng.uniform(0, 1, (2,) + geo.detector_shape), cuda, dtype)
    out = pl.cone_backprojection3d(p, geo.volume_shape, *geo.args(), out_dtype=torch.float32)
    ref = oracle.cone_backprojection3d(rounded(p), geo.volume_shape, *geo.args())
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5


@pytest.mark.parametrize("dtype", [torch.float16, torch.bfloat16])
@pytest.mark.parametrize("tilted", [False, True])
def test_cone_backprojection_paired_copy_is_bit_exact(cuda, dtype, tilted):
    """Given the queried workspace, a 16-bit backprojection stages a paired
    copy of the sinogram (tap u and u + 1 in one 32-bit element); given only
    the views' part, it stages the sinogram itself.  The lerps are the same
    operations on the same taps: the same bits, for the column loop of
    circular views and the general loop of tilted ones.  (The copy is made
    where a detector pixel serves at least 100 voxel updates per view.)"""
    geo = geometry.ConeBeam3D((64, 64, 64), (1.0, 1.0, 1.0), (40, 48), (2.4, 2.4), 12, 160.0, 260.0,
                              projection_multiplier=0.8)
    P = np.asarray(geo.projection_matrices).copy()
    if tilted:
        P[::2] = P[::2][:, :, [0, 2, 1, 3]]  # every other view rotates about y
    args = (geo.volume_origin, geo.volume_spacing, P, geo.step_size, geo.projection_multiplier)
    rng = np.random.Generator(np.random.PCG64(21))
    sino = t(rng.uniform(0, 1, (2,) + geo.detector_shape), cuda, dtype)
    gc = pl.ops.GeometryCone(2, cuda, *args, geo.detector_shape[0])
    code = pl.ops.storage_code(dtype)
    full = _capi.workspace_size("pyronn_cone_backprojection3d", 2, *geo.detector_shape, *geo.volume_shape, code, 0,
                                gc.g)
    views_only = 256 + (gc.g * geo.detector_shape[0] * 48 + 255) // 256 * 256
    assert full > views_only
    outs = []
    for ws_bytes in (full, views_only):
        ws = torch.empty(ws_bytes, dtype=torch.uint8, device=cuda)
        out = torch.empty((2,) + geo.volume_shape, device=cuda)
        _capi.call("pyronn_cone_backprojection3d", sino.data_ptr(), out.data_ptr(), code, 0, 0, 2,
                   *geo.detector_shape, *geo.volume_shape, *gc.pointers(), gc.g, ws.data_ptr(), ws_bytes,
                   torch.cuda.current_stream().cuda_stream)
        outs.append(out.cpu())
    assert torch.equal(outs[0], outs[1])
    ref = oracle.cone_backprojection3d(rounded(sino), geo.volume_shape, *args)
    assert rel_l2(outs[0].numpy(), ref) < 1e-5


def test_workspace_error_flag_clear(cuda):
    geo = _cone_geo()
    p = torch.rand((1,) + geo.detector_shape, device=cuda)
    gc = pl.ops.GeometryCone(1, cuda, *geo.args(), geo.detector_shape[0])
    ws_bytes = _capi.workspace_size("pyronn_cone_backprojection3d", 1, *geo.detector_shape, *geo.volume_shape, 0, 0, 1)
    ws = torch.full((ws_bytes,), 7, dtype=torch.uint8, device=cuda)
    out = torch.empty((1,) + geo.volume_shape, device=cuda)
    _capi.call("pyronn_cone_backprojection3d", p.data_ptr(), out.data_ptr(), 0, 0, 0, 1, *geo.detector_shape,
               *geo.volume_shape, *gc.pointers(), 1, ws.data_ptr(), ws_bytes, torch.cuda.current_stream().cuda_stream)
    flag = ctypes.c_int(-1)
    _capi.call("pyronn_workspace_error", ws.data_ptr(), torch.cuda.current_stream().cuda_stream,
               ctypes.byref(flag))
    assert flag.value == 0


def test_cone_batch_geometry_rows(cuda):
    """Per-batch-element geometry rows vs one shared row."""
    g1 = _cone_geo()
    g2 = geometry.ConeBeam3D(g1.volume_shape, (1.0, 1.0, 1.0), (30, 36), (1.2, 1.3), 16, 170.0, 250.0,
                             step_size=0.6)
    vol = np.stack([phantoms.ellipsoid_phantom_3d(g1.volume_shape, (1, 1, 1), seed=s, n=5)[0] for s in (7, 8)])
    stacked = [np.stack([a, b]) for a, b in zip(g1.args(), g2.args())]
    out = pl.cone_projection3d(t(vol, cuda), g1.detector_shape, *stacked).cpu().numpy()
    for b, g in enumerate((g1, g2)):
        single = pl.cone_projection3d(t(vol[b:b + 1], cuda), g.detector_shape, *g.args()).cpu().numpy()
        np.testing.assert_array_equal(out[b], single[0])


# ------------------------------------------------------------ golden (reference outputs)


def test_golden_parallel(cuda):
    g = load_golden("parallel2d")
    args = (g["volume_origin"], g["detector_origin"], g["volume_spacing"], g["detector_spacing"], g["ray_vectors"])
    out = pl.parallel_projection2d(t(g["volume"], cuda), g["projection_shape"], *args)
    assert rel_l2(out.cpu().numpy(), g["sinogram_ref"]) < 5e-5
    out = pl.parallel_backprojection2d(t(g["sinogram_in"], cuda), g["volume"].shape[1:], *args)
    assert rel_l2(out.cpu().numpy(), g["volume_ref"]) < 5e-4


def test_golden_fan(cuda):
    g = load_golden("fan2d")
    args = (g["volume_origin"], g["detector_origin"], g["volume_spacing"], g["detector_spacing"], g["sid"], g["sdd"],
            g["ray_vectors"])
    out = pl.fan_projection2d(t(g["volume"], cuda), g["projection_shape"], *args)
    assert rel_l2(out.cpu().numpy(), g["sinogram_ref"]) < 5e-5
    out = pl.fan_backprojection2d(t(g["sinogram_in"], cuda), g["volume"].shape[1:], *args)
    assert rel_l2(out.cpu().numpy(), g["volume_ref"]) < 5e-4


def test_golden_fan_degenerate_line(cuda):
    """Pixels on and near intersectLines2D's degenerate line (the source
    inside the field; cc/helper_headers/helper_geometry_gpu.h:30-36): the
    reference's NaN intersection reaches its texture as a NaN coordinate,
    which samples as coordinate 0 -- half of the view's first texel -- and
    just off the line its FP32 intersection lands far from the exact one; the
    kernel takes the reference's FP32 steps within 1e-2 mm of the source's
    depth.  Matched against the reference's own outputs (golden fixture) and
    the oracle, which follows the same rule."""
    g = load_golden("fan2d_degenerate")
    args = (g["volume_origin"], g["detector_origin"], g["volume_spacing"], g["detector_spacing"], g["sid"], g["sdd"],
            g["ray_vectors"])
    out = pl.fan_backprojection2d(t(g["sinogram_in"], cuda), tuple(g["volume_shape"]), *args).cpu().numpy()
    ref = g["volume_ref"]
    assert np.isfinite(out).all()
    assert rel_l2(out, ref) < 5e-4
    # the column of pixels at x = -SID for the view along +x (batch 0: SID 5.5,
    # column 10; batch 1: SID 15.5, column 0) carries the degenerate taps
    for b, col in ((0, 10), (1, 0)):
        np.testing.assert_allclose(out[b, :, col], ref[b, :, col], rtol=1e-3, atol=1e-3 * np.abs(ref[b, :, col]).max())
    # and the FP64 oracle follows the same rule
    orc = oracle.fan_backprojection2d(g["sinogram_in"], tuple(g["volume_shape"]), *args)
    assert rel_l2(out, orc) < 1e-5


@pytest.mark.parametrize("name", ["cone3d", "cone3d_edges"])
@pytest.mark.parametrize("hw", [0, 1])
def test_golden_cone(cuda, name, hw):
    g = load_golden(name)
    args = (g["volume_origin"], g["volume_spacing"], g["projection_matrices"], g["step_size"],
            g["projection_multiplier"])
    tol = 5e-5 if hw else 1e-5
    out = pl.cone_projection3d(t(g["volume"], cuda), g["projection_shape"], *args, hardware_interp=bool(hw))
    assert rel_l2(out.cpu().numpy(), g["sinogram_ref_hw%d" % hw]) < tol
    out = pl.cone_backprojection3d(t(g["sinogram_in"], cuda), g["volume"].shape[1:], *args,
                                   hardware_interp=bool(hw))
    assert rel_l2(out.cpu().numpy(), g["volume_ref_hw%d" % hw]) < tol


# ------------------------------------------------------------ gradients and errors


def test_gradients_are_paired_ops(cuda):
    geo = _cone_geo()
    x = torch.rand((1,) + geo.volume_shape, device=cuda, requires_grad=True)
    y = pl.cone_projection3d(x, geo.detector_shape, *geo.args())
    gy = torch.rand_like(y)
    (gx,) = torch.autograd.grad(y, x, gy)
    bp = pl.cone_backprojection3d(gy, geo.volume_shape, *geo.args())
    torch.testing.assert_close(gx, bp, rtol=0, atol=0)

    g2 = geometry.FanBeam2D((30, 30), (1, 1), 50, 1.0, 20, 80.0, 120.0)
    p = torch.rand((2,) + g2.detector_shape, device=cuda, requires_grad=True)
    v = pl.fan_backprojection2d(p, g2.volume_shape, *g2.args())
    gv = torch.rand_like(v)
    (gp,) = torch.autograd.grad(v, p, gv)
    torch.testing.assert_close(gp, pl.fan_projection2d(gv, g2.detector_shape, *g2.args()), rtol=0, atol=0)


def test_invalid_arguments_raise(cuda):
    geo = _cone_geo()
    x = torch.rand((1,) + geo.volume_shape, device=cuda)
    with pytest.raises(ValueError):
        pl.cone_projection3d(x, (16, 30), *geo.args())
    with pytest.raises(ValueError):
        pl.cone_projection3d(x[0], geo.detector_shape, *geo.args())
    with pytest.raises(TypeError):
        pl.cone_projection3d(x.double(), geo.detector_shape, *geo.args())
    # geom_batch that is neither 1 nor batch, straight through the C ABI
    lib = _capi.load()
    st = lib.pyronn_parallel_projection2d(x.data_ptr(), x.data_ptr(), 0, 0, 2, 4, 4, 3, 5, 1, 1, 1, 1, 1, 3, None, 0,
                                          None)
    assert st == _capi.ERROR_INVALID_ARGUMENT
    assert b"geom_batch" in lib.pyronn_last_error()
    st = lib.pyronn_cone_projection3d(x.data_ptr(), x.data_ptr(), 0, 0, 0, 1, 4, 4, 4, 3, 5, 5, 1, 1, 1, 1, 1, 1,
                                      None, 0, None)
    assert st == _capi.ERROR_WORKSPACE_TOO_SMALL


# ------------------------------------------------------------ matched adjoint


def _adjoint_geo():
    return geometry.ConeBeam3D((20, 24, 28), (1.0, 0.9, 1.1), (30, 36), (1.2, 1.3), 16, 160.0, 260.0,
                               step_size=0.6)


def test_matched_backprojection_vs_oracle(cuda):
    geo = _adjoint_geo()
    rng = np.random.Generator(np.random.PCG64(21))
    y = rng.uniform(-1, 1, (2,) + geo.detector_shape).astype(np.float32)
    out = pl.cone_backprojection3d_matched(t(y, cuda), geo.volume_shape, *geo.args())
    ref = oracle.cone_backprojection3d_matched(y, geo.volume_shape, *geo.args())
    assert out.dtype == torch.float32
    assert rel_l2(out.cpu().numpy(), ref) < 2e-5


def test_dot_product_adjoint(cuda):
    """<A x, y> = <x, A^T y> to 1e-6 (FP32 operators, FP64 dot products)."""
    geo = _adjoint_geo()
    rng = np.random.Generator(np.random.PCG64(22))
    x = t(rng.uniform(0.1, 1, (2,) + geo.volume_shape), cuda)
    y = t(rng.uniform(-1, 1, (2,) + geo.detector_shape), cuda)
    ax = pl.cone_projection3d(x, geo.detector_shape, *geo.args())
    aty = pl.cone_backprojection3d_matched(y, geo.volume_shape, *geo.args())
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-6
    # the unmatched (reference) pair, reported by the mismatch it has
    bp = pl.cone_backprojection3d(y, geo.volume_shape, *geo.args())
    assert abs(float((x.double() * bp.double()).sum()) - lhs) / abs(lhs) > 1e-3


def test_central_differences_of_the_loss(cuda):
    """d/dx 1/2 ||A x - y||^2 through autograd (matched adjoint) against FP64
    central differences, h = 1e-3, on 64 random voxels."""
    geo = _adjoint_geo()
    rng = np.random.Generator(np.random.PCG64(23))
    x0 = rng.uniform(0.2, 1, (1,) + geo.volume_shape)
    y = t(rng.uniform(0, 5, (1,) + geo.detector_shape), cuda)

    def loss(xv):
        r = pl.cone_projection3d(xv, geo.detector_shape, *geo.args(), matched_adjoint=True) - y
        return 0.5 * (r.double() ** 2).sum()

    x = t(x0, cuda).requires_grad_(True)
    (g,) = torch.autograd.grad(loss(x), x)
    idx = rng.choice(x0.size, 64, replace=False)
    h = 1e-3
    fd = []
    for i in idx:
        xp = x0.copy().reshape(-1)
        xm = x0.copy().reshape(-1)
        xp[i] += h
        xm[i] -= h
        lp = float(loss(t(xp.reshape(x0.shape), cuda)))
        lm = float(loss(t(xm.reshape(x0.shape), cuda)))
        fd.append((lp - lm) / (2 * h))
    ga = g.reshape(-1)[torch.as_tensor(idx, device=cuda)].double().cpu().numpy()
    assert rel_l2(ga, np.array(fd)) < 2e-3


def test_unrolled_reconstruction_with_checkpointing(cuda):
    """Config-4 pattern at small size: y = -log(Poisson(I0 exp(-A x)) / I0),
    K unrolled gradient steps through the ops; checkpointed and plain
    unrolling give the same loss gradient, and the loss decreases."""
    from pyronn_layers import recon
    geo = geometry.ConeBeam3D((16, 16, 16), (1.0, 1.0, 1.0), (24, 24), (1.5, 1.5), 18, 100.0, 170.0)
    x_true = t(phantoms.ellipsoid_phantom_3d(geo.volume_shape, (1, 1, 1), seed=3, n=4)[0][None] * 0.02, cuda)
    y = recon.poisson_sinogram(pl.cone_projection3d(x_true, geo.detector_shape, *geo.args()), 1e5, seed=1)
    grads = []
    for ckpt in (True, False):
        net = recon.UnrolledGradientDescent(geo, n_steps=4, init_lr=2e-3, checkpoint=ckpt).to(cuda)
        x0 = torch.zeros_like(x_true)
        xk = net(x0, y)
        loss = 0.5 * ((pl.cone_projection3d(xk, geo.detector_shape, *geo.args()) - y) ** 2).sum()
        loss.backward()
        grads.append(net.log_lr.grad.clone())
        loss0 = 0.5 * ((pl.cone_projection3d(x0, geo.detector_shape, *geo.args()) - y) ** 2).sum()
        assert float(loss) < float(loss0)
    torch.testing.assert_close(grads[0], grads[1], rtol=1e-5, atol=0)


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_cone_projection_non_circular_views(cuda, dtype):
    """Views whose detector v axis is not along z (a trajectory about the y
    axis: P's y and z columns swapped) take the forward projector's xy mode;
    mixing them with circular views exercises both modes in one launch."""
    geo = _cone_geo(n_proj=12)
    P = np.asarray(geo.projection_matrices).copy()
    P[::2] = P[::2][:, :, [0, 2, 1, 3]]  # every other view rotates about y
    args = (geo.volume_origin, geo.volume_spacing, P, geo.step_size, geo.projection_multiplier)
    vol = phantoms.ellipsoid_phantom_3d(geo.volume_shape, geo.volume_spacing, seed=9, n=6)[0][None]
    x = t(vol, cuda, dtype)
    out = pl.cone_projection3d(x, geo.detector_shape, *args, out_dtype=torch.float32)
    ref = oracle.cone_projection3d(rounded(x), geo.detector_shape, *args)
    assert rel_l2(out.cpu().numpy(), ref) < CONE_FWD_TOL[dtype]


@pytest.mark.parametrize("hw", [False, True])
def test_cone_projection_volume_partly_off_detector(cuda, hw):
    """Rays outside a view's detector footprint of the volume box skip their
    set-up; with the volume shifted so that it projects partly off the
    detector (and wholly off it in some views), the result still matches the
    oracle, zeros included."""
    geo = _cone_geo(n_proj=16)
    origin = np.asarray(geo.volume_origin, np.float32) + np.array([6.0, 14.0, -11.0], np.float32)
    args = (origin, geo.volume_spacing, geo.projection_matrices, geo.step_size, geo.projection_multiplier)
    vol = phantoms.ellipsoid_phantom_3d(geo.volume_shape, geo.volume_spacing, seed=8, n=6)[0][None]
    out = pl.cone_projection3d(t(vol, cuda), geo.detector_shape, *args, hardware_interp=hw)
    ref = oracle.cone_projection3d(vol, geo.detector_shape, *args, hardware_interp=hw)
    assert (ref == 0).any() and (ref != 0).any()
    assert rel_l2(out.cpu().numpy(), ref) < (5e-4 if hw else 2e-5)


def test_cone_projection_wide_fp16_range(cuda):
    """FP16 inputs whose magnitudes could overflow FP16 in the packed lerps'
    differences (above 32704) take FP32 y and x lerps: a scan of the input
    before the cell copy flags them, and the result matches the oracle as closely as a normal-range
    input's.  (The BF16 bound, 8.5e37, lies beyond what FP32 sums of a ray can
    hold anyway.)"""
    geo = _cone_geo()
    vol = phantoms.ellipsoid_phantom_3d(geo.volume_shape, geo.volume_spacing, seed=5, n=6)[0][None]
    x = t(vol / vol.max() * 40000.0, cuda, torch.float16)
    x[0, 3, 4, 5] = -40000.0  # a negative extreme beside positive ones
    out = pl.cone_projection3d(x, geo.detector_shape, *geo.args(), out_dtype=torch.float32)
    ref = oracle.cone_projection3d(rounded(x), geo.detector_shape, *geo.args())
    assert torch.isfinite(out).all()
    assert rel_l2(out.cpu().numpy(), ref) < 2e-5


@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
def test_cone_projection_padded_cell_pitch(cuda, dtype):
    """A volume (91 x 8 x 196, z y x) whose cell copy needs one cell of x
    pitch padding for the sampler's biased index not to wrap: the forward
    over that layout matches the oracle."""
    geo = geometry.ConeBeam3D((91, 8, 196), (1.0, 1.0, 1.0), (40, 60), (3.0, 3.0), 8, 300.0, 500.0,
                              step_size=0.5, projection_multiplier=0.8)
    vol = phantoms.ellipsoid_phantom_3d(geo.volume_shape, geo.volume_spacing, seed=9, n=6)[0][None]
    x = t(vol, cuda, dtype)
    out = pl.cone_projection3d(x, geo.detector_shape, *geo.args(), out_dtype=torch.float32)
    ref = oracle.cone_projection3d(rounded(x), geo.detector_shape, *geo.args())
    assert (ref != 0).any()
    assert rel_l2(out.cpu().numpy(), ref) < CONE_FWD_TOL[dtype]


# ------------------------------------------------------------ device geometry


@pytest.mark.parametrize("start,rng_", [(0.0, 2 * math.pi), (0.3, math.pi + 0.4)])
def test_device_geometry_matches_host_builder(cuda, start, rng_):
    """The FP64 device builders give the host builder's matrices and ray
    vectors (to FP32 rounding: CUDA's and the host's FP64 sin/cos may differ
    in the last bit)."""
    n, det, sp = 97, (40, 56), (1.3, 0.7)
    host = geometry.circular_projection_matrices(n, 640.0, 1100.0, det, sp, rng_, start)
    dev = pl.circular_projection_matrices(n, 640.0, 1100.0, det, sp, rng_, start, device=cuda)
    np.testing.assert_allclose(dev.cpu().numpy(), host, rtol=2e-7, atol=2e-7 * np.abs(host).max())
    rh = geometry.ray_vectors_2d(n, rng_, start)
    rd = pl.circular_ray_vectors_2d(n, rng_, start, device=cuda)
    np.testing.assert_allclose(rd.cpu().numpy(), rh, rtol=0, atol=1.2e-7)
    # the device matrices drive the projector like the host ones
    geo = geometry.ConeBeam3D((16, 20, 24), (1.0, 1.0, 1.0), det, sp, n, 640.0, 1100.0, rng_)
    vol = phantoms.ellipsoid_phantom_3d(geo.volume_shape, geo.volume_spacing, seed=2, n=4)[0][None]
    args = list(geo.args())
    args[2] = host
    a = pl.cone_projection3d(t(vol, cuda), geo.detector_shape, *args)
    args[2] = dev
    b = pl.cone_projection3d(t(vol, cuda), geo.detector_shape, *args)
    assert rel_l2(b.cpu().numpy(), a.cpu().numpy()) < 1e-6


# ------------------------------------------------------------ degenerate sizes


@pytest.mark.parametrize("vol_shape,det,n_proj,batch", [
    ((1, 1, 1), (1, 1), 1, 1),      # one voxel, one pixel, one view
    ((3, 5, 7), (2, 3), 3, 3),      # ragged odd sizes, batch of 3
    ((9, 1, 4), (5, 1), 2, 2),      # flat volume, one-column detector
])
@pytest.mark.parametrize("hw", [False, True])
def test_cone_tiny_and_ragged_shapes(cuda, vol_shape, det, n_proj, batch, hw):
    """Every cone path on sizes far below one tile or one TMA box, against the
    oracle: partial blocks, single views and one-pixel detectors."""
    geo = geometry.ConeBeam3D(vol_shape, (1.0, 0.9, 1.1), det, (1.2, 1.3), n_proj, 60.0, 100.0, step_size=0.5)
    rng = np.random.Generator(np.random.PCG64(31))
    vol = rng.uniform(0.2, 1.0, (batch,) + vol_shape).astype(np.float32)
    out = pl.cone_projection3d(t(vol, cuda), geo.detector_shape, *geo.args(), hardware_interp=hw)
    ref = oracle.cone_projection3d(vol, geo.detector_shape, *geo.args(), hardware_interp=hw)
    tol = 5e-3 if hw else 2e-5
    assert out.shape == (batch,) + geo.detector_shape
    assert rel_l2(out.cpu().numpy(), ref) < tol or np.abs(ref).max() == 0
    sino = rng.uniform(0.2, 1.0, (batch,) + geo.detector_shape).astype(np.float32)
    back = pl.cone_backprojection3d(t(sino, cuda), geo.volume_shape, *geo.args(), hardware_interp=hw)
    refb = oracle.cone_backprojection3d(sino, geo.volume_shape, *geo.args(), hardware_interp=hw)
    assert back.shape == (batch,) + vol_shape
    assert rel_l2(back.cpu().numpy(), refb) < (5e-3 if hw else 1e-5) or np.abs(refb).max() == 0


@pytest.mark.parametrize("n_proj", [256, 300, 513])
@pytest.mark.parametrize("fan", [False, True])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float16])
def test_2d_backprojection_view_chunks(cuda, n_proj, fan, dtype):
    """The 2D backprojector stages the views' constants in shared memory 256 at
    a time: one full chunk, a full chunk and a ragged one, and three chunks
    whose last holds one view, against the oracle."""
    if fan:
        geo = geometry.FanBeam2D((24, 20), (1.0, 0.8), 40, 1.1, n_proj, 40.0, 70.0)
        bwd, obwd = pl.fan_backprojection2d, oracle.fan_backprojection2d
    else:
        geo = geometry.ParallelBeam2D((24, 20), (1.0, 0.8), 40, 1.1, n_proj)
        bwd, obwd = pl.parallel_backprojection2d, oracle.parallel_backprojection2d
    rng = np.random.Generator(np.random.PCG64(n_proj))
    sino = t(rng.uniform(0.2, 1.0, (2,) + geo.detector_shape).astype(np.float32), cuda, dtype)
    back = bwd(sino, geo.volume_shape, *geo.args(), out_dtype=torch.float32)
    refb = obwd(rounded(sino), geo.volume_shape, *geo.args())
    assert rel_l2(back.cpu().numpy(), refb) < 1e-5


@pytest.mark.parametrize("vol_shape,det_w,n_proj,batch", [((1, 1), 1, 1, 1), ((5, 3), 7, 2, 3), ((2, 33), 4, 5, 1)])
@pytest.mark.parametrize("fan", [False, True])
def test_2d_tiny_and_ragged_shapes(cuda, vol_shape, det_w, n_proj, batch, fan):
    if fan:
        geo = geometry.FanBeam2D(vol_shape, (1.0, 0.8), det_w, 1.1, n_proj, 40.0, 70.0)
        fwd, bwd, ofwd, obwd = (pl.fan_projection2d, pl.fan_backprojection2d, oracle.fan_projection2d,
                                oracle.fan_backprojection2d)
    else:
        geo = geometry.ParallelBeam2D(vol_shape, (1.0, 0.8), det_w, 1.1, n_proj)
        fwd, bwd, ofwd, obwd = (pl.parallel_projection2d, pl.parallel_backprojection2d, oracle.parallel_projection2d,
                                oracle.parallel_backprojection2d)
    rng = np.random.Generator(np.random.PCG64(32))
    img = rng.uniform(0.2, 1.0, (batch,) + vol_shape).astype(np.float32)
    out = fwd(t(img, cuda), geo.detector_shape, *geo.args())
    ref = ofwd(img, geo.detector_shape, *geo.args())
    assert out.shape == (batch,) + geo.detector_shape
    assert rel_l2(out.cpu().numpy(), ref) < 2e-5 or np.abs(ref).max() == 0
    sino = rng.uniform(0.2, 1.0, (batch,) + geo.detector_shape).astype(np.float32)
    back = bwd(t(sino, cuda), geo.volume_shape, *geo.args())
    refb = obwd(sino, geo.volume_shape, *geo.args())
    assert rel_l2(back.cpu().numpy(), refb) < 1e-5 or np.abs(refb).max() == 0
