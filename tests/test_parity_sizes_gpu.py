"""Parity at the sizes the workloads are quoted on, against the FP64 oracle
(the CPU restatement of the reference kernels) on the same seeded inputs.

* config 1 -- 2D parallel beam, 256 x 256 at 1.0 mm, 180 views on [0, pi),
  367-pixel detector at 1.0 mm, the 10-ellipse phantom: forward and
  backprojection, FP32;
* config 2 -- one full slice of the fan-beam batch: 512 x 512 at 0.5 mm, 360
  views on [0, 2 pi), SID 750 / SDD 1200, 1024 pixels at 0.5 mm: FP32 and
  BF16 storage;
* config 4 -- the differentiable cone geometry: 128^3 at 1.0 mm, 180 views,
  256 x 256 at 1.5 mm, SID 600 / SDD 1000: forward, backprojection, the
  matched pair's dot-product test on the batch of 4 volumes, and the
  gradient of 1/2 |A x - y|^2 against FP64 central differences (h = 1e-3)
  on 64 random voxels;
* config 3 -- the 512^3 headline geometry (360 views, 1024 x 768 at 1 mm, SID
  750 / SDD 1200, step 0.5 voxel) with FP16 storage: two full views of the
  forward projection and four z-slices of the backprojection (the oracle's
  bounded samples of the full launch).

Tolerances (relative L2) are those of the small-size tests: 2e-5 for ray
marches and 1e-5 for backprojections in FP32 arithmetic on the same
(storage-rounded) input; storage rounding against the FP32 input is reported
separately with its own bound.
"""
import math

import numpy as np
import pytest
import torch

import oracle
import pyronn_layers as pl
from pyronn_layers import geometry, phantoms
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def t(a, dev, dtype=torch.float32):
    return torch.as_tensor(np.asarray(a, dtype=np.float32)).to(device=dev, dtype=dtype)


# ------------------------------------------------------------------ config 1


def test_config1_parallel_full_size(cuda):
    geo = geometry.ParallelBeam2D((256, 256), (1.0, 1.0), 367, 1.0, 180)
    vol, _ = phantoms.ellipse_phantom_2d((256, 256), (1.0, 1.0), seed=2024)
    x = t(vol[None], cuda)
    sino = pl.parallel_projection2d(x, geo.detector_shape, *geo.args())
    ref = oracle.parallel_projection2d(vol[None], geo.detector_shape, *geo.args())
    assert rel_l2(sino.cpu().numpy(), ref) < 2e-5
    p = sino.cpu().numpy()
    back = pl.parallel_backprojection2d(sino, geo.volume_shape, *geo.args())
    refb = oracle.parallel_backprojection2d(p, geo.volume_shape, *geo.args())
    assert rel_l2(back.cpu().numpy(), refb) < 1e-5


# ------------------------------------------------------------------ config 2


@pytest.mark.parametrize("dtype", [torch.float32, torch.bfloat16])
def test_config2_fan_slice_full_size(cuda, dtype):
    geo = geometry.FanBeam2D((512, 512), (0.5, 0.5), 1024, 0.5, 360, 750.0, 1200.0)
    vol, _ = phantoms.ellipse_phantom_2d((512, 512), (0.5, 0.5), seed=100)
    x = t(vol[None], cuda, dtype)
    xr = x.float().cpu().numpy()
    sino = pl.fan_projection2d(x, geo.detector_shape, *geo.args(), out_dtype=torch.float32)
    ref = oracle.fan_projection2d(xr, geo.detector_shape, *geo.args())
    assert rel_l2(sino.cpu().numpy(), ref) < 2e-5
    if dtype != torch.float32:
        # BF16 storage of the phantom against the FP32 phantom: its rounding only
        ref32 = oracle.fan_projection2d(vol[None], geo.detector_shape, *geo.args())
        assert rel_l2(sino.cpu().numpy(), ref32) < 4e-3
    p = sino.to(dtype)
    back = pl.fan_backprojection2d(p, geo.volume_shape, *geo.args(), out_dtype=torch.float32)
    refb = oracle.fan_backprojection2d(p.float().cpu().numpy(), geo.volume_shape, *geo.args())
    assert rel_l2(back.cpu().numpy(), refb) < 1e-5


# ------------------------------------------------------------------ config 4


def _config4_geo():
    return geometry.ConeBeam3D((128, 128, 128), (1.0, 1.0, 1.0), (256, 256), (1.5, 1.5), 180, 600.0, 1000.0)


def _config4_volumes(geo, batch):
    vols = [phantoms.ellipsoid_phantom_3d(geo.volume_shape, geo.volume_spacing, seed=400 + b)[0] for b in range(batch)]
    return np.stack(vols) * np.float32(0.02)  # attenuation per mm


def test_config4_cone_full_size(cuda):
    geo = _config4_geo()
    vol = _config4_volumes(geo, 1)
    sino = pl.cone_projection3d(t(vol, cuda), geo.detector_shape, *geo.args())
    ref = oracle.cone_projection3d(vol, geo.detector_shape, *geo.args())
    assert rel_l2(sino.cpu().numpy(), ref) < 2e-5
    back = pl.cone_backprojection3d(sino, geo.volume_shape, *geo.args())
    refb = oracle.cone_backprojection3d(sino.cpu().numpy(), geo.volume_shape, *geo.args())
    assert rel_l2(back.cpu().numpy(), refb) < 1e-5


def test_config4_dot_product_of_the_matched_pair(cuda):
    """<A x, y> = <x, A^T y> to 1e-6 (FP32 operators, FP64 sums) on the batch
    of four 128^3 volumes; the reference's unmatched pair is reported by its
    mismatch."""
    geo = _config4_geo()
    x = t(_config4_volumes(geo, 4), cuda)
    rng = np.random.Generator(np.random.PCG64(44))
    y = t(rng.uniform(0.0, 1.0, (4,) + geo.detector_shape), cuda)
    ax = pl.cone_projection3d(x, geo.detector_shape, *geo.args())
    aty = pl.cone_backprojection3d_matched(y, geo.volume_shape, *geo.args())
    lhs = float((ax.double() * y.double()).sum())
    rhs = float((x.double() * aty.double()).sum())
    assert abs(lhs - rhs) / abs(lhs) < 1e-6
    bp = pl.cone_backprojection3d(y, geo.volume_shape, *geo.args())
    assert abs(float((x.double() * bp.double()).sum()) - lhs) / abs(lhs) > 1e-3


def test_config4_gradient_against_central_differences(cuda):
    """d/dx 1/2 |A x - y|^2 through autograd (matched adjoint) against FP64
    central differences, h = 1e-3, on 64 random voxels of the batch of four
    128^3 volumes; y = -log(Poisson(1e5 exp(-A x_true)) / 1e5)."""
    from pyronn_layers import recon
    geo = _config4_geo()
    x_true = t(_config4_volumes(geo, 4), cuda)
    y = recon.poisson_sinogram(pl.cone_projection3d(x_true, geo.detector_shape, *geo.args()), 1e5, seed=4)
    x0 = (x_true * 0.5).contiguous()

    def loss(xv):
        r = pl.cone_projection3d(xv, geo.detector_shape, *geo.args(), matched_adjoint=True) - y
        return 0.5 * (r.double() ** 2).sum()

    x = x0.clone().requires_grad_(True)
    (g,) = torch.autograd.grad(loss(x), x)
    rng = np.random.Generator(np.random.PCG64(45))
    # voxels inside the field (rays through them exist in every view)
    idx = rng.choice(x0.numel(), 4096, replace=False)
    zyx = np.stack(np.unravel_index(idx, x0.shape), 1)
    centre = np.array([64, 64, 64])
    inside = np.linalg.norm(zyx[:, 1:] - centre, axis=1) < 50
    idx = idx[inside][:64]
    h = 1e-3
    flat = x0.reshape(-1)
    fd = []
    with torch.no_grad():
        for i in idx:
            xp = flat.clone()
            xp[i] += h
            xm = flat.clone()
            xm[i] -= h
            fd.append((float(loss(xp.reshape(x0.shape))) - float(loss(xm.reshape(x0.shape)))) / (2 * h))
    ga = g.reshape(-1)[torch.as_tensor(idx, device=cuda)].double().cpu().numpy()
    assert rel_l2(ga, np.array(fd)) < 2e-3


# ------------------------------------------------------------------ config 3 (512^3)


def test_config3_cone512_headline_samples(cuda):
    """The headline geometry at full size with FP16 storage (FP32 sums):
    views 0 and 97 of the forward projection and z-slices 254..257 of the
    backprojection against the oracle on the same FP16-rounded inputs."""
    geo = geometry.ConeBeam3D((512, 512, 512), (0.5, 0.5, 0.5), (768, 1024), (1.0, 1.0), 360, 750.0, 1200.0,
                              step_size=0.5)
    ell = phantoms.random_ellipsoids(2024, [256.0, 256.0, 256.0], n=32)
    vol = phantoms.rasterise_ellipsoids_torch(ell, geo.volume_shape, geo.volume_spacing, geo.volume_origin, cuda)
    x = vol[None].to(torch.float16).contiguous()
    del vol
    sino = pl.cone_projection3d(x, geo.detector_shape, *geo.args(), out_dtype=torch.float32)
    xr = x.float().cpu().numpy()
    for view in (0, 97):
        ref, _ = oracle.cone_projection3d_views(xr, geo.detector_shape, view, view + 1, geo.volume_origin,
                                                geo.volume_spacing, geo.projection_matrices, geo.step_size)
        assert rel_l2(sino[0, view].cpu().numpy(), ref[view]) < 2e-5, view
    p16 = sino.to(torch.float16)
    del sino
    back = pl.cone_backprojection3d(p16, geo.volume_shape, *geo.args(), out_dtype=torch.float32)
    z0, z1 = 254, 258
    refb = oracle.cone_backprojection3d_slab(p16.float().cpu().numpy(), geo.volume_shape, z0, z1, geo.volume_origin,
                                             geo.volume_spacing, geo.projection_matrices, geo.projection_multiplier)
    assert rel_l2(back[0, z0:z1].cpu().numpy(), refb[z0:z1]) < 1e-5
