"""Pins of the CPU oracle (no GPU): closed-form line integrals of analytic
phantoms, the projection-matrix decomposition, linearity, and -- once
generated -- the golden fixtures holding the reference's own outputs."""
import math

import numpy as np
import pytest

import oracle
from pyronn_layers import geometry, phantoms
from conftest import load_golden, rel_l2


def test_parallel_projection_matches_exact_line_integrals():
    # at 1 mm spacing the reference's mm box offset and spacing scale are exact
    shape, n_proj, W = (96, 96), 24, 135
    ell = phantoms.random_ellipses(1, (96.0, 96.0), n=6, axes_mm=(6.0, 20.0), inner=0.5)
    vol = phantoms.rasterise_ellipses(ell, shape, (1.0, 1.0), geometry.centered_origin(shape, (1.0, 1.0)))
    geo = geometry.ParallelBeam2D(shape, (1.0, 1.0), W, 1.0, n_proj)
    sino = oracle.parallel_projection2d(vol[None], geo.detector_shape, *geo.args())[0]
    exact = np.zeros_like(sino)
    for p, (c, s) in enumerate(geo.ray_vectors.astype(np.float64)):
        for u in range(W):
            uu = u * 1.0 + float(geo.detector_origin[0])
            exact[p, u] = phantoms.ellipse_line_integral(ell, (-s * uu, c * uu), (c, s))
    assert rel_l2(sino, exact) < 0.03


def test_cone_projection_matches_exact_line_integrals():
    vol_shape, spacing = (48, 48, 48), (1.0, 1.0, 1.0)
    geo = geometry.ConeBeam3D(vol_shape, spacing, (40, 48), (1.6, 1.6), 6, 200.0, 320.0, step_size=0.25)
    ell = phantoms.random_ellipsoids(2, (48.0, 48.0, 48.0), n=5, axes_mm=(4.0, 12.0), inner=0.5)
    vol = phantoms.rasterise_ellipsoids(ell, vol_shape, spacing, geometry.centered_origin(vol_shape, spacing))
    sino = oracle.cone_projection3d(vol[None], geo.detector_shape, *geo.args())[0]
    inv, src = oracle.cone_decompose(geo.projection_matrices, geo.volume_spacing, geo.volume_origin)
    origin_xyz = geo.volume_origin[::-1].astype(np.float64)
    exact = np.zeros_like(sino)
    for p in range(6):
        s_mm = src[p] * 1.0 + origin_xyz
        for v in range(0, 40):
            for u in range(0, 48):
                d = inv[p] @ np.array([u, v, 1.0])
                d /= np.linalg.norm(d)
                exact[p, v, u] = phantoms.ellipsoid_line_integral(ell, s_mm, d)
    # partial-volume error of 4-12 mm ellipsoids on a 1 mm grid; a wrong
    # geometry gives O(1) errors
    assert rel_l2(sino, exact) < 0.05


def test_decomposition_recovers_source_and_rays():
    geo = geometry.ConeBeam3D((10, 12, 14), (0.5, 0.7, 0.9), (20, 30), (1.0, 1.1), 8, 300.0, 500.0)
    inv, src = oracle.cone_decompose(geo.projection_matrices, geo.volume_spacing, geo.volume_origin)
    s_zyx = np.asarray(geo.volume_spacing, np.float64)
    o_zyx = np.asarray(geo.volume_origin, np.float64)
    for p, th in enumerate(geometry.view_angles(8)):
        src_mm = np.array([-300 * math.cos(th), -300 * math.sin(th), 0.0])
        expect = (src_mm - o_zyx[::-1]) / s_zyx[::-1]
        np.testing.assert_allclose(src[p], expect, rtol=0, atol=2e-3)
        # the ray through the principal point is the principal direction
        d = inv[p] @ np.array([(30 - 1) / 2.0, (20 - 1) / 2.0, 1.0]) * s_zyx[::-1]
        d /= np.linalg.norm(d)
        np.testing.assert_allclose(d, [math.cos(th), math.sin(th), 0.0], atol=1e-6)


def test_backprojection_is_linear():
    geo = geometry.ConeBeam3D((8, 10, 12), (1, 1, 1), (12, 14), (1.5, 1.5), 5, 120.0, 200.0)
    rng = np.random.Generator(np.random.PCG64(0))
    p = rng.uniform(0, 1, (1,) + geo.detector_shape).astype(np.float32)
    q = rng.uniform(0, 1, (1,) + geo.detector_shape).astype(np.float32)
    a = oracle.cone_backprojection3d(p, geo.volume_shape, *geo.args())
    b = oracle.cone_backprojection3d(q, geo.volume_shape, *geo.args())
    c = oracle.cone_backprojection3d(p + 2 * q, geo.volume_shape, *geo.args())
    np.testing.assert_allclose(c, a + 2 * b, rtol=1e-6, atol=1e-9)


def test_projection_sample_counts():
    geo = geometry.ConeBeam3D((16, 16, 16), (1, 1, 1), (8, 8), (2.0, 2.0), 3, 100.0, 150.0, step_size=0.5)
    vol = np.ones((1, 16, 16, 16), np.float32)
    sino, cnt = oracle.cone_projection3d(vol, geo.detector_shape, *geo.args(), counts=True)
    # every ray through the centre crosses ~16 voxels: ~32 samples at step 0.5
    assert cnt.shape == (3,) and np.all(cnt > 8 * 8 * 20)
    assert np.all(sino >= 0)


def test_fan_backprojection_closed_form_matches_intersection():
    # the oracle keeps the reference's intersectLines2D; the weight and the
    # detector coordinate must match the closed form used on the GPU
    geo = geometry.FanBeam2D((16, 16), (1, 1), 40, 1.0, 12, 60.0, 100.0)
    rng = np.random.Generator(np.random.PCG64(1))
    p = rng.uniform(0, 1, (1,) + geo.detector_shape).astype(np.float32)
    out = oracle.fan_backprojection2d(p, geo.volume_shape, *geo.args())
    assert np.isfinite(out).all() and out.max() > 0


# ------------------------------------------------------ golden fixtures


def test_oracle_matches_reference_parallel():
    g = load_golden("parallel2d")
    args = (g["volume_origin"], g["detector_origin"], g["volume_spacing"], g["detector_spacing"], g["ray_vectors"])
    # the reference samples with 8-bit texture weights: measured 1.1e-5 (its
    # forward averages them over 0.2 mm steps) and 1.2e-4 (one tap pair per view)
    sino = oracle.parallel_projection2d(g["volume"], g["projection_shape"], *args)
    assert rel_l2(sino, g["sinogram_ref"]) < 5e-5
    vol = oracle.parallel_backprojection2d(g["sinogram_in"], g["volume"].shape[1:], *args)
    assert rel_l2(vol, g["volume_ref"]) < 5e-4


def test_oracle_matches_reference_fan():
    g = load_golden("fan2d")
    args = (g["volume_origin"], g["detector_origin"], g["volume_spacing"], g["detector_spacing"], g["sid"], g["sdd"],
            g["ray_vectors"])
    sino = oracle.fan_projection2d(g["volume"], g["projection_shape"], *args)
    assert rel_l2(sino, g["sinogram_ref"]) < 5e-5  # measured 1.1e-5
    vol = oracle.fan_backprojection2d(g["sinogram_in"], g["volume"].shape[1:], *args)
    assert rel_l2(vol, g["volume_ref"]) < 5e-4  # measured 1.1e-4


@pytest.mark.parametrize("name", ["cone3d", "cone3d_edges"])
@pytest.mark.parametrize("hw", [0, 1])
def test_oracle_matches_reference_cone(name, hw):
    g = load_golden(name)
    args = (g["volume_origin"], g["volume_spacing"], g["projection_matrices"], g["step_size"],
            g["projection_multiplier"])
    # hardware_interp: exact weights here, 8-bit texture weights in the
    # reference: measured 5.1e-5 / 5.3e-5 (forward), 3.5e-4 / 6.0e-4 (back)
    sino = oracle.cone_projection3d(g["volume"], g["projection_shape"], *args, hardware_interp=hw)
    assert rel_l2(sino, g["sinogram_ref_hw%d" % hw]) < (2e-4 if hw else 1e-5)
    vol = oracle.cone_backprojection3d(g["sinogram_in"], g["volume"].shape[1:], *args, hardware_interp=hw)
    assert rel_l2(vol, g["volume_ref_hw%d" % hw]) < (2e-3 if hw else 1e-5)


def test_matched_backprojection_is_the_transpose():
    """<A x, y> = <x, A^T y> for the forward projector and the matched
    backprojector (positive x: the reference's end correction always runs)."""
    geo = geometry.ConeBeam3D((10, 12, 14), (1.0, 0.9, 1.1), (16, 18), (1.3, 1.3), 6, 120.0, 200.0, step_size=0.7)
    rng = np.random.Generator(np.random.PCG64(4))
    x = rng.uniform(0.1, 1, (1,) + geo.volume_shape).astype(np.float32)
    y = rng.uniform(-1, 1, (1,) + geo.detector_shape).astype(np.float32)
    ax = oracle.cone_projection3d(x, geo.detector_shape, *geo.args())
    aty = oracle.cone_backprojection3d_matched(y, geo.volume_shape, *geo.args())
    lhs, rhs = float((ax * y).sum()), float((x.astype(np.float64) * aty).sum())
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # the reference's voxel-driven backprojector is not the transpose
    bp = oracle.cone_backprojection3d(y, geo.volume_shape, *geo.args())
    assert abs(float((x.astype(np.float64) * bp).sum()) - lhs) > 1e-3 * abs(lhs)


# ------------------------------------------------------------ FDK / FBP filter


def test_ramp_kernels():
    """Kak & Slaney's spatial ramp kernels: Ram-Lak is zero at even offsets,
    both are symmetric, and their DC gain tau * sum h tends to 0 (the ramp
    vanishes at zero frequency; the truncated tail is O(1 / (W tau)))."""
    from oracle import filters
    for kind in (filters.RAM_LAK, filters.SHEPP_LOGAN):
        h = filters.ramp_kernel(513, 0.8, kind)
        np.testing.assert_allclose(h, h[::-1], rtol=0, atol=0)
        assert abs(h.sum()) < 2.0 / (np.pi ** 2 * 512 * 0.8)
    h = filters.ramp_kernel(9, 0.5, filters.RAM_LAK)
    assert h[8] == pytest.approx(1.0 / (4 * 0.5)) and h[10] == 0.0
    assert h[9] == pytest.approx(-1.0 / (np.pi ** 2 * 0.5))


def test_oracle_fdk_reconstructs_ellipsoids():
    """Pins the filter's scale by reconstruction: FDK (cosine weights, Ram-Lak,
    backprojection with multiplier SID * SDD * pi / N) of the oracle's own
    projections of an ellipsoid phantom gives back its densities."""
    from oracle import filters
    vs, sp = (48, 48, 48), (1.0, 1.0, 1.0)
    geo = geometry.ConeBeam3D(vs, sp, (80, 96), (1.6, 1.6), 180, 600.0, 1000.0)
    vol, _ = phantoms.ellipsoid_phantom_3d(vs, sp, seed=5, n=4)
    sino = oracle.cone_projection3d(vol[None].astype(np.float32), geo.detector_shape, *geo.args())
    H, W = geo.detector_shape[1:]
    q = filters.fdk_filter(sino, geo.sdd, 1.6, 1.6, (H - 1) / 2, (W - 1) / 2).astype(np.float32)
    args = list(geo.args())
    args[4] = np.array([geo.sid * geo.sdd * np.pi / 180], np.float32)
    rec = oracle.cone_backprojection3d(q, vs, *args)[0]
    c = slice(12, 36)
    assert abs(rec[c, c, c].mean() / vol[c, c, c].mean() - 1) < 0.01
    assert np.linalg.norm(rec[c, c, c] - vol[c, c, c]) / np.linalg.norm(vol[c, c, c]) < 0.08


def test_oracle_matches_reference_on_the_degenerate_fan_line():
    """intersectLines2D's NaN (parallel lines: pixels at the source's depth)
    reaches the reference's tex2D as a NaN coordinate, sampled as coordinate 0
    (half of the view's first texel); the oracle follows that rule and matches
    the reference's own outputs there."""
    g = load_golden("fan2d_degenerate")
    args = (g["volume_origin"], g["detector_origin"], g["volume_spacing"], g["detector_spacing"], g["sid"], g["sdd"],
            g["ray_vectors"])
    out = oracle.fan_backprojection2d(g["sinogram_in"], tuple(g["volume_shape"]), *args)
    assert np.isfinite(out).all()
    assert rel_l2(out, g["volume_ref"]) < 5e-4
    col = g["volume_ref"][0, :, 10]
    np.testing.assert_allclose(out[0, :, 10], col, rtol=1e-3, atol=1e-3 * np.abs(col).max())
