"""Trajectory builders and phantoms (host side, no GPU)."""
import math

import numpy as np

from pyronn_layers import geometry, phantoms


def test_projection_matrices_null_vector_is_the_source():
    P = geometry.circular_projection_matrices(12, 750.0, 1200.0, (768, 1024), (1.0, 1.0)).astype(np.float64)
    for p, th in enumerate(geometry.view_angles(12)):
        src = np.array([-750 * math.cos(th), -750 * math.sin(th), 0.0, 1.0])
        r = P[p] @ src
        assert np.abs(r).max() < 1e-3 * np.abs(P[p]).max()
        # the isocentre projects to the detector centre at depth SID
        c = P[p] @ np.array([0.0, 0.0, 0.0, 1.0])
        np.testing.assert_allclose(c[2], 750.0, rtol=1e-6)
        np.testing.assert_allclose(c[:2] / c[2], [(1024 - 1) / 2, (768 - 1) / 2], atol=1e-3)


def test_magnification_and_orientation():
    P = geometry.circular_projection_matrices(1, 750.0, 1200.0, (100, 100), (1.0, 1.0)).astype(np.float64)[0]
    # at angle 0 the detector u axis is +y, v is +z; 1 mm at the isocentre -> 1.6 px
    c = P @ np.array([0, 0, 0, 1.0])
    dy = P @ np.array([0, 1.0, 0, 1.0])
    dz = P @ np.array([0, 0, 1.0, 1.0])
    np.testing.assert_allclose(dy[0] / dy[2] - c[0] / c[2], 1.6, rtol=1e-6)
    np.testing.assert_allclose(dz[1] / dz[2] - c[1] / c[2], 1.6, rtol=1e-6)


def test_ray_vectors_and_origins():
    r = geometry.ray_vectors_2d(180, math.pi)
    np.testing.assert_allclose(np.linalg.norm(r, axis=1), 1.0, rtol=1e-6)
    np.testing.assert_allclose(r[90], [0.0, 1.0], atol=1e-6)
    np.testing.assert_allclose(geometry.centered_origin((256, 256), (1.0, 1.0)), [-127.5, -127.5])
    np.testing.assert_allclose(geometry.detector_origin_1d(367, 1.0), [-183.0])


def test_phantoms_are_seeded():
    a, ea = phantoms.ellipse_phantom_2d((64, 64), (1, 1), seed=5)
    b, eb = phantoms.ellipse_phantom_2d((64, 64), (1, 1), seed=5)
    c, _ = phantoms.ellipse_phantom_2d((64, 64), (1, 1), seed=6)
    np.testing.assert_array_equal(a, b)
    assert not np.array_equal(a, c)
    assert ea.shape == (10, 6) and a.max() > 0
    v, ell = phantoms.ellipsoid_phantom_3d((24, 24, 24), (2.0, 2.0, 2.0), seed=3, n=8)
    assert v.shape == (24, 24, 24) and len(ell) == 8 and v.max() > 0


def test_ellipse_line_integral_chord():
    ell = np.array([[0.0, 0.0, 10.0, 5.0, 0.0, 2.0]])
    # horizontal line through the centre: chord 20 mm, density 2
    assert abs(phantoms.ellipse_line_integral(ell, (-50.0, 0.0), (1.0, 0.0)) - 40.0) < 1e-9
    assert phantoms.ellipse_line_integral(ell, (-50.0, 6.0), (1.0, 0.0)) == 0.0
