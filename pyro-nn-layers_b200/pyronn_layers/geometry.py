"""Trajectory and grid helpers that produce the geometry tensors of the ops.

These are the callers' side of the projector ops (the PYRO-NN package builds
the same tensors in Python): ray vectors for 2D parallel/fan beam, the 3x4
projection matrices of a circular cone-beam trajectory, and centred origins.
Everything is computed in FP64 and handed to the ops as FP32.

Conventions (shared with the kernels):
* 2D: view angle theta has ray / central-ray vector (cos theta, sin theta); the
  detector axis is (-sin theta, cos theta); a fan source sits at
  -SID * (cos theta, sin theta).
* 3D: the source circles the z axis at -SID * (cos theta, sin theta, 0); the
  principal ray points along (cos theta, sin theta, 0); detector columns (u)
  run along (-sin theta, cos theta, 0), rows (v) along +z; the principal point
  is the detector centre unless an offset is given.  P maps homogeneous world
  mm (x, y, z, 1) to (u w, v w, w) in detector pixel indices, w being the
  depth from the source along the principal ray.
"""
from __future__ import annotations

import math

import numpy as np


def centered_origin(shape, spacing):
    """Origin (mm, same axis order as shape) that centres a grid on 0: -(N-1)/2 * s."""
    shape = np.asarray(shape, dtype=np.float64)
    spacing = np.asarray(spacing, dtype=np.float64)
    return (-(shape - 1.0) / 2.0 * spacing).astype(np.float32)


def view_angles(n_proj: int, angular_range: float = 2.0 * math.pi, start: float = 0.0):
    """n_proj angles evenly spaced on [start, start + angular_range)."""
    return start + np.arange(n_proj, dtype=np.float64) * (angular_range / n_proj)


def ray_vectors_2d(n_proj: int, angular_range: float = math.pi, start: float = 0.0):
    """[n_proj, 2] (cos, sin) of each view angle, float32."""
    a = view_angles(n_proj, angular_range, start)
    return np.stack([np.cos(a), np.sin(a)], axis=1).astype(np.float32)


def circular_projection_matrices(n_proj: int, sid: float, sdd: float, detector_shape, detector_spacing,
                                 angular_range: float = 2.0 * math.pi, start: float = 0.0,
                                 principal_point=None):
    """[n_proj, 3, 4] float32 projection matrices of a circular cone-beam scan.

    detector_shape = (H, W) pixels, detector_spacing = (dv, du) mm;
    principal_point = (cv, cu) in pixel indices (default: detector centre)."""
    H, W = int(detector_shape[0]), int(detector_shape[1])
    dv, du = float(detector_spacing[0]), float(detector_spacing[1])
    if principal_point is None:
        cv, cu = (H - 1) / 2.0, (W - 1) / 2.0
    else:
        cv, cu = float(principal_point[0]), float(principal_point[1])
    K = np.array([[sdd / du, 0.0, cu], [0.0, sdd / dv, cv], [0.0, 0.0, 1.0]], dtype=np.float64)
    out = np.empty((n_proj, 3, 4), dtype=np.float64)
    for i, th in enumerate(view_angles(n_proj, angular_range, start)):
        c, s = math.cos(th), math.sin(th)
        src = np.array([-sid * c, -sid * s, 0.0])
        R = np.array([[-s, c, 0.0], [0.0, 0.0, 1.0], [c, s, 0.0]])
        Rt = np.concatenate([R, (-R @ src)[:, None]], axis=1)
        out[i] = K @ Rt
    return out.astype(np.float32)


def detector_origin_1d(width: int, spacing: float):
    """Centred detector origin -(W-1)/2 * du (mm), shape [1]."""
    return np.array([-(width - 1) / 2.0 * spacing], dtype=np.float32)


class ParallelBeam2D:
    """Geometry tensors of a 2D parallel-beam scan, in the op argument order."""

    def __init__(self, volume_shape, volume_spacing, detector_width, detector_spacing, n_proj,
                 angular_range=math.pi):
        self.volume_shape = tuple(int(v) for v in volume_shape)
        self.volume_spacing = np.asarray(volume_spacing, dtype=np.float32)
        self.volume_origin = centered_origin(self.volume_shape, self.volume_spacing)
        self.detector_shape = (int(n_proj), int(detector_width))
        self.detector_spacing = np.array([detector_spacing], dtype=np.float32)
        self.detector_origin = detector_origin_1d(detector_width, detector_spacing)
        self.ray_vectors = ray_vectors_2d(n_proj, angular_range)

    def args(self):
        return (self.volume_origin, self.detector_origin, self.volume_spacing, self.detector_spacing,
                self.ray_vectors)


class FanBeam2D(ParallelBeam2D):
    """Geometry tensors of a 2D fan-beam scan with a flat equispaced detector."""

    def __init__(self, volume_shape, volume_spacing, detector_width, detector_spacing, n_proj, sid, sdd,
                 angular_range=2.0 * math.pi):
        super().__init__(volume_shape, volume_spacing, detector_width, detector_spacing, n_proj, angular_range)
        self.sid = np.array([sid], dtype=np.float32)
        self.sdd = np.array([sdd], dtype=np.float32)

    def args(self):
        return (self.volume_origin, self.detector_origin, self.volume_spacing, self.detector_spacing, self.sid,
                self.sdd, self.ray_vectors)


class ConeBeam3D:
    """Geometry tensors of a circular cone-beam scan, in the op argument order."""

    def __init__(self, volume_shape, volume_spacing, detector_shape, detector_spacing, n_proj, sid, sdd,
                 angular_range=2.0 * math.pi, step_size=0.5, projection_multiplier=None):
        self.volume_shape = tuple(int(v) for v in volume_shape)
        self.volume_spacing = np.asarray(volume_spacing, dtype=np.float32)
        self.volume_origin = centered_origin(self.volume_shape, self.volume_spacing)
        self.detector_shape = (int(n_proj),) + tuple(int(v) for v in detector_shape)
        self.detector_spacing = tuple(float(v) for v in detector_spacing)
        self.sid, self.sdd = float(sid), float(sdd)
        self.projection_matrices = circular_projection_matrices(n_proj, sid, sdd, detector_shape,
                                                                detector_spacing, angular_range)
        self.step_size = np.array([step_size], dtype=np.float32)
        if projection_multiplier is None:
            projection_multiplier = 1.0
        self.projection_multiplier = np.array([projection_multiplier], dtype=np.float32)

    def args(self):
        return (self.volume_origin, self.volume_spacing, self.projection_matrices, self.step_size,
                self.projection_multiplier)
