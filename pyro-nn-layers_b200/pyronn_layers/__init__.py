"""pyronn_layers -- B200-native projector ops with the PYRO-NN-Layers op surface.

The reference exposes its ops under the ``pyronn_layers`` namespace
(python/ops/pyronn_layers_ops.py:27-29); the same names live here:

    parallel_projection2d, parallel_backprojection2d,
    fan_projection2d, fan_backprojection2d,
    cone_projection3d, cone_backprojection3d

They run hand-written sm_100a CUDA kernels through the C ABI of
``include/pyronn_b200.h`` (``libpyronn_b200.so`` in this directory).
"""
from .ops import (  # noqa: F401
    check_device_errors,
    circular_projection_matrices,
    circular_ray_vectors_2d,
    cone_backprojection3d,
    cone_backprojection3d_matched,
    cone_projection3d,
    device_errors,
    fan_backprojection2d,
    fan_projection2d,
    parallel_backprojection2d,
    parallel_projection2d,
    release_cached_arrays,
    set_sync_error_checks,
)
from ._capi import PyronnDeviceError, PyronnError  # noqa: F401
from . import fbp, geometry, phantoms  # noqa: F401

__all__ = [
    "parallel_projection2d",
    "parallel_backprojection2d",
    "fan_projection2d",
    "fan_backprojection2d",
    "cone_projection3d",
    "cone_backprojection3d",
    "cone_backprojection3d_matched",
    "release_cached_arrays",
    "circular_projection_matrices",
    "circular_ray_vectors_2d",
    "PyronnError",
    "PyronnDeviceError",
    "check_device_errors",
    "device_errors",
    "set_sync_error_checks",
    "fbp",
    "geometry",
    "phantoms",
]
