"""Parity with the reference's own CUDA kernels (built unmodified from its
sources into oracle/_ref) at a larger size than the golden fixtures, and a
side-by-side timing on the same GPU.

Set PYRONN_TIMING_OUT=<file> to have the timings written as JSON."""
import ctypes
import json
import os

import numpy as np
import pytest
import torch

import oracle
import pyronn_layers as pl
from pyronn_layers import geometry, phantoms
from conftest import rel_l2

pytestmark = pytest.mark.gpu

KEEP = []  # buffers handed to the reference live until the module ends


def ref_lib():
    path = oracle.REF_LIB
    if not os.path.exists(path):
        pytest.skip("oracle/_ref/libpyronn_ref.so not built (needs the reference sources)")
    L = ctypes.CDLL(path)
    L.ref_cone_projection3d.restype = ctypes.c_int
    L.ref_cone_backprojection3d.restype = ctypes.c_int
    return L


def dptr(a, dev, slack=0):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32)).reshape(-1)
    t = torch.zeros(a.size + slack, dtype=torch.float32, device=dev)
    t[: a.size] = torch.from_numpy(a).to(dev)
    KEEP.append(t)
    return ctypes.c_void_p(t.data_ptr())


def timed(fn, reps=3):
    fn()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(reps):
        fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps


def test_cone_parity_and_speed_vs_reference(cuda):
    L = ref_lib()
    shape, n_proj, det = (256, 256, 256), 24, (512, 512)
    geo = geometry.ConeBeam3D(shape, (0.5, 0.5, 0.5), det, (1.0, 1.0), n_proj, 750.0, 1200.0, step_size=0.5)
    sp = np.asarray(geo.volume_spacing, np.float64)
    ell = phantoms.random_ellipsoids(11, [shape[k] * sp[k] for k in (2, 1, 0)], n=32)
    vol = phantoms.rasterise_ellipsoids_torch(ell, shape, sp, geo.volume_origin, cuda)[None].contiguous()
    vo, vs, P, st, mu = (np.asarray(a, np.float32)[None] for a in geo.args())
    H, W = det
    Z, Y, X = shape

    ours_s = pl.cone_projection3d(vol, geo.detector_shape, *geo.args())
    ref_s = torch.zeros(n_proj * H * W, device=cuda)
    args_f = (ctypes.c_void_p(vol.data_ptr()), ctypes.c_void_p(ref_s.data_ptr()), 0, 1, Z, Y, X, n_proj, H, W,
              dptr(vo, cuda), dptr(vs, cuda), dptr(P, cuda), dptr(st, cuda))
    assert L.ref_cone_projection3d(*args_f) == 0
    torch.cuda.synchronize()
    e_f = rel_l2(ours_s.cpu().numpy().ravel(), ref_s.cpu().numpy())

    sino = ours_s.contiguous()
    sino_pad = torch.zeros(sino.numel() + W + 8, device=cuda)  # slack for the reference's past-the-end taps
    sino_pad[: sino.numel()] = sino.reshape(-1)
    ours_v = pl.cone_backprojection3d(sino, geo.volume_shape, *geo.args())
    ref_v = torch.zeros(Z * Y * X, device=cuda)
    args_b = (ctypes.c_void_p(sino_pad.data_ptr()), ctypes.c_void_p(ref_v.data_ptr()), 0, 1, n_proj, H, W, Z, Y, X,
              dptr(vo, cuda), dptr(vs, cuda), dptr(P, cuda), dptr(mu, cuda))
    assert L.ref_cone_backprojection3d(*args_b) == 0
    torch.cuda.synchronize()
    e_b = rel_l2(ours_v.cpu().numpy().ravel(), ref_v.cpu().numpy())
    assert e_f < 2e-5, e_f
    assert e_b < 1e-5, e_b

    t = {
        "config": "cone 256^3 at 0.5 mm, %d views, 512x512 detector, step 0.5 voxel, FP32" % n_proj,
        "forward_rel_l2_vs_reference": e_f, "backprojection_rel_l2_vs_reference": e_b,
        "ours_forward_ms": timed(lambda: pl.cone_projection3d(vol, geo.detector_shape, *geo.args())),
        "reference_forward_ms": timed(lambda: L.ref_cone_projection3d(*args_f)),
        "ours_backprojection_ms": timed(lambda: pl.cone_backprojection3d(sino, geo.volume_shape, *geo.args())),
        "reference_backprojection_ms": timed(lambda: L.ref_cone_backprojection3d(*args_b)),
    }
    out = os.environ.get("PYRONN_TIMING_OUT")
    if out:
        with open(out, "w") as f:
            json.dump(t, f, indent=1)
