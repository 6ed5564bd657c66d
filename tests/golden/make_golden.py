"""Generates the golden fixtures tests/golden/*.npz from the reference itself.

    python tests/golden/make_golden.py [--out DIR] [--only NAME,...]     (needs a CUDA GPU)

Runs the reference's own CUDA launchers (cc/kernels/*.cu.cc of PYRO-NN-Layers,
compiled unmodified into oracle/_ref/libpyronn_ref.so by oracle.build_ref(),
with PYRONN_REFERENCE_ROOT set to the reference checkout)
on small seeded inputs through oracle/ref/ref_driver.cu, which restates the
TF op layer (per-batch-element launcher loop; FP64 projection-matrix
decomposition rounded to FP32).  Each fixture stores the inputs, the geometry
and the reference output, so the tests need neither the generator nor the
reference at run time.

The software cone backprojector of the reference can read up to W+1 elements
past the end of its sinogram (its `>` bounds, cone_backprojector_3D_CudaKernel.cu.cc:68-71);
every sinogram handed to it here is allocated with that much zeroed slack.
"""
from __future__ import annotations

import ctypes
import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "pyro-nn-layers_b200"))

import torch  # noqa: E402

import oracle  # noqa: E402
from pyronn_layers import geometry, phantoms  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


# every device buffer handed to the reference stays referenced here until the
# script ends: a temporary freed before the call would hand its block to the
# next allocation and the reference would read the wrong data
_KEEP = []


def dev(a, slack=0):
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    t = torch.zeros(a.size + slack, dtype=torch.float32, device="cuda")
    t[: a.size] = torch.from_numpy(a.reshape(-1)).cuda()
    _KEEP.append(t)
    return t


def check_geometry(step_like):
    """The reference's march loops forever on a zero step: refuse one."""
    if not np.all(np.asarray(step_like, np.float64) > 0):
        raise ValueError("non-positive spacing/step would stall the reference kernel")


def ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def load_ref():
    path = oracle.build_ref()
    if path is None or not os.path.exists(path):
        raise SystemExit("oracle/_ref/libpyronn_ref.so missing: build it where the reference sources exist "
                         "(PYRONN_REFERENCE_ROOT=<checkout> python -c 'import oracle; oracle.build_ref()')")
    return ctypes.CDLL(path)


def check(rc, what):
    if rc != 0:
        raise RuntimeError("%s returned CUDA error %d" % (what, rc))


def case_parallel(L):
    B, Y, X, n_proj, W = 2, 64, 64, 60, 95
    vols = np.stack([phantoms.ellipse_phantom_2d((Y, X), (1.0, 1.0), seed=10 + b, n=6)[0] for b in range(B)])
    vs = np.array([[1.0, 1.0], [1.0, 1.0]], np.float32)
    check_geometry(vs)
    vo = np.stack([geometry.centered_origin((Y, X), vs[b]) for b in range(B)])
    ds = np.array([[1.0], [1.0]], np.float32)
    do = np.stack([geometry.detector_origin_1d(W, 1.0)] * B)
    rays = np.stack([geometry.ray_vectors_2d(n_proj, math.pi), geometry.ray_vectors_2d(n_proj, math.pi, 0.05)])
    sino = torch.zeros(B * n_proj * W, device="cuda")
    check(L.ref_parallel_projection2d(ptr(dev(vols)), ptr(sino), B, Y, X, n_proj, W, ptr(dev(vo)), ptr(dev(do)),
                                      ptr(dev(vs)), ptr(dev(ds)), ptr(dev(rays))), "par fp")
    rng = np.random.Generator(np.random.PCG64(7))
    sino_in = rng.uniform(0.0, 1.0, (B, n_proj, W)).astype(np.float32)
    vol_out = torch.zeros(B * Y * X, device="cuda")
    check(L.ref_parallel_backprojection2d(ptr(dev(sino_in)), ptr(vol_out), B, n_proj, W, Y, X, ptr(dev(vo)),
                                          ptr(dev(do)), ptr(dev(vs)), ptr(dev(ds)), ptr(dev(rays))), "par bp")
    np.savez_compressed(os.path.join(OUT, "parallel2d.npz"), volume=vols, volume_origin=vo, volume_spacing=vs,
                        detector_origin=do, detector_spacing=ds, ray_vectors=rays, projection_shape=[n_proj, W],
                        sinogram_ref=sino.cpu().numpy().reshape(B, n_proj, W), sinogram_in=sino_in,
                        volume_ref=vol_out.cpu().numpy().reshape(B, Y, X))


def case_fan(L):
    B, Y, X, n_proj, W = 2, 64, 64, 72, 128
    vs = np.array([[0.5, 0.5], [0.5, 0.5]], np.float32)
    check_geometry(vs)
    vols = np.stack([phantoms.ellipse_phantom_2d((Y, X), (0.5, 0.5), seed=20 + b, n=6)[0] for b in range(B)])
    vo = np.stack([geometry.centered_origin((Y, X), vs[b]) for b in range(B)])
    ds = np.array([[0.5], [0.5]], np.float32)
    do = np.stack([geometry.detector_origin_1d(W, 0.5)] * B)
    sid = np.array([[75.0], [80.0]], np.float32)
    sdd = np.array([[120.0], [125.0]], np.float32)
    rays = np.stack([geometry.ray_vectors_2d(n_proj, 2 * math.pi), geometry.ray_vectors_2d(n_proj, 2 * math.pi,
                                                                                          0.1)])
    sino = torch.zeros(B * n_proj * W, device="cuda")
    check(L.ref_fan_projection2d(ptr(dev(vols)), ptr(sino), B, Y, X, n_proj, W, ptr(dev(vo)), ptr(dev(do)),
                                 ptr(dev(vs)), ptr(dev(ds)), ptr(dev(sid)), ptr(dev(sdd)), ptr(dev(rays))),
          "fan fp")
    rng = np.random.Generator(np.random.PCG64(8))
    sino_in = rng.uniform(0.0, 1.0, (B, n_proj, W)).astype(np.float32)
    vol_out = torch.zeros(B * Y * X, device="cuda")
    check(L.ref_fan_backprojection2d(ptr(dev(sino_in)), ptr(vol_out), B, n_proj, W, Y, X, ptr(dev(vo)),
                                     ptr(dev(do)), ptr(dev(vs)), ptr(dev(ds)), ptr(dev(sid)), ptr(dev(sdd)),
                                     ptr(dev(rays))), "fan bp")
    np.savez_compressed(os.path.join(OUT, "fan2d.npz"), volume=vols, volume_origin=vo, volume_spacing=vs,
                        detector_origin=do, detector_spacing=ds, sid=sid, sdd=sdd, ray_vectors=rays,
                        projection_shape=[n_proj, W], sinogram_ref=sino.cpu().numpy().reshape(B, n_proj, W),
                        sinogram_in=sino_in, volume_ref=vol_out.cpu().numpy().reshape(B, Y, X))


def case_fan_degenerate(L):
    """Fan backprojection with pixels on intersectLines2D's degenerate line:
    the source inside the field (SID 5.5 mm, then 15.5 mm: the column of
    pixels at x = -SID for the view along +x, and the row, column or row at
    distance SID for the other axis views), where the reference's lines are
    parallel and its intersection is NaN
    (cc/helper_headers/helper_geometry_gpu.h:30-36)."""
    B, Y, X, W = 2, 32, 32, 40
    vs = np.array([[1.0, 1.0], [1.0, 1.0]], np.float32)
    check_geometry(vs)
    vo = np.stack([geometry.centered_origin((Y, X), vs[b]) for b in range(B)])
    ds = np.array([[1.0], [1.0]], np.float32)
    do = np.stack([geometry.detector_origin_1d(W, 1.0)] * B)
    sid = np.array([[5.5], [15.5]], np.float32)
    sdd = sid + np.float32(30.0)
    views = np.array([[1.0, 0.0], [0.0, 1.0], [-1.0, 0.0], [0.0, -1.0], [0.6, 0.8],
                      [math.cos(1.0), math.sin(1.0)]], np.float32)
    rays = np.stack([views, views])
    n_proj = views.shape[0]
    rng = np.random.Generator(np.random.PCG64(9))
    sino_in = rng.uniform(0.5, 1.0, (B, n_proj, W)).astype(np.float32)
    vol_out = torch.zeros(B * Y * X, device="cuda")
    check(L.ref_fan_backprojection2d(ptr(dev(sino_in)), ptr(vol_out), B, n_proj, W, Y, X, ptr(dev(vo)),
                                     ptr(dev(do)), ptr(dev(vs)), ptr(dev(ds)), ptr(dev(sid)), ptr(dev(sdd)),
                                     ptr(dev(rays))), "fan bp degenerate")
    np.savez_compressed(os.path.join(OUT, "fan2d_degenerate.npz"), volume_shape=[Y, X], volume_origin=vo,
                        volume_spacing=vs, detector_origin=do, detector_spacing=ds, sid=sid, sdd=sdd,
                        ray_vectors=rays, sinogram_in=sino_in, volume_ref=vol_out.cpu().numpy().reshape(B, Y, X))


def cone_case(L, name, vol_shape, spacing, det_shape, det_spacing, n_proj, sid, sdd, step, seed):
    Z, Y, X = vol_shape
    H, W = det_shape
    g = geometry.ConeBeam3D(vol_shape, spacing, det_shape, det_spacing, n_proj, sid, sdd, step_size=step,
                            projection_multiplier=0.75)
    vol = phantoms.ellipsoid_phantom_3d(vol_shape, spacing, seed=seed, n=8)[0][None]
    vo, vs, P, st, mu = (np.asarray(a, np.float32) for a in g.args())
    vo, vs, st, mu = vo[None], vs[None], st[None], mu[None]
    P = P[None]
    check_geometry(vs)
    check_geometry(st)
    out = {}
    for hw in (0, 1):
        sino = torch.zeros(n_proj * H * W, device="cuda")
        check(L.ref_cone_projection3d(ptr(dev(vol)), ptr(sino), hw, 1, Z, Y, X, n_proj, H, W, ptr(dev(vo)),
                                      ptr(dev(vs)), ptr(dev(P)), ptr(dev(st))), "cone fp hw=%d" % hw)
        out["sinogram_ref_hw%d" % hw] = sino.cpu().numpy().reshape(1, n_proj, H, W)
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    sino_in = rng.uniform(0.0, 1.0, (1, n_proj, H, W)).astype(np.float32)
    for hw in (0, 1):
        v = torch.zeros(Z * Y * X, device="cuda")
        # W + 1 zeroed elements of slack for the reference's past-the-end taps
        check(L.ref_cone_backprojection3d(ptr(dev(sino_in, slack=W + 8)), ptr(v), hw, 1, n_proj, H, W, Z, Y, X,
                                          ptr(dev(vo)), ptr(dev(vs)), ptr(dev(P)), ptr(dev(mu))),
              "cone bp hw=%d" % hw)
        out["volume_ref_hw%d" % hw] = v.cpu().numpy().reshape(1, Z, Y, X)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), volume=vol, volume_origin=vo, volume_spacing=vs,
                        projection_matrices=P, step_size=st, projection_multiplier=mu,
                        projection_shape=[n_proj, H, W], sinogram_in=sino_in, **out)


def main():
    global OUT
    if "--out" in sys.argv:
        OUT = sys.argv[sys.argv.index("--out") + 1]
        os.makedirs(OUT, exist_ok=True)
    L = load_ref()
    for f in ("ref_parallel_projection2d", "ref_parallel_backprojection2d", "ref_fan_projection2d",
              "ref_fan_backprojection2d", "ref_cone_projection3d", "ref_cone_backprojection3d"):
        getattr(L, f).restype = ctypes.c_int
    torch.cuda.init()
    only = sys.argv[sys.argv.index("--only") + 1].split(",") if "--only" in sys.argv else None
    cases = {"parallel2d": lambda: case_parallel(L), "fan2d": lambda: case_fan(L),
             "fan2d_degenerate": lambda: case_fan_degenerate(L),
             # detector covers the whole volume shadow
             "cone3d": lambda: cone_case(L, "cone3d", (24, 32, 40), (1.0, 1.0, 1.0), (40, 56), (1.5, 1.5), 24, 200.0,
                                         320.0, 0.5, 30),
             # small detector: the shadow overflows every edge (out-of-detector
             # taps, the software backprojector's next-row / next-view taps)
             "cone3d_edges": lambda: cone_case(L, "cone3d_edges", (20, 28, 28), (1.0, 1.0, 1.0), (16, 20), (1.5, 1.5),
                                               12, 150.0, 260.0, 0.7, 40)}
    for name, run in cases.items():
        if only is None or name in only:
            run()
    print("golden fixtures written to", OUT)


if __name__ == "__main__":
    main()
