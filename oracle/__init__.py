"""CPU oracle and reference build for the projector ops -- TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference legs import this package, to check or time against it.  The product
(``pyro-nn-layers_b200``) never imports, links or calls anything here.

* ``liboracle.so`` (built from ``oracle.c`` by gcc): the FP64 restatement of
  the reference kernels, multithreaded with pthreads.
* ``_ref/libpyronn_ref.so`` (built by :func:`build_ref` from the reference's
  own ``cc/kernels/*.cu.cc`` where they lie, plus ``ref/compat.h`` and
  ``ref/ref_driver.cu``): the reference's CUDA launchers, for GPU-side
  comparisons and for generating golden fixtures.  Only buildable where the
  reference sources exist; the built file travels with the repository copy.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SRC = os.path.join(HERE, "oracle.c")
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libpyronn_ref.so")
# root of a PYRO-NN-Layers checkout whose cc/kernels/ build_ref compiles; no
# default: without it build_ref keeps an existing _ref/ library
REF_ROOT_ENV = "PYRONN_REFERENCE_ROOT"
REF_FILES = [
    "par_projector_2D_CudaKernel.cu.cc",
    "par_backprojector_2D_CudaKernel.cu.cc",
    "fan_projector_2D_CudaKernel.cu.cc",
    "fan_backprojector_2D_CudaKernel.cu.cc",
    "cone_projector_3D_CudaKernel.cu.cc",
    "cone_projector_3D_CudaKernel_hardware_interp.cu.cc",
    "cone_backprojector_3D_CudaKernel.cu.cc",
    "cone_backprojector_3D_CudaKernel_hardware_interp.cu.cc",
]


def build_oracle(force=False) -> str:
    if force or not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < os.path.getmtime(ORACLE_SRC):
        tmp = ORACLE_LIB + ".tmp"
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", "-pthread", "-o", tmp, ORACLE_SRC,
                        "-lm"], check=True)
        os.replace(tmp, ORACLE_LIB)
    return ORACLE_LIB


def reference_kernel_dir(root=None):
    """cc/kernels of the reference checkout given by `root` or by the
    PYRONN_REFERENCE_ROOT environment variable; None when neither is set."""
    root = root or os.environ.get(REF_ROOT_ENV)
    return os.path.join(root, "cc", "kernels") if root else None


def build_ref(force=False, root=None) -> str | None:
    """Compiles the reference's 8 kernel files unmodified (BUILD:44 flags:
    -DGOOGLE_CUDA=1, ftz=true) for sm_100a into _ref/, reading them where they
    lie under `root` (default: $PYRONN_REFERENCE_ROOT).  Without the reference
    sources (e.g. on a GPU box) it returns the existing library, or None."""
    src_dir = reference_kernel_dir(root)
    if src_dir is None or not os.path.isdir(src_dir):
        return REF_LIB if os.path.exists(REF_LIB) else None
    if os.path.exists(REF_LIB) and not force:
        return REF_LIB
    obj_dir = os.path.join(REF_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    nvcc = "nvcc" if subprocess.run(["which", "nvcc"], capture_output=True).returncode == 0 \
        else "/usr/local/cuda/bin/nvcc"
    common = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++14", "-ftz=true",
              "-Xcompiler", "-fPIC", "-w"]
    objs = []
    for f in REF_FILES:
        obj = os.path.join(obj_dir, f.replace(".cu.cc", ".o"))
        cmd = [nvcc] + common + ["-x", "cu", "-DGOOGLE_CUDA=1", "-include", os.path.join(HERE, "ref", "compat.h"),
                                 "-I", os.path.join(HERE, "ref", "stub"), "-c", os.path.join(src_dir, f), "-o", obj]
        subprocess.run(cmd, check=True)
        objs.append(obj)
    drv = os.path.join(obj_dir, "ref_driver.o")
    subprocess.run([nvcc] + common + ["-c", os.path.join(HERE, "ref", "ref_driver.cu"), "-o", drv], check=True)
    objs.append(drv)
    tmp = REF_LIB + ".tmp"
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] + objs, check=True)
    os.replace(tmp, REF_LIB)
    return REF_LIB


# ------------------------------------------------------------ CPU oracle API

_lib = None


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        L = ctypes.CDLL(ORACLE_LIB)
        P, I = ctypes.c_void_p, ctypes.c_int
        L.oracle_parallel_projection2d.argtypes = [P, P, I, I, I, I, I, P, P, P, P, P, I, I, P]
        L.oracle_fan_projection2d.argtypes = [P, P, I, I, I, I, I, P, P, P, P, P, P, P, I, I, P]
        L.oracle_parallel_backprojection2d.argtypes = [P, P, I, I, I, I, I, P, P, P, P, P, I, I]
        L.oracle_fan_backprojection2d.argtypes = [P, P, I, I, I, I, I, P, P, P, P, P, P, P, I, I]
        L.oracle_cone_projection3d.argtypes = [P, P, I, I, I, I, I, I, I, I, P, P, P, P, I, I, P]
        L.oracle_cone_backprojection3d.argtypes = [P, P, I, I, I, I, I, I, I, I, P, P, P, P, I, I]
        L.oracle_cone_decompose.argtypes = [P, P, P, I, P, P]
        L.oracle_cone_backprojection3d_slab.argtypes = [P, P, I, I, I, I, I, I, I, I, I, P, P, P, P, I]
        L.oracle_cone_projection3d_views.argtypes = [P, P, I, I, I, I, I, I, I, I, I, P, P, P, P, I, P]
        L.oracle_cone_backprojection3d_matched.argtypes = [P, P, I, I, I, I, I, I, I, P, P, P, P, I]
        for f in ("oracle_parallel_projection2d", "oracle_fan_projection2d", "oracle_parallel_backprojection2d",
                  "oracle_fan_backprojection2d", "oracle_cone_projection3d", "oracle_cone_backprojection3d",
                  "oracle_cone_decompose", "oracle_cone_backprojection3d_slab", "oracle_cone_projection3d_views",
                  "oracle_cone_backprojection3d_matched"):
            getattr(L, f).restype = None
        _lib = L
    return _lib


def default_threads():
    return os.cpu_count() or 1


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _geom_batch(batch, *arrays_and_rowsizes):
    g = 1
    for a, row in arrays_and_rowsizes:
        if a.size == row * batch and batch > 1:
            g = batch
    return g


def _rows(a, g, row):
    a = _f32(a).reshape(-1)
    if a.size == row and g > 1:
        a = np.tile(a, g)
    return np.ascontiguousarray(a)


def parallel_projection2d(volume, projection_shape, volume_origin, detector_origin, volume_spacing,
                          detector_spacing, ray_vectors, nthreads=None, counts=False):
    vol = _f32(volume)
    B, Y, X = vol.shape
    n_proj, W = (int(v) for v in projection_shape)
    g = _geom_batch(B, (_f32(volume_origin), 2), (_f32(ray_vectors), n_proj * 2))
    args = [_rows(volume_origin, g, 2), _rows(detector_origin, g, 1), _rows(volume_spacing, g, 2),
            _rows(detector_spacing, g, 1), _rows(ray_vectors, g, 2 * n_proj)]
    out = np.zeros((B, n_proj, W), dtype=np.float64)
    cnt = np.zeros(B * n_proj, dtype=np.int64)
    lib().oracle_parallel_projection2d(_ptr(vol), _ptr(out), B, Y, X, n_proj, W, *[_ptr(a) for a in args], g,
                                       nthreads or default_threads(), _ptr(cnt))
    return (out, cnt) if counts else out


def fan_projection2d(volume, projection_shape, volume_origin, detector_origin, volume_spacing, detector_spacing,
                     sid, sdd, central_ray_vectors, nthreads=None, counts=False):
    vol = _f32(volume)
    B, Y, X = vol.shape
    n_proj, W = (int(v) for v in projection_shape)
    g = _geom_batch(B, (_f32(volume_origin), 2), (_f32(central_ray_vectors), n_proj * 2))
    args = [_rows(volume_origin, g, 2), _rows(detector_origin, g, 1), _rows(volume_spacing, g, 2),
            _rows(detector_spacing, g, 1), _rows(sid, g, 1), _rows(sdd, g, 1), _rows(central_ray_vectors, g,
                                                                                    2 * n_proj)]
    out = np.zeros((B, n_proj, W), dtype=np.float64)
    cnt = np.zeros(B * n_proj, dtype=np.int64)
    lib().oracle_fan_projection2d(_ptr(vol), _ptr(out), B, Y, X, n_proj, W, *[_ptr(a) for a in args], g,
                                  nthreads or default_threads(), _ptr(cnt))
    return (out, cnt) if counts else out


def parallel_backprojection2d(sinogram, volume_shape, volume_origin, detector_origin, volume_spacing,
                              detector_spacing, ray_vectors, nthreads=None):
    sino = _f32(sinogram)
    B, n_proj, W = sino.shape
    Y, X = (int(v) for v in volume_shape)
    g = _geom_batch(B, (_f32(volume_origin), 2), (_f32(ray_vectors), n_proj * 2))
    args = [_rows(volume_origin, g, 2), _rows(detector_origin, g, 1), _rows(volume_spacing, g, 2),
            _rows(detector_spacing, g, 1), _rows(ray_vectors, g, 2 * n_proj)]
    out = np.zeros((B, Y, X), dtype=np.float64)
    lib().oracle_parallel_backprojection2d(_ptr(sino), _ptr(out), B, n_proj, W, Y, X, *[_ptr(a) for a in args], g,
                                           nthreads or default_threads())
    return out


def fan_backprojection2d(sinogram, volume_shape, volume_origin, detector_origin, volume_spacing, detector_spacing,
                         sid, sdd, central_ray_vectors, nthreads=None):
    sino = _f32(sinogram)
    B, n_proj, W = sino.shape
    Y, X = (int(v) for v in volume_shape)
    g = _geom_batch(B, (_f32(volume_origin), 2), (_f32(central_ray_vectors), n_proj * 2))
    args = [_rows(volume_origin, g, 2), _rows(detector_origin, g, 1), _rows(volume_spacing, g, 2),
            _rows(detector_spacing, g, 1), _rows(sid, g, 1), _rows(sdd, g, 1), _rows(central_ray_vectors, g,
                                                                                    2 * n_proj)]
    out = np.zeros((B, Y, X), dtype=np.float64)
    lib().oracle_fan_backprojection2d(_ptr(sino), _ptr(out), B, n_proj, W, Y, X, *[_ptr(a) for a in args], g,
                                      nthreads or default_threads())
    return out


def cone_projection3d(volume, projection_shape, volume_origin, volume_spacing, projection_matrices, step_size,
                      projection_multiplier=None, hardware_interp=False, nthreads=None, counts=False):
    vol = _f32(volume)
    B, Z, Y, X = vol.shape
    n_proj, H, W = (int(v) for v in projection_shape)
    g = _geom_batch(B, (_f32(volume_origin), 3), (_f32(projection_matrices), n_proj * 12))
    args = [_rows(volume_origin, g, 3), _rows(volume_spacing, g, 3), _rows(projection_matrices, g, 12 * n_proj),
            _rows(step_size, g, 1)]
    out = np.zeros((B, n_proj, H, W), dtype=np.float64)
    cnt = np.zeros(B * n_proj, dtype=np.int64)
    lib().oracle_cone_projection3d(_ptr(vol), _ptr(out), int(bool(hardware_interp)), B, Z, Y, X, n_proj, H, W,
                                   *[_ptr(a) for a in args], g, nthreads or default_threads(), _ptr(cnt))
    return (out, cnt) if counts else out


def cone_backprojection3d(sinogram, volume_shape, volume_origin, volume_spacing, projection_matrices,
                          step_size=None, projection_multiplier=1.0, hardware_interp=False, nthreads=None):
    sino = _f32(sinogram)
    B, n_proj, H, W = sino.shape
    Z, Y, X = (int(v) for v in volume_shape)
    g = _geom_batch(B, (_f32(volume_origin), 3), (_f32(projection_matrices), n_proj * 12))
    args = [_rows(volume_origin, g, 3), _rows(volume_spacing, g, 3), _rows(projection_matrices, g, 12 * n_proj),
            _rows(projection_multiplier, g, 1)]
    out = np.zeros((B, Z, Y, X), dtype=np.float64)
    lib().oracle_cone_backprojection3d(_ptr(sino), _ptr(out), int(bool(hardware_interp)), B, n_proj, H, W, Z, Y, X,
                                       *[_ptr(a) for a in args], g, nthreads or default_threads())
    return out


def cone_decompose(projection_matrices, volume_spacing, volume_origin):
    P = _f32(projection_matrices).reshape(-1, 12)
    n = P.shape[0]
    inv = np.zeros((n, 9), dtype=np.float64)
    src = np.zeros((n, 3), dtype=np.float64)
    lib().oracle_cone_decompose(_ptr(P), _ptr(_f32(volume_spacing)), _ptr(_f32(volume_origin)), n, _ptr(inv),
                                _ptr(src))
    return inv.reshape(n, 3, 3), src


def cone_backprojection3d_slab(sinogram, volume_shape, z_begin, z_end, volume_origin, volume_spacing,
                               projection_matrices, projection_multiplier=1.0, hardware_interp=False, nthreads=None):
    """Slices [z_begin, z_end) of batch element 0 (bounded CPU-baseline samples)."""
    sino = _f32(sinogram)
    n_proj, H, W = sino.shape[-3:]
    Z, Y, X = (int(v) for v in volume_shape)
    out = np.zeros((Z, Y, X), dtype=np.float64)
    lib().oracle_cone_backprojection3d_slab(
        _ptr(sino), _ptr(out), int(bool(hardware_interp)), n_proj, H, W, Z, Y, X, z_begin, z_end,
        _ptr(_f32(volume_origin)), _ptr(_f32(volume_spacing)), _ptr(_f32(projection_matrices)),
        _ptr(_f32(np.atleast_1d(projection_multiplier))), nthreads or default_threads())
    return out


def cone_projection3d_views(volume, projection_shape, p_begin, p_end, volume_origin, volume_spacing,
                            projection_matrices, step_size, hardware_interp=False, nthreads=None):
    """Views [p_begin, p_end) of batch element 0; returns (sinogram, sample counts)."""
    vol = _f32(volume)
    Z, Y, X = vol.shape[-3:]
    n_proj, H, W = (int(v) for v in projection_shape)
    out = np.zeros((n_proj, H, W), dtype=np.float64)
    cnt = np.zeros(n_proj, dtype=np.int64)
    lib().oracle_cone_projection3d_views(
        _ptr(vol), _ptr(out), int(bool(hardware_interp)), Z, Y, X, n_proj, H, W, p_begin, p_end,
        _ptr(_f32(volume_origin)), _ptr(_f32(volume_spacing)), _ptr(_f32(projection_matrices)),
        _ptr(_f32(np.atleast_1d(step_size))), nthreads or default_threads(), _ptr(cnt))
    return out, cnt


def cone_backprojection3d_matched(sinogram, volume_shape, volume_origin, volume_spacing, projection_matrices,
                                  step_size, projection_multiplier=None):
    """Exact transpose of the linear software forward projector (FP64)."""
    sino = _f32(sinogram)
    B, n_proj, H, W = sino.shape
    Z, Y, X = (int(v) for v in volume_shape)
    g = _geom_batch(B, (_f32(volume_origin), 3), (_f32(projection_matrices), n_proj * 12))
    args = [_rows(volume_origin, g, 3), _rows(volume_spacing, g, 3), _rows(projection_matrices, g, 12 * n_proj),
            _rows(step_size, g, 1)]
    out = np.zeros((B, Z, Y, X), dtype=np.float64)
    lib().oracle_cone_backprojection3d_matched(_ptr(sino), _ptr(out), B, n_proj, H, W, Z, Y, X,
                                               *[_ptr(a) for a in args], g)
    return out


from .filters import cosine_weights, fdk_filter, ramp_kernel  # noqa: E402,F401  (FDK / FBP pre-processing)
