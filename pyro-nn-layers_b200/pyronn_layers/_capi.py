"""ctypes binding of the C ABI in ``include/pyronn_b200.h``.

The library ``libpyronn_b200.so`` sits next to this file (built in-tree by
``pyro-nn-layers_b200/build.py``).  There is no fallback implementation: if the
library is missing or fails to load, every op raises.
"""
from __future__ import annotations

import ctypes
import os

LIB_NAME = "libpyronn_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

ABI_VERSION = 1

FLOAT32 = 0
BFLOAT16 = 1
FLOAT16 = 2

SUCCESS = 0
ERROR_INVALID_ARGUMENT = 1
ERROR_UNSUPPORTED = 2
ERROR_WORKSPACE_TOO_SMALL = 3
ERROR_CUDA = 4

_P = ctypes.c_void_p
_I = ctypes.c_int
_SZ = ctypes.c_size_t
_D = ctypes.c_double

# name -> (restype, argtypes); mirrors include/pyronn_b200.h
PROTOTYPES = {
    "pyronn_abi_version": (_I, []),
    "pyronn_status_string": (ctypes.c_char_p, [_I]),
    "pyronn_last_error": (ctypes.c_char_p, []),
    "pyronn_release_cached_arrays": (_I, []),
    "pyronn_workspace_error": (_I, [_P, _P, _P]),
    "pyronn_debug_starve_tma_wait": (_I, [_I]),
    "pyronn_noalloc_error": (_I, [_P, _P]),
    "pyronn_fdk_error": (_I, [_P, _P]),
    "pyronn_projection2d_workspace_size": (_SZ, [_I] * 4),
    "pyronn_parallel_projection2d": (
        _I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _I, _P, _SZ, _P]),
    "pyronn_parallel_backprojection2d": (_I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _I, _P]),
    "pyronn_fan_projection2d": (
        _I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _I, _P, _SZ, _P]),
    "pyronn_fan_backprojection2d": (_I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P, _I, _P]),
    "pyronn_cone_projection3d_workspace_size": (_SZ, [_I] * 10),
    "pyronn_cone_projection3d": (
        _I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _I, _P, _SZ, _P]),
    "pyronn_cone_backprojection3d_workspace_size": (_SZ, [_I] * 10),
    "pyronn_cone_backprojection3d": (
        _I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _I, _P, _SZ, _P]),
    "pyronn_cone_backprojection3d_matched_workspace_size": (_SZ, [_I, _I]),
    "pyronn_cone_backprojection3d_matched": (
        _I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _I, _P, _SZ, _P]),
    "pyronn_cone_backprojection3d_noalloc": (
        _I, [_P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _I, _P]),
    "pyronn_circular_projection_matrices": (_I, [_P, _I] + [_D] * 8 + [_P]),
    "pyronn_circular_ray_vectors_2d": (_I, [_P, _I, _D, _D, _P]),
    "pyronn_fdk_filter": (_I, [_P, _P, _I, _I, _I, _I, _I, _I] + [_D] * 5 + [_I, _I, _P]),
}

DEVICE_ERROR_NONE = 0  # PYRONN_DEVICE_ERROR_NONE
DEVICE_ERROR_WAIT_TIMEOUT = 1  # PYRONN_DEVICE_ERROR_WAIT_TIMEOUT

NOALLOC_MAX_VIEWS = 8192  # PYRONN_NOALLOC_MAX_VIEWS
FILTER_RAM_LAK = 0  # PYRONN_FILTER_RAM_LAK
FILTER_SHEPP_LOGAN = 1  # PYRONN_FILTER_SHEPP_LOGAN
FDK_MAX_WIDTH = 4096  # PYRONN_FDK_MAX_WIDTH


class PyronnError(RuntimeError):
    """A non-success status returned by the C ABI."""

    def __init__(self, func, status, detail):
        self.func = func
        self.status = status
        self.detail = detail
        super().__init__("%s failed: %s (status %d)%s" % (
            func, _status_name(status), status, (": " + detail) if detail else ""))


class PyronnDeviceError(RuntimeError):
    """A kernel reported a device-side failure (a bounded wait that gave up)
    after its call had returned: the affected results were not written."""

    def __init__(self, flags, what="device"):
        self.flags = flags
        super().__init__("%s error flags 0x%x: a bounded wait for an asynchronous copy or tensor-core "
                         "operation gave up; the affected output was not written" % (what, flags))


def _status_name(status):
    return {
        SUCCESS: "success",
        ERROR_INVALID_ARGUMENT: "invalid argument",
        ERROR_UNSUPPORTED: "unsupported",
        ERROR_WORKSPACE_TOO_SMALL: "workspace too small",
        ERROR_CUDA: "CUDA error",
    }.get(status, "unknown status")


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads (once) and returns the library; raises ImportError if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            "%s not found: build it with `python pyro-nn-layers_b200/build.py` "
            "(there is no CPU fallback for the projector ops)" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    ver = lib.pyronn_abi_version()
    if ver != ABI_VERSION:
        raise ImportError("%s has ABI version %d, expected %d" % (path, ver, ABI_VERSION))
    _lib = lib
    return lib


def call(name: str, *args) -> None:
    """Calls an entry point and raises PyronnError on a non-success status."""
    lib = load()
    status = getattr(lib, name)(*args)
    if status != SUCCESS:
        detail = lib.pyronn_last_error().decode("utf-8", "replace")
        raise PyronnError(name, status, detail)


def workspace_size(name: str, *args: int) -> int:
    """Workspace bytes of an entry point (``pyronn_projection2d`` for both 2D
    forward ops); args as the C query takes them."""
    return int(getattr(load(), name + "_workspace_size")(*args))
