"""C ABI surface checks that need no GPU: the library loads, exports every
symbol include/pyronn_b200.h declares, and rejects bad arguments with a
status code (no CUDA call happens before these checks)."""
import ctypes
import os
import re

import pytest

from pyronn_layers import _capi
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pyronn_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"PYRONN_API\s+[\w\s\*]+?\b(pyronn_\w+)\s*\(", text)))


def test_header_declares_the_six_ops():
    syms = declared_symbols()
    for op in ("parallel_projection2d", "parallel_backprojection2d", "fan_projection2d", "fan_backprojection2d",
               "cone_projection3d", "cone_backprojection3d"):
        assert "pyronn_" + op in syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_capi.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name
    assert set(declared_symbols()) == set(_capi.PROTOTYPES)


def test_abi_version_and_status_strings():
    lib = _capi.load()
    assert lib.pyronn_abi_version() == _capi.ABI_VERSION
    assert lib.pyronn_status_string(0) == b"success"
    assert lib.pyronn_status_string(_capi.ERROR_WORKSPACE_TOO_SMALL) == b"workspace too small"
    assert lib.pyronn_status_string(99) == b"unknown status"


def test_workspace_sizes():
    lib = _capi.load()
    # batch, vol z/y/x, views, det h/w, in_dtype, hardware_interp, geom_batch
    fp = lib.pyronn_cone_projection3d_workspace_size(2, 64, 64, 64, 360, 100, 120, 0, 0, 2)
    fp_hw = lib.pyronn_cone_projection3d_workspace_size(2, 64, 64, 64, 360, 100, 120, 0, 1, 2)
    fp16 = lib.pyronn_cone_projection3d_workspace_size(2, 64, 64, 64, 360, 100, 120, 1, 0, 2)
    bp = lib.pyronn_cone_backprojection3d_workspace_size(2, 360, 100, 120, 64, 64, 64, 0, 0, 2)
    assert fp_hw >= 256 + 2 * 360 * 96 and fp_hw % 256 == 0
    # zero-padded copies of one volume for the software forward path: x- and
    # y-fastest (67^3 each) and the z-fastest cell copy (66^3 cells of 8 taps)
    def align(n):
        return (n + 255) // 256 * 256
    assert fp - fp_hw == 2 * align(67 ** 3 * 4) + align(66 ** 3 * 32)
    assert fp16 - fp_hw == 2 * align(67 ** 3 * 2) + align(66 ** 3 * 16)
    assert bp >= 256 + 2 * 360 * 48 and bp % 256 == 0
    assert lib.pyronn_cone_projection3d_workspace_size(0, 8, 8, 8, 10, 4, 4, 0, 0, 1) == 0
    assert lib.pyronn_cone_projection3d_workspace_size(1, 8, 8, 8, 10, 4, 4, 9, 0, 1) == 0


def _cell_pitch(vol_x, vol_y, vol_z):
    """x pitch of the forward's cell copy: the least s_x >= (Y+2)(Z+2) for
    which the sampler's floor-biased cell index (bias 0x4B400000 per unit of
    the x and y strides plus the z floor's bias, 0x4B400000 or, for z in
    half-voxel units, 0x4BC00000; mod 2^32) plus any index of the copy stays
    in [0, 2^32)."""
    xc, yc, zc = vol_x + 2, vol_y + 2, vol_z + 2
    sx = yc * zc
    while True:
        biases = [(0x4B400000 * (sx + zc) + zb) % 2 ** 32 for zb in (0x4B400000, 0x4BC00000)]
        if all(b >= sx + zc + 1 and b + xc * sx <= 2 ** 32 for b in biases):
            return sx
        sx += 1


def test_cell_copy_pitch():
    """The forward's workspace holds the cell copy at the pitch its index
    arithmetic needs: (Y+2)(Z+2) cells for most shapes, one more where the
    biased index would otherwise wrap (vol 91 x 8 x 196, z y x)."""
    lib = _capi.load()

    def align(n):
        return (n + 255) // 256 * 256
    for z, y, x in [(64, 64, 64), (91, 8, 196), (512, 512, 512), (85, 150, 38)]:
        sx = _cell_pitch(x, y, z)
        fp16 = lib.pyronn_cone_projection3d_workspace_size(1, z, y, x, 16, 40, 60, 1, 0, 1)
        fp_hw = lib.pyronn_cone_projection3d_workspace_size(1, z, y, x, 16, 40, 60, 1, 1, 1)
        padded = (x + 3) * (y + 3) * (z + 3)
        assert fp16 - fp_hw == 2 * align(padded * 2) + align((x + 2) * sx * 16)
    assert _cell_pitch(196, 8, 91) == 10 * 93 + 1
    assert _cell_pitch(64, 64, 64) == 66 * 66
    # padded copies past 2^31 elements: the direct path, which needs no copies
    big = [lib.pyronn_cone_projection3d_workspace_size(1, 1300, 1300, 1300, 16, 40, 60, 1, hw, 1) for hw in (0, 1)]
    assert big[0] == big[1] > 0


FAKE = 4096  # non-null, never dereferenced: validation fails first


@pytest.mark.parametrize("in_dt,out_dt,batch,g,msg", [
    (7, 0, 1, 1, b"in_dtype"),
    (0, -1, 1, 1, b"out_dtype"),
    (0, 0, 0, 1, b"batch"),
    (0, 0, 2, 3, b"geom_batch"),
])
def test_2d_rejects_bad_arguments(in_dt, out_dt, batch, g, msg):
    lib = _capi.load()
    st = lib.pyronn_fan_backprojection2d(FAKE, FAKE, in_dt, out_dt, batch, 3, 5, 4, 4, FAKE, FAKE, FAKE, FAKE, FAKE,
                                         FAKE, FAKE, g, None)
    assert st == _capi.ERROR_INVALID_ARGUMENT
    assert msg in lib.pyronn_last_error()


def test_null_pointers_and_dims():
    lib = _capi.load()
    st = lib.pyronn_parallel_projection2d(None, FAKE, 0, 0, 1, 4, 4, 3, 5, FAKE, FAKE, FAKE, FAKE, FAKE, 1, None, 0,
                                          None)
    assert st == _capi.ERROR_INVALID_ARGUMENT and b"null data" in lib.pyronn_last_error()
    st = lib.pyronn_parallel_projection2d(FAKE, FAKE, 0, 0, 1, 4, 4, 3, 5, FAKE, None, FAKE, FAKE, FAKE, 1, None, 0,
                                          None)
    assert st == _capi.ERROR_INVALID_ARGUMENT and b"null geometry" in lib.pyronn_last_error()
    st = lib.pyronn_parallel_projection2d(FAKE, FAKE, 0, 0, 1, 4, 0, 3, 5, FAKE, FAKE, FAKE, FAKE, FAKE, 1, None, 0,
                                          None)
    assert st == _capi.ERROR_INVALID_ARGUMENT and b"positive" in lib.pyronn_last_error()


def test_2d_forward_workspace_size_and_checks():
    lib = _capi.load()
    # two cell copies of the batch (4 FP32 taps per cell whatever the storage
    # type, border of two cells below and one above), each rounded up to 256 bytes
    assert _capi.workspace_size("pyronn_projection2d", 3, 5, 7, 0) == 2 * 3840
    assert _capi.workspace_size("pyronn_projection2d", 2, 100, 100, 1) == 2 * 339712
    assert _capi.workspace_size("pyronn_projection2d", 0, 5, 7, 0) == 0
    assert _capi.workspace_size("pyronn_projection2d", 1, 5, 7, 9) == 0
    st = lib.pyronn_fan_projection2d(FAKE, FAKE, 0, 0, 2, 10, 10, 3, 5, FAKE, FAKE, FAKE, FAKE, FAKE, FAKE, FAKE, 1,
                                     FAKE, 2 * 5632 - 1, None)
    assert st == _capi.ERROR_WORKSPACE_TOO_SMALL and b"11264" in lib.pyronn_last_error()
    st = lib.pyronn_parallel_projection2d(FAKE, FAKE, 0, 0, 1, 4, 4, 3, 5, FAKE, FAKE, FAKE, FAKE, FAKE, 1, FAKE + 4,
                                          1 << 20, None)
    assert st == _capi.ERROR_INVALID_ARGUMENT and b"aligned" in lib.pyronn_last_error()


def test_cone_rejects_small_workspace_and_huge_sizes():
    lib = _capi.load()
    st = lib.pyronn_cone_backprojection3d(FAKE, FAKE, 0, 0, 0, 1, 8, 8, 8, 4, 4, 4, FAKE, FAKE, FAKE, FAKE, FAKE, 1,
                                          FAKE, 16, None)
    assert st == _capi.ERROR_WORKSPACE_TOO_SMALL
    st = lib.pyronn_cone_projection3d(FAKE, FAKE, 0, 0, 0, 1, 2048, 2048, 2048, 4, 4, 4, FAKE, FAKE, FAKE, FAKE,
                                      FAKE, 1, FAKE, 1 << 20, None)
    assert st == _capi.ERROR_UNSUPPORTED and b"2^31" in lib.pyronn_last_error()


def test_ops_refuse_cpu_tensors():
    torch = pytest.importorskip("torch")
    import pyronn_layers as pl
    from pyronn_layers import geometry
    geo = geometry.ConeBeam3D((8, 8, 8), (1, 1, 1), (8, 8), (1, 1), 4, 100, 150)
    with pytest.raises(ValueError, match="CUDA"):
        pl.cone_projection3d(torch.zeros(1, 8, 8, 8), geo.detector_shape, *geo.args())


def test_trajectory_builders_reject_bad_arguments():
    lib = _capi.load()
    f = lib.pyronn_circular_projection_matrices
    assert f(None, 4, 600.0, 1000.0, 1.0, 1.0, 1.0, 1.0, 6.28, 0.0, None) == _capi.ERROR_INVALID_ARGUMENT
    assert f(FAKE, 0, 600.0, 1000.0, 1.0, 1.0, 1.0, 1.0, 6.28, 0.0, None) == _capi.ERROR_INVALID_ARGUMENT
    assert f(FAKE, 4, -600.0, 1000.0, 1.0, 1.0, 1.0, 1.0, 6.28, 0.0, None) == _capi.ERROR_INVALID_ARGUMENT
    assert b"positive" in lib.pyronn_last_error()
    assert f(FAKE, 4, 600.0, 1000.0, 1.0, 1.0, float("nan"), 1.0, 6.28, 0.0, None) == _capi.ERROR_INVALID_ARGUMENT
    g = lib.pyronn_circular_ray_vectors_2d
    assert g(FAKE, -1, 3.14, 0.0, None) == _capi.ERROR_INVALID_ARGUMENT
    assert g(FAKE, 4, float("inf"), 0.0, None) == _capi.ERROR_INVALID_ARGUMENT


def test_host_geometry_cache_is_keyed_by_content():
    """Host geometry passed to the ops is copied to the device once per
    content (a copy from pageable memory would wait for the stream's queued
    work on every call); a changed array is a new entry, the cache is bounded."""
    np = pytest.importorskip("numpy")
    pytest.importorskip("torch")
    from pyronn_layers import ops
    a = np.arange(12, dtype=np.float32)
    d1 = ops._host_geometry_on_device(a, "cpu")
    assert ops._host_geometry_on_device(a.copy(), "cpu") is d1
    a[0] = 5.0
    d3 = ops._host_geometry_on_device(a, "cpu")
    assert d3 is not d1 and float(d3[0]) == 5.0 and float(d1[0]) == 0.0
    for k in range(ops._HOST_GEOM_CACHE_SIZE + 8):
        ops._host_geometry_on_device(np.full(3, float(k), np.float32), "cpu")
    assert len(ops._HOST_GEOM_CACHE) <= ops._HOST_GEOM_CACHE_SIZE
