"""The TensorFlow custom-op shim (tf_shim/pyronn_tf_ops.cc) compiles against
the C ABI header.

TensorFlow is not installed here, so the shim is compiled with
``g++ -fsyntax-only`` against tests/tf_stub/: declarations of the TensorFlow
names the shim uses, with TensorFlow 2.x signatures.  This catches drift
between the shim and include/pyronn_b200.h (argument lists of the entry
points and workspace queries, enum names), which a build that only runs where
TensorFlow exists would not.  The shim reproduces the reference's six
REGISTER_OPs (cc/ops/*_OPKernel.cc); the second test checks their names,
inputs and attrs textually against the reference's registrations.
"""
import os
import re
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(ROOT, "pyro-nn-layers_b200", "tf_shim", "pyronn_tf_ops.cc")
STUB = os.path.join(ROOT, "tests", "tf_stub")
CUDA_INC = "/usr/local/cuda/include"

# the reference's registrations (op name -> inputs in order, attrs), from
# cc/ops/par_projector_2D_OPKernel.cc:30-37, par_backprojector_2D_OPKernel.cc:26-33,
# fan_projector_2D_OPKernel.cc:26-35, fan_backprojector_2D_OPKernel.cc:26-35,
# cone_projector_3D_OPKernel.cc:34-42, cone_backprojector_3D_OPKernel.cc:27-35
REFERENCE_OPS = {
    "ParallelProjection2D": (["volume", "projection_shape", "volume_origin", "detector_origin", "volume_spacing",
                              "detector_spacing", "ray_vectors"], []),
    "ParallelBackprojection2D": (["sinogram", "volume_shape", "volume_origin", "detector_origin", "volume_spacing",
                                  "detector_spacing", "ray_vectors"], []),
    "FanProjection2D": (["volume", "projection_shape", "volume_origin", "detector_origin", "volume_spacing",
                         "detector_spacing", "source_2_isocenter_distance", "source_2_detector_distance",
                         "central_ray_vectors"], []),
    "FanBackprojection2D": (["sinogram", "volume_shape", "volume_origin", "detector_origin", "volume_spacing",
                             "detector_spacing", "source_2_isocenter_distance", "source_2_detector_distance",
                             "central_ray_vectors"], []),
    "ConeProjection3D": (["volume", "projection_shape", "volume_origin", "volume_spacing", "projection_matrices",
                          "step_size", "projection_multiplier"], ["hardware_interp"]),
    "ConeBackprojection3D": (["sinogram", "volume_shape", "volume_origin", "volume_spacing",
                              "projection_matrices", "step_size", "projection_multiplier"], ["hardware_interp"]),
}


def test_shim_compiles_against_the_c_abi():
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("g++ or the CUDA headers are not available")
    cmd = [gxx, "-std=c++17", "-fsyntax-only", "-Wall", "-Werror", "-DGOOGLE_CUDA=1", "-I", STUB, "-I",
           os.path.join(ROOT, "include"), "-I", CUDA_INC, SHIM]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


def test_shim_registers_the_reference_ops():
    src = open(SHIM).read()
    regs = re.findall(r'REGISTER_OP\("(\w+)"\)(.*?);', src, re.S)
    assert {name for name, _ in regs} == set(REFERENCE_OPS)
    for name, body in regs:
        inputs = [m.strip() for m in re.findall(r'\.Input\("\s*(\w+)\s*:', body)]
        attrs = [m.strip() for m in re.findall(r'\.Attr\("\s*(\w+)\s*:', body)]
        assert (inputs, attrs) == REFERENCE_OPS[name], name
        assert re.search(r"\.Attr\(\"hardware_interp : bool = false\"\)", body) or not attrs
    # every op has a GPU kernel whose shape input lives in host memory
    for name in REFERENCE_OPS:
        assert re.search(r'REGISTER_KERNEL_BUILDER\(Name\("%s"\)\.Device\(DEVICE_GPU\)\.HostMemory' % name, src)
