"""The serving wire format on CPU: geometry descriptors rebuild the same
geometry tensors, requests and results survive the byte framing, and
malformed messages are refused."""
import math

import numpy as np
import pytest

from pyronn_layers import geometry, wire


def test_cone_descriptor_round_trip_keeps_matrices():
    geo = geometry.ConeBeam3D((8, 10, 12), (1.0, 0.9, 1.1), (6, 7), (1.2, 1.3), 5, 300.0, 500.0,
                              step_size=0.4, projection_multiplier=0.7)
    d = wire.geometry_descriptor("cone", geo)
    kind, g2 = wire.geometry_from_descriptor(d)
    assert kind == "cone"
    for a, b in zip(geo.args(), g2.args()):
        np.testing.assert_array_equal(np.asarray(a), np.asarray(b))


def test_circular_descriptor_builds_the_trajectory():
    d = wire.circular_descriptor("cone", (8, 8, 8), (1, 1, 1), (6, 7), (1.5, 1.5), 9, 400.0, 700.0,
                                 angular_range=math.pi)
    _, g = wire.geometry_from_descriptor(d)
    ref = geometry.circular_projection_matrices(9, 400.0, 700.0, (6, 7), (1.5, 1.5), math.pi)
    np.testing.assert_array_equal(g.projection_matrices, ref)
    d2 = wire.circular_descriptor("fan", (16, 16), (0.5, 0.5), 33, 0.5, 12, 300.0, 500.0)
    kind, g2 = wire.geometry_from_descriptor(d2)
    assert kind == "fan" and g2.detector_shape == (12, 33)


@pytest.mark.parametrize("dtype", ["fp32", "fp16", "bf16"])
def test_request_and_result_framing(dtype):
    rng = np.random.Generator(np.random.PCG64(3))
    if dtype == "bf16":
        data = rng.integers(0, 2 ** 16, (3, 4, 5)).astype(np.uint16)
    else:
        data = rng.uniform(0, 1, (3, 4, 5)).astype(np.float32 if dtype == "fp32" else np.float16)
    msg = wire.encode_request(17, "cone_fwd", "scanner-a", dtype, data)
    r = wire.decode_request(msg)
    assert (r["id"], r["op"], r["geometry"], r["dtype"]) == (17, "cone_fwd", "scanner-a", dtype)
    np.testing.assert_array_equal(r["data"].view(data.dtype), data)
    res = wire.decode_result(wire.encode_result(17, dtype, data))
    assert res["id"] == 17
    np.testing.assert_array_equal(res["data"].view(data.dtype), data)


def test_malformed_messages_are_refused():
    msg = wire.encode_request(1, "fan_bp", "g", "fp32", np.zeros((2, 3), np.float32))
    with pytest.raises(ValueError):
        wire.decode_request(msg[:-4])            # truncated payload
    with pytest.raises(ValueError):
        wire.decode_request(msg[:3])             # truncated length
    with pytest.raises(ValueError):
        wire.decode_result(msg)                  # a request is not a result
    with pytest.raises(ValueError):
        wire.encode_request(1, "mri", "g", "fp32", np.zeros(2, np.float32))
    with pytest.raises(ValueError):
        wire.geometry_from_descriptor({"kind": "cone", "n_proj": 0, "sid": 1.0, "sdd": 2.0})
