"""Wire format of the serving loop: geometry and request descriptors a client
sends, and the framing of requests and results as bytes.

* A geometry descriptor is a JSON object that rebuilds a serving geometry
  entry: for a circular scan its parameters (the server builds the matrices
  or ray vectors itself), for any other cone trajectory the projection
  matrices themselves.  ``ProjectorServer.register_geometry`` adds it to the
  server's geometry table under a name; requests refer to that name.
* A request is one job: op (``fan_fwd``, ``fan_bp``, ``cone_fwd``,
  ``cone_bp``), geometry name, storage dtype and the input array.  A result
  carries the job id and the output array.
* Framing of a request or result: a 4-byte little-endian header length, the
  UTF-8 JSON header, then the array's raw little-endian bytes (C order); the
  header gives the array's shape and dtype and the payload's byte count, so a
  reader can check it got the whole message.

No reference counterpart: PYRO-NN-Layers has no serving layer.
"""
from __future__ import annotations

import json
import math
import struct
from typing import Tuple

import numpy as np

from . import geometry as _geometry

OPS = ("fan_fwd", "fan_bp", "cone_fwd", "cone_bp")
# array encodings on the wire; bf16 travels as its 16-bit pattern
_NP_NAMES = {"fp32": "<f4", "fp16": "<f2", "bf16": "<u2"}


# ------------------------------------------------------------- geometry


def geometry_descriptor(kind: str, geo) -> dict:
    """JSON-able descriptor of a geometry.FanBeam2D / ConeBeam3D.  Cone
    geometries carry their projection matrices (any trajectory)."""
    if kind == "fan":
        return {"kind": "fan", "volume_shape": list(geo.volume_shape),
                "volume_spacing": [float(v) for v in geo.volume_spacing],
                "detector_width": int(geo.detector_shape[1]), "detector_spacing": float(geo.detector_spacing[0]),
                "n_proj": int(geo.detector_shape[0]), "sid": float(geo.sid[0]), "sdd": float(geo.sdd[0]),
                "ray_vectors": np.asarray(geo.ray_vectors, np.float32).tolist()}
    if kind == "cone":
        return {"kind": "cone", "volume_shape": list(geo.volume_shape),
                "volume_spacing": [float(v) for v in geo.volume_spacing],
                "detector_shape": list(geo.detector_shape[1:]),
                "detector_spacing": [float(v) for v in geo.detector_spacing],
                "n_proj": int(geo.detector_shape[0]), "sid": float(geo.sid), "sdd": float(geo.sdd),
                "step_size": float(geo.step_size[0]), "projection_multiplier": float(geo.projection_multiplier[0]),
                "projection_matrices": np.asarray(geo.projection_matrices, np.float32).tolist()}
    raise ValueError("kind must be 'fan' or 'cone', got %r" % (kind,))


def circular_descriptor(kind: str, volume_shape, volume_spacing, detector, detector_spacing, n_proj: int,
                        sid: float, sdd: float, angular_range: float = 2.0 * math.pi, step_size: float = 0.5,
                        projection_multiplier: float = 1.0) -> dict:
    """Compact descriptor of a circular scan (no matrices: the server builds
    them).  detector: width (fan) or (H, W) (cone)."""
    d = {"kind": kind, "circular": True, "volume_shape": [int(v) for v in volume_shape],
         "volume_spacing": [float(v) for v in volume_spacing], "n_proj": int(n_proj), "sid": float(sid),
         "sdd": float(sdd), "angular_range": float(angular_range)}
    if kind == "fan":
        d.update(detector_width=int(detector), detector_spacing=float(detector_spacing))
    elif kind == "cone":
        d.update(detector_shape=[int(v) for v in detector], detector_spacing=[float(v) for v in detector_spacing],
                 step_size=float(step_size), projection_multiplier=float(projection_multiplier))
    else:
        raise ValueError("kind must be 'fan' or 'cone', got %r" % (kind,))
    return d


def geometry_from_descriptor(d: dict):
    """(kind, geometry object) from a descriptor (validated)."""
    kind = d.get("kind")
    n = int(d["n_proj"])
    if n <= 0 or d["sid"] <= 0 or d["sdd"] <= 0:
        raise ValueError("n_proj, sid and sdd must be positive")
    if kind == "fan":
        geo = _geometry.FanBeam2D(tuple(d["volume_shape"]), tuple(d["volume_spacing"]), int(d["detector_width"]),
                                  float(d["detector_spacing"]), n, float(d["sid"]), float(d["sdd"]),
                                  float(d.get("angular_range", 2.0 * math.pi)))
        if not d.get("circular"):
            rays = np.asarray(d["ray_vectors"], np.float32)
            if rays.shape != (n, 2):
                raise ValueError("ray_vectors must be [n_proj, 2]")
            geo.ray_vectors = rays
        return "fan", geo
    if kind == "cone":
        geo = _geometry.ConeBeam3D(tuple(d["volume_shape"]), tuple(d["volume_spacing"]), tuple(d["detector_shape"]),
                                   tuple(d["detector_spacing"]), n, float(d["sid"]), float(d["sdd"]),
                                   float(d.get("angular_range", 2.0 * math.pi)), float(d.get("step_size", 0.5)),
                                   float(d.get("projection_multiplier", 1.0)))
        if not d.get("circular"):
            pm = np.asarray(d["projection_matrices"], np.float32)
            if pm.shape != (n, 3, 4):
                raise ValueError("projection_matrices must be [n_proj, 3, 4]")
            geo.projection_matrices = pm
        return "cone", geo
    raise ValueError("kind must be 'fan' or 'cone', got %r" % (kind,))


# ------------------------------------------------------------- framing


def _pack(header: dict, payload: bytes) -> bytes:
    h = json.dumps(header, separators=(",", ":")).encode("utf-8")
    return struct.pack("<I", len(h)) + h + payload


def _unpack(msg: bytes) -> Tuple[dict, memoryview]:
    if len(msg) < 4:
        raise ValueError("truncated message")
    (n,) = struct.unpack_from("<I", msg, 0)
    if 4 + n > len(msg):
        raise ValueError("truncated header")
    header = json.loads(bytes(msg[4:4 + n]).decode("utf-8"))
    payload = memoryview(msg)[4 + n:]
    if len(payload) != header.get("nbytes", -1):
        raise ValueError("payload of %d bytes, header says %s" % (len(payload), header.get("nbytes")))
    return header, payload


def _array_bytes(a: np.ndarray, dtype: str) -> bytes:
    if dtype not in _NP_NAMES:
        raise ValueError("dtype must be one of %s" % sorted(_NP_NAMES))
    return np.ascontiguousarray(a, dtype=_NP_NAMES[dtype]).tobytes()


def encode_request(job_id: int, op: str, geometry: str, dtype: str, data: np.ndarray) -> bytes:
    """One job as bytes.  data: the op input without the batch dimension, in
    the storage dtype (bf16 as its uint16 bit pattern)."""
    if op not in OPS:
        raise ValueError("op must be one of %s" % (OPS,))
    payload = _array_bytes(data, dtype)
    return _pack({"type": "request", "id": int(job_id), "op": op, "geometry": geometry, "dtype": dtype,
                  "shape": [int(v) for v in data.shape], "nbytes": len(payload)}, payload)


def decode_request(msg: bytes) -> dict:
    """-> {"id", "op", "geometry", "dtype", "data" (numpy, storage dtype)}."""
    h, payload = _unpack(msg)
    if h.get("type") != "request" or h.get("op") not in OPS or h.get("dtype") not in _NP_NAMES:
        raise ValueError("not a valid request header")
    data = np.frombuffer(payload, dtype=_NP_NAMES[h["dtype"]]).reshape(h["shape"])
    return {"id": h["id"], "op": h["op"], "geometry": h["geometry"], "dtype": h["dtype"], "data": data}


def encode_result(job_id: int, dtype: str, data: np.ndarray) -> bytes:
    payload = _array_bytes(data, dtype)
    return _pack({"type": "result", "id": int(job_id), "dtype": dtype, "shape": [int(v) for v in data.shape],
                  "nbytes": len(payload)}, payload)


def decode_result(msg: bytes) -> dict:
    h, payload = _unpack(msg)
    if h.get("type") != "result" or h.get("dtype") not in _NP_NAMES:
        raise ValueError("not a valid result header")
    data = np.frombuffer(payload, dtype=_NP_NAMES[h["dtype"]]).reshape(h["shape"])
    return {"id": h["id"], "dtype": h["dtype"], "data": data}
