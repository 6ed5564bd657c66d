"""The continuous-batching server: results are the same alone and in the mix,
batches form, CUDA graphs are replayed, latencies are reported."""
import numpy as np
import pytest
import torch

import pyronn_layers as pl
from pyronn_layers import geometry, serving

pytestmark = pytest.mark.gpu


def small_geometries():
    fan = geometry.FanBeam2D((64, 64), (0.5, 0.5), 128, 0.5, 60, 75.0, 120.0)
    c1 = geometry.ConeBeam3D((24, 24, 24), (1.0, 1.0, 1.0), (32, 40), (1.5, 1.5), 20, 120.0, 200.0)
    c2 = geometry.ConeBeam3D((32, 32, 32), (0.5, 0.5, 0.5), (40, 48), (1.0, 1.0), 24, 150.0, 240.0)
    return {
        "fan": serving.GeometryEntry("fan", fan, fan.volume_shape, fan.detector_shape),
        "c1": serving.GeometryEntry("cone", c1, c1.volume_shape, c1.detector_shape),
        "c2": serving.GeometryEntry("cone", c2, c2.volume_shape, c2.detector_shape),
    }


def alone(job, geos, dev):
    g = geos[job.cls.geometry].geo
    x = job.data.to(dev)[None]
    if job.cls.op == "fan_fwd":
        return pl.fan_projection2d(x, g.detector_shape, *g.args())[0]
    if job.cls.op == "fan_bp":
        return pl.fan_backprojection2d(x, g.volume_shape, *g.args(), out_dtype=torch.float32)[0]
    if job.cls.op == "cone_fwd":
        return pl.cone_projection3d(x, g.detector_shape, *g.args())[0]
    return pl.cone_backprojection3d(x, g.volume_shape, *g.args(), out_dtype=torch.float32)[0]


def test_results_alone_equal_results_in_the_mix(cuda):
    geos = small_geometries()
    trace = serving.poisson_trace(60, rate_hz=2000.0, seed=3, mix={"fan": 0.5, "c1": 0.3, "c2": 0.2})
    jobs = serving.make_jobs(trace, geos, seed=1)
    server = serving.ProjectorServer(geos, device=cuda, max_inflight=6, max_batch=4, n_streams=3)
    stats = server.run_trace(jobs, realtime=False)
    assert np.isfinite(stats.p50_ms) and stats.p99_ms >= stats.p50_ms
    assert stats.mean_batch > 1.0  # jobs were batched
    assert stats.gups > 0
    for j in jobs:
        ref = alone(j, geos, cuda)
        assert j.result is not None and j.result.shape == ref.shape
        # same kernels, same per-element arithmetic: bitwise equal
        assert torch.equal(j.result, ref), (j.id, j.cls)


def test_graphs_are_replayed_and_memory_is_admitted(cuda):
    geos = small_geometries()
    trace = serving.poisson_trace(80, rate_hz=5000.0, seed=4, mix={"c1": 1.0})
    jobs = serving.make_jobs(trace, geos, seed=2)
    server = serving.ProjectorServer(geos, device=cuda, max_inflight=4, max_batch=2, n_streams=2)
    stats = server.run_trace(jobs, realtime=False)
    assert stats.graph_replays > 0
    assert all(j.done >= j.admit >= 0 for j in jobs)
    # a reserve larger than the device refuses every job
    tight = serving.ProjectorServer(geos, device=cuda, hbm_reserve=1 << 50)
    with pytest.raises(MemoryError):
        tight.run_trace(serving.make_jobs(trace[:2], geos, seed=2), realtime=False)


def test_wire_requests_through_the_server(cuda):
    """Geometries registered from wire descriptors and jobs decoded from wire
    requests give, as wire results, the same arrays as the ops called directly."""
    from pyronn_layers import wire
    server = serving.ProjectorServer({}, device=cuda, max_batch=2)
    server.register_geometry("cone-a", wire.circular_descriptor("cone", (24, 24, 24), (1.0, 1.0, 1.0), (32, 40),
                                                                (1.5, 1.5), 20, 120.0, 200.0))
    fan = geometry.FanBeam2D((64, 64), (0.5, 0.5), 128, 0.5, 60, 75.0, 120.0)
    server.register_geometry("fan-b", wire.geometry_descriptor("fan", fan))
    with pytest.raises(ValueError):
        server.register_geometry("fan-b", wire.geometry_descriptor("fan", fan))
    rng = np.random.Generator(np.random.PCG64(9))
    reqs = []
    for i, (op, name, dtype) in enumerate([("cone_fwd", "cone-a", "fp32"), ("cone_bp", "cone-a", "fp16"),
                                            ("fan_fwd", "fan-b", "bf16"), ("fan_bp", "fan-b", "fp32"),
                                            ("cone_fwd", "cone-a", "fp32")]):
        e = server.geometries[name]
        shape = e.volume_shape if op.endswith("fwd") else e.sinogram_shape
        x = torch.as_tensor(rng.uniform(0, 1, shape), dtype={"fp32": torch.float32, "fp16": torch.float16,
                                                              "bf16": torch.bfloat16}[dtype])
        payload = x.view(torch.int16).numpy().view(np.uint16) if dtype == "bf16" else x.numpy()
        reqs.append((wire.encode_request(i, op, name, dtype, payload), x))
    jobs = [serving.job_from_request(wire.decode_request(m), server.geometries) for m, _ in reqs]
    server.run_trace(jobs, realtime=False)
    for j, (_, x) in zip(jobs, reqs):
        res = wire.decode_result(serving.result_message(j))
        assert res["id"] == j.id
        j.data = x
        ref = alone(j, server.geometries, cuda).cpu()
        got = torch.from_numpy(np.array(res["data"]))
        if res["dtype"] == "bf16":
            got = got.view(torch.int16).view(torch.bfloat16)
        assert torch.equal(got, ref), (j.id, j.cls)
    with pytest.raises(ValueError):  # wrong input shape for the geometry
        serving.job_from_request(wire.decode_request(wire.encode_request(
            9, "cone_fwd", "cone-a", "fp32", np.zeros((3, 3, 3), np.float32))), server.geometries)
