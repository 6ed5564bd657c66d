"""Host-side pieces of the serving loop (no GPU): the seeded trace, the job
classes and the percentile helper."""
import collections

import numpy as np

from pyronn_layers import serving


def test_trace_is_seeded_and_follows_the_mix():
    a = serving.poisson_trace(4000, rate_hz=100.0, seed=5)
    b = serving.poisson_trace(4000, rate_hz=100.0, seed=5)
    assert a == b
    times = np.array([t for t, _ in a])
    assert np.all(np.diff(times) > 0)
    # mean inter-arrival 1/rate
    assert abs(np.diff(times).mean() - 0.01) < 0.001
    geo = collections.Counter(c.geometry for _, c in a)
    assert abs(geo["fan512"] / 4000 - 0.6) < 0.03
    assert abs(geo["cone128"] / 4000 - 0.3) < 0.03
    assert abs(geo["cone256"] / 4000 - 0.1) < 0.02
    ops = collections.Counter(c.op.split("_")[1] for _, c in a)
    dts = collections.Counter(c.dtype for _, c in a)
    assert abs(ops["fwd"] / 4000 - 0.5) < 0.03 and abs(dts["bf16"] / 4000 - 0.5) < 0.03


def test_job_classes_group_compatible_jobs():
    c1 = serving.JobClass("cone_fwd", "cone128", "bf16")
    c2 = serving.JobClass("cone_fwd", "cone128", "bf16")
    c3 = serving.JobClass("cone_fwd", "cone128", "fp32")
    assert c1 == c2 and hash(c1) == hash(c2) and c1 != c3


def test_percentiles_and_updates():
    assert serving.percentile([1, 2, 3, 4], 50) == 2.5
    assert np.isnan(serving.percentile([], 99))
    g = serving.standard_geometries()
    assert g["fan512"].updates == 512 * 512 * 360
    assert g["cone128"].updates == 128 ** 3 * 180
    assert g["cone256"].updates == 256 ** 3 * 360
