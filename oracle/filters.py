"""FP64 restatement of the FDK / FBP pre-processing -- TEST INFRASTRUCTURE.

The projector ops of PYRO-NN-Layers have no filtering step (the PYRO-NN
package around them filters in Python), so there is no reference code to
follow: this restates the published algorithms the library's
``pyronn_fdk_filter`` implements.

* Cosine pre-weighting of a flat-detector cone-beam (or fan-beam) projection
  (L. A. Feldkamp, L. C. Davis, J. W. Kress, "Practical cone-beam algorithm",
  JOSA A 1(6), 1984): g(u, v) = p(u, v) * SDD / sqrt(SDD^2 + u^2 + v^2), with
  (u, v) the pixel's detector coordinates in mm relative to the principal
  point.  SDD = 0 means no weighting (parallel beam).
* Discrete ramp filtering of every detector row with the spatial kernels of
  A. C. Kak, M. Slaney, "Principles of Computerized Tomographic Imaging"
  (IEEE Press 1988), ch. 3: sample spacing tau = the detector column pitch,
  Ram-Lak h[0] = 1 / (4 tau^2), h[n odd] = -1 / (pi^2 n^2 tau^2), h[n even] = 0;
  Shepp-Logan h[n] = -2 / (pi^2 tau^2 (4 n^2 - 1)); the row is convolved
  linearly (zero outside the detector): q[j] = tau * sum_k h[j - k] g[k].

Parity is pinned by the analytic reconstruction tests (an FDK of projected
ellipsoids reproduces their densities); no golden vectors exist.
"""
from __future__ import annotations

import math

import numpy as np

RAM_LAK = 0
SHEPP_LOGAN = 1


def ramp_kernel(width: int, tau: float, kind: int = RAM_LAK) -> np.ndarray:
    """tau * h[m] for m = -(width-1) .. width-1 (FP64)."""
    m = np.arange(-(width - 1), width, dtype=np.float64)
    if kind == RAM_LAK:
        h = np.zeros_like(m)
        odd = (np.abs(m) % 2) == 1
        h[odd] = -1.0 / (math.pi ** 2 * m[odd] ** 2 * tau ** 2)
        h[m == 0] = 1.0 / (4.0 * tau ** 2)
    elif kind == SHEPP_LOGAN:
        h = -2.0 / (math.pi ** 2 * tau ** 2 * (4.0 * m ** 2 - 1.0))
    else:
        raise ValueError("unknown filter kind %r" % kind)
    return tau * h


def cosine_weights(det_h: int, det_w: int, sdd: float, det_spacing_v: float, det_spacing_u: float,
                   principal_v: float, principal_u: float) -> np.ndarray:
    """[det_h, det_w] SDD / sqrt(SDD^2 + u^2 + v^2); ones when sdd == 0."""
    if sdd == 0.0:
        return np.ones((det_h, det_w))
    v = (np.arange(det_h, dtype=np.float64) - principal_v) * det_spacing_v
    u = (np.arange(det_w, dtype=np.float64) - principal_u) * det_spacing_u
    return sdd / np.sqrt(sdd ** 2 + u[None, :] ** 2 + v[:, None] ** 2)


def fdk_filter(projections, sdd: float, det_spacing_v: float, det_spacing_u: float, principal_v: float,
               principal_u: float, kind: int = RAM_LAK, weight_output: bool = False) -> np.ndarray:
    """[..., det_h, det_w] -> filtered rows (FP64).  weight_output applies the
    cosine weights after the filter instead of before (the adjoint)."""
    p = np.asarray(projections, dtype=np.float64)
    det_h, det_w = p.shape[-2:]
    c = cosine_weights(det_h, det_w, sdd, det_spacing_v, det_spacing_u, principal_v, principal_u)
    h = ramp_kernel(det_w, det_spacing_u, kind)
    g = p if weight_output else p * c
    rows = g.reshape(-1, det_w)
    out = np.empty_like(rows)
    for r in range(rows.shape[0]):
        out[r] = np.convolve(rows[r], h)[det_w - 1:2 * det_w - 1]
    out = out.reshape(p.shape)
    return out * c if weight_output else out
