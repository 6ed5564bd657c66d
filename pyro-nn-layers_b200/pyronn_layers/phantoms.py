"""Seeded ellipse / ellipsoid phantoms with closed-form line integrals.

Every phantom is a sum of constant-density ellipses (2D) or ellipsoids (3D),
drawn from ``numpy.random.Generator(PCG64(seed))``.  The parameter lists are
returned with the rasterised grid so tests can compare projections with the
exact (continuous) line integrals.
"""
from __future__ import annotations

import numpy as np


def _rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def random_ellipses(seed, field_mm, n=10, axes_mm=(10.0, 100.0), density=(0.1, 1.0), inner=0.8):
    """n ellipses: centre uniform in the inner fraction of the field, semi-axes
    uniform in axes_mm, rotation uniform [0, pi), density uniform.
    Returns an array [n, 6] of (cx, cy, a, b, phi, rho), mm and radians."""
    r = _rng(seed)
    fx, fy = float(field_mm[0]), float(field_mm[1])
    cx = r.uniform(-inner * fx / 2, inner * fx / 2, n)
    cy = r.uniform(-inner * fy / 2, inner * fy / 2, n)
    a = r.uniform(axes_mm[0], axes_mm[1], n)
    b = r.uniform(axes_mm[0], axes_mm[1], n)
    phi = r.uniform(0.0, np.pi, n)
    rho = r.uniform(density[0], density[1], n)
    return np.stack([cx, cy, a, b, phi, rho], axis=1)


def rasterise_ellipses(ellipses, shape, spacing, origin):
    """Sums the ellipses at pixel centres. shape/spacing/origin in (y, x) order."""
    Y, X = int(shape[0]), int(shape[1])
    ys = origin[0] + np.arange(Y) * spacing[0]
    xs = origin[1] + np.arange(X) * spacing[1]
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    img = np.zeros((Y, X), dtype=np.float64)
    for cx, cy, a, b, phi, rho in ellipses:
        c, s = np.cos(phi), np.sin(phi)
        dx, dy = xx - cx, yy - cy
        u = c * dx + s * dy
        v = -s * dx + c * dy
        img += rho * ((u / a) ** 2 + (v / b) ** 2 <= 1.0)
    return img.astype(np.float32)


def ellipse_phantom_2d(shape, spacing, seed, n=10):
    """Rasterised sum of n random ellipses (10-100 mm semi-axes) and their parameters."""
    from .geometry import centered_origin
    spacing = np.asarray(spacing, dtype=np.float64)
    origin = centered_origin(shape, spacing).astype(np.float64)
    field = (shape[1] * spacing[1], shape[0] * spacing[0])
    ell = random_ellipses(seed, field, n)
    return rasterise_ellipses(ell, shape, spacing, origin), ell


def ellipse_line_integral(ellipses, p0, d):
    """Exact integral along the line p0 + t d (|d| = 1) of the ellipse sum."""
    total = 0.0
    for cx, cy, a, b, phi, rho in ellipses:
        c, s = np.cos(phi), np.sin(phi)
        px, py = p0[0] - cx, p0[1] - cy
        pu, pv = c * px + s * py, -s * px + c * py
        du, dv = c * d[0] + s * d[1], -s * d[0] + c * d[1]
        A = (du / a) ** 2 + (dv / b) ** 2
        B = 2 * (pu * du / a ** 2 + pv * dv / b ** 2)
        C = (pu / a) ** 2 + (pv / b) ** 2 - 1.0
        disc = B * B - 4 * A * C
        if disc > 0:
            total += rho * np.sqrt(disc) / A
    return total


def _rotation(r):
    # random rotation from a uniform unit quaternion
    q = r.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def random_ellipsoids(seed, field_mm, n=32, axes_mm=(5.0, 60.0), density=(0.1, 1.0), inner=0.8):
    """n ellipsoids: list of (centre[3] (x,y,z) mm, semi-axes[3] mm, R[3,3], rho)."""
    r = _rng(seed)
    out = []
    for _ in range(n):
        c = np.array([r.uniform(-inner * f / 2, inner * f / 2) for f in field_mm])
        ax = r.uniform(axes_mm[0], axes_mm[1], 3)
        R = _rotation(r)
        rho = r.uniform(density[0], density[1])
        out.append((c, ax, R, rho))
    return out


def rasterise_ellipsoids(ellipsoids, shape, spacing, origin):
    """Sums ellipsoids at voxel centres; shape/spacing/origin in (z, y, x) order."""
    Z, Y, X = (int(v) for v in shape)
    zs = origin[0] + np.arange(Z) * spacing[0]
    ys = origin[1] + np.arange(Y) * spacing[1]
    xs = origin[2] + np.arange(X) * spacing[2]
    vol = np.zeros((Z, Y, X), dtype=np.float32)
    for c, ax, R, rho in ellipsoids:
        # bounding box of the ellipsoid to limit work
        ext = np.sqrt((R ** 2) @ (ax ** 2))
        lo = c - ext
        hi = c + ext
        zi = np.nonzero((zs >= lo[2]) & (zs <= hi[2]))[0]
        yi = np.nonzero((ys >= lo[1]) & (ys <= hi[1]))[0]
        xi = np.nonzero((xs >= lo[0]) & (xs <= hi[0]))[0]
        if len(zi) == 0 or len(yi) == 0 or len(xi) == 0:
            continue
        zz, yy, xx = np.meshgrid(zs[zi], ys[yi], xs[xi], indexing="ij")
        d = np.stack([xx - c[0], yy - c[1], zz - c[2]], axis=-1)
        loc = d @ R  # coordinates in the ellipsoid frame (R columns are its axes)
        inside = ((loc / ax) ** 2).sum(axis=-1) <= 1.0
        sub = vol[zi[0]:zi[-1] + 1, yi[0]:yi[-1] + 1, xi[0]:xi[-1] + 1]
        sub += (rho * inside).astype(np.float32)
    return vol


def ellipsoid_phantom_3d(shape, spacing, seed, n=32):
    """Rasterised sum of n random ellipsoids (5-60 mm semi-axes) and their parameters."""
    from .geometry import centered_origin
    spacing = np.asarray(spacing, dtype=np.float64)
    origin = centered_origin(shape, spacing).astype(np.float64)
    field = (shape[2] * spacing[2], shape[1] * spacing[1], shape[0] * spacing[0])
    ell = random_ellipsoids(seed, field, n)
    return rasterise_ellipsoids(ell, shape, spacing, origin), ell


def ellipsoid_line_integral(ellipsoids, p0, d):
    """Exact integral along p0 + t d (|d| = 1, (x,y,z) mm) of the ellipsoid sum."""
    total = 0.0
    for c, ax, R, rho in ellipsoids:
        p = (np.asarray(p0) - c) @ R / ax
        q = (np.asarray(d) @ R) / ax
        A = q @ q
        B = 2 * p @ q
        C = p @ p - 1.0
        disc = B * B - 4 * A * C
        if disc > 0:
            total += rho * np.sqrt(disc) / A
    return total


def rasterise_ellipsoids_torch(ellipsoids, shape, spacing, origin, device, dtype=None):
    """rasterise_ellipsoids on a torch device (for large grids); float32 result."""
    import torch
    Z, Y, X = (int(v) for v in shape)
    zs = origin[0] + torch.arange(Z, device=device, dtype=torch.float64) * spacing[0]
    ys = origin[1] + torch.arange(Y, device=device, dtype=torch.float64) * spacing[1]
    xs = origin[2] + torch.arange(X, device=device, dtype=torch.float64) * spacing[2]
    vol = torch.zeros((Z, Y, X), device=device, dtype=torch.float32)
    for c, ax, R, rho in ellipsoids:
        ext = np.sqrt((R ** 2) @ (ax ** 2))
        lo, hi = c - ext, c + ext
        zi = torch.nonzero((zs >= lo[2]) & (zs <= hi[2])).flatten()
        yi = torch.nonzero((ys >= lo[1]) & (ys <= hi[1])).flatten()
        xi = torch.nonzero((xs >= lo[0]) & (xs <= hi[0])).flatten()
        if zi.numel() == 0 or yi.numel() == 0 or xi.numel() == 0:
            continue
        z0, z1 = int(zi[0]), int(zi[-1]) + 1
        y0, y1 = int(yi[0]), int(yi[-1]) + 1
        x0, x1 = int(xi[0]), int(xi[-1]) + 1
        zz, yy, xx = torch.meshgrid(zs[z0:z1], ys[y0:y1], xs[x0:x1], indexing="ij")
        d = torch.stack([xx - c[0], yy - c[1], zz - c[2]], dim=-1)
        loc = d @ torch.as_tensor(R, device=device, dtype=torch.float64)
        inside = ((loc / torch.as_tensor(ax, device=device, dtype=torch.float64)) ** 2).sum(-1) <= 1.0
        vol[z0:z1, y0:y1, x0:x1] += float(rho) * inside.to(torch.float32)
    return vol if dtype is None else vol.to(dtype)
