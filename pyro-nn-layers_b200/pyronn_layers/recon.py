"""Differentiable reconstruction helpers built on the projector ops.

``UnrolledGradientDescent`` runs K steps of x <- x - lr_k * A^T (A x - y) for
a cone-beam geometry, each step differentiable (the ops' backward passes are
the paired projector / backprojector, or the exact transpose with
``matched_adjoint=True``).  With ``checkpoint=True`` every step is wrapped in
``torch.utils.checkpoint`` so only the step inputs are kept for the backward
pass and each step's projections are recomputed there -- the memory of K
unrolled steps stays that of one.
"""
from __future__ import annotations

import torch
import torch.utils.checkpoint as tcp

from . import ops


class UnrolledGradientDescent(torch.nn.Module):
    def __init__(self, geo, n_steps: int = 20, init_lr: float = 1e-4, matched_adjoint: bool = True,
                 checkpoint: bool = True):
        super().__init__()
        self.geo = geo
        self.n_steps = n_steps
        self.matched_adjoint = matched_adjoint
        self.checkpoint = checkpoint
        # one learnable step length per iteration (the "learned" part)
        self.log_lr = torch.nn.Parameter(torch.full((n_steps,), float(torch.log(torch.tensor(init_lr)))))

    def project(self, x):
        g = self.geo
        return ops.cone_projection3d(x, g.detector_shape, *g.args(), matched_adjoint=self.matched_adjoint)

    def backproject(self, r):
        g = self.geo
        if self.matched_adjoint:
            return ops.cone_backprojection3d_matched(r, g.volume_shape, *g.args())
        return ops.cone_backprojection3d(r, g.volume_shape, *g.args())

    def _step(self, x, y, lr):
        return x - lr * self.backproject(self.project(x) - y)

    def forward(self, x0, y):
        x = x0
        for k in range(self.n_steps):
            lr = self.log_lr[k].exp()
            if self.checkpoint and torch.is_grad_enabled():
                x = tcp.checkpoint(self._step, x, y, lr, use_reentrant=False)
            else:
                x = self._step(x, y, lr)
        return x


def poisson_sinogram(clean, i0: float = 1e5, seed: int = 0):
    """y = -log(Poisson(I0 exp(-p)) / I0) of a line-integral sinogram p
    (counts clamped at 1 to keep the log finite)."""
    gen = torch.Generator(device=clean.device).manual_seed(seed)
    counts = torch.poisson(i0 * torch.exp(-clean.float()), generator=gen).clamp_min(1.0)
    return -torch.log(counts / i0)
