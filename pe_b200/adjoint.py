"""Gradients of the DEM step: loss helpers and a torch.autograd.Function around the C ABI's
adjoint (pe_b200_adjoint_forward / pe_b200_adjoint_backward).

The autograd Function exists as a gradient-check harness (torch.autograd.gradcheck); the
gradient itself is computed by the library's adjoint kernel.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import _abi, scenes
from .engine import Engine


def sphere_masses(s) -> np.ndarray:
    """pe's sphere mass 4/3 pi r^3 rho (SphereBase.h:169-171)."""
    rho = s.materials[s.mat, 0]
    return 4.0 / 3.0 * math.pi * s.r * s.r * s.r * rho


def make_single_material(s, k_n, c_n, c_t, mu, density=1.0):
    """Copy of scene s with one material (spheres and walls) of the given contact coefficients."""
    t = s.copy()
    t.materials = scenes.material(density, k_n, c_n, c_t, mu)[None, :]
    t.mat = np.zeros_like(s.mat)
    t.plane_mat = np.zeros_like(s.plane_mat)
    t.box_mat = np.zeros_like(s.box_mat)
    return t


def set_params(s, k_n, c_n, c_t, mu):
    """Copy of a single-material scene with new contact coefficients."""
    t = s.copy()
    t.materials = scenes.material(float(s.materials[0, 0]), k_n, c_n, c_t, mu)[None, :]
    return t


@dataclasses.dataclass
class LossSpec:
    """Final centre-of-mass height plus the fraction of mass below an opening height z_open.

    The fraction uses a logistic step of width `width` (a hard indicator has zero gradient almost
    everywhere, for finite differences as much as for the adjoint)."""
    m: np.ndarray
    z_open: float
    width: float = 0.1

    @staticmethod
    def for_scene(s, z_open=None, width=0.1):
        z = float(np.median(s.x[:, 2])) if z_open is None else float(z_open)
        return LossSpec(m=sphere_masses(s), z_open=z, width=width)

    def value(self, x) -> float:
        M = self.m.sum()
        z = x[:, 2]
        sig = 1.0 / (1.0 + np.exp(-(self.z_open - z) / self.width))
        return float((self.m * z).sum() / M + (self.m * sig).sum() / M)

    def diff(self, xp, xm) -> float:
        """value(xp) - value(xm), summed term by term so that the large common part cancels
        exactly (central differences of a loss of order 10 with h = 1e-6 would otherwise lose
        most of their digits)."""
        M = self.m.sum()
        zp, zm = xp[:, 2], xm[:, 2]
        sp = 1.0 / (1.0 + np.exp(-(self.z_open - zp) / self.width))
        sm = 1.0 / (1.0 + np.exp(-(self.z_open - zm) / self.width))
        return float((self.m * (zp - zm)).sum() / M + (self.m * (sp - sm)).sum() / M)

    def grad(self, x) -> np.ndarray:
        M = self.m.sum()
        z = x[:, 2]
        sig = 1.0 / (1.0 + np.exp(-(self.z_open - z) / self.width))
        g = np.zeros_like(x)
        g[:, 2] = self.m / M - self.m / M * sig * (1.0 - sig) / self.width
        return g


def difference_ladder(diff, hs, smooth_tol=1e-4):
    """Finite differences of a loss at each step h of the ladder `hs` (largest first).

    diff(a, b) returns loss(input + a) - loss(input + b), summed term by term (LossSpec.diff of
    two runs).  For each h: the forward difference (L(p+h) - L(p)) / h, the backward difference
    (L(p) - L(p-h)) / h and the central difference (their mean).  A DEM loss is only piecewise
    smooth: pe's dashpot force jumps from 0 to c_n v_n when a contact starts, so when a
    perturbation moves some contact's first step across a step boundary inside [p - h, p + h],
    the difference quotient picks up that jump.  The forward and backward differences then
    disagree; `smooth` marks the steps where they agree to smooth_tol (relative).  `chosen` is
    the largest smooth step (the smallest step when none is), the one a derivative is checked
    against."""
    rows = []
    for h in hs:
        fwd = diff(h, 0.0) / h
        bwd = diff(0.0, -h) / h
        cen = 0.5 * (fwd + bwd)
        rows.append({"h": h, "forward": fwd, "backward": bwd, "central": cen,
                     "smooth": bool(abs(fwd - bwd) <= smooth_tol * max(abs(cen), 1e-300))})
    chosen = next((r for r in rows if r["smooth"]), rows[-1])
    return rows, chosen


def _coeffs(s):
    m = s.materials[0]
    return {"k_n": m[6] / 2.0, "c_n": m[7] / 2.0, "c_t": m[8] / 2.0, "mu": m[2] + m[2]}


def dem_loss(v0, scales, s, spec: LossSpec, nsteps: int, every: int):
    """Loss after nsteps FP64 DEM steps as a function of the initial velocities v0 (n x 3) and
    scale factors of (k_n, c_n, mu) around scene s's single material."""
    import torch

    class _DemLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, v, sc):
            c = _coeffs(s)
            base = np.array([c["k_n"], c["c_n"], c["mu"]])
            p = base * sc.detach().cpu().numpy()
            t = set_params(s, p[0], p[1], c["c_t"], p[2])
            t.v = v.detach().cpu().numpy().astype(np.float64).copy()
            e = Engine(solver=_abi.DEM, precision=_abi.FP64).load_scene(t)
            e.adjoint_forward(nsteps, t.dt, every)
            x = e.download()[0]
            ctx.e, ctx.x, ctx.base = e, x, base
            return torch.tensor(spec.value(x), dtype=torch.float64)

        @staticmethod
        def backward(ctx, g):
            gx = spec.grad(ctx.x)
            z = np.zeros_like(gx)
            # the engine keeps its checkpoints, so backward may run more than once
            _, gv0, _, gp = ctx.e.adjoint_backward(gx, z, z)
            gs = np.array([gp[0], gp[1], gp[3]]) * ctx.base
            gval = float(g)
            return (torch.tensor(gv0 * gval, dtype=torch.float64),
                    torch.tensor(gs * gval, dtype=torch.float64))

    return _DemLoss.apply(v0, scales)
