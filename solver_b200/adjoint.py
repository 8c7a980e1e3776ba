"""Discrete adjoint of the projection step for checking harnesses.

`ProjectionLoss` is a thin ``torch.autograd.Function`` over the C ABI's
``of_adjoint_gradient``: its forward runs the steps on the device and returns
loss = 1/2 |u(T) - target|^2 over the unique velocity entries, its backward
hands back the gradients the adjoint run computed (initial velocity and
viscosity).  It exists so that test code can drive the hand-written adjoint
through torch's interface; the compute is the CUDA path behind the ABI.

`perturbed_taylor_green` builds the adjoint check's initial field: the
Taylor-Green velocity plus a seeded solenoidal perturbation (Fourier modes
|k| <= kmax with Gaussian amplitudes, scaled to a given RMS) made discretely
divergence-free by the device's own projection.
"""
from __future__ import annotations

import math

import numpy as np

from . import Context, Grid, PERIODIC, step_params


def unique_view(a, comp):
    """Active entries of a padded face field without the duplicated periodic
    face (the entries the loss and its seed are defined on)."""
    s = [slice(1, -1)] * 3
    axis = {"u": 2, "v": 1, "w": 0}[comp]
    s[axis] = slice(1, -2)
    return a[tuple(s)]


def unique_loss(vel, target):
    return 0.5 * sum(float(np.sum((unique_view(vel[c], n) - unique_view(target[c], n)) ** 2))
                     for c, n in enumerate("uvw"))


def _axis_coords(grid: Grid, loc):
    """1-D storage coordinates (x, y, z) of a padded field, ghosts included."""
    shape = grid.shape(loc)
    out = []
    for axis, (h, name) in enumerate(zip((grid.dx, grid.dy, grid.dz), "xyz")):
        idx = np.arange(shape[2 - axis]) - 1.0
        face = (loc, name) in (("u", "x"), ("v", "y"), ("w", "z"))
        out.append(idx * h if face else (idx + 0.5) * h)
    return out


def smooth_field(grid: Grid, seed, rms=1.0, kmax=4):
    """Velocity-shaped random field: Fourier modes 0 < |k| <= kmax with
    standard-normal cosine and sine amplitudes from numpy's Generator(seed)
    (drawn per component, modes in (kx, ky, kz) lexicographic order), scaled
    to the given RMS over the active entries (padded arrays, edges and corners
    zero).  a cos(k.x) + b sin(k.x) = Re((a - ib) e^{ik.x}) is summed axis by
    axis, so a 512^3 field costs three small contractions and one matrix
    product instead of a pass over the grid per mode."""
    g = grid
    rng = np.random.default_rng(seed)
    ks = np.arange(-kmax, kmax + 1)
    modes = [(kx, ky, kz) for kx in ks for ky in ks for kz in ks
             if 0 < kx * kx + ky * ky + kz * kz <= kmax * kmax and (g.nz > 1 or kz == 0)]
    out = []
    for comp in "uvw":
        f = np.zeros(g.shape(comp))
        if not (comp == "w" and g.nz == 1):
            coef = np.zeros((ks.size, ks.size, ks.size), dtype=np.complex128)  # [kz, ky, kx]
            for (kx, ky, kz) in modes:
                a, b = rng.standard_normal(2)
                coef[kz + kmax, ky + kmax, kx + kmax] += a - 1j * b
            x, y, z = _axis_coords(g, comp)
            ex = np.exp(1j * np.outer(ks, x))  # [kx, i]
            ey = np.exp(1j * np.outer(ks, y))  # [ky, j]
            ez = np.exp(1j * np.outer(ks, z))  # [kz, k]
            t = np.einsum("abc,ci->abi", coef, ex)  # [kz, ky, i]
            t = np.einsum("bj,abi->aji", ey, t).reshape(ks.size, -1)  # [kz, j*i]
            f = (ez.real.T @ t.real - ez.imag.T @ t.imag).reshape(g.shape(comp))
        out.append(f)
    cur_rms = math.sqrt(sum(float(np.mean(a[1:-1, 1:-1, 1:-1] ** 2)) for a in out) / 3.0)
    for a in out:
        a *= rms / cur_rms
        _zero_edges(a)
    return out


def perturbed_taylor_green(ctx: Context, viscosity, dt, seed, rms=1.0e-2, kmax=4,
                           max_iterations=400, tolerance=1.0e-13):
    """Taylor-Green (the u = sin x cos y cos z phase) plus a seeded
    solenoidal perturbation (smooth_field, then the device's discrete
    projection); returns the padded (u, v, w, p) host arrays."""
    g = ctx.grid
    ctx.tg_init(viscosity, dt, mode=1)
    st = ctx.download_state()
    pert = smooth_field(g, seed, rms, kmax)
    vel = [st[c] + pert[i] for i, c in enumerate("uvw")]
    for a in vel:  # edges and corners stay zero, as the reference never writes them
        _zero_edges(a)
    (u, v, w), _, _, _ = ctx.project_velocity(vel, dt, 1.0, max_iterations, tolerance)
    return u, v, w, st["p"]


def _zero_edges(a):
    sz, sy, sx = a.shape
    for k in (0, sz - 1):
        for j in (0, sy - 1):
            a[k, j, :] = 0.0
        for i in (0, sx - 1):
            a[k, :, i] = 0.0
    for j in (0, sy - 1):
        for i in (0, sx - 1):
            a[:, j, i] = 0.0


def upload_initial(ctx: Context, state):
    """Makes (u, v, w, p) the resident state at step 0 (no AB2 history)."""
    u, v, w, p = state
    g = ctx.grid
    z = [g.zeros(c) for c in "uvw"]
    ctx.upload_state(u, v, w, z[0], z[1], z[2], p, False, None)


def _torch():
    import torch
    return torch


class ProjectionLoss:
    """torch.autograd.Function: loss(u0, v0, w0, nu) for a fixed target.

    apply(ctx, state_p, steps, every, target, dt, max_iterations, tolerance,
          u0, v0, w0, nu) with u0, v0, w0 float64 CPU tensors in padded storage
    and nu a 0-d float64 tensor; returns the 0-d loss tensor."""

    @staticmethod
    def _function():
        torch = _torch()

        class _F(torch.autograd.Function):
            @staticmethod
            def forward(fctx, ctx, p0, steps, every, target, dt, max_iterations, tolerance, u0, v0,
                        w0, nu):
                upload_initial(ctx, (u0.detach().numpy().copy(), v0.detach().numpy().copy(),
                                     w0.detach().numpy().copy(), p0))
                prm = step_params(float(nu), dt, max_iterations, tolerance)
                grad, info = ctx.adjoint_gradient(prm, steps, target, checkpoint_every=every)
                fctx.save_for_backward(*(torch.from_numpy(gr) for gr in grad),
                                       torch.tensor(info["grad_viscosity"], dtype=torch.float64))
                return torch.tensor(info["loss"], dtype=torch.float64)

            @staticmethod
            def backward(fctx, g_loss):
                gu, gv, gw, gnu = fctx.saved_tensors
                return (None, None, None, None, None, None, None, None, g_loss * gu, g_loss * gv,
                        g_loss * gw, g_loss * gnu)

        return _F

    @classmethod
    def apply(cls, *args):
        return cls._function().apply(*args)


__all__ = ["ProjectionLoss", "perturbed_taylor_green", "smooth_field", "unique_loss",
           "unique_view", "upload_initial", "PERIODIC"]
