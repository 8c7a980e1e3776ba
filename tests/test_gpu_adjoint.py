"""Tangent-linear and adjoint runs of the projection step (periodic grids).

There is no reference code for derivatives; they are pinned by the checks the
adjoint check configuration names: central finite differences of the forward
run (tangent-linear velocity, gradient along a direction, viscosity
derivative), the dot-product test <J d, w> = <d, J^T w> between the FP64
tangent-linear and adjoint runs, invariance under the checkpoint interval, the
torch.autograd.Function wrapper, and the mixed-precision gradient against the
FP64 one.

Tolerances: dot-product test 1e-10 (both sides are exact transposes up to
rounding and the pressure-solve tolerance 1e-12); finite differences 1e-6
relative.  The finite differences run along smooth directions (Fourier modes
|k| <= 4) with eps = 1e-8 on O(1) fields.  The limiter, upwind-side and
first-order switches of the TVD advection make the step only piecewise
smooth: a central difference sees the derivative only while no van Leer ratio
crosses its kink at r = 0 within +-eps, and on the Taylor-Green base state
some ratios sit within ~1e-6 of it (measured on 16^3, 4 steps: relative
differences 7e-5, 2e-7 and 7e-9 at eps = 1e-6, 1e-7 and 1e-8).  The runs at
+-eps take the same pressure iterations, so the solve does not add noise.
"""
import math

import numpy as np
import pytest

import solver_b200 as sb
from solver_b200.adjoint import (ProjectionLoss, perturbed_taylor_green, smooth_field, unique_loss,
                                 unique_view, upload_initial)

pytestmark = pytest.mark.gpu

NU = 0.01
STEPS = 4
TOL = 1e-12
FD_TOL = 1e-6
DOT_TOL = 1e-10
EPS = 1e-8
EPS_NU = 1e-6  # relative step of the viscosity (the loss changes by ~1e-8 of itself)


def _setup(n=16, precision=sb.OF_FP64, seed=1):
    h = 2.0 * math.pi / n
    g = sb.Grid(n, n, n, h, h, h)
    ctx = sb.Context(g, [sb.PERIODIC] * 6, precision=precision)
    dt = h / 6.0  # CFL 0.5 with the velocity-free bound
    state = perturbed_taylor_green(ctx, NU, dt, seed=seed)
    prm = sb.step_params(NU, dt, 400, TOL)
    return ctx, g, dt, prm, state


def _direction(g, seed):
    rng = np.random.default_rng(seed)
    d = []
    for c in "uvw":
        a = g.zeros(c)
        a[1:-1, 1:-1, 1:-1] = rng.standard_normal(a[1:-1, 1:-1, 1:-1].shape)
        d.append(a)
    return d


def _smooth_direction(g, seed):
    return smooth_field(g, seed, rms=1.0)


def _shifted(state, d, eps):
    u, v, w, p = state
    return (u + eps * d[0], v + eps * d[1], w + eps * d[2], p)


def _forward(ctx, state, prm, steps):
    upload_initial(ctx, state)
    ctx.run_steps(prm, steps)
    st = ctx.download_state()
    return [st[c] for c in "uvw"]


def _unique_dot(a, b):
    return sum(float(np.sum(unique_view(a[i], c) * unique_view(b[i], c))) for i, c in enumerate("uvw"))


def _active_dot(a, b):
    return sum(float(np.sum(a[i][1:-1, 1:-1, 1:-1] * b[i][1:-1, 1:-1, 1:-1])) for i in range(3))


@pytest.fixture(scope="module")
def case():
    ctx, g, dt, prm, state = _setup()
    yield ctx, g, dt, prm, state
    ctx.close()


def test_perturbed_initial_field_is_divergence_free(case):
    ctx, g, dt, prm, state = case
    u, v, w, _ = state
    div = ((u[1:-1, 1:-1, 2:-1] - u[1:-1, 1:-1, 1:-2]) / g.dx + (v[1:-1, 2:-1, 1:-1] - v[1:-1, 1:-2, 1:-1]) / g.dy
           + (w[2:-1, 1:-1, 1:-1] - w[1:-2, 1:-1, 1:-1]) / g.dz)
    assert np.sqrt(np.mean(div ** 2)) < 1e-10


def test_tangent_linear_matches_central_difference(case):
    ctx, g, dt, prm, state = case
    d = _smooth_direction(g, 7)
    upload_initial(ctx, state)
    tl = ctx.tangent_linear(prm, STEPS, d)
    eps = EPS
    fp = _forward(ctx, _shifted(state, d, eps), prm, STEPS)
    fm = _forward(ctx, _shifted(state, d, -eps), prm, STEPS)
    fd = [(a - b) / (2 * eps) for a, b in zip(fp, fm)]
    num = math.sqrt(sum(float(np.sum((unique_view(tl[i], c) - unique_view(fd[i], c)) ** 2))
                        for i, c in enumerate("uvw")))
    den = math.sqrt(_unique_dot(fd, fd))
    assert num / den <= FD_TOL, num / den


def test_dot_product_tangent_linear_vs_adjoint(case):
    ctx, g, dt, prm, state = case
    d = _direction(g, 11)
    w = _direction(g, 12)
    uT = _forward(ctx, state, prm, STEPS)
    target = [uT[i] - w[i] for i in range(3)]
    upload_initial(ctx, state)
    grad, info = ctx.adjoint_gradient(prm, STEPS, target, checkpoint_every=2)
    upload_initial(ctx, state)
    tl = ctx.tangent_linear(prm, STEPS, d)
    lhs = _unique_dot(tl, w)
    rhs = _active_dot(d, grad)
    assert abs(lhs - rhs) <= DOT_TOL * max(abs(lhs), abs(rhs)), (lhs, rhs)
    assert abs(info["loss"] - 0.5 * _unique_dot(w, w)) <= 1e-12 * info["loss"]


def test_gradient_matches_central_difference(case):
    ctx, g, dt, prm, state = case
    rng = np.random.default_rng(3)
    uT = _forward(ctx, state, prm, STEPS)
    target = [a + 0.1 * rng.standard_normal(a.shape) for a in uT]
    upload_initial(ctx, state)
    grad, info = ctx.adjoint_gradient(prm, STEPS, target, checkpoint_every=STEPS)
    d = _smooth_direction(g, 5)
    eps = EPS
    lp = unique_loss(_forward(ctx, _shifted(state, d, eps), prm, STEPS), target)
    lm = unique_loss(_forward(ctx, _shifted(state, d, -eps), prm, STEPS), target)
    fd = (lp - lm) / (2 * eps)
    ad = _active_dot(d, grad)
    assert abs(fd - ad) <= FD_TOL * abs(fd), (fd, ad)
    assert abs(info["loss"] - unique_loss(uT, target)) <= 1e-12 * info["loss"]


def test_viscosity_gradient_matches_central_difference(case):
    ctx, g, dt, prm, state = case
    rng = np.random.default_rng(4)
    uT = _forward(ctx, state, prm, STEPS)
    target = [a + 0.1 * rng.standard_normal(a.shape) for a in uT]
    upload_initial(ctx, state)
    _, info = ctx.adjoint_gradient(prm, STEPS, target, checkpoint_every=3)
    eps = EPS_NU * NU
    lp = unique_loss(_forward(ctx, state, sb.step_params(NU + eps, dt, 400, TOL), STEPS), target)
    lm = unique_loss(_forward(ctx, state, sb.step_params(NU - eps, dt, 400, TOL), STEPS), target)
    fd = (lp - lm) / (2 * eps)
    assert abs(fd - info["grad_viscosity"]) <= FD_TOL * abs(fd), (fd, info["grad_viscosity"])


def test_gradient_independent_of_checkpoint_interval(case):
    ctx, g, dt, prm, state = case
    w = _direction(g, 21)
    uT = _forward(ctx, state, prm, STEPS)
    target = [uT[i] - w[i] for i in range(3)]
    grads = []
    for every in (1, 3, STEPS):
        upload_initial(ctx, state)
        grad, info = ctx.adjoint_gradient(prm, STEPS, target, checkpoint_every=every)
        grads.append((grad, info))
        # the last segment's states are kept by the first pass; the others are
        # recomputed from their checkpoints
        segs = list(range(0, STEPS, every))
        expected_forward = STEPS + sum(min(every, STEPS - k) - 1 for k in segs[:-1])
        assert info["forward_steps"] == expected_forward
    ref = np.concatenate([a.ravel() for a in grads[0][0]])
    for grad, info in grads[1:]:
        cur = np.concatenate([a.ravel() for a in grad])
        assert np.max(np.abs(cur - ref)) <= 1e-12 * np.max(np.abs(ref))
        assert abs(info["grad_viscosity"] - grads[0][1]["grad_viscosity"]) <= \
            1e-12 * abs(grads[0][1]["grad_viscosity"])


@pytest.mark.parametrize("snapshots", [0, 1, 2, 3])
def test_binomial_schedule_gives_the_stored_state_gradient(case, snapshots):
    """of_adjoint_gradient_binomial reverses 9 steps with 1, 2 or 3 snapshots
    (recursion of the binomial schedule, the one-snapshot case recomputing
    from the initial state) or as many as fit (0: all 8): the gradient, the
    loss and the viscosity derivative equal those of the run that keeps every
    state (one segment) to rounding (1e-12 relative; the transposed advection
    scatters with atomics, so two runs of either schedule differ in the last
    bits), the loss bitwise (it is formed by the forward pass), and the
    number of forward steps is the schedule's published minimum."""
    ctx, g, dt, prm, state = case
    steps = 9
    w = _direction(g, 23)
    uT = _forward(ctx, state, prm, steps)
    target = [uT[i] - w[i] for i in range(3)]
    upload_initial(ctx, state)
    ref, ref_info = ctx.adjoint_gradient(prm, steps, target, checkpoint_every=steps)
    upload_initial(ctx, state)
    grad, info = ctx.adjoint_gradient_binomial(prm, steps, target, snapshots=snapshots)
    used = snapshots if snapshots else steps - 1
    assert info["snapshots"] == used
    assert info["forward_steps"] == steps + sb.adjoint_schedule_cost(steps, used)[1]
    gmax = max(float(np.max(np.abs(b))) for b in ref)
    for a, b in zip(grad, ref):
        assert np.max(np.abs(a - b)) <= 1e-12 * gmax
    assert info["loss"] == ref_info["loss"]
    assert abs(info["grad_viscosity"] - ref_info["grad_viscosity"]) <= \
        1e-12 * abs(ref_info["grad_viscosity"])
    # the resident state is left at step `steps`, as of_run_steps leaves it
    st = ctx.download_state()
    assert st["metrics"]["step"] == steps
    assert np.array_equal(st["u"], uT[0])


def test_torch_autograd_function_returns_adjoint_gradients(case):
    torch = pytest.importorskip("torch")
    ctx, g, dt, prm, state = case
    w = _direction(g, 31)
    uT = _forward(ctx, state, prm, STEPS)
    target = [uT[i] - w[i] for i in range(3)]
    upload_initial(ctx, state)
    grad, info = ctx.adjoint_gradient(prm, STEPS, target, checkpoint_every=2)
    u0 = [torch.from_numpy(a.copy()).requires_grad_(True) for a in state[:3]]
    nu = torch.tensor(NU, dtype=torch.float64, requires_grad=True)
    loss = ProjectionLoss.apply(ctx, state[3], STEPS, 2, target, dt, 400, TOL, u0[0], u0[1], u0[2], nu)
    loss.backward()
    assert abs(loss.item() - info["loss"]) <= 1e-14 * info["loss"]
    for t, a in zip(u0, grad):
        assert np.max(np.abs(t.grad.numpy() - a)) <= 1e-12 * np.max(np.abs(a))
    assert abs(nu.grad.item() - info["grad_viscosity"]) <= 1e-12 * abs(info["grad_viscosity"])


def test_mixed_precision_gradient_matches_fp64():
    ctx, g, dt, prm, state = _setup(precision=sb.OF_FP64)
    w = _direction(g, 41)
    uT = _forward(ctx, state, prm, STEPS)
    target = [uT[i] - w[i] for i in range(3)]
    upload_initial(ctx, state)
    g64, i64 = ctx.adjoint_gradient(prm, STEPS, target, checkpoint_every=2)
    ctx.set_precision(sb.OF_MIXED)
    upload_initial(ctx, state)
    g32, i32 = ctx.adjoint_gradient(prm, STEPS, target, checkpoint_every=2)
    ref = np.concatenate([a.ravel() for a in g64])
    cur = np.concatenate([a.ravel() for a in g32])
    assert np.max(np.abs(cur - ref)) <= 1e-8 * np.max(np.abs(ref))
    assert abs(i32["grad_viscosity"] - i64["grad_viscosity"]) <= 1e-8 * abs(i64["grad_viscosity"])
    ctx.close()


def test_adjoint_rejects_walls():
    g = sb.Grid(8, 8, 1, 1 / 8, 1 / 8, 1.0)
    bc = [sb.NO_SLIP_WALL] * 4 + [sb.PERIODIC] * 2
    ctx = sb.Context(g, bc)
    z = [g.zeros(c) for c in "uvw"]
    ctx.upload_state(*z, *[g.zeros(c) for c in "uvw"], g.zeros("p"))
    with pytest.raises(ValueError, match="periodic boundaries only"):
        ctx.adjoint_gradient(sb.step_params(0.01, 0.01, 100, 1e-10), 1, z)
    ctx.close()
