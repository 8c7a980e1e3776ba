"""GPU parity against the CPU oracle, through the C ABI (include/orchard_b200.h).

Tolerances: the FP64 path must match the reference's deterministic CPU build
to a max-norm relative difference of 1e-11 (velocity and pressure after N
steps); single operators are compared at 1e-12.  Sums on the GPU use a
different (tree) order than the CPU's sequential loops, so results differ at
the rounding level, never more.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_maxdiff, to_gpu_bc, to_gpu_grid, to_gpu_pbc

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-11
OP_TOL = 1e-12


@pytest.fixture(scope="module")
def sb():
    import solver_b200
    return solver_b200


def _random_velocity(grid, rng, amp=1.0):
    return [rng.standard_normal(po.shape(grid, c)) * amp for c in "uvw"]


def _tg_gpu_run(sb, oracle, cfg, steps, mode=0, variant=0):
    g = oracle.tg_grid(cfg)
    bc = oracle.tg_bc(cfg)
    dt = oracle.tg_dt(cfg)
    s0 = oracle.tg_init(cfg, 0)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(bc))
    ctx.upload_state(s0.u, s0.v, s0.w, s0.adv_u, s0.adv_v, s0.adv_w, s0.p, s0.has_previous_advection,
                     s0.metrics)
    prm = sb.step_params(cfg.viscosity, dt, cfg.poisson_max_iterations, cfg.poisson_tolerance)
    metrics = ctx.run_steps(prm, steps)
    out = ctx.download_state()
    ref = oracle.tg_steps(cfg, steps, s0.copy())
    return out, ref, metrics


# 32^2 and 64x32x16 exercise the shared-memory tiled stencil kernels (nx % 32 == 0,
# ny % 8 == 0); 16^3 and 12x10x8 the general kernels.
@pytest.mark.parametrize("n,steps", [((32, 32, 1), 5), ((16, 16, 16), 3), ((12, 10, 8), 3),
                                     ((64, 32, 16), 2)])
def test_taylor_green_steps_match_oracle(sb, oracle, n, steps):
    cfg = po.steps_config(*n, 0.01, 0.5, steps, 1e-12)
    out, ref, metrics = _tg_gpu_run(sb, oracle, cfg, steps)
    for name in ("u", "v", "w", "p", "adv_u", "adv_v", "adv_w"):
        d = rel_maxdiff(out[name], getattr(ref, name))
        assert d <= STEP_TOL, (name, d)
    assert metrics["step"] == ref.metrics["step"] == steps
    assert metrics["pressure_iterations"] == ref.metrics["pressure_iterations"]
    assert abs(metrics["max_cfl"] - ref.metrics["max_cfl"]) <= 1e-12 * ref.metrics["max_cfl"]
    assert metrics["divergence_l2"] <= 1e-10


def test_cavity_steps_match_oracle(sb, oracle):
    cc = po.cavity_config(32, 32, poisson_tolerance=1e-12)
    g = oracle.cavity_grid(cc)
    bc = oracle.cavity_bc(cc)
    s0 = oracle.cavity_init(cc)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(bc))
    ctx.upload_state(s0.u, s0.v, s0.w, s0.adv_u, s0.adv_v, s0.adv_w, s0.p, 0, s0.metrics)
    nu = cc.lid_velocity / cc.reynolds
    prm = sb.step_params(nu, oracle.cavity_dt(cc), cc.poisson_max_iterations, cc.poisson_tolerance,
                         variant=sb.OF_CORRECTION_CAVITY)
    m = ctx.run_steps(prm, 6)
    out = ctx.download_state()
    ref = oracle.cavity_steps(cc, 6, s0.copy())
    for name in ("u", "v", "p"):
        d = rel_maxdiff(out[name], getattr(ref, name))
        assert d <= STEP_TOL, (name, d)
    assert m["pressure_iterations"] == ref.metrics["pressure_iterations"]


def test_advection_matches_oracle(sb, oracle):
    rng = np.random.default_rng(1)
    g = po.Grid(12, 9, 7, 0.3, 0.25, 0.4)
    u, v, w = _random_velocity(g, rng)
    ctx = sb.Context(to_gpu_grid(g), [sb.PERIODIC] * 6)
    got = ctx.compute_advection_term(u, v, w)
    exp = oracle.advection(g, u, v, w)
    for a, b in zip(got, exp):
        assert rel_maxdiff(a, b) <= OP_TOL


@pytest.mark.parametrize("types", [
    [po.PERIODIC] * 6,
    [po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.PRESCRIBED_VELOCITY, po.SYMMETRY,
     po.SYMMETRY],
    [po.PERIODIC, po.PERIODIC, po.NO_SLIP_WALL, po.PRESCRIBED_VELOCITY, po.PERIODIC, po.PERIODIC],
])
def test_predictor_adi_matches_oracle(sb, oracle, types):
    rng = np.random.default_rng(2)
    g = po.Grid(10, 8, 6, 0.2, 0.3, 0.25)
    vel = [None] * 6
    vel[3] = (0.7, 0.0, 0.1)
    bc = po.bc_from(types, vel)
    rhs = _random_velocity(g, rng)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(bc))
    got, lines = ctx.solve_predictor_adi(rhs, 0.05)
    exp, lines_ref = oracle.predictor_adi(g, bc, 0.05, *rhs)
    assert lines == lines_ref
    for a, b in zip(got, exp):
        assert rel_maxdiff(a, b) <= OP_TOL


@pytest.mark.parametrize("types", [
    [po.PERIODIC] * 6,
    [po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.PRESCRIBED_VELOCITY, po.SYMMETRY,
     po.SYMMETRY],
    [po.PERIODIC, po.PERIODIC, po.NO_SLIP_WALL, po.PRESCRIBED_VELOCITY, po.PERIODIC, po.PERIODIC],
])
def test_predictor_adi_partition_solver_matches_oracle(sb, oracle, types):
    """Lines of 64 and 96 unknowns take the warp-per-line partition solver."""
    rng = np.random.default_rng(5)
    g = po.Grid(64, 96, 64, 0.02, 0.03, 0.025)
    vel = [None] * 6
    vel[3] = (0.7, 0.0, 0.1)
    bc = po.bc_from(types, vel)
    rhs = _random_velocity(g, rng)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(bc))
    got, lines = ctx.solve_predictor_adi(rhs, 0.3)
    exp, lines_ref = oracle.predictor_adi(g, bc, 0.3, *rhs)
    assert lines == lines_ref
    for a, b in zip(got, exp):
        assert rel_maxdiff(a, b) <= OP_TOL


@pytest.mark.parametrize("shape", [(200, 130, 1), (1000, 40, 1), (96, 70, 12)])
def test_predictor_adi_padded_wall_lines_match_oracle(sb, oracle, shape):
    """Wall lines whose length is not a multiple of 32 (199, 999, 95 ...
    unknowns) take the warp-scan solver padded to a multiple of 32; few long
    lines (2D) use blocks of four lines."""
    rng = np.random.default_rng(9)
    nx, ny, nz = shape
    g = po.Grid(nx, ny, nz, 1.0 / nx, 1.0 / ny, 1.0 if nz == 1 else 1.0 / nz)
    types = [po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.PRESCRIBED_VELOCITY, po.SYMMETRY,
             po.SYMMETRY]
    vel = [None] * 6
    vel[3] = (1.0, 0.0, 0.0)
    bc = po.bc_from(types, vel)
    rhs = _random_velocity(g, rng)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(bc))
    got, lines = ctx.solve_predictor_adi(rhs, 0.5 * 0.01 * 0.5 / (nx + ny))
    exp, lines_ref = oracle.predictor_adi(g, bc, 0.5 * 0.01 * 0.5 / (nx + ny), *rhs)
    assert lines == lines_ref
    for a, b in zip(got, exp):
        assert rel_maxdiff(a, b) <= OP_TOL


@pytest.mark.parametrize("case", ["dirichlet2d", "neumann2d", "periodic3d", "mixed3d",
                                  "mixed3d_tiled"])
def test_poisson_matches_oracle(sb, oracle, case):
    rng = np.random.default_rng(3)
    if case == "dirichlet2d":
        g = po.Grid(32, 32, 1, 1 / 32, 1 / 32, 1.0)
        types = [po.P_DIRICHLET] * 4 + [po.P_NEUMANN] * 2
        vals = [0.3, -0.1, 0.2, 0.0, 0.0, 0.0]
        pbc = po.pbc_from(types, vals)
    elif case == "neumann2d":
        g = po.Grid(24, 24, 1, 1 / 24, 1 / 24, 1.0)
        pbc = po.pbc_from([po.P_NEUMANN] * 6, gradients=[0.1, 0.1, -0.2, -0.2, 0.0, 0.0])
    elif case == "periodic3d":
        g = po.Grid(16, 16, 16, 0.39, 0.39, 0.39)
        pbc = po.pbc_from([po.P_PERIODIC] * 6)
    elif case == "mixed3d":
        g = po.Grid(16, 8, 12, 0.1, 0.2, 0.15)
        pbc = po.pbc_from([po.P_PERIODIC, po.P_PERIODIC, po.P_NEUMANN, po.P_DIRICHLET,
                           po.P_NEUMANN, po.P_NEUMANN])
    else:
        g = po.Grid(64, 32, 16, 0.1, 0.2, 0.15)
        pbc = po.pbc_from([po.P_NEUMANN, po.P_DIRICHLET, po.P_PERIODIC, po.P_PERIODIC,
                           po.P_DIRICHLET, po.P_NEUMANN], values=[0, 0.2, 0, 0, -0.1, 0])
    rhs = rng.standard_normal(po.shape(g, "p"))
    ctx = sb.Context(to_gpu_grid(g), [sb.PERIODIC] * 6)
    p_gpu, d = ctx.solve_pressure_poisson(rhs, to_gpu_pbc(pbc), 200, 1e-12)
    p_ref = np.zeros(po.shape(g, "p"))
    dref, hist = oracle.poisson_solve(g, pbc, 200, 1e-12, rhs, p_ref)
    info = (d["iterations"], dref.iterations, d["relative_residual"], dref.relative_residual,
            rel_maxdiff(p_gpu, p_ref))
    assert d["converged"] and dref.converged, info
    assert d["multigrid_levels"] == dref.multigrid_levels
    assert d["coarse_unknowns"] == dref.coarse_unknowns
    assert d["zero_mean_enforced"] == bool(dref.zero_mean_enforced)
    n = min(len(hist), len(d["residual_history"]))
    # near convergence the norms are rounding-dominated: compare against r0
    np.testing.assert_allclose(d["residual_history"][:n], hist[:n], rtol=1e-9,
                               atol=1e-10 * hist[0], err_msg=str(info))
    if d["iterations"] == dref.iterations:
        assert rel_maxdiff(p_gpu, p_ref) <= 1e-11, info
    else:
        # the two runs straddle the stopping threshold (relative residual within
        # rounding of the tolerance): one extra iteration, solutions agree to the
        # tolerance's order
        assert abs(d["iterations"] - dref.iterations) == 1, info
        assert rel_maxdiff(p_gpu, p_ref) <= 1e-9, info


def test_project_velocity_matches_oracle(sb, oracle):
    rng = np.random.default_rng(4)
    g = po.Grid(16, 12, 10, 0.2, 0.25, 0.3)
    bc = po.periodic_bc()
    pred = _random_velocity(g, rng)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(bc))
    (cu, cv, cw), phi, rhs, d = ctx.project_velocity(pred, 0.01, 1.0, 200, 1e-12)
    exp, rhs_ref, dref = oracle.project_velocity(g, bc, 0.01, 1.0, 200, 1e-12, *pred,
                                                 np.zeros(po.shape(g, "p")))
    for a, b in zip((cu, cv, cw), exp):
        assert rel_maxdiff(a, b) <= OP_TOL * 10
    assert rel_maxdiff(rhs, rhs_ref) <= OP_TOL
    assert d["pressure_solve"]["iterations"] == dref.pressure_solve.iterations
    assert d["divergence_l2_after"] <= 1e-10
    assert abs(d["divergence_l2_before"] - dref.divergence_l2_before) <= 1e-12 * dref.divergence_l2_before


def test_host_loop_and_graph_paths_agree(sb, oracle, monkeypatch):
    """The PCG loop runs as one CUDA graph with a device-controlled WHILE node;
    the host-driven loop (one launch per kernel) must give the same result."""
    cfg = po.steps_config(16, 16, 16, 0.01, 0.5, 2, 1e-12)
    outs = []
    for no_graph in ("0", "1"):
        monkeypatch.setenv("ORCHARD_B200_NO_GRAPH", no_graph)
        out, ref, m = _tg_gpu_run(sb, oracle, cfg, 2)
        outs.append((out, m))
        for name in ("u", "v", "w", "p"):
            assert rel_maxdiff(out[name], getattr(ref, name)) <= STEP_TOL
    (a, ma), (b, mb) = outs
    assert ma["pressure_iterations"] == mb["pressure_iterations"]
    for name in ("u", "v", "w", "p"):
        assert np.array_equal(a[name], b[name]), name


def test_poisson_nonconvergence_reports_like_reference(sb, oracle):
    # tests/test_runtime.cpp:1777-1792: one iteration at tolerance 1e-30 must fail
    cfg = po.tg_config(16, 16, 1, 0.01, 0.25, 0.01, 1, 1e-30)
    g = oracle.tg_grid(cfg)
    s0 = oracle.tg_init(cfg, 0)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(oracle.tg_bc(cfg)))
    ctx.upload_state(s0.u, s0.v, s0.w, s0.adv_u, s0.adv_v, s0.adv_w, s0.p, 0, s0.metrics)
    with pytest.raises(sb.NotConvergedError,
                       match="Taylor-Green pressure solve did not converge at step 1"):
        ctx.run_steps(sb.step_params(cfg.viscosity, oracle.tg_dt(cfg), 1, 1e-30), 1)
    st = ctx.download_state()
    assert st["metrics"]["step"] == 0  # the state is left at the last completed step
    assert np.array_equal(st["u"], s0.u)


@pytest.mark.parametrize("n", [(32, 32, 32), (64, 32, 16), (48, 40, 8)])
def test_mixed_precision_matches_fp64(sb, oracle, n):
    """OF_MIXED (FP32 inner MG-PCG inside FP64 defect correction) converges to
    the same relative residual as the FP64 path, so the states agree to the
    solve tolerance (1e-12): checked at 1e-9 relative after 8 steps, and the
    mixed state against the oracle at the same bound."""
    cfg = po.steps_config(*n, 0.01, 0.5, 8, 1e-12)
    g = oracle.tg_grid(cfg)
    s0 = oracle.tg_init(cfg, 0)
    outs = {}
    for prec in (sb.OF_FP64, sb.OF_MIXED):
        ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(oracle.tg_bc(cfg)), precision=prec)
        ctx.upload_state(s0.u, s0.v, s0.w, s0.adv_u, s0.adv_v, s0.adv_w, s0.p, 0, s0.metrics)
        prm = sb.step_params(cfg.viscosity, oracle.tg_dt(cfg), cfg.poisson_max_iterations,
                             cfg.poisson_tolerance)
        m = ctx.run_steps(prm, 8)
        outs[prec] = (ctx.download_state(), m)
        ctx.close()
    (a, ma), (b, mb) = outs[sb.OF_FP64], outs[sb.OF_MIXED]
    assert mb["pressure_relative_residual"] <= 1e-12
    ref = oracle.tg_steps(cfg, 8, s0.copy())
    for name in ("u", "v", "w"):
        assert rel_maxdiff(b[name], a[name]) <= 1e-9, name
        assert rel_maxdiff(b[name], getattr(ref, name)) <= 1e-9, name


def _host_state(st, pinned):
    import torch
    out = {}
    for name in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p"):
        a = np.ascontiguousarray(getattr(st, name) if not isinstance(st, dict) else st[name])
        if pinned:
            t = torch.empty(a.shape, dtype=torch.float64, pin_memory=True)
            t.numpy()[...] = a
            out[name] = t.numpy()
            out["_keep_" + name] = t
        else:
            out[name] = a.copy()
    return out


@pytest.mark.parametrize("pinned", [False, True])
def test_step_host_equals_upload_step_download(sb, oracle, pinned):
    """of_step_host (one call per step on host arrays; with pinned arrays the
    AB2 history comes back while the pressure solve runs) gives bitwise the
    state of of_state_upload + of_run_steps(1) + of_state_download."""
    cfg = po.steps_config(32, 32, 16, 0.01, 0.5, 4, 1e-12)
    g = oracle.tg_grid(cfg)
    s0 = oracle.tg_init(cfg, 0)
    prm = sb.step_params(cfg.viscosity, oracle.tg_dt(cfg), cfg.poisson_max_iterations,
                         cfg.poisson_tolerance)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(oracle.tg_bc(cfg)))
    host = _host_state(s0, pinned)
    host["has_previous_advection"] = 0
    host["metrics"] = dict(s0.metrics)
    ref = {k: getattr(s0, k).copy() for k in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")}
    ref_hp, ref_m = 0, dict(s0.metrics)
    ctx2 = sb.Context(to_gpu_grid(g), to_gpu_bc(oracle.tg_bc(cfg)))
    for _ in range(4):
        m = ctx.step_host(prm, host)
        ctx2.upload_state(ref["u"], ref["v"], ref["w"], ref["adv_u"], ref["adv_v"], ref["adv_w"],
                          ref["p"], ref_hp, ref_m)
        ref_m = ctx2.run_steps(prm, 1)
        st = ctx2.download_state()
        ref = {k: st[k] for k in ref}
        ref_hp = st["has_previous_advection"]
        for name in ref:
            assert np.array_equal(host[name], ref[name]), name
        assert host["has_previous_advection"] == ref_hp == 1
        assert m == ref_m
    assert m["step"] == 4


def test_step_host_failure_leaves_host_state_unchanged(sb, oracle):
    """A failed step (one CG iteration at tolerance 1e-30) raises like
    of_run_steps and leaves every host array -- the pinned AB2 history that
    was being copied back during the step included -- as it was passed in."""
    cfg = po.steps_config(32, 32, 16, 0.01, 0.5, 2, 1e-12)
    g = oracle.tg_grid(cfg)
    s0 = oracle.tg_init(cfg, 0)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(oracle.tg_bc(cfg)))
    host = _host_state(s0, True)
    host["has_previous_advection"] = 0
    host["metrics"] = dict(s0.metrics)
    dt = oracle.tg_dt(cfg)
    ctx.step_host(sb.step_params(cfg.viscosity, dt, cfg.poisson_max_iterations, 1e-12), host)
    before = {k: host[k].copy() for k in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")}
    assert np.abs(before["adv_u"]).max() > 0
    with pytest.raises(sb.NotConvergedError,
                       match="Taylor-Green pressure solve did not converge at step 2"):
        ctx.step_host(sb.step_params(cfg.viscosity, dt, 1, 1e-30), host)
    for name, a in before.items():
        assert np.array_equal(host[name], a), name
    assert host["has_previous_advection"] == 1
    assert host["metrics"]["step"] == 1
