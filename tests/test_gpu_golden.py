"""GPU path against the golden fixtures generated by the reference's own
sources (tests/golden/make_golden.py), through the C ABI.  FP64 tolerance:
max-norm relative difference <= 1e-11 after the recorded steps."""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_maxdiff, to_gpu_bc, to_gpu_grid
from test_oracle import grid_of, load

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sb():
    import solver_b200
    return solver_b200


@pytest.mark.parametrize("name", ["tg2d_16", "tg3d_8"])
def test_gpu_taylor_green_matches_golden(sb, oracle, name):
    d = load(name)
    c = d["config"]
    cfg = po.tg_config(int(c[0]), int(c[1]), int(c[2]), c[3], c[4], c[5], int(c[6]), c[7])
    g = oracle.tg_grid(cfg)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(oracle.tg_bc(cfg)))
    ctx.upload_state(*(d[f"in_{n}"] for n in po.FIELDS), 0, None)
    m = ctx.run_steps(sb.step_params(cfg.viscosity, oracle.tg_dt(cfg), cfg.poisson_max_iterations,
                                     cfg.poisson_tolerance), int(d["steps"]))
    out = ctx.download_state()
    for n in ("u", "v", "w", "p", "adv_u", "adv_v", "adv_w"):
        assert rel_maxdiff(out[n], d[f"out_{n}"]) <= 1e-11, n
    assert m["pressure_iterations"] == int(d["out_m_pressure_iterations"])


def test_gpu_cavity_matches_golden(sb, oracle):
    d = load("cavity_16")
    cc = po.cavity_config(16, 16, poisson_tolerance=1e-12)
    g = oracle.cavity_grid(cc)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(oracle.cavity_bc(cc)))
    ctx.upload_state(*(d[f"in_{n}"] for n in po.FIELDS), 0, None)
    prm = sb.step_params(cc.lid_velocity / cc.reynolds, oracle.cavity_dt(cc),
                         cc.poisson_max_iterations, cc.poisson_tolerance,
                         variant=sb.OF_CORRECTION_CAVITY)
    m = ctx.run_steps(prm, int(d["steps"]))
    out = ctx.download_state()
    for n in ("u", "v", "p"):
        assert rel_maxdiff(out[n], d[f"out_{n}"]) <= 1e-11, n
    assert m["pressure_iterations"] == int(d["out_m_pressure_iterations"])


@pytest.mark.parametrize("name", ["poisson_dirichlet_8", "poisson_neumann_864", "poisson_periodic_8"])
def test_gpu_poisson_matches_golden(sb, name):
    d = load(name)
    g = grid_of(d["grid"])
    pb = d["pbc"]
    pbc = [(int(pb[f, 0]), float(pb[f, 1]), float(pb[f, 2])) for f in range(6)]
    ctx = sb.Context(to_gpu_grid(g), [sb.PERIODIC] * 6)
    p, diag = ctx.solve_pressure_poisson(d["rhs"], pbc, 200, 1e-12)
    assert diag["iterations"] == int(d["iterations"])
    assert diag["multigrid_levels"] == int(d["levels"])
    assert rel_maxdiff(p, d["pressure"]) <= 1e-11
