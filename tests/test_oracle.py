"""The CPU oracle (plain-C restatement) pinned against the reference.

Three independent pins: (1) the golden fixtures generated by the reference's
own sources (tests/golden/make_golden.py), bit for bit; (2) the reference
build itself when oracle/_ref is present, bit for bit; (3) the reference's
published validation numbers for Taylor-Green 2D 128^2
(validation/latest/benchmark_summary.csv:5, taylor_green_temporal.csv:4).
"""
import glob
import math
import os

import numpy as np
import pytest

import pyoracle as po

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def state_from(d, prefix):
    s = po.State(*(d[f"{prefix}_{n}"].copy() for n in po.FIELDS))
    s.has_previous_advection = int(d[f"{prefix}_has_prev"])
    s.metrics = {k[len(prefix) + 3:]: d[k].item() for k in d if k.startswith(prefix + "_m_")}
    return s


def grid_of(a):
    return po.Grid(int(a[0]), int(a[1]), int(a[2]), float(a[3]), float(a[4]), float(a[5]))


def assert_state_equal(s, d, prefix):
    for n in po.FIELDS:
        assert np.array_equal(getattr(s, n), d[f"{prefix}_{n}"]), n
    for k, v in s.metrics.items():
        assert v == d[f"{prefix}_m_{k}"].item(), k


@pytest.mark.parametrize("name", ["tg2d_16", "tg3d_8"])
def test_oracle_taylor_green_matches_golden(oracle, name):
    d = load(name)
    c = d["config"]
    cfg = po.tg_config(int(c[0]), int(c[1]), int(c[2]), c[3], c[4], c[5], int(c[6]), c[7])
    s0 = oracle.tg_init(cfg, 0)
    assert_state_equal(s0, d, "in")
    s1 = oracle.tg_steps(cfg, int(d["steps"]), s0)
    assert_state_equal(s1, d, "out")


def test_oracle_cavity_matches_golden(oracle):
    d = load("cavity_16")
    cc = po.cavity_config(16, 16, poisson_tolerance=1e-12)
    s0 = oracle.cavity_init(cc)
    assert_state_equal(s0, d, "in")
    s1 = oracle.cavity_steps(cc, int(d["steps"]), s0)
    assert_state_equal(s1, d, "out")


@pytest.mark.parametrize("name", ["poisson_dirichlet_8", "poisson_neumann_864", "poisson_periodic_8"])
def test_oracle_poisson_matches_golden(oracle, name):
    d = load(name)
    g = grid_of(d["grid"])
    pb = d["pbc"]
    pbc = po.pbc_from([int(x) for x in pb[:, 0]], list(pb[:, 1]), list(pb[:, 2]))
    p = np.zeros(po.shape(g, "p"))
    diag, hist = oracle.poisson_solve(g, pbc, 200, 1e-12, d["rhs"], p)
    assert diag.iterations == int(d["iterations"])
    assert diag.multigrid_levels == int(d["levels"])
    assert np.array_equal(p, d["pressure"])
    assert np.array_equal(hist, d["history"])


def test_oracle_adi_advection_projection_match_golden(oracle):
    d = load("adi_walls")
    g = grid_of(d["grid"])
    vel = [None] * 6
    vel[3] = (0.7, 0.0, 0.1)
    bc = po.bc_from([int(t) for t in d["types"]], vel)
    out, lines = oracle.predictor_adi(g, bc, float(d["alpha"]), d["rhs_u"], d["rhs_v"], d["rhs_w"])
    assert lines == int(d["lines"])
    for a, c in zip(out, "uvw"):
        assert np.array_equal(a, d[f"out_{c}"])
    d = load("advection")
    g = grid_of(d["grid"])
    for a, c in zip(oracle.advection(g, d["u"], d["v"], d["w"]), "uvw"):
        assert np.array_equal(a, d[f"a{c}"])
    d = load("projection_periodic")
    g = grid_of(d["grid"])
    corr, rhs, diag = oracle.project_velocity(g, po.periodic_bc(), 0.01, 1.0, 200, 1e-12,
                                              d["pu"], d["pv"], d["pw"], np.zeros(po.shape(g, "p")))
    for a, c in zip(corr, "uvw"):
        assert np.array_equal(a, d[f"c{c}"])
    assert np.array_equal(rhs, d["rhs"])
    assert diag.pressure_solve.iterations == int(d["iterations"])


def test_oracle_reproduces_published_taylor_green_128(oracle):
    # benchmarks/taylor_green_128.cfg: nx=ny=128, nu=0.01, CFL 0.25, T=0.25, tol 1e-10
    cfg = po.tg_config(128, 128, 1, 0.01, 0.25, 0.25, 200, 1e-10)
    s = oracle.tg_init(cfg, 0)
    steps = math.ceil(cfg.final_time / oracle.tg_dt(cfg))
    s = oracle.tg_steps(cfg, steps, s)
    v = oracle.tg_validate(cfg, s, s.metrics["time"])
    assert s.metrics["step"] == 41
    assert f"{v['normalized_energy_error']:.5e}" == "7.01798e-04"
    assert f"{v['velocity_relative_l2_error']:.5e}" == "2.58575e-03"
    assert s.metrics["divergence_l2"] <= 1e-10


def test_oracle_bitwise_equal_to_reference_build(oracle, ref):
    rng = np.random.default_rng(7)
    for n, steps in (((12, 10, 1), 3), ((8, 6, 6), 2)):
        cfg = po.steps_config(*n, 0.02, 0.5, steps, 1e-12)
        s_ref = ref.tg_init(cfg, 0)
        # perturb the state so that every branch of the limiter is exercised
        for name in ("u", "v"):
            po.active(getattr(s_ref, name))[...] += 0.05 * rng.standard_normal(
                po.active(getattr(s_ref, name)).shape)
        s_ref = ref.tg_init_tail(cfg, s_ref)
        s_ora = s_ref.copy()
        ref.tg_steps(cfg, steps, s_ref)
        oracle.tg_steps(cfg, steps, s_ora)
        for name in po.FIELDS:
            assert np.array_equal(getattr(s_ref, name), getattr(s_ora, name)), name
        assert s_ref.metrics == s_ora.metrics


def test_oracle_rejects_nonconverged_pressure_projection(oracle):
    # tests/test_runtime.cpp:1777-1792: poisson_max_iterations=1, tolerance=1e-30
    cfg = po.tg_config(16, 16, 1, 0.01, 0.25, 0.01, 1, 1e-30)
    s = oracle.tg_init(cfg, 0)
    with pytest.raises(po.OracleError, match="Taylor-Green pressure solve did not converge"):
        oracle.tg_steps(cfg, 1, s)


def test_golden_manifest_lists_every_fixture():
    import json
    with open(os.path.join(GOLDEN, "manifest.json")) as f:
        m = json.load(f)
    names = {os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))}
    assert set(m["cases"]) <= names
