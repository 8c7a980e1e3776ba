"""The reference's own unit tests, run through the B200 bodies of its seams.

`make -C oracle binding` (run by __graft_entry__.build() where the reference
tree is present) links solver_b200/binding/projection_b200.cpp -- the file a
maintainer adds to the reference tree -- over the reference's own objects,
whose CPU bodies of project_velocity, solve_predictor_adi,
linsolve::solve_pressure_poisson and compute_advection_term are made weak, so
that every call of those four (from the tests and from the reference's case
drivers alike) goes through the C ABI to the GPU.  The tests themselves are
the reference's tests/test_runtime.cpp functions, unchanged, run one by one
(oracle/binding_tests_main.inc).  Among them the MG-PCG Dirichlet and
pure-Neumann recovery tests (tests/test_runtime.cpp:1178-1285), the ADI
against the dense factorised operator (:1009-1056), the quiescent and
pure-Neumann projections (:1447-1539) and the non-convergence message
(:1777-1792).
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "solver_tests_b200")

TESTS = [
    "test_predictor_adi_preserves_quiescent_state",
    "test_predictor_adi_preserves_periodic_couette_state",
    "test_predictor_adi_matches_factorized_dense_reference",
    "test_lid_driven_cavity_predictor_rhs_matches_manual_formula",
    "test_poisson_mgpcg_discrete_dirichlet_recovery",
    "test_poisson_mgpcg_pure_neumann_zero_mean_recovery",
    "test_diffusion_term_matches_scaled_laplacian",
    "test_taylor_green_step_behavior",
    "test_bounded_advection_regression_case",
    "test_static_projection_preserves_quiescent_fluid",
    "test_pure_neumann_projection_recovers_zero_mean_pressure",
    "test_taylor_green_smoke_validation",
    "test_taylor_green_3d_smoke_validation",
    "test_taylor_green_rejects_nonconverged_pressure_projection",
    "test_channel_flow_couette_profile_validation",
    "test_channel_flow_poiseuille_profile_validation",
    "test_channel_flow_rejects_nonconverged_pressure_projection",
    "test_lid_driven_cavity_rejects_nonconverged_pressure_projection",
    "test_lid_driven_cavity_restart_is_bitwise_deterministic",
    "test_lid_driven_cavity_smoke_run",
    "test_lid_driven_cavity_reference_validation_gate",
]

needs_binary = pytest.mark.skipif(not os.path.exists(BIN),
                                  reason="binding test binary not built (needs the reference tree)")


@needs_binary
def test_binary_binds_the_b200_seam_bodies():
    """The four seam functions of the linked binary are the binding's (the
    reference's own definitions were weak and dropped) and it loads the
    in-tree CUDA library."""
    syms = subprocess.run(["nm", "-C", BIN], capture_output=True, text=True, check=True).stdout
    assert "solver::b200_binding::context_for(" in syms
    for seam in ("solver::project_velocity(", "solver::solve_predictor_adi(",
                 "solver::linsolve::solve_pressure_poisson(", "solver::compute_advection_term("):
        defs = [line for line in syms.splitlines() if f" T {seam}" in line]
        assert len(defs) == 1, (seam, defs)
    libs = subprocess.run(["ldd", BIN], capture_output=True, text=True, check=True).stdout
    assert os.path.join("solver_b200", "liborchard_b200.so") in libs or "liborchard_b200.so" in libs


@pytest.fixture(scope="module")
def binding_run():
    env = dict(os.environ, ORCHARD_B200_BINDING_VERBOSE="1")
    p = subprocess.run([BIN] + TESTS, capture_output=True, text=True, env=env, timeout=1200)
    results = {}
    for line in p.stdout.splitlines():
        kind, _, rest = line.partition(" ")
        name = rest.split(":", 1)[0]
        results[name] = (kind, line)
    return results, p.stderr


@needs_binary
@pytest.mark.gpu
@pytest.mark.parametrize("name", TESTS)
def test_reference_test_passes_through_b200_binding(binding_run, name):
    results, stderr = binding_run
    assert "b200 binding: context on CUDA device 0" in stderr
    kind, line = results.get(name, ("MISSING", name))
    assert kind == "PASS", line
