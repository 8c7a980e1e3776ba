"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The CPU oracle (oracle/liborchard_oracle.so, a plain-C restatement of the
reference) is the checker for every parity test; oracle/_ref/liborchard_ref.so
(the reference's own sources compiled in place) pins the oracle when present.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import pyoracle  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def _ensure_oracle_built():
    if not os.path.exists(pyoracle.ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])


@pytest.fixture(scope="session")
def oracle():
    _ensure_oracle_built()
    return pyoracle.Oracle(pyoracle.ORACLE_SO)


@pytest.fixture(scope="session")
def ref():
    if not os.path.exists(pyoracle.REF_SO):
        pytest.skip("reference build (oracle/_ref) not present")
    return pyoracle.Oracle(pyoracle.REF_SO)


def rel_maxdiff(a, b):
    """Max-norm relative difference over active entries: max|a-b| / max|b|."""
    a = pyoracle.active(np.asarray(a))
    b = pyoracle.active(np.asarray(b))
    scale = np.max(np.abs(b))
    d = np.max(np.abs(a - b))
    return d / scale if scale > 0 else d


def to_gpu_bc(bc):
    """pyoracle.BC -> solver_b200 boundary spec."""
    return [(bc.faces[f].type, tuple(bc.faces[f].velocity), bc.faces[f].pressure) for f in range(6)]


def to_gpu_pbc(pbc):
    return [(pbc.faces[f].type, pbc.faces[f].value, pbc.faces[f].gradient) for f in range(6)]


def to_gpu_grid(g):
    import solver_b200
    return solver_b200.Grid(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz)
