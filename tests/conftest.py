"""Shared fixtures.  GPU tests are marked ``gpu``; everything else runs on CPU.

The CPU oracle (oracle/liborchard_oracle.so, a plain-C restatement of the
reference) is the checker for every parity test; oracle/_ref/liborchard_ref.so
(the reference's own sources compiled in place) pins the oracle when present.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import pyoracle  # noqa: E402

# Background reference runs (tests/refjob.py): name -> (process, outdir, log file)
_JOBS = {}


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "refjob(name): needs the result of a long CPU reference "
                                       "run (tests/refjob.py), started at the session's start")


def pytest_collection_finish(session):
    """Start, one process each, the reference runs the selected tests need, so
    they run on host cores while the GPU tests before them run."""
    names = sorted({n for it in session.items for m in it.iter_markers("refjob") for n in m.args})
    if not names or not os.path.exists(pyoracle.REF_SO):
        return
    outdir = tempfile.mkdtemp(prefix="orchard_refjobs_")
    for name in names:
        log = open(os.path.join(outdir, name + ".log"), "w")
        proc = subprocess.Popen([sys.executable, os.path.join(HERE, "refjob.py"), name, outdir],
                                stdout=log, stderr=subprocess.STDOUT)
        _JOBS[name] = (proc, outdir, log)


def pytest_sessionfinish(session, exitstatus):
    import shutil
    for proc, outdir, log in _JOBS.values():
        if proc.poll() is None:
            proc.kill()
            proc.wait()
        log.close()
    for outdir in {v[1] for v in _JOBS.values()}:
        shutil.rmtree(outdir, ignore_errors=True)


@pytest.fixture(scope="session")
def refjob_result():
    """refjob_result(name) -> the state a background reference run ended with
    (waits for it): dict of padded fields, 'metrics' and 'wall' seconds."""
    import json

    def get(name, timeout=1800):
        if name not in _JOBS:
            pytest.skip("reference build (oracle/_ref) not present")
        proc, outdir, _ = _JOBS[name]
        rc = proc.wait(timeout=timeout)
        if rc != 0:
            with open(os.path.join(outdir, name + ".log")) as f:
                pytest.fail(f"reference run {name} failed (rc {rc}):\n{f.read()[-3000:]}")
        with np.load(os.path.join(outdir, name + ".npz")) as z:
            out = {k: z[k] for k in z.files}
        out["metrics"] = json.loads(str(out["metrics"]))
        out["wall"] = float(out["wall"])
        return out

    return get


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
