"""Long CPU reference runs for the GPU parity tests at the bench's sizes.

TEST INFRASTRUCTURE ONLY.  The reference build (oracle/_ref/liborchard_ref.so,
the reference's own C++ sources compiled in place) needs minutes for one
256^3 step on one core, so ``tests/conftest.py`` starts every job that the
selected tests need as its own process at the start of the session (one core
each, next to the GPU tests), and the tests wait for the result files.

Each job runs the reference's own initial state and ``run_taylor_green_steps``
/ ``run_lid_driven_cavity_steps`` (solver/taylor_green.cpp:540-634,
solver/lid_driven_cavity.cpp:562-623) and writes the state after its steps
to ``<outdir>/<name>.npz`` (padded fields, metrics, wall time), then
``<name>.done``.

    python tests/refjob.py <name> <outdir>
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))

import numpy as np  # noqa: E402

import pyoracle as po  # noqa: E402

# name -> (kind, grid, physics, steps).  Taylor-Green: (nx, ny, nz), viscosity,
# CFL, Poisson tolerance; cavity: (nx, ny), Poisson tolerance.
JOBS = {
    # 3D Taylor-Green at Re 1600 (viscosity 1/1600), CFL 0.5, tolerance 1e-12:
    # the headline workload's physics at 128^3 and at its own 256^3
    "tg3d_128_3": ("tg", (128, 128, 128), (1.0 / 1600.0, 0.5, 1e-12), 3),
    "tg3d_256_2": ("tg", (256, 256, 256), (1.0 / 1600.0, 0.5, 1e-12), 2),
    # Re 100 lid-driven cavity at 1024^2 with the shipped config's Poisson
    # tolerance (1e-8), its first 20 steps
    "cavity_1024_20": ("cavity", (1024, 1024), (1e-8,), 20),
}


def config(name):
    kind, n, phys, steps = JOBS[name]
    if kind == "tg":
        nu, cfl, tol = phys
        return po.steps_config(*n, nu, cfl, steps, tol)
    return po.cavity_config(n[0], n[1], reynolds=100.0, lid_velocity=1.0, cfl_limit=0.5,
                            max_steps=1000000, min_steps=1, steady_tolerance=1e-8,
                            poisson_max_iterations=400, poisson_tolerance=phys[0])


def initial_state(lib, name):
    kind = JOBS[name][0]
    cfg = config(name)
    return lib.tg_init(cfg, 0) if kind == "tg" else lib.cavity_init(cfg)


def run(name, outdir):
    kind, _, _, steps = JOBS[name]
    ref = po.Oracle(po.REF_SO)
    cfg = config(name)
    s = initial_state(ref, name)
    t0 = time.time()
    s = ref.tg_steps(cfg, steps, s) if kind == "tg" else ref.cavity_steps(cfg, steps, s)
    wall = time.time() - t0
    tmp = os.path.join(outdir, name + ".tmp.npz")
    np.savez(tmp, **{f: getattr(s, f) for f in po.FIELDS},
             has_previous_advection=s.has_previous_advection,
             metrics=json.dumps(s.metrics), wall=wall)
    os.replace(tmp, os.path.join(outdir, name + ".npz"))
    with open(os.path.join(outdir, name + ".done"), "w") as f:
        f.write(f"{wall:.1f}\n")


if __name__ == "__main__":
    run(sys.argv[1], sys.argv[2])
