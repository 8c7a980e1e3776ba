"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs the reference's own C++ sources, compiled in place from the reference
tree by ``make -C oracle ref`` (oracle/_ref/liborchard_ref.so), on small
seeded inputs and stores inputs and outputs as .npz files.  The fixtures pin
the plain-C oracle (bit for bit) and the GPU path (within the parity
tolerance) on machines where the reference tree is absent.

Usage:  make -C oracle ref && python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402


def save(name, **arrays):
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **arrays)


def state_arrays(prefix, s):
    out = {f"{prefix}_{n}": getattr(s, n) for n in po.FIELDS}
    out[f"{prefix}_has_prev"] = np.array(s.has_previous_advection)
    for k, v in s.metrics.items():
        out[f"{prefix}_m_{k}"] = np.array(v)
    return out


def main():
    ref = po.Oracle(po.REF_SO)
    rng = np.random.default_rng(20261203)
    meta = {}

    # Taylor-Green steps from the reference's own initial state
    for name, n, steps in (("tg2d_16", (16, 16, 1), 3), ("tg3d_8", (8, 8, 8), 2)):
        cfg = po.steps_config(*n, 0.01, 0.5, steps, 1e-12)
        s0 = ref.tg_init(cfg, 0)
        s1 = ref.tg_steps(cfg, steps, s0.copy())
        cfg_arr = np.array([cfg.nx, cfg.ny, cfg.nz, cfg.viscosity, cfg.cfl_limit, cfg.final_time,
                            cfg.poisson_max_iterations, cfg.poisson_tolerance])
        save(name, config=cfg_arr, steps=np.array(steps), **state_arrays("in", s0),
             **state_arrays("out", s1))
        meta[name] = {"steps": steps, "pressure_iterations": s1.metrics["pressure_iterations"]}

    # lid-driven cavity steps
    cc = po.cavity_config(16, 16, poisson_tolerance=1e-12)
    s0 = ref.cavity_init(cc)
    s1 = ref.cavity_steps(cc, 4, s0.copy())
    save("cavity_16", steps=np.array(4), **state_arrays("in", s0), **state_arrays("out", s1))
    meta["cavity_16"] = {"steps": 4, "pressure_iterations": s1.metrics["pressure_iterations"]}

    # Poisson solves
    cases = {
        "poisson_dirichlet_8": (po.Grid(8, 8, 1, 0.125, 0.125, 1.0),
                                po.pbc_from([po.P_DIRICHLET] * 4 + [po.P_NEUMANN] * 2,
                                            values=[0.3, -0.1, 0.2, 0.0, 0.0, 0.0])),
        "poisson_neumann_864": (po.Grid(8, 6, 4, 0.1, 0.2, 0.3),
                                po.pbc_from([po.P_NEUMANN] * 6,
                                            gradients=[0.1, 0.1, -0.2, -0.2, 0.0, 0.0])),
        "poisson_periodic_8": (po.Grid(8, 8, 8, 0.4, 0.4, 0.4), po.pbc_from([po.P_PERIODIC] * 6)),
    }
    for name, (g, pbc) in cases.items():
        rhs = rng.standard_normal(po.shape(g, "p"))
        p = np.zeros(po.shape(g, "p"))
        d, hist = ref.poisson_solve(g, pbc, 200, 1e-12, rhs, p)
        save(name, grid=np.array([g.nx, g.ny, g.nz, g.dx, g.dy, g.dz]),
             pbc=np.array([[pbc.faces[f].type, pbc.faces[f].value, pbc.faces[f].gradient]
                           for f in range(6)]), rhs=rhs, pressure=p, history=hist,
             iterations=np.array(d.iterations), levels=np.array(d.multigrid_levels))
        meta[name] = {"iterations": d.iterations, "levels": d.multigrid_levels}

    # ADI predictor with walls, advection, projection
    g = po.Grid(6, 5, 4, 0.2, 0.3, 0.25)
    types = [po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.PRESCRIBED_VELOCITY,
             po.SYMMETRY, po.SYMMETRY]
    bc = po.bc_from(types, [None, None, None, (0.7, 0.0, 0.1), None, None])
    rhs = [rng.standard_normal(po.shape(g, c)) for c in "uvw"]
    out, lines = ref.predictor_adi(g, bc, 0.05, *rhs)
    save("adi_walls", grid=np.array([g.nx, g.ny, g.nz, g.dx, g.dy, g.dz]), types=np.array(types),
         alpha=np.array(0.05), rhs_u=rhs[0], rhs_v=rhs[1], rhs_w=rhs[2], out_u=out[0],
         out_v=out[1], out_w=out[2], lines=np.array(lines))
    vel = [rng.standard_normal(po.shape(g, c)) for c in "uvw"]
    adv = ref.advection(g, *vel)
    save("advection", grid=np.array([g.nx, g.ny, g.nz, g.dx, g.dy, g.dz]), u=vel[0], v=vel[1],
         w=vel[2], au=adv[0], av=adv[1], aw=adv[2])
    gp = po.Grid(8, 6, 4, 0.2, 0.25, 0.3)
    pred = [rng.standard_normal(po.shape(gp, c)) for c in "uvw"]
    phi = np.zeros(po.shape(gp, "p"))
    corr, prhs, d = ref.project_velocity(gp, po.periodic_bc(), 0.01, 1.0, 200, 1e-12, *pred, phi)
    save("projection_periodic", grid=np.array([gp.nx, gp.ny, gp.nz, gp.dx, gp.dy, gp.dz]),
         pu=pred[0], pv=pred[1], pw=pred[2], cu=corr[0], cv=corr[1], cw=corr[2], phi=phi,
         rhs=prhs, iterations=np.array(d.pressure_solve.iterations))

    with open(os.path.join(HERE, "manifest.json"), "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py",
                   "source": "the reference's C++ sources compiled in place (oracle/_ref)",
                   "cases": meta}, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
