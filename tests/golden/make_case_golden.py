"""Generates the case-layer golden fixtures in tests/golden/cases/ from the
reference itself (its sources compiled in place by ``make -C oracle ref``).

* ``tg2d_32.cfg`` / ``cavity_32.cfg``: config files of our own in the
  reference's ``key = value`` format, and ``ref_cli_*.txt``: the reports the
  reference's CLIs (tools/taylor_green_main.cpp, tools/lid_driven_cavity_main.cpp)
  print for them.
* ``cavity_24.chk``: an SLVCHKP1 checkpoint written by the reference's
  write_lid_driven_cavity_checkpoint of a 24x24 cavity state after 7 steps,
  ``cavity_24.npz`` the same state as arrays, ``cavity_24.json`` the
  reference's build description, checkpoint hashes and finalize outputs on
  that state, and ``cavity_24.vtk`` the reference's write_mac_fields_vtk of it.

* ``ref_cli_cavity_128_steady.txt`` (only with ``--with-steady``, about a
  quarter of an hour of CPU): the reference's ``solver_cavity`` report for
  the shipped config solver_b200/configs/lid_driven_cavity_re100_128.cfg,
  marched to the steady state.

Usage:  make -C oracle ref && python tests/golden/make_case_golden.py [--with-steady]
"""
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "cases")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import pyoracle as po  # noqa: E402

TG_CFG = """# Taylor-Green vortex, 2D 32x32, a short decay run
nx = 32
ny = 32
nz = 1
viscosity = 0.01
cfl_limit = 0.25
final_time = 0.25
poisson_max_iterations = 200
poisson_tolerance = 1e-10
validate_energy = true
"""

CAVITY_CFG = """# lid-driven cavity, Re 100 on 32x32
nx = 32
ny = 32
reynolds = 100
lid_velocity = 1.0
cfl_limit = 0.5
max_steps = 400
min_steps = 50
steady_tolerance = 1e-7
poisson_max_iterations = 200
poisson_tolerance = 1e-10
validate_reference = true
"""

CAVITY_STEPS = 60


def run_cli(binary, *args, cwd=OUT):
    p = subprocess.run([os.path.join(ROOT, "oracle", "_ref", binary), *args], capture_output=True,
                       text=True, cwd=cwd)
    return p.stdout


def main():
    os.makedirs(OUT, exist_ok=True)
    with open(os.path.join(OUT, "tg2d_32.cfg"), "w") as f:
        f.write(TG_CFG)
    with open(os.path.join(OUT, "cavity_32.cfg"), "w") as f:
        f.write(CAVITY_CFG)
    with open(os.path.join(OUT, "ref_cli_tg2d_32.txt"), "w") as f:
        f.write(run_cli("solver_taylor_green", "tg2d_32.cfg"))
    with open(os.path.join(OUT, f"ref_cli_cavity_32_steps{CAVITY_STEPS}.txt"), "w") as f:
        f.write(run_cli("solver_cavity", "cavity_32.cfg", "--steps", str(CAVITY_STEPS)))

    ref = po.ReferenceIO()
    cc = po.cavity_config(24, 24, max_steps=500, min_steps=20, steady_tolerance=1e-7,
                          poisson_tolerance=1e-12)
    s = ref.cavity_steps(cc, 7, ref.cavity_init(cc))
    chk = os.path.join(OUT, "cavity_24.chk")
    ref.cavity_checkpoint_write(chk, cc, True, s)
    _, meta = ref.cavity_checkpoint_load(chk, cc, True)
    fin = ref.cavity_finalize(cc, True, s)
    ref.write_vtk(os.path.join(OUT, "cavity_24.vtk"), ref.cavity_grid(cc), s)
    np.savez_compressed(os.path.join(OUT, "cavity_24.npz"),
                        **{n: getattr(s, n) for n in po.FIELDS},
                        has_prev=np.array(s.has_previous_advection))
    info = {
        "config": {k: getattr(cc, k) for k, _ in po.CavityConfig._fields_},
        "validate_reference": True,
        "metrics": s.metrics,
        "build_description": ref.build_description(),
        "checksum": str(meta["checksum"]),
        "build_hash": str(meta["build_hash"]),
        "configuration_hash": str(meta["configuration_hash"]),
        "finalize": {k: (v.hex() if isinstance(v, float) else
                         [x.hex() for x in v] if isinstance(v, list) else v)
                     for k, v in fin.items()},
    }
    with open(os.path.join(OUT, "cavity_24.json"), "w") as f:
        json.dump(info, f, indent=1, sort_keys=True)
    if "--with-steady" in sys.argv:
        report = run_cli("solver_cavity", os.path.join("solver_b200", "configs",
                                                       "lid_driven_cavity_re100_128.cfg"), cwd=ROOT)
        with open(os.path.join(OUT, "ref_cli_cavity_128_steady.txt"), "w") as f:
            f.write(report)
    print("wrote", sorted(os.listdir(OUT)))


if __name__ == "__main__":
    main()
