"""ctypes view of the CPU oracle interface (oracle/orchard_oracle.h).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()``
and the ``cpu_baseline`` leg of ``bench.py`` as the checker; the product
package ``solver_b200`` never imports it.

Two libraries export the interface:

* ``oracle/liborchard_oracle.so`` -- the plain-C restatement (the oracle);
* ``oracle/_ref/liborchard_ref.so`` -- the reference's own C++ sources compiled
  in place (present only where the reference tree was available at build time).

Arrays are numpy float64 in the reference's padded MAC storage, shaped
``(sz, sy, sx)`` so that ``a[k, j, i]`` is the reference's ``field(i, j, k)``
(core/field_layout.hpp:178-183).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liborchard_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "liborchard_ref.so")

# PhysicalBoundaryType / PressureBoundaryType (bc/boundary_conditions.hpp:10-22)
NO_SLIP_WALL, PRESCRIBED_VELOCITY, SYMMETRY, FIXED_PRESSURE, PERIODIC = range(5)
P_NEUMANN, P_DIRICHLET, P_PERIODIC = range(3)


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class FaceBC(C.Structure):
    _fields_ = [("type", C.c_int), ("velocity", C.c_double * 3), ("pressure", C.c_double),
                ("pressure_gradient", C.c_double)]


class BC(C.Structure):
    _fields_ = [("faces", FaceBC * 6)]


class PFaceBC(C.Structure):
    _fields_ = [("type", C.c_int), ("value", C.c_double), ("gradient", C.c_double)]


class PBC(C.Structure):
    _fields_ = [("faces", PFaceBC * 6)]


class PoissonDiag(C.Structure):
    _fields_ = [("iterations", C.c_int), ("initial_residual_l2", C.c_double),
                ("final_residual_l2", C.c_double), ("relative_residual", C.c_double),
                ("removed_rhs_mean", C.c_double), ("multigrid_levels", C.c_int),
                ("coarse_unknowns", C.c_int), ("pre_smoothing_steps", C.c_int),
                ("post_smoothing_steps", C.c_int), ("converged", C.c_int),
                ("zero_mean_enforced", C.c_int)]


class ProjectionDiag(C.Structure):
    _fields_ = [("rhs_l2", C.c_double), ("divergence_l2_before", C.c_double),
                ("divergence_l2_after", C.c_double), ("pressure_mean", C.c_double),
                ("pressure_solve", PoissonDiag)]


class StepMetrics(C.Structure):
    _fields_ = [("step", C.c_int), ("time", C.c_double), ("dt", C.c_double),
                ("max_cfl", C.c_double), ("max_velocity_change", C.c_double),
                ("divergence_l2", C.c_double), ("max_divergence_l2", C.c_double),
                ("pressure_iterations", C.c_int), ("pressure_relative_residual", C.c_double)]


class TGConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("viscosity", C.c_double),
                ("cfl_limit", C.c_double), ("final_time", C.c_double),
                ("poisson_max_iterations", C.c_int), ("poisson_tolerance", C.c_double)]


class TGValidation(C.Structure):
    _fields_ = [("kinetic_energy", C.c_double), ("exact_kinetic_energy", C.c_double),
                ("normalized_energy_error", C.c_double),
                ("velocity_relative_l2_error", C.c_double)]


class CavityConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("reynolds", C.c_double),
                ("lid_velocity", C.c_double), ("cfl_limit", C.c_double), ("max_steps", C.c_int),
                ("min_steps", C.c_int), ("steady_tolerance", C.c_double),
                ("poisson_max_iterations", C.c_int), ("poisson_tolerance", C.c_double)]


DP = C.POINTER(C.c_double)


class CState(C.Structure):
    _fields_ = [("u", DP), ("v", DP), ("w", DP), ("adv_u", DP), ("adv_v", DP), ("adv_w", DP),
                ("p", DP), ("has_previous_advection", C.c_int), ("metrics", StepMetrics)]


def shape(grid, loc):
    """Storage shape (sz, sy, sx) of a field at location loc: 'p', 'u', 'v' or 'w'."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    ext = {"p": (nx, ny, nz), "u": (nx + 1, ny, nz), "v": (nx, ny + 1, nz),
           "w": (nx, ny, nz + 1)}[loc]
    return (ext[2] + 2, ext[1] + 2, ext[0] + 2)


def active(a):
    """Active (non-ghost) view of a padded array."""
    return a[1:-1, 1:-1, 1:-1]


def zeros(grid, loc):
    return np.zeros(shape(grid, loc), dtype=np.float64)


def ptr(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(DP)


@dataclass
class State:
    """A Taylor-Green / cavity state: padded velocity, AB2 history and total pressure."""
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    adv_u: np.ndarray
    adv_v: np.ndarray
    adv_w: np.ndarray
    p: np.ndarray
    has_previous_advection: int = 0
    metrics: dict = field(default_factory=dict)

    @staticmethod
    def empty(grid):
        return State(zeros(grid, "u"), zeros(grid, "v"), zeros(grid, "w"), zeros(grid, "u"),
                     zeros(grid, "v"), zeros(grid, "w"), zeros(grid, "p"))

    def copy(self):
        return State(*(getattr(self, n).copy() for n in FIELDS), self.has_previous_advection,
                     dict(self.metrics))

    def to_c(self):
        cs = CState(*(ptr(getattr(self, n)) for n in FIELDS))
        cs.has_previous_advection = self.has_previous_advection
        for k, v in self.metrics.items():
            setattr(cs.metrics, k, v)
        return cs

    def from_c(self, cs):
        self.has_previous_advection = cs.has_previous_advection
        self.metrics = {k: getattr(cs.metrics, k) for k, _ in StepMetrics._fields_}


FIELDS = ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")


class OracleError(RuntimeError):
    pass


class Oracle:
    """Python face of one oracle library (the restatement or the reference build)."""

    def __init__(self, path=ORACLE_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = C.CDLL(path)
        L = self.lib
        L.oo_last_error.restype = C.c_char_p
        L.oo_tg_dt.restype = C.c_double
        L.oo_cavity_dt.restype = C.c_double

    def _check(self, rc):
        if rc != 0:
            msg = self.lib.oo_last_error().decode()
            if rc == 1:
                raise ValueError(msg)
            raise OracleError(msg)

    # --- operators -------------------------------------------------------
    def advection(self, grid, u, v, w):
        out = [zeros(grid, c) for c in "uvw"]
        self._check(self.lib.oo_advection(C.byref(grid), ptr(u), ptr(v), ptr(w), *map(ptr, out)))
        return out

    def diffusion(self, grid, nu, u, v, w):
        out = [zeros(grid, c) for c in "uvw"]
        self._check(self.lib.oo_diffusion(C.byref(grid), C.c_double(nu), ptr(u), ptr(v), ptr(w),
                                          *map(ptr, out)))
        return out

    def apply_velocity_bc(self, grid, bc, u, v, w):
        self._check(self.lib.oo_apply_velocity_bc(C.byref(grid), C.byref(bc), ptr(u), ptr(v),
                                                  ptr(w)))

    def apply_pressure_bc(self, grid, pbc, p):
        self._check(self.lib.oo_apply_pressure_bc(C.byref(grid), C.byref(pbc), ptr(p)))

    def derive_pressure_correction_bc(self, bc):
        out = PBC()
        self._check(self.lib.oo_derive_pressure_correction_bc(C.byref(bc), C.byref(out)))
        return out

    def apply_total_pressure_bc(self, grid, bc, su, sv, sw, p):
        self._check(self.lib.oo_apply_total_pressure_bc(C.byref(grid), C.byref(bc), ptr(su),
                                                        ptr(sv), ptr(sw), ptr(p)))

    def gradient(self, grid, p):
        out = [zeros(grid, c) for c in "uvw"]
        self._check(self.lib.oo_gradient(C.byref(grid), ptr(p), *map(ptr, out)))
        return out

    def divergence(self, grid, u, v, w):
        out = zeros(grid, "p")
        self._check(self.lib.oo_divergence(C.byref(grid), ptr(u), ptr(v), ptr(w), ptr(out)))
        return out

    def predictor_adi(self, grid, bc, alpha, ru, rv, rw):
        out = [zeros(grid, c) for c in "uvw"]
        ls = C.c_int(0)
        self._check(self.lib.oo_predictor_adi(C.byref(grid), C.byref(bc), C.c_double(alpha),
                                              ptr(ru), ptr(rv), ptr(rw), *map(ptr, out),
                                              C.byref(ls)))
        return out, ls.value

    def poisson_solve(self, grid, pbc, max_iterations, tolerance, rhs, pressure, hist_cap=4096):
        d = PoissonDiag()
        hist = np.zeros(hist_cap)
        self._check(self.lib.oo_poisson_solve(C.byref(grid), C.byref(pbc), max_iterations,
                                              C.c_double(tolerance), ptr(rhs), ptr(pressure),
                                              C.byref(d), ptr(hist), hist_cap))
        n = min(d.iterations + 1, hist_cap)
        return d, hist[:n].copy()

    def project_velocity(self, grid, bc, dt, density, max_iterations, tolerance, pu, pv, pw,
                         phi):
        out = [zeros(grid, c) for c in "uvw"]
        rhs = zeros(grid, "p")
        d = ProjectionDiag()
        self._check(self.lib.oo_project_velocity(
            C.byref(grid), C.byref(bc), C.c_double(dt), C.c_double(density), max_iterations,
            C.c_double(tolerance), ptr(pu), ptr(pv), ptr(pw), ptr(phi), *map(ptr, out), ptr(rhs),
            C.byref(d)))
        return out, rhs, d

    # --- Taylor-Green -----------------------------------------------------
    def tg_grid(self, cfg):
        g = Grid()
        self._check(self.lib.oo_tg_grid(C.byref(cfg), C.byref(g)))
        return g

    def tg_dt(self, cfg):
        return self.lib.oo_tg_dt(C.byref(cfg))

    def tg_bc(self, cfg):
        bc = BC()
        self._check(self.lib.oo_tg_bc(C.byref(cfg), C.byref(bc)))
        return bc

    def tg_init(self, cfg, mode=0):
        s = State.empty(self.tg_grid(cfg))
        cs = s.to_c()
        self._check(self.lib.oo_tg_init(C.byref(cfg), mode, C.byref(cs)))
        s.from_c(cs)
        return s

    def tg_init_tail(self, cfg, s):
        cs = s.to_c()
        self._check(self.lib.oo_tg_init_tail(C.byref(cfg), C.byref(cs)))
        s.from_c(cs)
        return s

    def tg_steps(self, cfg, steps, s):
        cs = s.to_c()
        self._check(self.lib.oo_tg_steps(C.byref(cfg), steps, C.byref(cs)))
        s.from_c(cs)
        return s

    def tg_validate(self, cfg, s_or_fields, time, mode=0):
        u, v, w = (s_or_fields.u, s_or_fields.v, s_or_fields.w) if hasattr(s_or_fields, "u") \
            else s_or_fields
        out = TGValidation()
        self._check(self.lib.oo_tg_validate(C.byref(cfg), mode, ptr(u), ptr(v), ptr(w),
                                            C.c_double(time), C.byref(out)))
        return {k: getattr(out, k) for k, _ in TGValidation._fields_}

    # --- cavity -------------------------------------------------------------
    def cavity_grid(self, cfg):
        g = Grid()
        self._check(self.lib.oo_cavity_grid(C.byref(cfg), C.byref(g)))
        return g

    def cavity_dt(self, cfg):
        return self.lib.oo_cavity_dt(C.byref(cfg))

    def cavity_bc(self, cfg):
        bc = BC()
        self._check(self.lib.oo_cavity_bc(C.byref(cfg), C.byref(bc)))
        return bc

    def cavity_init(self, cfg):
        s = State.empty(self.cavity_grid(cfg))
        cs = s.to_c()
        self._check(self.lib.oo_cavity_init(C.byref(cfg), C.byref(cs)))
        s.from_c(cs)
        return s

    def cavity_steps(self, cfg, steps, s):
        cs = s.to_c()
        self._check(self.lib.oo_cavity_steps(C.byref(cfg), steps, C.byref(cs)))
        s.from_c(cs)
        return s


class ReferenceIO(Oracle):
    """The reference build's drivers and I/O around the step (config files,
    describe, SLVCHKP1 checkpoint, finalize, VTK): liborchard_ref.so only."""

    def __init__(self, path=REF_SO):
        super().__init__(path)

    def tg_config_load(self, path):
        c, val, buf = TGConfig(), C.c_int(), C.create_string_buffer(4096)
        self._check(self.lib.oo_ref_tg_config_load(str(path).encode(), C.byref(c), C.byref(val), buf,
                                                   C.c_size_t(4096)))
        return c, bool(val.value), buf.value.decode()

    def cavity_config_load(self, path):
        c, val, buf = CavityConfig(), C.c_int(), C.create_string_buffer(4096)
        self._check(self.lib.oo_ref_cavity_config_load(str(path).encode(), C.byref(c), C.byref(val),
                                                       buf, C.c_size_t(4096)))
        return c, bool(val.value), buf.value.decode()

    def build_description(self):
        buf = C.create_string_buffer(1024)
        self._check(self.lib.oo_ref_build_description(buf, C.c_size_t(1024)))
        return buf.value.decode()

    def cavity_checkpoint_write(self, path, cfg, validate_reference, s):
        cs = s.to_c()
        self._check(self.lib.oo_ref_cavity_checkpoint_write(str(path).encode(), C.byref(cfg),
                                                            int(validate_reference), C.byref(cs)))

    def cavity_checkpoint_load(self, path, cfg, validate_reference):
        s = State.empty(self.cavity_grid(cfg))
        cs = s.to_c()
        meta = (C.c_ulonglong * 3)()
        self._check(self.lib.oo_ref_cavity_checkpoint_load(str(path).encode(), C.byref(cfg),
                                                           int(validate_reference), C.byref(cs), meta))
        s.from_c(cs)
        return s, {"checksum": meta[0], "build_hash": meta[1], "configuration_hash": meta[2]}

    def cavity_finalize(self, cfg, validate_reference, s):
        cs = s.to_c()
        ext, smp, err = (C.c_double * 4)(), (C.c_double * 4)(), (C.c_double * 4)()
        worst, ok = C.c_double(), C.c_int()
        self._check(self.lib.oo_ref_cavity_finalize(C.byref(cfg), int(validate_reference), C.byref(cs),
                                                    ext, smp, err, C.byref(worst), C.byref(ok)))
        return {"u_vertical_max": ext[0], "u_vertical_min": ext[1], "v_horizontal_max": ext[2],
                "v_horizontal_min": ext[3], "samples": list(smp), "errors": list(err),
                "max_relative_error": worst.value, "pass": bool(ok.value)}

    def write_vtk(self, path, grid, s):
        cs = s.to_c()
        self._check(self.lib.oo_ref_write_vtk(str(path).encode(), C.byref(grid), C.byref(cs)))


def tg_config(nx, ny, nz, viscosity=0.01, cfl_limit=0.5, final_time=0.5,
              poisson_max_iterations=200, poisson_tolerance=1e-10):
    """TaylorGreenConfig with the reference's defaults (solver/taylor_green.hpp:18-30)."""
    return TGConfig(nx, ny, nz, viscosity, cfl_limit, final_time, poisson_max_iterations,
                    poisson_tolerance)


def cavity_config(nx, ny, reynolds=100.0, lid_velocity=1.0, cfl_limit=0.5, max_steps=8000,
                  min_steps=200, steady_tolerance=1e-7, poisson_max_iterations=200,
                  poisson_tolerance=1e-10):
    """LidDrivenCavityConfig with the reference's defaults (solver/lid_driven_cavity.hpp:12-25)."""
    return CavityConfig(nx, ny, reynolds, lid_velocity, cfl_limit, max_steps, min_steps,
                        steady_tolerance, poisson_max_iterations, poisson_tolerance)


def periodic_bc():
    bc = BC()
    for f in range(6):
        bc.faces[f].type = PERIODIC
    return bc


def bc_from(types, velocities=None):
    bc = BC()
    for f, t in enumerate(types):
        bc.faces[f].type = t
        if velocities and velocities[f] is not None:
            for c in range(3):
                bc.faces[f].velocity[c] = velocities[f][c]
    return bc


def pbc_from(types, values=None, gradients=None):
    pbc = PBC()
    for f, t in enumerate(types):
        pbc.faces[f].type = t
        if values:
            pbc.faces[f].value = values[f]
        if gradients:
            pbc.faces[f].gradient = gradients[f]
    return pbc


def steps_config(nx, ny, nz, viscosity, cfl, steps, tol, max_it=400):
    """A TaylorGreenConfig whose final_time gives exactly ``steps`` steps.

    The reference takes dt = T / ceil(T / dt_max) with dt_max = cfl / sum(1/h)
    (solver/taylor_green.cpp:397-401, 519-525); T slightly below steps*dt_max
    makes the ceiling exactly ``steps``."""
    g = 2.0 * np.pi
    dx, dy = g / nx, g / ny
    inv = 1.0 / dx + 1.0 / dy + (1.0 / (g / nz) if nz > 1 else 0.0)
    dt_max = cfl / inv
    return tg_config(nx, ny, nz, viscosity, cfl, steps * dt_max * (1.0 - 1e-9), max_it, tol)
