"""Case drivers, config files, checkpoints and VTK export of the B200 step.

Python face of ``include/orchard_b200_cases.h``, mirroring the reference's
drivers and I/O:

==========================================  ==========================================
here                                        reference
==========================================  ==========================================
``TaylorGreenConfig``                       TaylorGreenConfig (solver/taylor_green.hpp:18-30)
``load_taylor_green_config``                solver/taylor_green.cpp:425-481
``TaylorGreenCase`` (init, steps, run)      initialize_taylor_green_state,
                                            run_taylor_green_steps, run_taylor_green
``TaylorGreenCase.finalize``                finalize_taylor_green_result
``LidDrivenCavityConfig``                   solver/lid_driven_cavity.hpp:12-25
``load_lid_driven_cavity_config``           solver/lid_driven_cavity.cpp:296-336
``LidDrivenCavityCase``                     initialize_lid_driven_cavity_state,
                                            run_lid_driven_cavity_steps, run_lid_driven_cavity,
                                            finalize_lid_driven_cavity_result
``*.write_checkpoint`` / ``load_checkpoint``  io/checkpoint.cpp:313-461 (SLVCHKP1)
``*.write_vtk``                             io/vtk_export.cpp:18-73
==========================================  ==========================================

The case state stays resident on the GPU; every computation runs there.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _capi
from . import Context, Grid, _dp, _struct_dict

SCHEMES = ("tvd", "upwind", "central")
LIMITERS = ("van_leer",)
BACKENDS = ("cpu", "metal")


class OfTgConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("viscosity", C.c_double),
                ("cfl_limit", C.c_double), ("final_time", C.c_double),
                ("poisson_max_iterations", C.c_int), ("poisson_tolerance", C.c_double),
                ("validate_energy", C.c_int), ("backend", C.c_int), ("advection_scheme", C.c_int),
                ("advection_limiter", C.c_int)]


class OfTgResult(C.Structure):
    _fields_ = [("final_step", _capi.OfStepMetrics), ("initial_kinetic_energy", C.c_double),
                ("final_kinetic_energy", C.c_double), ("reference_dataset", C.c_char * 64),
                ("normalized_energy_error", C.c_double), ("velocity_relative_l2_error", C.c_double),
                ("exact_kinetic_energy", C.c_double), ("pass_", C.c_int),
                ("accelerator_name", C.c_char * 64), ("elapsed_seconds", C.c_double)]


class OfCavityConfig(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("reynolds", C.c_double),
                ("lid_velocity", C.c_double), ("cfl_limit", C.c_double), ("max_steps", C.c_int),
                ("min_steps", C.c_int), ("steady_tolerance", C.c_double),
                ("poisson_max_iterations", C.c_int), ("poisson_tolerance", C.c_double),
                ("validate_reference", C.c_int), ("advection_scheme", C.c_int),
                ("advection_limiter", C.c_int)]


class OfCavityPoint(C.Structure):
    _fields_ = [("label", C.c_char * 32), ("line", C.c_int), ("coordinate", C.c_double),
                ("reference_value", C.c_double), ("reference_lower_bound", C.c_double),
                ("reference_upper_bound", C.c_double), ("sample_value", C.c_double),
                ("relative_error", C.c_double)]


class OfCavityResult(C.Structure):
    _fields_ = [("final_step", _capi.OfStepMetrics), ("u_vertical_max", C.c_double),
                ("u_vertical_min", C.c_double), ("v_horizontal_max", C.c_double),
                ("v_horizontal_min", C.c_double), ("reference_dataset", C.c_char * 64),
                ("points", OfCavityPoint * 4), ("max_relative_error", C.c_double),
                ("divergence_l2", C.c_double), ("pass_", C.c_int), ("elapsed_seconds", C.c_double)]


class OfCheckpointMeta(C.Structure):
    _fields_ = [("format_version", C.c_uint32), ("scalar_bytes", C.c_uint32),
                ("checksum", C.c_uint64), ("build_hash", C.c_uint64),
                ("configuration_hash", C.c_uint64)]


CASE_SYMBOLS = (
    "of_rest_init", "of_kinetic_energy", "of_tg_velocity_error", "of_sample_line", "of_get_grid",
    "of_tg_config_default", "of_tg_config_load", "of_tg_config_describe", "of_tg_case",
    "of_tg_create", "of_tg_run_steps", "of_tg_finalize", "of_tg_run",
    "of_cavity_config_default", "of_cavity_config_load", "of_cavity_config_describe",
    "of_cavity_case", "of_cavity_create", "of_cavity_run_steps", "of_cavity_run_to_steady",
    "of_cavity_finalize", "of_cavity_run", "of_cavity_centerlines",
    "of_fnv1a64", "of_build_hash", "of_library_build_hash",
    "of_cavity_checkpoint_write", "of_cavity_checkpoint_load",
    "of_cavity_checkpoint_write_host", "of_cavity_checkpoint_load_host",
    "of_tg_checkpoint_write", "of_tg_checkpoint_load", "of_write_vtk",
)

_bound = None


def _lib():
    global _bound
    lib = _capi.load()
    if _bound is lib:
        return lib
    V, I, D, S = C.c_void_p, C.c_int, C.c_double, C.c_char_p
    PG, PB, PM = C.POINTER(_capi.OfGrid), C.POINTER(_capi.OfBC), C.POINTER(_capi.OfStepMetrics)
    PT, PC = C.POINTER(OfTgConfig), C.POINTER(OfCavityConfig)
    DP = _capi.DP
    lib.of_rest_init.argtypes = [V, D, D]
    lib.of_kinetic_energy.argtypes = [V, DP]
    lib.of_tg_velocity_error.argtypes = [V, D, D, I, DP]
    lib.of_sample_line.argtypes = [V, I, I, I, I, I, DP, C.POINTER(I)]
    lib.of_get_grid.argtypes = [V, PG]
    lib.of_tg_config_default.argtypes = [PT]
    lib.of_tg_config_load.argtypes = [S, PT]
    lib.of_tg_config_describe.argtypes = [PT, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    lib.of_tg_case.argtypes = [PT, PG, PB, DP, C.POINTER(I)]
    lib.of_tg_create.argtypes = [PT, I, C.POINTER(V)]
    lib.of_tg_run_steps.argtypes = [V, PT, I, PM]
    lib.of_tg_finalize.argtypes = [V, PT, C.POINTER(OfTgResult)]
    lib.of_tg_run.argtypes = [V, PT, C.POINTER(OfTgResult)]
    lib.of_cavity_config_default.argtypes = [PC]
    lib.of_cavity_config_load.argtypes = [S, PC]
    lib.of_cavity_config_describe.argtypes = [PC, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)]
    lib.of_cavity_case.argtypes = [PC, PG, PB, DP, DP]
    lib.of_cavity_create.argtypes = [PC, I, C.POINTER(V)]
    lib.of_cavity_run_steps.argtypes = [V, PC, I, PM]
    lib.of_cavity_run_to_steady.argtypes = [V, PC, PM]
    lib.of_cavity_finalize.argtypes = [V, PC, C.POINTER(OfCavityResult)]
    lib.of_cavity_run.argtypes = [V, PC, C.POINTER(OfCavityResult)]
    lib.of_cavity_centerlines.argtypes = [V, DP, DP, DP, DP]
    lib.of_fnv1a64.argtypes = [C.c_void_p, C.c_size_t]
    lib.of_fnv1a64.restype = C.c_uint64
    lib.of_build_hash.argtypes = [S, S, S, S, S, I]
    lib.of_build_hash.restype = C.c_uint64
    lib.of_library_build_hash.argtypes = []
    lib.of_library_build_hash.restype = C.c_uint64
    PMeta = C.POINTER(OfCheckpointMeta)
    lib.of_cavity_checkpoint_write.argtypes = [V, S, PC, C.c_uint64]
    lib.of_cavity_checkpoint_load.argtypes = [V, S, PC, C.c_uint64, PMeta]
    lib.of_cavity_checkpoint_write_host.argtypes = [S, PC, C.c_uint64] + [DP] * 7 + [I, PM]
    lib.of_cavity_checkpoint_load_host.argtypes = [S, PC, C.c_uint64] + [DP] * 7 + \
        [C.POINTER(I), PM, PMeta]
    lib.of_tg_checkpoint_write.argtypes = [V, S, PT, C.c_uint64]
    lib.of_tg_checkpoint_load.argtypes = [V, S, PT, C.c_uint64, PMeta]
    lib.of_write_vtk.argtypes = [V, S]
    _bound = lib
    return lib


def _path(p):
    return str(p).encode()


def _text(b):
    return b.decode() if isinstance(b, bytes) else b


# ---- configs -------------------------------------------------------------------

@dataclass
class TaylorGreenConfig:
    """TaylorGreenConfig (solver/taylor_green.hpp:18-30), same defaults."""
    nx: int = 128
    ny: int = 128
    nz: int = 1
    viscosity: float = 0.01
    cfl_limit: float = 0.5
    final_time: float = 0.5
    poisson_max_iterations: int = 200
    poisson_tolerance: float = 1.0e-10
    validate_energy: bool = True
    backend: str = "cpu"
    advection_scheme: str = "tvd"
    advection_limiter: str = "van_leer"

    def to_c(self):
        return OfTgConfig(self.nx, self.ny, self.nz, self.viscosity, self.cfl_limit, self.final_time,
                          self.poisson_max_iterations, self.poisson_tolerance,
                          int(bool(self.validate_energy)), BACKENDS.index(self.backend),
                          SCHEMES.index(self.advection_scheme),
                          LIMITERS.index(self.advection_limiter))

    @classmethod
    def from_c(cls, c):
        return cls(c.nx, c.ny, c.nz, c.viscosity, c.cfl_limit, c.final_time, c.poisson_max_iterations,
                   c.poisson_tolerance, bool(c.validate_energy), BACKENDS[c.backend],
                   SCHEMES[c.advection_scheme], LIMITERS[c.advection_limiter])


@dataclass
class LidDrivenCavityConfig:
    """LidDrivenCavityConfig (solver/lid_driven_cavity.hpp:12-25), same defaults."""
    nx: int = 128
    ny: int = 128
    reynolds: float = 100.0
    lid_velocity: float = 1.0
    cfl_limit: float = 0.5
    max_steps: int = 8000
    min_steps: int = 200
    steady_tolerance: float = 1.0e-7
    poisson_max_iterations: int = 200
    poisson_tolerance: float = 1.0e-10
    validate_reference: bool = True
    advection_scheme: str = "tvd"
    advection_limiter: str = "van_leer"

    def to_c(self):
        return OfCavityConfig(self.nx, self.ny, self.reynolds, self.lid_velocity, self.cfl_limit,
                              self.max_steps, self.min_steps, self.steady_tolerance,
                              self.poisson_max_iterations, self.poisson_tolerance,
                              int(bool(self.validate_reference)), SCHEMES.index(self.advection_scheme),
                              LIMITERS.index(self.advection_limiter))

    @classmethod
    def from_c(cls, c):
        return cls(c.nx, c.ny, c.reynolds, c.lid_velocity, c.cfl_limit, c.max_steps, c.min_steps,
                   c.steady_tolerance, c.poisson_max_iterations, c.poisson_tolerance,
                   bool(c.validate_reference), SCHEMES[c.advection_scheme],
                   LIMITERS[c.advection_limiter])


def load_taylor_green_config(path) -> TaylorGreenConfig:
    c = OfTgConfig()
    _capi.check(_lib().of_tg_config_load(_path(path), C.byref(c)))
    return TaylorGreenConfig.from_c(c)


def load_lid_driven_cavity_config(path) -> LidDrivenCavityConfig:
    c = OfCavityConfig()
    _capi.check(_lib().of_cavity_config_load(_path(path), C.byref(c)))
    return LidDrivenCavityConfig.from_c(c)


def describe(config) -> str:
    """describe(config) (solver/taylor_green.cpp:483-495, lid_driven_cavity.cpp:338-349)."""
    lib = _lib()
    fn = lib.of_tg_config_describe if isinstance(config, TaylorGreenConfig) else \
        lib.of_cavity_config_describe
    c = config.to_c()
    n = C.c_size_t()
    _capi.check(fn(C.byref(c), None, 0, C.byref(n)))
    buf = C.create_string_buffer(n.value + 1)
    _capi.check(fn(C.byref(c), buf, n.value + 1, None))
    return buf.value.decode()


def _grid(g):
    return Grid(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz)


def taylor_green_case(config: TaylorGreenConfig):
    """(grid, boundary set, dt, steps) of make_taylor_green_grid & co."""
    g, bc, dt, steps = _capi.OfGrid(), _capi.OfBC(), C.c_double(), C.c_int()
    c = config.to_c()
    _capi.check(_lib().of_tg_case(C.byref(c), C.byref(g), C.byref(bc), C.byref(dt), C.byref(steps)))
    return _grid(g), bc, dt.value, steps.value


def lid_driven_cavity_case(config: LidDrivenCavityConfig):
    """(grid, boundary set, viscosity, dt) of make_lid_driven_cavity_grid & co."""
    g, bc, nu, dt = _capi.OfGrid(), _capi.OfBC(), C.c_double(), C.c_double()
    c = config.to_c()
    _capi.check(_lib().of_cavity_case(C.byref(c), C.byref(g), C.byref(bc), C.byref(nu), C.byref(dt)))
    return _grid(g), bc, nu.value, dt.value


# ---- hashes ------------------------------------------------------------------------

def fnv1a64(data: bytes) -> int:
    return _lib().of_fnv1a64(data, len(data))


def build_hash(project_name, project_version, compiler_id, compiler_version, build_profile,
               fast_math=False) -> int:
    """build_hash of a BuildInfo (io/checkpoint.cpp:42-49)."""
    return _lib().of_build_hash(project_name.encode(), project_version.encode(), compiler_id.encode(),
                                compiler_version.encode(), build_profile.encode(), int(bool(fast_math)))


def library_build_hash() -> int:
    return _lib().of_library_build_hash()


def _meta_dict(m):
    return {name: getattr(m, name) for name, _ in m._fields_}


# ---- cases -----------------------------------------------------------------------

class _Case(Context):
    """A Context created by a case constructor of the C ABI."""

    def _adopt(self, handle):
        self._lib = _capi.load()
        self._h = handle
        g = _capi.OfGrid()
        _capi.check(self._lib.of_get_grid(self._h, C.byref(g)))
        self.grid = _grid(g)

    def kinetic_energy(self):
        e = C.c_double()
        _capi.check(_lib().of_kinetic_energy(self._h, C.byref(e)))
        return e.value

    def write_vtk(self, path):
        _capi.check(_lib().of_write_vtk(self._h, _path(path)))


class TaylorGreenCase(_Case):
    """A Taylor-Green run resident on the GPU (TaylorGreenState)."""

    def __init__(self, config: TaylorGreenConfig, device: int = 0, precision: int = _capi.OF_FP64):
        lib = _lib()
        self.config = config
        self._c = config.to_c()
        h = C.c_void_p()
        _capi.check(lib.of_tg_create(C.byref(self._c), int(device), C.byref(h)))
        self._adopt(h)
        if precision != _capi.OF_FP64:
            self.set_precision(precision)

    def run_case_steps(self, steps):
        """run_taylor_green_steps(config, steps, state)."""
        m = _capi.OfStepMetrics()
        _capi.check(_lib().of_tg_run_steps(self._h, C.byref(self._c), int(steps), C.byref(m)))
        return _struct_dict(m)

    def finalize(self):
        r = OfTgResult()
        _capi.check(_lib().of_tg_finalize(self._h, C.byref(self._c), C.byref(r)))
        return _tg_result(r)

    def run(self):
        """run_taylor_green(config, &state): re-initialise, step to final_time, finalize."""
        r = OfTgResult()
        _capi.check(_lib().of_tg_run(self._h, C.byref(self._c), C.byref(r)))
        return _tg_result(r)

    def velocity_error(self, time, mode=0):
        e = C.c_double()
        _capi.check(_lib().of_tg_velocity_error(self._h, self.config.viscosity, float(time), int(mode),
                                                C.byref(e)))
        return e.value

    def write_checkpoint(self, path, build_hash=0):
        _capi.check(_lib().of_tg_checkpoint_write(self._h, _path(path), C.byref(self._c), int(build_hash)))

    def load_checkpoint(self, path, build_hash=0):
        m = OfCheckpointMeta()
        _capi.check(_lib().of_tg_checkpoint_load(self._h, _path(path), C.byref(self._c), int(build_hash),
                                                 C.byref(m)))
        return _meta_dict(m)


def _tg_result(r):
    out = {name: getattr(r, name) for name, _ in r._fields_}
    out["final_step"] = _struct_dict(r.final_step)
    out["pass"] = bool(out.pop("pass_"))
    out["reference_dataset"] = _text(out["reference_dataset"])
    out["accelerator_name"] = _text(out["accelerator_name"])
    return out


class LidDrivenCavityCase(_Case):
    """A lid-driven-cavity run resident on the GPU (LidDrivenCavityState)."""

    def __init__(self, config: LidDrivenCavityConfig, device: int = 0, precision: int = _capi.OF_FP64):
        lib = _lib()
        self.config = config
        self._c = config.to_c()
        h = C.c_void_p()
        _capi.check(lib.of_cavity_create(C.byref(self._c), int(device), C.byref(h)))
        self._adopt(h)
        if precision != _capi.OF_FP64:
            self.set_precision(precision)

    def run_case_steps(self, steps):
        """run_lid_driven_cavity_steps(config, steps, state)."""
        m = _capi.OfStepMetrics()
        _capi.check(_lib().of_cavity_run_steps(self._h, C.byref(self._c), int(steps), C.byref(m)))
        return _struct_dict(m)

    def run_to_steady(self):
        """The solver_cavity loop: steps until steady or max_steps."""
        m = _capi.OfStepMetrics()
        _capi.check(_lib().of_cavity_run_to_steady(self._h, C.byref(self._c), C.byref(m)))
        return _struct_dict(m)

    def centerlines(self):
        g = self.grid
        uc, uv, vc, vv = (np.zeros(g.ny), np.zeros(g.ny), np.zeros(g.nx), np.zeros(g.nx))
        _capi.check(_lib().of_cavity_centerlines(self._h, _dp(uc), _dp(uv), _dp(vc), _dp(vv)))
        return {"u_vertical": (uc, uv), "v_horizontal": (vc, vv)}

    def finalize(self):
        r = OfCavityResult()
        _capi.check(_lib().of_cavity_finalize(self._h, C.byref(self._c), C.byref(r)))
        return _cavity_result(r)

    def run(self):
        """run_lid_driven_cavity(config) on the resident state."""
        r = OfCavityResult()
        _capi.check(_lib().of_cavity_run(self._h, C.byref(self._c), C.byref(r)))
        return _cavity_result(r)

    def write_checkpoint(self, path, build_hash=0):
        _capi.check(_lib().of_cavity_checkpoint_write(self._h, _path(path), C.byref(self._c),
                                                      int(build_hash)))

    def load_checkpoint(self, path, build_hash=0):
        m = OfCheckpointMeta()
        _capi.check(_lib().of_cavity_checkpoint_load(self._h, _path(path), C.byref(self._c),
                                                     int(build_hash), C.byref(m)))
        return _meta_dict(m)


def _cavity_result(r):
    out = {name: getattr(r, name) for name, _ in r._fields_ if name != "points"}
    out["final_step"] = _struct_dict(r.final_step)
    out["pass"] = bool(out.pop("pass_"))
    out["reference_dataset"] = _text(out["reference_dataset"])
    pts = []
    for p in r.points:
        d = {name: getattr(p, name) for name, _ in p._fields_}
        d["label"] = _text(d["label"])
        if d["label"]:
            pts.append(d)
    out["points"] = pts
    return out


# ---- host-side checkpoint codec ------------------------------------------------------

def write_cavity_checkpoint_host(path, config: LidDrivenCavityConfig, state, build_hash=0):
    """write_lid_driven_cavity_checkpoint on host arrays: state is a dict with
    u, v, w, adv_u, adv_v, adv_w, p (padded storage), has_previous_advection and
    metrics (dict of of_step_metrics fields)."""
    c = config.to_c()
    m = _capi.OfStepMetrics()
    for k, v in state.get("metrics", {}).items():
        setattr(m, k, v)
    arrs = [np.ascontiguousarray(state[k], dtype=np.float64)
            for k in ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")]
    _capi.check(_lib().of_cavity_checkpoint_write_host(_path(path), C.byref(c), int(build_hash),
                                                       *map(_dp, arrs),
                                                       int(bool(state.get("has_previous_advection"))),
                                                       C.byref(m)))


def load_cavity_checkpoint_host(path, config: LidDrivenCavityConfig, build_hash=0):
    """load_lid_driven_cavity_checkpoint into host arrays; returns (state, meta)."""
    grid, _, _, _ = lid_driven_cavity_case(config)
    arrs = [grid.zeros(c) for c in "uvwuvwp"]
    hp = C.c_int()
    m = _capi.OfStepMetrics()
    meta = OfCheckpointMeta()
    c = config.to_c()
    _capi.check(_lib().of_cavity_checkpoint_load_host(_path(path), C.byref(c), int(build_hash),
                                                      *map(_dp, arrs), C.byref(hp), C.byref(m),
                                                      C.byref(meta)))
    names = ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")
    state = dict(zip(names, arrs))
    state["has_previous_advection"] = hp.value
    state["metrics"] = _struct_dict(m)
    return state, _meta_dict(meta)


__all__ = [n for n in dir() if not n.startswith("_") and n not in ("C", "np", "dataclass", "fields")]
