"""B200-native projection time step of Orchard Flow (zfifteen/solver).

Python face of the C ABI (include/orchard_b200.h).  ``Context`` mirrors the
reference's projection-step seams, each a C++ free function in the reference:

====================================  ==============================================
``Context`` method                    reference function
====================================  ==============================================
``compute_advection_term``            solver/momentum_terms.hpp:36-38
``solve_predictor_adi``               solver/projection.hpp:49-52
``solve_pressure_poisson``            linsolve/poisson_solver.hpp:34-37
``project_velocity``                  solver/projection.hpp:65-70
``run_steps`` on the resident state   run_taylor_green_steps, solver/taylor_green.hpp:87;
                                      run_lid_driven_cavity_steps,
                                      solver/lid_driven_cavity.hpp:119-121
====================================  ==============================================

Arrays are float64 numpy arrays in the reference's padded storage, shaped
``(sz, sy, sx)`` so that ``a[k, j, i]`` is the reference's ``field(i, j, k)``.
Every computation runs on the GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import (OF_CORRECTION_CAVITY, OF_CORRECTION_TAYLOR_GREEN, OF_FP64, OF_MIXED,  # noqa
                    NonFiniteError, NotConvergedError, OfError)

# PhysicalBoundaryType / PressureBoundaryType (bc/boundary_conditions.hpp:10-22)
NO_SLIP_WALL, PRESCRIBED_VELOCITY, SYMMETRY, FIXED_PRESSURE, PERIODIC = range(5)
P_NEUMANN, P_DIRICHLET, P_PERIODIC = range(3)

POISSON_LABELS = {"solver": "mgpcg", "preconditioner": "geometric_multigrid",
                  "cycle": "v_cycle", "smoother": "damped_jacobi"}


@dataclass(frozen=True)
class Grid:
    """Grid (core/grid.hpp:57-87) with one ghost layer."""
    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float

    def shape(self, loc):
        """Padded storage shape (sz, sy, sx) of 'p', 'u', 'v' or 'w'."""
        ext = {"p": (self.nx, self.ny, self.nz), "u": (self.nx + 1, self.ny, self.nz),
               "v": (self.nx, self.ny + 1, self.nz), "w": (self.nx, self.ny, self.nz + 1)}[loc]
        return (ext[2] + 2, ext[1] + 2, ext[0] + 2)

    def zeros(self, loc):
        return np.zeros(self.shape(loc))


def _dp(a):
    if a is None:
        return None
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("arrays must be C-contiguous float64")
    return a.ctypes.data_as(_capi.DP)


def _check_shape(grid, a, loc, what):
    if a.shape != grid.shape(loc):
        raise ValueError(f"{what}: incompatible field layouts (expected {grid.shape(loc)}, "
                         f"got {a.shape})")


def make_bc(faces):
    """BoundaryConditionSet from six (type, velocity[3], pressure) tuples or types."""
    bc = _capi.OfBC()
    for f, spec in enumerate(faces):
        if isinstance(spec, int):
            spec = (spec,)
        bc.faces[f].type = spec[0]
        if len(spec) > 1 and spec[1] is not None:
            for c in range(3):
                bc.faces[f].velocity[c] = spec[1][c]
        if len(spec) > 2:
            bc.faces[f].pressure = spec[2]
    return bc


def make_pbc(faces):
    """PressureBoundarySet from six (type, value, gradient) tuples or types."""
    pbc = _capi.OfPBC()
    for f, spec in enumerate(faces):
        if isinstance(spec, int):
            spec = (spec,)
        pbc.faces[f].type = spec[0]
        if len(spec) > 1:
            pbc.faces[f].value = spec[1]
        if len(spec) > 2:
            pbc.faces[f].gradient = spec[2]
    return pbc


def _struct_dict(s):
    return {name: getattr(s, name) for name, _ in s._fields_}


def poisson_diag_dict(d):
    out = _struct_dict(d)
    out["converged"] = bool(out["converged"])
    out["zero_mean_enforced"] = bool(out["zero_mean_enforced"])
    out.update(POISSON_LABELS)
    return out


class Context:
    """A device context: one grid, one velocity boundary set, one stream."""

    def __init__(self, grid: Grid, bc, device: int = 0, precision: int = OF_FP64):
        lib = _capi.load()
        self.grid = grid
        self._bc = bc if isinstance(bc, _capi.OfBC) else make_bc(bc)
        g = _capi.OfGrid(grid.nx, grid.ny, grid.nz, grid.dx, grid.dy, grid.dz)
        h = C.c_void_p()
        _capi.check(lib.of_create(C.byref(g), C.byref(self._bc), device, C.byref(h)))
        self._h = h
        self._lib = lib
        if precision != OF_FP64:
            self.set_precision(precision)

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            _capi.check(self._lib.of_destroy(self._h))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_precision(self, precision):
        _capi.check(self._lib.of_set_precision(self._h, precision))

    def device_bytes(self):
        n = C.c_size_t()
        _capi.check(self._lib.of_device_bytes(self._h, C.byref(n)))
        return n.value

    # ---- operator entry points -------------------------------------------
    def compute_advection_term(self, u, v, w, out=None):
        g = self.grid
        for a, loc in zip((u, v, w), "uvw"):
            _check_shape(g, a, loc, "compute_advection_term")
        out = out if out is not None else [g.zeros(c) for c in "uvw"]
        _capi.check(self._lib.of_compute_advection_term(self._h, _dp(u), _dp(v), _dp(w),
                                                        *map(_dp, out)))
        return out

    def solve_predictor_adi(self, rhs, alpha):
        g = self.grid
        for a, loc in zip(rhs, "uvw"):
            _check_shape(g, a, loc, "solve_predictor_adi")
        out = [g.zeros(c) for c in "uvw"]
        ls = C.c_int()
        _capi.check(self._lib.of_solve_predictor_adi(self._h, float(alpha), *map(_dp, rhs),
                                                     *map(_dp, out), C.byref(ls)))
        return out, ls.value

    def solve_pressure_poisson(self, rhs, pbc, max_iterations, tolerance, pressure=None,
                               history_cap=4096):
        g = self.grid
        _check_shape(g, rhs, "p", "solve_pressure_poisson")
        pressure = pressure if pressure is not None else g.zeros("p")
        _check_shape(g, pressure, "p", "solve_pressure_poisson")
        pbc = pbc if isinstance(pbc, _capi.OfPBC) else make_pbc(pbc)
        d = _capi.OfPoissonDiag()
        hist = np.zeros(history_cap)
        _capi.check(self._lib.of_solve_pressure_poisson(self._h, C.byref(pbc), int(max_iterations),
                                                        float(tolerance), _dp(rhs), _dp(pressure),
                                                        C.byref(d), _dp(hist), history_cap))
        diag = poisson_diag_dict(d)
        diag["residual_history"] = hist[:min(d.iterations + 1, history_cap)].copy()
        return pressure, diag

    def project_velocity(self, predicted, dt, density, max_iterations, tolerance,
                         pressure_correction=None, pressure_rhs=None):
        g = self.grid
        for a, loc in zip(predicted, "uvw"):
            _check_shape(g, a, loc, "project_velocity")
        phi = pressure_correction if pressure_correction is not None else g.zeros("p")
        rhs = pressure_rhs if pressure_rhs is not None else g.zeros("p")
        out = [g.zeros(c) for c in "uvw"]
        d = _capi.OfProjectionDiag()
        _capi.check(self._lib.of_project_velocity(self._h, float(dt), float(density),
                                                  int(max_iterations), float(tolerance),
                                                  *map(_dp, predicted), _dp(phi), *map(_dp, out),
                                                  _dp(rhs), C.byref(d)))
        diag = {"rhs_l2": d.rhs_l2, "divergence_l2_before": d.divergence_l2_before,
                "divergence_l2_after": d.divergence_l2_after, "pressure_mean": d.pressure_mean,
                "pressure_solve": poisson_diag_dict(d.pressure_solve)}
        return out, phi, rhs, diag

    # ---- resident state ------------------------------------------------------
    def upload_state(self, u, v, w, adv_u, adv_v, adv_w, p_total, has_previous_advection=False,
                     metrics=None):
        m = _capi.OfStepMetrics()
        for k, val in (metrics or {}).items():
            setattr(m, k, val)
        _capi.check(self._lib.of_state_upload(self._h, _dp(u), _dp(v), _dp(w), _dp(adv_u),
                                              _dp(adv_v), _dp(adv_w), _dp(p_total),
                                              int(bool(has_previous_advection)), C.byref(m)))

    def download_state(self):
        g = self.grid
        arrs = [g.zeros(c) for c in "uvw"] + [g.zeros(c) for c in "uvw"] + [g.zeros("p")]
        hp = C.c_int()
        m = _capi.OfStepMetrics()
        _capi.check(self._lib.of_state_download(self._h, *map(_dp, arrs), C.byref(hp), C.byref(m)))
        return {"u": arrs[0], "v": arrs[1], "w": arrs[2], "adv_u": arrs[3], "adv_v": arrs[4],
                "adv_w": arrs[5], "p": arrs[6], "has_previous_advection": hp.value,
                "metrics": _struct_dict(m)}

    def download_state_into(self, arrs):
        """Downloads the resident state into caller arrays (dict of u, v, w,
        adv_u, adv_v, adv_w, p); returns the step metrics."""
        names = ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")
        for name, loc in zip(names, "uvwuvwp"):
            _check_shape(self.grid, arrs[name], loc, "download_state")
        hp = C.c_int()
        m = _capi.OfStepMetrics()
        _capi.check(self._lib.of_state_download(self._h, *(_dp(arrs[k]) for k in names),
                                                C.byref(hp), C.byref(m)))
        return _struct_dict(m)

    def tg_init(self, viscosity, dt, mode=0):
        _capi.check(self._lib.of_tg_init(self._h, float(viscosity), float(dt), int(mode)))

    def step_host(self, params: _capi.OfStepParams, state):
        """One step of a host-resident state (dict of u, v, w, adv_u, adv_v,
        adv_w, p arrays, has_previous_advection, metrics), updated in place:
        upload, step and download in one call; pinned adv_* arrays get the new
        AB2 history while the pressure solve runs.  Returns the metrics."""
        names = ("u", "v", "w", "adv_u", "adv_v", "adv_w", "p")
        for name, loc in zip(names, "uvwuvwp"):
            _check_shape(self.grid, state[name], loc, "step_host")
        hp = C.c_int(int(bool(state.get("has_previous_advection", 0))))
        m = _capi.OfStepMetrics()
        for k, val in (state.get("metrics") or {}).items():
            setattr(m, k, val)
        _capi.check(self._lib.of_step_host(self._h, C.byref(params), *(_dp(state[k]) for k in names),
                                           C.byref(hp), C.byref(m)))
        state["has_previous_advection"] = hp.value
        state["metrics"] = _struct_dict(m)
        return state["metrics"]

    def run_steps(self, params: _capi.OfStepParams, steps: int):
        m = _capi.OfStepMetrics()
        _capi.check(self._lib.of_run_steps(self._h, C.byref(params), int(steps), C.byref(m)))
        return _struct_dict(m)

    # ---- derivatives (periodic grids, Taylor-Green predictor) ----------------
    def tangent_linear(self, params: _capi.OfStepParams, steps: int, du):
        """Runs `steps` steps from the resident state and returns the
        tangent-linear velocity for the perturbation `du` (three padded arrays)
        of the resident velocity's active entries."""
        g = self.grid
        for a, loc in zip(du, "uvw"):
            _check_shape(g, a, loc, "tangent_linear")
        out = [g.zeros(c) for c in "uvw"]
        _capi.check(self._lib.of_tangent_linear(self._h, C.byref(params), int(steps),
                                                *map(_dp, du), *map(_dp, out)))
        return out

    def adjoint_gradient(self, params: _capi.OfStepParams, steps: int, target,
                         checkpoint_every: int = 10):
        """Runs `steps` steps from the resident state; returns (grad, info) with
        grad the gradient of 1/2 |u(T) - target|^2 (unique entries) with respect
        to the resident velocity's active entries and info the loss, the
        viscosity derivative and the run's timings."""
        g = self.grid
        for a, loc in zip(target, "uvw"):
            _check_shape(g, a, loc, "adjoint_gradient")
        grad = [g.zeros(c) for c in "uvw"]
        info = _capi.OfAdjointInfo()
        _capi.check(self._lib.of_adjoint_gradient(self._h, C.byref(params), int(steps),
                                                  int(checkpoint_every), *map(_dp, target),
                                                  *map(_dp, grad), C.byref(info)))
        return grad, _struct_dict(info)

    def adjoint_gradient_binomial(self, params: _capi.OfStepParams, steps: int, target,
                                  snapshots: int = 0):
        """adjoint_gradient with the optimal binomial checkpoint schedule and
        `snapshots` saved states (0: as many as fit in device memory)."""
        g = self.grid
        for a, loc in zip(target, "uvw"):
            _check_shape(g, a, loc, "adjoint_gradient_binomial")
        grad = [g.zeros(c) for c in "uvw"]
        info = _capi.OfAdjointInfo()
        _capi.check(self._lib.of_adjoint_gradient_binomial(
            self._h, C.byref(params), int(steps), int(snapshots), *map(_dp, target),
            *map(_dp, grad), C.byref(info)))
        return grad, _struct_dict(info)


def adjoint_schedule_cost(steps: int, snapshots: int):
    """(reverse_cost, after_forward_cost): forward steps the binomial schedule
    recomputes for `steps` steps and `snapshots` free snapshots (host only)."""
    a, b = C.c_longlong(), C.c_longlong()
    _capi.check(_capi.load().of_adjoint_schedule_cost(int(steps), int(snapshots), C.byref(a),
                                                      C.byref(b)))
    return a.value, b.value


def step_params(viscosity, dt, max_iterations, tolerance, variant=OF_CORRECTION_TAYLOR_GREEN,
                density=1.0, name=None):
    """Parameters of one projection step (the run_*_steps locals)."""
    if name is None:
        name = "Taylor-Green" if variant == OF_CORRECTION_TAYLOR_GREEN else "lid-driven cavity"
    return _capi.OfStepParams(float(viscosity), float(dt), float(density), int(max_iterations),
                              float(tolerance), int(variant),
                              1 if variant == OF_CORRECTION_TAYLOR_GREEN else 0,
                              name.encode())


# ---- instrumentation ---------------------------------------------------------

def kernel_classes():
    lib = _capi.load()
    return [lib.of_kernel_class_name(i).decode() for i in range(lib.of_kernel_class_count())]


def profile_enable(on=True):
    _capi.check(_capi.load().of_profile_enable(1 if on else 0))


def profile_reset():
    _capi.check(_capi.load().of_profile_reset())


def profile_read():
    """{class name: (launches, timed launches, total device ms)}."""
    lib = _capi.load()
    out = {}
    for i, name in enumerate(kernel_classes()):
        n, t, ms = C.c_longlong(), C.c_longlong(), C.c_double()
        _capi.check(lib.of_profile_read(i, C.byref(n), C.byref(t), C.byref(ms)))
        out[name] = (n.value, t.value, ms.value)
    return out


def profile_coarse_chain(ctx, reps=200):
    """(microseconds, kernels) of one V-cycle coarse-level chain (levels 1 ..
    coarsest) replayed `reps` times from a CUDA graph of that chain alone, on
    the level-1 rhs of the context's last solve."""
    us, n = C.c_double(), C.c_int()
    _capi.check(ctx._lib.of_profile_coarse_chain(ctx._h, int(reps), C.byref(us), C.byref(n)))
    return us.value, n.value


def context_stream(ctx):
    """The context's cudaStream_t as an integer handle."""
    p = C.c_void_p()
    _capi.check(ctx._lib.of_stream(ctx._h, C.byref(p)))
    return p.value or 0
