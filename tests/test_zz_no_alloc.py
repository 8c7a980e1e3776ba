"""of_pressure_rhs_noalloc: the allocation-free pressure right-hand side pass.

The entry point works on caller-owned device buffers with a static device
scratch.  It must give what the context path gives: the pressure rhs and the
two norms that of_project_velocity reports (rhs, rhs_l2, divergence_l2_before)
for the same boundary-consistent velocity, within the single-operator
tolerance (1e-12 relative), on consecutive calls that reuse the scratch.
"""
import ctypes as C

import numpy as np
import pytest

import pyoracle as po
from conftest import rel_maxdiff, to_gpu_bc, to_gpu_grid

OP_TOL = 1e-12


def _abi_grid(g):
    from solver_b200 import _capi
    return _capi.OfGrid(g.nx, g.ny, g.nz, g.dx, g.dy, g.dz)


def _consistent_velocity(oracle, g, bc, rng):
    """Random velocity with its boundary conditions applied (the `working`
    field project_velocity builds its rhs from)."""
    vel = [rng.standard_normal(po.shape(g, c)) for c in "uvw"]
    oracle.apply_velocity_bc(g, bc, *vel)
    return vel


def _noalloc(g, vel, dt, density, stream, with_norms=True):
    import torch
    from solver_b200 import _capi
    lib = _capi.load()
    dev = [torch.from_numpy(a).to("cuda:0") for a in vel]
    rhs = torch.zeros(po.shape(g, "p"), dtype=torch.float64, device="cuda:0")
    norms = np.full(2, np.nan)
    grid = _abi_grid(g)
    st = lib.of_pressure_rhs_noalloc(C.byref(grid), dt, density, *[t.data_ptr() for t in dev],
                                     rhs.data_ptr(),
                                     norms.ctypes.data_as(_capi.DP) if with_norms else None,
                                     stream.cuda_stream)
    _capi.check(st)
    stream.synchronize()
    return rhs.cpu().numpy(), norms


CASES = [
    # periodic box, several k chunks per column
    (po.Grid(64, 32, 48, 0.1, 0.2, 0.15), [po.PERIODIC] * 6),
    # walls on x and y, periodic z; ragged tiles (nx % 32, ny % 8 != 0)
    (po.Grid(40, 20, 12, 0.05, 0.07, 0.09),
     [po.NO_SLIP_WALL, po.NO_SLIP_WALL, po.SYMMETRY, po.PRESCRIBED_VELOCITY, po.PERIODIC,
      po.PERIODIC]),
]


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(CASES)))
def test_noalloc_matches_project_velocity_twice(oracle, case):
    import torch
    import solver_b200 as sb
    g, types = CASES[case]
    vels = [None] * 6
    if types[3] == po.PRESCRIBED_VELOCITY:
        vels[3] = (0.3, 0.0, -0.2)
    bc = po.bc_from(types, vels)
    rng = np.random.default_rng(11 + case)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(bc))
    stream = torch.cuda.Stream(device="cuda:0")
    # two calls in a row on different inputs; the second reuses the scratch
    for call, (dt, density) in enumerate(((0.01, 1.0), (0.003, 1.7))):
        vel = _consistent_velocity(oracle, g, bc, rng)
        _, _, rhs_ctx, d = ctx.project_velocity(vel, dt, density, 200, 1e-10)
        rhs, norms = _noalloc(g, vel, dt, density, stream)
        assert rel_maxdiff(rhs, rhs_ctx) <= OP_TOL, call
        assert abs(norms[0] - d["divergence_l2_before"]) <= OP_TOL * d["divergence_l2_before"], call
        assert abs(norms[1] - d["rhs_l2"]) <= OP_TOL * d["rhs_l2"], call
        # ghosts are left as passed in (zero)
        ghost = rhs.copy()
        ghost[1:-1, 1:-1, 1:-1] = 0.0
        assert not ghost.any(), call


@pytest.mark.gpu
def test_noalloc_enqueue_only_then_norms(oracle):
    """norms == NULL only enqueues; a following call with norms still gives
    the context path's norms (the ticket started from zero both times)."""
    import torch
    import solver_b200 as sb
    g, types = CASES[0]
    bc = po.bc_from(types)
    rng = np.random.default_rng(5)
    vel = _consistent_velocity(oracle, g, bc, rng)
    stream = torch.cuda.Stream(device="cuda:0")
    rhs0, _ = _noalloc(g, vel, 0.02, 1.0, stream, with_norms=False)
    rhs1, norms = _noalloc(g, vel, 0.02, 1.0, stream)
    assert np.array_equal(rhs0, rhs1)
    ctx = sb.Context(to_gpu_grid(g), to_gpu_bc(bc))
    _, _, rhs_ctx, d = ctx.project_velocity(vel, 0.02, 1.0, 200, 1e-10)
    assert rel_maxdiff(rhs1, rhs_ctx) <= OP_TOL
    assert abs(norms[1] - d["rhs_l2"]) <= OP_TOL * d["rhs_l2"]


def test_noalloc_rejects_oversized_plane():
    """Host-side checks fire before any device work (runs without a GPU):
    a k plane needing more reduction blocks than the scratch holds."""
    from solver_b200 import _capi
    lib = _capi.load()
    fake = 1 << 20  # never dereferenced: the call fails during validation
    big = _capi.OfGrid(32 * 8192 + 32, 8, 1, 1.0, 1.0, 1.0)
    norms = np.zeros(2)
    st = lib.of_pressure_rhs_noalloc(C.byref(big), 0.1, 1.0, fake, fake, fake, fake,
                                     norms.ctypes.data_as(_capi.DP), None)
    assert st == _capi.OF_INVALID_ARGUMENT
    msg = lib.of_last_error().decode()
    assert "static scratch holds 8192" in msg and "2097152 cells per k plane" in msg
    g = _capi.OfGrid(8, 8, 8, 1.0, 1.0, 1.0)
    st = lib.of_pressure_rhs_noalloc(C.byref(g), 0.0, 1.0, fake, fake, fake, fake, None, None)
    assert st == _capi.OF_INVALID_ARGUMENT
    assert lib.of_last_error().decode() == "build_pressure_rhs expects dt > 0"


@pytest.mark.gpu
def test_noalloc_calls_allocate_no_device_memory(oracle):
    """The property the entry point exists for: after a first call (which
    looks up the scratch address and loads the kernel), further calls leave
    the device's free memory unchanged."""
    import torch
    from solver_b200 import _capi
    lib = _capi.load()
    g, types = CASES[0]
    bc = po.bc_from(types)
    vel = _consistent_velocity(oracle, g, bc, np.random.default_rng(8))
    dev = [torch.from_numpy(a).to("cuda:0") for a in vel]
    rhs = torch.zeros(po.shape(g, "p"), dtype=torch.float64, device="cuda:0")
    norms = np.zeros(2)
    grid = _abi_grid(g)
    stream = torch.cuda.Stream(device="cuda:0")

    def call():
        st = lib.of_pressure_rhs_noalloc(C.byref(grid), 0.01, 1.0, *[t.data_ptr() for t in dev],
                                         rhs.data_ptr(), norms.ctypes.data_as(_capi.DP),
                                         stream.cuda_stream)
        _capi.check(st)

    call()
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(0)
    for _ in range(10):
        call()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info(0)
    assert free_after == free_before
