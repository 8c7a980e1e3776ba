"""Host-side pieces of the adjoint check harness (no GPU).

`smooth_field` builds the seeded perturbation of the adjoint workloads by
summing its Fourier modes axis by axis; here it is checked against the
direct sum over the grid of a cos(k.x) + b sin(k.x) per mode, with the same
amplitudes drawn in the same order, on staggered 2D and 3D grids."""
import math

import numpy as np

import solver_b200 as sb
from solver_b200.adjoint import smooth_field, unique_view


def _direct(grid, seed, rms=1.0, kmax=4):
    g = grid
    rng = np.random.default_rng(seed)
    ks = range(-kmax, kmax + 1)
    modes = [(kx, ky, kz) for kx in ks for ky in ks for kz in ks
             if 0 < kx * kx + ky * ky + kz * kz <= kmax * kmax and (g.nz > 1 or kz == 0)]
    out = []
    for comp in "uvw":
        shape = g.shape(comp)
        axes = []
        for axis, (h, name) in enumerate(zip((g.dx, g.dy, g.dz), "xyz")):
            idx = np.arange(shape[2 - axis]) - 1.0
            face = (comp, name) in (("u", "x"), ("v", "y"), ("w", "z"))
            axes.append(idx * h if face else (idx + 0.5) * h)
        zz, yy, xx = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
        f = np.zeros(shape)
        if not (comp == "w" and g.nz == 1):
            for (kx, ky, kz) in modes:
                a, b = rng.standard_normal(2)
                ph = kx * xx + ky * yy + kz * zz
                f += a * np.cos(ph) + b * np.sin(ph)
        out.append(f)
    cur = math.sqrt(sum(float(np.mean(a[1:-1, 1:-1, 1:-1] ** 2)) for a in out) / 3.0)
    for a in out:
        a *= rms / cur
        sz, sy, sx = a.shape
        for k in (0, sz - 1):
            for j in (0, sy - 1):
                a[k, j, :] = 0.0
            for i in (0, sx - 1):
                a[k, :, i] = 0.0
        for j in (0, sy - 1):
            for i in (0, sx - 1):
                a[:, j, i] = 0.0
    return out


def test_smooth_field_equals_the_direct_mode_sum():
    for n, nz in ((16, 16), (24, 1), (20, 12)):
        h = 2.0 * math.pi / n
        g = sb.Grid(n, n, nz, h, h, h if nz > 1 else 1.0)
        fast = smooth_field(g, 3, rms=0.5)
        ref = _direct(g, 3, rms=0.5)
        for a, b in zip(fast, ref):
            assert a.shape == b.shape
            assert np.max(np.abs(a - b)) <= 1e-13
        rms = math.sqrt(sum(float(np.mean(a[1:-1, 1:-1, 1:-1] ** 2)) for a in fast) / 3.0)
        assert abs(rms - 0.5) <= 1e-14
        if nz == 1:
            assert not np.any(fast[2])


def test_smooth_field_is_periodic_on_the_unique_entries():
    # the duplicated periodic face equals the first face, so the field is a
    # sample of a 2 pi-periodic function
    n = 12
    h = 2.0 * math.pi / n
    g = sb.Grid(n, n, n, h, h, h)
    u = smooth_field(g, 7)[0]
    assert np.allclose(u[1:-1, 1:-1, 1], u[1:-1, 1:-1, n + 1], atol=1e-13)
    assert unique_view(u, "u").shape == (n, n, n)
