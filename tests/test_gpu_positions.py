"""Interpolation and spreading at awkward positions, through the C ABI
against the oracle: points exactly on cell faces and at cell centres (ties
of the nearest node), on and just beyond the periodic ends in x and y
(wrapped), at and beyond the walls in z (stencil clipped to 1..kmax), mixed
with interior points.  Tolerances: FP64 relative L2 <= 1e-12 (the spread
also within 1e-12 of its largest value everywhere); mixed <= 1e-5 for the
interpolated velocity and <= 1e-4 for the spread field."""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep
from util import rel_l2

pytestmark = pytest.mark.gpu


def _positions(grid, n, seed):
    itot, jtot, ktot, dx, dy, dz = grid
    lx, ly, lz = itot * dx, jtot * dy, ktot * dz
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, lx, n)
    y = rng.uniform(0.0, ly, n)
    z = rng.uniform(0.2 * lz, 0.8 * lz, n)
    kind = rng.integers(0, 5, n)
    m = kind == 0  # on faces, the ends of each axis included
    x[m] = rng.integers(0, itot + 1, m.sum()) * dx
    y[m] = rng.integers(0, jtot + 1, m.sum()) * dy
    z[m] = rng.integers(0, ktot + 1, m.sum()) * dz
    m = kind == 1  # at cell centres
    x[m] = (rng.integers(0, itot, m.sum()) + 0.5) * dx
    y[m] = (rng.integers(0, jtot, m.sum()) + 0.5) * dy
    z[m] = (rng.integers(0, ktot, m.sum()) + 0.5) * dz
    m = kind == 2  # just beyond the periodic ends
    lo = rng.uniform(size=m.sum()) < 0.5
    x[m] = np.where(lo, -rng.uniform(0.0, 2.0, m.sum()) * dx, lx + rng.uniform(0.0, 2.0, m.sum()) * dx)
    lo = rng.uniform(size=m.sum()) < 0.5
    y[m] = np.where(lo, -rng.uniform(0.0, 2.0, m.sum()) * dy, ly + rng.uniform(0.0, 2.0, m.sum()) * dy)
    m = kind == 3  # at and beyond the walls
    lo = rng.uniform(size=m.sum()) < 0.5
    z[m] = np.where(lo, rng.uniform(-1.5, 1.5, m.sum()) * dz, lz + rng.uniform(-1.5, 1.5, m.sum()) * dz)
    return x, y, z


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_interp_awkward_positions(cuda, precision):
    wl = W.small_config()
    x, y, z = _positions(wl.grid, wl.npts, 41)
    u, v, w = wl.velocity()
    ref = O.interp(wl.grid, u, v, w, x, y, z)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision)
    dt = np.float64 if precision == "fp64" else np.float32
    got = cs.eulr2lagr(u.astype(dt), v.astype(dt), w.astype(dt), x, y, z)
    tol = 1e-12 if precision == "fp64" else 1e-5
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= tol


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spread_awkward_positions(cuda, precision):
    wl = W.small_config()
    x, y, z = _positions(wl.grid, wl.npts, 42)
    rng = np.random.default_rng(43)
    f = rng.normal(size=(3, wl.npts))
    a = rng.uniform(0.5, 1.5, wl.npts) * wl.grid[3] ** 2
    ref = O.spread(wl.grid, x, y, z, f[0], f[1], f[2], a)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision)
    dt = np.float64 if precision == "fp64" else np.float32
    got = cs.lagr2eulr(x, y, z, *(v.astype(dt) for v in f), a.astype(dt))
    for g, r in zip(got, ref):
        if precision == "fp64":
            assert rel_l2(g, r) <= 1e-12
            assert np.abs(g - r).max() <= 1e-12 * np.abs(r).max()
        else:
            assert rel_l2(g, r) <= 1e-4
