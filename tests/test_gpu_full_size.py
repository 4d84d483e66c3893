"""The coupling step at the full sizes of the benchmark workloads.

  - dense suspension: 256 capsules, L = 15, 524,288 points, grid 256x256x128;
  - uneven batch: 1024 capsules, L = 7..23, 1,526,248 points, grid 512x256x256.

Both are compared with the FP64 oracle over every point and cell (its C step,
threaded over capsules, takes seconds at these sizes), with the tolerances of
the small parity cases: FP64 velocity and field 1e-12, force, normals and
area 1e-10 (relative L2); mixed 1e-4.  Properties that hold at any size are
checked on the full sizes too:

  - spreading conserves force: per component, the field summed over its cells
    (the periodic x and y halo copies left out) times dV equals the sum of
    force x area (FP64 1e-12, mixed 1e-6 of sum |force| x area);
  - a constant velocity interpolates to itself, the 3-point weights summing
    to one (FP64 1e-14, mixed 4e-6 = 32 units in the last place of 1);
  - the spread field does not depend on the order of the points: a permuted
    point list gives the same field bit for bit (integer sums, and a
    fixed-point scale made of order-independent quantities);
  - a repeated step gives the same bits.
"""
import os

import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep
from util import rel_l2

pytestmark = pytest.mark.gpu

_CASES = {}


def _case(name):
    if name not in _CASES:
        _CASES.clear()  # one full-size case in host memory at a time
        wl = W.config1() if name == "dense" else W.config2()
        u, v, w = wl.velocity()
        ref = O.coupling_step(wl.grid, wl.degree, wl.radius, u, v, w, wl.x, wl.y, wl.z, wl.gs, wl.csk,
                              nthreads=os.cpu_count() or 1)
        _CASES[name] = (wl, (u, v, w), ref)
    return _CASES[name]


def _tol(precision):
    return (1e-12, 1e-10) if precision == "fp64" else (1e-4, 1e-4)


@pytest.mark.parametrize("name", ["dense", "uneven"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_against_oracle(cuda, name, precision):
    wl, vel, ref = _case(name)
    dt = np.float64 if precision == "fp64" else np.float32
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    out = cs.step(*(x.astype(dt) for x in vel), wl.x, wl.y, wl.z)
    t_eul, t_lag = _tol(precision)
    for c in range(3):
        assert rel_l2(out["u"][c], ref["u"][c]) <= t_eul, ("u", c)
        assert rel_l2(out["fgrid"][c], ref["fgrid"][c]) <= t_eul, ("fgrid", c)
        assert rel_l2(out["f"][c], ref["f"][c]) <= t_lag, ("f", c)
        assert rel_l2(out["n"][c], ref["n"][c]) <= t_lag, ("n", c)
    assert rel_l2(out["area"], ref["area"]) <= t_lag


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spread_conserves_force(cuda, precision):
    wl, vel, _ = _case("dense")
    itot, jtot, ktot, dx, dy, dz = wl.grid
    dt = np.float64 if precision == "fp64" else np.float32
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    out = cs.step(*(x.astype(dt) for x in vel), wl.x, wl.y, wl.z)
    a = np.asarray(out["area"], np.float64)
    tol = 1e-12 if precision == "fp64" else 1e-6
    for c in range(3):
        f = np.asarray(out["f"][c], np.float64)
        g = np.asarray(out["fgrid"][c], np.float64)[:, 1:jtot + 1, 1:itot + 1]
        total = g.sum() * dx * dy * dz
        assert abs(total - (f * a).sum()) <= tol * np.abs(f * a).sum(), c


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_constant_velocity_interpolates_to_itself(cuda, precision):
    wl, _, _ = _case("dense")
    dt = np.float64 if precision == "fp64" else np.float32
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    const = (1.25, 0.0, -0.5)
    fields = [np.full(cs.field_shape, c, dt) for c in const]
    got = cs.eulr2lagr(*fields, wl.x, wl.y, wl.z)
    tol = 1e-14 if precision == "fp64" else 4e-6
    for g, c in zip(got, const):
        assert np.abs(np.asarray(g, np.float64) - c).max() <= tol * max(abs(c), 1.0)


@pytest.mark.parametrize("name", ["dense", "uneven"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_spread_independent_of_point_order(cuda, name, precision):
    wl, _, _ = _case(name)
    dt = np.float64 if precision == "fp64" else np.float32
    rng = np.random.default_rng(41)
    f = rng.normal(size=(3, wl.npts)).astype(dt)
    a = (rng.uniform(0.5, 1.5, wl.npts) * wl.grid[3] ** 2).astype(dt)
    perm = rng.permutation(wl.npts)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    g0 = [x.copy() for x in cs.lagr2eulr(wl.x, wl.y, wl.z, *f, a)]
    g1 = cs.lagr2eulr(wl.x[perm], wl.y[perm], wl.z[perm], *(x[perm] for x in f), a[perm])
    for c in range(3):
        assert np.array_equal(g0[c], g1[c]), c


def test_repeated_step_is_bitwise_identical(cuda):
    wl, vel, _ = _case("dense")
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="mixed")
    v32 = [x.astype(np.float32) for x in vel]
    o1 = cs.step(*v32, wl.x, wl.y, wl.z)
    o1 = {k: ([x.copy() for x in v] if isinstance(v, list) else v.copy()) for k, v in o1.items()}
    o2 = cs.step(*v32, wl.x, wl.y, wl.z)
    for k in ("u", "f", "n", "fgrid"):
        for c in range(3):
            assert np.array_equal(o1[k][c], o2[k][c]), (k, c)
    assert np.array_equal(o1["area"], o2["area"])
