"""Wall collision force (collisions.f90:10-32) on the GPU.

Capsules close to the wall z = 0 (the nearest points within 1-2 cells of it,
inside the cutoff rad0 = 2.5 dz) and one far from it:

  - sg_collisions against the oracle's restatement: FP64 relative L2
    <= 1e-13, mixed (FP32 force, FP64 wall term, one rounding) <= 1e-6;
  - sg_step with the force applied between the membrane force and the
    spreading (main.f90:229-233) against the oracle's complagrforces,
    collisions and lagr2eulr in that order: FP64 force 1e-10, field 1e-10,
    mixed 1e-4 (the tolerances of the step parity tests);
  - sg_membrane_force (complagrforces) never includes it, and sg_step
    without it is bitwise the plain step;
  - sg_collisions before any parameters are set, and invalid parameters,
    are refused.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep, SgError
from util import rel_l2

pytestmark = pytest.mark.gpu


def wall_case():
    dx = 1.0 / 16
    grid = (64, 48, 40, dx, dx, dx)
    degree = [11, 15, 7]
    radius = np.array([4.0, 5.0, 4.0]) * dx
    centre = np.array([[1.0, 1.0, 5.0 * dx], [2.6, 1.7, 6.2 * dx], [3.0, 2.0, 1.25]])
    rng = np.random.default_rng(17)
    modes = W.velocity_modes(rng)
    wl = W._build("wall", grid, degree, radius, centre, 0.05 * radius, rng, modes, 0.5)
    assert wl.z.min() > 0.5 * dx
    return wl


@pytest.fixture(scope="module")
def case():
    wl = wall_case()
    dz = wl.grid[5]
    off = wl.offsets
    F = np.zeros((3, wl.npts))
    A = np.zeros(wl.npts)
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        f, _, a = O.complagrforces(int(wl.degree[k]), float(wl.radius[k]), wl.x[s], wl.y[s], wl.z[s], wl.gs, wl.csk)
        F[:, s], A[s] = f, a
    Fc = F.copy()
    Fc[2] = O.collisions(wl.z, A, F[2], wl.grid[3], wl.grid[4], dz=dz)
    assert np.count_nonzero(Fc[2] != F[2]) > 100  # the wall term is active
    fgrid = O.spread(wl.grid, wl.x, wl.y, wl.z, Fc[0], Fc[1], Fc[2], A)
    return wl, F, Fc, A, fgrid


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_collisions_against_oracle(cuda, case, precision):
    wl, F, Fc, A, _ = case
    dt = np.float64 if precision == "fp64" else np.float32
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    cs.set_wall_collisions(in_step=False)
    fz = F[2].astype(dt)
    a = A.astype(dt)
    ref = O.collisions(wl.z, a.astype(np.float64), fz.astype(np.float64), wl.grid[3], wl.grid[4], dz=wl.grid[5])
    got = cs.collisions(wl.z, a, fz.copy())
    assert rel_l2(got, ref) <= (1e-13 if precision == "fp64" else 1e-6)
    far = ref == fz.astype(np.float64)
    assert np.array_equal(got[far], fz[far])  # no wall term: FZ unchanged


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_step_with_collisions(cuda, case, precision):
    wl, F, Fc, A, fgrid = case
    dt = np.float64 if precision == "fp64" else np.float32
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    cs.set_wall_collisions(in_step=True)
    u, v, w = wl.velocity(dtype=dt)
    out = cs.step(u, v, w, wl.x, wl.y, wl.z)
    tol = 1e-10 if precision == "fp64" else 1e-4
    for c in range(3):
        assert rel_l2(out["f"][c], Fc[c]) <= tol, c
        assert rel_l2(out["fgrid"][c], fgrid[c]) <= tol, c
    # the force that sg_membrane_force returns is complagrforces alone
    f, _, _ = cs.complagrforces(wl.x, wl.y, wl.z)
    assert rel_l2(f[2], F[2]) <= tol


def test_step_without_collisions_is_the_plain_step(cuda, case):
    wl = case[0]
    u, v, w = wl.velocity(dtype=np.float32)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="mixed")
    o1 = cs.step(u, v, w, wl.x, wl.y, wl.z)
    o1 = {k: [x.copy() for x in o1[k]] for k in ("f", "fgrid")}
    cs.set_wall_collisions(in_step=False)
    o2 = cs.step(u, v, w, wl.x, wl.y, wl.z)
    for k in ("f", "fgrid"):
        for c in range(3):
            assert np.array_equal(o1[k][c], o2[k][c]), (k, c)


def test_refusals(cuda, case):
    wl = case[0]
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="fp64")
    z = wl.z.copy()
    with pytest.raises(SgError) as e:
        cs.collisions(z, np.ones(wl.npts), np.zeros(wl.npts))
    assert e.value.code == 6  # SG_ERR_STATE
    for bad in (dict(rad0=0.0), dict(rep=0.0), dict(col=np.nan), dict(betacol=np.inf)):
        with pytest.raises(SgError) as e:
            cs.set_wall_collisions(**bad)
        assert e.value.code == 5  # SG_ERR_ARG
