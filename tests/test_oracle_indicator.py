"""The oracle's indicator function (indicator.f90:19-182) on the CPU.

  - the Poisson solve (solver1d after initsolver(0)) satisfies the discrete
    equation it solves: the second-order Laplacian, periodic in x and y, with
    the Neumann rows of initsolver.f90:33-39 in z, to 1e-10 relative, for a
    right-hand side of zero mean (the mean mode is fixed by the reference's
    zero last pivot);
  - for a spherical capsule the indicator is 1 at the centre, 0 far away, and
    its integral is the sphere's volume within 3 %;
  - the viscosity and the centrifugal terms follow from the indicator as
    written (visc0 (1 + (lambda - 1) I), 0.5 (I_j + I_j+1) sin(theta) (ta/Rep^2)^1/4).
"""
import numpy as np

import oracle as O
from suguru_b200 import workloads as W


def laplacian(p, dx, dy, dz):
    """The operator solver1d inverts, on interior values [kmax, jtot, itot]."""
    lap = (np.roll(p, -1, 2) - 2 * p + np.roll(p, 1, 2)) / dx ** 2 + (np.roll(p, -1, 1) - 2 * p + np.roll(p, 1, 1)) / dy ** 2
    pz = np.concatenate([p[:1], p, p[-1:]], axis=0)  # Neumann: b(1) += a(1), b(kmax) += c(kmax)
    return lap + (pz[2:] - 2 * p + pz[:-2]) / dz ** 2


def test_poisson_solves_the_discrete_laplacian():
    rng = np.random.default_rng(8)
    rhs = rng.normal(size=(12, 10, 16))
    rhs -= rhs.mean()
    dx, dy, dz = 1 / 16, 1 / 20, 1 / 32
    p = O.poisson_solver1d(rhs, dx, dy, dz)
    assert np.abs(laplacian(p, dx, dy, dz) - rhs).max() <= 1e-10 * np.abs(rhs).max()


def sphere_case():
    dx = 1.0 / 16
    grid = (48, 48, 48, dx, dx, dx)
    R = 7 * dx
    L = 11
    x, y, z = W.capsule_points(L, R, np.array([1.5, 1.5, 1.3]))
    _, n, a = O.complagrforces(L, R, x, y, z)
    return grid, R, (x, y, z), n, a


def test_indicator_of_a_sphere():
    grid, R, (x, y, z), n, a = sphere_case()
    out = O.indicator(grid, x, y, z, *n, a)
    dx = grid[3]
    I = out["indic"][1:-1, 1:-1, 1:-1]
    vol = I.sum() * dx ** 3
    assert abs(vol - 4 / 3 * np.pi * R ** 3) <= 0.03 * (4 / 3 * np.pi * R ** 3)
    k, j, i = (int(c / dx) for c in (1.3, 1.5, 1.5))  # the cell whose corner is the centre
    assert I[k, j, i] == 1.0 and I[2, 2, 2] == 0.0
    assert I.min() >= 0.0


def test_viscosity_and_centrifugal_terms():
    grid, R, (x, y, z), n, a = sphere_case()
    out = O.indicator(grid, x, y, z, *n, a, visc0=3.0, lam=5.0, thetainc=0.3, ta=2.0, rep=0.5)
    Ic = out["indic"]
    assert np.allclose(out["visc"][1:-1, 1:-1, 1:-1], 3.0 * (1 + 4.0 * Ic[1:-1, 1:-1, 1:-1]), rtol=0, atol=1e-15)
    amp = (2.0 / 0.25) ** 0.25
    fy = 0.5 * (Ic[1:-1, 1:-1, 1:-1] + Ic[1:-1, 2:, 1:-1]) * np.sin(0.3) * amp
    assert np.allclose(out["fy"][1:-1, 1:-1, 1:-1], fy, rtol=0, atol=1e-14)
    assert np.all(out["fy"][0] == 0)  # halos untouched
