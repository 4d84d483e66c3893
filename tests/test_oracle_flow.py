"""The oracle's FFT flow solver (fsolver = 'f': fftuvw, fillps, solver1d, correc,
bounduvw; main.f90:333-347) on the CPU.

  - the Helmholtz solves of initsolver(2) (u, v: no-slip ghost rows) and
    initsolver(3) (w: zero at the top face) satisfy the discrete equations
    they solve, to 1e-10 relative;
  - after a step the velocity is discretely divergence-free (fillps of the
    new field below 1e-10 of the field's scale / dx) and meets bounduvw;
  - a uniform body force on a fluid at rest accelerates it by f dt in the
    interior, away from the walls' viscous layers (the no-slip rows hold the
    first cells back).
"""
import numpy as np

import oracle as O


def helmholtz(p, dx, dy, dz, e, shift):
    """The operator solver1d inverts after initsolver(e), on interior values [kmax, jtot, itot]."""
    a, b, c = O.solver_rows(p.shape[0], dz, e, shift)
    lap = (np.roll(p, -1, 2) - 2 * p + np.roll(p, 1, 2)) / dx ** 2 + (np.roll(p, -1, 1) - 2 * p + np.roll(p, 1, 1)) / dy ** 2
    if e == 3:  # the last row is the identity: w(kmax) = rhs(kmax)
        lap[-1] = 0.0
    out = lap + b[:, None, None] * p
    out[1:] += a[1:, None, None] * p[:-1]
    out[:-1] += c[:-1, None, None] * p[1:]
    return out


def test_helmholtz_solves():
    rng = np.random.default_rng(2)
    dx, dy, dz = 1 / 16, 1 / 12, 1 / 20
    for e in (2, 3):
        rhs = rng.normal(size=(10, 12, 16))
        if e == 3:
            rhs[-1] = 0.0
        p = O.poisson_solver1d(rhs, dx, dy, dz, e=e, shift=37.0)
        assert np.abs(helmholtz(p, dx, dy, dz, e, 37.0) - rhs).max() <= 1e-10 * np.abs(rhs).max()


def _state(seed=3, grid=(16, 12, 10)):
    itot, jtot, ktot = grid
    dx = 1.0 / 16
    g = (itot, jtot, ktot, dx, dx, dx)
    rng = np.random.default_rng(seed)
    shape = (ktot + 2, jtot + 2, itot + 2)
    uo, vo, wo, uoo, voo, woo = (rng.normal(size=shape) * 0.1 for _ in range(6))
    O.bounduvw(uo, vo, wo)
    O.bounduvw(uoo, voo, woo)
    p = rng.normal(size=shape) * 0.01
    O.boundp(p)
    f = [rng.normal(size=shape) for _ in range(3)]
    return g, (uo, vo, wo, uoo, voo, woo), p, f


def test_step_is_divergence_free_and_meets_the_walls():
    g, vel, p, f = _state()
    dx = g[3]
    u, v, w, pn = O.flow_step(g, 1e-3, 0.5, *vel, p, *f)
    S = O._sh
    div = (S(w, 0, 0, 0) - S(w, -1, 0, 0)) / dx + (S(v, 0, 0, 0) - S(v, 0, -1, 0)) / dx + (S(u, 0, 0, 0) - S(u, 0, 0, -1)) / dx
    assert np.abs(div).max() <= 1e-10 * np.abs(u).max() / dx
    assert np.array_equal(u[0], -u[1]) and np.array_equal(v[-1], -v[-2])
    assert np.all(w[0] == 0) and np.all(w[-2] == 0)
    assert np.array_equal(u[:, :, 0], u[:, :, -2]) and np.array_equal(pn[:, -1, :], pn[:, 1, :])


def test_uniform_force_accelerates_the_core():
    g = (16, 12, 24, 1 / 16, 1 / 16, 1 / 16)
    shape = (26, 14, 18)
    zero = np.zeros(shape)
    fx = np.zeros(shape)
    fx[...] = 2.0
    dt = 1e-4
    u, v, w, _ = O.flow_step(g, dt, 1.0, zero, zero, zero, zero, zero, zero, zero, fx, zero, zero)
    core = u[6:-6, 1:-1, 1:-1]
    assert np.allclose(core, 2.0 * dt, rtol=1e-6)
    assert np.abs(v).max() <= 1e-15 and np.abs(w).max() <= 1e-15
