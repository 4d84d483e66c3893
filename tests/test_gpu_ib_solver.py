"""The coupled solver (main.f90:172-347 with fsolver = 'f') against the oracle's
main loop built from the same stages: coupling_step, indicator, Update_Pos
(with the periodic shift) and flow_step, fed back step after step.

Three steps of the small mixed-degree batch, FP64, with and without the
indicator's centrifugal terms: positions within 1e-11 of the domain size,
velocities and pressure within 1e-9 of their largest value.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.ib_solver import IBSolver

pytestmark = pytest.mark.gpu

IND = dict(visc0=2.0, lam=3.0, thetainc=1.2, ta=2.0, rep=0.5)


def oracle_run(wl, steps, dt, rep, u0, indicator):
    g = wl.grid
    lx, ly, lz = (g[q] * g[q + 3] for q in range(3))
    x, y, z = wl.x.copy(), wl.y.copy(), wl.z.copy()
    u = [a.copy() for a in u0]
    uo = [a.copy() for a in u0]
    p = np.zeros_like(u0[0])
    for _ in range(steps):
        uoo, uo = uo, [a.copy() for a in u]
        r = O.coupling_step(g, wl.degree, wl.radius, *u, x, y, z, wl.gs, wl.csk)
        fx, fy, fz = r["fgrid"]
        if indicator:
            o = O.indicator(g, x, y, z, *r["n"], r["area"], fy=fy, fz=fz, **indicator)
            fy, fz = o["fy"], o["fz"]
        x, y, z = O.update_pos_capsules(wl.offsets, dt, lx, ly, lz, x, y, z, *r["u"])
        a, b, c, p = O.flow_step(g, dt, rep, *uo, *uoo, p, fx, fy, fz)
        u = [a, b, c]
    return (x, y, z), u, p


@pytest.mark.parametrize("indicator", [None, IND])
def test_coupled_steps_against_oracle(cuda, indicator):
    wl = W.small_config()
    u0 = list(wl.velocity())
    O.bounduvw(*u0)
    dt, rep, steps = 0.01 * wl.grid[3], 0.5, 3
    solver = IBSolver(wl, dt, rep, u0, indicator=indicator)
    solver.run(steps)
    got = solver.state()
    X, u, p = oracle_run(wl, steps, dt, rep, u0, indicator)
    size = wl.grid[0] * wl.grid[3]
    for g, r in zip(got["X"], X):
        assert np.abs(g - r).max() <= 1e-11 * size
    for g, r in zip(got["u"] + [got["p"]], u + [p]):
        assert np.abs(g - r).max() <= 1e-9 * np.abs(r).max()
    assert np.abs(u[0] - u0[0]).max() > 1e-6  # the flow did move


def test_graph_replay_is_bitwise_the_eager_loop(cuda):
    wl = W.small_config()
    u0 = list(wl.velocity())
    O.bounduvw(*u0)
    dt, rep = 0.01 * wl.grid[3], 0.5
    a = IBSolver(wl, dt, rep, u0, indicator=IND)
    a.run(5)
    b = IBSolver(wl, dt, rep, u0, indicator=IND)
    b.run(5, graph=True)
    sa, sb = a.state(), b.state()
    for k in ("X", "u"):
        for x, y in zip(sa[k], sb[k]):
            assert np.array_equal(x, y), k
    assert np.array_equal(sa["p"], sb["p"])


def test_mixed_coupling_step_within_the_mixed_tolerance(cuda):
    wl = W.small_config()
    u0 = list(wl.velocity())
    O.bounduvw(*u0)
    dt, rep = 0.01 * wl.grid[3], 0.5
    a = IBSolver(wl, dt, rep, u0, indicator=IND)
    a.run(3)
    b = IBSolver(wl, dt, rep, u0, indicator=IND, precision="mixed")
    b.run(3, graph=True)
    sa, sb = a.state(), b.state()
    size = wl.grid[0] * wl.grid[3]
    for x, y in zip(sa["X"], sb["X"]):
        assert np.abs(x - y).max() <= 1e-7 * size
    for x, y in zip(sa["u"], sb["u"]):
        assert np.abs(x - y).max() <= 1e-4 * np.abs(x).max()
