"""The FFT flow solver (fsolver = 'f', main.f90:333-347) on the GPU against the oracle.

  - one step from a random state (velocities at two levels meeting bounduvw,
    a pressure meeting boundp, random IB forces): u, v, w and p within 1e-10
    of their largest value, with no-slip and with Couette wall values;
  - five steps fed back as the reference's main loop does (uoo <- uo <- u)
    within 1e-9; the final field is discretely divergence-free;
  - host and device memory give the same bits; mixed contexts and calls
    before sg_set_flow_params are refused.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200.coupling import CouplingStep, SgError

pytestmark = pytest.mark.gpu


def _state(grid, seed):
    itot, jtot, ktot = grid[:3]
    rng = np.random.default_rng(seed)
    shape = (ktot + 2, jtot + 2, itot + 2)
    uo, vo, wo, uoo, voo, woo = (rng.normal(size=shape) * 0.1 for _ in range(6))
    O.bounduvw(uo, vo, wo)
    O.bounduvw(uoo, voo, woo)
    p = rng.normal(size=shape) * 0.01
    O.boundp(p)
    f = [rng.normal(size=shape) for _ in range(3)]
    return [uo, vo, wo, uoo, voo, woo], p, f


def _ctx(grid, precision="fp64", mem="host"):
    return CouplingStep(grid, np.array([3], np.int32), np.array([0.1]), precision=precision, mem=mem)


GRID = (32, 24, 20, 1 / 16, 1 / 16, 1 / 16)


@pytest.mark.parametrize("walls", [(0.0, 0.0), (20 / 16 * 1.0, -20 / 16 * 1.0)])
def test_one_step(cuda, walls):
    vel, p, f = _state(GRID, 4)
    dt, rep = 2e-3, 0.7
    ru, rv, rw, rp = O.flow_step(GRID, dt, rep, *vel, p, *f, vb2=walls[0], vt2=walls[1])
    cs = _ctx(GRID)
    cs.set_flow_params(rep, *walls)
    pg = p.copy()
    u, v, w = cs.flow_step(dt, *vel, pg, *f)
    for g, r in ((u, ru), (v, rv), (w, rw), (pg, rp)):
        assert np.abs(g - r).max() <= 1e-10 * np.abs(r).max()


@pytest.mark.parametrize("grid", [(64, 64, 12, 1 / 16, 1 / 16, 1 / 16), (256, 128, 8, 1 / 32, 1 / 16, 1 / 8),
                                  (128, 256, 6, 1 / 16, 1 / 32, 1 / 8), (512, 32, 5, 1 / 64, 1 / 8, 1 / 8),
                                  (32, 24, 300, 1 / 16, 1 / 16, 1 / 64)])
def test_one_step_transform_paths(cuda, grid):
    """Register-resident transforms for power-of-two lengths (rows of 32 to
    256 complex values, columns of 32 to 256) beside the mixed-radix ones, and
    the elimination kept in shared memory (ktot <= 288) or streamed through
    global memory (ktot = 300)."""
    vel, p, f = _state(grid, 9)
    dt, rep = 1e-3, 0.8
    ru, rv, rw, rp = O.flow_step(grid, dt, rep, *vel, p, *f)
    cs = _ctx(grid)
    cs.set_flow_params(rep)
    pg = p.copy()
    u, v, w = cs.flow_step(dt, *vel, pg, *f)
    for g, r in ((u, ru), (v, rv), (w, rw), (pg, rp)):
        assert np.abs(g - r).max() <= 1e-10 * np.abs(r).max()


def test_five_steps_and_divergence(cuda):
    vel, p, f = _state(GRID, 5)
    dt, rep = 1e-3, 0.5
    cs = _ctx(GRID)
    cs.set_flow_params(rep)
    ro = [x.copy() for x in vel]
    rp = p.copy()
    go = [x.copy() for x in vel]
    gp = p.copy()
    for _ in range(5):
        u, v, w, rp = O.flow_step(GRID, dt, rep, *ro, rp, *f)
        ro = [u, v, w] + ro[:3]
        gu, gv, gw = cs.flow_step(dt, *go, gp, *f)
        go = [gu.copy(), gv.copy(), gw.copy()] + go[:3]
    for g, r in zip(go[:3] + [gp], ro[:3] + [rp]):
        assert np.abs(g - r).max() <= 1e-9 * np.abs(r).max()
    u, v, w = go[:3]
    S, dx = O._sh, GRID[3]
    div = (S(w, 0, 0, 0) - S(w, -1, 0, 0)) / dx + (S(v, 0, 0, 0) - S(v, 0, -1, 0)) / dx + (S(u, 0, 0, 0) - S(u, 0, 0, -1)) / dx
    assert np.abs(div).max() <= 1e-9 * np.abs(u).max() / dx


def test_device_memory_same_bits(cuda):
    torch = cuda
    vel, p, f = _state(GRID, 6)
    cs = _ctx(GRID)
    cs.set_flow_params(0.9)
    ph = p.copy()
    host = cs.flow_step(1e-3, *vel, ph, *f)
    cd = _ctx(GRID, mem="device")
    cd.set_flow_params(0.9)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    pd = dev(p)
    out = cd.flow_step(1e-3, *map(dev, vel), pd, *map(dev, f))
    torch.cuda.synchronize()
    for a, b in zip(host, out):
        assert np.array_equal(a, b.cpu().numpy())
    assert np.array_equal(ph, pd.cpu().numpy())


def test_refusals(cuda):
    vel, p, f = _state(GRID, 7)
    cs = _ctx(GRID)
    with pytest.raises(SgError) as e:
        cs.flow_step(1e-3, *vel, p, *f)
    assert e.value.code == 6
    cm = _ctx(GRID, precision="mixed")
    with pytest.raises(SgError) as e:
        cm.set_flow_params(1.0)
    assert e.value.code == 1


def test_one_step_on_non_cubic_cells(cuda):
    grid = (32, 24, 20, 1 / 16, 1 / 12, 1 / 20)
    vel, p, f = _state(grid, 8)
    dt, rep = 1e-3, 0.6
    ru, rv, rw, rp = O.flow_step(grid, dt, rep, *vel, p, *f)
    cs = _ctx(grid)
    cs.set_flow_params(rep)
    pg = p.copy()
    u, v, w = cs.flow_step(dt, *vel, pg, *f)
    for g, r in ((u, ru), (v, rv), (w, rw), (pg, rp)):
        assert np.abs(g - r).max() <= 1e-10 * np.abs(r).max()
