"""GPU parity of the CUDA coupling step against the CPU FP64 oracle.

Tolerances (relative L2 over all points / cells, FP64 plain path):
  interpolated velocity, spread field   <= 1e-12
  membrane force, normals, area          <= 1e-10
Mixed path (FP32 + Legendre contractions) against the FP64 oracle:
  force, velocity, spread field          <= 1e-4
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep
from util import rel_l2, rel_max

pytestmark = pytest.mark.gpu


def _forces_oracle(wl):
    off = wl.offsets
    F = np.zeros((3, wl.npts))
    Nn = np.zeros((3, wl.npts))
    A = np.zeros(wl.npts)
    for c in range(wl.ncap):
        s = slice(off[c], off[c + 1])
        f, n, a = O.complagrforces(int(wl.degree[c]), float(wl.radius[c]), wl.x[s], wl.y[s], wl.z[s], wl.gs, wl.csk)
        F[:, s], Nn[:, s], A[s] = f, n, a
    return F, Nn, A


@pytest.fixture(scope="module", params=["small", "c0"])
def wl(request):
    return W.small_config() if request.param == "small" else W.config0()


def test_interp_fp64(cuda, wl):
    u, v, w = wl.velocity()
    ref = O.interp(wl.grid, u, v, w, wl.x, wl.y, wl.z)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    got = cs.eulr2lagr(u, v, w, wl.x, wl.y, wl.z)
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-12


def test_spread_fp64(cuda, wl):
    rng = np.random.default_rng(5)
    f = rng.normal(size=(3, wl.npts))
    a = rng.uniform(0.5, 1.5, wl.npts) * (wl.grid[3] ** 2)
    ref = O.spread(wl.grid, wl.x, wl.y, wl.z, f[0], f[1], f[2], a)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    got = cs.lagr2eulr(wl.x, wl.y, wl.z, f[0].copy(), f[1].copy(), f[2].copy(), a)
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-12
        assert np.abs(g - r).max() <= 1e-12 * np.abs(r).max()


def test_spread_deterministic(cuda, wl):
    rng = np.random.default_rng(6)
    f = rng.normal(size=(3, wl.npts))
    a = rng.uniform(0.5, 1.5, wl.npts)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    g1 = cs.lagr2eulr(wl.x, wl.y, wl.z, f[0].copy(), f[1].copy(), f[2].copy(), a)
    g2 = cs.lagr2eulr(wl.x, wl.y, wl.z, f[0].copy(), f[1].copy(), f[2].copy(), a)
    for x, y in zip(g1, g2):
        assert np.array_equal(x, y)


def test_forces_fp64(cuda, wl):
    F, Nn, A = _forces_oracle(wl)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    f, n, a = cs.complagrforces(wl.x, wl.y, wl.z)
    for c in range(3):
        assert rel_l2(f[c], F[c]) <= 1e-10
        assert rel_l2(n[c], Nn[c]) <= 1e-10
    assert rel_l2(a, A) <= 1e-10


def test_step_fp64(cuda, wl):
    u, v, w = wl.velocity()
    ref = O.coupling_step(wl.grid, wl.degree, wl.radius, u, v, w, wl.x, wl.y, wl.z, wl.gs, wl.csk)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    out = cs.step(u, v, w, wl.x, wl.y, wl.z)
    for c in range(3):
        assert rel_l2(out["u"][c], ref["u"][c]) <= 1e-12
        assert rel_l2(out["f"][c], ref["f"][c]) <= 1e-10
        assert rel_l2(out["fgrid"][c], ref["fgrid"][c]) <= 1e-10
    assert rel_l2(out["area"], ref["area"]) <= 1e-10


def test_step_mixed(cuda, wl):
    u, v, w = wl.velocity()
    ref = O.coupling_step(wl.grid, wl.degree, wl.radius, u, v, w, wl.x, wl.y, wl.z, wl.gs, wl.csk)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
    out = cs.step(u.astype(np.float32), v.astype(np.float32), w.astype(np.float32), wl.x, wl.y, wl.z)
    errs = {}
    for c in range(3):
        errs["u%d" % c] = rel_l2(out["u"][c], ref["u"][c])
        errs["f%d" % c] = rel_l2(out["f"][c], ref["f"][c])
        errs["n%d" % c] = rel_l2(out["n"][c], ref["n"][c])
        errs["g%d" % c] = rel_l2(out["fgrid"][c], ref["fgrid"][c])
    errs["area"] = rel_l2(out["area"], ref["area"])
    print(errs)
    for k, e in errs.items():
        assert e <= 1e-4, (k, e)
