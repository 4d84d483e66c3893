"""Edge inputs of the coupling step through the C ABI.

  - no capsules: every call succeeds, the spread field (halos included) is
    zero and the Lagrangian outputs are empty;
  - the largest SH degrees the boundary accepts (up to L = 31, 8192 points a
    capsule, beside smaller ones): force, normals and area per capsule
    against the oracle, FP64 <= 1e-10 and mixed <= 1e-4 (the path
    tolerances), and the spread field and velocity likewise.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep
from util import rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_no_capsules(cuda, precision):
    wl = W.small_config()
    dt = np.float64 if precision == "fp64" else np.float32
    cs = CouplingStep(wl.grid, np.zeros(0, np.int32), np.zeros(0), precision=precision)
    assert cs.npts == 0
    u, v, w = (a.astype(dt) for a in wl.velocity())
    e = np.zeros(0)
    out = cs.step(u, v, w, e, e, e)
    for g in out["fgrid"]:
        assert g.shape == u.shape and not np.any(g)
    for k in ("u", "f", "n"):
        assert all(x.size == 0 for x in out[k])
    assert out["area"].size == 0
    fz = [np.zeros(0, dt) for _ in range(4)]
    for g in cs.lagr2eulr(e, e, e, *fz):
        assert not np.any(g)


@pytest.fixture(scope="module")
def big():
    wl = W.small_config(ncap=3, seed=19, grid=(128, 96, 64), degrees=(24, 28, 31))
    ref = O.coupling_step(wl.grid, wl.degree, wl.radius, *wl.velocity(), wl.x, wl.y, wl.z, wl.gs, wl.csk)
    return wl, ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_largest_degrees(cuda, big, precision):
    wl, ref = big
    dt = np.float64 if precision == "fp64" else np.float32
    u, v, w = (a.astype(dt) for a in wl.velocity())
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision)
    out = cs.step(u, v, w, wl.x, wl.y, wl.z)
    tol_f, tol_u = (1e-10, 1e-12) if precision == "fp64" else (1e-4, 1e-4)
    off = wl.offsets
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        for c in range(3):
            assert rel_l2(out["f"][c][s], ref["f"][c][s]) <= tol_f, (int(wl.degree[k]), c)
            assert rel_l2(out["n"][c][s], ref["n"][c][s]) <= tol_f, (int(wl.degree[k]), c)
        assert rel_l2(out["area"][s], ref["area"][s]) <= tol_f, int(wl.degree[k])
    for c in range(3):
        assert rel_l2(out["u"][c], ref["u"][c]) <= tol_u
        assert rel_l2(out["fgrid"][c], ref["fgrid"][c]) <= max(tol_f, tol_u)
