"""Membrane laws per capsule: Skalak and neo-Hookean (membmodel.c:60-99; the
reference picks one at compile time, -DSKALAK or -DNONHOOK).

A batch that mixes the two laws must give, capsule by capsule, the oracle's
force, normals and area for each capsule's own law: FP64 within 1e-10, mixed
within 1e-4 (relative L2).  Switching one capsule's law leaves every other
capsule's force bit for bit unchanged.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep, SgError
from util import rel_l2

pytestmark = pytest.mark.gpu

LAWS = np.array([1, 0, 1, 1], dtype=np.int32)  # neo-Hookean, Skalak, neo-Hookean, neo-Hookean


@pytest.fixture(scope="module")
def case():
    wl = W.small_config(ncap=4, seed=23, grid=(64, 48, 40), degrees=(7, 11, 15, 16))
    off = wl.offsets
    ref = []
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        ref.append(O.complagrforces(int(wl.degree[k]), float(wl.radius[k]), wl.x[s], wl.y[s], wl.z[s],
                                    wl.gs, wl.csk, law=int(LAWS[k])))
    return wl, ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_mixed_law_batch(cuda, case, precision):
    wl, ref = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    cs.set_capsule_law(LAWS)
    f, n, a = cs.complagrforces(wl.x, wl.y, wl.z)
    tol = 1e-10 if precision == "fp64" else 1e-4
    off = wl.offsets
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        fr, nr, ar = ref[k]
        for c in range(3):
            assert rel_l2(f[c][s], fr[c]) <= tol, (k, c)
            assert rel_l2(n[c][s], nr[c]) <= tol, (k, c)
        assert rel_l2(a[s], ar) <= tol, k


def test_law_is_per_capsule(cuda, case):
    wl, _ = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="fp64")
    f0, _, _ = cs.complagrforces(wl.x, wl.y, wl.z)
    f0 = [x.copy() for x in f0]
    law = np.zeros(wl.ncap, np.int32)
    law[2] = 1
    cs.set_capsule_law(law)
    f1, _, _ = cs.complagrforces(wl.x, wl.y, wl.z)
    off = wl.offsets
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        same = all(np.array_equal(f0[c][s], f1[c][s]) for c in range(3))
        assert same == (k != 2), k
    with pytest.raises(SgError):
        cs.set_capsule_law(np.full(wl.ncap, 2, np.int32))
