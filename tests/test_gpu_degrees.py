"""Uneven SH degrees in one context (the config-2 shape of work, small).

Capsules of degree 2, 8 (odd N = 9), 16 (N = 17), 22 and 23 (N = 24: the
largest tensor-core operands, J = 3 nD = 144 columns, 256 TMEM columns) are
stepped together.  FP64 against the oracle at the FP64 tolerances, mixed
within 1e-4 for every capsule, for every capsule split of the persistent
kernels, with the mixed path's force stage fused (one kernel per capsule,
FP32 contractions) and staged (tensor cores).  The staged mixed path's
automatic split mode runs degrees >= 16 in BF16x6:
forced to BF16x3, the degree-22 capsule's force error exceeds 1e-4 (the
second derivatives of the shape amplify the ~2^-17 product error about as
L^2), which the last test shows.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep
from util import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    wl = W.small_config(ncap=5, seed=17, grid=(96, 64, 48), degrees=(2, 8, 16, 22, 23))
    ref = O.coupling_step(wl.grid, wl.degree, wl.radius, *wl.velocity(), wl.x, wl.y, wl.z, wl.gs, wl.csk)
    return wl, ref


@pytest.mark.parametrize("precision,fused", [("fp64", False), ("mixed", False), ("mixed", True)])
@pytest.mark.parametrize("split", [1, 8])
def test_uneven_degrees(cuda, case, precision, fused, split):
    wl, ref = case
    dt = np.float64 if precision == "fp64" else np.float32
    u, v, w = (a.astype(dt) for a in wl.velocity())
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision)
    if precision == "mixed":
        cs.set_fused_force(fused)
    cs.set_point_split(split)
    out = cs.step(u, v, w, wl.x, wl.y, wl.z)
    tol_f, tol_u = (1e-10, 1e-12) if precision == "fp64" else (1e-4, 1e-4)
    off = wl.offsets
    for k in range(wl.ncap):  # every degree on its own
        s = slice(off[k], off[k + 1])
        for c in range(3):
            assert rel_l2(out["f"][c][s], ref["f"][c][s]) <= tol_f, (int(wl.degree[k]), c)
            assert rel_l2(out["n"][c][s], ref["n"][c][s]) <= tol_f, (int(wl.degree[k]), c)
        assert rel_l2(out["area"][s], ref["area"][s]) <= tol_f, int(wl.degree[k])
    for c in range(3):
        assert rel_l2(out["u"][c], ref["u"][c]) <= tol_u
        assert rel_l2(out["fgrid"][c], ref["fgrid"][c]) <= max(tol_f, tol_u)


def _force_errors(wl, ref, out):
    off = wl.offsets
    return {int(wl.degree[k]): max(rel_l2(out["f"][c][off[k]:off[k + 1]], ref["f"][c][off[k]:off[k + 1]])
                                   for c in range(3)) for k in range(wl.ncap)}


def test_split_modes(cuda, case):
    wl, ref = case
    u, v, w = (a.astype(np.float32) for a in wl.velocity())
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
    cs.set_fused_force(False)  # the staged force stage, contractions on the tensor cores
    assert [cs.legendre_terms(L) for L in (2, 15, 16, 23)] == [3, 3, 6, 6]
    err = {}
    for terms in (3, 6):
        cs.set_legendre_terms(terms)
        err[terms] = _force_errors(wl, ref, cs.step(u, v, w, wl.x, wl.y, wl.z))
    print(err)
    assert max(err[6].values()) <= 2e-5       # FP32-level at every degree
    assert err[3][22] > 1e-4                   # why the automatic mode switches at high degree
    assert err[3][22] > 10 * err[6][22]
    cs.set_legendre_terms(0)
    assert cs.legendre_terms(22) == 6 and cs.legendre_terms(8) == 3
