"""Bending (ibend = 1; sph.f90:479-731, 1236-1454, 1705-1709) through the C
ABI against the oracle.

A batch of five capsules of four degrees with per-capsule bending moduli (one
of them 0) must give, capsule by capsule, the oracle's force, normals and area for its own
modulus: FP64 within 1e-10, mixed within 1e-4 (relative L2).  The modulus is
the reference's ebend = cbend gscell (param.f90:90-91, cbend = 0.3) in units
of the capsule radius, eb = cbend gs R^2.  Setting every modulus back to 0
gives the plain force bit for bit; bending capsules never take the
surrogate; a non-finite modulus is refused.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep, SgError
from util import rel_l2

pytestmark = pytest.mark.gpu

CBEND = np.array([0.3, 0.0, 0.3, 0.05, 1.0])


@pytest.fixture(scope="module")
def case():
    wl = W.small_config(ncap=5, seed=29, grid=(64, 48, 40), degrees=(7, 11, 15, 16, 23))
    eb = CBEND * wl.gs * wl.radius**2
    off = wl.offsets
    ref = []
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        ref.append(O.complagrforces(int(wl.degree[k]), float(wl.radius[k]), wl.x[s], wl.y[s], wl.z[s],
                                    wl.gs, wl.csk, eb=float(eb[k])))
    return wl, eb, ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bending_batch(cuda, case, precision):
    wl, eb, ref = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    cs.set_capsule_bending(eb)
    f, n, a = cs.complagrforces(wl.x, wl.y, wl.z)
    tol = 1e-10 if precision == "fp64" else 1e-4
    off = wl.offsets
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        fr, nr, ar = ref[k]
        for c in range(3):
            assert rel_l2(f[c][s], fr[c]) <= tol, (k, c, rel_l2(f[c][s], fr[c]))
            assert rel_l2(n[c][s], nr[c]) <= tol, (k, c)
        assert rel_l2(a[s], ar) <= tol, k


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bending_in_the_coupling_step(cuda, case, precision):
    # interp -> force with bending -> spread, against the oracle's force
    # spread onto the grid
    wl, eb, ref = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
    cs.set_capsule_bending(eb)
    dt = np.float64 if precision == "fp64" else np.float32
    out = cs.step(*(u.astype(dt) for u in wl.velocity()), wl.x, wl.y, wl.z)
    fref = np.concatenate([r[0] for r in ref], axis=1)
    aref = np.concatenate([r[2] for r in ref])
    Fref = O.spread(wl.grid, wl.x, wl.y, wl.z, fref[0], fref[1], fref[2], aref)
    tol = 1e-10 if precision == "fp64" else 1e-4
    for c in range(3):
        assert rel_l2(out["f"][c], fref[c]) <= tol
        assert rel_l2(out["fgrid"][c], Fref[c]) <= tol


def test_zero_modulus_is_the_plain_force(cuda, case):
    wl, eb, _ = case
    for precision in ("fp64", "mixed"):
        plain = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
        f0 = [x.copy() for x in plain.complagrforces(wl.x, wl.y, wl.z)[0]]
        cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision)
        terms = [cs.legendre_terms(d) for d in wl.degree]
        cs.set_capsule_bending(eb)
        cs.complagrforces(wl.x, wl.y, wl.z)
        cs.set_capsule_bending(0.0)
        assert [cs.legendre_terms(d) for d in wl.degree] == terms
        f1 = cs.complagrforces(wl.x, wl.y, wl.z)[0]
        for c in range(3):
            assert np.array_equal(f0[c], f1[c]), (precision, c)


def test_bending_capsules_never_take_the_surrogate(cuda):
    # four L = 15 capsules on a surrogate context with a nonzero linear
    # response, its network marked ready (its parameters written back as they
    # are) and trust limits that admit everything: exactly the two capsules
    # without bending take it
    wl = W.small_config(ncap=4, seed=31, grid=(64, 48, 40), degrees=(15,))
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="mixed", surrogate=True)
    n = 3 * 16 * 16
    cs.surrogate_set_linear(np.eye(n, dtype=np.float32), np.zeros((n, n), np.float32))
    cs.surrogate_params(cs.surrogate_params())
    cs.surrogate_set_trust(1e30, 1e30)
    vel = [u.astype(np.float32) for u in wl.velocity()]
    cs.step(*vel, wl.x, wl.y, wl.z)
    assert cs.surrogate_counts() == (4, 0)
    eb = np.array([0.0, 0.3, 0.0, 0.1]) * wl.gs * wl.radius**2
    cs.set_capsule_bending(eb)
    cs.step(*vel, wl.x, wl.y, wl.z)
    assert cs.surrogate_counts() == (2, 2)


def test_non_finite_modulus_is_refused(cuda, case):
    wl, eb, _ = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="fp64")
    bad = eb.copy()
    bad[1] = np.nan
    with pytest.raises(SgError):
        cs.set_capsule_bending(bad)
