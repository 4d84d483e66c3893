"""CPU known-answer tests of the oracle's bending terms (ibend = 1,
sph.f90:479-731, 1236-1454, 1705-1709; param.f90:90-91).

The reference's moment law M = eb (B_ref - b) (mixed with the contravariant
metric, sph.f90:1258-1290) has a classical small-deformation limit on a
sphere of radius R: for a radial displacement w = eps R Pbar_l^0(theta) the
bending part of the load is, to first order in eps,

    normal      eb l(l+1)(l-1)(l+2) / R^4  w          (along the inward normal)
    tangential  eb (l(l+1) - 2) / R^4  dw/dtheta      (along e_theta)

(the operator eb (lap^2 + 2 lap / R^2) w of a pre-curved shell, and the
curvature times the transverse shear Q for the in-plane part).  A rigid
translation (l = 1) bends nothing; a uniform dilation changes the moment
uniformly, so it has no transverse shear and leaves the Laplace-law force
unchanged; the reference sphere carries no force at all.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W

L, R, EB = 15, 0.25, 0.3


def _mode(l, eps):
    ca = np.zeros((L + 1, L + 1))
    cb = np.zeros((L + 1, L + 1))
    ca[0, l] = eps * R
    x, y, z = W.capsule_points(L, R, (1.0, 1.0, 1.0), ca, cb)
    w = W.shape_radius(L, R, ca, cb).ravel() - R
    f1, n1, _ = O.complagrforces(L, R, x, y, z, eb=EB)
    f0, _, _ = O.complagrforces(L, R, x, y, z, eb=0.0)
    return f1 - f0, n1, w


def test_reference_sphere_carries_no_bending_force():
    x, y, z = W.capsule_points(L, R, (2.0, 1.0, 1.0))
    f, _, _ = O.complagrforces(L, R, x, y, z, eb=EB)
    assert np.abs(f).max() < 1e-8 * EB / R**3


@pytest.mark.parametrize("lam", [0.95, 1.1])
def test_uniform_dilation_bends_nothing(lam):
    x, y, z = W.capsule_points(L, lam * R, (1.0, 1.0, 1.0))
    f1, _, _ = O.complagrforces(L, R, x, y, z, gs=1.3, eb=EB)
    f0, _, _ = O.complagrforces(L, R, x, y, z, gs=1.3)
    assert np.abs(f1 - f0).max() < 1e-7 * np.abs(f0).max()


@pytest.mark.parametrize("l", [2, 3, 4, 6])
def test_linear_normal_load(l):
    eps = 1e-5
    df, n, w = _mode(l, eps)
    dn = (df * n).sum(0)
    mask = np.abs(w) > 0.3 * np.abs(w).max()
    ratio = dn[mask] / w[mask]
    pred = EB * l * (l + 1) * (l - 1) * (l + 2) / R**4
    assert abs(ratio.mean() / pred - 1) < 1e-4
    assert ratio.std() / pred < 1e-3


# Pbar_l^0 up to a constant, and its theta derivative (c = cos, s = sin)
_P = {2: (lambda c: 3 * c * c - 1, lambda c, s: -6 * c * s),
      3: (lambda c: 5 * c**3 - 3 * c, lambda c, s: -(15 * c * c - 3) * s)}


@pytest.mark.parametrize("l", [2, 3])
def test_linear_tangential_load(l):
    eps = 1e-5
    df, _, w = _mode(l, eps)
    th, _, ph = W.force_grid(L)
    T, PH = np.meshgrid(th, ph, indexing="ij")
    c, s, PH = np.cos(T).ravel(), np.sin(T).ravel(), PH.ravel()
    dw = w * _P[l][1](c, s) / _P[l][0](c)
    et = np.stack([c * np.sin(PH), c * np.cos(PH), -s])
    ft = (df * et).sum(0)
    mask = np.abs(dw) > 0.3 * np.abs(dw).max()
    ratio = ft[mask] / dw[mask]
    pred = EB * (l * (l + 1) - 2) / R**4
    assert abs(ratio.mean() / pred - 1) < 1e-4
    assert ratio.std() / pred < 1e-3


def test_translation_bends_nothing():
    # l = 1 is a rigid shift to first order: what bending load it has is of
    # second order (about 0.3 eps of the l = 2 load of the same amplitude)
    df1, _, _ = _mode(1, 1e-5)
    df2, _, _ = _mode(2, 1e-5)
    assert np.abs(df1).max() < 1e-4 * np.abs(df2).max()


def test_bending_is_linear_in_the_modulus():
    rng = np.random.default_rng(5)
    ca, cb = W.random_shape(rng, L, 0.05 * R)
    x, y, z = W.capsule_points(L, R, (1.0, 1.0, 1.0), ca, cb)
    f0, _, _ = O.complagrforces(L, R, x, y, z)
    f1, _, _ = O.complagrforces(L, R, x, y, z, eb=EB)
    f2, _, _ = O.complagrforces(L, R, x, y, z, eb=2 * EB)
    assert np.abs((f2 - f0) - 2 * (f1 - f0)).max() < 1e-9 * np.abs(f1 - f0).max()
