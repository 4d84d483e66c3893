"""surf_vol (surf_vol.f90:12-131) on the GPU against the oracle's restatement.

sg_surf_vol computes, per capsule in FP64: the centroid, the volume of the
1000-layer radial quadrature, the total area, exy1 from the inertia tensor's
principal moments and exy2 = (r_max - r_min) / (r_max + r_min).  The oracle's
or_surf_vol restates the same routine.  Both get the same positions, normals
and areas (the oracle's complagrforces of each capsule), so the test isolates
the integrals:

  - config 0 (one capsule, SH degree 15, perturbed sphere);
  - an uneven subset of config 2: one capsule of every degree it draws (7-18);
  - axis-aligned and tilted ellipsoids, so that exy1 takes both branches of
    the reference (a principal moment equal to Ixx sets it; otherwise the
    previous value exy1_prev is kept).

Tolerances: FP64 inputs, relative error <= 1e-12 for volume, area and
centroid, absolute <= 1e-12 for exy2 and <= 1e-10 for exy1.  exy1 comes from
the principal moments through the trigonometric cubic formula of the
reference, which is ill-conditioned when two moments nearly coincide (a
nearly spherical capsule): the GPU's tree sums and the oracle's sequential
sums differ in the last bits, and that difference reaches exy1 amplified by
the inverse gap between the moments (1.1e-11 observed).  FP32 normals and
areas (the mixed path's outputs): against the oracle on the same FP32 values
at the same tolerances, and against the FP64 inputs <= 1e-6.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep

pytestmark = pytest.mark.gpu

GRID = (64, 48, 40, 1.0 / 16, 1.0 / 16, 1.0 / 16)


def ellipsoid(L, R, centre, axes, tilt):
    """Points of an ellipsoid with semi-axes R * axes on the force grid of
    degree L, rotated by `tilt` radians about the z axis then the x axis."""
    th, _, ph = W.force_grid(L)
    T, P = np.meshgrid(th, ph, indexing="ij")
    p = np.stack([axes[0] * np.sin(T) * np.sin(P), axes[1] * np.sin(T) * np.cos(P), axes[2] * np.cos(T)]) * R
    c, s = np.cos(tilt), np.sin(tilt)
    rz = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    rx = np.array([[1.0, 0.0, 0.0], [0.0, c, -s], [0.0, s, c]])
    p = (rx @ rz @ p.reshape(3, -1))
    return [centre[q] + p[q] for q in range(3)]


def capsules():
    """(degree, radius, x, y, z) per capsule of the three cases."""
    out = []
    c0 = W.config0()
    out.append((15, float(c0.radius[0]), c0.x, c0.y, c0.z))
    c2 = W.config2()
    off = c2.offsets
    for L in sorted(set(c2.degree.tolist())):
        k = int(np.where(c2.degree == L)[0][0])
        s = slice(off[k], off[k + 1])
        out.append((L, float(c2.radius[k]), c2.x[s], c2.y[s], c2.z[s]))
    R = 0.3
    for axes, tilt in (((1.2, 0.9, 1.0), 0.0), ((1.15, 0.95, 0.9), 0.0), ((1.2, 0.9, 1.0), 0.4)):
        out.append((12, R, *ellipsoid(12, R, (1.5, 1.4, 1.2), axes, tilt)))
    return out


@pytest.fixture(scope="module")
def case():
    caps = capsules()
    degree = np.array([c[0] for c in caps], np.int32)
    radius = np.array([c[1] for c in caps])
    x = np.concatenate([c[2] for c in caps])
    y = np.concatenate([c[3] for c in caps])
    z = np.concatenate([c[4] for c in caps])
    nrm, area = [], []
    for L, R, cx, cy, cz in caps:
        _, n, a = O.complagrforces(L, R, cx, cy, cz, 1.0, 1.0)
        nrm.append(n)
        area.append(a)
    n = np.concatenate(nrm, axis=1)
    a = np.concatenate(area)
    exy_prev = np.linspace(0.01, 0.02, len(caps))  # distinct, so a kept value is recognisable
    return degree, radius, x, y, z, n, a, exy_prev


def oracle_rows(degree, x, y, z, n, a, exy_prev):
    off = np.concatenate([[0], np.cumsum([W.npts_of(int(L)) for L in degree])])
    rows = []
    for k in range(degree.size):
        s = slice(off[k], off[k + 1])
        rows.append(O.surf_vol(x[s], y[s], z[s], n[0][s], n[1][s], n[2][s], a[s], exy_prev[k]))
    return np.array(rows)


def check(got, ref, tol):
    # volume, area, centroid: relative; exy1, exy2: absolute
    for q in (0, 1, 4, 5, 6):
        assert np.abs(got[:, q] - ref[:, q]).max() <= tol * np.abs(ref[:, q]).max(), q
    assert np.abs(got[:, 3] - ref[:, 3]).max() <= max(tol, 1e-12)  # exy2
    assert np.abs(got[:, 2] - ref[:, 2]).max() <= max(tol, 1e-10)  # exy1


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_surf_vol_against_oracle(cuda, case, precision):
    degree, radius, x, y, z, n, a, exy_prev = case
    dt = np.float64 if precision == "fp64" else np.float32
    cs = CouplingStep(GRID, degree, radius, precision=precision)
    nn = [q.astype(dt) for q in n]
    aa = a.astype(dt)
    got = np.asarray(cs.surf_vol(x, y, z, *nn, aa, exy1_prev=exy_prev))
    # the oracle on the same (possibly FP32-rounded) inputs
    ref_same = oracle_rows(degree, x, y, z, [q.astype(np.float64) for q in nn], aa.astype(np.float64), exy_prev)
    check(got, ref_same, 1e-12)
    if precision == "mixed":  # against the FP64 inputs: the rounding of normals and areas only
        check(got, oracle_rows(degree, x, y, z, n, a, exy_prev), 1e-6)
    # both exy1 branches occur: the aligned ellipsoids set it, the tilted one keeps exy1_prev
    assert got[-1, 2] == exy_prev[-1]
    assert got[-3, 2] != exy_prev[-3] and got[-2, 2] != exy_prev[-2]

