"""The indicator function (indicator.f90:19-182) on the GPU against the oracle.

Capsules from the small mixed-degree batch (some across the periodic faces)
and a sphere; normals and areas from the oracle's complagrforces, so that
only the indicator itself is compared:

  - FP64: G (the lagr2eulrind spread) is exercised through the result;
    indic, visc and the centrifugal terms added to fy, fz match the oracle
    to 1e-10 of their largest value (the Poisson solve runs through cuFFT
    against numpy's FFT), leaving out the few cells whose value before the
    0.01 / 0.9 thresholds lies within 10 times the tolerance of one;
  - mixed: FP32 inputs and outputs, the same computation in FP64 inside,
    within 1e-6;
  - the sphere's indicator integrates to its volume within 3 %;
  - host and device memory give the same bits;
  - sg_indicator before sg_set_indicator_params is refused.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep, SgError

pytestmark = pytest.mark.gpu

PARAMS = dict(visc0=2.0, lam=5.0, thetainc=70.0 * np.pi / 180.0, ta=1160000.0, rep=0.0016)


def _normals(wl):
    off = wl.offsets
    N = np.zeros((3, wl.npts))
    A = np.zeros(wl.npts)
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        _, n, a = O.complagrforces(int(wl.degree[k]), float(wl.radius[k]), wl.x[s], wl.y[s], wl.z[s])
        N[:, s], A[s] = n, a
    return N, A


@pytest.fixture(scope="module")
def case():
    wl = W.small_config(ncap=3, grid=(64, 48, 40))
    N, A = _normals(wl)
    rng = np.random.default_rng(9)
    shape = (wl.grid[2] + 2, wl.grid[1] + 2, wl.grid[0] + 2)
    fy0, fz0 = rng.normal(size=shape), rng.normal(size=shape)
    ref = O.indicator(wl.grid, wl.x, wl.y, wl.z, *N, A, fy=fy0, fz=fz0, **PARAMS)
    return wl, N, A, fy0, fz0, ref


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_indicator_against_oracle(cuda, case, precision):
    wl, N, A, fy0, fz0, ref = case
    dt = np.float64 if precision == "fp64" else np.float32
    tol = 1e-10 if precision == "fp64" else 1e-6
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision)
    cs.set_indicator_params(**PARAMS)
    fy, fz = fy0.astype(dt), fz0.astype(dt)
    indic, visc = cs.indicator(wl.x, wl.y, wl.z, *(n.astype(dt) for n in N), A.astype(dt), fy=fy, fz=fz)
    assert ref["indic"].max() == 1.0  # the capsules' interiors reach the upper threshold
    # cells whose value before the thresholds lies within rounding of 0.01 or 0.9 may be
    # thresholded differently by the two sides; they (and the terms that read them) are left out
    kt, q = wl.grid[2], wl.grid[2] // 4
    raw = np.zeros_like(ref["indi"])
    raw[1:kt - q + 1, 1:-1, 1:-1] = ref["indi"][1 + q:kt + 1, 1:-1, 1:-1]
    O.boundp(raw)
    eps = 10 * tol
    near = (np.abs(raw - 0.01) < eps) | (np.abs(raw - 0.9) < eps)
    near_y = near.copy()
    near_y[:, :-1, :] |= near[:, 1:, :]
    near_z = near.copy()
    near_z[:-1] |= near[1:]
    for got, want, skip in ((indic, ref["indic"], near), (visc, ref["visc"], near), (fy, ref["fy"], near_y),
                            (fz, ref["fz"], near_z)):
        err = np.abs(np.asarray(got, np.float64) - want)[~skip]
        assert err.max() <= tol * np.abs(want).max(), err.max()
    assert near.mean() < 1e-3


def test_sphere_volume(cuda):
    dx = 1.0 / 16
    grid = (48, 48, 48, dx, dx, dx)
    R, L = 7 * dx, 11
    x, y, z = W.capsule_points(L, R, np.array([1.5, 1.5, 1.3]))
    _, n, a = O.complagrforces(L, R, x, y, z)
    cs = CouplingStep(grid, np.array([L], np.int32), np.array([R]), precision="fp64")
    cs.set_indicator_params(**PARAMS)
    indic, _ = cs.indicator(x, y, z, *n, a)
    vol = indic[1:-1, 1:-1, 1:-1].sum() * dx ** 3
    assert abs(vol - 4 / 3 * np.pi * R ** 3) <= 0.03 * 4 / 3 * np.pi * R ** 3


def test_refused_before_setup(cuda, case):
    wl, N, A = case[:3]
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    with pytest.raises(SgError) as e:
        cs.indicator(wl.x, wl.y, wl.z, *N, A)
    assert e.value.code == 6


def test_device_memory_same_bits(cuda, case):
    torch = cuda
    wl, N, A, fy0, fz0, _ = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    cs.set_indicator_params(**PARAMS)
    fy, fz = fy0.copy(), fz0.copy()
    ih, vh = cs.indicator(wl.x, wl.y, wl.z, *N, A, fy=fy, fz=fz)
    cd = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64", mem="device")
    cd.set_indicator_params(**PARAMS)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    fyd, fzd = dev(fy0), dev(fz0)
    idv, vdv = cd.indicator(*map(dev, (wl.x, wl.y, wl.z)), *map(dev, N), dev(A), fy=fyd, fz=fzd)
    torch.cuda.synchronize()
    for h, d in ((ih, idv), (vh, vdv), (fy, fyd), (fz, fzd)):
        assert np.array_equal(h, d.cpu().numpy())
