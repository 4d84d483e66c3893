"""Spreading on grids whose sizes are not multiples of the tile, and into
fields that do not start on an aligned address.

  - ragged grids (last tile in x or y narrower than the tile, down to 3
    cells) give the oracle's field;
  - a grid whose every tile shape would leave a last tile of 1 or 2 cells in
    a periodic dimension is refused at set-up (a stencil that wraps around
    the periodic end could reach three tiles there, and the binning records
    two per dimension);
  - output arrays offset by one element from an aligned allocation give the
    same field, bit for bit, as aligned ones, and nothing is written outside.
Tolerances: FP64 relative L2 <= 1e-12, mixed <= 1e-4 (the path tolerances).
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep, SgError
from util import rel_l2

pytestmark = pytest.mark.gpu


def _case(grid, seed=31):
    wl = W.small_config(grid=grid)
    rng = np.random.default_rng(seed)
    f = rng.normal(size=(3, wl.npts))
    a = rng.uniform(0.5, 1.5, wl.npts) * wl.grid[3] ** 2
    ref = O.spread(wl.grid, wl.x, wl.y, wl.z, f[0], f[1], f[2], a)
    return wl, f, a, ref


@pytest.mark.parametrize("grid", [(61, 45, 40), (67, 53, 37), (75, 48, 40), (35, 43, 37)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_ragged_grids(cuda, grid, precision):
    wl, f, a, ref = _case(grid)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision)
    dt = np.float64 if precision == "fp64" else np.float32
    tol = 1e-12 if precision == "fp64" else 1e-4
    got = cs.lagr2eulr(wl.x, wl.y, wl.z, *(x.astype(dt) for x in f), a.astype(dt))
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= tol


def test_grid_without_a_valid_tile_shape_is_refused(cuda):
    # 66 = 2 mod 8, 16 and 32: every tile shape leaves a 2-cell last tile in x
    wl = W.small_config()
    grid = (66,) + tuple(wl.grid[1:])
    with pytest.raises(SgError):
        CouplingStep(grid, wl.degree, wl.radius, precision="fp64")


def test_grid_only_a_wide_tile_fits(cuda):
    # jtot = 25 = 1 mod 8: of the tile shapes only 16x16x8 fits, which the
    # FP32 spread has and the FP64 spread (at most 1024 cells per tile) has
    # not.  The FP64 context is refused at set-up with SG_ERR_CONFIG, before
    # any launch; the mixed context spreads on 16x16x8 tiles and matches the
    # oracle.
    grid = (64, 25, 40)
    wl, f, a, ref = _case(grid, seed=33)
    with pytest.raises(SgError) as e:
        CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    assert e.value.code == 1  # SG_ERR_CONFIG
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
    assert cs.tile_shape()[1] == (16, 16, 8)
    got = cs.lagr2eulr(wl.x, wl.y, wl.z, *(x.astype(np.float32) for x in f), a.astype(np.float32))
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_unaligned_output_fields(cuda, precision):
    torch = cuda
    wl, f, a, ref = _case((64, 48, 40), seed=32)
    td = torch.float64 if precision == "fp64" else torch.float32
    dt = np.float64 if precision == "fp64" else np.float32
    dev = torch.device("cuda", 0)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision, mem="device")
    X = [torch.from_numpy(x).to(dev) for x in (wl.x, wl.y, wl.z)]
    F = [torch.from_numpy(x.astype(dt)).to(dev) for x in f]
    A = torch.from_numpy(a.astype(dt)).to(dev)
    shape = cs.field_shape
    n = int(np.prod(shape))
    aligned = [torch.empty(shape, dtype=td, device=dev) for _ in range(3)]
    bufs = [torch.full((n + 1,), 7.0, dtype=td, device=dev) for _ in range(3)]
    shifted = [b[1:].view(shape) for b in bufs]  # one element past a 256-byte boundary
    cs.lagr2eulr(*X, *F, A, out=aligned)
    cs.lagr2eulr(*X, *F, A, out=shifted)
    torch.cuda.synchronize()
    tol = 1e-12 if precision == "fp64" else 1e-4
    for g, s, b, r in zip(aligned, shifted, bufs, ref):
        assert torch.equal(g, s)
        assert float(b[0]) == 7.0  # nothing written before the field
        assert rel_l2(g.cpu().numpy(), r) <= tol


@pytest.mark.parametrize("shape", [4, 5])
@pytest.mark.parametrize("grid", [(61, 47, 40), (67, 51, 37), (64, 48, 40)])
def test_row_tiles(cuda, grid, shape):
    # whole-x-row tiles (FP32): ragged y and z, periodic x inside the tile,
    # halos written row by row; into an output shifted off its alignment, with
    # nothing written outside the field; bitwise equal on a repeat
    torch = cuda
    wl, f, a, ref = _case(grid, seed=34)
    dev = torch.device("cuda", 0)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed", mem="device")
    cs.set_tile_shape(shape)
    X = [torch.from_numpy(x).to(dev) for x in (wl.x, wl.y, wl.z)]
    F = [torch.from_numpy(x.astype(np.float32)).to(dev) for x in f]
    A = torch.from_numpy(a.astype(np.float32)).to(dev)
    n = int(np.prod(cs.field_shape))
    bufs = [torch.full((n + 2,), 7.0, dtype=torch.float32, device=dev) for _ in range(3)]
    shifted = [b[1:n + 1].view(cs.field_shape) for b in bufs]
    cs.lagr2eulr(*X, *F, A, out=shifted)
    again = [o.clone() for o in cs.lagr2eulr(*X, *F, A)]
    torch.cuda.synchronize()
    for s_, b, g2, r in zip(shifted, bufs, again, ref):
        assert float(b[0]) == 7.0 and float(b[-1]) == 7.0
        assert torch.equal(s_, g2)
        assert rel_l2(s_.cpu().numpy(), r) <= 1e-4



@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dense_tiles(cuda, precision):
    # 24,576 points inside a box of 2 x 2 x 2 cells, so that a handful of
    # tiles hold up to 24,576 entries each: the FP64 limbs are folded over
    # several passes of 4,096 contributions, and the FP32 scales take the
    # exact integer sum bound of dense tiles; forces of mixed magnitudes
    dx = 1.0 / 16
    grid = (64, 48, 40, dx, dx, dx)
    degree = np.array([31, 31, 31], np.int32)  # 8 (L + 1)^2 = 8192 points each
    radius = np.full(3, 0.25)
    n = int(np.sum(8 * (degree + 1) ** 2))
    rng = np.random.default_rng(37)
    x = (20.3 + rng.uniform(0.0, 2.0, n)) * dx
    y = (10.2 + rng.uniform(0.0, 2.0, n)) * dx
    z = (17.6 + rng.uniform(0.0, 2.0, n)) * dx
    f = rng.normal(size=(3, n)) * rng.choice([1e-3, 1.0, 30.0], size=(3, n))
    a = rng.uniform(0.5, 1.5, n) * dx**2
    ref = O.spread(grid, x, y, z, f[0], f[1], f[2], a)
    cs = CouplingStep(grid, degree, radius, precision=precision)
    dt = np.float64 if precision == "fp64" else np.float32
    tol = 1e-12 if precision == "fp64" else 1e-4
    args = (x, y, z, *(v.astype(dt) for v in f), a.astype(dt))
    got = [g.copy() for g in cs.lagr2eulr(*args)]
    again = cs.lagr2eulr(*args)
    for g, g2, r in zip(got, again, ref):
        assert np.array_equal(g, g2)
        assert rel_l2(g, r) <= tol
