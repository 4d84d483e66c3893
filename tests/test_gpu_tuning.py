"""Spreading tile shapes, the autotuner and CUDA-graph replay of the step.

Every tile shape must give the oracle's spread field within the path's
tolerance (FP64 relative L2 <= 1e-12, mixed <= 1e-4) and be bitwise
reproducible; the autotuner must leave the context on a valid shape with the
same results; a captured graph must reproduce sg_step bit for bit on the same
device arrays, also after their contents change.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import TILE_SHAPES, CouplingStep, SgError
from util import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    wl = W.small_config()
    rng = np.random.default_rng(21)
    f = rng.normal(size=(3, wl.npts))
    a = rng.uniform(0.5, 1.5, wl.npts) * wl.grid[3] ** 2
    ref = O.spread(wl.grid, wl.x, wl.y, wl.z, f[0], f[1], f[2], a)
    return wl, f, a, ref


@pytest.mark.parametrize("shape", range(len(TILE_SHAPES)))
def test_tile_shape_mixed(cuda, case, shape):
    wl, f, a, ref = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
    cs.set_tile_shape(shape)
    tx, ty, tz = TILE_SHAPES[shape]
    assert cs.tile_shape() == (shape, (tx or wl.grid[0], ty, tz))  # 0: whole x rows
    f32 = [x.astype(np.float32) for x in f]
    g1 = cs.lagr2eulr(wl.x, wl.y, wl.z, *f32, a.astype(np.float32))
    g2 = cs.lagr2eulr(wl.x, wl.y, wl.z, *f32, a.astype(np.float32))
    for x, y, r in zip(g1, g2, ref):
        assert np.array_equal(x, y)
        assert rel_l2(x, r) <= 1e-4


@pytest.mark.parametrize("shape", range(len(TILE_SHAPES)))
def test_tile_shape_fp64(cuda, case, shape):
    wl, f, a, ref = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    if shape not in (0, 3):  # three-limb FP64 accumulators: 32x8x4 and 8x8x4 tiles only
        with pytest.raises(SgError):
            cs.set_tile_shape(shape)
        return
    cs.set_tile_shape(shape)
    got = cs.lagr2eulr(wl.x, wl.y, wl.z, f[0].copy(), f[1].copy(), f[2].copy(), a)
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-12


def test_autotune_mixed(cuda):
    wl = W.small_config()
    u, v, w = (x.astype(np.float32) for x in wl.velocity())
    ref = O.coupling_step(wl.grid, wl.degree, wl.radius, *wl.velocity(), wl.x, wl.y, wl.z, wl.gs, wl.csk)
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
    best, ms = cs.autotune(u, v, w, wl.x, wl.y, wl.z, reps=2)
    assert 0 <= best < len(TILE_SHAPES) and ms > 0
    assert cs.tile_shape()[0] == best
    out = cs.step(u, v, w, wl.x, wl.y, wl.z)
    for c in range(3):
        assert rel_l2(out["fgrid"][c], ref["fgrid"][c]) <= 1e-4
        assert rel_l2(out["u"][c], ref["u"][c]) <= 1e-4


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay(cuda, precision):
    torch = cuda
    wl = W.small_config()
    dt = torch.float64 if precision == "fp64" else torch.float32
    dev = lambda a, t=dt: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", t)
    st = torch.cuda.Stream()
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision, mem="device",
                      stream=st.cuda_stream)
    u, v, w = (dev(x) for x in wl.velocity())
    X, Y, Z = (dev(x, torch.float64) for x in (wl.x, wl.y, wl.z))
    lag = [torch.zeros(wl.npts, dtype=dt, device="cuda") for _ in range(10)]
    eul = [torch.zeros_like(u) for _ in range(3)]
    torch.cuda.synchronize()  # inputs were written on torch's stream
    cs.step(u, v, w, X, Y, Z, lag_out=lag, eul_out=eul)
    torch.cuda.synchronize()
    want = [t.clone() for t in lag + eul]
    n_launch = cs.last_launch_count()
    cs.graph_capture(u, v, w, X, Y, Z, lag, eul)
    for t in lag + eul:
        t.fill_(float("nan"))
    torch.cuda.synchronize()
    cs.graph_launch()
    torch.cuda.synchronize()
    assert cs.last_launch_count() == n_launch
    for a, b in zip(lag + eul, want):
        assert torch.equal(a, b)
    # new contents, same arrays: the replay follows them
    u.mul_(0.5)
    X.add_(0.25 * wl.grid[3])
    torch.cuda.synchronize()
    cs.graph_launch()
    torch.cuda.synchronize()
    got = [t.clone() for t in lag + eul]
    cs.graph_release()
    cs.step(u, v, w, X, Y, Z, lag_out=lag, eul_out=eul)
    torch.cuda.synchronize()
    for a, b in zip(got, lag + eul):
        assert torch.equal(a, b)
    with pytest.raises(SgError):
        cs.graph_launch()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_point_split_does_not_change_results(cuda, precision):
    """Every capsule cut into 1, 2, 4 or 8 work items: bitwise the same step."""
    wl = W.small_config()
    dt = np.float64 if precision == "fp64" else np.float32
    u, v, w = (a.astype(dt) for a in wl.velocity())
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision=precision)
    outs = []
    for sp in (1, 2, 4, 8):
        cs.set_point_split(sp)
        assert cs.point_split() == sp
        o = cs.step(u, v, w, wl.x, wl.y, wl.z)
        outs.append([x.copy() for x in list(o["u"]) + list(o["f"]) + list(o["n"]) + [o["area"]] + list(o["fgrid"])])
    for o in outs[1:]:
        for a, b in zip(o, outs[0]):
            assert np.array_equal(a, b)
    with pytest.raises(SgError):
        cs.set_point_split(9)


def test_legendre_tile_rows_do_not_change_results(cuda):
    # 64-row tiles (M = 64 products, rows in the first half of each TMEM
    # quadrant) against 128-row tiles: every row is the same dot product
    wl = W.small_config()
    u, v, w = (a.astype(np.float32) for a in wl.velocity())
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
    cs.set_fused_force(False)  # the tensor-core contractions of the staged force stage
    assert cs.legendre_tile_rows() == 128
    a = cs.step(u, v, w, wl.x, wl.y, wl.z)
    a = {k: [x.copy() for x in val] if isinstance(val, tuple) or isinstance(val, list) else val.copy()
         for k, val in a.items()}
    cs.set_legendre_tile_rows(64)
    assert cs.legendre_tile_rows() == 64
    b = cs.step(u, v, w, wl.x, wl.y, wl.z)
    for k in ("u", "f", "n", "fgrid"):
        for x, y in zip(a[k], b[k]):
            assert np.array_equal(x, y), k
    assert np.array_equal(a["area"], b["area"])
    with pytest.raises(SgError):
        cs.set_legendre_tile_rows(96)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_with_bending_and_collisions(cuda, precision):
    # the captured step with every optional stage on: bending moduli (the
    # extra contraction launch and the bending membrane kernel) and the wall
    # force inside the step, capsules moved next to the bottom wall; the
    # replay gives the eager step's bits
    torch = cuda
    wl = W.small_config(ncap=3, seed=23, degrees=(7, 16, 11))
    dt = torch.float64 if precision == "fp64" else torch.float32
    dev = lambda a, t=dt: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", t)
    st = torch.cuda.Stream()
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision, mem="device",
                      stream=st.cuda_stream)
    cs.set_capsule_bending(0.3 * wl.gs * wl.radius**2)
    cs.set_wall_collisions(in_step=True)
    z = wl.z - wl.z.min() + 0.5 * wl.grid[5]  # the lowest point half a cell above the wall
    u, v, w = (dev(x) for x in wl.velocity())
    X, Y, Z = (dev(x, torch.float64) for x in (wl.x, wl.y, z))
    lag = [torch.zeros(wl.npts, dtype=dt, device="cuda") for _ in range(10)]
    eul = [torch.zeros_like(u) for _ in range(3)]
    torch.cuda.synchronize()
    cs.step(u, v, w, X, Y, Z, lag_out=lag, eul_out=eul)
    torch.cuda.synchronize()
    want = [t.clone() for t in lag + eul]
    cs.graph_capture(u, v, w, X, Y, Z, lag, eul)
    for t in lag + eul:
        t.fill_(float("nan"))
    torch.cuda.synchronize()
    cs.graph_launch()
    torch.cuda.synchronize()
    for a, b in zip(lag + eul, want):
        assert torch.equal(a, b)
    cs.graph_release()
