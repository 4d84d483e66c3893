"""sg_spread_noalloc: spreading for callers that cannot allocate device memory.

A host code whose device memory all belongs to its own pool, or code that may
not call cudaMalloc or create an sg_ctx, calls sg_spread_noalloc with its own
device arrays; the binning scratch is a fixed array inside the library.  This
test calls it through the C ABI twice in a row and compares each result with
the context-based sg_spread on the same inputs, at the FP64 spread tolerance
used by the parity tests (relative L2 <= 1e-12).  It lives in its own file,
collected last, and runs either alone or after the other tests.
"""
import ctypes

import numpy as np
import pytest

from suguru_b200 import coupling, workloads as W
from util import rel_l2

pytestmark = pytest.mark.gpu


def _spread_noalloc(torch, grid, X, Y, Z, F, A):
    itot, jtot, ktot, dx, dy, dz = grid
    shape = (ktot + 2, jtot + 2, itot + 2)
    out = [torch.full(shape, float("nan"), dtype=torch.float64, device="cuda") for _ in range(3)]
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = coupling.lib().sg_spread_noalloc(itot, jtot, ktot, itot * dx, jtot * dy, ktot * dz, X.numel(),
                                          p(X), p(Y), p(Z), p(F[0]), p(F[1]), p(F[2]), p(A),
                                          p(out[0]), p(out[1]), p(out[2]), None)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return [o.cpu().numpy() for o in out]


def test_spread_noalloc_matches_context_spread(cuda):
    torch = cuda
    wl = W.small_config()
    rng = np.random.default_rng(11)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    X, Y, Z = dev(wl.x), dev(wl.y), dev(wl.z)
    cs = coupling.CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64", mem="device")
    for call in range(2):  # two calls in a row share the scratch array
        F = [dev(rng.normal(size=wl.npts)) for _ in range(3)]
        A = dev(rng.uniform(0.5, 1.5, wl.npts) * wl.grid[3] ** 2)
        ref = [o.cpu().numpy() for o in cs.lagr2eulr(X, Y, Z, F[0], F[1], F[2], A)]
        got = _spread_noalloc(torch, wl.grid, X, Y, Z, F, A)
        for g, r in zip(got, ref):
            assert np.isfinite(g).all()
            assert rel_l2(g, r) <= 1e-12, call


def test_spread_noalloc_rejects_oversize(cuda):
    torch = cuda
    wl = W.small_config()
    itot, jtot, ktot, dx, dy, dz = wl.grid
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    too_many = 65536 + 1  # SG_NOALLOC_MAX_POINTS + 1: rejected before any device work
    rc = coupling.lib().sg_spread_noalloc(itot, jtot, ktot, itot * dx, jtot * dy, ktot * dz, too_many,
                                          p, p, p, p, p, p, p, p, p, p, None)
    assert rc == 7  # SG_ERR_TOO_LARGE


def test_spread_noalloc_rejects_too_many_tiles(cuda):
    # 512 x 256 x 256 cells on 32x8x4 tiles: 32768 tiles > SG_NOALLOC_MAX_TILES
    # (16384).  The arrays are real and of full size, although the call
    # refuses on the host before it queues anything.
    torch = cuda
    itot, jtot, ktot, dx = 512, 256, 256, 1.0 / 32
    fld = [torch.zeros((ktot + 2, jtot + 2, itot + 2), dtype=torch.float64, device="cuda") for _ in range(3)]
    pts = torch.full((7, 64), 1.0, dtype=torch.float64, device="cuda")
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    rc = coupling.lib().sg_spread_noalloc(itot, jtot, ktot, itot * dx, jtot * dx, ktot * dx, 64,
                                          *[p(pts[q]) for q in range(7)], p(fld[0]), p(fld[1]), p(fld[2]), None)
    assert rc == 7  # SG_ERR_TOO_LARGE
    torch.cuda.synchronize()
    assert all(float(f.abs().max()) == 0.0 for f in fld)  # nothing was written

