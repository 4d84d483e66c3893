"""The overlap mesh's lid (interpolation.f90:10-69) through the C ABI: bitwise
the oracle's for random fields (FP64, host and device memory, nr = 2 and 4,
planes near the wall and at the top), and refusals of nr < 2 and of planes
outside the mesh."""
import numpy as np
import pytest

import oracle as O
from suguru_b200.coupling import CouplingStep, SgError

pytestmark = pytest.mark.gpu

GRID = (64, 48, 40, 1 / 16, 1 / 12, 1 / 20)


def _fields(seed):
    rng = np.random.default_rng(seed)
    shape = (GRID[2] + 2, GRID[1] + 2, GRID[0] + 2)
    return [rng.normal(size=shape) for _ in range(5)]


def _ctx(mem="host"):
    return CouplingStep(GRID, np.array([3], np.int32), np.array([0.1]), mem=mem)


@pytest.mark.parametrize("nf,nr", [(16, 2), (1, 4), (0, 2), (40, 2)])
def test_lid_equals_oracle(cuda, nf, nr):
    f = _fields(nf + nr)
    ref = O.overlap_lid(GRID, nf, nr, *f)
    got = _ctx().overlap_lid(nf, nr, *f)
    for g, r in zip(got, ref):
        assert g.shape == r.shape
        assert np.array_equal(g, r)


def test_device_memory(cuda):
    torch = cuda
    f = _fields(7)
    ref = O.overlap_lid(GRID, 16, 2, *f)
    got = _ctx("device").overlap_lid(16, 2, *[torch.from_numpy(a).cuda() for a in f])
    torch.cuda.synchronize()
    for g, r in zip(got, ref):
        assert np.array_equal(g.cpu().numpy(), r)


def test_refusals(cuda):
    f = _fields(8)
    cs = _ctx()
    for nf, nr in ((16, 1), (-1, 2), (41, 2)):
        with pytest.raises(SgError) as e:
            cs.overlap_lid(nf, nr, *f)
        assert e.value.code == 5  # SG_ERR_ARG
