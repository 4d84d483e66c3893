"""The fused force stage of the mixed path (one kernel, one CTA per capsule;
opt-in through sg_set_fused_force).

  - bit for bit the staged force stage with its contractions on CUDA cores
    (sg_set_tensor_cores(0)): the pointwise stages are the same device code
    and the per-capsule contraction sums in the same order of k as the
    staged CUDA-core kernel; uneven degrees 2..23 in one batch;
  - against the oracle within the mixed path's 1e-4 (the FP32 contractions
    make it FP32-level: 2e-5 per capsule);
  - one launch for the whole stage;
  - capsules that bend take the staged stage: the step is the same bits
    with the fused stage switched on or off;
  - FP64 contexts refuse it.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import workloads as W
from suguru_b200.coupling import CouplingStep, SgError
from util import rel_l2

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    wl = W.small_config(ncap=6, seed=41, grid=(96, 64, 48), degrees=(2, 8, 15, 16, 22, 23))
    ref = O.coupling_step(wl.grid, wl.degree, wl.radius, *wl.velocity(), wl.x, wl.y, wl.z, wl.gs, wl.csk)
    return wl, ref


def _step(cs, wl):
    u, v, w = (a.astype(np.float32) for a in wl.velocity())
    out = cs.step(u, v, w, wl.x, wl.y, wl.z)
    return {k: ([x.copy() for x in val] if isinstance(val, (list, tuple)) else val.copy()) for k, val in out.items()}


def test_fused_equals_staged_cuda_core(cuda, case):
    wl, _ = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
    assert not cs.fused_force()  # the staged stage is the default
    cs.set_fused_force(True)
    a = _step(cs, wl)
    n_fused = cs.last_launch_count()
    cs.set_fused_force(False)
    cs.set_tensor_cores(False)
    b = _step(cs, wl)
    n_staged = cs.last_launch_count()
    for k in ("u", "f", "n", "fgrid"):
        for x, y in zip(a[k], b[k]):
            assert np.array_equal(x, y), k
    assert np.array_equal(a["area"], b["area"])
    assert n_fused < n_staged


def test_fused_against_oracle(cuda, case):
    wl, ref = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
    cs.set_fused_force(True)
    out = _step(cs, wl)
    off = wl.offsets
    for k in range(wl.ncap):
        s = slice(off[k], off[k + 1])
        for c in range(3):
            assert rel_l2(out["f"][c][s], ref["f"][c][s]) <= 2e-5, (int(wl.degree[k]), c)
            assert rel_l2(out["n"][c][s], ref["n"][c][s]) <= 2e-5, (int(wl.degree[k]), c)
        assert rel_l2(out["area"][s], ref["area"][s]) <= 2e-5, int(wl.degree[k])
    for c in range(3):
        assert rel_l2(out["u"][c], ref["u"][c]) <= 1e-4
        assert rel_l2(out["fgrid"][c], ref["fgrid"][c]) <= 1e-4


def test_bending_takes_the_staged_stage(cuda, case):
    wl, _ = case
    eb = 0.3 * wl.gs * wl.radius**2
    outs = []
    for fused in (True, False):
        cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="mixed")
        cs.set_fused_force(fused)
        cs.set_capsule_bending(eb)
        outs.append(_step(cs, wl))
    for k in ("f", "n", "fgrid"):
        for x, y in zip(outs[0][k], outs[1][k]):
            assert np.array_equal(x, y), k


def test_fp64_refuses(cuda, case):
    wl, _ = case
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, precision="fp64")
    assert not cs.fused_force()
    with pytest.raises(SgError):
        cs.set_fused_force(True)
