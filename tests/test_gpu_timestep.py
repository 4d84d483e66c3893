"""Time-stepped coupling (config 4 on a small case): prescribed flow, Update_Pos.

1. The GPU evaluation of the prescribed time-varying flow equals the numpy
   form (workloads.velocity_field) to 1e-12 in FP64 and 1e-6 in FP32.
2. Three FP64 steps (interp -> Update_Pos) follow the CPU oracle's trajectory
   to 1e-12 relative in the positions.
3. Twenty steps, mixed vs FP64 from the same start: positions agree to 1e-6
   of the capsule radius, and the per-capsule volume and area (surf_vol from
   each path's own normals and areas) within the mixed tolerance 1e-4.
"""
import numpy as np
import pytest

import oracle as O
from suguru_b200 import timestep as TS
from suguru_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_prescribed_flow_matches_numpy(cuda):
    torch = cuda
    wl = W.small_config()
    om = TS.frequencies(len(wl.modes["phase"]))
    flow = TS.PrescribedFlow(wl.grid, wl.modes, 0.7, om, torch.float64)
    flow32 = TS.PrescribedFlow(wl.grid, wl.modes, 0.7, om, torch.float32)
    for t in (0.0, 0.37):
        got = [x.cpu().numpy() for x in flow(t)]
        got32 = [x.cpu().numpy() for x in flow32(t)]
        ref = W.velocity_field(wl.grid, wl.modes, 0.7, t=t, omega=om)
        for g, g32, r in zip(got, got32, ref):
            assert np.abs(g - r).max() <= 1e-12 * np.abs(r).max()
            assert np.abs(g32 - r).max() <= 1e-6 * np.abs(r).max()  # FP32 output: a few roundings


def test_fp64_trajectory_matches_oracle(cuda):
    wl = W.small_config()
    om = TS.frequencies(len(wl.modes["phase"]))
    steps, dt = 3, 0.01 * wl.grid[3]
    got = TS.run(wl, steps, precision="fp64", omega=om)
    x, y, z = wl.x.copy(), wl.y.copy(), wl.z.copy()
    lz = wl.grid[2] * wl.grid[5]
    for s in range(steps):
        u, v, w = wl.velocity(t=s * dt, omega=om)
        ul, vl, wlv = O.interp(wl.grid, u, v, w, x, y, z)
        x, y, z = O.update_pos(dt, lz, x, y, z, ul, vl, wlv)
    for g, r in zip(got["positions"], (x, y, z)):
        assert np.abs(g - r).max() <= 1e-12 * np.abs(r).max()


def test_mixed_vs_fp64_drift(cuda):
    wl = W.small_config()
    r = TS.compare(wl, 20)
    print(r)
    assert r["position_mixed_vs_fp64"] <= 1e-6 * float(wl.radius.min())
    assert r["volume_mixed_vs_fp64"] <= 1e-4
    assert r["area_mixed_vs_fp64"] <= 1e-4
    assert r["mixed_steps_per_s"] > 0 and r["fp64_steps_per_s"] > 0
