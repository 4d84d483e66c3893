"""Time-stepped coupling (config 4): capsules advected through a prescribed flow.

Each step runs the library's coupling step (interpolation, membrane force,
spreading; main.f90:225-233) and then Update_Pos (forward Euler with the
interpolated velocity, Update_Pos.f90:95-126).  The Eulerian velocity is
prescribed: the shear u = gamma z plus seeded random Fourier modes whose phases
advance with seeded frequencies, sampled at each component's staggered
location (the numpy form is workloads.velocity_field; here it is evaluated on
the GPU every step).  There is no flow solver on this path, so the spread
force is computed, as the reference does, but does not feed back.

`run` returns the per-capsule volume and area (surf_vol, FP64) at the first
and last step and the CUDA-event time of the stepping loop; `compare` runs the
mixed and the FP64 paths from the same start and reports the drift of each
and their difference.
"""
import os

import numpy as np

from . import workloads as W
from .coupling import CouplingStep


def frequencies(nmodes=16, seed=7):
    return np.random.default_rng(seed).uniform(0.5, 2.0, size=nmodes) * 2.0 * np.pi


class PrescribedFlow:
    """u, v, w on the MAC grid (with halos) at time t, from the library's flow
    kernels (include/sg_workload.h) on the current torch stream.

    Called with a float t, or with a 0-d float64 CUDA tensor that the work
    reads when it runs (a captured CUDA graph can then advance it)."""

    def __init__(self, grid, modes, shear, omega, dtype, device="cuda"):
        import torch
        self.torch = torch
        self.grid = grid
        itot, jtot, ktot = grid[:3]
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        self.modes = [f64(modes["nx"]), f64(modes["ny"]), f64(modes["phase"]), f64(modes["amp"]).reshape(-1, 3),
                      f64(omega)]
        self.shear = float(shear)
        self.dtype = dtype
        self.out = [torch.empty((ktot + 2, jtot + 2, itot + 2), dtype=dtype, device=device) for _ in range(3)]
        self.work = torch.empty(3 * (jtot + 2) * (itot + 2), dtype=torch.float64, device=device)
        self.t = torch.zeros((), dtype=torch.float64, device=device)

    def __call__(self, t):
        import ctypes
        from .coupling import SgError, lib
        torch = self.torch
        if isinstance(t, torch.Tensor):
            tt = t
        else:
            self.t.fill_(float(t))
            tt = self.t
        itot, jtot, ktot, dx, dy, dz = self.grid
        nx, ny, ph, amp, om = self.modes
        p = lambda a: ctypes.c_void_p(a.ctypes.data)
        d = lambda x: ctypes.c_void_p(x.data_ptr())
        rc = lib().sg_prescribed_flow(itot, jtot, ktot, dx, dy, dz, len(ph), p(nx), p(ny), p(ph), p(amp), p(om),
                                      self.shear, d(tt), int(self.dtype == torch.float32), *map(d, self.out),
                                      d(self.work), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
        if rc:
            raise SgError(rc, "sg_prescribed_flow")
        return self.out


def run(wl, steps, precision="mixed", dt=None, surrogate_params=None, trust=None, omega=None, stream=None,
        graph=True, tune=True, output_dir=None, output_every=100, restart_every=None):
    """Advect the capsules of `wl` for `steps` steps; returns diagnostics and timing.

    graph: capture one step (flow evaluation, coupling step, Update_Pos and
    the time increment, which lives on the device) in a CUDA graph and replay
    it `steps` times, so that no host work is left between the steps.
    tune: let the library's autotuner pick the spreading tile and the capsule
    split first (untimed; the points do not move).
    output_dir: every `output_every` steps write the reference's outputs there
    (Capsule###step#######.txt, center_velocity.txt, epsilonxy.txt; main.f90:
    455-476), and every `restart_every` steps its restart file
    allpartdata####### (loadd.f90:147-670; capsules of one degree only).  The
    host writes between the replays, so a run with outputs times them too.
    """
    import torch
    if restart_every and len(set(int(L) for L in wl.degree)) > 1:
        raise ValueError("allpartdata holds capsules of one point count; this batch has several degrees")
    dx = wl.grid[3]
    dt = 0.01 * dx if dt is None else dt
    omega = frequencies(len(wl.modes["phase"])) if omega is None else omega
    td = torch.float64 if precision == "fp64" else torch.float32
    st = torch.cuda.Stream() if stream is None else stream
    cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision, mem="device",
                      stream=st.cuda_stream, async_=True, surrogate=surrogate_params is not None)
    if surrogate_params is not None:
        cs.surrogate_params(surrogate_params)
        cs.surrogate_set_trust(*trust)
    with torch.cuda.stream(st):  # every torch op below is ordered with the library's work
        flow = PrescribedFlow(wl.grid, wl.modes, wl.shear, omega, td)
        X = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (wl.x, wl.y, wl.z)]
        n = wl.npts
        lag = [torch.empty(n, dtype=td, device="cuda") for _ in range(10)]
        eul = [torch.empty_like(flow.out[0]) for _ in range(3)]

        def diag():
            cs.step(*flow(0.0), *X, lag_out=lag, eul_out=eul)  # normals and area of the current shape
            out = cs.surf_vol(*X, lag[6], lag[7], lag[8], lag[9])
            cs.synchronize()
            return out.cpu().numpy()

        d0 = diag()
        start = [x.cpu().numpy() for x in X]

        def outputs(done):  # the state after `done` steps
            from . import particle_io as PIO
            cs.synchronize()
            pos = [x.cpu().numpy() for x in X]
            vel = [lag[q].double().cpu().numpy() for q in range(3)]
            sv = cs.surf_vol(*X, lag[6], lag[7], lag[8], lag[9]).cpu().numpy()
            PIO.write_step_outputs(output_dir, done, done * dt, wl.offsets, pos, vel, sv[-1, 2], sv[-1, 3])
            if restart_every and done % restart_every == 0:
                frc = [lag[q].double().cpu().numpy() for q in range(3, 6)]
                scal, arr = PIO.particle_state(wl.offsets, pos, velocity=vel, force=frc,
                                               area=lag[9].double().cpu().numpy(), volume=sv[:, 0],
                                               volume0=d0[:, 0], initial=start)
                PIO.write_allpartdata(os.path.join(output_dir, PIO.allpartdata_name(done)), scal, arr)

        def due(done):
            return output_dir is not None and done % output_every == 0
        on_sur = fb = 0
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if tune:  # tile shape and capsule split from the library's autotuner (does not move the points)
            cs.autotune(*flow(0.0), *X, lag_out=lag, eul_out=eul, reps=2)
        if graph:
            t_dev = torch.zeros((), dtype=torch.float64, device="cuda")
            flow(t_dev)  # library handles of the flow's products exist before the capture
            cs.update_pos(0.0, *X, lag[0], lag[1], lag[2])  # loads the kernel; X + 0 U leaves X as it is
            st.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=st):
                u, v, w = flow(t_dev)
                cs.step(u, v, w, *X, lag_out=lag, eul_out=eul)
                cs.update_pos(dt, *X, lag[0], lag[1], lag[2])
                t_dev.add_(dt)
            e0.record(st)
            for s in range(steps):
                g.replay()
                if due(s + 1):
                    outputs(s + 1)
            e1.record(st)
        else:
            e0.record(st)
            for s in range(steps):
                u, v, w = flow(s * dt)
                cs.step(u, v, w, *X, lag_out=lag, eul_out=eul)
                cs.update_pos(dt, *X, lag[0], lag[1], lag[2])
                if due(s + 1):
                    outputs(s + 1)
            e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if graph:
            del g
        if surrogate_params is not None:
            on_sur, fb = cs.surrogate_counts()
        d1 = diag()
        final = [x.cpu().numpy() for x in X]
    cs.close()
    return dict(vol0=d0[:, 0], area0=d0[:, 1], vol=d1[:, 0], area=d1[:, 1], positions=final,
                steps_per_s=steps / (ms / 1e3), ms=ms, on_surrogate=on_sur, fallback=fb)


def compare(wl, steps, **kw):
    """Mixed vs FP64 trajectories from the same start."""
    a = run(wl, steps, precision="mixed", **kw)
    b = run(wl, steps, precision="fp64")
    rel = lambda x, y: float(np.max(np.abs(x - y) / np.abs(y)))
    return dict(
        steps=steps,
        mixed_steps_per_s=a["steps_per_s"], fp64_steps_per_s=b["steps_per_s"],
        volume_drift_mixed=rel(a["vol"], a["vol0"]), volume_drift_fp64=rel(b["vol"], b["vol0"]),
        area_drift_mixed=rel(a["area"], a["area0"]), area_drift_fp64=rel(b["area"], b["area0"]),
        volume_mixed_vs_fp64=rel(a["vol"], b["vol"]), area_mixed_vs_fp64=rel(a["area"], b["area"]),
        position_mixed_vs_fp64=float(max(np.abs(p - q).max() for p, q in zip(a["positions"], b["positions"]))),
        on_surrogate=a["on_surrogate"], fallback=a["fallback"])


def config4(ncap=1024):
    """200 steps of config 2, dt = 0.01 dx, time-varying modes."""
    return W.config2(ncap)
