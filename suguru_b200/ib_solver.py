"""The coupled immersed-boundary solver: the reference's main loop with its FFT
flow solver (main.f90:172-347, fsolver = 'f'), every stage on the GPU, FP64.

One step, in the reference's order:
  uoo <- uo <- unew                      (main.f90:186-209)
  eulr2lagr, complagrforces, [collisions], lagr2eulr    sg_step (main.f90:225-233)
  [indicator: indic, visc, centrifugal terms into forcey, forcez]   (main.f90:237)
  Update_Pos                             sg_update_pos (main.f90:239)
  fftuvw, bounduvw, fillps, solver1d, boundp, correc, bounduvw, pnew += p
                                         sg_flow_step (main.f90:333-347)
The spread force of the step drives the flow, and the flow moves the
capsules: no prescribed velocity is involved.
"""
import numpy as np

from .coupling import CouplingStep


class IBSolver:
    """State on the device (torch tensors): positions X, velocities u (unew),
    uo, uoo, pressure p, the force fields and, with the indicator, indic and
    visc.  u0: initial (u, v, w) fields meeting bounduvw (numpy, FP64).

    precision: "fp64" runs every stage in FP64; "mixed" runs the coupling step
    (interpolation, membrane force, spread) and Update_Pos on a mixed-precision
    context, from an FP32 copy of the velocity, and widens its force fields,
    normals and areas to FP64 for the indicator and the flow solver, which
    stay FP64."""

    def __init__(self, wl, dt, rep, u0, walls=(0.0, 0.0), indicator=None, collisions=False, stream=None,
                 precision="fp64"):
        import torch
        self.torch = torch
        self.dt = float(dt)
        self.st = torch.cuda.Stream() if stream is None else stream
        self.cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="fp64", mem="device",
                               stream=self.st.cuda_stream, async_=True)
        self.mixed = precision == "mixed"
        self.cs_ib = self.cs
        if self.mixed:
            self.cs_ib = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="mixed",
                                      mem="device", stream=self.st.cuda_stream, async_=True)
        self.cs.set_flow_params(rep, *walls)
        self.indicator = indicator is not None
        if self.indicator:
            self.cs.set_indicator_params(**indicator)
        if collisions:
            self.cs_ib.set_wall_collisions(in_step=True)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()
        with torch.cuda.stream(self.st):
            self.X = [dev(a) for a in (wl.x, wl.y, wl.z)]
            self.u = [dev(a) for a in u0]
            self.uo = [a.clone() for a in self.u]
            self.uoo = [a.clone() for a in self.u]
            self.p = torch.zeros_like(self.u[0])
            self.lag = [torch.zeros(wl.npts, dtype=torch.float64, device="cuda") for _ in range(10)]
            self.force = [torch.zeros_like(self.u[0]) for _ in range(3)]
            self.ind = [torch.zeros_like(self.u[0]) for _ in range(2)]
            self.unext = [torch.zeros_like(self.u[0]) for _ in range(3)]
            if self.mixed:  # the mixed step's own buffers
                self.u32 = [torch.zeros(self.u[0].shape, dtype=torch.float32, device="cuda") for _ in range(3)]
                self.lag32 = [torch.zeros(wl.npts, dtype=torch.float32, device="cuda") for _ in range(10)]
                self.force32 = [torch.zeros_like(self.u32[0]) for _ in range(3)]
        self.stepped = False

    def step(self, marks=None):
        """One step; marks: optional list of 5 CUDA events recorded between the stages
        (coupling step, indicator, Update_Pos, flow step)."""
        cs, L = self.cs, self.lag
        mark = (lambda q: marks[q].record(self.st)) if marks else (lambda q: None)
        with self.torch.cuda.stream(self.st):
            # uoo <- uo <- unew (buffers rotate; u still holds unew for the interpolation)
            self.uoo, self.uo = self.uo, self.uoo
            for a, b in zip(self.uo, self.u):
                a.copy_(b)
            mark(0)
            if self.mixed:
                for a, b in zip(self.u32, self.u):
                    a.copy_(b)
                self.cs_ib.step(*self.u32, *self.X, lag_out=self.lag32, eul_out=self.force32)
                for a, b in zip(self.force, self.force32):
                    a.copy_(b)
                for q in range(6, 10):  # normals and areas for the indicator
                    L[q].copy_(self.lag32[q])
            else:
                cs.step(*self.u, *self.X, lag_out=L, eul_out=self.force)
            mark(1)
            if self.indicator:
                cs.indicator(*self.X, L[6], L[7], L[8], L[9], fy=self.force[1], fz=self.force[2], out=self.ind)
            mark(2)
            if self.mixed:
                self.cs_ib.update_pos(self.dt, *self.X, *self.lag32[0:3])
            else:
                cs.update_pos(self.dt, *self.X, L[0], L[1], L[2])
            mark(3)
            cs.flow_step(self.dt, *self.uo, *self.uoo, self.p, *self.force, out=self.unext)
            mark(4)
            self.u, self.unext = self.unext, self.u
        self.stepped = True

    def stage_times(self, steps):
        """Mean ms per stage over `steps` steps: coupling step, indicator, Update_Pos, flow step."""
        torch = self.torch
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
        acc = np.zeros(4)
        for _ in range(steps):
            self.step(marks=ev)
            torch.cuda.synchronize()
            acc += [ev[q].elapsed_time(ev[q + 1]) for q in range(4)]
        return dict(zip(("coupling_step", "indicator", "update_pos", "flow_step"), (acc / steps).tolist()))

    def run(self, steps, graph=False):
        """Advance `steps` steps; returns the CUDA-event time in ms.

        graph: capture two steps in one CUDA graph (the buffers rotate every
        step, so a pair returns them to their places) and replay it, an odd
        last step running eagerly; the work is the same, without host launches
        between the kernels.  A solver that has not stepped yet runs its first
        step eagerly and outside the timed region, so that first launches stay
        outside the capture."""
        torch = self.torch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g = None
        if graph and not self.stepped and steps > 0:
            # the libraries' first launches (module loads, FFT plans' first use) happen outside the capture
            self.step()
            steps -= 1
            torch.cuda.synchronize()
        if graph and steps >= 2:
            torch.cuda.synchronize()
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=self.st):
                self.step()
                self.step()
        e0.record(self.st)
        if g is not None:
            # the capture recorded the work without running it; the pair's buffer
            # rotation already happened on the host, which a pair restores.  The
            # replays go to the solver's stream, between the timing events.
            with torch.cuda.stream(self.st):
                for _ in range(steps // 2):
                    g.replay()
            if steps % 2:
                self.step()
        else:
            for _ in range(steps):
                self.step()
        e1.record(self.st)
        torch.cuda.synchronize()
        del g
        return e0.elapsed_time(e1)

    def state(self):
        self.torch.cuda.synchronize()
        h = lambda ts: [t.cpu().numpy() for t in ts]
        return dict(X=h(self.X), u=h(self.u), p=self.p.cpu().numpy(), force=h(self.force), lag=h(self.lag),
                    indic=self.ind[0].cpu().numpy(), visc=self.ind[1].cpu().numpy())
