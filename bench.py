#!/usr/bin/env python
"""Benchmark: Lagrangian points/s per IB coupling step on one B200.

One step = interpolation of the Eulerian velocity to every force point
(eulr2lagr), the spectral Skalak membrane force with normals and areas
(complagrforces), and spreading of force*area onto the Eulerian grid
(lagr2eulr), for the dense-suspension workload: 256 capsules of SH degree 15
(524,288 points) on a 256x256x128 grid, seeded synthetic shapes and velocity.

`value` is the headline path (mixed precision: FP32 fields, FP32 pointwise,
Legendre contractions batched per degree), device-resident inputs, points/s
summed over ranks.  The FP64 plain path is measured beside it.  `e2e` is the
same metric through the public C ABI with host (pinned) buffers, H2D/D2H copies
inside the timed region.  `--impl reference` times the CPU FP64 restatement of
the reference path (the oracle, reference loop structure) on the host cores.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from suguru_b200 import workloads as W  # noqa: E402

L2_BYTES = 126 * 2**20


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="c1", choices=["c0", "c1", "c2", "c4", "coupled"],
                   help="c4: the 200-step time-stepped run of config 2 (steps/s, area/volume drift); "
                        "coupled: the IB solver with the FFT flow solver on config 1's grid and capsules (FP64)")
    p.add_argument("--c4-steps", type=int, default=200)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--only", default=None, choices=["mixed", "fp64"],
                   help="time one path only, no e2e (for profiler captures)")
    p.add_argument("--bending", action="store_true",
                   help="with --only: the reference's default bending (ibend = 1, cbend = 0.3) on every capsule")
    p.add_argument("--cpu-sample-caps", type=int, default=64)
    p.add_argument("--no-surrogate", action="store_true", help="skip training and timing the surrogate path")
    p.add_argument("--tile", type=int, default=None, choices=[0, 1, 2, 3, 4, 5, 6],
                   help="fixed spreading tile shape (index into TILE_SHAPES; FP64 takes shape 0) instead of the "
                        "autotuner, so that profiler captures see one launch sequence")
    p.add_argument("--legendre-terms", type=int, default=0, choices=[0, 3, 6],
                   help="mixed path: split products of the tensor-core Legendre contractions (0: automatic by degree)")
    p.add_argument("--sur-samples", type=int, default=200000)
    p.add_argument("--sur-epochs", type=int, default=40)
    p.add_argument("--sur-loose-tol", type=float, default=3e-2)
    return p.parse_args()


WORKLOAD_LABELS = {
    "c0": "single capsule, SH degree 15 (2,048 points), grid 128x64x64, dx=1/32, Skalak Gs=1 C=1",
    "c1": "dense suspension: 256 capsules, SH degree 15 (524,288 points), grid 256x256x128, dx=1/32, "
          "Skalak Gs=1 C=1",
    "c2": "uneven batch: 1024 capsules, SH degree 7-23 (1,526,248 points), grid 512x256x256, dx=1/32, "
          "Skalak Gs=1 C=1",
}


def workload(name):
    return {"c0": W.config0, "c1": W.config1, "c2": W.config2, "coupled": W.config1}[name]()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


def load_traffic():
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.3)
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 8:
                    continue
                try:
                    sm.append(float(parts[0]))
                    smax.append(float(parts[1]))
                except ValueError:
                    continue
                for nm, val in zip(names, parts[4:8]):
                    if val.lower() == "active":
                        reasons.add(nm)
        os.remove(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def spread_bytes(wl, s):
    """Algorithmic bytes of one spread launch: the whole force field written
    (lagr2eulr zeroes and writes every cell) plus, per point, its force record
    (force * area / dV and the largest component: 4 reals), base cell indices
    (3 int32), fractional offsets (3 reals) and the sorted index (int32)."""
    itot, jtot, ktot = wl.grid[:3]
    nfield = (itot + 2) * (jtot + 2) * (ktot + 2)
    return 3 * nfield * s + wl.npts * (4 * s + 12 + 3 * s + 4)


def cs_tile_shape(shape):
    from suguru_b200.coupling import TILE_SHAPES
    t = TILE_SHAPES[shape]
    return ("rows",) + t[1:] if t[0] == 0 else t


def rel_l2_t(a, b):
    import torch
    d = torch.linalg.vector_norm((a.double() - b.double()).ravel())
    return float(d / torch.clamp(torch.linalg.vector_norm(b.double().ravel()), min=1e-300))


def legendre_roofline(r, tc_peak, peak_kind):
    """Tensor-pipe roofline of the Legendre contractions of one step: the
    algorithmic flops (2 x multiply-adds of the transforms, triangular zeros
    left out) over the summed CUDA-event time of the contraction launches,
    against the measured dense bf16 peak divided by the split products per
    product (3 for BF16x3, 6 for BF16x6: each FP32-accurate product costs that
    many bf16 products).  issue_frac is the issued tensor-core work (padded
    tiles x split products) over the bf16 peak: how busy the tensor pipe was."""
    w, t_ms, terms = r["work"], r["stages"]["contract"], max(r["terms"], 1)
    if t_ms <= 0 or w["issued_flops"] <= 0:
        return None
    achieved = w["flops"] / (t_ms / 1e3) / 1e12
    peak = tc_peak / terms
    return {"kernel": "legendre_mma_kernel (tcgen05, BF16x%d), %d launches per step" % (terms, w["launches"]),
            "bound": "tensor", "flops_per_step": w["flops"], "issued_flops_per_step": w["issued_flops"],
            "ms_per_step": t_ms, "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_kind": "%s bf16 dense / %d (BF16x%d)" % (peak_kind, terms, terms),
            "issue_frac": w["issued_flops"] / (t_ms / 1e3) / 1e12 / tc_peak}


def run_ours(args):
    import torch
    import torch.distributed as dist
    from suguru_b200.coupling import CouplingStep
    from suguru_b200 import replicas as R

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", local)
    # a dedicated stream: the library launches on it and the timing events are
    # recorded on it (torch's default stream has the null handle)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    wl = workload(args.config)
    n = wl.npts
    hbm_peak, tc_peak, peak_kind = load_peaks()

    def dev_inputs(dtype):
        u, v, w = wl.velocity(dtype=dtype)
        td = torch.float64 if dtype == np.float64 else torch.float32
        return [torch.from_numpy(a).to(dev) for a in (u, v, w)], td

    X = [torch.from_numpy(a).to(dev) for a in (wl.x, wl.y, wl.z)]
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=dev)

    def make_cs(precision, surrogate=False):
        cs = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision=precision, mem="device",
                          device=local, stream=stream.cuda_stream, async_=True, surrogate=surrogate)
        if precision != "fp64":
            cs.set_legendre_terms(args.legendre_terms)
        return cs

    capidx = torch.repeat_interleave(torch.arange(wl.ncap, device=dev),
                                     torch.from_numpy(np.diff(wl.offsets).astype(np.int64)).to(dev))

    def worst_capsule(out, ref):
        """Largest per-capsule relative L2 error of the force vectors."""
        num = torch.zeros(wl.ncap, dtype=torch.float64, device=dev)
        den = torch.zeros_like(num)
        for c in range(3):
            num.index_add_(0, capidx, (out[3 + c].double() - ref[3 + c].double()) ** 2)
            den.index_add_(0, capidx, ref[3 + c].double() ** 2)
        return float(torch.sqrt(num / torch.clamp(den, min=1e-300)).max())

    def time_path(cs, precision, tune=True):
        dtype = np.float64 if precision == "fp64" else np.float32
        uvw, td = dev_inputs(dtype)
        lag = [torch.empty(n, dtype=td, device=dev) for _ in range(10)]
        eul = [torch.empty(cs.field_shape, dtype=td, device=dev) for _ in range(3)]
        tile = 0
        if args.tile is not None:  # a fixed tile shape, no autotuning (profiler captures)
            cs.set_tile_shape(args.tile if precision != "fp64" else 0)
            tune = False
        if tune:  # the library's autotuner picks the spreading tile shape (untimed set-up)
            cs.set_profiling(False)
            tile, _ = cs.autotune(*uvw, *X, lag_out=lag, eul_out=eul, reps=3)
        else:
            tile = cs.tile_shape()[0]
        cs.set_profiling(True)
        for _ in range(args.warmup):
            cs.step(*uvw, *X, lag_out=lag, eul_out=eul)
        # stage split of one step (CUDA events between the stages)
        stages = {k: 0.0 for k in ("bin", "interp", "membrane", "spread", "contract")}
        nst = 3
        for _ in range(nst):
            flush.zero_()
            cs.step(*uvw, *X, lag_out=lag, eul_out=eul)
            st = cs.stage_times()
            for key in stages:
                stages[key] += st[key] / nst
        # the timed steps replay one captured CUDA graph of the step
        cs.set_profiling(False)
        torch.cuda.synchronize()
        cs.graph_capture(*uvw, *X, lag, eul)
        cs.graph_launch()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        e1 = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        launches = 0
        with Clocks(local) as clk:
            for k in range(args.steps):
                flush.zero_()  # L2 flush between timed iterations (outside the events)
                e0[k].record(stream)
                cs.graph_launch()
                e1[k].record(stream)
                launches += cs.last_launch_count()
            torch.cuda.synchronize()
        cs.graph_release()
        ms = R.max_over_ranks(sum(a.elapsed_time(b) for a, b in zip(e0, e1)))
        return dict(ms_per_step=ms / args.steps, stages=stages, work=cs.contraction_work(),
                    terms=cs.legendre_terms(15) if precision != "fp64" else 0,
                    launches=launches, clocks=clk.summary(), s=4 if precision != "fp64" else 8,
                    tile="x".join(map(str, cs_tile_shape(tile))), out=[t.clone() for t in lag + eul])

    def errors(out, ref):
        """Relative L2 of the mixed-path results against the FP64 plain path (itself within 1e-10 of the oracle)."""
        return {"velocity": max(rel_l2_t(out[c], ref[c]) for c in range(3)),
                "force": max(rel_l2_t(out[3 + c], ref[3 + c]) for c in range(3)),
                "spread_field": max(rel_l2_t(out[10 + c], ref[10 + c]) for c in range(3)),
                "force_worst_capsule": worst_capsule(out, ref)}

    if args.only:
        cs = make_cs(args.only)
        if args.bending:
            cs.set_capsule_bending(0.3 * wl.gs * wl.radius**2)
        r = time_path(cs, args.only)
        cs.close()
        if rank == 0:
            print(json.dumps({"only": args.only, "ms_per_step": r["ms_per_step"], "stages_ms": r["stages"],
                              "points_per_s": world * n / (r["ms_per_step"] / 1e3)}))
        if world > 1:
            dist.destroy_process_group()
        return None

    cs64 = make_cs("fp64")
    fp64 = time_path(cs64, "fp64")
    cs64.close()
    csm = make_cs("mixed")
    mixed = time_path(csm, "mixed")  # the staged force stage, contractions on the tensor cores
    # the force stage as one fused kernel (FP32 contractions on CUDA cores), as the comparison
    csm.set_fused_force(True)
    fused = time_path(csm, "mixed")
    # the reference's default bending (ibend = 1, ebend = cbend gscell with cbend = 0.3, in
    # units of the capsule radius)
    csm.set_fused_force(False)
    csm.set_capsule_bending(0.3 * wl.gs * wl.radius**2)
    bending = time_path(csm, "mixed")
    csm.close()

    # ---- surrogate: linear response, plain-model training data, the library's training kernels
    sur = None
    if not args.no_surrogate:
        from suguru_b200 import surrogate as S
        t0 = time.perf_counter()
        L0, L1 = S.linear_response()
        Xtr, Ytr, _ = S.make_dataset(args.sur_samples, seed=31)
        Xv, Yv, Av = S.make_dataset(8192, seed=32)
        t1 = time.perf_counter()
        css = make_cs("mixed", surrogate=True)
        hist = S.train(css, Xtr, Ytr, L0, L1, epochs=args.sur_epochs, batch=1024, lr=1e-3, seed=3)
        t2 = time.perf_counter()
        e_lin = S.rel_err_rows(css.surrogate_predict(Xv, parts=1), Yv)
        e_net = S.rel_err_rows(css.surrogate_predict(Xv, parts=3), Yv)
        variants = {}
        # residual-check limits calibrated for 1e-4 (the headline) and for a
        # loose tolerance, and with no limit (every capsule on the network)
        for tol in (1e-4, args.sur_loose_tol, None):
            if tol is None:
                css.surrogate_set_trust(1e30, 1e30, 0.0, 1e30)
                info = dict(amp_max=float("inf"), ratio_max=float("inf"))
            else:
                info = S.calibrate_trust(css, Xv, Yv, tol=tol)
            css.set_tile_shape(-1)
            r = time_path(css, "mixed", tune=True)
            ns, nf = css.surrogate_counts()
            variants[tol] = dict(r=r, on_surrogate=ns, fallback=nf, amp_max=info["amp_max"],
                                 ratio_max=info["ratio_max"], errors=errors(r["out"], fp64["out"]))
        params = css.surrogate_params()
        css.close()
        sur = dict(variants=variants, hist=hist, t_data=t1 - t0, t_train=t2 - t1, params=params,
                   med_lin=float(np.median(e_lin)), med_net=float(np.median(e_net)))

    # e2e through the public API with pinned host buffers (the headline path)
    u32, v32, w32 = wl.velocity(dtype=np.float32)
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hu, hv, hw = pin(u32), pin(v32), pin(w32)
    hX = [pin(a) for a in (wl.x, wl.y, wl.z)]
    cs_h = CouplingStep(wl.grid, wl.degree, wl.radius, wl.gs, wl.csk, precision="mixed", mem="host", device=local,
                        surrogate=sur is not None)
    if sur is not None:  # the headline path: trained network, limits for 1e-4
        cs_h.surrogate_params(sur["params"])
        v = sur["variants"][1e-4]
        cs_h.surrogate_set_trust(v["amp_max"], v["ratio_max"], 0.5, 2.0)
    hlag = [torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(10)]
    heul = [torch.empty(cs_h.field_shape, dtype=torch.float32).pin_memory() for _ in range(3)]
    for _ in range(max(1, args.warmup // 2)):
        cs_h.step(hu, hv, hw, *hX, lag_out=hlag, eul_out=heul)
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cs_h.step(hu, hv, hw, *hX, lag_out=hlag, eul_out=heul)
    e2e_s = R.max_over_ranks((time.perf_counter() - t0) / args.steps)
    cs_h.close()
    nfield = int(np.prod(cs_h.field_shape))
    h2d = 3 * nfield * 4 + 3 * n * 8
    d2h = 10 * n * 4 + 3 * nfield * 4

    result = None
    if rank == 0:
        head = mixed
        path = "mixed (surrogate off)"
        if sur is not None:
            v4 = sur["variants"][1e-4]
            head = v4["r"]
            if v4["on_surrogate"] > 0:
                path = ("mixed + surrogate: %d of %d capsules on the network, per-capsule checks calibrated "
                        "for 1e-4 force error" % (v4["on_surrogate"], v4["on_surrogate"] + v4["fallback"]))
            else:
                path = ("mixed plain: the surrogate's limits calibrated for 1e-4 force error admit no capsule "
                        "(held-out median error %.1e), so the step runs without it" % sur["med_net"])
        value = world * n / (head["ms_per_step"] / 1e3)
        fp64_value = world * n / (fp64["ms_per_step"] / 1e3)
        sp_ms = head["stages"]["spread"]
        sbytes = spread_bytes(wl, 4)
        achieved = sbytes / (sp_ms / 1e3) / 1e9
        traffic = load_traffic().get("spread_%s_mixed_bytes_per_launch" % args.config)  # this workload's capture only
        result = {
            "metric": "Lagrangian pts/s per IB step, mixed+surrogate vs FP64 plain, 1 B200, <=1e-4 err",
            "value": value,
            "unit": "points/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": head["ms_per_step"],
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (Legendre contractions on tcgen05 tensor cores, BF16x3 below SH degree 16 and "
                     "BF16x6 from 16 up unless --legendre-terms forces one, FP32 accumulation; "
                     "FP64 positions, centroids, tables)",
            "data": "synthetic (seeded shapes and velocity modes, no reference fixtures exist)",
            "config": {"workload": WORKLOAD_LABELS[args.config],
                       "path": path, "points": n, "parallelism": "replicas" if world > 1 else
                       "single GPU", "l2": "flushed (256 MB write) between timed iterations",
                       "spread_tile": head["tile"], "spread_tile_fp64": fp64["tile"],
                       "timed": "replays of one captured CUDA graph of the step (autotuned tile and schedule)"},
            "fp64_plain": {"value": fp64_value, "unit": "points/s", "ms_per_step": fp64["ms_per_step"],
                           "stages_ms": fp64["stages"]},
            "mixed_plain": {"value": world * n / (mixed["ms_per_step"] / 1e3), "unit": "points/s",
                            "ms_per_step": mixed["ms_per_step"], "stages_ms": mixed["stages"],
                            "errors_vs_fp64": errors(mixed["out"], fp64["out"])},
            "speedup_vs_fp64_plain": value / fp64_value,
            "stages_ms": head["stages"],
            "roofline": {"kernel": "spread_kernel<float> (deterministic gather spread)", "bound": "hbm",
                         "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                         "peak_kind": peak_kind, "algorithmic_bytes": sbytes, "traffic": traffic},
            "roofline_legendre": legendre_roofline(mixed, tc_peak, peak_kind),
            "mixed_bending": {
                "value": world * n / (bending["ms_per_step"] / 1e3), "unit": "points/s",
                "ms_per_step": bending["ms_per_step"], "stages_ms": bending["stages"],
                "note": "the same step with the reference's default bending (ibend = 1, cbend = 0.3): "
                        "one more contraction for the third and fourth derivatives, the bending "
                        "membrane kernel, BF16x6 products"},
            "mixed_fused_force": {
                "value": world * n / (fused["ms_per_step"] / 1e3), "unit": "points/s",
                "ms_per_step": fused["ms_per_step"], "stages_ms": fused["stages"],
                "errors_vs_fp64": errors(fused["out"], fp64["out"]),
                "note": "the force stage as one kernel, one CTA per capsule, Legendre contractions in FP32 "
                        "on CUDA cores (sg_set_fused_force); the headline's force stage is the staged one"},
            "e2e": {"value": world * n / e2e_s, "unit": "points/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3},
            "gpu_launches": head["launches"],
            "clocks": head["clocks"],
        }
        if sur is not None:
            vv = {}
            for tol, v in sur["variants"].items():
                vv["no limit" if tol is None else "%g" % tol] = {"points_per_s": world * n / (v["r"]["ms_per_step"] / 1e3),
                                  "ms_per_step": v["r"]["ms_per_step"], "on_surrogate": v["on_surrogate"],
                                  "fallback": v["fallback"], "amp_max": min(v["amp_max"], 1e30),
                                  "ratio_max": min(v["ratio_max"], 1e30),
                                  "errors_vs_fp64": v["errors"], "stages_ms": v["r"]["stages"]}
            result["surrogate"] = {
                "training": {"samples": args.sur_samples, "epochs": args.sur_epochs, "batch": 1024,
                             "data_s": sur["t_data"], "train_s": sur["t_train"],
                             "loss_first_last": [float(sur["hist"][0]), float(sur["hist"][-1])]},
                "heldout_median_rel_err": {"linear_response": sur["med_lin"], "linear_plus_network": sur["med_net"]},
                "by_tolerance": vv}
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return result


def run_c4(args, rank):
    """Config 4: 200 coupling steps of config 2 with forward-Euler advection, mixed vs FP64."""
    import torch
    from suguru_b200 import timestep as TS
    if rank != 0:
        return 0
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    wl = TS.config4()
    TS.run(wl, 3, precision="mixed")  # warm-up (module load, first launches)
    r = TS.compare(wl, args.c4_steps)
    print(json.dumps({
        "metric": "coupling steps/s, time-stepped config 2 (1024 capsules, L 7-23, grid 512x256x256)",
        "value": r["mixed_steps_per_s"], "unit": "steps/s", "n_gpus": 1, "steps": args.c4_steps,
        "higher_is_better": True, "dtype": "f32 mixed (FP64 positions)",
        "data": "synthetic (seeded shapes, prescribed shear + time-varying modes)",
        "config": {"workload": "config 2 advected for %d steps, dt = 0.01 dx, forward Euler" % args.c4_steps,
                   "points": int(wl.npts)},
        "points_per_s": r["mixed_steps_per_s"] * wl.npts,
        "fp64_plain": {"steps_per_s": r["fp64_steps_per_s"]},
        "drift": {k: r[k] for k in ("volume_drift_mixed", "volume_drift_fp64", "area_drift_mixed", "area_drift_fp64",
                                    "volume_mixed_vs_fp64", "area_mixed_vs_fp64", "position_mixed_vs_fp64")},
    }))
    return 0


def run_coupled(args, rank):
    """The coupled IB + flow solver (main.f90:172-347, fsolver 'f') on config 1's grid and
    capsules in FP64: steps/s with and without the indicator, the stages, and the oracle's
    main loop timed on the host for one step."""
    import torch
    from suguru_b200.ib_solver import IBSolver
    if rank != 0:
        return 0
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    wl = W.config1()
    u0 = list(wl.velocity())
    O.bounduvw(*u0)
    dt, rep = 0.01 * wl.grid[3], 0.0016  # Rep of param.f90:57
    ind = dict(visc0=1.0 / rep, lam=1.0, thetainc=70.0 * np.pi / 180.0, ta=1160000.0, rep=rep)
    out = {}
    for name, indicator, prec in (("without_indicator", None, "fp64"), ("with_indicator", ind, "fp64"),
                                  ("with_indicator_mixed_ib_step", ind, "mixed")):
        sol = IBSolver(wl, dt, rep, u0, indicator=indicator, precision=prec)
        sol.run(args.warmup)
        ms = sol.run(args.steps, graph=True)
        out[name] = {"steps_per_s": args.steps / (ms / 1e3), "ms_per_step": ms / args.steps,
                     "timed": "replays of a CUDA graph of two steps", "stages_ms": sol.stage_times(3)}
        del sol
    cpu = None
    if not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        x, y, z = wl.x.copy(), wl.y.copy(), wl.z.copy()
        t0 = time.perf_counter()
        r = O.coupling_step(wl.grid, wl.degree, wl.radius, *u0, x, y, z, wl.gs, wl.csk, nthreads=cores)
        o = O.indicator(wl.grid, x, y, z, *r["n"], r["area"], fy=r["fgrid"][1], fz=r["fgrid"][2], **ind)
        lx, ly, lz = (wl.grid[q] * wl.grid[q + 3] for q in range(3))
        O.update_pos_capsules(wl.offsets, dt, lx, ly, lz, x, y, z, *r["u"])
        O.flow_step(wl.grid, dt, rep, *u0, *u0, np.zeros_like(u0[0]), r["fgrid"][0], o["fy"], o["fz"])
        sec = time.perf_counter() - t0
        cpu = {"value": 1.0 / sec, "unit": "steps/s", "cores": cores, "kind": "port",
               "sample": "one full step of the oracle's main loop with the indicator at this size (C coupling "
                         "step on all host threads, numpy indicator and flow step)"}
    head = out["with_indicator"]
    print(json.dumps({
        "metric": "coupled IB + FFT flow solver steps/s, config 1 grid and capsules, 1 B200",
        "value": head["steps_per_s"], "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "dtype": "f64", "data": "synthetic (seeded shapes and initial velocity modes)",
        "config": {"workload": "256 capsules, L = 15 (524,288 points), grid 256x256x128, Rep = 0.0016, "
                               "dt = 0.01 dx, indicator on (visc0 = 1/Rep, lambda = 1, thetainc = 70 deg, "
                               "ta = 1.16e6)", "points": int(wl.npts)},
        "with_indicator": head, "without_indicator": out["without_indicator"],
        "with_indicator_mixed_ib_step": out["with_indicator_mixed_ib_step"], "cpu_baseline": cpu}))
    return 0


def cpu_reference(wl, ncaps, steps, warmup, faithful=True, cores=None):
    """The CPU FP64 restatement of the reference path (oracle, reference loop
    structure) on a bounded sample of the workload: the first `ncaps` capsules,
    all host threads (or `cores` of them)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    ncaps = min(ncaps, wl.ncap)
    npts = int(wl.offsets[ncaps])
    u, v, w = wl.velocity()
    x, y, z = wl.x[:npts], wl.y[:npts], wl.z[:npts]
    cores = cores or os.cpu_count() or 1
    for _ in range(warmup):
        O.coupling_step(wl.grid, wl.degree[:ncaps], wl.radius[:ncaps], u, v, w, x, y, z, wl.gs, wl.csk,
                        faithful=faithful, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(steps):
        O.coupling_step(wl.grid, wl.degree[:ncaps], wl.radius[:ncaps], u, v, w, x, y, z, wl.gs, wl.csk,
                        faithful=faithful, nthreads=cores)
    dt = (time.perf_counter() - t0) / steps
    return npts / dt, cores, npts, dt


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        wl = workload(args.config)
        steps, warmup = max(1, args.steps), max(0, args.warmup)
        val, cores, npts, dt = cpu_reference(wl, args.cpu_sample_caps, steps, warmup)
        sample = "first %d of %d capsules (%d points), full grid, %d OpenMP threads, FP64" % (
            min(args.cpu_sample_caps, wl.ncap), wl.ncap, npts, cores)
        print(json.dumps({
            "impl": "reference",
            "metric": "Lagrangian pts/s per IB step, mixed+surrogate vs FP64 plain, 1 B200, <=1e-4 err",
            "value": val, "unit": "points/s", "n_gpus": 0, "steps": steps,
            "warmup": warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
            "config": {"workload": WORKLOAD_LABELS.get(args.config, WORKLOAD_LABELS["c1"]), "sample": sample},
            "cpu_baseline": {"value": val, "unit": "points/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }))
        return 0
    if args.config == "c4":
        return run_c4(args, rank)
    if args.config == "coupled":
        return run_coupled(args, rank)
    res = run_ours(args)
    if rank == 0 and res is not None:
        if not args.no_cpu_baseline:
            wl = workload(args.config)
            val, cores, npts, dt = cpu_reference(wl, args.cpu_sample_caps, 1, 0)
            res["cpu_baseline"] = {"value": val, "unit": "points/s", "cores": cores, "kind": "port",
                                   "sample": "oracle (reference loop structure, FP64) on the first %d capsules "
                                             "(%d points) of the workload, full grid, %.2f s/step"
                                             % (min(args.cpu_sample_caps, wl.ncap), npts, dt)}
            # the same restatement on one host core, over a smaller sample
            c1 = max(1, min(8, args.cpu_sample_caps))
            v1, _, n1, t1 = cpu_reference(wl, c1, 1, 0, cores=1)
            res["cpu_baseline"]["single_core"] = {
                "value": v1, "unit": "points/s", "cores": 1,
                "sample": "first %d capsules (%d points), full grid, one thread, %.2f s/step" % (c1, n1, t1)}
        print(json.dumps(res))
    return 0


if __name__ == "__main__":
    sys.exit(main())
