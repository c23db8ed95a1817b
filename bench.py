#!/usr/bin/env python
"""Benchmark of the closed-form alpha solve on B200.

Metric: Mpix/s of soft-constraint closed-form alpha solves, each to FP64
relative residual 1e-7, on the 1920x1080 synthetic workload (one image per
GPU): assembly of the matting Laplacian, V-cycle hierarchy setup and the
preconditioned CG solve, from image + trimap resident in HBM to alpha
resident in HBM. ``value`` is the mixed-precision path (FP32 inner V-cycle
PCG inside FP64 iterative refinement); the plain FP64 path is reported
beside it. ``e2e`` is the same metric through the public ``solve_alpha`` API
with host numpy buffers (uploads and the alpha download inside the timed
region). ``--impl reference`` times the CPU restatement of PyMatting's own
path (cf_laplacian + make_linear_system + vcycle + cg) on host cores.

``--workload foreground`` instead times estimate_foreground_ml (the step
after alpha in PyMatting's cutout) on a 1920x1080 image and matte: the
multi-level Gauss-Seidel sweeps in the reference's exact order, bit-identical
to it for equal seed colours; its reference arm is the oracle's C
restatement on one host core.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: launched by torch.distributed.run, one rank per GPU; every rank
solves its own image (weak scaling, no collective on the data path).
"""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "Mpix/s of cf alpha solves at FP64 rel-residual 1e-7: mixed vs FP64 GPU; % HBM"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["1080p", "4096", "batch64", "foreground"],
                    default="1080p",
                    help="foreground: estimate_foreground_ml on a 1920x1080 image + matte")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune", choices=["auto", "none"], default="none",
                    help="auto: run the launch-shape autotuner before timing; none (default): "
                         "the built-in launch shapes, which matched or beat the tuner's "
                         "picks at 1080p with L2 flushed between steps")
    ap.add_argument("--profile", choices=["apply", "solve", "solve-fp64", "solve-mixed"],
                    default=None,
                    help="profiling case: a few operator applies, or one solve per precision "
                         "(or of one precision)")
    return ap.parse_args()


WORKLOADS = {
    # name: list of (h, w, seed offset, unknown fraction)
    "1080p": dict(sizes=[(1080, 1920, 0.08)], sigma=3.0, band=10),
    "4096": dict(sizes=[(4096, 4096, 0.15)], sigma=3.0, band=10),
}


def make_inputs(workload, rank):
    from pymatting_b200.synthetic import make_matting_problem, batch_sizes
    if workload == "batch64":
        spec = [(h, w, frac, seed) for (h, w, frac, seed) in batch_sizes(64, 1000)]
        from pymatting_b200.shard import shard_sizes
        world = int(os.environ.get("WORLD_SIZE", "1"))
        mine = shard_sizes([(h, w) for h, w, _, _ in spec], world)[rank]
        spec = [spec[k] for k in mine]
        sigma, band = 3.0, 10
    else:
        wl = WORKLOADS[workload]
        spec = [(h, w, frac, 100 + rank) for (h, w, frac) in wl["sizes"]]
        sigma, band = wl["sigma"], wl["band"]
    imgs, tris, fracs = [], [], []
    for h, w, frac, seed in spec:
        img, tri, _a, real = make_matting_problem(h, w, seed, sigma=sigma, band=band,
                                                  unknown_fraction=frac)
        imgs.append(img)
        tris.append(tri)
        fracs.append(real)
    return imgs, tris, fracs


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons (every 100 ms).

    Started before the warm-up so that the sampler's own start-up never falls
    inside a timed region; only samples taken inside the timed windows are
    reported."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []       # (time, line)
        self.windows = []     # (t0, t1) of timed regions
        self.thread = None
        self.first = threading.Event()

    def start(self, wait=5.0):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        self.first.wait(wait)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))
            self.first.set()

    def window(self, t0, t1):
        self.windows.append((t0, t1))

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        inside = [ln for (t, ln) in self.lines
                  if any(a <= t <= b for (a, b) in self.windows)]
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in inside:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax = max(smax, float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(HERE, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_per_launch(kind, npx):
    """DRAM bytes per apply launch from the committed ncu summary, scaled."""
    path = os.path.join(HERE, "profiles", "apply_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    e = d.get(kind)
    if not e:
        return None
    return float(e["dram_bytes"]) * npx / float(e["pixels"])


def run_reference(args, rank, world):
    """CPU restatement of the reference path on host cores (rank 0 only)."""
    if rank != 0:
        return None
    import oracle
    imgs, tris, fracs = make_inputs(args.workload if args.workload != "batch64" else "1080p", 0)
    img, tri = imgs[0], tris[0]
    h, w = tri.shape
    # Bound the run to a few minutes: full image for short runs, a crop
    # otherwise (throughput per pixel is close to size-independent).
    steps = args.steps + args.warmup
    if steps > 6:
        hh, ww = h // 2, w // 2
        y0, x0 = (h - hh) // 2, (w - ww) // 2
        img, tri = img[y0:y0 + hh, x0:x0 + ww].copy(), tri[y0:y0 + hh, x0:x0 + ww].copy()
    sample = "%dx%d soft system from the %s workload" % (tri.shape[1], tri.shape[0], args.workload)
    times = []
    for s in range(steps):
        t0 = time.perf_counter()
        x, iters = oracle.solve_soft(img, tri, preconditioner="vcycle", rtol=1e-7)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    npx = tri.size
    value = npx * len(times) / sum(times) / 1e6
    line = {
        "metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": {"workload": "cf_alpha_soft_vcycle_rtol1e-7_" + args.workload,
                   "image": "%dx%d" % (tri.shape[1], tri.shape[0]),
                   "path": "cf_laplacian + make_linear_system + vcycle + cg (CPU restatement)"},
        "cpu_baseline": {"value": value, "unit": "Mpix/s", "cores": 1, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "iters": iters,
    }
    print(json.dumps(line), flush=True)
    return line


FG_METRIC = "Mpix/s of estimate_foreground_ml (reference sweep order, bit-exact for equal seeds)"


def foreground_inputs(rank):
    from pymatting_b200.synthetic import make_matting_problem
    img, _tri, alpha, _ = make_matting_problem(1080, 1920, 1 + rank, sigma=2.0, band=7,
                                               unknown_fraction=0.12, dtype=np.float32)
    return img, alpha


def run_foreground_reference(args, rank):
    """The oracle's C restatement of estimate_foreground_ml on one host core."""
    if rank != 0:
        return
    import oracle
    img, alpha = foreground_inputs(0)
    times = []
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.estimate_foreground_ml(img, alpha, return_background=True)
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            times.append(dt)
    npx = alpha.size
    value = npx * len(times) / sum(times) / 1e6
    line = {"metric": FG_METRIC, "value": value, "unit": "Mpix/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "estimate_foreground_ml_1920x1080",
                       "path": "oracle C restatement of _estimate_fb_ml, 1 core"},
            "cpu_baseline": {"value": value, "unit": "Mpix/s", "cores": 1, "kind": "port",
                             "sample": "full 1920x1080 image per step"},
            "e2e": {"value": value, "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_foreground(args, rank, world, local):
    """estimate_foreground_ml on one 1920x1080 image per GPU (weak scaling)."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import pymatting_b200 as pm
    from pymatting_b200 import _ffi
    lib = _ffi.lib()
    img, alpha = foreground_inputs(rank)
    h, w, depth = img.shape
    npx = h * w
    ti = torch.as_tensor(img, device=dev)
    ta = torch.as_tensor(alpha, device=dev)
    nb = int(lib.pmb_fg_workspace_bytes(h, w, depth))
    ws = torch.empty(nb, dtype=torch.uint8, device=dev)
    F = torch.empty((h, w, depth), dtype=torch.float32, device=dev)
    B = torch.empty_like(F)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    st = torch.cuda.current_stream().cuda_stream
    levels = pm.foreground.foreground_levels(h, w)

    def step():
        rc = lib.pmb_fg_ml(ti.data_ptr(), ta.data_ptr(), h, w, depth, 1e-5, 10, 2, 32, 1.0,
                           None, F.data_ptr(), B.data_ptr(), ws.data_ptr(), nb, st)
        assert rc == 0, _ffi.last_error()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if world > 1:
            t = torch.tensor([v], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return v

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(args.warmup):
        step()
    _ffi.check(lib.pmb_fg_status(ws.data_ptr(), st), "pmb_fg_ml")
    barrier()
    t0 = time.time()
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        step()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    clocks.window(t0, time.time())
    _ffi.check(lib.pmb_fg_status(ws.data_ptr(), st), "pmb_fg_ml")
    barrier()
    ms = max_over_ranks(sum(times) / len(times))
    # the reference's GPU backend (estimate_foreground_ml_cupy, Jacobi), same timing rules
    nbj = int(lib.pmb_fg_jacobi_workspace_bytes(h, w))
    wsj = torch.empty(nbj, dtype=torch.uint8, device=dev)

    def step_jacobi():
        rc = lib.pmb_fg_ml_jacobi(ti.data_ptr(), ta.data_ptr(), h, w, 1e-5, 10, 2, 32,
                                  F.data_ptr(), B.data_ptr(), wsj.data_ptr(), nbj, st)
        assert rc == 0, _ffi.last_error()

    for _ in range(args.warmup):
        step_jacobi()
    tj = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        step_jacobi()
        e1.record()
        torch.cuda.synchronize()
        tj.append(e0.elapsed_time(e1))
    ms_j = max_over_ranks(sum(tj) / len(tj))
    # end to end through the public API with host numpy buffers
    e2e_times = []
    for s in range(args.warmup + max(3, args.steps // 4)):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        Fh, Bh = pm.estimate_foreground_ml(img, alpha, return_background=True)
        dt = time.perf_counter() - t1
        if s >= args.warmup:
            e2e_times.append(dt)
    e2e_ms = max_over_ranks(1e3 * sum(e2e_times) / len(e2e_times))
    clock_rec = clocks.stop()
    if rank == 0:
        peak, peak_kind = measured_peaks()
        alg_bytes = npx * (depth * 4 + 4 + 2 * depth * 4)
        gbs = alg_bytes / (ms * 1e-3) / 1e9
        line = {
            "metric": FG_METRIC, "value": world * npx / (ms * 1e-3) / 1e6, "unit": "Mpix/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": "estimate_foreground_ml_1920x1080", "image": "1920x1080x3",
                       "levels": len(levels), "regularization": 1e-5,
                       "iterations": "10 on levels <= 32x32, 2 above",
                       "l2": "flushed between steps (256 MB write)",
                       "parallelism": "weak: one image per GPU, no collective"},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                         "frac": gbs / peak, "peak_source": peak_kind, "traffic": None,
                         "bytes_per_launch": alg_bytes,
                         "note": "latency-bound: each level is a wavefront of about "
                                 "h + w diagonal steps; bytes are image + alpha in, F + B out"},
            "e2e": {"value": world * npx / (e2e_ms * 1e-3) / 1e6, "unit": "Mpix/s",
                    "h2d_bytes_per_step": int(npx * (depth + 1) * 4),
                    "d2h_bytes_per_step": int(npx * 2 * depth * 4)},
            "gpu_launches": int((2 + 2 * len(levels)) * args.steps),
            "cupy_variant": {"value": world * npx / (ms_j * 1e-3) / 1e6, "unit": "Mpix/s",
                             "ms_per_step": ms_j,
                             "path": "estimate_foreground_ml_cupy drop-in (Jacobi, float32)"},
            "clocks": clock_rec,
        }
        if world == 1 and not args.no_cpu_baseline:
            import oracle
            t1 = time.perf_counter()
            oracle.estimate_foreground_ml(img, alpha, return_background=True)
            dt = time.perf_counter() - t1
            line["cpu_baseline"] = {"value": npx / dt / 1e6, "unit": "Mpix/s", "cores": 1,
                                    "kind": "port",
                                    "sample": "one full 1920x1080 estimate_foreground_ml "
                                              "(oracle C restatement), %.0f ms" % (1e3 * dt)}
            line["max_abs_vs_oracle"] = float(np.abs(Fh - oracle.estimate_foreground_ml(
                img, alpha)).max())
        print(json.dumps(line), flush=True)
    if world > 1:
        barrier()
        dist.destroy_process_group()


def cpu_baseline(img, tri):
    import oracle
    t0 = time.perf_counter()
    x, iters = oracle.solve_soft(img, tri, preconditioner="vcycle", rtol=1e-7)
    dt = time.perf_counter() - t0
    return {"value": tri.size / dt / 1e6, "unit": "Mpix/s", "cores": 1, "kind": "port",
            "sample": "one %dx%d soft-constraint vcycle CG solve to rtol 1e-7 (oracle: C "
                      "cf_laplacian, scipy make_linear_system / vcycle / cg), %d iterations, "
                      "%.1f s" % (tri.shape[1], tri.shape[0], iters, dt)}, x


def run_profile_case(args, imgs_d, tris_d, npx):
    """Small fixed cases for ncu captures (no timing is reported)."""
    import torch
    from pymatting_b200.batch import AlphaBatch
    out = {"profile": args.profile, "workload": args.workload, "pixels": int(npx)}
    precisions = {"solve-fp64": ["fp64"], "solve-mixed": ["mixed"]}.get(args.profile,
                                                                      ["fp64", "mixed"])
    for precision in precisions:
        batch = AlphaBatch(imgs_d, tris_d, precision=precision)
        if args.profile == "apply":
            batch.system.time_apply(2)
        else:
            batch.solve()
            st = batch.stats()[0]
            out[precision] = {"iters": st.iters, "outer": st.outer_iters,
                              "launches": batch.system.launch_count()}
        torch.cuda.synchronize()
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.workload == "foreground":
        if args.impl == "reference":
            run_foreground_reference(args, rank)
        else:
            run_foreground(args, rank, world, local)
        return
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    import pymatting_b200  # noqa: F401
    from pymatting_b200.batch import AlphaBatch, solve_alpha

    imgs, tris, fracs = make_inputs(args.workload, rank)
    npx = sum(t.size for t in tris)
    imgs_d = [torch.as_tensor(i, device=dev) for i in imgs]
    tris_d = [torch.as_tensor(t, device=dev) for t in tris]
    if args.profile:
        run_profile_case(args, imgs_d, tris_d, npx)
        return
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    clocks = ClockSampler(local)

    def device_step(precision):
        batch = AlphaBatch(imgs_d, tris_d, precision=precision, tune="cached")
        x = batch.solve()
        alphas = batch.alphas(x)
        return batch, x, alphas

    def timed(fn, steps):
        times, info = [], None
        t_start = time.time()
        for _ in range(steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            info = fn()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
        clocks.window(t_start, time.time())
        return times, info

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if world > 1:
            t = torch.tensor([v], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return v

    # Launch shapes: the autotuner runs once per precision before any timing
    # (its result is a cached launch configuration, not a cached output).
    tunings = {p: (AlphaBatch(imgs_d, tris_d, precision=p, tune="auto").tuning
                   if args.tune == "auto" else None) for p in ["fp64", "mixed"]}
    results = {}
    clocks.start()
    for precision in ["fp64", "mixed"]:
        for _ in range(args.warmup):
            device_step(precision)
        barrier()
        times, info = timed(lambda: device_step(precision), args.steps)
        barrier()
        total_ms = max_over_ranks(sum(times))
        batch = info[0]
        launches = sum(batch.system.launch_count() for _ in [0]) + 4 * len(imgs)
        results[precision] = dict(total_ms=total_ms, batch=batch, x=info[1],
                                  launches_per_step=launches)

    # FP64 relative residual of the mixed result, measured with the FP64
    # operator of an FP64 system on the same inputs.
    b64 = results["fp64"]["batch"]
    ax = b64.system.apply(results["mixed"]["x"])
    rel_mixed = float(torch.linalg.norm(b64.b - ax) / torch.linalg.norm(b64.b))
    ax = b64.system.apply(results["fp64"]["x"])
    rel_fp64 = float(torch.linalg.norm(b64.b - ax) / torch.linalg.norm(b64.b))
    alpha_diff = float((torch.clamp(results["mixed"]["x"], 0, 1) -
                        torch.clamp(results["fp64"]["x"], 0, 1)).abs().max())
    # Error of both results against a tight FP64 solve (rel-res 1e-12) of the
    # same system, outside the timed region: at rel-res 1e-7 weakly
    # constrained unknown regions still move, in either precision.
    stats_timed = {p: results[p]["batch"].stats()[0] for p in ["fp64", "mixed"]}
    x_tight = AlphaBatch(imgs_d, tris_d, precision="fp64").solve(rtol=1e-12)
    alpha_err = {p: float((torch.clamp(results[p]["x"], 0, 1) - torch.clamp(x_tight, 0, 1))
                          .abs().max()) for p in ["fp64", "mixed"]}

    # End to end through the public API with host buffers: pinned CPU
    # tensors in, alphas back in host memory, both copies inside the timing.
    imgs_h = [torch.from_numpy(i).pin_memory() for i in imgs]
    tris_h = [torch.from_numpy(t).pin_memory() for t in tris]
    for _ in range(max(1, args.warmup)):
        solve_alpha(imgs_h, tris_h, precision="mixed", tune="cached")
    barrier()
    e2e_times, _ = timed(lambda: solve_alpha(imgs_h, tris_h, precision="mixed", tune="cached"),
                         args.steps)
    e2e_ms = max_over_ranks(sum(e2e_times))
    clock_rec = clocks.stop()

    # Roofline of the Laplacian apply (the operator kernel of the solve).
    peak, peak_kind = measured_peaks()
    apply = {}
    for precision, es in [("mixed", 4), ("fp64", 8)]:
        ms = results[precision]["batch"].system.time_apply(50)
        bytes_alg = npx * 15 * es
        apply[precision] = dict(ms=ms, bytes=bytes_alg, gbs=bytes_alg / (ms * 1e-3) / 1e9)
    traffic = traffic_per_launch("fp32", npx)

    if rank == 0:
        k = args.steps
        value = world * npx * k / (results["mixed"]["total_ms"] * 1e-3) / 1e6
        value64 = world * npx * k / (results["fp64"]["total_ms"] * 1e-3) / 1e6
        e2e_value = world * npx * k / (e2e_ms * 1e-3) / 1e6
        st_m = stats_timed["mixed"]
        st_d = stats_timed["fp64"]
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "Mpix/s",
            "n_gpus": world,
            "steps": k,
            "warmup": args.warmup,
            "ms_per_step": results["mixed"]["total_ms"] / k,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 inner / f64 refinement",
            "data": "synthetic",
            "config": {
                "workload": "cf_alpha_soft_vcycle_rtol1e-7_" + args.workload,
                "images_per_gpu": len(imgs),
                "image": "x".join(str(s) for s in (tris[0].shape[1], tris[0].shape[0])),
                "unknown_fraction": round(float(np.mean(fracs)), 4),
                "lambda": 100.0, "epsilon": 1e-7, "preconditioner": "vcycle",
                "precision": "mixed (FP32 inner rtol 1e-4, FP64 refinement)",
                "l2": "flushed between steps (256 MB write); planes exceed L2",
                "parallelism": "weak: one image per GPU, no collective",
                "launch_shapes": {p: (t or {}).get("knobs") for p, t in tunings.items()},
            },
            "fp64_value": value64,
            "mixed_over_fp64": value / value64,
            "iters": {"mixed_inner_total": st_m.iters, "mixed_outer": st_m.outer_iters,
                      "fp64": st_d.iters},
            "rel_residual_fp64": {"mixed": rel_mixed, "fp64": rel_fp64},
            "alpha_maxabs_mixed_vs_fp64": alpha_diff,
            "alpha_maxabs_vs_fp64_rtol1e-12": alpha_err,
            "roofline": {
                "bound": "hbm",
                "kernel": "half-stencil Laplacian apply y = (L + lambda D) x, FP32",
                "achieved": apply["mixed"]["gbs"],
                "peak": peak,
                "unit": "GB/s",
                "frac": apply["mixed"]["gbs"] / peak,
                "peak_source": peak_kind,
                "traffic": traffic,
                "bytes_per_launch": apply["mixed"]["bytes"],
                "bytes_formula": "pixels x 15 values (13 half-stencil planes + x + y) x 4 B",
                "fp64": {"achieved": apply["fp64"]["gbs"], "frac": apply["fp64"]["gbs"] / peak,
                         "bytes_per_launch": apply["fp64"]["bytes"]},
            },
            "e2e": {"value": e2e_value, "unit": "Mpix/s",
                    "h2d_bytes_per_step": int(npx * (24 + 8)),
                    "d2h_bytes_per_step": int(npx * 8)},
            "gpu_launches": int(results["mixed"]["launches_per_step"] * k),
            "clocks": clock_rec,
        }
        if world == 1 and not args.no_cpu_baseline and args.workload == "1080p":
            cb, _x = cpu_baseline(imgs[0], tris[0])
            line["cpu_baseline"] = cb
        print(json.dumps(line), flush=True)
    if world > 1:
        barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
