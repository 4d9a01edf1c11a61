"""Benchmark of the B200 gas step: cell-updates/s on the 256x384 plain scene.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload plain|fine]

One step = one full gas step (advect -> diffuse -> sources -> forces ->
pressure solve to the configured tolerance -> project) of the seeded synthetic
scene: 256x384 MAC grid over 0.8 m x 1.2 m, three square logs of half-side
2.5 cm injecting fuel at 5e-3 kg/m2/s, a 1800 K Gaussian hot spot; pressure by
FP32 V(2,2) cycles inside an FP64 defect-correction loop to ||r||/||rhs|| <= 1e-6.
The state (~25 MB) fits in L2, so L2 is flushed (a 256 MB write) before every
timed step; each step is timed alone with CUDA events on the library's stream.

N > 1 runs independent replicas (one scene per rank, seeds differ): the gas
step has no data-path collective; value = all ranks' cell-updates / max-over-
ranks time ("scaling": "weak").

--impl reference times the reference's CPU implementation of the step on this
box's host cores: the C++ restatement of the WGSL (the reference's WGSL needs a
WebGPU stack that does not exist here), FP32, OpenMP over all host threads.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (nx, ny, scene kind, seed, solver mode, tol, max cycles)
    "plain": (256, 384, 0, 1235, 2, 1e-6, 200),
    "fine": (512, 768, 1, 1236, 2, 1e-10, 300),
}
METRIC = "cell-updates/s"
PLAIN_CFL, PLAIN_DT_CAP = 0.5, 2e-3   # the plain workload's time step: CFL 0.5, at most 2 ms
# algorithmic bytes per cell-update (reference schedule, one read + one write per element at storage width):
# advect 156, diffuse 48 per sub-step, sources 68, forces 28, coef 20, rhs0 28, coefRestrict 13.3, project 32,
# V(2,2) cycle 216.8, FP64 defect-correction iteration 40, FP64 rhs assembly 12
B_FIXED = 156 + 68 + 28 + 20 + 28 + 13.3 + 32


# DRAM bytes (read + write) per launch of a kernel, from one ncu capture of the workload
NCU_TRAFFIC = {("plain", "mg_coarse"): 123904, ("plain", "advect"): 2967808}


def bytes_per_cell(diff_sub: int, cycles: float, fp64: bool) -> float:
    b = B_FIXED + 48.0 * diff_sub + 216.8 * cycles
    if fp64:
        b += 40.0 * cycles + 12.0
    return b


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0])); mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_cpu(workload: str, steps: int, warmup: int, threads: int):
    """The CPU restatement of the reference step (oracle, f32), same scene and solver."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    from oracle import oracle
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[workload]
    sc = cb.generate_scene(kind, nx, ny, 0.8, seed)
    o = oracle.OracleSim(nx, ny, 0.8, sc["dt"])
    load_scene(o, sc)
    o.set_solver(mode, 1, tol, maxc)
    o.set_cfl(PLAIN_CFL, PLAIN_DT_CAP)
    o.step(warmup)
    cyc = 0.0
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step(1)
        cyc += o.info()["last_cycles"]
    dt = time.perf_counter() - t0
    return nx * ny * steps / dt, dt, cyc / max(steps, 1)


BATCH_CLASSES = ((96, 144), (128, 192), (192, 288), (256, 384))


def batch_scenes(n: int = 64, seed: int = 2000):
    """64 floor-log scenes of uneven size: size class uniform, 2-6 logs, B x logU[0.5,2], YOamb ~ U[0.18,0.233]."""
    import numpy as np
    import campfire_b200 as cb
    idx = np.random.default_rng(seed).integers(0, len(BATCH_CLASSES), n)
    return [cb.generate_scene(2, *BATCH_CLASSES[i], 0.8, seed + k) for k, i in enumerate(idx)]


def run_batched(dev, stream, flush, steps: int, warmup: int, tol: float, max_cycles: int, plain_steps: int):
    """Batched gas step of 64 uneven scenes (one launch per kernel for all scenes, one graph per step)
    against the same scenes stepped one by one with the plain single-scene step."""
    import torch
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    scenes = batch_scenes()
    cells = sum(s["nx"] * s["ny"] for s in scenes)
    b = cb.Batch([(s["nx"], s["ny"]) for s in scenes], 0.8, [s["dt"] for s in scenes], device=dev.index)
    for v, s in zip(b.scenes, scenes):
        load_scene(v, s)
    b.set_solver(cb.SOLVE_FP64, 1, tol, max_cycles)
    b.set_coarse_solve("pipelined")
    b.set_krylov(True)
    tune = cb.autotune([(s["nx"], s["ny"]) for s in scenes], iters=10, device=dev.index, coarse_direct=True)
    b.set_coarse_cells(tune["best"])
    b.set_stream(stream.cuda_stream)
    b.step(warmup)
    b.synchronize()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        b.step(1)
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    b.synchronize()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    cyc = [v.info()["last_cycles"] for v in b.scenes]
    rel = max(v.info()["last_rel"] for v in b.scenes)
    launches = b.launch_count()
    b.close()
    batched = cells * steps / (ms / 1e3)

    # the same scenes, one by one, through the plain single-scene step (same solver, same tolerance)
    plain_ms, plain_cells = 0.0, 0
    best = {d: cb.autotune([d], iters=10, device=dev.index, coarse_direct=True)["best"] for d in BATCH_CLASSES}
    for s in scenes:
        g = cb.FluidSim(dev.index, {"nx": s["nx"], "ny": s["ny"], "dt": s["dt"]}, width=0.8).init()
        load_scene(g, s)
        g.set_solver(cb.SOLVE_FP64, 1, tol, max_cycles)
        g.set_coarse_solve("pipelined")
        g.set_krylov(True)
        g.set_coarse_cells(best[(s["nx"], s["ny"])])
        g.set_stream(stream.cuda_stream)
        g.step(warmup)
        g.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        flush.fill_(0.0)
        e0.record(stream)
        g.step(plain_steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        g.synchronize()
        plain_ms += e0.elapsed_time(e1)
        plain_cells += s["nx"] * s["ny"] * plain_steps
        g.close()
    plain = plain_cells / (plain_ms / 1e3)
    return {"value": batched, "unit": METRIC, "scenes": len(scenes), "cells": cells, "steps": steps,
            "schedule": {"coarse_cells": tune["best"],
                         "autotune_ms_per_cycle": {str(k): round(v, 5) for k, v in tune["ms_per_cycle"].items()}},
            "ms_per_step": ms / steps, "launches_per_step": launches,
            "pressure": {"mode": "fp64_defect_correction", "tol": tol, "max_cycles": max_cycles,
                         "cycles_last_step": {"min": min(cyc), "max": max(cyc)}, "max_rel_residual": rel},
            "sizes": {f"{nx}x{ny}": sum(1 for s in scenes if (s["nx"], s["ny"]) == (nx, ny))
                      for nx, ny in BATCH_CLASSES},
            "plain_one_by_one": {"value": plain, "unit": METRIC, "steps_per_scene": plain_steps},
            "batched_over_plain": batched / plain}


def field_errors(g, ref):
    """max|gpu - ref| / max|ref| of T, u (U and V faces), Y_F and Y_S."""
    import numpy as np
    out = {}
    for name, get in (("T", lambda s, r: (s("T"),)), ("u", lambda s, r: (s("U"), s("V"))),
                      ("Y_F", lambda s, r: (s("Y").reshape(-1, 4)[:, 0],)),
                      ("Y_S", lambda s, r: (s("Y").reshape(-1, 4)[:, 3],))):
        a = np.concatenate([np.asarray(x, np.float64).ravel() for x in get(g.readBuffer, None)])
        b = np.concatenate([np.asarray(x, np.float64).ravel() for x in get(ref.read, None)])
        scale = float(np.max(np.abs(b))) or 1.0
        out[name] = float(np.max(np.abs(a - b))) / scale
    return out


def run_fp64_error(dev, workload: str, steps: int, every: int, threads: int):
    """The GPU step (FP32, FP64 defect correction) and the FP64 oracle (the same algorithm in
    double precision) from the same scene, side by side; errors every `every` steps."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    from oracle import oracle
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[workload]
    sc = cb.generate_scene(kind, nx, ny, 0.8, seed)
    g = cb.FluidSim(dev.index, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    g.set_solver(mode, 1, tol, maxc)
    g.set_coarse_solve("pipelined")
    g.set_krylov(True)
    g.set_cfl(PLAIN_CFL, PLAIN_DT_CAP)
    o = oracle.OracleSim(nx, ny, 0.8, sc["dt"], fp64=True)
    load_scene(o, sc)
    o.set_solver(mode, 1, tol, maxc)
    o.set_cfl(PLAIN_CFL, PLAIN_DT_CAP)
    rows = []
    for k in range(1, steps + 1):
        g.step(1)
        o.step(1)
        if k % every == 0 or k == 1:
            rows.append(dict(step=k, **field_errors(g, o)))
    g.close()
    return {"workload": workload, "steps": steps, "every": every, "errors": rows,
            "metric": "max|gpu - fp64 oracle| / max|fp64 oracle| per field"}


SERVE_CLASSES = ((96, 144), (128, 192), (192, 288), (256, 384), (512, 768))


def served_jobs(lam: float, njobs: int, steps_lo: int, steps_hi: int, seed: int):
    """Poisson arrivals at rate lam; size class uniform; tepee scenes (scene kind 1); N uniform."""
    import numpy as np
    rng = np.random.default_rng(seed)
    t, jobs = 0.0, []
    for k in range(njobs):
        t += float(rng.exponential(1.0 / lam))
        jobs.append({"size_class": int(rng.integers(0, len(SERVE_CLASSES))), "kind": 1, "seed": 9000 + k,
                     "nsteps": int(rng.integers(steps_lo, steps_hi + 1)), "arrival_s": t})
    return jobs


def run_served(dev, stream, lams, njobs: int, steps_lo: int, steps_hi: int, slots: int, budget: float, tol: float):
    """The serving loop (continuous batching, HBM-budget admission) at several arrival rates, against the
    same jobs served one by one by the plain single-scene step (FIFO; each job's time from the measured
    plain ms/step of its size class)."""
    import numpy as np
    import torch
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    # plain per-step time of each size class (same solver), for the one-by-one schedule
    plain_ms = {}
    for c, (nx, ny) in enumerate(SERVE_CLASSES):
        sc = cb.generate_scene(1, nx, ny, 0.8, 9000)
        g = cb.FluidSim(dev.index, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
        load_scene(g, sc)
        g.set_solver(cb.SOLVE_FP64, 1, tol, 300)
        g.set_coarse_solve("pipelined")
        g.set_krylov(True)
        g.set_stream(stream.cuda_stream)
        g.step(3)
        g.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        g.step(5)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        plain_ms[c] = e0.elapsed_time(e1) / 5
        g.close()
    srv = cb.Server(SERVE_CLASSES, [slots] * len(SERVE_CLASSES), budget, device=dev.index)
    srv.set_solver(cb.SOLVE_FP64, 1, tol, 300, "pipelined", krylov=True)
    out = []
    for lam in lams:
        jobs = served_jobs(lam, njobs, steps_lo, steps_hi, seed=int(lam) + 17)
        res, wall, cu = srv.run(jobs)
        lat = np.array([r["done_s"] - r["arrival_s"] for r in res])
        # one by one, first come first served, with the plain step
        t_free, lat1 = 0.0, []
        for j in sorted(jobs, key=lambda q: q["arrival_s"]):
            start = max(j["arrival_s"], t_free)
            t_free = start + j["nsteps"] * plain_ms[j["size_class"]] / 1e3
            lat1.append(t_free - j["arrival_s"])
        lat1 = np.array(lat1)
        cells = sum(SERVE_CLASSES[j["size_class"]][0] * SERVE_CLASSES[j["size_class"]][1] * j["nsteps"] for j in jobs)
        out.append({"lambda_jobs_per_s": lam, "jobs": njobs, "value": cu / wall, "unit": METRIC,
                    "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                    "wall_s": wall, "max_rel_residual": max(r["last_rel"] for r in res),
                    "one_by_one": {"value": cells / t_free if t_free > 0 else None, "unit": METRIC,
                                   "p50_latency_s": float(np.percentile(lat1, 50)),
                                   "p99_latency_s": float(np.percentile(lat1, 99))}})
    srv.close()
    return {"classes": [f"{a}x{b}" for a, b in SERVE_CLASSES], "slots_per_class": slots, "budget_bytes": budget,
            "steps_per_job": [steps_lo, steps_hi], "scene": "tepee (five logs of half 5 cm), FP64 defect correction "
            f"to {tol:g}, pipelined direct coarsest", "one_by_one_model": "FIFO over the same jobs with each class's measured "
            "plain single-scene ms/step", "plain_ms_per_step": {f"{a}x{b}": plain_ms[c] for c, (a, b) in
                                                                enumerate(SERVE_CLASSES)},
            "runs": out}


APP_MODE = (224, 320, 0.003)    # the app's "balanced" grid (js/config.js:8), width 0.7 m
APP_IMAGE = (734, 1080)          # a canvas 1080 pixels high with the domain's aspect (ground strip included)


def run_app_frames(dev, stream, frames: int, warmup: int):
    """The campfire app's frame (js/main.js:247-283) on its default scene (defaultScene, :132-155):
    the rigid bodies advance and exchange heat at their contacts, the wood model steps on the host,
    pieces are uploaded and rasterised, the frame's gas steps run (reference solver: one V-cycle per
    step), then radiation, the synchronous readback and the wood coupling, and the photo view is
    rendered into device memory. Wall-clock per frame with a stream synchronisation at its end."""
    import numpy as np
    import torch
    import campfire_b200 as cb
    from campfire_b200.render import Renderer, render_device
    from campfire_b200.wood import WoodScene, app_rigid_options, default_scene
    nx, ny, dt = APP_MODE
    W, H = APP_IMAGE
    sim = cb.FluidSim(dev.index, {"nx": nx, "ny": ny, "dt": dt}, width=0.7).init()
    sim.set_stream(stream.cuda_stream)
    sim.set_solver(cb.SOLVE_FIXED, 1)
    sim.writeParams()
    sim.reset()
    ws = WoodScene(sim, rigid=app_rigid_options())
    npieces = len(default_scene(ws))
    ren = Renderer(sim)
    img = torch.empty(H * W * 4, dtype=torch.float32, device=dev)
    frame_dt = 1.0 / 60.0
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(frames)]
    steps = 0
    wall = 0.0
    for k in range(warmup + frames):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        n = ws.frame(frame_dt)
        ren.writeParams({"view": 0, "exposure": 1.0, "time": sim.info()["time"]})
        ren.writeWood(ws)
        if k >= warmup:
            ev[k - warmup][0].record(stream)
        render_device(sim, ren.rp, W, H, img.data_ptr(), ren.wood)
        if k >= warmup:
            ev[k - warmup][1].record(stream)
        stream.synchronize()
        if k >= warmup:
            wall += time.perf_counter() - t0
            steps += n
    render_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    st = ws.stats()
    ws.close()
    sim.close()
    px = W * H
    return {"scene": f"the app's default fire ({npieces} moving pieces: 7 coals, 2 logs, 7 sticks), {nx}x{ny} "
                     f"cells, dt {dt}, one V-cycle per step", "frame_sim_dt_s": frame_dt, "frames": frames,
            "warmup_frames": warmup, "image": [W, H], "frames_per_s": frames / wall,
            "ms_per_frame": 1e3 * wall / frames, "gas_steps_per_frame": steps / frames,
            "sim_time_per_wall_time": steps * dt / wall,
            "render_ms": float(np.median(render_ms)), "render_mpixel_per_s": px / (np.median(render_ms) / 1e3) / 1e6,
            "last_frame_stats": {"hrr_w_per_m": st["hrr"], "rad_w_per_m": st["rad"], "tmax_k": st["tmax"]}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-sample", type=int, default=3, help="steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batched-steps", type=int, default=10,
                    help="timed steps of the 64-scene batched measurement added to the line (0: skip)")
    ap.add_argument("--served-jobs", type=int, default=40,
                    help="jobs per arrival rate of the serving measurement added to the line (0: skip)")
    ap.add_argument("--served-steps", type=int, nargs=2, default=(20, 200), metavar=("LO", "HI"),
                    help="steps per served job, uniform in [LO, HI]")
    ap.add_argument("--served-rates", type=float, nargs="+", default=(10.0, 100.0, 1000.0))
    ap.add_argument("--app-frames", type=int, default=120,
                    help="timed frames of the app frame measurement (wood coupling + gas steps + render) "
                         "added to the line (0: skip)")
    ap.add_argument("--fp64-error-every", type=int, default=0,
                    help="with --fp64-error-steps S: run the workload beside the FP64 oracle for S steps and "
                         "report the field errors every this many steps (0: skip)")
    ap.add_argument("--fp64-error-steps", type=int, default=2000)
    ap.add_argument("--coarse-cells", type=int, default=0,
                    help="start the coarse block at the first level with at most this many cells instead of "
                         "autotuning (0: autotune); for profiling runs whose launch indices must not depend on "
                         "the autotuner")
    ap.add_argument("--launch", default="graph", choices=["graph", "stream"],
                    help="graph: one CUDA graph per step (pressure loop as a device-side WHILE node); "
                         "stream: kernel by kernel, the host polling the loop decision (for profilers that "
                         "do not list kernels inside conditional graph nodes)")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(a.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[a.workload]
    config = {"workload": f"{a.workload} gas step {nx}x{ny}, 3 logs, FP32 V(2,2) in FP64 defect correction "
                          f"to rel residual {tol:g}", "nx": nx, "ny": ny, "scene_seed": seed,
              "pressure": {"mode": "fp64_defect_correction", "tol": tol, "max_cycles": maxc},
              "l2": "flushed before every timed step (256 MB write)", "parallelism": f"replicas{world}"}

    if a.impl == "reference":
        if rank != 0:
            return
        th = cpu_threads()
        val, secs, cyc = run_cpu(a.workload, a.steps, a.warmup, th)
        line = {"metric": METRIC, "value": val, "unit": METRIC, "impl": "reference", "n_gpus": a.gpus,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * secs / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(config, cycles_per_step=cyc),
                "cpu_baseline": {"value": val, "unit": METRIC, "cores": th, "kind": "port",
                                 "sample": f"{a.steps} steps of the {nx}x{ny} workload after {a.warmup} warm-up steps "
                                           "(C++ restatement of the reference WGSL, f32, OpenMP)"},
                "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # one non-default stream shared by the library, the L2 flush and the timing events
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)

    sc = cb.generate_scene(kind, nx, ny, 0.8, seed + 1000 * rank)
    sim = cb.FluidSim(local, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(sim, sc)
    sim.set_solver(mode, 1, tol, maxc)
    sim.set_coarse_solve("pipelined")
    sim.set_krylov(True)
    sim.set_cfl(PLAIN_CFL, PLAIN_DT_CAP)   # dt set by CFL 0.5 each step, capped at 2 ms
    config["dt"] = {"cfl": PLAIN_CFL, "cap_s": PLAIN_DT_CAP}
    config["pressure"]["coarsest"] = "direct: inverse factored beside the pressure loop, applied from the next step (pipelined)"
    config["pressure"]["outer"] = "flexible preconditioned CG in FP64, FP32 V(2,2) as preconditioner"
    # smoother schedule picked by the autotuner (fused V-cycles timed on a scratch scene of this size)
    if a.coarse_cells > 0:
        sim.set_coarse_cells(a.coarse_cells)
        config["schedule"] = {"coarse_cells": a.coarse_cells, "autotune": "skipped"}
    else:
        tune = cb.autotune([(nx, ny)], iters=20, device=local, coarse_direct=True)
        sim.set_coarse_cells(tune["best"])
        config["schedule"] = {"coarse_cells": tune["best"],
                              "autotune_ms_per_cycle": {str(k): round(v, 5) for k, v in tune["ms_per_cycle"].items()}}
    sim.set_stream(stream.cuda_stream)
    sim.set_graphs(a.launch == "graph")
    config["launch"] = a.launch
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    sim.step(a.warmup)
    sim.synchronize()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    cycles = []
    clocks = ClockSampler(local)
    clocks.start()
    for k in range(a.steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        sim.step(1)
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clk = clocks.stop()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    info = sim.info()
    sim.synchronize()
    launches = sim.launch_count()
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * nx * ny * a.steps / (ms_max / 1e3)

    # ---- end to end through the C ABI: per step upload params + pieces from pinned host
    # memory, step, read the accumulators back (the frame data flow of js/main.js:266-283)
    pin_pieces = torch.from_numpy(sc["pieces"].copy()).pin_memory()
    acc = torch.zeros(528, dtype=torch.int32).pin_memory()
    rad = torch.zeros(320 * 4, dtype=torch.float32).pin_memory()
    fw = torch.zeros(256, dtype=torch.int32).pin_memory()
    L = cb.lib()
    fptr = ctypes.cast(pin_pieces.data_ptr(), ctypes.POINTER(ctypes.c_float))
    i32 = ctypes.POINTER(ctypes.c_int32)
    e2e_steps = max(5, min(50, a.steps // 4))
    barrier()
    e2e_s = 0.0
    for k in range(e2e_steps):
        flush.fill_(float(k))
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        cb._lib.check(L.cfg_upload_pieces(sim._h, fptr, sc["npieces"]))
        cb._lib.check(L.cfg_write_params(sim._h))
        cb._lib.check(L.cfg_step(sim._h, 1))
        cb._lib.check(L.cfg_readback(sim._h, ctypes.cast(acc.data_ptr(), i32),
                                     ctypes.cast(rad.data_ptr(), ctypes.POINTER(ctypes.c_float)),
                                     ctypes.cast(fw.data_ptr(), i32)))
        e2e_s += time.perf_counter() - t0
    t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * nx * ny * e2e_steps / float(t.item())

    # ---- roofline of the dominant kernel (device time per step share), measured after the timed region
    hbm, peak_kind = peaks()
    kern = {}
    for name in ("advect", "diffuse_sources", "forces", "mg_down0", "mg_up0", "mg_coarse", "pcg_step", "defect64",
                 "project"):
        m, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        cb._lib.check(L.cfg_time_kernel(sim._h, name.encode(), 50, ctypes.byref(m), ctypes.byref(b), ctypes.byref(n)))
        kern[name] = {"ms": m.value, "bytes": b.value, "per_step": n.value, "share_ms": m.value * n.value}
    dom = max(kern, key=lambda k: kern[k]["share_ms"])
    dk = kern[dom]
    achieved = dk["bytes"] / (dk["ms"] / 1e3) / 1e9
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_source": f"{peak_kind} hbm_gbs (copy bandwidth)",
            "traffic": NCU_TRAFFIC.get((a.workload, dom)), "traffic_source": "ncu dram__bytes_read.sum + "
            "dram__bytes_write.sum, one capture of this workload (--set full)",
            "bytes_per_launch": dk["bytes"], "launch_ms": dk["ms"],
            "step_bytes_per_cell": bytes_per_cell(info["diffSub"], info["last_cycles"], True),
            "step_frac": (value / world) * bytes_per_cell(info["diffSub"], info["last_cycles"], True) / 1e9 / hbm,
            "kernels": {k: {"ms": round(v["ms"], 5), "per_step": v["per_step"]} for k, v in kern.items()}}

    batched = None
    if a.batched_steps > 0:
        batched = run_batched(dev, stream, flush, a.batched_steps, 3, 1e-10, 300, 3)

    fp64_error = None
    if a.fp64_error_every > 0 and rank == 0:
        fp64_error = run_fp64_error(dev, a.workload, a.fp64_error_steps, a.fp64_error_every, cpu_threads())

    served = None
    if a.served_jobs > 0:
        served = run_served(dev, stream, a.served_rates, a.served_jobs, a.served_steps[0], a.served_steps[1],
                            slots=12, budget=150e9, tol=1e-10)

    app = None
    if a.app_frames > 0:
        app = run_app_frames(dev, stream, a.app_frames, 30)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        th = cpu_threads()
        val, secs, cyc = run_cpu(a.workload, a.cpu_sample, 1, th)
        cpu = {"value": val, "unit": METRIC, "cores": th, "kind": "port",
               "sample": f"{a.cpu_sample} steps of the same {nx}x{ny} workload after 1 warm-up step "
                         f"(C++ restatement of the reference WGSL, f32, OpenMP; the reference's V-cycle and "
                         f"coarsest sweeps in the plain FP64 defect correction to the same tolerance: "
                         f"{cyc:.1f} V-cycles/step)"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(config, cycles_last_step=info["last_cycles"], diff_sub=info["diffSub"],
                               levels=info["levels"]),
                # H2D: the piece buffer, the descriptor's parameter block (uniform + step controls, 204 B)
                # and dx/alpha of the diffusion rule (16 B); D2H: acc + rad + faceW
                "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 64 * 20 * 4 + 204 + 16,
                        "d2h_bytes_per_step": 528 * 4 + 320 * 16 + 256 * 4},
                "gpu_launches": launches * a.steps, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
                "batched": batched, "served": served, "app_frame": app, "fp64_oracle_error": fp64_error}
        print(json.dumps(line))
    sim.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
