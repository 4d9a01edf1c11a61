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
# cycle shape of each workload's pressure loop: the W tail (the level two above the coarsest visits the
# level below it twice per cycle, inside the one-CTA coarse block) when that level has at most this many
# cells; 0: the reference's V(2,2) cycle. On the tepee scenes the coarse levels limit the FP64 loop's
# convergence: the W tail takes ~19% fewer cycles to 1e-10 at 512x768 (oracle: 18.8 -> 15.2 per step) for
# a few more coarse-block phases per cycle; the three-log scene at 1e-6 gains nothing.
W_CELLS = {"plain": 0, "fine": 1536}
SERVE_W_CELLS = 1536                  # the served jobs are tepee scenes too
METRIC = "cell-updates/s"
PLAIN_CFL, PLAIN_DT_CAP = 0.5, 2e-3   # the plain workload's time step: CFL 0.5, at most 2 ms
# algorithmic bytes per cell-update (reference schedule, one read + one write per element at storage width):
# advect 156, diffuse 48 per sub-step, sources 68, forces 28, coef 20, rhs0 28, coefRestrict 13.3, project 32,
# V(2,2) cycle 216.8, FP64 defect-correction iteration 40, FP64 rhs assembly 12
B_FIXED = 156 + 68 + 28 + 20 + 28 + 13.3 + 32


# DRAM bytes (read + write) per launch of a kernel, from one ncu capture of the workload
NCU_TRAFFIC = {("plain", "mg_coarse"): 157440, ("plain", "advect"): 2967808,
               ("fine", "mg_up0_krylov"): 16266752, ("fine", "mg_down0_krylov"): 20596736,
               ("batched", "mg_down0"): 43902464}


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
    """SM clocks and clock-event (throttle) reasons sampled during the timed region: NVML read every 2 ms
    from a thread (read-only queries), so that even a timed region of a few tens of milliseconds holds
    samples; nvidia-smi at its 20 ms period when NVML is not importable."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []
        self.nvml, self.samples, self.reasons, self.max_mhz = None, [], set(), None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = self._handle(pynvml, index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            self.bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                         "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                         "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                         "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
        except Exception:
            self.nvml = None

    @staticmethod
    def _handle(pynvml, index: int):
        """The NVML handle of CUDA device `index` (matched by PCI bus id: NVML numbers every GPU of the
        machine, CUDA only the visible ones)."""
        try:
            import torch
            p = torch.cuda.get_device_properties(index)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(index)

    def start(self):
        if self.nvml is not None:
            self.stop_evt = threading.Event()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _sample(self):
        nv = self.nvml
        self.samples.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
        r = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
        for n, b in self.bits.items():
            if r & b:
                self.reasons.add(n)

    def _poll(self):
        try:
            while True:
                self._sample()
                if self.stop_evt.wait(0.002):
                    break
        except Exception:
            pass

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_evt.set()
            self.t.join(timeout=5)
            sm = sorted(self.samples)
            return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": self.max_mhz,
                    "reasons": sorted(self.reasons), "samples": len(sm), "source": "nvml, 2 ms period"}
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0])); mx = float(f[1])
            except ValueError:
                continue
            for n, v in zip(self.NAMES, f[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 20 ms period"}


def cpu_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def workload_config(workload: str, world: int, w_cells=None) -> dict:
    """The workload as both arms run it (scene, grid, solver, time step, L2 policy): the same dict in the
    line of this implementation and of the reference arm (w_cells: the cycle shape's override)."""
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[workload]
    w = W_CELLS[workload] if w_cells is None else w_cells
    scene = {0: "3 logs", 1: "5-log tepee"}[kind]
    return {"workload": f"{workload} gas step {nx}x{ny}, {scene}, FP32 V(2,2) in FP64 defect correction "
                        f"to rel residual {tol:g}", "nx": nx, "ny": ny, "scene_kind": kind, "scene_seed": seed,
            "pressure": {"mode": "fp64_defect_correction", "tol": tol, "max_cycles": maxc,
                         "outer": "flexible preconditioned CG in FP64, FP32 multigrid cycle as preconditioner",
                         "cycle": cycle_name(w),
                         "coarsest": "direct: inverse factored beside the pressure loop, applied from the next "
                                     "step (pipelined)"},
            "dt": {"cfl": PLAIN_CFL, "cap_s": PLAIN_DT_CAP},
            "l2": "flushed before every timed step (256 MB write)", "parallelism": f"replicas{world}"}


def configure_solver(sim, workload: str, w_cells=None) -> None:
    """The workload's solver on a FluidSim or an OracleSim (same calls on both); w_cells overrides the
    workload's cycle shape."""
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[workload]
    sim.set_solver(mode, 1, tol, maxc)
    sim.set_coarse_solve("pipelined")
    sim.set_krylov(True)
    sim.set_cfl(PLAIN_CFL, PLAIN_DT_CAP)   # dt set by CFL 0.5 each step, capped at 2 ms
    sim.set_coarse_w(W_CELLS[workload] if w_cells is None else w_cells)


def cycle_name(w_cells: int) -> str:
    return ("V(2,2)" if w_cells <= 0 else
            f"V(2,2) with a W tail: the level two above the coarsest (at most {w_cells} cells) visits the level "
            "below it twice per cycle (inside the one-CTA coarse block)")


def run_cpu(workload: str, steps: int, warmup: int, threads: int, w_cells=None):
    """The CPU restatement of the reference step (oracle, f32) on the same scene with the same solver.
    Inputs come from the oracle's own scene restatement: the product library is not loaded."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle, scene_ref
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[workload]
    sc = scene_ref.generate_scene(kind, nx, ny, 0.8, seed)
    o = oracle.OracleSim(nx, ny, 0.8, sc["dt"])
    scene_ref.load_scene(o, sc)
    configure_solver(o, workload, w_cells)
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
    tt = cb.autotune_tiles([(s["nx"], s["ny"]) for s in scenes], iters=10, device=dev.index)
    b.set_tiles(*tt["best"])
    b.set_stream(stream.cuda_stream)
    b.step(warmup)
    b.synchronize()
    # the Krylov update: its own kernel per cycle, or folded into the level-0 smoother kernels (a
    # one-CTA-per-scene decision kernel ends each cycle), which needs every scene's coarse block
    # below level 0. Candidates: the autotuner's coarse level with the update kernel, and the
    # largest timed coarse level below every scene's level 0 with the fold; each timed over
    # whole steps, interleaved (the scenes' cycle counts drift from step to step), the faster kept
    min_cells = min(s["nx"] * s["ny"] for s in scenes)
    cands = [(tune["best"], 3)]
    below = [c for c in tune["ms_per_cycle"] if c < min_cells]
    if below:
        cands.append((max(below), 2))
    cand_ms = {c: 0.0 for c in cands}
    folded = {}
    for rnd in range(2):
        for c in cands:
            b.set_coarse_cells(c[0])
            b.set_krylov(c[1])
            folded[c] = b.krylov_folded()
            b.step(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.step(3)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            b.synchronize()
            cand_ms[c] += e0.elapsed_time(e1) / 6
    kept = min(cand_ms, key=cand_ms.get)
    b.set_coarse_cells(kept[0])
    b.set_krylov(kept[1])
    fold = kept[1] if folded[kept] else 3
    b.step(1)
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
    infos = [v.info() for v in b.scenes]
    cyc = [i["last_cycles"] for i in infos]
    rel = max(i["last_rel"] for i in infos)
    launches = b.launch_count()
    b.close()
    batched = cells * steps / (ms / 1e3)
    # algorithmic bytes of the last step: each scene's cells x its own bytes per cell-update (its cycles)
    step_bytes = sum(sc_["nx"] * sc_["ny"] * bytes_per_cell(i["diffSub"], i["last_cycles"], True)
                     for sc_, i in zip(scenes, infos))
    hbm, peak_kind = peaks()
    achieved = step_bytes / (ms / steps / 1e3) / 1e9

    # the same scenes, one by one, through the plain single-scene step (same solver, same tolerance)
    plain_ms, plain_cells = 0.0, 0
    best = {d: cb.autotune([d], iters=10, device=dev.index, coarse_direct=True)["best"] for d in BATCH_CLASSES}
    best_tiles = {d: cb.autotune_tiles([d], iters=10, device=dev.index)["best"] for d in BATCH_CLASSES}
    for s in scenes:
        g = cb.FluidSim(dev.index, {"nx": s["nx"], "ny": s["ny"], "dt": s["dt"]}, width=0.8).init()
        load_scene(g, s)
        g.set_solver(cb.SOLVE_FP64, 1, tol, max_cycles)
        g.set_coarse_solve("pipelined")
        g.set_krylov(True)
        g.set_coarse_cells(best[(s["nx"], s["ny"])])
        g.set_tiles(*best_tiles[(s["nx"], s["ny"])])
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
            "schedule": {"coarse_cells": kept[0],
                         "autotune_ms_per_cycle": {str(k): round(v, 5) for k, v in tune["ms_per_cycle"].items()},
                         "krylov_update": "folded into the level-0 kernels" if fold == 2 else "own kernel",
                         "candidates_ms_per_step": {f"coarse {c[0]}, " + ("folded" if folded[c] else "own kernel"):
                                                    round(v, 4) for c, v in cand_ms.items()},
                         "tiles": {"advect": cb.TILE_SHAPES[tt["best"][0]],
                                   "diffuse_sources": cb.TILE_SHAPES[tt["best"][1]],
                                   "forces": cb.TILE_SHAPES[tt["best"][2]],
                                   "autotune_ms": {k: [round(x, 5) for x in v] for k, v in tt["ms"].items()}}},
            "ms_per_step": ms / steps, "launches_per_step": launches,
            "pressure": {"mode": "fp64_defect_correction", "tol": tol, "max_cycles": max_cycles,
                         "cycles_last_step": {"min": min(cyc), "max": max(cyc)}, "max_rel_residual": rel},
            "sizes": {f"{nx}x{ny}": sum(1 for s in scenes if (s["nx"], s["ny"]) == (nx, ny))
                      for nx, ny in BATCH_CLASSES},
            "plain_one_by_one": {"value": plain, "unit": METRIC, "steps_per_scene": plain_steps},
            "batched_over_plain": batched / plain,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "peak_source": f"{peak_kind} hbm_gbs (copy bandwidth)",
                         "step_bytes": step_bytes, "bytes_per_cell": step_bytes / cells,
                         "basis": "algorithmic bytes of the last step (each scene's cycles) / mean ms per step",
                         "traffic": {"kernel": "mg_down0", "bytes": NCU_TRAFFIC[("batched", "mg_down0")],
                                     "algorithmic_bytes": 82.0 * cells,
                                     "source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one launch of "
                                               "the level-0 down kernel of this batch (cold replay)"}}}


ERR_FIELDS = ("T", "u", "Y_F", "Y_S")


def _err_arrays(read):
    """T, u (U and V faces), Y_F and Y_S of a sim, as float64 arrays (`read`: readBuffer or OracleSim.read)."""
    import numpy as np
    y = np.asarray(read("Y"), np.float64).reshape(-1, 4)
    return {"T": np.asarray(read("T"), np.float64),
            "u": np.concatenate([np.asarray(read("U"), np.float64), np.asarray(read("V"), np.float64)]),
            "Y_F": y[:, 0], "Y_S": y[:, 3]}


def field_errors(read_a, read_ref, detail: bool = False):
    """Per field |a - ref| / max|ref|: its maximum, and with `detail` its 99.9th percentile and the fraction of
    values above 1e-4 (a single cell whose limiter or chemistry branch flips under a rounding difference sets
    the maximum; the percentile shows the rest of the field)."""
    import numpy as np
    a, b = _err_arrays(read_a), _err_arrays(read_ref)
    out = {}
    for f in ERR_FIELDS:
        d = np.abs(a[f] - b[f]) / (float(np.max(np.abs(b[f]))) or 1.0)
        out[f] = {"max": float(d.max()), "p99_9": float(np.quantile(d, 0.999)),
                  "frac_above_1e-4": float(np.mean(d > 1e-4))} if detail else float(d.max())
    return out


def run_fp64_error(dev, workload: str, steps: int, every: int, threads: int):
    """Accuracy of the GPU step (FP32 arithmetic, FP64 pressure to the workload's tolerance) against the FP64
    oracle (the same algorithm in double precision), reported at step 1 and every `every` steps:
      one_step    the step after the report, from the GPU's state: that state is copied into an FP64 oracle
                  and into the CPU FP32 restatement, and all three take the step; errors against the FP64 one
      trajectory  the GPU run and an FP64 oracle run from the same initial scene, and the FP32 restatement's
                  own run against the FP64 one (the flame amplifies rounding: FP32 drift, not a defect; the
                  FP64 oracle also rasterises the pieces in FP64, so a face that is barely open in FP32 can
                  be closed there, which moves u at that face from the first step on)"""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    from oracle import oracle, scene_ref
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[workload]
    sc = cb.generate_scene(kind, nx, ny, 0.8, seed)
    g = cb.FluidSim(dev.index, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    configure_solver(g, workload)

    def osim(fp64):
        o = oracle.OracleSim(nx, ny, 0.8, sc["dt"], fp64=fp64)
        scene_ref.load_scene(o, sc)
        configure_solver(o, workload)
        return o

    traj64, traj32 = osim(True), osim(False)
    t0 = time.perf_counter()
    reports, probe, k = [], None, 0
    while k < steps or probe is not None:   # the last report's probed step may run past `steps`
        if probe is not None:    # the probed step: the GPU state copied into fresh oracles first
            one64, one32 = osim(True), osim(False)
            one64.copy_state_from(g, PLAIN_CFL, PLAIN_DT_CAP)
            one32.copy_state_from(g, PLAIN_CFL, PLAIN_DT_CAP)
        g.step(1)
        traj64.step(1)
        traj32.step(1)
        k += 1
        if probe is not None:
            one64.step(1)
            one32.step(1)
            probe["one_step"] = {"step": k, "gpu": field_errors(g.readBuffer, one64.read, detail=True),
                                 "cpu_fp32": field_errors(one32.read, one64.read, detail=True),
                                 "cycles": {"gpu": g.info()["last_cycles"], "fp64_oracle": one64.info()["last_cycles"]}}
            one64.close()
            one32.close()
            probe = None
        if k <= steps and (k == 1 or k % every == 0):
            probe = {"step": k, "trajectory": {"gpu": field_errors(g.readBuffer, traj64.read),
                                               "cpu_fp32": field_errors(traj32.read, traj64.read)},
                     "one_step": None}
            reports.append(probe)
    g.close()
    return {"workload": workload, "steps": steps, "every": every, "reports": reports,
            "steps_note": f"{steps} of the workload's 2000 steps (bounded so the line finishes in minutes)",
            "metric": "|x - fp64 oracle| / max|fp64 oracle| per field (T; u = U and V faces; Y_F; Y_S)",
            "cpu_threads": threads, "seconds": time.perf_counter() - t0}


SERVE_CLASSES = ((96, 144), (128, 192), (192, 288), (256, 384), (512, 768))


def served_jobs(njobs: int, steps_lo: int, steps_hi: int, seed: int = 5):
    """One job set for every arrival rate: size class uniform over the classes, tepee scenes (scene kind 1),
    N uniform in [steps_lo, steps_hi]; `gap` holds unit-rate exponential inter-arrival gaps (divided by
    lambda for a rate), so every rate serves the same jobs in the same order."""
    import numpy as np
    rng = np.random.default_rng(seed)
    jobs = []
    for k in range(njobs):
        jobs.append({"size_class": int(rng.integers(0, len(SERVE_CLASSES))), "kind": 1, "seed": 9000 + k,
                     "nsteps": int(rng.integers(steps_lo, steps_hi + 1)), "gap": float(rng.exponential(1.0))})
    return jobs


def diff_sub(dx: float, dt: float) -> int:
    """Diffusion sub-steps for dt (js/fluid.js:190-198 with the default diffMult)."""
    import math
    tmax, rho_amb, t_amb = 2200.0, 101325 * 0.0289 / (8.314462 * 293.15), 293.15
    mu = 1.716e-5 * (tmax / 273.15) ** 1.5 * 383.55 / (tmax + 110.4)
    alpha = mu / 0.7 / (rho_amb * t_amb / tmax)
    n = math.ceil(dt / (dx * dx / (4.5 * alpha)))
    return max(1, min(5, n if n % 2 else n + 1))


def run_one_by_one(dev, jobs, tol: float):
    """Each job alone through the plain single-scene FluidSim (same scene, solver and step count as served):
    wall seconds from generating its scene to its fields read back, one job after the other."""
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    service = []
    for j in jobs:
        nx, ny = SERVE_CLASSES[j["size_class"]]
        t0 = time.perf_counter()
        sc = cb.generate_scene(j["kind"], nx, ny, 0.8, j["seed"])
        g = cb.FluidSim(dev.index, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
        load_scene(g, sc)
        g.set_solver(cb.SOLVE_FP64, 1, tol, 300)
        g.set_coarse_solve("pipelined")
        g.set_krylov(True)
        g.set_coarse_w(SERVE_W_CELLS)
        g.step(j["nsteps"])
        g.synchronize()
        cb.field_hash(g)
        service.append(time.perf_counter() - t0)
        g.close()
    return service


def run_served(dev, stream, lams, njobs: int, steps_lo: int, steps_hi: int, slots: int, budget: float, tol: float):
    """The serving loop (continuous batching, HBM-budget admission) at several arrival rates, against the same
    jobs run one by one through the plain single-scene step: each job's one-by-one service time is measured
    (scene set-up, steps, fields read back), and each rate's first-come-first-served schedule is built from
    those measured times and the rate's arrivals."""
    import numpy as np
    import campfire_b200 as cb
    jobs = served_jobs(njobs, steps_lo, steps_hi)
    service = run_one_by_one(dev, jobs, tol)
    srv = cb.Server(SERVE_CLASSES, [slots] * len(SERVE_CLASSES), budget, device=dev.index)
    srv.set_solver(cb.SOLVE_FP64, 1, tol, 300, "pipelined", krylov=2,   # the Krylov update folded (as the batch)
                   coarse_w=SERVE_W_CELLS)
    hbm, peak_kind = peaks()
    cells = sum(SERVE_CLASSES[j["size_class"]][0] * SERVE_CLASSES[j["size_class"]][1] * j["nsteps"] for j in jobs)
    out = []
    for lam in lams:
        t, run_jobs = 0.0, []
        for j in jobs:
            t += j["gap"] / lam
            run_jobs.append(dict(j, arrival_s=t))
        res, wall, cu = srv.run(run_jobs)
        lat = np.array([r["done_s"] - r["arrival_s"] for r in res])
        t_free, lat1 = 0.0, []
        for j, svc in zip(run_jobs, service):          # arrival order
            t_free = max(j["arrival_s"], t_free) + svc
            lat1.append(t_free - j["arrival_s"])
        lat1 = np.array(lat1)
        # algorithmic bytes: each job's cells x steps x bytes per cell-update at its last solve's cycle count
        byts = sum(SERVE_CLASSES[j["size_class"]][0] * SERVE_CLASSES[j["size_class"]][1] * j["nsteps"] *
                   bytes_per_cell(diff_sub(0.8 / SERVE_CLASSES[j["size_class"]][0], 2e-3), r["last_cycles"], True)
                   for j, r in zip(run_jobs, res))
        value = cu / wall
        one = cells / t_free
        out.append({"lambda_jobs_per_s": lam, "jobs": njobs, "value": value, "unit": METRIC,
                    "p50_latency_s": float(np.percentile(lat, 50)), "p99_latency_s": float(np.percentile(lat, 99)),
                    "wall_s": wall, "max_rel_residual": max(r["last_rel"] for r in res),
                    "roofline": {"achieved": byts / wall / 1e9, "peak": hbm, "unit": "GB/s",
                                 "frac": byts / wall / 1e9 / hbm, "peak_source": f"{peak_kind} hbm_gbs"},
                    "one_by_one": {"value": one, "unit": METRIC, "makespan_s": t_free,
                                   "p50_latency_s": float(np.percentile(lat1, 50)),
                                   "p99_latency_s": float(np.percentile(lat1, 99))},
                    "served_over_one_by_one": value / one})
    srv.close()
    return {"classes": [f"{a}x{b}" for a, b in SERVE_CLASSES], "slots_per_class": slots, "budget_bytes": budget,
            "jobs": njobs, "steps_per_job": [steps_lo, steps_hi], "job_steps_total": sum(j["nsteps"] for j in jobs),
            "scene": f"tepee (five logs of half 5 cm), FP64 defect correction to {tol:g}, pipelined direct coarsest, "
                     f"cycle {cycle_name(SERVE_W_CELLS)}",
            "one_by_one": "measured: each job alone through the plain FluidSim (scene set-up, steps, fields read "
                          "back), first come first served at each rate's arrivals",
            "one_by_one_service_s": float(sum(service)), "runs": out}


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
    ws.set_readback_lag(-1)   # readbacks through the ring, applied when they arrive (js/fluid.js:315-342)
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
    rbs = ws.readbacks()
    ws.close()
    sim.close()
    px = W * H
    return {"scene": f"the app's default fire ({npieces} moving pieces: 7 coals, 2 logs, 7 sticks), {nx}x{ny} "
                     f"cells, dt {dt}, one V-cycle per step", "frame_sim_dt_s": frame_dt, "frames": frames,
            "readback": "asynchronous ring, applied when arrived", "readbacks": rbs,
            "warmup_frames": warmup, "image": [W, H], "frames_per_s": frames / wall,
            "ms_per_frame": 1e3 * wall / frames, "gas_steps_per_frame": steps / frames,
            "sim_time_per_wall_time": steps * dt / wall,
            "render_ms": float(np.median(render_ms)), "render_mpixel_per_s": px / (np.median(render_ms) / 1e3) / 1e6,
            "last_frame_stats": {"hrr_w_per_m": st["hrr"], "rad_w_per_m": st["rad"], "tmax_k": st["tmax"]}}


def run_e2e(sim, sc, stream, flush, steps: int, barrier, dev, world: int, ckpt=None) -> dict:
    """Wall-clock steps through the C ABI with the host-side inputs and outputs of the app's frame (see main).
    ckpt: the state measure_gpu saved two warm-up steps before its timed steps; it is loaded and the two steps are
    taken the same way untimed, so that the timed steps are the device-timed ones."""
    import torch
    import torch.distributed as dist
    import campfire_b200 as cb
    L = cb.lib()
    pin_pieces = torch.from_numpy(sc["pieces"].copy()).pin_memory()
    acc = torch.zeros(528, dtype=torch.int32).pin_memory()
    rad = torch.zeros(320 * 4, dtype=torch.float32).pin_memory()
    fw = torch.zeros(256, dtype=torch.int32).pin_memory()
    fptr = ctypes.cast(pin_pieces.data_ptr(), ctypes.POINTER(ctypes.c_float))
    i32 = ctypes.POINTER(ctypes.c_int32)
    accp, radp, fwp = (ctypes.cast(acc.data_ptr(), i32), ctypes.cast(rad.data_ptr(), ctypes.POINTER(ctypes.c_float)),
                       ctypes.cast(fw.data_ptr(), i32))
    tag, ready, slot = ctypes.c_uint64(), ctypes.c_int(), ctypes.c_int()
    if ckpt:
        sim.load_checkpoint(ckpt)
        for k in range(2):
            flush.fill_(float(k))
            cb._lib.check(L.cfg_upload_pieces(sim._h, fptr, sc["npieces"]))
            cb._lib.check(L.cfg_write_params(sim._h))
            cb._lib.check(L.cfg_step(sim._h, 1))
            cb._lib.check(L.cfg_readback_begin(sim._h, k, ctypes.byref(slot)))
            cb._lib.check(L.cfg_readback_wait(sim._h, accp, radp, fwp, ctypes.byref(tag)))
    collected, skipped, lag = 0, 0, []
    # the L2 flush's device time, measured apart (so that the timed loop carries no extra events)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    f0.record(stream)
    for k in range(steps):
        flush.fill_(float(k))
    f1.record(stream)
    torch.cuda.synchronize(dev)
    flush_ms = f0.elapsed_time(f1) / steps

    def collect(k, wait):
        nonlocal collected
        while True:
            if wait:
                rc = L.cfg_readback_wait(sim._h, accp, radp, fwp, ctypes.byref(tag))
                if rc == -2:
                    return
                cb._lib.check(rc)
            else:
                cb._lib.check(L.cfg_readback_poll(sim._h, accp, radp, fwp, ctypes.byref(tag), ctypes.byref(ready)))
                if not ready.value:
                    return
            collected += 1
            lag.append(k - tag.value)

    barrier()
    t0 = time.perf_counter()
    for k in range(steps):
        flush.fill_(float(k))
        cb._lib.check(L.cfg_upload_pieces(sim._h, fptr, sc["npieces"]))
        cb._lib.check(L.cfg_write_params(sim._h))
        cb._lib.check(L.cfg_step(sim._h, 1))
        rc = L.cfg_readback_begin(sim._h, k, ctypes.byref(slot))
        if rc == -16:   # three readbacks in flight: every step's result is read, so wait for the oldest
            skipped += 1
            rc = L.cfg_readback_wait(sim._h, accp, radp, fwp, ctypes.byref(tag))
            cb._lib.check(rc)
            collected += 1
            lag.append(k - tag.value)
            rc = L.cfg_readback_begin(sim._h, k, ctypes.byref(slot))
        cb._lib.check(rc)
        collect(k, False)
    collect(steps, True)
    wall = time.perf_counter() - t0
    torch.cuda.synchronize(dev)
    flush_s = steps * flush_ms / 1e3
    t = torch.tensor([wall - flush_s], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return {"steps": steps, "seconds": float(t.item()), "wall_s": wall, "flush_s": flush_s,
            "collected": collected, "waited_on_full_ring": skipped,
            "lag_steps": {"max": max(lag) if lag else None, "mean": sum(lag) / len(lag) if lag else None}}


def measure_gpu(dev, stream, flush, workload: str, steps: int, warmup: int, launch: str, coarse_cells: int,
                world: int, rank: int, barrier, clocks=None, w_cells=None, ckpt=None) -> dict:
    """The plain single-scene step of `workload` on this rank's GPU: `steps` steps timed one by one with CUDA
    events on the library's stream after an L2 flush each; value = all ranks' cell-updates / max-over-ranks time.
    ckpt: a file that receives the scene's state two warm-up steps before the timed steps (cfg_checkpoint_save),
    so that the end-to-end measurement can take the same steps."""
    import torch
    import torch.distributed as dist
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[workload]
    sc = cb.generate_scene(kind, nx, ny, 0.8, seed + 1000 * rank)
    sim = cb.FluidSim(dev.index, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(sim, sc)
    configure_solver(sim, workload, w_cells)
    # smoother schedule picked by the autotuner (fused V-cycles timed on a scratch scene of this size)
    if coarse_cells > 0:
        sim.set_coarse_cells(coarse_cells)
        schedule = {"coarse_cells": coarse_cells, "autotune": "skipped"}
    else:
        tune = cb.autotune([(nx, ny)], iters=20, device=dev.index, coarse_direct=True)
        sim.set_coarse_cells(tune["best"])
        schedule = {"coarse_cells": tune["best"],
                    "autotune_ms_per_cycle": {str(k): round(v, 5) for k, v in tune["ms_per_cycle"].items()}}
    # tile shapes of the advection, diffusion + sources and forces kernels (same bits for every shape)
    tt = cb.autotune_tiles([(nx, ny)], iters=20, device=dev.index)
    sim.set_tiles(*tt["best"])
    schedule["tiles"] = {"advect": cb.TILE_SHAPES[tt["best"][0]], "diffuse_sources": cb.TILE_SHAPES[tt["best"][1]],
                         "forces": cb.TILE_SHAPES[tt["best"][2]],
                         "autotune_ms": {k: [round(x, 5) for x in v] for k, v in tt["ms"].items()}}
    sim.set_stream(stream.cuda_stream)
    sim.set_graphs(launch == "graph")
    if ckpt:
        sim.step(warmup - 2)
        sim.synchronize()
        sim.save_checkpoint(ckpt)
        sim.step(2)
    else:
        sim.step(warmup)
    sim.synchronize()
    barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    if clocks:
        clocks.start()
    for k in range(steps):
        flush.fill_(float(k))
        ev[k][0].record(stream)
        sim.step(1)
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    barrier()
    clk = clocks.stop() if clocks else None
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    info = sim.info()
    sim.synchronize()
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    return {"sim": sim, "scene": sc, "value": world * nx * ny * steps / (ms_max / 1e3), "ms_max": ms_max,
            "info": info, "launches": sim.launch_count(), "schedule": schedule, "clocks": clk}


def kernel_roofline(sim, workload: str, value_per_gpu: float, info: dict) -> dict:
    """The dominant kernel's achieved HBM bandwidth (algorithmic bytes per launch / CUDA-event time of back-to-back
    launches on the library's stream) and the whole step's (algorithmic bytes per cell-update x cell-updates/s)."""
    import campfire_b200 as cb
    L = cb.lib()
    hbm, peak_kind = peaks()
    kern = {}
    for name in ("advect", "diffuse_sources", "forces", "mg_down0_krylov", "mg_up0_krylov", "mg_down0", "mg_up0",
                 "mg_coarse", "pcg_decide", "pcg_step", "defect64", "project"):
        m, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        rc = L.cfg_time_kernel(sim._h, name.encode(), 50, ctypes.byref(m), ctypes.byref(b), ctypes.byref(n))
        if rc == -2:   # a variant this engine does not run (the folded Krylov kernels, or the plain ones)
            continue
        cb._lib.check(rc)
        if name in ("mg_down0", "mg_up0") and name + "_krylov" in kern:
            continue       # the step runs the folded variants: the plain ones are not on its path
        kern[name] = {"ms": m.value, "bytes": b.value, "per_step": n.value, "share_ms": m.value * n.value}
    dom = max(kern, key=lambda k: kern[k]["share_ms"])
    dk = kern[dom]
    achieved = dk["bytes"] / (dk["ms"] / 1e3) / 1e9
    bpc = bytes_per_cell(info["diffSub"], info["last_cycles"], True)
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_source": f"{peak_kind} hbm_gbs (copy bandwidth)",
            "traffic": NCU_TRAFFIC.get((workload, dom)), "traffic_source": "ncu dram__bytes_read.sum + "
            "dram__bytes_write.sum per launch, one capture of this workload",
            "bytes_per_launch": dk["bytes"], "launch_ms": dk["ms"],
            "step_bytes_per_cell": bpc, "step_achieved_gbs": value_per_gpu * bpc / 1e9,
            "step_frac": value_per_gpu * bpc / 1e9 / hbm,
            "kernels": {k: {"ms": round(v["ms"], 5), "per_step": v["per_step"]} for k, v in kern.items()}}


def profile_batch(warm: int, coarse_cells: int, krylov: int) -> None:
    """The batched workload (the 64 scenes of run_batched, FP64 to 1e-10, pipelined coarsest inverse) launched
    kernel by kernel with a fixed schedule: `warm` steps, then one more."""
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    scenes = batch_scenes()
    b = cb.Batch([(s["nx"], s["ny"]) for s in scenes], 0.8, [s["dt"] for s in scenes])
    for v, s in zip(b.scenes, scenes):
        load_scene(v, s)
    b.set_solver(cb.SOLVE_FP64, 1, 1e-10, 300)
    b.set_coarse_solve("pipelined")
    b.set_coarse_cells(coarse_cells)
    b.set_krylov(krylov)
    b.set_graphs(False)
    b.step(warm)
    b.synchronize()
    b.step(1)
    b.synchronize()
    print(json.dumps({"workload": "batched", "profile_steps": warm + 1, "coarse_cells": coarse_cells,
                      "krylov_folded": b.krylov_folded(),
                      "cycles_last_step": max(v.info()["last_cycles"] for v in b.scenes)}))
    b.close()


def profile_steps(workload: str, warm: int, w_cells) -> None:
    """The workload's scene and solver launched kernel by kernel: `warm` steps, then one more, synchronised
    between (a profiler's capture selects launches of the last step by skipping the earlier ones)."""
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[workload]
    sc = cb.generate_scene(kind, nx, ny, 0.8, seed)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    configure_solver(g, workload, w_cells)
    g.set_coarse_cells(1536)
    g.set_graphs(False)
    g.step(warm)
    g.synchronize()
    g.step(1)
    g.synchronize()
    print(json.dumps({"workload": workload, "profile_steps": warm + 1, "cycles_last_step": g.info()["last_cycles"]}))
    g.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain", choices=sorted(WORKLOADS))
    ap.add_argument("--cpu-sample", type=int, default=3, help="steps of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fine-steps", type=int, default=20,
                    help="timed steps of the 512x768 tepee workload (FP64 to 1e-10) added to the line as `fine` "
                         "(0: skip; ignored with --workload fine)")
    ap.add_argument("--batched-steps", type=int, default=500,
                    help="timed steps of the 64-scene batched measurement added to the line (0: skip)")
    ap.add_argument("--served-jobs", type=int, default=24,
                    help="jobs of the serving measurement (the same jobs at every arrival rate; 0: skip)")
    ap.add_argument("--served-steps", type=int, nargs=2, default=(100, 2000), metavar=("LO", "HI"),
                    help="steps per served job, uniform in [LO, HI]")
    ap.add_argument("--served-rates", type=float, nargs="+", default=(10.0, 100.0, 1000.0))
    ap.add_argument("--app-frames", type=int, default=120,
                    help="timed frames of the app frame measurement (wood coupling + gas steps + render) "
                         "added to the line (0: skip)")
    ap.add_argument("--fp64-error-every", type=int, default=100,
                    help="report the field errors against the FP64 oracle every this many steps (0: skip)")
    ap.add_argument("--fp64-error-steps", type=int, default=200,
                    help="steps of the FP64-oracle comparison (the workload defines 2000)")
    ap.add_argument("--fp64-error-workload", default="fine", choices=sorted(WORKLOADS))
    ap.add_argument("--coarse-cells", type=int, default=0,
                    help="start the coarse block at the first level with at most this many cells instead of "
                         "autotuning (0: autotune); for profiling runs whose launch indices must not depend on "
                         "the autotuner")
    ap.add_argument("--launch", default="graph", choices=["graph", "stream"],
                    help="graph: one CUDA graph per step (pressure loop as a device-side WHILE node); "
                         "stream: kernel by kernel, the host polling the loop decision (for profilers that "
                         "do not list kernels inside conditional graph nodes)")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="profiling driver: step the workload's scene this many times, then once more, kernel by "
                         "kernel (stream launches, coarse block from 1536 cells, no autotuning), print its cycle "
                         "count and exit without a benchmark line (for ncu's launch lists and captures)")
    ap.add_argument("--profile-batch", action="store_true",
                    help="with --profile-steps: the batched workload (coarse block from 6144 cells, the Krylov "
                         "update folded, as the benchmark's batch keeps it in its runs) instead of --workload")
    ap.add_argument("--w-cells", type=int, default=None,
                    help="override the main workload's cycle shape (cfg_set_coarse_w; 0: the V-cycle) in both "
                         "arms, the profiling driver included")
    a = ap.parse_args()
    a.warmup = max(a.warmup, 3)
    if a.profile_steps > 0:
        if a.profile_batch:
            profile_batch(a.profile_steps, 6144, 2)
        else:
            profile_steps(a.workload, a.profile_steps, a.w_cells)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(a.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nx, ny, kind, seed, mode, tol, maxc = WORKLOADS[a.workload]
    config = workload_config(a.workload, world, a.w_cells)

    if a.impl == "reference":
        # the CPU restatement of the reference step on this box's host cores: oracle library only
        if rank != 0:
            return
        th = cpu_threads()
        val, secs, cyc = run_cpu(a.workload, a.steps, a.warmup, th, a.w_cells)
        line = {"metric": METRIC, "value": val, "unit": METRIC, "impl": "reference", "n_gpus": a.gpus,
                "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * secs / a.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
                "solve": {"cycles_per_step": cyc, "arithmetic": "f32 (FP64 outer loop), host cores"},
                "cpu_baseline": {"value": val, "unit": METRIC, "cores": th, "kind": "port",
                                 "sample": f"{a.steps} steps of the {nx}x{ny} workload after {a.warmup} warm-up steps "
                                           "(C++ restatement of the reference WGSL, f32, OpenMP, same solver)"},
                "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist
    import campfire_b200 as cb

    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # one non-default stream shared by the library, the L2 flush and the timing events
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    import tempfile
    fd, ckpt = tempfile.mkstemp(prefix="campfire_bench_", suffix=".ckpt")
    os.close(fd)
    m = measure_gpu(dev, stream, flush, a.workload, a.steps, a.warmup, a.launch, a.coarse_cells, world, rank,
                    barrier, ClockSampler(local), w_cells=a.w_cells, ckpt=ckpt)
    sim, sc, value, ms_max, info = m["sim"], m["scene"], m["value"], m["ms_max"], m["info"]

    # ---- end to end through the C ABI, the app's frame data flow (js/main.js:266-283): per step the piece
    # buffer from pinned host memory and the parameter block go up, the step runs, and the step's
    # accumulators, radiation output and face weights come back through the asynchronous readback ring
    # (cfg_readback_begin / cfg_readback_poll, js/fluid.js:315-342), collected as they arrive; every step's
    # readback is taken: when the ring's three slots are in flight the host waits for the oldest (at most
    # three steps queued ahead of the GPU). The timed region ends when the last readback has been collected.
    # The L2 flush before each step (as in the device-timed loop) sits on the same stream; its device time,
    # measured with CUDA events over the same number of flushes just before, is taken out of the wall time.
    # The timed steps are the device-timed ones: the scene resumes from the state saved before them.
    e2e = run_e2e(sim, sc, stream, flush, a.steps, barrier, dev, world, ckpt=ckpt)
    os.unlink(ckpt)
    e2e_value = world * nx * ny * e2e["steps"] / e2e["seconds"]

    # ---- roofline of the dominant kernel, measured after the timed region
    roof = kernel_roofline(sim, a.workload, value / world, info)
    sim.close()

    # ---- the 512x768 tepee workload (FP64 to 1e-10): the plain step where the roofline target is set
    fine = None
    if a.fine_steps > 0 and a.workload != "fine":
        mf = measure_gpu(dev, stream, flush, "fine", a.fine_steps, a.warmup, a.launch, 0, world, rank, barrier,
                         ClockSampler(local))
        fi = mf["info"]
        fine = {"value": mf["value"], "unit": METRIC, "steps": a.fine_steps, "ms_per_step": mf["ms_max"] / a.fine_steps,
                "config": workload_config("fine", world), "schedule": mf["schedule"],
                "solve": {"cycles_last_step": fi["last_cycles"], "diff_sub": fi["diffSub"], "levels": fi["levels"],
                          "last_rel": fi["last_rel"]},
                "roofline": kernel_roofline(mf["sim"], "fine", mf["value"] / world, fi), "clocks": mf["clocks"]}
        mf["sim"].close()
        # the same workload with the V(2,2) cycle throughout (the cycle shape's effect)
        mv = measure_gpu(dev, stream, flush, "fine", a.fine_steps, a.warmup, a.launch, 0, world, rank, barrier,
                         w_cells=0)
        fine["v_cycle"] = {"value": mv["value"], "unit": METRIC, "ms_per_step": mv["ms_max"] / a.fine_steps,
                           "cycle": cycle_name(0), "cycles_last_step": mv["info"]["last_cycles"],
                           "last_rel": mv["info"]["last_rel"]}
        mv["sim"].close()

    batched = None
    if a.batched_steps > 0:
        batched = run_batched(dev, stream, flush, a.batched_steps, 3, 1e-10, 300, 10)

    fp64_error = None
    if a.fp64_error_every > 0 and rank == 0:
        fp64_error = run_fp64_error(dev, a.fp64_error_workload, a.fp64_error_steps, a.fp64_error_every, cpu_threads())

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
        val, secs, cyc = run_cpu(a.workload, a.cpu_sample, 1, th, a.w_cells)
        cpu = {"value": val, "unit": METRIC, "cores": th, "kind": "port",
               "sample": f"{a.cpu_sample} steps of the same {nx}x{ny} workload after 1 warm-up step "
                         f"(C++ restatement of the reference WGSL, f32, OpenMP, same solver: "
                         f"{cyc:.1f} V-cycles/step)"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": a.steps,
                "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
                "launch": a.launch, "schedule": m["schedule"],
                "solve": {"cycles_last_step": info["last_cycles"], "diff_sub": info["diffSub"],
                          "levels": info["levels"], "last_rel": info["last_rel"]},
                # H2D: the piece buffer and the descriptor's parameter block (uniform + step controls, 204 B), each
                # the parameter of a one-CTA kernel (dx and alpha of the diffusion rule go up only when they change);
                # D2H: acc + rad + faceW of every collected readback
                "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 64 * 20 * 4 + 204,
                        "d2h_bytes_per_step": (528 * 4 + 320 * 16 + 256 * 4) * e2e["collected"] / e2e["steps"],
                        "steps": e2e["steps"], "steps_timed": "the device-timed steps, resumed from a checkpoint",
                        "readback": "asynchronous ring of three pinned slots (js/fluid.js:315-342)",
                        "readbacks": {k: e2e[k] for k in ("collected", "waited_on_full_ring", "lag_steps")},
                        "wall_s": e2e["wall_s"], "l2_flush_s_removed": e2e["flush_s"]},
                "gpu_launches": m["launches"] * a.steps, "roofline": roof, "cpu_baseline": cpu, "clocks": m["clocks"],
                "fine": fine, "batched": batched, "served": served, "app_frame": app, "fp64_oracle_error": fp64_error}
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
