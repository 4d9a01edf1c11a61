"""FluidSim: the reference's gas-solver host interface over the B200 C ABI.

Mirrors `class FluidSim` of js/fluid.js:26-356 (names, argument meaning and
error behaviour) so a caller of the reference finds the same surface:

    sim = FluidSim(device=0, mode={"nx": 224, "ny": 320, "dt": 0.003})
    sim.init()                      # allocates; raises on 'coarsest level too large'
    sim.setParam("heaterT", 1200)   # applied by the next writeParams()
    sim.writeParams()
    sim.uploadPieces(pieces, n)     # Float32Array(64*20) packing of js/main.js:196-199
    sim.clearGeometry(); sim.encodeGeometry()
    for _ in range(n): sim.encodeStep()
    sim.encodeRadiation()
    out = sim.readback()            # {acc, rad, faceW}, then acc is cleared
    T = sim.readBuffer("T")

WebGPU's encoder/pass arguments have no counterpart: each call enqueues CUDA
work on the handle's stream in call order. Extensions beyond the reference
(solver modes, CFL step, FP64 budgets, batches) are snake_case methods.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

from . import _lib
from ._lib import CampfireError, CfgInfo, CfgParams, check

SCENE_WIDTH = 0.7   # js/config.js:3
STAGES = ("advect", "diffuse", "sources", "forces", "coef/rhs", "vcycle", "project")


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _coarse_mode(direct) -> int:
    if direct == "pipelined" or (not isinstance(direct, bool) and direct == 2):
        return 2
    return 1 if direct else 0


class _SceneOps:
    """Per-scene FluidSim surface shared by FluidSim and batch scene views."""

    _h: Optional[int]
    _cfl = 0.0

    # FluidSim.time (js/fluid.js:252): advanced by dt per step on the host; with a CFL step the
    # device owns dt and the clock, so it is read from the device (cfg_get_info)
    @property
    def time(self) -> float:
        if self._cfl > 0 and getattr(self, "_h", None):
            return self.info()["time"]
        return self.__dict__.get("_time", 0.0)

    @time.setter
    def time(self, v: float):
        self.__dict__["_time"] = float(v)

    # -- FluidSim methods
    def reset(self):
        check(_lib.lib().cfg_reset(self._h))
        self.time = 0.0

    def setParam(self, k: str, v: float):
        check(_lib.lib().cfg_set_param(self._h, k.encode(), float(v)))

    def getParam(self, k: str) -> float:
        v = ctypes.c_double()
        check(_lib.lib().cfg_get_param(self._h, k.encode(), ctypes.byref(v)))
        return v.value

    @property
    def params(self) -> dict:
        return {n: self.getParam(n) for n, _ in _lib.PARAM_FIELDS}

    def writeParams(self):
        check(_lib.lib().cfg_write_params(self._h))

    def uploadPieces(self, data, n: int):
        a = np.zeros(_lib.MAX_PIECES * _lib.PIECE_FLOATS, np.float32)
        d = np.asarray(data, np.float32).ravel()
        a[: min(d.size, a.size)] = d[: a.size]
        check(_lib.lib().cfg_upload_pieces(self._h, _fp(a), int(n)))

    def clearGeometry(self, encoder=None):
        check(_lib.lib().cfg_clear_geometry(self._h))

    def encodeGeometry(self, pass_=None):
        check(_lib.lib().cfg_geometry(self._h))

    def encodeRadiation(self, pass_=None):
        check(_lib.lib().cfg_radiation(self._h))

    def readback(self) -> dict:
        """encodeReadback + afterSubmit: {acc: int32[528], rad: float32[320*4], faceW: int32[256]}."""
        acc = np.zeros(_lib.ACC_LEN, np.int32)
        rad = np.zeros(_lib.RAD_LEN * 4, np.float32)
        fw = np.zeros(_lib.MAX_PIECES * 4, np.int32)
        i32p = ctypes.POINTER(ctypes.c_int32)
        check(_lib.lib().cfg_readback(self._h, acc.ctypes.data_as(i32p), _fp(rad), fw.ctypes.data_as(i32p)))
        return {"acc": acc, "rad": rad, "faceW": fw}

    def encodeReadback(self, tag: int = 0):
        """encodeReadback + afterSubmit, asynchronous (cfg_readback_begin): the ring slot used, or None when
        the next slot is still pending (the frame's readback is skipped and acc keeps accumulating)."""
        slot = ctypes.c_int(-1)
        rc = _lib.lib().cfg_readback_begin(self._h, tag, ctypes.byref(slot))
        if rc == -16:
            return None
        check(rc)
        return slot.value

    def pollReadback(self, wait: bool = False):
        """The oldest pending readback once its copies are done: (data, tag), data as readback() gives it;
        None if nothing is ready (wait=True blocks for the oldest pending one)."""
        acc = np.zeros(_lib.ACC_LEN, np.int32)
        rad = np.zeros(_lib.RAD_LEN * 4, np.float32)
        fw = np.zeros(_lib.MAX_PIECES * 4, np.int32)
        i32p = ctypes.POINTER(ctypes.c_int32)
        tag = ctypes.c_uint64()
        L = _lib.lib()
        if wait:
            rc = L.cfg_readback_wait(self._h, acc.ctypes.data_as(i32p), _fp(rad), fw.ctypes.data_as(i32p),
                                     ctypes.byref(tag))
            if rc == -2:
                return None
            check(rc)
        else:
            ready = ctypes.c_int()
            check(L.cfg_readback_poll(self._h, acc.ctypes.data_as(i32p), _fp(rad), fw.ctypes.data_as(i32p),
                                      ctypes.byref(tag), ctypes.byref(ready)))
            if not ready.value:
                return None
        return {"acc": acc, "rad": rad, "faceW": fw}, tag.value

    def field_size(self, name: str) -> int:
        n = ctypes.c_size_t()
        check(_lib.lib().cfg_field_size(self._h, name.encode(), ctypes.byref(n)))
        return n.value

    def readBuffer(self, name: str) -> np.ndarray:
        """Float32 copy of a field in the reference's dense layout (js/fluid.js:345-355)."""
        n = self.field_size(name)
        out = np.empty(n, np.float32)
        check(_lib.lib().cfg_read_field(self._h, name.encode(), _fp(out), n))
        return out

    def writeBuffer(self, name: str, data) -> None:
        a = np.ascontiguousarray(np.asarray(data, np.float32).ravel())
        check(_lib.lib().cfg_write_field(self._h, name.encode(), _fp(a), a.size))

    def read_p64(self) -> np.ndarray:
        out = np.empty(self.nx * self.ny, np.float64)
        check(_lib.lib().cfg_read_p64(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size))
        return out

    def info(self) -> dict:
        i = CfgInfo()
        check(_lib.lib().cfg_get_info(self._h, ctypes.byref(i)))
        return {"nx": i.nx, "ny": i.ny, "levels": i.levels, "diffSub": i.diff_sub, "dx": i.dx, "dt": i.dt,
                "height": i.height, "time": i.time, "frame": i.frame, "last_cycles": i.last_cycles,
                "last_rel": i.last_rel,
                "level_dims": [(i.level_nx[l], i.level_ny[l]) for l in range(i.levels)]}

    @property
    def diffSub(self) -> int:
        return self.info()["diffSub"]

    @property
    def levels(self) -> list:
        return [{"nx": a, "ny": b} for a, b in self.info()["level_dims"]]

    def setFrame(self, f: int):
        self.frame = int(f)
        check(_lib.lib().cfg_set_frame(self._h, int(f)))

    # -- extensions
    def set_dt(self, dt: float):
        check(_lib.lib().cfg_set_dt(self._h, float(dt)))
        self.dt = float(dt)

    def set_cfl(self, cfl: float, dt_cap: float):
        t = self.time   # the clock so far (the device's while a CFL step was on)
        check(_lib.lib().cfg_set_cfl(self._h, float(cfl), float(dt_cap)))
        self._cfl = float(cfl)
        if cfl <= 0:
            self.time = t

    def set_nray(self, n: int):
        check(_lib.lib().cfg_set_nray(self._h, int(n)))

    def pressure_residual(self) -> float:
        v = ctypes.c_double()
        check(_lib.lib().cfg_pressure_residual(self._h, ctypes.byref(v)))
        return v.value

    def save_checkpoint(self, path: str):
        """The scene's state to a file (cfg_checkpoint_save)."""
        check(_lib.lib().cfg_checkpoint_save(self._h, os.fsencode(path)))

    def load_checkpoint(self, path: str):
        """Resume from a checkpoint of a scene of the same grid size (cfg_checkpoint_load)."""
        check(_lib.lib().cfg_checkpoint_load(self._h, os.fsencode(path)))
        inf = self.info()
        self.time, self.frame = inf["time"], inf["frame"]

    def budgets(self) -> np.ndarray:
        o = np.zeros(8, np.float64)
        check(_lib.lib().cfg_budgets(self._h, o.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return o


class FluidSim(_SceneOps):
    """new FluidSim(device, mode) + init() (js/fluid.js:27-160) on a CUDA device."""

    def __init__(self, device: int = 0, mode: Optional[dict] = None, width: float = SCENE_WIDTH, **kw):
        mode = dict(mode or {}, **kw)
        self.device, self.nx, self.ny, self.dt = device, int(mode["nx"]), int(mode["ny"]), float(mode["dt"])
        self.dx = width / self.nx
        self.height = self.dx * self.ny
        self.width = width
        self.time = 0.0
        self.frame = 0
        self._h = None

    def init(self):
        h = ctypes.c_void_p()
        check(_lib.lib().cfg_create(self.nx, self.ny, self.width, self.dt, self.device, ctypes.byref(h)))
        self._h = h.value
        return self

    def close(self):
        if self._h:
            _lib.lib().cfg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def encodeStep(self, pass_=None, n: int = 1):
        """One gas step (js/fluid.js:225-253); time += dt."""
        check(_lib.lib().cfg_step(self._h, int(n)))
        if self._cfl <= 0:
            self.time += n * self.dt

    def step(self, n: int = 1):
        self.encodeStep(n=n)

    def encodeStepProfiled(self) -> dict:
        """One step with per-stage device ms, names of js/fluid.js:291."""
        ms = np.zeros(7, np.float32)
        check(_lib.lib().cfg_step_profiled(self._h, _fp(ms)))
        if self._cfl <= 0:
            self.time += self.dt
        return dict(zip(STAGES, ms.tolist()))

    def vcycle(self, pass_=None, nu: int = 2):
        check(_lib.lib().cfg_vcycle(self._h, int(nu)))

    def run_stage(self, name: str):
        check(_lib.lib().cfg_run_stage(self._h, name.encode()))

    def set_coarse_cells(self, cells: int):
        """Smoother schedule: the one-CTA coarse block starts at the first level with <= cells cells."""
        check(_lib.lib().cfg_set_coarse_cells(self._h, int(cells)))

    def set_coarse_cluster(self, cs: int):
        """The coarse phase on one CTA (0) or on a cluster of cs CTAs (2, 4, 8, 16); bit-identical."""
        check(_lib.lib().cfg_set_coarse_cluster(self._h, int(cs)))

    def set_coarse_w(self, cells: int):
        """Cycle shape: the W tail (the level two above the coarsest, if it has <= cells cells, visits the
        next level twice per cycle); 0: the V-cycle."""
        check(_lib.lib().cfg_set_coarse_w(self._h, int(cells)))

    def set_coarse_solve(self, direct):
        """TOL/FP64 modes: the coarsest level by its inverse (True), by 120 sweeps (False), or by the
        inverse factored beside the previous step's solve ("pipelined")."""
        check(_lib.lib().cfg_set_coarse_solve(self._h, _coarse_mode(direct)))

    def set_krylov(self, on):
        """FP64 mode: preconditioned CG around the V-cycle (True) or plain defect correction (False);
        2 / 3: CG with its update folded into the level-0 kernels / as its own kernel."""
        check(_lib.lib().cfg_set_krylov(self._h, int(on)))

    def krylov_folded(self) -> bool:
        """Whether the pressure loop folds the Krylov update into the level-0 kernels."""
        f = ctypes.c_int()
        check(_lib.lib().cfg_krylov_folded(self._h, ctypes.byref(f)))
        return bool(f.value)

    def set_tiles(self, advect: int, diffuse_sources: int, forces: int):
        """Tile shapes (TILE_SHAPES indices) of the advection, diffusion + sources and forces kernels."""
        check(_lib.lib().cfg_set_tiles(self._h, advect, diffuse_sources, forces))

    def set_solver(self, mode: int = _lib.SOLVE_FIXED, ncycles: int = 1, tol: float = 1e-6, max_cycles: int = 50):
        check(_lib.lib().cfg_set_solver(self._h, mode, ncycles, tol, max_cycles))

    def set_stream(self, stream_ptr: int):
        check(_lib.lib().cfg_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def synchronize(self):
        check(_lib.lib().cfg_synchronize(self._h))

    def set_graphs(self, on: bool):
        check(_lib.lib().cfg_set_graphs(self._h, 1 if on else 0))

    def launch_count(self) -> int:
        n = ctypes.c_int()
        check(_lib.lib().cfg_launch_count(self._h, ctypes.byref(n)))
        return n.value


class _SceneView(_SceneOps):
    def __init__(self, h, nx, ny, width):
        self._h, self.nx, self.ny, self.width = h, nx, ny, width
        self.dx = width / nx
        self.time, self.frame = 0.0, 0


class Batch:
    """Many independent scenes of uneven size stepped together (one launch per kernel for all)."""

    def __init__(self, dims, width=0.8, dts=None, device: int = 0):
        n = len(dims)
        nx = (ctypes.c_int * n)(*[d[0] for d in dims])
        ny = (ctypes.c_int * n)(*[d[1] for d in dims])
        widths = [width] * n if np.isscalar(width) else list(width)
        dts = dts or [0.002] * n
        wa = (ctypes.c_double * n)(*widths)
        da = (ctypes.c_double * n)(*dts)
        h = ctypes.c_void_p()
        check(_lib.lib().cfg_batch_create(n, nx, ny, wa, da, device, ctypes.byref(h)))
        self._h = h.value
        self.scenes = []
        for i in range(n):
            v = ctypes.c_void_p()
            check(_lib.lib().cfg_batch_scene(self._h, i, ctypes.byref(v)))
            self.scenes.append(_SceneView(v.value, dims[i][0], dims[i][1], widths[i]))

    def close(self):
        if self._h:
            _lib.lib().cfg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        check(_lib.lib().cfg_batch_step(self._h, int(n)))

    def set_solver(self, mode=_lib.SOLVE_FIXED, ncycles=1, tol=1e-6, max_cycles=50):
        check(_lib.lib().cfg_batch_set_solver(self._h, mode, ncycles, tol, max_cycles))

    def set_coarse_cells(self, cells: int):
        check(_lib.lib().cfg_batch_set_coarse_cells(self._h, int(cells)))

    def set_coarse_solve(self, direct):
        check(_lib.lib().cfg_batch_set_coarse_solve(self._h, _coarse_mode(direct)))

    def set_coarse_cluster(self, cs: int):
        check(_lib.lib().cfg_batch_set_coarse_cluster(self._h, int(cs)))

    def set_coarse_w(self, cells: int):
        check(_lib.lib().cfg_batch_set_coarse_w(self._h, int(cells)))

    def set_krylov(self, on):
        """True / 1: on (the update kernel for a batch); 2: on, update folded into the level-0 kernels;
        3: on, separate update kernel; False / 0: plain defect correction."""
        check(_lib.lib().cfg_batch_set_krylov(self._h, int(on)))

    def krylov_folded(self) -> bool:
        f = ctypes.c_int()
        check(_lib.lib().cfg_batch_krylov_folded(self._h, ctypes.byref(f)))
        return bool(f.value)

    def set_tiles(self, advect: int, diffuse_sources: int, forces: int):
        check(_lib.lib().cfg_batch_set_tiles(self._h, advect, diffuse_sources, forces))

    def set_graphs(self, on: bool):
        check(_lib.lib().cfg_batch_set_graphs(self._h, 1 if on else 0))

    def set_active(self, i: int, on: bool):
        check(_lib.lib().cfg_batch_set_active(self._h, i, 1 if on else 0))

    def set_stream(self, stream_ptr: int):
        check(_lib.lib().cfg_batch_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def synchronize(self):
        check(_lib.lib().cfg_batch_synchronize(self._h))

    def launch_count(self) -> int:
        n = ctypes.c_int()
        check(_lib.lib().cfg_batch_launch_count(self._h, ctypes.byref(n)))
        return n.value

    def write_params(self):
        check(_lib.lib().cfg_batch_write_params(self._h))

    def geometry(self):
        check(_lib.lib().cfg_batch_geometry(self._h))


class Server:
    """Continuous-batching server of gas-step jobs (cfg_server_*): resident slots per size
    class, admission by an HBM budget, one batched step per loop iteration."""

    def __init__(self, classes, slots, budget_bytes: float, device: int = 0, width: float = 0.8):
        n = len(classes)
        nx = (ctypes.c_int * n)(*[c[0] for c in classes])
        ny = (ctypes.c_int * n)(*[c[1] for c in classes])
        sl = (ctypes.c_int * n)(*slots)
        h = ctypes.c_void_p()
        check(_lib.lib().cfg_server_create(device, n, nx, ny, sl, float(budget_bytes), width, ctypes.byref(h)))
        self._h = h.value
        self.classes = list(classes)

    def close(self):
        if self._h:
            _lib.lib().cfg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_solver(self, mode=_lib.SOLVE_FP64, ncycles=1, tol=1e-10, max_cycles=300, coarse_direct=True,
                   coarse_cells=0, krylov=False, coarse_w=0):
        check(_lib.lib().cfg_server_set_solver(self._h, mode, ncycles, tol, max_cycles, _coarse_mode(coarse_direct),
                                               coarse_cells, int(krylov)))
        check(_lib.lib().cfg_server_set_coarse_w(self._h, int(coarse_w)))

    def slot_bytes(self, size_class: int) -> int:
        b = ctypes.c_size_t()
        check(_lib.lib().cfg_server_slot_bytes(self._h, size_class, ctypes.byref(b)))
        return b.value

    def run(self, jobs):
        """jobs: dicts with size_class, kind, seed, nsteps, arrival_s. Returns (results, wall_s, cell_updates)."""
        n = len(jobs)
        arr = (_lib.CfgJob * max(n, 1))()
        for i, j in enumerate(jobs):
            arr[i] = _lib.CfgJob(j["size_class"], j.get("kind", 1), j["seed"], j["nsteps"], 0, j["arrival_s"])
        res = (_lib.CfgJobResult * max(n, 1))()
        wall, cu = ctypes.c_double(), ctypes.c_double()
        check(_lib.lib().cfg_server_run(self._h, arr, n, res, ctypes.byref(wall), ctypes.byref(cu)))
        out = [{k: getattr(res[i], k) for k, _ in _lib.CfgJobResult._fields_ if k != "pad"} for i in range(n)]
        return out, wall.value, cu.value

    # -- the asynchronous service (a host thread runs the loop on submitted jobs)
    def submit(self, size_class: int, kind: int, seed: int, nsteps: int, keep_fields: bool = False) -> int:
        """Hand a job to the service; returns its ticket."""
        job = _lib.CfgJob(size_class, kind, seed, nsteps, _lib.CFG_JOB_KEEP_FIELDS if keep_fields else 0, 0.0)
        t = ctypes.c_uint64()
        check(_lib.lib().cfg_server_submit(self._h, ctypes.byref(job), ctypes.byref(t)))
        return t.value

    @staticmethod
    def _result(r) -> dict:
        return {k: getattr(r, k) for k, _ in _lib.CfgJobResult._fields_ if k != "pad"}

    def poll(self, ticket: int):
        """The job's result once it has finished (then released), else None."""
        r, done = _lib.CfgJobResult(), ctypes.c_int()
        check(_lib.lib().cfg_server_poll(self._h, ticket, ctypes.byref(r), ctypes.byref(done)))
        return self._result(r) if done.value else None

    def wait(self, ticket: int, timeout_s: float = 60.0) -> dict:
        r = _lib.CfgJobResult()
        check(_lib.lib().cfg_server_wait(self._h, ticket, float(timeout_s), ctypes.byref(r)))
        return self._result(r)

    def drain(self):
        check(_lib.lib().cfg_server_drain(self._h))

    def fetch(self, ticket: int, name: str, count: int) -> np.ndarray:
        """A finished keep_fields job's final field (dense float32)."""
        out = np.empty(count, np.float32)
        check(_lib.lib().cfg_server_fetch(self._h, ticket, name.encode(), _fp(out), count))
        return out

    def release(self, ticket: int):
        check(_lib.lib().cfg_server_release(self._h, ticket))


def field_hash(sim) -> int:
    """FNV-1a 64 of the dense T, Y, U, V float32 bytes (the hash cfg_server_run reports)."""
    h = 1469598103934665603
    for f in ("T", "Y", "U", "V"):
        for b in np.ascontiguousarray(sim.readBuffer(f), np.float32).tobytes():
            h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def autotune(dims, iters: int = 20, device: int = 0, coarse_direct: bool = False) -> dict:
    """Time the fused V-cycle under every coarse-block threshold on a scratch batch of these
    sizes (cfg_autotune); {"best": cells, "ms_per_cycle": {cells: ms}}."""
    n = len(dims)
    nx = (ctypes.c_int * n)(*[d[0] for d in dims])
    ny = (ctypes.c_int * n)(*[d[1] for d in dims])
    cap = 16
    cells = (ctypes.c_int * cap)()
    ms = (ctypes.c_double * cap)()
    k = ctypes.c_int(cap)
    best = ctypes.c_int()
    check(_lib.lib().cfg_autotune(device, n, nx, ny, 1 if coarse_direct else 0, iters, ctypes.byref(best), cells, ms,
                                  ctypes.byref(k)))
    return {"best": best.value, "ms_per_cycle": {cells[i]: ms[i] for i in range(k.value)}}


TILE_SHAPES = ((32, 8), (64, 8), (32, 16))


def autotune_tiles(dims, iters: int = 20, device: int = 0) -> dict:
    """Time the advection, diffusion + sources and forces kernels under every tile shape on a scratch
    batch of these sizes (cfg_autotune_tiles); {"best": (advect, diffuse_sources, forces) shape indices,
    "ms": {kernel: [ms per shape]}}."""
    n = len(dims)
    nx = (ctypes.c_int * n)(*[d[0] for d in dims])
    ny = (ctypes.c_int * n)(*[d[1] for d in dims])
    best = (ctypes.c_int * 3)()
    ms = (ctypes.c_double * 9)()
    check(_lib.lib().cfg_autotune_tiles(device, n, nx, ny, iters, best, ms))
    names = ("advect", "diffuse_sources", "forces")
    return {"best": tuple(best), "ms": {k: [ms[i * 3 + s] for s in range(3)] for i, k in enumerate(names)}}


def generate_scene(kind: int, nx: int, ny: int, width: float = 0.8, seed: int = 1234) -> dict:
    """Seeded synthetic scene (cfg_scene_generate): initial fields, pieces, params, dt."""
    T = np.empty(nx * ny, np.float32)
    Y = np.empty(4 * nx * ny, np.float32)
    U = np.empty((nx + 1) * ny, np.float32)
    V = np.empty(nx * (ny + 1), np.float32)
    pieces = np.zeros(_lib.MAX_PIECES * _lib.PIECE_FLOATS, np.float32)
    npc = ctypes.c_int()
    P = CfgParams()
    dt = ctypes.c_double()
    check(_lib.lib().cfg_scene_generate(kind, nx, ny, width, seed, _fp(T), _fp(Y), _fp(U), _fp(V), _fp(pieces),
                                        ctypes.byref(npc), ctypes.byref(P), ctypes.byref(dt)))
    params = {n: getattr(P, n) for n, _ in _lib.PARAM_FIELDS}
    return {"T": T, "Y": Y, "U": U, "V": V, "pieces": pieces, "npieces": npc.value, "params": params,
            "dt": dt.value, "nx": nx, "ny": ny, "width": width, "kind": kind, "seed": seed}


# parameters that the scene sets; the rest keep FluidSim's defaults
SCENE_PARAM_KEYS = ("Tamb", "rhoAmb", "YOamb", "reactB", "reactTa", "dHc", "Pr", "exchAlpha", "depth")


def load_scene(sim, scene: dict) -> None:
    """Apply a generated scene to a FluidSim-like object (product or oracle) and rasterise the wood."""
    for k in SCENE_PARAM_KEYS:
        sim_set = getattr(sim, "setParam", None) or getattr(sim, "set_param")
        sim_set(k, scene["params"][k])
    up = getattr(sim, "uploadPieces", None) or getattr(sim, "upload_pieces")
    up(scene["pieces"], scene["npieces"])
    (getattr(sim, "writeParams", None) or getattr(sim, "write_params"))()
    (getattr(sim, "reset", None))()
    wr = getattr(sim, "writeBuffer", None) or getattr(sim, "write")
    for k in ("T", "Y", "U", "V"):
        wr(k, scene[k])
    # the advected copies start equal to the state (reset() fills them the same way)
    wr("T2", scene["T"])
    wr("Y2", scene["Y"])
    (getattr(sim, "clearGeometry", None) or getattr(sim, "clear_geometry"))()
    (getattr(sim, "encodeGeometry", None) or getattr(sim, "geometry"))()
