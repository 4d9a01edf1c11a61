"""ORACLE — test infrastructure, not product code.

ctypes wrappers over the CPU checkers:
  * oracle/liboracle_gas.so  — the C++ restatement of the reference WGSL gas step
    (gas_ref.hpp) and the 1D flame restatement (flame1d.c);
  * oracle/_ref/libwgslref.so — the reference's own WGSL translated mechanically
    to C++ (wgsl2cpp.py) under the FluidSim harness (wgsl_harness.cpp); built
    only where the reference checkout exists.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module, as the checker. Method names follow js/fluid.js's FluidSim so the parity
tests read like the reference's own harness (dev/gas_test.html).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle_gas.so")
REF_LIB_PATH = os.path.join(_HERE, "_ref", "libwgslref.so")
# the reference checkout, where one exists: CAMPFIRE_REF (environment); unset: the translated WGSL is not built
REFERENCE_ROOT = os.environ.get("CAMPFIRE_REF", "")

SOLVE_FIXED, SOLVE_TOL, SOLVE_FP64 = 0, 1, 2
STAGES = ("advect", "diffuse", "sources", "forces", "coef_rhs", "pressure", "project")


def build(force: bool = False) -> str:
    """Compile the restatement with its Makefile (g++ -O3 -fopenmp -ffp-contract=off)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True, stdout=subprocess.DEVNULL)
    return LIB_PATH


def build_ref(checkout: str | None = None) -> str | None:
    """Translate and compile the reference WGSL from the checkout at `checkout` (default: CAMPFIRE_REF);
    nothing is built where no checkout exists."""
    root = checkout or REFERENCE_ROOT
    if root and os.path.isdir(os.path.join(root, "shaders")):
        subprocess.run(["make", "-C", _HERE, "ref", f"REF={root}"], check=True, stdout=subprocess.DEVNULL)
    return REF_LIB_PATH if os.path.exists(REF_LIB_PATH) else None


def _declare(L, pfx):
    vp, ci, cd, cs = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p
    dp = ctypes.POINTER(ctypes.c_double)
    getattr(L, pfx + "error").restype = cs
    getattr(L, pfx + "create").restype = vp
    getattr(L, pfx + "create").argtypes = [ci, ci, cd, cd, ci]
    sigs = {
        "destroy": [vp], "reset": [vp], "write_params": [vp],
        "set_param": [vp, cs, cd], "get_param": [vp, cs, dp],
        "set_dt": [vp, cd], "set_cfl": [vp, cd, cd], "set_frame": [vp, ctypes.c_uint],
        "set_nray": [vp, ci], "set_solver": [vp, ci, ci, cd, ci],
        "upload_pieces": [vp, ctypes.POINTER(ctypes.c_float), ci],
        "clear_geometry": [vp], "geometry": [vp], "radiation": [vp],
        "step": [vp, ci], "vcycle": [vp, ci], "stage": [vp, cs],
        "read_field": [vp, cs, dp, ctypes.c_size_t], "write_field": [vp, cs, dp, ctypes.c_size_t],
        "readback": [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float),
                     ctypes.POINTER(ctypes.c_int32)],
        "budgets": [vp, dp], "info": [vp, dp], "level_dims": [vp, ci, ctypes.POINTER(ctypes.c_int)],
        "pressure_residual": [vp, dp], "set_coarse_solve": [vp, ci], "set_krylov": [vp, ci],
        "set_coarse_w": [vp, ci],
        "render": [vp, vp, ctypes.POINTER(ctypes.c_float), ci, ci, ctypes.POINTER(ctypes.c_float)],
    }
    for name, args in sigs.items():
        fn = getattr(L, pfx + name, None)
        if fn is not None:
            fn.restype = ci
            fn.argtypes = args


_libs = {}


def lib(which: str = "restatement"):
    """The restatement ("restatement") or the translated reference WGSL ("wgsl")."""
    if which not in _libs:
        if which == "restatement":
            if not os.path.exists(LIB_PATH):
                build()
            L = ctypes.CDLL(LIB_PATH)
            _declare(L, "orc_")
            L.flame1d_speed.restype = ctypes.c_double
            L.flame1d_speed.argtypes = [ctypes.c_double] * 7 + [ctypes.POINTER(ctypes.c_double)]
        else:
            if not os.path.exists(REF_LIB_PATH):
                raise OracleError("oracle/_ref/libwgslref.so is not built (needs the reference checkout)")
            L = ctypes.CDLL(REF_LIB_PATH)
            _declare(L, "wref_")
        _libs[which] = L
    return _libs[which]


def flame_speed(B=2e10, Ta=15000.0, dx=5e-5, F=1.0, phi=1.0, L=0.03, tEnd=1.0):
    """S_L and peak T of the restated tests/flame1d.mjs solver."""
    tb = ctypes.c_double()
    sl = lib().flame1d_speed(B, Ta, dx, F, phi, L, tEnd, ctypes.byref(tb))
    return sl, tb.value


class OracleError(RuntimeError):
    pass


class _Fns:
    def __init__(self, L, pfx):
        self._L, self._pfx = L, pfx

    def __getattr__(self, name):
        fn = getattr(self._L, self._pfx + name, None)
        if fn is None:
            raise OracleError(f"{self._pfx}{name} is not provided by this checker")
        return fn


class OracleSim:
    """FluidSim-shaped CPU checker.

    impl="restatement": the C++ restatement (fp64=False: f32 parity oracle, True: FP64).
    impl="wgsl": the reference's WGSL, mechanically translated (f32, one V-cycle per step).
    """

    def __init__(self, nx: int, ny: int, width: float, dt: float, fp64: bool = False, impl: str = "restatement"):
        L = lib(impl)
        self._f = _Fns(L, "orc_" if impl == "restatement" else "wref_")
        h = self._f.create(nx, ny, width, dt, 1 if fp64 else 0)
        if not h:
            raise OracleError(self._f.error().decode())
        self._h = h
        self.nx, self.ny, self.fp64, self.impl = nx, ny, fp64, impl

    def _chk(self, rc):
        if rc != 0:
            raise OracleError(self._f.error().decode())

    def close(self):
        if getattr(self, "_h", None):
            self._f.destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- FluidSim surface
    def reset(self): self._chk(self._f.reset(self._h))
    def set_param(self, k, v): self._chk(self._f.set_param(self._h, k.encode(), float(v)))

    def get_param(self, k):
        v = ctypes.c_double()
        self._chk(self._f.get_param(self._h, k.encode(), ctypes.byref(v)))
        return v.value

    def write_params(self): self._chk(self._f.write_params(self._h))
    def set_dt(self, dt): self._chk(self._f.set_dt(self._h, dt))
    def set_cfl(self, cfl, dt_cap): self._chk(self._f.set_cfl(self._h, cfl, dt_cap))
    def set_frame(self, f): self._chk(self._f.set_frame(self._h, f))
    def set_nray(self, n): self._chk(self._f.set_nray(self._h, n))

    def set_solver(self, mode=SOLVE_FIXED, ncycles=1, tol=1e-6, max_cycles=50):
        self._chk(self._f.set_solver(self._h, mode, ncycles, tol, max_cycles))

    def set_coarse_solve(self, direct):
        self._chk(self._f.set_coarse_solve(self._h, 2 if (direct == "pipelined" or (not isinstance(direct, bool) and direct == 2)) else (1 if direct else 0)))

    def set_krylov(self, on):
        self._chk(self._f.set_krylov(self._h, 1 if on else 0))

    def set_coarse_w(self, cells: int):
        """The solve loop's cycle: the W tail when the level two above the coarsest has <= cells cells (0: V-cycle)."""
        self._chk(self._f.set_coarse_w(self._h, int(cells)))

    def upload_pieces(self, data, n):
        a = np.zeros(64 * 20, np.float32)
        d = np.asarray(data, np.float32).ravel()
        a[: d.size] = d
        self._chk(self._f.upload_pieces(self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n))

    def clear_geometry(self): self._chk(self._f.clear_geometry(self._h))
    def geometry(self): self._chk(self._f.geometry(self._h))
    def radiation(self): self._chk(self._f.radiation(self._h))

    def render(self, rp: bytes, wood, width: int, height: int) -> np.ndarray:
        """render.wgsl's fragment stage (translated reference only): float32 [height, width, 4], row 0 at the top.
        rp: the 48-byte RP uniform; wood: 64 x 12 float32 or None."""
        out = np.zeros((height, width, 4), np.float32)
        rb = ctypes.create_string_buffer(bytes(rp), 48)
        w = None if wood is None else np.ascontiguousarray(np.asarray(wood, np.float32).ravel())
        wp = None if w is None else w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        self._chk(self._f.render(self._h, ctypes.cast(rb, ctypes.c_void_p), wp, width, height,
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out
    def step(self, n=1): self._chk(self._f.step(self._h, n))
    def vcycle(self, nu=2): self._chk(self._f.vcycle(self._h, nu))
    def stage(self, name): self._chk(self._f.stage(self._h, name.encode()))

    def field_size(self, name):
        nx, ny = self.nx, self.ny
        base = name.split(".")[0]
        lvl = int(name.split(".")[1]) if "." in name else 0
        if name in ("U", "Uh", "U2", "fx"):
            return (nx + 1) * ny
        if name in ("V", "Vh", "V2", "fy"):
            return nx * (ny + 1)
        if name in ("T", "Th", "T2", "p64"):
            return nx * ny
        if name in ("Y", "Yh", "Y2"):
            return 4 * nx * ny
        if name in ("SQ", "cellG"):
            return 2 * nx * ny
        if name == "rad":
            return 320 * 4
        d = (ctypes.c_int * 2)()
        self._chk(self._f.level_dims(self._h, lvl, d))
        lx, ly = d[0], d[1]
        return {"p": lx * ly, "rhs": lx * ly, "ax": (lx + 1) * ly, "ay": lx * (ly + 1)}[base]

    def read(self, name):
        n = self.field_size(name)
        out = np.empty(n, np.float64)
        self._chk(self._f.read_field(self._h, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))
        return out

    def write(self, name, arr):
        a = np.ascontiguousarray(np.asarray(arr, np.float64).ravel())
        self._chk(self._f.write_field(self._h, name.encode(), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size))

    def readback(self):
        acc = np.zeros(528, np.int32)
        rad = np.zeros(320 * 4, np.float32)
        fw = np.zeros(256, np.int32)
        self._chk(self._f.readback(self._h, acc.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                   rad.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                   fw.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return {"acc": acc, "rad": rad, "faceW": fw}

    def budgets(self):
        o = np.zeros(8, np.float64)
        self._chk(self._f.budgets(self._h, o.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return o

    def info(self):
        o = np.zeros(16, np.float64)
        self._chk(self._f.info(self._h, o.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        keys = ["nx", "ny", "dx", "dt", "time", "frame", "diffSub", "levels", "last_cycles",
                "last_rel", "height", "last_rel0"]
        return dict(zip(keys, o[: len(keys)].tolist()))

    def copy_state_from(self, sim, cfl: float = 0.0, dt_cap: float = 0.0):
        """Take over the state of a FluidSim-like object (readBuffer / read_p64 / info): every field a step
        reads or keeps (the gas fields and their advected copies, sources, geometry, the multigrid levels,
        the FP64 pressure) and its time step, so that the next step starts from identical values (f32
        values are exact in either arithmetic). cfl > 0: the CFL step with this cap continues."""
        for f in ("T", "Y", "U", "V", "T2", "Y2", "U2", "V2", "SQ", "fx", "fy"):
            self.write(f, sim.readBuffer(f))
        cg = np.ascontiguousarray(sim.readBuffer("cellG"), np.float32)
        g = np.empty(cg.size, np.float64)
        g[0::2] = cg[0::2]
        g[1::2] = cg.view(np.uint32)[1::2]          # bitcast<f32>(piece*4+face) -> its integer value
        self.write("cellG", g)
        for lvl in range(int(self.info()["levels"])):
            for f in ("p", "rhs", "ax", "ay"):
                name = f if lvl == 0 else f"{f}.{lvl}"
                self.write(name, sim.readBuffer(name))
        self.write("p64", sim.read_p64())
        self.set_dt(float(sim.info()["dt"]))
        if cfl > 0:
            self.set_cfl(cfl, dt_cap)
        self.write_params()

    def pressure_residual(self):
        v = ctypes.c_double()
        self._chk(self._f.pressure_residual(self._h, ctypes.byref(v)))
        return v.value
