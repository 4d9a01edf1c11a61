"""ORACLE — test infrastructure, not product code.

ctypes wrapper over oracle/liboracle_gas.so: the CPU restatement of the
reference WGSL gas step (gas_ref.hpp) and the 1D flame restatement
(flame1d.c). Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg import this module, as the checker. The method names follow
js/fluid.js's FluidSim so the parity tests read like the reference's own
harness (dev/gas_test.html).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liboracle_gas.so")

SOLVE_FIXED, SOLVE_TOL, SOLVE_FP64 = 0, 1, 2
STAGES = ("advect", "diffuse", "sources", "forces", "coef_rhs", "pressure", "project")


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O3 -fopenmp -ffp-contract=off)."""
    if force or not os.path.exists(LIB_PATH):
        subprocess.run(["make", "-C", _HERE, "-B" if force else "all"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, ci, cd, cs = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p
        dp = ctypes.POINTER(ctypes.c_double)
        L.orc_error.restype = cs
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ci, ci, cd, cd, ci]
        for name, args in {
            "orc_destroy": [vp], "orc_reset": [vp], "orc_write_params": [vp],
            "orc_set_param": [vp, cs, cd], "orc_get_param": [vp, cs, dp],
            "orc_set_dt": [vp, cd], "orc_set_cfl": [vp, cd, cd], "orc_set_frame": [vp, ctypes.c_uint],
            "orc_set_nray": [vp, ci], "orc_set_solver": [vp, ci, ci, cd, ci],
            "orc_upload_pieces": [vp, ctypes.POINTER(ctypes.c_float), ci],
            "orc_clear_geometry": [vp], "orc_geometry": [vp], "orc_radiation": [vp],
            "orc_step": [vp, ci], "orc_vcycle": [vp, ci], "orc_stage": [vp, cs],
            "orc_read_field": [vp, cs, dp, ctypes.c_size_t],
            "orc_write_field": [vp, cs, dp, ctypes.c_size_t],
            "orc_readback": [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float),
                             ctypes.POINTER(ctypes.c_int32)],
            "orc_budgets": [vp, dp], "orc_info": [vp, dp],
            "orc_level_dims": [vp, ci, ctypes.POINTER(ctypes.c_int)],
            "orc_pressure_residual": [vp, dp],
        }.items():
            fn = getattr(L, name)
            fn.restype = ci
            fn.argtypes = args
        L.flame1d_speed.restype = cd
        L.flame1d_speed.argtypes = [cd] * 7 + [dp]
        _lib = L
    return _lib


def flame_speed(B=2e10, Ta=15000.0, dx=5e-5, F=1.0, phi=1.0, L=0.03, tEnd=1.0):
    """S_L and peak T of the restated tests/flame1d.mjs solver."""
    tb = ctypes.c_double()
    sl = lib().flame1d_speed(B, Ta, dx, F, phi, L, tEnd, ctypes.byref(tb))
    return sl, tb.value


class OracleError(RuntimeError):
    pass


def _chk(rc):
    if rc != 0:
        raise OracleError(lib().orc_error().decode())


class OracleSim:
    """FluidSim-shaped wrapper over the CPU oracle (fp64=False: f32 parity oracle)."""

    def __init__(self, nx: int, ny: int, width: float, dt: float, fp64: bool = False):
        self._L = lib()
        h = self._L.orc_create(nx, ny, width, dt, 1 if fp64 else 0)
        if not h:
            raise OracleError(self._L.orc_error().decode())
        self._h = h
        self.nx, self.ny, self.fp64 = nx, ny, fp64

    def close(self):
        if self._h:
            self._L.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- FluidSim surface
    def reset(self): _chk(self._L.orc_reset(self._h))
    def set_param(self, k, v): _chk(self._L.orc_set_param(self._h, k.encode(), float(v)))

    def get_param(self, k):
        v = ctypes.c_double()
        _chk(self._L.orc_get_param(self._h, k.encode(), ctypes.byref(v)))
        return v.value

    def write_params(self): _chk(self._L.orc_write_params(self._h))
    def set_dt(self, dt): _chk(self._L.orc_set_dt(self._h, dt))
    def set_cfl(self, cfl, dt_cap): _chk(self._L.orc_set_cfl(self._h, cfl, dt_cap))
    def set_frame(self, f): _chk(self._L.orc_set_frame(self._h, f))
    def set_nray(self, n): _chk(self._L.orc_set_nray(self._h, n))

    def set_solver(self, mode=SOLVE_FIXED, ncycles=1, tol=1e-6, max_cycles=50):
        _chk(self._L.orc_set_solver(self._h, mode, ncycles, tol, max_cycles))

    def upload_pieces(self, data, n):
        a = np.zeros(64 * 20, np.float32)
        d = np.asarray(data, np.float32).ravel()
        a[: d.size] = d
        _chk(self._L.orc_upload_pieces(self._h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), n))

    def clear_geometry(self): _chk(self._L.orc_clear_geometry(self._h))
    def geometry(self): _chk(self._L.orc_geometry(self._h))
    def radiation(self): _chk(self._L.orc_radiation(self._h))
    def step(self, n=1): _chk(self._L.orc_step(self._h, n))
    def vcycle(self, nu=2): _chk(self._L.orc_vcycle(self._h, nu))
    def stage(self, name): _chk(self._L.orc_stage(self._h, name.encode()))

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
        d = (ctypes.c_int * 2)()
        _chk(self._L.orc_level_dims(self._h, lvl, d))
        lx, ly = d[0], d[1]
        return {"p": lx * ly, "rhs": lx * ly, "ax": (lx + 1) * ly, "ay": lx * (ly + 1)}[base]

    def read(self, name):
        n = self.field_size(name)
        out = np.empty(n, np.float64)
        _chk(self._L.orc_read_field(self._h, name.encode(), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n))
        return out

    def write(self, name, arr):
        a = np.ascontiguousarray(np.asarray(arr, np.float64).ravel())
        _chk(self._L.orc_write_field(self._h, name.encode(), a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size))

    def readback(self):
        acc = np.zeros(528, np.int32)
        rad = np.zeros(320 * 4, np.float32)
        fw = np.zeros(256, np.int32)
        _chk(self._L.orc_readback(self._h, acc.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                  rad.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                  fw.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return {"acc": acc, "rad": rad, "faceW": fw}

    def budgets(self):
        o = np.zeros(8, np.float64)
        _chk(self._L.orc_budgets(self._h, o.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return o

    def info(self):
        o = np.zeros(16, np.float64)
        _chk(self._L.orc_info(self._h, o.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        keys = ["nx", "ny", "dx", "dt", "time", "frame", "diffSub", "levels", "last_cycles",
                "last_rel", "height", "last_rel0"]
        return dict(zip(keys, o[: len(keys)].tolist()))

    def pressure_residual(self):
        v = ctypes.c_double()
        _chk(self._L.orc_pressure_residual(self._h, ctypes.byref(v)))
        return v.value
