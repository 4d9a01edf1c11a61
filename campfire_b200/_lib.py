"""ctypes binding of libcampfire_gas.so (include/campfire_gas.h).

The library is built in-tree by campfire_b200.build. There is no CPU fallback:
importing works without a GPU, but every computing call fails with
CampfireError (CFG_ERR_NODEV) when no CUDA device is present.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcampfire_gas.so")
HEADER = os.path.join(HERE, "..", "include", "campfire_gas.h")

CFG_OK = 0
ERRORS = {-2: "CFG_ERR_NOENT", -5: "CFG_ERR_IO", -12: "CFG_ERR_NOMEM", -16: "CFG_ERR_BUSY",
          -19: "CFG_ERR_NODEV", -22: "CFG_ERR_INVAL", -34: "CFG_ERR_RANGE", -110: "CFG_ERR_TIMEDOUT"}
SOLVE_FIXED, SOLVE_TOL, SOLVE_FP64 = 0, 1, 2
MAX_PIECES, PIECE_FLOATS, ACC_GLOBAL, ACC_LEN = 64, 20, 512, 528
E_SCALE, M_SCALE, G_SCALE, N_FLOOR, RAD_LEN = 1e6, 1e12, 1e3, 64, 320
MAX_LEVELS = 7
CFG_JOB_KEEP_FIELDS = 1

PARAM_FIELDS = [
    ("nx", "i"), ("ny", "i"), ("dx", "f"), ("dt", "f"),
    ("Tamb", "f"), ("rhoAmb", "f"), ("YOamb", "f"), ("grav", "f"),
    ("cp", "f"), ("Pr", "f"), ("viscMult", "f"), ("diffMult", "f"),
    ("reactB", "f"), ("reactTa", "f"), ("dHc", "f"), ("sO2", "f"),
    ("sootFormA", "f"), ("sootFormTa", "f"), ("sootOxA", "f"), ("sootOxTa", "f"),
    ("kappaSootC", "f"), ("kappaGas", "f"), ("exchAlpha", "f"), ("depth", "f"),
    ("charA", "f"), ("charTa", "f"), ("nPieces", "i"), ("frame", "u"),
    ("heaterX0", "f"), ("heaterX1", "f"), ("heaterY1", "f"), ("heaterT", "f"),
    ("burnerX0", "f"), ("burnerX1", "f"), ("burnerFlux", "f"), ("burnerT", "f"),
    ("sootDensity", "f"), ("sigma", "f"), ("charO2", "f"), ("time", "f"),
]
_CT = {"i": ctypes.c_int32, "f": ctypes.c_float, "u": ctypes.c_uint32}


class CfgParams(ctypes.Structure):
    """The 40-field uniform of shaders/common.wgsl:4-15."""
    _fields_ = [(n, _CT[t]) for n, t in PARAM_FIELDS]


class CfgInfo(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("levels", ctypes.c_int32),
                ("diff_sub", ctypes.c_int32), ("dx", ctypes.c_double), ("dt", ctypes.c_double),
                ("height", ctypes.c_double), ("time", ctypes.c_double), ("frame", ctypes.c_uint32),
                ("last_cycles", ctypes.c_int32), ("last_rel", ctypes.c_double),
                ("level_nx", ctypes.c_int32 * MAX_LEVELS), ("level_ny", ctypes.c_int32 * MAX_LEVELS)]


class CfgJob(ctypes.Structure):
    _fields_ = [("size_class", ctypes.c_int32), ("kind", ctypes.c_int32), ("seed", ctypes.c_uint64),
                ("nsteps", ctypes.c_int32), ("flags", ctypes.c_int32), ("arrival_s", ctypes.c_double)]


class CfgJobResult(ctypes.Structure):
    _fields_ = [("arrival_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double),
                ("slot", ctypes.c_int32), ("steps", ctypes.c_int32), ("last_cycles", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("last_rel", ctypes.c_double), ("hash", ctypes.c_uint64),
                ("t_sum", ctypes.c_double)]


class CfgWoodPiece(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("side", "rhoV", "rhoC", "mv", "mc", "Tc", "gasRate")] + \
               [(n, ctypes.c_double * 4) for n in ("Ts", "Tp", "d", "mflux", "charCov", "exposure")] + \
               [("dead", ctypes.c_int32), ("pad", ctypes.c_int32)]


class CfgRenderParams(ctypes.Structure):
    """The uniform RP of shaders/render.wgsl:13-17 (js/render.js:41-53)."""
    _fields_ = [("view", ctypes.c_int32), ("nPieces", ctypes.c_int32)] + \
               [(n, ctypes.c_float) for n in ("exposure", "width", "height", "ground", "time", "tmax", "chemi",
                                               "camX", "camY", "zoom")]


class CfgRigidParams(ctypes.Structure):
    """RIGID_DEFAULTS of js/rigid.js:12-27."""
    _fields_ = [("gravity", ctypes.c_double * 2), ("width", ctypes.c_double), ("dt", ctypes.c_double),
                ("substeps", ctypes.c_int32), ("pad", ctypes.c_int32)] + \
               [(n, ctypes.c_double) for n in ("slop", "contact_hertz", "contact_damping", "max_pushout", "mu_static",
                                               "mu_kinetic", "stick_speed", "max_speed", "drag_hertz",
                                               "drag_strength")]


class CfgRigidBody(ctypes.Structure):
    _fields_ = [("id", ctypes.c_int32), ("dragging", ctypes.c_int32)] + \
               [(n, ctypes.c_double) for n in ("x", "y", "a", "vx", "vy", "w", "half", "density", "mass")]


class CampfireError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


def declared_symbols() -> list[str]:
    """Entry points declared in include/campfire_gas.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*int\s+(cfg_\w+)\s*\(", text, re.M)))


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CampfireError(-5, f"{LIB_PATH} is missing: build it with `python -m campfire_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, ci, cd, cs, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_char_p, ctypes.c_size_t
    fp, dp, ip = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int)
    i32p = ctypes.POINTER(ctypes.c_int32)
    sigs = {
        "cfg_version": [], "cfg_last_error": [ctypes.c_char_p, sz],
        "cfg_default_params": [ctypes.POINTER(CfgParams)], "cfg_device_count": [ip],
        "cfg_create": [ci, ci, cd, cd, ci, ctypes.POINTER(vp)], "cfg_destroy": [vp], "cfg_reset": [vp],
        "cfg_set_param": [vp, cs, cd], "cfg_get_param": [vp, cs, dp], "cfg_set_dt": [vp, cd],
        "cfg_write_params": [vp], "cfg_upload_pieces": [vp, fp, ci], "cfg_clear_geometry": [vp],
        "cfg_geometry": [vp], "cfg_step": [vp, ci], "cfg_step_profiled": [vp, fp],
        "cfg_run_stage": [vp, cs], "cfg_vcycle": [vp, ci], "cfg_radiation": [vp],
        "cfg_set_frame": [vp, ctypes.c_uint32], "cfg_readback": [vp, i32p, fp, i32p],
        "cfg_readback_begin": [vp, ctypes.c_uint64, ip],
        "cfg_readback_poll": [vp, i32p, fp, i32p, ctypes.POINTER(ctypes.c_uint64), ip],
        "cfg_readback_wait": [vp, i32p, fp, i32p, ctypes.POINTER(ctypes.c_uint64)],
        "cfg_field_size": [vp, cs, ctypes.POINTER(sz)], "cfg_read_field": [vp, cs, fp, sz],
        "cfg_write_field": [vp, cs, fp, sz], "cfg_read_p64": [vp, dp, sz],
        "cfg_get_info": [vp, ctypes.POINTER(CfgInfo)], "cfg_set_solver": [vp, ci, ci, cd, ci],
        "cfg_set_cfl": [vp, cd, cd], "cfg_set_nray": [vp, ci], "cfg_pressure_residual": [vp, dp],
        "cfg_budgets": [vp, dp], "cfg_set_stream": [vp, vp], "cfg_synchronize": [vp],
        "cfg_set_graphs": [vp, ci], "cfg_launch_count": [vp, ip],
        "cfg_scene_generate": [ci, ci, ci, cd, ctypes.c_uint64, fp, fp, fp, fp, fp, ip,
                               ctypes.POINTER(CfgParams), dp],
        "cfg_batch_create": [ci, ip, ip, dp, dp, ci, ctypes.POINTER(vp)], "cfg_batch_destroy": [vp],
        "cfg_batch_scene": [vp, ci, ctypes.POINTER(vp)], "cfg_batch_set_solver": [vp, ci, ci, cd, ci],
        "cfg_batch_set_active": [vp, ci, ci], "cfg_batch_step": [vp, ci], "cfg_batch_set_stream": [vp, vp],
        "cfg_batch_synchronize": [vp], "cfg_batch_launch_count": [vp, ip], "cfg_batch_set_graphs": [vp, ci], "cfg_batch_write_params": [vp],
        "cfg_batch_geometry": [vp],
        "cfg_time_kernel": [vp, cs, ci, dp, dp, dp],
        "cfg_pressure_residual_noalloc": [vp, vp, vp, vp, ci, ci, cd, vp, dp],
        "cfg_set_coarse_cells": [vp, ci], "cfg_batch_set_coarse_cells": [vp, ci],
        "cfg_set_coarse_cluster": [vp, ci], "cfg_batch_set_coarse_cluster": [vp, ci],
        "cfg_set_coarse_w": [vp, ci], "cfg_batch_set_coarse_w": [vp, ci], "cfg_server_set_coarse_w": [vp, ci],
        "cfg_autotune": [ci, ci, ip, ip, ci, ci, ip, ip, dp, ip],
        "cfg_set_coarse_solve": [vp, ci], "cfg_batch_set_coarse_solve": [vp, ci],
        "cfg_set_tiles": [vp, ci, ci, ci], "cfg_batch_set_tiles": [vp, ci, ci, ci],
        "cfg_autotune_tiles": [ci, ci, ip, ip, ci, ip, dp],
        "cfg_checkpoint_save": [vp, cs], "cfg_checkpoint_load": [vp, cs],
        "cfg_wood_piece_init": [ctypes.POINTER(CfgWoodPiece), cd, cd, cd],
        "cfg_wood_piece_preheat": [ctypes.POINTER(CfgWoodPiece), cd, cd, cd, cd],
        "cfg_wood_piece_step": [ctypes.POINTER(CfgWoodPiece), cd, dp, dp, dp, cd, cd],
        "cfg_wood_create": [vp, cd, cd, ctypes.POINTER(vp)], "cfg_wood_destroy": [vp],
        "cfg_wood_add": [vp, cd, cd, cd, cd, cd, dp, dp, ip], "cfg_wood_remove": [vp, ci],
        "cfg_wood_frame": [vp, cd, ip], "cfg_wood_get": [vp, ci, ctypes.POINTER(CfgWoodPiece), dp, dp],
        "cfg_wood_stats": [vp, dp, dp, dp], "cfg_wood_render_data": [vp, fp],
        "cfg_wood_set_readback_lag": [vp, ci],
        "cfg_wood_readbacks": [vp, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)],
        "cfg_render_defaults": [vp, ctypes.POINTER(CfgRenderParams)],
        "cfg_render": [vp, ctypes.POINTER(CfgRenderParams), fp, ci, ci, fp],
        "cfg_render_device": [vp, ctypes.POINTER(CfgRenderParams), fp, ci, ci, vp],
        "cfg_wood_set": [vp, ci, ctypes.POINTER(CfgWoodPiece)],
        "cfg_wood_set_rigid": [vp, ctypes.POINTER(CfgRigidParams)], "cfg_wood_rigid": [vp, ctypes.POINTER(vp)],
        "cfg_wood_body": [vp, ci, ip],
        "cfg_rigid_defaults": [ctypes.POINTER(CfgRigidParams)],
        "cfg_rigid_create": [ctypes.POINTER(CfgRigidParams), ctypes.POINTER(vp)], "cfg_rigid_destroy": [vp],
        "cfg_rigid_get_params": [vp, ctypes.POINTER(CfgRigidParams)],
        "cfg_rigid_set_params": [vp, ctypes.POINTER(CfgRigidParams)],
        "cfg_rigid_add": [vp, cd, cd, cd, cd, cd, ip], "cfg_rigid_remove": [vp, ci],
        "cfg_rigid_resize": [vp, ci, cd], "cfg_rigid_set_density": [vp, ci, cd],
        "cfg_rigid_step": [vp, cd, ci], "cfg_rigid_advance": [vp, cd],
        "cfg_rigid_bodies": [vp, ctypes.POINTER(CfgRigidBody), ci, ip],
        "cfg_rigid_get": [vp, ci, ctypes.POINTER(CfgRigidBody)], "cfg_rigid_pick": [vp, cd, cd, ip, dp, dp],
        "cfg_rigid_drag_start": [vp, ci, cd, cd, cd, cd], "cfg_rigid_drag_move": [vp, ci, cd, cd],
        "cfg_rigid_drag_end": [vp, ci], "cfg_rigid_max_penetration": [vp, dp], "cfg_rigid_contacts": [vp, ip, ip],
        "cfg_server_create": [ci, ci, ip, ip, ip, cd, cd, ctypes.POINTER(vp)], "cfg_server_destroy": [vp],
        "cfg_server_set_solver": [vp, ci, ci, cd, ci, ci, ci, ci],
        "cfg_set_krylov": [vp, ci], "cfg_batch_set_krylov": [vp, ci],
        "cfg_krylov_folded": [vp, ctypes.POINTER(ci)], "cfg_batch_krylov_folded": [vp, ctypes.POINTER(ci)],
        "cfg_server_slot_bytes": [vp, ci, ctypes.POINTER(sz)],
        "cfg_server_run": [vp, ctypes.POINTER(CfgJob), ci, ctypes.POINTER(CfgJobResult), dp, dp],
        "cfg_server_submit": [vp, ctypes.POINTER(CfgJob), ctypes.POINTER(ctypes.c_uint64)],
        "cfg_server_poll": [vp, ctypes.c_uint64, ctypes.POINTER(CfgJobResult), ip],
        "cfg_server_wait": [vp, ctypes.c_uint64, cd, ctypes.POINTER(CfgJobResult)],
        "cfg_server_drain": [vp], "cfg_server_fetch": [vp, ctypes.c_uint64, cs, fp, sz],
        "cfg_server_release": [vp, ctypes.c_uint64],
    }
    for name, args in sigs.items():
        f = getattr(L, name)
        f.restype = ci
        f.argtypes = args
    _lib = L
    return L


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().cfg_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != CFG_OK:
        raise CampfireError(rc, last_error())


def device_count() -> int:
    n = ctypes.c_int()
    check(lib().cfg_device_count(ctypes.byref(n)))
    return n.value
