"""Helpers of the GPU parity tests: the same scene and state on the CUDA path
(through the C ABI) and on the CPU oracle."""
import numpy as np

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

STATE = ("T", "Y", "U", "V", "T2", "Y2", "U2", "V2", "SQ")
# stage -> fields it writes (js/fluid.js:225-253 with the bindings of :120-154)
STAGE_OUT = {
    "advect": ("T2", "Y2", "U2", "V2"),
    "diffuse": ("T", "Y"),
    "sources": ("T", "Y", "SQ"),
    "forces": ("U", "V"),
    "coef_rhs": ("ax", "ay", "rhs"),
    "pressure": ("p",),
    "project": ("U", "V"),
}


def make_pair(oracle_mod, nx=128, ny=192, kind=0, seed=1234, warm_steps=8, width=0.8, mode=None, ncycles=1,
              tol=1e-6, max_cycles=50):
    """A GPU FluidSim and an f32 oracle holding the same scene after `warm_steps` oracle steps."""
    sc = cb.generate_scene(kind, nx, ny, width, seed)
    o = oracle_mod.OracleSim(nx, ny, width, sc["dt"])
    load_scene(o, sc)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=width).init()
    load_scene(g, sc)
    mode = oracle_mod.SOLVE_FIXED if mode is None else mode
    o.set_solver(mode, ncycles, tol, max_cycles)
    g.set_solver(mode, ncycles, tol, max_cycles)
    if warm_steps:
        o.set_solver(oracle_mod.SOLVE_FIXED, 1)
        o.step(warm_steps)
        o.set_solver(mode, ncycles, tol, max_cycles)
        sync(o, g)
    return g, o, sc


def levels_of(o):
    return int(o.info()["levels"])


def sync(o, g, fields=STATE, levels=True):
    """Copy the oracle's state into the GPU sim (f32 values: exact)."""
    for f in fields:
        g.writeBuffer(f, o.read(f).astype(np.float32))
    if levels:
        for l in range(levels_of(o)):
            for f in ("p", "rhs", "ax", "ay"):
                name = f if l == 0 else f"{f}.{l}"
                g.writeBuffer(name, o.read(name).astype(np.float32))


def fields_of(stage, o):
    out = list(STAGE_OUT[stage])
    if stage == "coef_rhs":
        out = ["rhs"] + [f"{f}.{l}" if l else f for l in range(levels_of(o)) for f in ("ax", "ay")]
    return out
