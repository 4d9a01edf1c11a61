"""The Krylov FP64 mode: flexible preconditioned CG on the level-0 operator in FP64
with the FP32 V-cycle as preconditioner (an extension of the FP64 defect
correction; the oracle runs the same iteration with sequential dot products).
"""
import numpy as np
import pytest

import campfire_b200 as cb
from conftest import norm_err
from gpu_pairs import make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nx,ny,kind,tol", [(128, 192, 0, 1e-10), (96, 144, 2, 1e-8), (256, 384, 0, 1e-6)])
def test_krylov_step_matches_oracle(oracle_mod, nx, ny, kind, tol):
    g, o, _ = make_pair(oracle_mod, nx, ny, kind=kind, seed=1400 + nx, warm_steps=4, mode=cb.SOLVE_FP64, tol=tol,
                        max_cycles=200)
    for s in (g, o):
        s.set_coarse_solve(True)
        s.set_krylov(True)
    g.step(1); o.step(1)
    gi, oi = g.info(), o.info()
    assert abs(gi["last_cycles"] - oi["last_cycles"]) <= 1, (gi["last_cycles"], oi["last_cycles"])
    assert gi["last_rel"] <= tol
    assert norm_err(g.read_p64(), o.read("p64")) <= 1e-5
    for f in ("T", "Y", "U", "V", "SQ"):
        assert norm_err(g.readBuffer(f), o.read(f)) <= 1e-4, f
    g.close()


def test_krylov_needs_fewer_cycles_for_the_same_pressure(oracle_mod):
    out = {}
    for kr in (False, True):
        g, o, _ = make_pair(oracle_mod, 256, 384, kind=0, seed=1235, warm_steps=4, mode=cb.SOLVE_FP64, tol=1e-10,
                            max_cycles=300)
        g.set_coarse_solve(True)
        g.set_krylov(kr)
        g.step(1)
        out[kr] = (g.info()["last_cycles"], g.read_p64())
        g.close()
    assert out[True][0] <= 0.7 * out[False][0], (out[True][0], out[False][0])
    assert norm_err(out[True][1], out[False][1]) <= 1e-5


def test_graph_and_host_loops_agree_in_krylov_mode(oracle_mod):
    res = []
    for graphs in (True, False):
        g, o, _ = make_pair(oracle_mod, 96, 144, kind=2, seed=2001, warm_steps=3, mode=cb.SOLVE_FP64, tol=1e-9,
                            max_cycles=100)
        g.set_coarse_solve(True)
        g.set_krylov(True)
        g.set_graphs(graphs)
        g.step(2)
        res.append((g.info()["last_cycles"], g.read_p64().tobytes(), cb.field_hash(g)))
        g.close()
    assert res[0] == res[1]


def _krylov_run(cells, nx=64, ny=96, steps=3):
    from campfire_b200.fluid import load_scene
    sc = cb.generate_scene(0, nx, ny, 0.8, 1235)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    g.set_solver(cb.SOLVE_FP64, 1, 1e-8, 100)
    g.set_coarse_solve("pipelined")
    g.set_krylov(True)
    g.set_coarse_cells(cells)
    g.step(steps)
    out = {f: g.readBuffer(f) for f in ("T", "U", "V")}
    out["p64"] = g.read_p64()
    out["cycles"] = g.info()["last_cycles"]
    out["rel"] = g.info()["last_rel"]
    import ctypes
    m, b, n = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    cb._lib.check(cb.lib().cfg_time_kernel(g._h, b"pcg_step", 1, ctypes.byref(m), ctypes.byref(b), ctypes.byref(n)))
    out["pcg_step_per_step"] = n.value
    g.close()
    return out


def test_fused_krylov_update_matches_the_separate_kernel():
    """64x96: coarse block from level 1 (the level-0 smoother kernels carry the Krylov update
    and decide from the dot-product recurrence) against a coarse block that covers level 0
    (the separate update kernel, direct ||r||): the V-cycles give the same bits, so only the
    reduction order and the stopping test's rounding differ."""
    fused, sep = _krylov_run(1536), _krylov_run(100000)
    assert fused["pcg_step_per_step"] == 0 and sep["pcg_step_per_step"] > 0
    assert abs(fused["cycles"] - sep["cycles"]) <= 1, (fused["cycles"], sep["cycles"])
    assert fused["rel"] <= 1e-8 and sep["rel"] <= 1e-8
    assert norm_err(fused["p64"], sep["p64"]) <= 1e-7
    for f in ("T", "U", "V"):
        assert norm_err(fused[f], sep[f]) <= 1e-6, f
