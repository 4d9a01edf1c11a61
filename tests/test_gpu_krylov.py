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
