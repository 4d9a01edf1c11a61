"""The direct coarsest solve of the TOL and FP64 modes (an extension: the coarsest
operator inverted once per step instead of 120 red-black sweeps per cycle).

The inversion and the per-cycle product follow one operation order on the GPU
and in the oracle, so a cycle stays bit-exact; over a whole FP64 solve only the
FP64 norms' summation order differs.
"""
import numpy as np
import pytest

import campfire_b200 as cb
from conftest import norm_err
from gpu_pairs import levels_of, make_pair, sync

pytestmark = pytest.mark.gpu


def test_direct_cycles_are_bit_exact(oracle_mod):
    g, o, _ = make_pair(oracle_mod, 128, 192, kind=0, seed=1234, warm_steps=6, mode=cb.SOLVE_TOL, tol=1e-30,
                        max_cycles=3)
    g.set_coarse_solve(True); o.set_coarse_solve(True)
    g.run_stage("coef_rhs"); o.stage("coef_rhs")
    sync(o, g)
    g.run_stage("pressure"); o.stage("pressure")
    assert g.info()["last_cycles"] == o.info()["last_cycles"] == 3
    # the fused cycle keeps the coarse block's levels in shared memory: level 0 is the result
    a, b = g.readBuffer("p").astype(np.float64), o.read("p")
    assert np.array_equal(a, b), norm_err(a, b)
    g.close()


@pytest.mark.parametrize("nx,ny,kind", [(128, 192, 0), (96, 144, 2)])
def test_direct_fp64_step_matches_oracle(oracle_mod, nx, ny, kind):
    g, o, _ = make_pair(oracle_mod, nx, ny, kind=kind, seed=1300 + nx, warm_steps=5, mode=cb.SOLVE_FP64, tol=1e-10,
                        max_cycles=200)
    g.set_coarse_solve(True); o.set_coarse_solve(True)
    g.step(1); o.step(1)
    gi, oi = g.info(), o.info()
    assert abs(gi["last_cycles"] - oi["last_cycles"]) <= 1, (gi, oi)
    assert gi["last_rel"] <= 1e-10
    # the step's rhs comes through stages with transcendental functions (within 1e-4 per
    # field), and the stop decision's FP64 norms are summed in another order
    e = norm_err(g.read_p64(), o.read("p64"))
    assert e <= 1e-5, (e, gi["last_cycles"], oi["last_cycles"])
    for f in ("T", "Y", "U", "V", "SQ"):
        assert norm_err(g.readBuffer(f), o.read(f)) <= 1e-4, f
    g.close()


def test_direct_and_sweeps_reach_the_same_pressure(oracle_mod):
    out = {}
    for direct in (False, True):
        g, o, _ = make_pair(oracle_mod, 128, 192, kind=0, seed=1234, warm_steps=6, mode=cb.SOLVE_FP64, tol=1e-10,
                            max_cycles=200)
        g.set_coarse_solve(direct)
        g.step(1)
        out[direct] = (g.info()["last_cycles"], g.read_p64())
        g.close()
    assert abs(out[True][0] - out[False][0]) <= 2
    assert norm_err(out[True][1], out[False][1]) <= 1e-5


def test_singular_coarsest_keeps_the_sweeps(oracle_mod):
    """A gas pocket sealed on the coarsest level (pure Neumann: singular operator) is
    not inverted; the cycle then runs the reference's sweeps, on the GPU as in the oracle."""
    g, o, _ = make_pair(oracle_mod, 128, 192, kind=0, seed=1234, warm_steps=6, mode=cb.SOLVE_TOL, tol=1e-30,
                        max_cycles=2)
    g.set_coarse_solve(True); o.set_coarse_solve(True)
    g.run_stage("coef_rhs"); o.stage("coef_rhs")
    L = levels_of(o) - 1
    ax, ay = o.read(f"ax.{L}"), o.read(f"ay.{L}")
    cnx, cny = g.info()["level_dims"][L]
    ax = ax.reshape(cny, cnx + 1).copy(); ay = ay.reshape(cny + 1, cnx).copy()
    # seal cells (2..3, 2..3) from the rest: close every face on the pocket's boundary
    ax[2:4, 2] = 0.0; ax[2:4, 4] = 0.0; ay[2, 2:4] = 0.0; ay[4, 2:4] = 0.0
    o.write(f"ax.{L}", ax.ravel()); o.write(f"ay.{L}", ay.ravel())
    sync(o, g)
    g.run_stage("pressure"); o.stage("pressure")
    a, b = g.readBuffer("p").astype(np.float64), o.read("p")
    assert np.array_equal(a, b), norm_err(a, b)
    g.close()


def test_pipelined_stages_are_bit_exact(oracle_mod):
    """Pipelined coarse solve: the first solve after a reset has no inverse (sweeps) and factors
    its operator for the next; the second solve applies that inverse. Both bit-exact."""
    g, o, _ = make_pair(oracle_mod, 128, 192, kind=0, seed=1234, warm_steps=6, mode=cb.SOLVE_TOL, tol=1e-30,
                        max_cycles=3)
    g.set_coarse_solve("pipelined"); o.set_coarse_solve("pipelined")
    g.run_stage("coef_rhs"); o.stage("coef_rhs")
    sync(o, g)
    for k in range(2):
        g.run_stage("pressure"); o.stage("pressure")
        a, b = g.readBuffer("p").astype(np.float64), o.read("p")
        assert np.array_equal(a, b), (k, norm_err(a, b))
    g.close()


def test_pipelined_fp64_steps_match_oracle(oracle_mod):
    g, o, _ = make_pair(oracle_mod, 128, 192, kind=0, seed=1400, warm_steps=4, mode=cb.SOLVE_FP64, tol=1e-10,
                        max_cycles=200)
    g.set_krylov(True); o.set_krylov(True)
    g.set_coarse_solve("pipelined"); o.set_coarse_solve("pipelined")
    for k in range(3):
        g.step(1); o.step(1)
        gi, oi = g.info(), o.info()
        assert abs(gi["last_cycles"] - oi["last_cycles"]) <= 1, (k, gi, oi)
        assert gi["last_rel"] <= 1e-10
        e = norm_err(g.read_p64(), o.read("p64"))
        assert e <= 1e-5 * (k + 1), (k, e)
    g.close()


def test_pipelined_and_direct_take_the_same_cycles():
    """On the benchmark scene the previous step's coarsest inverse costs no cycles in the
    Krylov mode (the oracle: 121 cycles over 14 steps either way at 256x384, 1e-6)."""
    sc = cb.generate_scene(0, 128, 192, 0.8, 1234)
    from campfire_b200.fluid import load_scene
    cyc = {}
    for mode in (True, "pipelined"):
        g = cb.FluidSim(0, {"nx": 128, "ny": 192, "dt": sc["dt"]}, width=0.8).init()
        load_scene(g, sc)
        g.set_solver(cb.SOLVE_FP64, 1, 1e-6, 100)
        g.set_krylov(True)
        g.set_coarse_solve(mode)
        c = 0
        for k in range(8):
            g.step(1)
            g.synchronize()
            c += g.info()["last_cycles"]
        cyc[mode] = c
        g.close()
    assert abs(cyc["pipelined"] - cyc[True]) <= 2, cyc
