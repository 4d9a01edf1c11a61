"""The smoother schedule (where the one-CTA coarse block starts) and its autotuner.

The fused V-cycle reads exactly the values the reference dispatches read at
every level, whichever kernel runs the level, so every schedule gives the same
bits; the autotuner only picks the fastest.
"""
import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu


def run(nx, ny, cells, mode, steps=2, direct=False):
    sc = cb.generate_scene(0, nx, ny, 0.8, 1235)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    g.set_solver(mode, 2, 1e-8, 60)
    g.set_coarse_solve(direct)
    if cells:
        g.set_coarse_cells(cells)
    g.step(steps)
    out = {f: g.readBuffer(f) for f in ("T", "Y", "U", "V", "p")}
    out["p64"] = g.read_p64()
    out["cycles"] = g.info()["last_cycles"]
    g.close()
    return out


@pytest.mark.parametrize("mode,direct", [(cb.SOLVE_FIXED, False), (cb.SOLVE_FP64, False), (cb.SOLVE_FP64, True)])
def test_every_schedule_gives_the_same_bits(mode, direct):
    ref = run(256, 384, None, mode, direct=direct)
    for cells in (24576, 1536, 384, 96):
        got = run(256, 384, cells, mode, direct=direct)
        assert got["cycles"] == ref["cycles"], cells
        for f in ("T", "Y", "U", "V", "p", "p64"):
            assert np.array_equal(got[f], ref[f]), (cells, f)


def test_autotuner_times_the_candidates():
    r = cb.autotune([(256, 384)], iters=5)
    assert r["best"] in r["ms_per_cycle"]
    assert len(r["ms_per_cycle"]) >= 3
    assert all(v > 0 for v in r["ms_per_cycle"].values())
    rb = cb.autotune([(96, 144), (256, 384), (128, 192)], iters=3, coarse_direct=True)
    assert rb["best"] > 0
