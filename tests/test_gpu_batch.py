"""Batched scenes of uneven size: every kernel serves all scenes in one launch.

The batch must give each scene exactly what the single-scene path gives it
(the kernels compute scenes independently; the only atomics are integer)."""
import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu

DIMS = [(96, 144), (128, 192), (192, 288), (256, 384), (96, 144)]


def _single(sc, mode, tol, steps):
    s = cb.FluidSim(0, {"nx": sc["nx"], "ny": sc["ny"], "dt": sc["dt"]}, width=0.8).init()
    load_scene(s, sc)
    s.set_solver(mode, 2, tol, 60)
    s.step(steps)
    out = {f: s.readBuffer(f) for f in ("T", "Y", "U", "V", "p")}
    out["cycles"] = s.info()["last_cycles"]
    s.close()
    return out


@pytest.mark.parametrize("mode,tol", [(cb.SOLVE_FIXED, 0.0), (cb.SOLVE_TOL, 1e-4), (cb.SOLVE_FP64, 1e-8)])
def test_batch_equals_single_scenes(mode, tol):
    scenes = [cb.generate_scene(2, nx, ny, 0.8, 2000 + k) for k, (nx, ny) in enumerate(DIMS)]
    b = cb.Batch(DIMS, width=0.8, dts=[s["dt"] for s in scenes])
    for v, sc in zip(b.scenes, scenes):
        load_scene(v, sc)
    b.set_solver(mode, 2, tol if tol else 1e-6, 60)
    b.step(3)
    for k, (v, sc) in enumerate(zip(b.scenes, scenes)):
        ref = _single(sc, mode, tol if tol else 1e-6, 3)
        for f in ("T", "Y", "U", "V"):
            assert np.array_equal(v.readBuffer(f), ref[f]), (k, f)
        assert v.info()["last_cycles"] == ref["cycles"]
    b.close()


def test_inactive_scene_is_left_untouched():
    scenes = [cb.generate_scene(2, nx, ny, 0.8, 3000 + k) for k, (nx, ny) in enumerate(DIMS[:3])]
    b = cb.Batch(DIMS[:3], width=0.8, dts=[s["dt"] for s in scenes])
    for v, sc in zip(b.scenes, scenes):
        load_scene(v, sc)
    b.set_solver(cb.SOLVE_TOL, 1, 1e-4, 40)
    before = b.scenes[1].readBuffer("T")
    b.set_active(1, False)
    b.step(2)
    assert np.array_equal(b.scenes[1].readBuffer("T"), before)
    assert not np.array_equal(b.scenes[0].readBuffer("T"), scenes[0]["T"])
    b.set_active(1, True)
    b.step(1)
    assert not np.array_equal(b.scenes[1].readBuffer("T"), before)
    b.close()


def test_batch_krylov_update_folded_matches_its_own_kernel():
    """The Krylov direction update of a batch folded into the level-0 smoother kernels (krylov 2) or
    run as its own kernel per cycle (krylov 3): the same iteration, so the same cycle counts (within
    one: the stopping test's rounding) and pressures to 1e-7. Each cycle ends with one kernel in
    both forms (the folded form's per-scene sums and decision, or the update kernel); the folded
    form adds one launch per step, its last update after the loop."""
    from conftest import norm_err
    dims = [(96, 144), (128, 192), (64, 96)]
    scenes = [cb.generate_scene(2, nx, ny, 0.8, 2100 + k) for k, (nx, ny) in enumerate(dims)]
    out = {}
    for mode in (3, 2):
        b = cb.Batch(dims, 0.8, [s["dt"] for s in scenes])
        for v, s in zip(b.scenes, scenes):
            load_scene(v, s)
        b.set_solver(cb.SOLVE_FP64, 1, 1e-9, 100)
        b.set_coarse_solve("pipelined")
        b.set_coarse_cells(1536)
        b.set_krylov(mode)
        assert b.krylov_folded() == (mode == 2)
        b.step(3)
        b.synchronize()
        out[mode] = ([v.info()["last_cycles"] for v in b.scenes], [v.read_p64() for v in b.scenes],
                     [{f: v.readBuffer(f) for f in ("T", "U", "V")} for v in b.scenes], b.launch_count())
        b.close()
    for k in range(len(dims)):
        assert abs(out[2][0][k] - out[3][0][k]) <= 1, (k, out[2][0], out[3][0])
        assert norm_err(out[2][1][k], out[3][1][k]) <= 1e-7, k
        for f in ("T", "U", "V"):
            assert norm_err(out[2][2][k][f], out[3][2][k][f]) <= 1e-6, (k, f)
    if out[2][0][0] == out[3][0][0]:   # launches per step are counted with scene 0's cycles
        assert out[2][3] == out[3][3] + 1, (out[2][3], out[3][3])


def test_krylov_fold_needs_every_coarse_block_below_level_0():
    """The fold asked for (krylov 2) runs only while every scene's coarse block starts below level 0:
    a coarse block that covers a scene's level 0 falls back to the update kernel, and says so."""
    dims = [(96, 144), (64, 96)]
    b = cb.Batch(dims, 0.8, [1e-3, 1e-3])
    b.set_solver(cb.SOLVE_FP64, 1, 1e-9, 100)
    b.set_krylov(2)
    b.set_coarse_cells(1536)
    assert b.krylov_folded()
    b.set_coarse_cells(6144)          # 64x96 is 6144 cells: its whole hierarchy in the block
    assert not b.krylov_folded()
    b.set_krylov(3)
    b.set_coarse_cells(1536)
    assert not b.krylov_folded()
    b.close()
