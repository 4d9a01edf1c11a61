"""CFL steps driven like the app's frame loop: cfg_write_params before every step keeps the
device's CFL dt (the step leaves a copy of it behind an event), so graph and stream
launches give the same bits, and the dt the host sees is the one the step chose."""
import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu


def _run(graphs, steps=4):
    sc = cb.generate_scene(0, 96, 144, 0.8, 77)
    g = cb.FluidSim(0, {"nx": 96, "ny": 144, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    g.set_solver(cb.SOLVE_FP64, 1, 1e-8, 100)
    g.set_cfl(0.5, 2e-3)
    g.set_graphs(graphs)
    dts = []
    for _ in range(steps):
        g.writeParams()
        dts.append(g.info()["dt"])
        g.step(1)
    g.synchronize()
    out = {f: g.readBuffer(f) for f in ("T", "U", "V")}
    # the clock: the sum of the dt each step used, kept on the device (and by the Python mirror)
    t = 0.0
    for d in dts:
        t += d
    assert g.info()["time"] == t and g.time == t
    g.close()
    return out, dts


def test_write_params_keeps_the_cfl_dt_in_graph_and_stream_launches():
    a, da = _run(True)
    b, db = _run(False)
    assert da == db
    assert all(0 < d <= 2e-3 + 1e-12 for d in da[1:])   # the steps' CFL dt, capped at 2 ms
    for f in ("T", "U", "V"):
        assert np.array_equal(a[f], b[f]), f


def _cfl_dt(sim, cfl, cap):
    """dt = min(cap, cfl dx / max|u|) from the scene's own faces, in the device's f32 arithmetic."""
    m = np.float32(max(np.abs(sim.readBuffer("U")).max(), np.abs(sim.readBuffer("V")).max()))
    dx = np.float32(sim.info()["dx"])
    cand = np.float32(np.float32(cfl) * dx) / m if m > 0 else np.float32(cap)
    return float(min(np.float32(cap), cand))


def test_cfl_dt_per_scene_with_a_scene_disabled_and_reenabled():
    """Two CFL scenes in a batch: each step sets each enabled scene's dt from its own max|u|; a scene
    disabled for a step keeps its dt and its clock; cfg_write_params (the app calls it every frame)
    leaves the device's dt as the step set it; after re-enabling, the rule holds again."""
    dims = [(96, 144), (64, 96)]
    scenes = [cb.generate_scene(0, nx, ny, 0.8, 300 + k) for k, (nx, ny) in enumerate(dims)]
    b = cb.Batch(dims, 0.8, [s["dt"] for s in scenes])
    for v, s in zip(b.scenes, scenes):
        load_scene(v, s)
        v.set_cfl(0.5, 2e-3)
    b.set_solver(cb.SOLVE_FP64, 1, 1e-8, 100)
    b.step(3)
    b.synchronize()
    for v in b.scenes:
        assert v.info()["dt"] == _cfl_dt(v, 0.5, 2e-3)
    one = b.scenes[1]
    kept = (one.info()["dt"], one.info()["time"])
    b.set_active(1, False)
    b.step(1)
    b.synchronize()
    assert (one.info()["dt"], one.info()["time"]) == kept
    assert b.scenes[0].info()["dt"] == _cfl_dt(b.scenes[0], 0.5, 2e-3)
    b.set_active(1, True)
    for v in b.scenes:
        before = v.info()["dt"]
        v.writeParams()
        assert v.info()["dt"] == before
    b.step(2)
    b.synchronize()
    for v in b.scenes:
        assert v.info()["dt"] == _cfl_dt(v, 0.5, 2e-3)
    t1 = one.info()["time"]
    assert t1 > kept[1]
    b.close()
