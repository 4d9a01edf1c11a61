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
    g.close()
    return out, dts


def test_write_params_keeps_the_cfl_dt_in_graph_and_stream_launches():
    a, da = _run(True)
    b, db = _run(False)
    assert da == db
    assert all(0 < d <= 2e-3 + 1e-12 for d in da[1:])   # the steps' CFL dt, capped at 2 ms
    for f in ("T", "U", "V"):
        assert np.array_equal(a[f], b[f]), f
