"""Tile shapes of the advection, diffusion + sources and forces kernels (cfg_set_tiles) and
their autotuner (cfg_autotune_tiles). A cell's arithmetic does not depend on the tile it
falls in, and the 8x8 blocks of the heat-release reduction (sources.wgsl:160-172) stay whole
in every shape, so every shape must give the same bits, for single scenes and uneven batches,
with 1, 3 and 5 diffusion sub-steps (5: the widest halo, the largest shared-memory footprint)."""
import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu

SHAPES = [(0, 0, 0), (1, 1, 1), (2, 2, 2), (1, 2, 0), (2, 0, 1)]


def _single(shape, nx, ny, dt=None, steps=3):
    sc = cb.generate_scene(0, nx, ny, 0.8, 1234)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": dt or sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    if dt:
        g.set_dt(dt)
        g.writeParams()
    g.set_solver(cb.SOLVE_FIXED, 2)
    g.set_tiles(*shape)
    g.step(steps)
    out = (cb.field_hash(g), g.readback()["acc"].tobytes(), g.info()["diffSub"])
    g.close()
    return out


@pytest.mark.parametrize("nx,ny,dt,sub", [(128, 192, None, 1), (384, 576, 0.0035, 3), (192, 288, 0.03, 5)])
def test_tile_shapes_give_the_same_bits(nx, ny, dt, sub):
    ref = _single(SHAPES[0], nx, ny, dt)
    assert ref[2] == sub
    for shape in SHAPES[1:]:
        assert _single(shape, nx, ny, dt) == ref, shape


def test_tile_shapes_in_an_uneven_batch():
    dims = [(96, 144), (128, 192), (64, 96)]
    scenes = [cb.generate_scene(2, nx, ny, 0.8, 2000 + k) for k, (nx, ny) in enumerate(dims)]
    res = []
    for shape in SHAPES[:3]:
        b = cb.Batch(dims, 0.8, [s["dt"] for s in scenes])
        for v, s in zip(b.scenes, scenes):
            load_scene(v, s)
        b.set_solver(cb.SOLVE_FP64, 1, 1e-8, 100)
        b.set_tiles(*shape)
        b.step(3)
        b.synchronize()
        res.append([cb.field_hash(v) for v in b.scenes])
        b.close()
    assert res[1] == res[0] and res[2] == res[0]


def test_autotuner_picks_valid_shapes():
    t = cb.autotune_tiles([(256, 384)], iters=5)
    assert all(0 <= s < 3 for s in t["best"])
    for k, ms in t["ms"].items():
        assert all(m > 0 for m in ms), (k, ms)
        assert ms[t["best"][("advect", "diffuse_sources", "forces").index(k)]] == min(ms)
