"""The pressure loop's W tail (cfg_set_coarse_w): a cycle shape of the library's FP64 loop, not
of the reference (whose V(2,2) cycle, js/fluid.js:294-312, stays the default). The level two
above the coarsest, when it has at most W cells, visits the level below it twice per cycle,
inside the one-CTA coarse block; the oracle's solve loop runs the same cycle (oracle/gas_ref.hpp,
cycle_at). Checked here: parity with the oracle from the same state, fewer cycles than the
V-cycle on a tepee scene on both sides, results independent of the coarse block's start level,
a batch's scenes equal to the same scenes alone, and the setting's errors.
"""
import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene
from conftest import norm_err

pytestmark = pytest.mark.gpu

W = 1536


def _setup(sim, w, tol=1e-10):
    sim.set_solver(cb.SOLVE_FP64, 1, tol, 300)
    sim.set_coarse_solve("pipelined")
    sim.set_krylov(True)
    sim.set_coarse_w(w)


def _gpu(nx, ny, kind, seed, w, coarse_cells=1536, warm=3):
    sc = cb.generate_scene(kind, nx, ny, 0.8, seed)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    g.set_coarse_cells(coarse_cells)
    _setup(g, w)
    g.step(warm)
    return g, sc


@pytest.mark.parametrize("nx,ny", [(128, 192), (256, 384)])
def test_w_cycle_matches_oracle(oracle_mod, nx, ny):
    """From the GPU's state, two steps on both sides: fields within 1e-4, cycles within two
    (the GPU's pipelined inverse comes from its own previous step), both to 1e-10."""
    g, sc = _gpu(nx, ny, 1, 1240, W)
    o = oracle_mod.OracleSim(nx, ny, 0.8, sc["dt"])
    load_scene(o, sc)
    _setup(o, W)
    o.copy_state_from(g)
    for k in range(2):
        g.step(1)
        o.step(1)
        gi, oi = g.info(), o.info()
        assert gi["last_rel"] <= 1e-10 and oi["last_rel"] <= 1e-10, (k, gi["last_rel"], oi["last_rel"])
        assert abs(gi["last_cycles"] - oi["last_cycles"]) <= 2, (k, gi["last_cycles"], oi["last_cycles"])
        for f in ("T", "Y", "U", "V"):
            assert norm_err(g.readBuffer(f), o.read(f)) <= 1e-4, (k, f)
        assert norm_err(g.read_p64(), o.read("p64")) <= 1e-4
    g.close()


def test_w_cycle_needs_fewer_cycles_on_the_tepee(oracle_mod):
    """128x192 tepee, 1e-10: the W tail (its level has 1536 cells) saves cycles on the GPU and on the
    oracle alike, and the converged pressures agree (the solve's tolerance)."""
    cyc, p = {}, {}
    for w in (0, W):
        g, sc = _gpu(128, 192, 1, 1241, w, warm=2)
        c = []
        for _ in range(3):
            g.step(1)
            c.append(g.info()["last_cycles"])
        cyc[w], p[w] = c, g.read_p64()
        g.close()
    assert sum(cyc[W]) < sum(cyc[0]), cyc
    assert norm_err(p[W], p[0]) <= 1e-6
    oc = {}
    for w in (0, W):
        sc = cb.generate_scene(1, 128, 192, 0.8, 1241)
        o = oracle_mod.OracleSim(128, 192, 0.8, sc["dt"])
        load_scene(o, sc)
        _setup(o, w)
        o.step(5)
        oc[w] = o.info()["last_cycles"]
    assert oc[W] < oc[0], oc


def test_w_cycle_does_not_depend_on_the_coarse_block_start():
    """The W tail's level always runs inside the coarse block, and a level gives the same bits in the
    block and in the tiled kernels: starting the block at 384, 1536 or 6144 cells changes nothing."""
    hashes = []
    for cells in (384, 1536, 6144):
        g, sc = _gpu(128, 192, 1, 1242, W, coarse_cells=cells, warm=3)
        hashes.append((cb.field_hash(g), g.read_p64().tobytes(), g.info()["last_cycles"]))
        g.close()
    assert hashes[0] == hashes[1] == hashes[2]


def test_w_cycle_batch_matches_single_scenes():
    """A batch of scenes of three sizes with the W tail: each scene's bits equal the scene stepped
    alone (its decision, its cycle count, its block's cycle are its own)."""
    dims = [(128, 192), (96, 144), (192, 288)]
    scenes = [cb.generate_scene(1, nx, ny, 0.8, 1250 + k) for k, (nx, ny) in enumerate(dims)]
    b = cb.Batch(dims, 0.8, [s["dt"] for s in scenes])
    for v, s in zip(b.scenes, scenes):
        load_scene(v, s)
    b.set_solver(cb.SOLVE_FP64, 1, 1e-10, 300)
    b.set_coarse_solve("pipelined")
    b.set_krylov(2)
    b.set_coarse_cells(1536)
    b.set_coarse_w(W)
    b.step(3)
    b.synchronize()
    got = [(cb.field_hash(v), v.info()["last_cycles"]) for v in b.scenes]
    b.close()
    for (nx, ny), s, (h, c) in zip(dims, scenes, got):
        g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": s["dt"]}, width=0.8).init()
        load_scene(g, s)
        g.set_coarse_cells(1536)
        _setup(g, W)
        g.set_krylov(2)
        g.step(3)
        assert (cb.field_hash(g), g.info()["last_cycles"]) == (h, c), (nx, ny)
        g.close()


def test_w_cycle_setting_errors():
    g = cb.FluidSim(0, {"nx": 64, "ny": 96, "dt": 1e-3}, width=0.8).init()
    with pytest.raises(cb.CampfireError, match="INVAL"):
        g.set_coarse_w(-1)
    g.set_coarse_w(W)
    with pytest.raises(cb.CampfireError, match="INVAL"):
        g.set_coarse_cluster(4)   # the W tail runs in the one-CTA block only
    g.set_coarse_w(0)
    g.set_coarse_cluster(4)
    with pytest.raises(cb.CampfireError, match="INVAL"):
        g.set_coarse_w(W)
    g.set_coarse_cluster(0)
    g.set_coarse_w(W)
    g.close()
