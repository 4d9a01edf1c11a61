"""Checkpoint / resume of a scene (cfg_checkpoint_save / cfg_checkpoint_load).

A scene saved after k steps and loaded into a fresh scene (or a batch slot) of the
same grid size continues bit for bit: the state after k + m steps equals that of
an uninterrupted run (FNV-1a hashes of T, Y, U, V and the FP64 pressure).
"""
import os

import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu


def make(nx, ny, sc, dt=None, coarse=True):
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": dt or sc["dt"]}, width=0.8).init()
    g.set_solver(cb.SOLVE_FP64, 1, 1e-9, 100)
    g.set_coarse_solve(coarse)
    return g


def state(g):
    return cb.field_hash(g), g.read_p64().tobytes()


@pytest.mark.parametrize("cfl,coarse", [(0.0, True), (0.5, True), (0.0, "pipelined")])
def test_resume_is_bit_exact(tmp_path, cfl, coarse):
    # pipelined: the inverse factored during the last saved step is part of the state
    nx, ny = 96, 144
    sc = cb.generate_scene(1, nx, ny, 0.8, 4321)
    a = make(nx, ny, sc, coarse=coarse)
    load_scene(a, sc)
    if cfl:
        a.set_cfl(cfl, sc["dt"])
    a.step(6)
    ref = state(a)
    b = make(nx, ny, sc, coarse=coarse)
    load_scene(b, sc)
    if cfl:
        b.set_cfl(cfl, sc["dt"])
    b.step(3)
    path = str(tmp_path / "scene.ckpt")
    b.save_checkpoint(path)
    b.close()
    c = make(nx, ny, sc, dt=0.001, coarse=coarse)   # another dt and an empty state: all of it comes from the file
    if cfl:
        c.set_cfl(cfl, sc["dt"])
    c.load_checkpoint(path)
    assert abs(c.info()["time"] - 3 * a.info()["dt"]) < 1e-9 or cfl
    c.step(3)
    assert state(c) == ref
    a.close(); c.close()


def test_resume_into_a_batch_slot(tmp_path):
    nx, ny = 64, 96
    sc = cb.generate_scene(2, nx, ny, 0.8, 77)
    a = make(nx, ny, sc)
    load_scene(a, sc)
    a.step(2)
    path = str(tmp_path / "a.ckpt")
    a.save_checkpoint(path)
    a.step(2)
    ref = state(a)
    b = cb.Batch([(96, 144), (nx, ny)], 0.8, [0.002, sc["dt"]])
    b.set_solver(cb.SOLVE_FP64, 1, 1e-9, 100)
    b.set_coarse_solve(True)
    load_scene(b.scenes[0], cb.generate_scene(1, 96, 144, 0.8, 5))
    b.scenes[1].load_checkpoint(path)
    b.step(2)
    assert state(b.scenes[1]) == ref
    b.close(); a.close()


def test_bad_checkpoints_are_rejected(tmp_path):
    sc = cb.generate_scene(0, 64, 96, 0.8, 1)
    a = make(64, 96, sc)
    load_scene(a, sc)
    path = str(tmp_path / "s.ckpt")
    a.save_checkpoint(path)
    other = make(96, 144, sc)
    with pytest.raises(cb.CampfireError) as e:
        other.load_checkpoint(path)
    assert e.value.code == -34
    with pytest.raises(cb.CampfireError) as e:
        other.load_checkpoint(str(tmp_path / "missing.ckpt"))
    assert e.value.code == -2
    raw = bytearray(open(path, "rb").read())
    raw[len(raw) // 2] ^= 0xFF
    bad = str(tmp_path / "bad.ckpt")
    open(bad, "wb").write(bytes(raw))
    before = state(a)
    with pytest.raises(cb.CampfireError) as e:
        a.load_checkpoint(bad)
    assert e.value.code == -22
    assert state(a) == before   # a rejected file leaves the scene as it was
    a.close(); other.close()


def test_resumed_scene_matches_oracle(tmp_path, oracle_mod):
    """A checkpoint holds the whole state of a step: loaded into a fresh scene, its next steps equal the
    CPU oracle's from that state (the benchmark's solver: FP64 outer loop by flexible CG, pipelined
    coarsest inverse, CFL step), and the clock and dt come back as saved."""
    from conftest import norm_err
    nx, ny = 128, 192
    sc = cb.generate_scene(0, nx, ny, 0.8, 1234)

    def configure(s):
        s.set_solver(cb.SOLVE_FP64, 1, 1e-8, 200)
        s.set_coarse_solve("pipelined")
        s.set_krylov(True)
        s.set_cfl(0.5, 2e-3)

    a = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(a, sc)
    configure(a)
    a.step(5)
    saved = a.info()
    path = str(tmp_path / "scene.ckpt")
    a.save_checkpoint(path)
    a.close()
    c = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": 1e-3}, width=0.8).init()
    configure(c)
    c.load_checkpoint(path)
    got = c.info()
    assert got["dt"] == saved["dt"] and abs(got["time"] - saved["time"]) <= 1e-12
    o = oracle_mod.OracleSim(nx, ny, 0.8, sc["dt"])
    load_scene(o, sc)
    configure(o)
    o.copy_state_from(c, 0.5, 2e-3)
    for k in range(2):
        c.step(1)
        o.step(1)
        for f in ("T", "Y", "U", "V", "SQ"):
            e = norm_err(c.readBuffer(f), o.read(f))
            assert e <= 1e-4, (k, f, e)
        assert norm_err(c.read_p64(), o.read("p64")) <= 1e-4
    c.close()
