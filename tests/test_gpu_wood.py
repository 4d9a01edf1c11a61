"""The frame coupling of js/main.js (wood step on the last readback, piece upload,
geometry, gas steps, radiation, readback) on the GPU gas step (cfg_wood_frame)
against the oracle's restatement of the same loop over the CPU gas step.

The gas fields agree within 1e-4 per step, so after a frame of ~8 steps the
radiative (T^4) and convective heat inputs of a face agree within a few 1e-3
and the wood state, which integrates them slowly, within 1e-4. The flame
amplifies ulp-level differences (the CPU FP32 restatement itself drifts ~10% in
T from the FP64 oracle within 40 steps), so from the third frame on the face
inputs are compared by their totals per piece and the wood within 1e-3."""
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene
from campfire_b200.wood import WoodScene
from oracle.wood_ref import WoodScene as RefScene

pytestmark = pytest.mark.gpu


def pieces():
    # two preheated logs on the floor and a stick above them (frozen)
    return [(0.33, 0.03, 0.0, 0.05, 500.0, (900.0, 0.004, 500.0)),
            (0.47, 0.03, 0.0, 0.05, 500.0, (900.0, 0.004, 500.0)),
            (0.40, 0.085, 0.3, 0.025, 500.0, None)]


def rel(a, b, floor):
    return abs(a - b) / max(abs(b), floor)


def test_frames_match_the_oracle(oracle_mod):
    nx, ny = 96, 144
    sc = cb.generate_scene(0, nx, ny, 0.8, 4242)
    sc["npieces"] = 0
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    o = oracle_mod.OracleSim(nx, ny, 0.8, sc["dt"])
    load_scene(o, sc)
    ws, rs = WoodScene(g), RefScene(o)
    for p in pieces():
        assert ws.add(*p[:5], preheat=p[5]) == rs.add(*p[:5], preheat=p[5])
    for k in range(6):
        n = ws.frame(1 / 60)
        assert n == rs.frame(1 / 60) and n >= 1
        got = [ws.piece(s) for s in range(3)]
        # heat inputs: error relative to the largest input of the frame (as the field errors)
        sc_c = max(abs(q) for r in rs.slots[:3] for q in r["qConv"])
        sc_i = max(abs(q) for r in rs.slots[:3] for q in r["qInc"])
        early = k < 2
        for s in range(3):
            a, qc, qi = got[s]
            r = rs.slots[s]
            w = r["wood"]
            for f in range(4):
                assert rel(a["Ts"][f], w.Ts[f], 1.0) <= (1e-4 if early else 1e-3), (k, s, f, a["Ts"][f], w.Ts[f])
                if early:
                    assert abs(a["mflux"][f] - w.mflux[f]) <= 1e-3 * max(max(w.mflux), 1e-6), (k, s, f)
                    assert abs(qi[f] - r["qInc"][f]) <= 5e-3 * sc_i, (k, s, f, qi[f], r["qInc"][f])
                    assert abs(qc[f] - r["qConv"][f]) <= 5e-3 * sc_c, (k, s, f, qc[f], r["qConv"][f])
            if not early:   # the flame near the wood has begun to drift: the piece's totals
                assert rel(sum(qi), sum(r["qInc"]), 1.0) <= 3e-2, (k, s)
                assert abs(sum(qc) - sum(r["qConv"])) <= 3e-2 * 4 * sc_c, (k, s)
            assert rel(a["mv"], w.mv, 1e-12) <= 1e-5
    st = ws.stats()
    assert rel(st["hrr"], rs.hrr, 1.0) <= 5e-3
    assert abs(st["tmax"] - rs.tmax) <= 2
    ws.close(); g.close()


def test_slots_and_errors():
    sc = cb.generate_scene(0, 64, 96, 0.8, 1)
    g = cb.FluidSim(0, {"nx": 64, "ny": 96, "dt": sc["dt"]}, width=0.8).init()
    ws = WoodScene(g)
    s0 = ws.add(0.3, 0.03, 0.0, 0.05)
    s1 = ws.add(0.5, 0.03, 0.0, 0.05)
    assert (s0, s1) == (0, 1)
    ws.remove(s0)
    assert ws.piece(s0) is None
    assert ws.add(0.2, 0.03, 0.0, 0.03) == 0
    with pytest.raises(cb.CampfireError):
        ws.remove(7)
    with pytest.raises(cb.CampfireError):
        ws.add(0.2, 0.03, 0.0, -1.0)
    ws.close(); g.close()


def test_default_scene_matches_oracle(oracle_mod):
    """The app's default fire (js/main.js:132-155) set up through cfg_wood_add/cfg_wood_set is the
    oracle's exactly, and its first frames agree as above."""
    from campfire_b200.wood import default_scene
    from oracle.wood_ref import default_scene as ref_default_scene
    nx, ny, dt = 112, 160, 0.004
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": dt}, width=0.7).init()
    g.writeParams()
    g.reset()
    o = oracle_mod.OracleSim(nx, ny, 0.7, dt)
    o.write_params()
    o.reset()
    ws, rs = WoodScene(g), RefScene(o)
    slots = default_scene(ws)
    ref_default_scene(rs)
    assert slots == list(range(16))
    for s in slots:
        a = ws.piece(s)[0]
        w = rs.slots[s]["wood"]
        for k in ("side", "mv", "mc", "Tc", "rhoV", "rhoC"):
            assert a[k] == getattr(w, k), (s, k)
        for k in ("Ts", "Tp", "d", "charCov"):
            assert a[k] == [float(v) for v in getattr(w, k)], (s, k)
    for k in range(2):
        assert ws.frame(1 / 60) == rs.frame(1 / 60)
        for s in slots:
            a = ws.piece(s)[0]
            w = rs.slots[s]["wood"]
            for f in range(4):
                assert rel(a["Ts"][f], w.Ts[f], 1.0) <= 1e-4, (k, s, f)
            assert rel(a["mc"], w.mc, 1e-12) <= 1e-5
    ws.close(); g.close()


def test_moving_pieces_match_oracle(oracle_mod):
    """Moving pieces (js/rigid.js world in the frame, js/contact.js heat exchange): a stick dropped
    on two preheated logs. The bodies depend on the gas only through the wood's size and mass, so
    they agree with the oracle's to 1e-9 m over these frames; the wood as in the frozen case."""
    from campfire_b200.wood import app_rigid_options
    from oracle.rigid_ref import RigidWorld as RefWorld
    nx, ny, dt = 112, 160, 0.004
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": dt}, width=0.7).init()
    g.writeParams()
    g.reset()
    o = oracle_mod.OracleSim(nx, ny, 0.7, dt)
    o.write_params()
    o.reset()
    opts = app_rigid_options()
    ws = WoodScene(g, rigid=opts)
    rs = RefScene(o, world=RefWorld(**opts))
    for sc in (ws, rs):
        sc.add(0.30, 0.025, 0.0, 0.05, 500.0, preheat=(950.0, 0.004, 450.0))
        sc.add(0.40, 0.025, 0.0, 0.05, 500.0, preheat=(950.0, 0.004, 450.0))
        sc.add(0.35, 0.09, 0.4, 0.025, 500.0)
    y0 = ws.body(2).y
    for k in range(15):
        assert ws.frame(1 / 60) == rs.frame(1 / 60)
        for s in range(3):
            b, rb = ws.body(s), rs.slots[s]["body"]
            for f in ("x", "y", "a"):
                assert abs(getattr(b, f) - getattr(rb, f)) <= 1e-9, (k, s, f, getattr(b, f), getattr(rb, f))
            a = ws.piece(s)[0]
            w = rs.slots[s]["wood"]
            for f in range(4):
                assert rel(a["Ts"][f], w.Ts[f], 1.0) <= 1e-3, (k, s, f, a["Ts"][f], w.Ts[f])
    stick = ws.body(2)
    assert stick.y < y0 - 0.01                       # it fell
    assert ws.world.contacts()[0] >= 4               # and rests on the logs (floor + log contacts)
    assert abs(stick.vy) < 0.05
    ws.close(); g.close()


def test_lagged_readbacks_match_the_oracle(oracle_mod):
    """The reference applies each frame's readback when it arrives, frames later (afterSubmit's tag,
    js/fluid.js:327-342, onReadback js/main.js:210-230). With a fixed lag of two frames the GPU loop
    (readback ring, cfg_wood_set_readback_lag) and the oracle's loop apply the same readbacks at the
    same frames, with their own frames' gas time; a piece removed meanwhile does not receive its old
    slot's data."""
    nx, ny = 96, 144
    sc = cb.generate_scene(0, nx, ny, 0.8, 4242)
    sc["npieces"] = 0
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    o = oracle_mod.OracleSim(nx, ny, 0.8, sc["dt"])
    load_scene(o, sc)
    ws, rs = WoodScene(g), RefScene(o, lag=2)
    ws.set_readback_lag(2)
    for p in pieces():
        assert ws.add(*p[:5], preheat=p[5]) == rs.add(*p[:5], preheat=p[5])
    for k in range(5):
        if k == 3:   # replace the stick: its old slot's readbacks in flight must not reach the new one
            ws.remove(2)
            rs.slots[2] = None
            p = (0.41, 0.09, 0.0, 0.02, 500.0, None)
            assert ws.add(*p[:5]) == rs.add(*p[:5]) == 2
        assert ws.frame(1 / 60) == rs.frame(1 / 60)
        sc_c = max(abs(q) for r in rs.slots[:3] for q in r["qConv"]) or 1.0
        for s in range(3):
            a, qc, qi = ws.piece(s)
            r = rs.slots[s]
            w = r["wood"]
            for f in range(4):
                assert rel(a["Ts"][f], w.Ts[f], 1.0) <= 1e-4, (k, s, f, a["Ts"][f], w.Ts[f])
                assert abs(qc[f] - r["qConv"][f]) <= 5e-3 * sc_c, (k, s, f, qc[f], r["qConv"][f])
    assert ws.readbacks() == {"applied": 3, "skipped": 0}   # frames 0-2 applied at the starts of 2-4
    ws.close(); g.close()


def test_readbacks_applied_when_they_arrive():
    """lag < 0, the reference's own timing: frames never wait for the GPU, every readback is applied
    once, in order, or skipped while the ring is full; switching back to the synchronous mode delivers
    the rest. Paced like the app (a frame every 8 ms, js/main.js's requestAnimationFrame), the GPU keeps
    up and nearly every readback is applied, a frame or so late."""
    import time
    from campfire_b200.wood import default_scene
    g = cb.FluidSim(0, {"nx": 224, "ny": 320, "dt": 0.003}, width=0.7).init()
    g.writeParams()
    g.reset()
    ws = WoodScene(g)
    default_scene(ws)
    ws.set_readback_lag(-1)
    frames = 40
    for _ in range(frames):
        t0 = time.perf_counter()
        ws.frame(1 / 60)
        assert time.perf_counter() - t0 < 0.5       # the frame enqueues its work; it does not wait for it
        time.sleep(max(0.0, 0.008 - (time.perf_counter() - t0)))
    ws.set_readback_lag(0)
    rb = ws.readbacks()
    assert rb["applied"] + rb["skipped"] == frames and rb["applied"] >= frames - 5, rb
    st = ws.stats()
    assert st["hrr"] > 0 and 1000 < st["tmax"] < 3000, st
    ws.close(); g.close()
