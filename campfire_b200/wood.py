"""The campfire app's wood model and frame coupling around the gas step, through
the C ABI (cfg_wood_*): WoodPiece mirrors js/wood.js's class, WoodScene the
frame loop of js/main.js for pieces frozen in place."""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from ._lib import CfgWoodPiece, check


def _d4(v):
    return (ctypes.c_double * 4)(*[float(x) for x in v])


class WoodPiece:
    """new WoodPiece(side, rhoV, T0) of js/wood.js; fields as attributes (Ts, Tp, d, ...)."""

    def __init__(self, side: float, rhoV: float, T0: float = 293.15):
        self._s = CfgWoodPiece()
        check(_lib.lib().cfg_wood_piece_init(ctypes.byref(self._s), side, rhoV, T0))

    def __getattr__(self, name):
        s = object.__getattribute__(self, "_s")
        v = getattr(s, name)
        return list(v) if isinstance(v, ctypes.Array) else v

    @property
    def half(self):
        return 0.5 * self._s.side

    @property
    def dead(self):
        return bool(self._s.dead)

    def set_exposure(self, ex):
        for f in range(4):
            self._s.exposure[f] = ex[f]

    def preheat(self, Tsurf, charDepth, Tcore, charYield=0.25):
        check(_lib.lib().cfg_wood_piece_preheat(ctypes.byref(self._s), Tsurf, charDepth, Tcore, charYield))

    def step(self, dt, qConv, qInc, charBurnt, charYield=0.25, pyroMult=1.0):
        check(_lib.lib().cfg_wood_piece_step(ctypes.byref(self._s), dt, _d4(qConv), _d4(qInc), _d4(charBurnt),
                                             charYield, pyroMult))


class WoodScene:
    """The pieces of a FluidSim and the per-frame coupling (cfg_wood_frame)."""

    def __init__(self, sim, charYield: float = 0.25, pyroMult: float = 1.0, rigid=None):
        """rigid: None for pieces frozen in place, or the rigid world's options (app_rigid_options()
        for the app's world) for moving pieces."""
        h = ctypes.c_void_p()
        check(_lib.lib().cfg_wood_create(sim._h, charYield, pyroMult, ctypes.byref(h)))
        self._h = h.value
        self._world = None
        if rigid is not None:
            from .rigid import to_params
            check(_lib.lib().cfg_wood_set_rigid(self._h, ctypes.byref(to_params(dict(rigid)))))

    @property
    def world(self):
        """The scene's RigidWorld (moving pieces), or None."""
        if self._world is None:
            from .rigid import RigidWorld
            h = ctypes.c_void_p()
            rc = _lib.lib().cfg_wood_rigid(self._h, ctypes.byref(h))
            if rc == -2:
                return None
            check(rc)
            self._world = RigidWorld(_handle=h.value)
        return self._world

    def body(self, slot: int):
        """The rigid body of a moving piece."""
        i = ctypes.c_int()
        check(_lib.lib().cfg_wood_body(self._h, slot, ctypes.byref(i)))
        return self.world.body(i.value) if i.value else None

    def close(self):
        if self._h:
            self._world = None
            _lib.lib().cfg_wood_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, x, y, angle, side, density=500.0, preheat=None, faceT=None) -> int:
        slot = ctypes.c_int()
        pre = (ctypes.c_double * 3)(*preheat) if preheat else None
        ft = _d4(faceT) if faceT else None
        check(_lib.lib().cfg_wood_add(self._h, x, y, angle, side, density, pre, ft, ctypes.byref(slot)))
        return slot.value

    def remove(self, slot: int):
        check(_lib.lib().cfg_wood_remove(self._h, slot))

    def frame(self, sim_dt: float) -> int:
        n = ctypes.c_int()
        check(_lib.lib().cfg_wood_frame(self._h, sim_dt, ctypes.byref(n)))
        return n.value

    def set_readback_lag(self, lag: int):
        """0: synchronous readback; < 0: through the ring, applied when arrived (the reference);
        1..3: applied exactly `lag` frames later (cfg_wood_set_readback_lag)."""
        check(_lib.lib().cfg_wood_set_readback_lag(self._h, lag))

    def readbacks(self) -> dict:
        a, k = ctypes.c_uint64(), ctypes.c_uint64()
        check(_lib.lib().cfg_wood_readbacks(self._h, ctypes.byref(a), ctypes.byref(k)))
        return {"applied": a.value, "skipped": k.value}

    def piece(self, slot: int):
        """(state dict, qConv[4], qInc[4]) or None for an empty slot."""
        st = CfgWoodPiece()
        qc, qi = (ctypes.c_double * 4)(), (ctypes.c_double * 4)()
        rc = _lib.lib().cfg_wood_get(self._h, slot, ctypes.byref(st), qc, qi)
        if rc == -2:
            return None
        check(rc)
        d = {k: (list(getattr(st, k)) if isinstance(getattr(st, k), ctypes.Array) else getattr(st, k))
             for k, _ in CfgWoodPiece._fields_ if k != "pad"}
        return d, list(qc), list(qi)

    def set_piece(self, slot: int, state: dict):
        """Replace a piece's wood state (keys of piece()'s state dict; missing keys keep their value)."""
        cur = self.piece(slot)
        if cur is None:
            raise _lib.CampfireError(-2, "no piece in this slot")
        st = dict(cur[0], **state)
        c = CfgWoodPiece()
        for k, _ in CfgWoodPiece._fields_:
            if k == "pad":
                continue
            v = st[k]
            if isinstance(getattr(c, k), ctypes.Array):
                getattr(c, k)[:] = [float(x) for x in v]
            else:
                setattr(c, k, int(v) if k == "dead" else float(v))
        check(_lib.lib().cfg_wood_set(self._h, slot, ctypes.byref(c)))

    def render_data(self) -> np.ndarray:
        """The renderer's wood buffer (64 x 12 float32) of the last upload (js/main.js:188-207)."""
        out = np.zeros(64 * 12, np.float32)
        check(_lib.lib().cfg_wood_render_data(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def stats(self):
        h, r, t = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        check(_lib.lib().cfg_wood_stats(self._h, ctypes.byref(h), ctypes.byref(r), ctypes.byref(t)))
        return {"hrr": h.value, "rad": r.value, "tmax": t.value}


SCENE_WIDTH = 0.7   # js/config.js:3


def app_rigid_options(friction: float = 0.7) -> dict:
    """The app's rigid world: walls at the scene width (js/main.js:61) and the friction control
    (applyControls, :93-94)."""
    return {"width": SCENE_WIDTH, "muStatic": friction, "muKinetic": 0.75 * friction}


def default_scene(ws: WoodScene, char_yield: float = 0.25, density: float = 500.0) -> list:
    """The app's pre-lit fire (defaultScene, js/main.js:132-155): a bed of seven glowing coals,
    two logs flanking it and seven sticks piled on it. Returns the slots."""
    cx, S = SCENE_WIDTH / 2, 0.0125
    slots = []

    def coal(x, y, sz, T):
        s = ws.add(x, y, 0.0, sz, density, preheat=(T, sz, T - 30))
        st, _, _ = ws.piece(s)
        mc = st["rhoC"] * sz * sz
        side = math.sqrt(0.0 / st["rhoV"] + mc / st["rhoC"])     # WoodPiece.updateSide with mv = 0
        ws.set_piece(s, {"mv": 0.0, "mc": mc, "side": side, "d": [sz / 2] * 4, "charCov": [1.0] * 4,
                         "Tp": [T - 20] * 4})
        b = ws.body(s) if ws.world is not None else None
        if b is not None:   # p.body.density = w.mc / (sz * sz); world.resize(p.body, w.half)
            b.density = mc / (sz * sz)
            ws.world.resize(b, 0.5 * side)
        slots.append(s)

    def lit(x, y, sz):
        s = ws.add(x, y, 0.0, sz, density, preheat=(880.0, 0.003 if sz > 0.03 else 0.002, 380.0))
        ws.set_piece(s, {"Tp": [590.0] * 4})
        slots.append(s)

    x = cx - 0.06
    for sz in (0.016, 0.02, 0.015, 0.018, 0.02, 0.016, 0.017):
        coal(x + sz / 2, sz / 2, sz, 1050.0)
        x += sz + 0.0015
    lit(cx - 0.093, 0.025, 0.05)
    lit(cx + 0.093, 0.025, 0.05)
    y1 = 0.02 + S + 0.001
    for dx in (-0.045, -0.016, 0.013, 0.042):
        lit(cx + dx, y1, 0.025)
    for dx in (-0.03, 0.0, 0.028):
        lit(cx + dx, y1 + 2 * S + 0.002, 0.025)
    return slots
