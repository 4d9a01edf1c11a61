"""The campfire app's 2D rigid bodies (js/rigid.js) through the C ABI (cfg_rigid_*).

    w = RigidWorld({"width": 0.7})
    b = w.add(Body(0.35, 0.0125, 0.0125, 500))
    w.advance(1 / 60)
    print(b.x, b.y, b.a)

`Body` objects are handles: their fields read the world's current state. The
world runs on the host in double precision (no GPU needed).
"""
from __future__ import annotations

import ctypes

from . import _lib
from ._lib import CfgRigidBody, CfgRigidParams, check

_KEYS = {"gravity": "gravity", "width": "width", "dt": "dt", "substeps": "substeps", "slop": "slop",
         "contactHertz": "contact_hertz", "contactDamping": "contact_damping", "maxPushout": "max_pushout",
         "muStatic": "mu_static", "muKinetic": "mu_kinetic", "stickSpeed": "stick_speed", "maxSpeed": "max_speed",
         "dragHertz": "drag_hertz", "dragStrength": "drag_strength"}


def defaults() -> dict:
    """RIGID_DEFAULTS (js/rigid.js:12-27) with the reference's option names."""
    p = CfgRigidParams()
    check(_lib.lib().cfg_rigid_defaults(ctypes.byref(p)))
    return {k: (list(getattr(p, c)) if k == "gravity" else getattr(p, c)) for k, c in _KEYS.items()}


def to_params(opts: dict) -> CfgRigidParams:
    p = CfgRigidParams()
    check(_lib.lib().cfg_rigid_defaults(ctypes.byref(p)))
    for k, v in opts.items():
        if k not in _KEYS:
            raise KeyError(f"unknown rigid option {k}")
        if k == "gravity":
            p.gravity[0], p.gravity[1] = float(v[0]), float(v[1])
        elif k == "substeps":
            p.substeps = int(v)
        else:
            setattr(p, _KEYS[k], float(v))
    return p


class Body:
    """A square piece: new Body(x, y, half, density, angle) (js/rigid.js:40-49). Added to a world
    with RigidWorld.add; afterwards its attributes read the world's state."""

    def __init__(self, x, y, half, density, angle=0.0):
        self._init = (float(x), float(y), float(half), float(density), float(angle))
        self.world = None
        self.id = 0

    def _state(self) -> CfgRigidBody:
        b = CfgRigidBody()
        check(_lib.lib().cfg_rigid_get(self.world._h, self.id, ctypes.byref(b)))
        return b

    def __getattr__(self, name):
        if name in ("x", "y", "a", "vx", "vy", "w", "half", "density", "mass"):
            if self.world is None:
                x, y, half, density, angle = self._init
                return {"x": x, "y": y, "a": angle, "vx": 0.0, "vy": 0.0, "w": 0.0, "half": half,
                        "density": density, "mass": density * (2 * half) ** 2}[name]
            return getattr(self._state(), name)
        if name == "drag":
            return bool(self._state().dragging) if self.world is not None else False
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name == "density" and self.__dict__.get("world") is not None:
            check(_lib.lib().cfg_rigid_set_density(self.world._h, self.id, float(value)))
            return
        object.__setattr__(self, name, value)


class RigidWorld:
    """RigidWorld of js/rigid.js:159-468 (options as RIGID_DEFAULTS' keys)."""

    def __init__(self, opts: dict | None = None, _handle=None):
        if _handle is not None:
            self._h, self._own = _handle, False
        else:
            h = ctypes.c_void_p()
            check(_lib.lib().cfg_rigid_create(ctypes.byref(to_params(opts or {})), ctypes.byref(h)))
            self._h, self._own = h.value, True
        self._bodies = {}

    def close(self):
        if self._h and self._own:
            _lib.lib().cfg_rigid_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def p(self) -> dict:
        c = CfgRigidParams()
        check(_lib.lib().cfg_rigid_get_params(self._h, ctypes.byref(c)))
        return {k: (list(getattr(c, n)) if k == "gravity" else getattr(c, n)) for k, n in _KEYS.items()}

    def set_params(self, **opts):
        cur = self.p
        cur.update(opts)
        check(_lib.lib().cfg_rigid_set_params(self._h, ctypes.byref(to_params(cur))))

    def add(self, body: Body) -> Body:
        x, y, half, density, angle = body._init
        i = ctypes.c_int()
        check(_lib.lib().cfg_rigid_add(self._h, x, y, half, density, angle, ctypes.byref(i)))
        body.world, body.id = self, i.value
        self._bodies[i.value] = body
        return body

    def body(self, id_: int) -> Body:
        """The handle of a body by id (bodies the world made itself, e.g. a wood scene's)."""
        if id_ not in self._bodies:
            b = Body(0, 0, 1, 1)
            b.world, b.id = self, id_
            self._bodies[id_] = b
        return self._bodies[id_]

    def remove(self, body: Body):
        check(_lib.lib().cfg_rigid_remove(self._h, body.id))
        self._bodies.pop(body.id, None)

    def resize(self, body: Body, half: float):
        check(_lib.lib().cfg_rigid_resize(self._h, body.id, float(half)))

    def step(self, dt: float, n: int = 1):
        check(_lib.lib().cfg_rigid_step(self._h, float(dt), int(n)))

    def advance(self, dt: float):
        check(_lib.lib().cfg_rigid_advance(self._h, float(dt)))

    def states(self) -> list:
        """All bodies in world order: dicts of id, x, y, a, vx, vy, w, half, density, mass, dragging."""
        n = ctypes.c_int()
        check(_lib.lib().cfg_rigid_bodies(self._h, None, 0, ctypes.byref(n)))
        arr = (CfgRigidBody * max(n.value, 1))()
        check(_lib.lib().cfg_rigid_bodies(self._h, arr, n.value, ctypes.byref(n)))
        return [{k: getattr(arr[i], k) for k, _ in CfgRigidBody._fields_} for i in range(n.value)]

    @property
    def bodies(self) -> list:
        return [self.body(s["id"]) for s in self.states()]

    def pick(self, x: float, y: float):
        i, lx, ly = ctypes.c_int(), ctypes.c_double(), ctypes.c_double()
        check(_lib.lib().cfg_rigid_pick(self._h, float(x), float(y), ctypes.byref(i), ctypes.byref(lx),
                                        ctypes.byref(ly)))
        return None if i.value == 0 else {"body": self.body(i.value), "lx": lx.value, "ly": ly.value}

    def startDrag(self, body: Body, lx, ly, tx, ty):
        check(_lib.lib().cfg_rigid_drag_start(self._h, body.id, float(lx), float(ly), float(tx), float(ty)))

    def moveDrag(self, body: Body, tx, ty):
        check(_lib.lib().cfg_rigid_drag_move(self._h, body.id, float(tx), float(ty)))

    def endDrag(self, body: Body):
        check(_lib.lib().cfg_rigid_drag_end(self._h, body.id))

    def maxPenetration(self) -> float:
        v = ctypes.c_double()
        check(_lib.lib().cfg_rigid_max_penetration(self._h, ctypes.byref(v)))
        return v.value

    def contacts(self):
        m, p = ctypes.c_int(), ctypes.c_int()
        check(_lib.lib().cfg_rigid_contacts(self._h, ctypes.byref(m), ctypes.byref(p)))
        return m.value, p.value
