"""Headless renderer: `class Renderer` of js/render.js over the C ABI.

The reference draws shaders/render.wgsl's full-screen triangle into the canvas;
here the fragment stage runs as a CUDA kernel into an RGBA float image (row 0
at the top) that is copied to the host, so frames can be written to files:

    ren = Renderer(sim)
    ren.writeParams({"view": VIEWS["photo"], "nPieces": n, "exposure": 1.0, "time": t})
    ren.writeWood(wood)            # Float32Array(64*12) of js/main.js:188-207, or a WoodScene
    img = ren.encode(400, 700)     # float32 [700, 400, 4]
    write_png("frame.png", img)
"""
from __future__ import annotations

import ctypes
import struct
import zlib

import numpy as np

from . import _lib
from ._lib import CfgRenderParams, check

VIEWS = {"photo": 0, "temperature": 1, "reaction": 2, "oxygen": 3, "fuel": 4, "velocity": 5, "soot": 6}   # :5
GROUND = 0.03   # m of ground shown below the floor line, js/render.js:6
WOOD_FLOATS = 12


def _fp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def render_defaults(sim) -> CfgRenderParams:
    """The uniform as the app writes it for this scene (cfg_render_defaults)."""
    rp = CfgRenderParams()
    check(_lib.lib().cfg_render_defaults(sim._h, ctypes.byref(rp)))
    return rp


def render(sim, rp: CfgRenderParams, width: int, height: int, wood=None) -> np.ndarray:
    """One frame of the fragment stage: float32 [height, width, 4] (cfg_render)."""
    out = np.empty((int(height), int(width), 4), np.float32)
    w = None
    if wood is not None:
        w = np.ascontiguousarray(np.asarray(wood, np.float32).ravel())
        if w.size != _lib.MAX_PIECES * WOOD_FLOATS:
            raise ValueError(f"wood must hold {_lib.MAX_PIECES * WOOD_FLOATS} floats")
    check(_lib.lib().cfg_render(sim._h, ctypes.byref(rp), None if w is None else _fp(w), int(width), int(height),
                                _fp(out)))
    return out


def render_device(sim, rp: CfgRenderParams, width: int, height: int, rgba_device_ptr: int, wood=None) -> None:
    """Enqueue one frame into device memory (width * height * 4 float32 at rgba_device_ptr) on the
    scene's stream, without waiting (cfg_render_device)."""
    w = None
    if wood is not None:
        w = np.ascontiguousarray(np.asarray(wood, np.float32).ravel())
        if w.size != _lib.MAX_PIECES * WOOD_FLOATS:
            raise ValueError(f"wood must hold {_lib.MAX_PIECES * WOOD_FLOATS} floats")
    check(_lib.lib().cfg_render_device(sim._h, ctypes.byref(rp), None if w is None else _fp(w), int(width),
                                       int(height), ctypes.c_void_p(int(rgba_device_ptr))))


class Renderer:
    """js/render.js:8-71 for a FluidSim (or a batch scene view)."""

    def __init__(self, sim):
        self.sim = sim
        self.rp = render_defaults(sim)
        self.wood = np.zeros(_lib.MAX_PIECES * WOOD_FLOATS, np.float32)

    def writeParams(self, o: dict):
        """Renderer.writeParams (js/render.js:41-53): view, nPieces, exposure, time, and optional
        tmax (1800), chemi (3e-7) and cam {x, y, zoom} (default: the whole domain and the ground)."""
        d = render_defaults(self.sim)
        view = o["view"]
        d.view = VIEWS[view] if isinstance(view, str) else int(view)
        d.nPieces = int(o.get("nPieces", d.nPieces))
        d.exposure = float(o.get("exposure", d.exposure))
        d.time = float(o.get("time", d.time))
        d.tmax = float(o["tmax"]) if o.get("tmax") is not None else 1800.0
        d.chemi = float(o["chemi"]) if o.get("chemi") is not None else 3e-7
        cam = o.get("cam") or {"x": 0.0, "y": -GROUND, "zoom": 1.0}
        d.camX, d.camY, d.zoom = float(cam["x"]), float(cam["y"]), float(cam["zoom"])
        self.rp = d

    def writeWood(self, data):
        """Renderer.writeWood (:55): the 64 x 12 wood buffer, or a WoodScene's as its last upload built it."""
        if hasattr(data, "render_data"):
            data = data.render_data()
        w = np.zeros(_lib.MAX_PIECES * WOOD_FLOATS, np.float32)
        a = np.asarray(data, np.float32).ravel()
        w[: a.size] = a
        self.wood = w

    def encode(self, width: int, height: int) -> np.ndarray:
        """Renderer.encode (:57-70) into an image of width x height pixels."""
        return render(self.sim, self.rp, width, height, self.wood)


def to_rgba8(img: np.ndarray) -> np.ndarray:
    """A unorm8 colour target's conversion: clamp to [0, 1], scale by 255, round to nearest."""
    return np.rint(np.clip(np.asarray(img, np.float32), 0.0, 1.0) * 255.0).astype(np.uint8)


def write_png(path: str, img: np.ndarray) -> None:
    """8-bit RGBA PNG of a float [H, W, 4] image (or a uint8 one)."""
    a = img if img.dtype == np.uint8 else to_rgba8(img)
    h, w = a.shape[:2]
    raw = b"".join(b"\x00" + a[y].tobytes() for y in range(h))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xffffffff)

    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0))
    png += chunk(b"IDAT", zlib.compress(raw, 6)) + chunk(b"IEND", b"")
    with open(path, "wb") as f:
        f.write(png)
