"""ORACLE — test infrastructure, not product code.

The seeded synthetic scenes of the benchmark workloads, restated on the host in
Python so that the CPU checker (and bench.py's reference arm, which times it)
can build its inputs without loading the product library. The product's own
generator is `cfg_scene_generate`; `tests/test_scene_ref.py` checks that both
give the same bits for every scene kind.

The scenes follow the workload definitions (no reference file defines them:
the reference builds its scene interactively, js/main.js:132-155):
  kind 0  three square logs of half-side 0.025*sqrt(pi)/2 (a circle of radius
          2.5 cm at equal area) at (0.35,0.025), (0.45,0.025), (0.40,0.068) m,
          fuel flux 5e-3 kg/m^2/s at 600 K;
  kind 1  five logs of radius 5 cm (as squares of equal area) in a seeded tepee,
          flux 8e-3;
  kind 2  2-6 seeded floor logs of radius 2.5 or 5 cm, B scaled by a factor
          log-uniform in [0.5, 2], ambient Y_O uniform in [0.18, 0.233].
Gas: T = 300 + 1500 g, g = exp(-r^2 / (2 * 0.05^2)) around (0.40, 0.12) m;
Y_F = 0.3 g, Y_O = YOamb (1 - Y_F), soot 0, products the rest; U, V uniform in
[-0.01, 0.01] m/s from a counter-based hash of the seed; dt = min(2 ms,
0.5 dx / max|u|). Pieces use the packing of js/main.js:196-199 (x, y, angle,
half, vel, omega, alive, Ts[4], mflux[4], charCov[4]).

Arithmetic is IEEE double as in the product's generator, with the C library's
exp/log/sin/cos/sqrt (Python's math module), evaluated in the same order.
"""
from __future__ import annotations

import math

import numpy as np

MASK = (1 << 64) - 1
MAX_PIECES, PIECE_FLOATS = 64, 20
# parameters a scene sets; the rest keep FluidSim's defaults (js/fluid.js:35-45)
SCENE_PARAM_KEYS = ("Tamb", "rhoAmb", "YOamb", "reactB", "reactTa", "dHc", "Pr", "exchAlpha", "depth")


def _splitmix(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & MASK
    x = ((x ^ (x >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    x = ((x ^ (x >> 27)) * 0x94D049BB133111EB) & MASK
    return x ^ (x >> 31)


def _hash01(seed: int, stream: int, k: int) -> float:
    base = _splitmix((seed ^ ((stream * 0xD1B54A32D192ED03) & MASK)) & MASK)
    return (_splitmix((base + k) & MASK) >> 11) * (1.0 / 9007199254740992.0)


def _hash01_array(seed: int, stream: int, n: int) -> np.ndarray:
    """_hash01(seed, stream, k) for k = 0..n-1 (vectorised splitmix, wrapping uint64)."""
    base = np.uint64(_splitmix((seed ^ ((stream * 0xD1B54A32D192ED03) & MASK)) & MASK))
    with np.errstate(over="ignore"):
        x = base + np.arange(n, dtype=np.uint64)
        x = x + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x = x ^ (x >> np.uint64(31))
    return (x >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class _Rng:
    def __init__(self, seed: int, stream: int):
        self.seed, self.stream, self.n = seed, stream, 0

    def u(self, a: float | None = None, b: float | None = None) -> float:
        v = _hash01(self.seed, self.stream, self.n)
        self.n += 1
        return v if a is None else a + (b - a) * v


def _corners(b):
    x, y, a, h = b
    c, s = math.cos(a), math.sin(a)
    lx, ly = (-h, h, h, -h), (-h, -h, h, h)
    return [x + c * lx[k] - s * ly[k] for k in range(4)], [y + s * lx[k] + c * ly[k] for k in range(4)]


def _overlap(p, q, margin: float) -> bool:
    """Separating-axis test of two rotated squares with a clearance margin."""
    px, py = _corners(p)
    qx, qy = _corners(q)
    axes = ((math.cos(p[2]), math.sin(p[2])), (-math.sin(p[2]), math.cos(p[2])),
            (math.cos(q[2]), math.sin(q[2])), (-math.sin(q[2]), math.cos(q[2])))
    for ax in axes:
        pmin, pmax, qmin, qmax = 1e30, -1e30, 1e30, -1e30
        for k in range(4):
            dp = px[k] * ax[0] + py[k] * ax[1]
            dq = qx[k] * ax[0] + qy[k] * ax[1]
            pmin, pmax = min(pmin, dp), max(pmax, dp)
            qmin, qmax = min(qmin, dq), max(qmax, dq)
        if pmax + margin < qmin or qmax + margin < pmin:
            return False
    return True


def _inside(b, W: float, H: float) -> bool:
    cx, cy = _corners(b)
    return all(not (cx[k] < 0.005 or cx[k] > W - 0.005 or cy[k] < -1e-9 or cy[k] > H - 0.005) for k in range(4))


def _fits(b, placed, W: float, H: float) -> bool:
    if not _inside(b, W, H):
        return False
    return not any(_overlap(b, q, 0.006) for q in placed)


def _f32(v: float) -> float:
    return float(np.float32(v))


def generate_scene(kind: int, nx: int, ny: int, width: float = 0.8, seed: int = 1234) -> dict:
    """The scene as a dict: T, Y, U, V (float32, dense reference layouts), pieces (64 x 20 float32),
    npieces, params (the scene's parameters, rounded to f32 as the uniform holds them), dt."""
    if kind not in (0, 1, 2):
        raise ValueError("scene kind must be 0, 1 or 2")
    dx = width / nx
    H = dx * ny
    rng = _Rng(seed, 7)
    Tamb, YOamb, Bmul, flux = 300.0, 0.233, 1.0, 5e-3
    if kind == 1:
        flux = 8e-3
    if kind == 2:
        Bmul = math.exp(rng.u(math.log(0.5), math.log(2.0)))
        YOamb = rng.u(0.18, 0.233)
    params = {"Tamb": _f32(Tamb), "rhoAmb": _f32(101325.0 * 0.0289 / (8.314462 * Tamb)), "YOamb": _f32(YOamb),
              "reactB": _f32(2.0e10 * Bmul), "reactTa": 15000.0, "dHc": _f32(15.0e6), "Pr": _f32(0.7),
              "exchAlpha": _f32(0.05), "depth": _f32(0.3)}
    area_half = 0.5 * math.sqrt(3.14159265358979323846)
    boxes = []
    if kind == 0:
        hf = 0.025 * area_half
        boxes = [(0.35, 0.025, 0.0, hf), (0.45, 0.025, 0.0, hf), (0.40, 0.068, 0.0, hf)]
    elif kind == 1:
        hf = 0.05 * area_half
        cx = 0.5 * width
        for k in range(5):
            for _ in range(4000):
                sg = -1.0 if k % 2 == 0 else 1.0
                if k < 2:
                    b = (cx + sg * rng.u(0.13, 0.17), hf, 0.0, hf)
                elif k < 4:
                    bx = cx + sg * rng.u(0.04, 0.08)
                    by = rng.u(0.12, 0.17)
                    b = (bx, by, -sg * rng.u(0.45, 0.75), hf)
                else:
                    bx = cx + rng.u(-0.02, 0.02)
                    by = rng.u(0.24, 0.30)
                    b = (bx, by, rng.u(-0.3, 0.3), hf)
                if _fits(b, boxes, width, H):
                    boxes.append(b)
                    break
    else:
        want = 2 + min(4, int(rng.u() * 5))
        for _ in range(want):
            hf = (0.025 if rng.u() < 0.5 else 0.05) * area_half
            for _ in range(2000):
                b = (rng.u(0.05 + hf, width - 0.05 - hf), hf, 0.0, hf)
                ok = _fits(b, boxes, width, H)
                for q in boxes:
                    ok = ok and abs(b[0] - q[0]) >= b[3] + q[3] + 0.01
                if ok:
                    boxes.append(b)
                    break
    pieces = np.zeros(MAX_PIECES * PIECE_FLOATS, np.float32)
    for n, (x, y, a, h) in enumerate(boxes):
        p = pieces[n * PIECE_FLOATS:(n + 1) * PIECE_FLOATS]
        p[0], p[1], p[2], p[3], p[7] = x, y, a, h, 1.0
        p[8:12], p[12:16], p[16:20] = 600.0, flux, 0.0
    # initial gas: one exp per cell, evaluated as the product's generator does
    s2 = 2.0 * 0.05 * 0.05
    g = np.empty(nx * ny, np.float64)
    k = 0
    for j in range(ny):
        y = (j + 0.5) * dx - 0.12
        yy = y * y
        for i in range(nx):
            x = (i + 0.5) * dx - 0.40
            g[k] = math.exp(-(x * x + yy) / s2)
            k += 1
    yf = 0.3 * g
    yo = YOamb * (1.0 - yf)
    ys = np.zeros_like(g)
    yp = 1.0 - yf - yo - ys
    T = (300.0 + 1500.0 * g).astype(np.float32)
    Y = np.stack([yf, yo, yp, ys], axis=1).astype(np.float32).ravel()
    U = ((2.0 * _hash01_array(seed, 1, (nx + 1) * ny) - 1.0) * 0.01).astype(np.float32)
    V = ((2.0 * _hash01_array(seed, 2, nx * (ny + 1)) - 1.0) * 0.01).astype(np.float32)
    umax = max(float(np.max(np.abs(U.astype(np.float64)))), float(np.max(np.abs(V.astype(np.float64)))))
    dt = min(2e-3, 0.5 * dx / umax) if umax > 0 else 2e-3
    return {"T": T, "Y": Y, "U": U, "V": V, "pieces": pieces, "npieces": len(boxes), "params": params, "dt": dt,
            "nx": nx, "ny": ny, "width": width, "kind": kind, "seed": seed}


def load_scene(sim, scene: dict) -> None:
    """Apply a scene to an OracleSim in FluidSim's set-up order (params, pieces, writeParams, reset,
    fields, geometry), as the product's loader does."""
    for k in SCENE_PARAM_KEYS:
        sim.set_param(k, scene["params"][k])
    sim.upload_pieces(scene["pieces"], scene["npieces"])
    sim.write_params()
    sim.reset()
    for k in ("T", "Y", "U", "V"):
        sim.write(k, scene[k])
    sim.write("T2", scene["T"])
    sim.write("Y2", scene["Y"])
    sim.clear_geometry()
    sim.geometry()
