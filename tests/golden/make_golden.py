"""Generates the golden fixtures of the gas step (tests/golden/*.npz).

The outputs come from the reference itself: its WGSL kernels (shaders/*.wgsl and
the sampler text of js/gpu.js) translated mechanically to C++ by
oracle/wgsl2cpp.py and driven in FluidSim's dispatch order (js/fluid.js) by
oracle/wgsl_harness.cpp, built by `make -C oracle ref` into oracle/_ref/.
Needs the reference checkout (its path in $CAMPFIRE_REF, or the first argument) and
the product library for the scene generator; the fixtures themselves are
self-contained (inputs and outputs), so the tests read only the .npz files.

Each fixture holds, for one seeded scene:
  in_*      the scene: parameter names/values, pieces, npieces, T, Y, U, V
  geo_*     encodeGeometry: cellG (sdf, piece id), fx, fy, faceW
  acc       the acc readback after each of `steps` steps (frame = step index)
  fin_*     the state after those steps
  st_<stage>_<field>
            the fields each stage writes, stage by stage, during one more step
  rad       encodeRadiation after that step
  rnd_*     (cases in RENDER_CASES) render.wgsl's fragment stage on that final state:
            per image k the 48-byte RP uniform rnd_rp_k and the RGB image rnd_img_k
            (row 0 at the top; alpha is 1), with the seeded wood buffer rnd_wood

    CAMPFIRE_REF=<reference checkout> python tests/golden/make_golden.py   # rewrite the fixtures
"""
from __future__ import annotations

import glob
import hashlib
import os
import struct
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# the reference checkout: CAMPFIRE_REF (environment) or the first argument
REF = os.environ.get("CAMPFIRE_REF") or (sys.argv[1] if len(sys.argv) > 1 else "")
if not REF:
    sys.exit("make_golden.py: set CAMPFIRE_REF (or pass the path) to the reference checkout")
STATE = ("T", "Y", "U", "V", "T2", "Y2", "U2", "V2", "SQ", "p")
STAGE_OUT = {
    "advect": ("T2", "Y2", "U2", "V2"),
    "diffuse": ("T", "Y"),
    "sources": ("T", "Y", "SQ"),
    "forces": ("U", "V"),
    "coef_rhs": ("rhs", "ax", "ay"),
    "pressure": ("p",),
    "project": ("U", "V"),
}
STAGES = tuple(STAGE_OUT)

# name, scene kind, nx, ny, width, seed, steps, extra parameters
CASES = [
    ("logs_32x48", 0, 32, 48, 0.8, 101, 12, {}),
    ("tepee_diff3_40x64", 1, 40, 64, 0.5, 102, 10, {"diffMult": 40.0}),
    ("floor_heater_burner_32x48", 2, 32, 48, 0.4, 103, 10,
     {"diffMult": 200.0, "heaterX0": 0.1, "heaterX1": 0.2, "heaterY1": 0.03, "heaterT": 900.0,
      "burnerX0": 0.25, "burnerX1": 0.3, "burnerFlux": 0.02, "burnerT": 600.0}),
]
RENDER_CASES = ("logs_32x48", "tepee_diff3_40x64")
GROUND = 0.03   # js/render.js:6


def shader_digest(ref: str) -> str:
    h = hashlib.sha256()
    for f in sorted(glob.glob(os.path.join(ref, "shaders", "*.wgsl"))) + [os.path.join(ref, "js", "gpu.js")]:
        with open(f, "rb") as fh:
            h.update(os.path.relpath(f, ref).encode())
            h.update(fh.read())
    return h.hexdigest()


def level_fields(sim, base):
    nl = int(sim.info()["levels"])
    return [base if l == 0 else f"{base}.{l}" for l in range(nl)]


def stage_fields(sim, stage):
    out = []
    for f in STAGE_OUT[stage]:
        out += level_fields(sim, f) if f in ("ax", "ay") else [f]
    return out


def make_case(om, cb, name, kind, nx, ny, width, seed, steps, extra):
    from campfire_b200.fluid import SCENE_PARAM_KEYS
    sc = cb.generate_scene(kind, nx, ny, width, seed)
    s = om.OracleSim(nx, ny, width, sc["dt"], impl="wgsl")
    names = list(SCENE_PARAM_KEYS) + list(extra)
    vals = [sc["params"][k] for k in SCENE_PARAM_KEYS] + [extra[k] for k in extra]
    d = {
        "meta_name": np.array(name), "meta_dims": np.array([nx, ny], np.int32), "meta_width": np.float64(width),
        "meta_dt": np.float64(sc["dt"]), "meta_steps": np.int32(steps), "meta_shaders_sha256": np.array(shader_digest(REF)),
        "in_param_names": np.array(names), "in_param_values": np.array(vals, np.float64),
        "in_pieces": np.asarray(sc["pieces"], np.float32).ravel(), "in_npieces": np.int32(sc["npieces"]),
    }
    for k in ("T", "Y", "U", "V"):
        d["in_" + k] = np.asarray(sc[k], np.float32).ravel()
    apply_inputs(s, d)
    d["meta_levels"] = np.int32(s.info()["levels"])
    d["meta_diffsub"] = np.int32(s.info()["diffSub"])
    cg = s.read("cellG").reshape(-1, 2)
    d["geo_cellG_sdf"] = cg[:, 0].astype(np.float32)
    d["geo_cellG_id"] = cg[:, 1].astype(np.uint32)
    d["geo_fx"] = s.read("fx").astype(np.float32)
    d["geo_fy"] = s.read("fy").astype(np.float32)
    d["geo_faceW"] = s.readback()["faceW"].astype(np.int32)
    acc = []
    for i in range(steps):
        s.set_frame(i)
        s.write_params()
        s.step()
        acc.append(s.readback()["acc"].copy())
    d["acc"] = np.stack(acc).astype(np.int32)
    for f in STATE:
        d["fin_" + f] = s.read(f).astype(np.float32)
    for f in ("rhs", "ax", "ay"):
        for lf in level_fields(s, f):
            d["fin_" + lf] = s.read(lf).astype(np.float32)
    for lf in level_fields(s, "p")[1:]:
        d["fin_" + lf] = s.read(lf).astype(np.float32)
    s.set_frame(steps)
    s.write_params()
    for st in STAGES:
        s.stage(st)
        for f in stage_fields(s, st):
            d[f"st_{st}_{f}"] = s.read(f).astype(np.float32)
    d["st_acc"] = s.readback()["acc"].astype(np.int32)
    s.radiation()
    d["rad"] = s.readback()["rad"].astype(np.float32)
    if name in RENDER_CASES:
        add_renders(s, d, seed)
    s.close()
    return d


def render_uniform(view, npieces, width, height, cam=None, exposure=1.0, time=0.0, tmax=1800.0, chemi=3e-7):
    """The RP uniform as Renderer.writeParams packs it (js/render.js:41-53)."""
    cx, cy, zoom = cam if cam else (0.0, -GROUND, 1.0)
    return struct.pack("<ii10f", view, npieces, exposure, width, height, GROUND, time, tmax, chemi, cx, cy, zoom)


def wood_buffer(npieces, seed):
    """A seeded renderer wood buffer (Tp[4], d[4], char fraction, Tcore, visAvg, hasVirgin per piece)."""
    rng = np.random.default_rng(seed)
    w = np.zeros((64, 12), np.float32)
    for n in range(npieces):
        w[n, 0:4] = rng.uniform(550.0, 900.0, 4)
        w[n, 4:8] = rng.uniform(0.5e-3, 6e-3, 4)
        w[n, 8:12] = [rng.uniform(0.05, 0.6), rng.uniform(350.0, 600.0), rng.uniform(1e3, 2e4), float(n % 3 != 2)]
    return w.ravel()


def add_renders(s, d, seed):
    inf = s.info()
    nx, ny, dx = int(inf["nx"]), int(inf["ny"]), float(inf["dx"])
    W, H = nx * dx, ny * dx
    npc = int(d["in_npieces"])
    wood = wood_buffer(npc, seed)
    d["rnd_wood"] = wood
    # a camera zoomed 4x on the lowest piece (the app's ?zoom=4&cx=..&cy=.. inspection view, js/main.js:70-80)
    pcs = d["in_pieces"].reshape(64, 20)
    j = int(np.argmin(np.where(pcs[:npc, 7] > 0, pcs[:npc, 1], 1e9)))
    zoom = 4.0
    cam = (float(pcs[j, 0]) - W / 2 / zoom, float(pcs[j, 1]) - (H + GROUND) / 2 / zoom, zoom)
    shots = [(f"v{v}", render_uniform(v, npc, W, H, time=float(inf["time"])), 40, 62) for v in range(7)]
    shots += [("v0_zoom", render_uniform(0, npc, W, H, cam=cam, exposure=2.0), 48, 72),
              ("v1_zoom", render_uniform(1, npc, W, H, cam=cam, tmax=1500.0), 48, 72)]
    for k, rp, w, h in shots:
        img = s.render(rp, wood, w, h)
        assert np.all(img[..., 3] == 1.0)
        d["rnd_rp_" + k] = np.frombuffer(rp, np.uint8).copy()
        d["rnd_img_" + k] = img[..., :3].copy()


def apply_inputs(sim, d):
    """Scene set-up in FluidSim's order: params, pieces, writeParams, reset, fields, geometry."""
    for k, v in zip(d["in_param_names"].tolist(), d["in_param_values"].tolist()):
        sim.set_param(k, v)
    sim.upload_pieces(d["in_pieces"], int(d["in_npieces"]))
    sim.write_params()
    sim.reset()
    for k in ("T", "Y", "U", "V"):
        sim.write(k, d["in_" + k])
    sim.write("T2", d["in_T"])
    sim.write("Y2", d["in_Y"])
    sim.clear_geometry()
    sim.geometry()


def main():
    from oracle import oracle as om
    import campfire_b200 as cb
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={REF}"], check=True)
    for case in CASES:
        d = make_case(om, cb, *case)
        path = os.path.join(HERE, case[0] + ".npz")
        np.savez_compressed(path, **d)
        print(f"{path}: {os.path.getsize(path)} bytes, levels {int(d['meta_levels'])}, diffSub {int(d['meta_diffsub'])}")


if __name__ == "__main__":
    main()
