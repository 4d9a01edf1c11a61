"""The headless renderer (CUDA k_render through cfg_render) against the render fixtures.

The fixtures hold render.wgsl's fragment stage run by the reference's WGSL
translated to C++ on each case's final state (tests/golden/make_golden.py). The
state is written into the CUDA scene as it is, so the images differ only by the
device's and the host's transcendental functions (exp, log, pow, sin, cos within
a few ulp). The value noise of the wood end grain and the ground hashes
fract(sin(x) * 43758.5453): an ulp of sin(x) moves that by about 3e-3, and
where the product crosses an integer the hash jumps by up to 1. So per image:
the median pixel error is below 1e-6, at least 99% of the pixels agree within
2e-3 (max over channels), and the mean absolute error is below 1e-4. Measured
on B200: views 1-6 within 2e-6 everywhere (most bit-exact); the photo view's
median error is at most 2.4e-7 with 99.88% of the pixels or more within 2e-3.
"""
import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200._lib import CfgRenderParams
from campfire_b200.render import Renderer, render
from test_gpu_golden import gpu_sim
from test_golden import load
from test_render import IDS, RENDER_FIXTURES, shots, uniform

pytestmark = pytest.mark.gpu
CLOSE, FRAC, MEDIAN, MEAN = 2e-3, 0.99, 1e-6, 1e-4


def state_sim(d):
    g = gpu_sim(d)
    g.setFrame(int(d["meta_steps"]))
    g.writeParams()
    for f, key in (("T", "st_sources_T"), ("Y", "st_sources_Y"), ("SQ", "st_sources_SQ"),
                   ("U", "st_project_U"), ("V", "st_project_V"), ("rad", "rad")):
        g.writeBuffer(f, d[key])
    return g


def image_error(out, ref):
    e = np.abs(out[..., :3].astype(np.float64) - ref).max(axis=2)
    return float(np.median(e)), float(np.mean(e <= CLOSE)), float(e.mean()), float(e.max())


@pytest.mark.parametrize("path", RENDER_FIXTURES, ids=IDS)
def test_render_matches_fixture(path):
    d = load(path)
    g = state_sim(d)
    try:
        for k in shots(d):
            ref = d["rnd_img_" + k]
            out = render(g, uniform(d, k), ref.shape[1], ref.shape[0], d["rnd_wood"])
            assert out.shape == (ref.shape[0], ref.shape[1], 4)
            assert np.all(out[..., 3] == 1.0), k
            med, frac, mean, mx = image_error(out, ref)
            print(f"{k}: median {med:.2e} close {frac:.4f} mean {mean:.2e} max {mx:.2e}")
            assert med <= MEDIAN and frac >= FRAC and mean <= MEAN, (k, med, frac, mean, mx)
    finally:
        g.close()


def test_renderer_params_and_errors():
    d = load(RENDER_FIXTURES[0])
    g = state_sim(d)
    try:
        ren = Renderer(g)
        ren.writeParams({"view": "photo", "nPieces": int(d["in_npieces"]), "exposure": 1.0, "time": 0.0})
        ref = uniform(d, "v0")
        for f, _ in CfgRenderParams._fields_:
            if f != "time":
                assert getattr(ren.rp, f) == pytest.approx(getattr(ref, f), rel=1e-6), f
        ren.writeWood(d["rnd_wood"])
        img = ren.encode(40, 62)
        med, frac, _, _ = image_error(img, d["rnd_img_v0"])
        assert med <= MEDIAN and frac >= FRAC
        bad = uniform(d, "v0")
        bad.nPieces = 65
        with pytest.raises(cb.CampfireError, match="INVAL"):
            render(g, bad, 8, 8)
        with pytest.raises(cb.CampfireError, match="INVAL"):
            render(g, uniform(d, "v0"), 0, 8)
        with pytest.raises(ValueError):
            render(g, uniform(d, "v0"), 8, 8, np.zeros(10, np.float32))
        # a larger image than before reallocates the device image
        big = render(g, uniform(d, "v1"), 320, 496, d["rnd_wood"])
        assert big.shape == (496, 320, 4) and np.all(big[..., 3] == 1.0)
    finally:
        g.close()


def test_wood_scene_render_data():
    """WoodScene's render buffer is uploadPieces' woodData (js/main.js:200-203)."""
    from campfire_b200.wood import WoodScene
    from campfire_b200.fluid import load_scene
    sc = cb.generate_scene(0, 64, 96, 0.8, 1)
    g = cb.FluidSim(0, {"nx": 64, "ny": 96, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    g.uploadPieces(np.zeros(64 * 20, np.float32), 0)
    ws = WoodScene(g)
    try:
        a = ws.add(0.35, 0.026, 0.0, 0.05, 500.0, preheat=(900.0, 0.004, 350.0))
        b = ws.add(0.45, 0.026, 0.3, 0.05, 450.0)
        for _ in range(4):
            ws.frame(0.01)
        w = ws.render_data().reshape(64, 12)
        for s in (a, b):
            st, _, _ = ws.piece(s)
            np.testing.assert_array_equal(w[s, 0:4], np.float32(st["Tp"]))
            np.testing.assert_array_equal(w[s, 4:8], np.float32(st["d"]))
            cf = st["mc"] / st["rhoC"] / (st["mv"] / st["rhoV"] + st["mc"] / st["rhoC"] + 1e-12)
            assert w[s, 8] == np.float32(cf)
            assert w[s, 9] == np.float32(st["Tc"])
            assert w[s, 11] == (1.0 if st["mv"] > 0 else 0.0)
        assert np.all(w[2:] == 0)
        ren = Renderer(g)
        ren.writeParams({"view": 0, "nPieces": 2, "exposure": 1.0, "time": g.info()["time"]})
        ren.writeWood(ws)
        img = ren.encode(64, 98)
        assert np.all(np.isfinite(img)) and np.all(img[..., 3] == 1.0)
    finally:
        ws.close()
        g.close()
