"""The headless renderer's fixtures and host helpers (no GPU).

The render fixtures (rnd_* in tests/golden) are images of render.wgsl's fragment
stage computed by the reference's own WGSL translated to C++; here they are
re-rendered from the fixture's state through that translation (when it is
built) to pin them, and the PNG writer is checked by decoding its output.
"""
import ctypes
import os
import struct
import zlib

import numpy as np
import pytest

from campfire_b200._lib import CfgRenderParams
from campfire_b200.render import to_rgba8, write_png
from test_golden import FIXTURES, load

RENDER_FIXTURES = [f for f in FIXTURES if any(k.startswith("rnd_img_") for k in np.load(f).files)]
IDS = [f.rsplit("/", 1)[-1][:-4] for f in RENDER_FIXTURES]


def shots(d):
    return sorted(k[len("rnd_img_"):] for k in d if k.startswith("rnd_img_"))


def uniform(d, k) -> CfgRenderParams:
    return CfgRenderParams.from_buffer_copy(d["rnd_rp_" + k].tobytes())


def test_render_fixtures_present():
    assert len(RENDER_FIXTURES) >= 2
    for f in RENDER_FIXTURES:
        d = load(f)
        ks = shots(d)
        assert {f"v{v}" for v in range(7)} <= set(ks)
        assert d["rnd_wood"].shape == (64 * 12,)
        for k in ks:
            rp = uniform(d, k)
            assert rp.view == int(k[1])
            assert rp.nPieces == int(d["in_npieces"])
            img = d["rnd_img_" + k]
            assert img.dtype == np.float32 and img.ndim == 3 and img.shape[2] == 3
            # view 3 mixes by an unclamped oxygen fraction: the colour target clamps it
            assert np.all(np.isfinite(img)) and img.min() >= 0.0 and img.max() <= 1.01


def test_render_params_layout():
    # the RP uniform of render.wgsl:13-17: 2 i32 then 10 f32, 48 bytes
    assert struct.calcsize("<ii10f") == 48 == ctypes.sizeof(CfgRenderParams)
    rp = CfgRenderParams.from_buffer_copy(struct.pack("<ii10f", 3, 5, 1.5, 0.8, 1.2, 0.03, 2.0, 1800, 3e-7,
                                                      0.1, -0.03, 2.0))
    assert (rp.view, rp.nPieces, rp.exposure, rp.zoom) == (3, 5, 1.5, 2.0)


@pytest.mark.parametrize("path", RENDER_FIXTURES, ids=IDS)
def test_oracle_reproduces_render_fixtures(path):
    """The translated reference renders the fixture state into exactly the stored images."""
    from oracle import oracle as om
    if not os.path.exists(om.REF_LIB_PATH):
        pytest.skip("translated reference not built (needs the reference checkout)")
    d = load(path)
    nx, ny = (int(v) for v in d["meta_dims"])
    s = om.OracleSim(nx, ny, float(d["meta_width"]), float(d["meta_dt"]), impl="wgsl")
    try:
        for k, v in zip(d["in_param_names"].tolist(), d["in_param_values"].tolist()):
            s.set_param(k, v)
        s.upload_pieces(d["in_pieces"], int(d["in_npieces"]))
        s.set_frame(int(d["meta_steps"]))
        s.write_params()
        for f, key in (("T", "st_sources_T"), ("Y", "st_sources_Y"), ("SQ", "st_sources_SQ"),
                       ("U", "st_project_U"), ("V", "st_project_V"), ("rad", "rad")):
            s.write(f, d[key])
        for k in shots(d):
            img = d["rnd_img_" + k]
            out = s.render(d["rnd_rp_" + k].tobytes(), d["rnd_wood"], img.shape[1], img.shape[0])
            np.testing.assert_array_equal(out[..., :3], img, err_msg=k)
            assert np.all(out[..., 3] == 1.0)
    finally:
        s.close()


def _decode_png(path):
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, hdr = 8, b"", None
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        crc = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        assert crc == zlib.crc32(tag + body) & 0xffffffff
        if tag == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    w, h, depth, ctype = hdr[:4]
    assert (depth, ctype) == (8, 6)
    raw = zlib.decompress(idat)
    rows = [raw[y * (4 * w + 1):(y + 1) * (4 * w + 1)] for y in range(h)]
    assert all(r[0] == 0 for r in rows)
    return np.frombuffer(b"".join(r[1:] for r in rows), np.uint8).reshape(h, w, 4)


def test_png_writer_round_trip(tmp_path):
    d = load(RENDER_FIXTURES[0])
    img = d["rnd_img_v0"]
    rgba = np.concatenate([img, np.ones(img.shape[:2] + (1,), np.float32)], axis=2)
    p = str(tmp_path / "v0.png")
    write_png(p, rgba)
    back = _decode_png(p)
    np.testing.assert_array_equal(back, to_rgba8(rgba))
    assert back.shape == (img.shape[0], img.shape[1], 4)
    # unorm8 conversion: clamp, scale, round to nearest
    np.testing.assert_array_equal(to_rgba8(np.array([-1.0, 0.0, 0.5, 1.0 / 255 * 0.49, 1.0, 2.0], np.float32)),
                                  np.array([0, 0, 128, 0, 255, 255], np.uint8))
