"""The oracle's restatement of the seeded benchmark scenes equals the product's generator
(cfg_scene_generate, host code: no GPU needed) bit for bit, so the CPU checker and the
reference arm of the benchmark build their inputs without the product library."""
import numpy as np
import pytest

import campfire_b200 as cb
from oracle import scene_ref


@pytest.mark.parametrize("kind,nx,ny,seed", [(0, 64, 96, 1234), (0, 256, 384, 1235), (1, 512, 768, 1236),
                                             (1, 96, 144, 9003), (2, 96, 144, 2000), (2, 192, 288, 2017),
                                             (2, 128, 192, 2063)])
def test_scene_restatement_is_bit_exact(kind, nx, ny, seed):
    a = cb.generate_scene(kind, nx, ny, 0.8, seed)
    b = scene_ref.generate_scene(kind, nx, ny, 0.8, seed)
    for f in ("T", "Y", "U", "V", "pieces"):
        assert np.array_equal(a[f].view(np.uint32), b[f].view(np.uint32)), f
    assert a["npieces"] == b["npieces"]
    assert a["dt"] == b["dt"]
    for k in scene_ref.SCENE_PARAM_KEYS:
        assert a["params"][k] == b["params"][k], k
