"""The C-ABI library without computing on a GPU: exports, errors, host logic."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200 import _lib


def test_library_exports_every_declared_symbol():
    L = cb.lib()
    syms = cb.declared_symbols()
    assert len(syms) >= 40
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_exported_symbols_match_header_exactly():
    # nm -D lists the dynamic exports; every cfg_* export is declared in the header
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T cfg_" in ln}
    assert exported == set(cb.declared_symbols())


def test_params_struct_is_the_40_field_uniform():
    assert ctypes.sizeof(_lib.CfgParams) == 160   # common.wgsl:4-15
    p = _lib.CfgParams()
    _lib.check(cb.lib().cfg_default_params(ctypes.byref(p)))
    # js/fluid.js:35-45 defaults from js/config.js PHYS
    assert p.Tamb == np.float32(293.15) and p.YOamb == np.float32(0.232) and p.depth == np.float32(0.8)
    assert p.reactB == np.float32(2e10) and p.sO2 == np.float32(15e6 / 13.1e6)
    assert abs(p.rhoAmb - 101325 * 0.0289 / (8.314462 * 293.15)) < 1e-6


def test_no_cpu_fallback_without_device():
    if cb.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(cb.CampfireError) as e:
        cb.FluidSim(0, {"nx": 64, "ny": 96, "dt": 0.002}).init()
    assert e.value.code == -19   # CFG_ERR_NODEV


def test_coarsest_level_too_large_is_a_range_error():
    # js/fluid.js:91 throws 'coarsest level too large'; here the cap is 7 levels
    with pytest.raises(cb.CampfireError) as e:
        cb.FluidSim(0, {"nx": 1024, "ny": 1536, "dt": 0.002}).init()
    assert e.value.code == -34 and "coarsest level too large" in str(e.value)
    # an odd size stops halving at once: 257*258 cells on one level
    with pytest.raises(cb.CampfireError) as e:
        cb.FluidSim(0, {"nx": 257, "ny": 258, "dt": 0.002}).init()
    assert e.value.code == -34


def test_bad_arguments_are_rejected():
    with pytest.raises(cb.CampfireError) as e:
        cb.FluidSim(0, {"nx": 1, "ny": 96, "dt": 0.002}).init()
    assert e.value.code == -22
    with pytest.raises(cb.CampfireError):
        cb.FluidSim(0, {"nx": 64, "ny": 96, "dt": -1.0}).init()


def test_scene_generator_is_deterministic_and_matches_the_workload():
    a = cb.generate_scene(0, 128, 192, 0.8, 1234)
    b = cb.generate_scene(0, 128, 192, 0.8, 1234)
    for k in ("T", "Y", "U", "V", "pieces"):
        assert np.array_equal(a[k], b[k])
    c = cb.generate_scene(0, 128, 192, 0.8, 1235)
    assert not np.array_equal(a["U"], c["U"])
    # three logs of radius 2.5 cm at the stated centres as squares of equal area, 600 K faces, 5e-3 kg/m2/s
    P = a["pieces"].reshape(64, 20)
    h = 0.025 * np.sqrt(np.pi) / 2
    assert a["npieces"] == 3
    assert np.allclose(P[:3, :4], [[0.35, 0.025, 0, h], [0.45, 0.025, 0, h], [0.40, 0.068, 0, h]])
    assert np.all(P[:3, 8:12] == 600) and np.allclose(P[:3, 12:16], 5e-3)
    # Gaussian hot spot 1800 K at (0.40, 0.12), velocities within +-0.01 m/s, dt = 2 ms by CFL cap
    T = a["T"].reshape(192, 128)
    assert 1700 < T.max() <= 1800 and T.min() >= 300
    Y = a["Y"].reshape(-1, 4)
    assert np.allclose(Y.sum(1), 1.0, atol=1e-6) and np.all(Y[:, 3] == 0)
    assert np.abs(a["U"]).max() <= 0.01 and np.abs(a["V"]).max() <= 0.01
    assert a["dt"] == 0.002
    assert a["params"]["Tamb"] == 300 and abs(a["params"]["depth"] - 0.3) < 1e-7


def test_tepee_and_floor_scenes_have_no_overlaps():
    for kind, seed in ((1, 1236), (2, 2000), (2, 2001), (2, 2063)):
        s = cb.generate_scene(kind, 192, 288, 0.8, seed)
        n = s["npieces"]
        P = s["pieces"].reshape(64, 20)[:n]
        assert (kind == 1 and n == 5) or (kind == 2 and 2 <= n <= 6)
        # corners above the floor, inside the domain
        for x, y, a, h in P[:, :4]:
            c, si = np.cos(a), np.sin(a)
            for lx, ly in ((-h, -h), (h, -h), (h, h), (-h, h)):
                assert y + si * lx + c * ly >= -1e-6
                assert 0 <= x + c * lx - si * ly <= 0.8
        if kind == 2:
            assert 0.5 * 2e10 <= s["params"]["reactB"] <= 2 * 2e10 * 1.0001
            assert 0.18 <= s["params"]["YOamb"] <= 0.233


def test_autotuner_needs_a_device_and_valid_arguments():
    import ctypes
    L = cb.lib()
    one = (ctypes.c_int * 1)(64)
    cells = (ctypes.c_int * 4)()
    ms = (ctypes.c_double * 4)()
    best = ctypes.c_int()
    k = ctypes.c_int(0)
    assert L.cfg_autotune(0, 1, one, one, 0, 5, ctypes.byref(best), cells, ms, ctypes.byref(k)) == -22   # no capacity
    if cb.device_count() == 0:
        with pytest.raises(cb.CampfireError) as e:
            cb.autotune([(64, 96)], iters=2)
        assert e.value.code == -19


def test_server_structs_match_the_header():
    import ctypes
    assert ctypes.sizeof(cb._lib.CfgJob) == 32
    assert ctypes.sizeof(cb._lib.CfgJobResult) == 64
    if cb.device_count() == 0:
        with pytest.raises(cb.CampfireError) as e:
            cb.Server([(64, 96)], [1], 1e9)
        assert e.value.code == -19
