"""The CPU oracle against known answers.

The reference has no golden vectors for its WGSL kernels; these cases pin the
restatement to answers derived by hand from the WGSL text, plus the one known
answer the reference publishes (the 1D flame speed, README.md:89,
tests/flame1d.mjs).
"""
import math

import numpy as np
import pytest

from conftest import norm_err


def test_flame_speed_known_answer(oracle_mod):
    # README.md:89, js/config.js:26: B = 2e10, Ta = 15000 K -> S_L = 0.38 m/s (resolved: dx = 5e-5)
    sl, tb = oracle_mod.flame_speed(B=2e10, Ta=15000.0, dx=5e-5, L=0.03, tEnd=1.0)
    assert abs(sl - 0.38) <= 0.02 * 0.38, sl
    assert 2100 < tb < 2400


def test_flame_speed_scales_with_B(oracle_mod):
    # tests/flame1d.mjs calibrate mode: S_L grows like sqrt(B) for a one-step flame
    s1, _ = oracle_mod.flame_speed(B=1e10, dx=5e-5, L=0.03)
    s4, _ = oracle_mod.flame_speed(B=4e10, dx=5e-5, L=0.03)
    assert 1.8 < s4 / s1 < 2.5


@pytest.mark.parametrize("fp64", [False, True])
def test_ambient_is_a_fixed_point(oracle_mod, fp64):
    # reset() state (js/fluid.js:162-176), no wood: every stage leaves it unchanged
    o = oracle_mod.OracleSim(32, 48, 0.7, 0.003, fp64=fp64)
    o.set_solver(oracle_mod.SOLVE_FIXED, 2)
    o.clear_geometry(); o.geometry()
    o.step(3)
    T, Y, U, V = o.read("T"), o.read("Y").reshape(-1, 4), o.read("U"), o.read("V")
    assert np.all(T == np.float32(293.15))
    assert np.all(Y[:, 1] == np.float32(0.232)) and np.all(Y[:, [0, 2, 3]] == 0)
    assert np.all(U == 0) and np.all(V == 0)
    rb = o.readback()
    assert rb["acc"][512] == 0 and rb["acc"][513] == 0 and rb["acc"][514] == 293


def test_geometry_open_fractions(oracle_mod):
    # geometry.wgsl:44-51: fx = clamp(0.5 + d/dx, 0, 1) with d the signed distance to the square
    nx, ny, width = 40, 40, 0.4
    dx = width / nx
    o = oracle_mod.OracleSim(nx, ny, width, 0.002)
    p = np.zeros(64 * 20, np.float32)
    p[0:8] = [0.2, 0.1, 0.0, 0.025, 0, 0, 0, 1]   # square centred on a face line
    p[8:12] = 600
    o.upload_pieces(p, 1)
    o.write_params()
    o.clear_geometry(); o.geometry()
    fx = o.read("fx").reshape(ny, nx + 1)
    fy = o.read("fy").reshape(ny + 1, nx)
    # U face (i, j) at ((i)*dx, (j+0.5)*dx): for j inside the square's y-span the distance is |x-0.2|-0.025
    j = 10   # y = 0.105
    for i in range(nx + 1):
        d = abs(np.float32(i) * np.float32(dx) - np.float32(0.2)) - 0.025
        want = min(max(0.5 + d / dx, 0.0), 1.0)
        assert abs(fx[j, i] - want) < 1e-5, (i, fx[j, i], want)
    assert np.all(fy[0] == 0)                       # floor V faces closed
    assert fx[j, 20] == 0.0                           # face through the centre is closed
    cg = o.read("cellG").reshape(ny, nx, 2)
    # a cell inside: negative sdf and face id of the nearest side
    assert cg[10, 20, 0] < 0 and int(cg[10, 20, 1]) // 4 == 0
    assert int(cg[0, 0, 1]) == 4294967295 or cg[0, 0, 0] > 0


def test_uniform_flow_advects_linear_field_exactly(oracle_mod):
    # advect.wgsl: bilinear sampling is exact for a linear field, so with a uniform
    # velocity the first-order and MacCormack values both equal T(x - u dt) in the interior
    nx, ny, width, dt = 32, 32, 0.32, 0.002
    dx = width / nx
    o = oracle_mod.OracleSim(nx, ny, width, dt, fp64=True)
    u0 = 0.5
    U = np.full((ny, nx + 1), u0)
    o.write("U", U)
    o.write("V", np.zeros((ny + 1, nx)))
    x = (np.arange(nx) + 0.5) * dx
    T = np.tile(400.0 + 1000.0 * x, (ny, 1))
    o.write("T", T)
    o.stage("advect")
    T2 = o.read("T2").reshape(ny, nx)
    # the uniform carries dx and dt as f32 (js/fluid.js:185): the shift in cells is u0*f32(dt)/f32(dx)
    shift = u0 * float(np.float32(dt)) / float(np.float32(dx))
    want = 400.0 + 1000.0 * dx * (np.arange(nx) + 0.5 - shift)
    inner = T2[4:-4, 4:-4]
    assert np.allclose(inner, np.tile(want, (ny, 1))[4:-4, 4:-4], rtol=0, atol=1e-9)


def test_diffusion_conserves_species_at_uniform_temperature(oracle_mod):
    # diffuse.wgsl: antisymmetric face fluxes, zero flux at the domain edges
    nx, ny = 24, 36
    o = oracle_mod.OracleSim(nx, ny, 0.24, 0.002, fp64=True)
    o.clear_geometry(); o.geometry()
    rng = np.random.default_rng(0)
    Y = np.zeros((nx * ny, 4))
    Y[:, 0] = rng.uniform(0, 0.1, nx * ny)
    Y[:, 1] = 0.232 - Y[:, 0]
    o.write("Y2", Y.ravel())
    o.write("T2", np.full(nx * ny, 600.0))
    s0 = Y[:, 0].sum()
    o.stage("diffuse")
    Yd = o.read("Y").reshape(-1, 4)
    assert abs(Yd[:, 0].sum() - s0) < 1e-12 * nx * ny
    assert Yd[:, 0].std() < Y[:, 0].std()


def test_floor_probe_sees_black_ambient(oracle_mod):
    # radiation.wgsl: with transparent gas, an upward floor probe sees only the ambient:
    # q = sum_rays (pi/N) cos(a_k) * sigma Tamb^4 / 2 (first frame: no smoothing)
    nx, ny = 32, 48
    o = oracle_mod.OracleSim(nx, ny, 0.7, 0.003)
    o.set_nray(64)
    o.radiation()
    rad = o.readback()["rad"].reshape(-1, 4)
    N = 64
    q = rad[0, 0]   # first floor probe (no pieces)
    jit = (0 * 0.7548777 + 0 * 0.5698403) % 1.0
    want = sum(math.pi / N * math.cos(((k + jit) / N - 0.5) * math.pi) for k in range(N)) * 5.670374e-8 * 293.15 ** 4 / 2
    assert abs(q - want) / want < 1e-5, (q, want)


def test_fp64_projection_is_divergence_consistent(oracle_mod):
    # dev/gas_test.html:101-111 (H.divErr): after projection div(f u) - S -> 0 as the solve converges
    from campfire_b200.fluid import load_scene
    import campfire_b200 as cb
    sc = cb.generate_scene(0, 64, 96, 0.8, 7)
    o = oracle_mod.OracleSim(64, 96, 0.8, sc["dt"], fp64=True)
    load_scene(o, sc)
    o.set_solver(oracle_mod.SOLVE_TOL, 1, 1e-10, 400)
    o.step(1)
    nx, ny, dx = 64, 96, 0.8 / 64
    U, V = o.read("U").reshape(ny, nx + 1), o.read("V").reshape(ny + 1, nx)
    fx, fy = o.read("fx").reshape(ny, nx + 1), o.read("fy").reshape(ny + 1, nx)
    S = o.read("SQ").reshape(ny, nx, 2)[..., 0]
    div = (fx[:, 1:] * U[:, 1:] - fx[:, :-1] * U[:, :-1] + fy[1:] * V[1:] - fy[:-1] * V[:-1]) / dx
    openc = (fx[:, 1:] + fx[:, :-1] + fy[1:] + fy[:-1]) > 0
    err = np.abs(div - S)[openc]
    assert err.max() < 1e-6 * max(1.0, np.abs(S).max())


def test_direct_coarsest_falls_back_to_sweeps_when_singular(oracle_mod):
    """Direct coarsest solve (TOL/FP64 extension): a pocket sealed on the coarsest level
    makes the operator singular; the oracle then keeps the 120 sweeps, bit for bit."""
    import campfire_b200 as cb
    from campfire_b200.fluid import load_scene
    sc = cb.generate_scene(0, 64, 96, 0.8, 1234)
    res = {}
    for direct, seal in ((False, True), (True, True), (False, False), (True, False)):
        o = oracle_mod.OracleSim(64, 96, 0.8, sc["dt"])
        load_scene(o, sc)
        o.set_solver(oracle_mod.SOLVE_FIXED, 1)
        o.step(3)
        o.set_solver(oracle_mod.SOLVE_TOL, 1, 1e-30, 2)
        o.set_coarse_solve(direct)
        o.stage("coef_rhs")
        L = int(o.info()["levels"]) - 1
        if seal:
            ax, ay = o.read(f"ax.{L}"), o.read(f"ay.{L}")
            cnx, cny = 8, 12   # the coarsest level of 64x96
            ax = ax.reshape(cny, cnx + 1).copy(); ay = ay.reshape(cny + 1, cnx).copy()
            ax[2:4, 2] = 0.0; ax[2:4, 4] = 0.0; ay[2, 2:4] = 0.0; ay[4, 2:4] = 0.0
            o.write(f"ax.{L}", ax.ravel()); o.write(f"ay.{L}", ay.ravel())
        o.stage("pressure")
        res[(direct, seal)] = o.read("p")
    assert np.array_equal(res[(True, True)], res[(False, True)])        # singular: sweeps
    assert not np.array_equal(res[(True, False)], res[(False, False)])  # regular: the inverse
