"""The allocation-free residual check, through the C ABI, against cfg_pressure_residual.

cfg_pressure_residual_noalloc serves callers that cannot allocate device memory
when they need the check (their memory is committed to scenes already, or they
must not stall on the device-wide synchronisation an allocation can cause). It
must agree with the allocating entry point on the same pressure field, on
consecutive calls that share its fixed scratch array. This file is collected
last so that a run stopping at the first failure has run every other test.
"""
import ctypes

import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200 import _lib
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu

REL_TOL = 1e-9   # both sum f32 residuals in FP64; only the summation order differs


def _device_copy(torch, arr, dev):
    return torch.from_numpy(np.ascontiguousarray(arr, dtype=np.float32)).to(dev)


@pytest.mark.parametrize("nx,ny,kind,seed", [(128, 192, 0, 1234), (96, 144, 2, 2002)])
def test_noalloc_residual_matches_allocating_entry_point(nx, ny, kind, seed):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    sc = cb.generate_scene(kind, nx, ny, 0.8, seed)
    sim = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(sim, sc)
    sim.set_solver(cb.SOLVE_FIXED, 1)
    L = cb.lib()
    try:
        for _ in range(2):   # two steps, a check after each: consecutive calls reuse the scratch
            sim.step(1)
            want = sim.pressure_residual()
            bufs = {f: _device_copy(torch, sim.readBuffer(f), dev) for f in ("p", "rhs", "ax", "ay")}
            torch.cuda.synchronize(dev)
            h2 = (0.8 / nx) ** 2
            for call in range(2):
                rel = ctypes.c_double(-1.0)
                rc = L.cfg_pressure_residual_noalloc(
                    ctypes.c_void_p(bufs["p"].data_ptr()), ctypes.c_void_p(bufs["rhs"].data_ptr()),
                    ctypes.c_void_p(bufs["ax"].data_ptr()), ctypes.c_void_p(bufs["ay"].data_ptr()),
                    nx, ny, h2, ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream), ctypes.byref(rel))
                _lib.check(rc)
                assert want > 0
                assert abs(rel.value - want) <= REL_TOL * want, (call, rel.value, want)
    finally:
        sim.close()


def _residual_fp64(p, rhs, ax, ay, nx, ny, h2):
    """The residual sums of pressure.wgsl:77-101 in numpy: r in f32 with the kernel's operation order
    (each product and sum rounded separately), the squares summed in FP64."""
    f32 = np.float32
    P = p.reshape(ny, nx)
    AX = ax.reshape(ny, nx + 1)
    AY = ay.reshape(ny + 1, nx)
    w, e, s, n = AX[:, :-1], AX[:, 1:], AY[:-1, :], AY[1:, :]
    off = np.zeros((ny, nx), f32)
    diag = np.zeros((ny, nx), f32)
    pl = np.zeros_like(P); pl[:, 1:] = P[:, :-1]
    pr = np.zeros_like(P); pr[:, :-1] = P[:, 1:]
    pb = np.zeros_like(P); pb[1:, :] = P[:-1, :]
    pt = np.zeros_like(P); pt[:-1, :] = P[1:, :]
    col = np.arange(nx)[None, :]
    row = np.arange(ny)[:, None]
    m = (col > 0)
    off = np.where(m, off + w * pl, off); diag = np.where(m, diag + w, diag + f32(2) * w)
    m = (col < nx - 1)
    off = np.where(m, off + e * pr, off); diag = np.where(m, diag + e, diag + f32(2) * e)
    m = (row > 0)
    off = np.where(m, off + s * pb, off); diag = np.where(m, diag + s, diag)
    m = (row < ny - 1)
    off = np.where(m, off + n * pt, off); diag = np.where(m, diag + n, diag + f32(2) * n)
    R = rhs.reshape(ny, nx)
    r = np.where(diag <= 0, f32(0), R - (off - diag * P) / f32(h2)).astype(f32)
    return float(np.sum(r.astype(np.float64) ** 2)), float(np.sum(R.astype(np.float64) ** 2))


@pytest.mark.parametrize("nx,ny", [(1024, 1024), (700, 900)])
def test_noalloc_residual_at_and_below_the_block_limit(nx, ny):
    """1024x1024 fills exactly the 4096 blocks the scratch holds; 700x900 (2461 blocks) makes every
    thread of the combine kernel sum several partials. Random coefficients with closed faces (zeros)."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(nx + ny)
    f32 = np.float32
    p = rng.standard_normal(nx * ny).astype(f32)
    rhs = rng.standard_normal(nx * ny).astype(f32)
    ax = (rng.random((nx + 1) * ny) * (rng.random((nx + 1) * ny) > 0.1)).astype(f32)
    ay = (rng.random(nx * (ny + 1)) * (rng.random(nx * (ny + 1)) > 0.1)).astype(f32)
    h2 = (0.8 / nx) ** 2
    rr, bb = _residual_fp64(p, rhs, ax, ay, nx, ny, h2)
    want = np.sqrt(rr / bb)
    bufs = [_device_copy(torch, a, dev) for a in (p, rhs, ax, ay)]
    torch.cuda.synchronize(dev)
    L = cb.lib()
    for call in range(2):
        rel = ctypes.c_double(-1.0)
        _lib.check(L.cfg_pressure_residual_noalloc(*[ctypes.c_void_p(b.data_ptr()) for b in bufs], nx, ny, h2,
                                                   ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream),
                                                   ctypes.byref(rel)))
        assert abs(rel.value - want) <= REL_TOL * want, (call, rel.value, want)


def test_noalloc_rejects_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x = torch.zeros(16, device=dev)
    rel = ctypes.c_double()
    p = ctypes.c_void_p(x.data_ptr())
    rc = cb.lib().cfg_pressure_residual_noalloc(p, p, p, p, 2048, 1024, 1e-6, None, ctypes.byref(rel))
    assert rc == -34 and "1048576" in _lib.last_error()
