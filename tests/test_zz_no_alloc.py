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


def test_noalloc_rejects_grids_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    x = torch.zeros(16, device=dev)
    rel = ctypes.c_double()
    p = ctypes.c_void_p(x.data_ptr())
    rc = cb.lib().cfg_pressure_residual_noalloc(p, p, p, p, 2048, 1024, 1e-6, None, ctypes.byref(rel))
    assert rc == -34 and "1048576" in _lib.last_error()
