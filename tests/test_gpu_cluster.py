"""The cluster coarse phase (k_mg_cluster, cfg_set_coarse_cluster): levels lc..coarsest
shared out over a thread-block cluster give bit-identical fields to the one-CTA coarse
block, for cluster sizes 2 to 16, coarse phases starting at level 1 or deeper, the direct
coarsest solve and the reference's sweeps. The thresholds keep level 0 out of the
one-CTA block too (a block that covers level 0 also finishes the cycle's FP64 dot
products, in another summation order)."""
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu


def run(nx, ny, kind, cs, cells, mode, steps, coarse):
    sc = cb.generate_scene(kind, nx, ny, 0.8, 4000 + nx)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    if mode == "fixed":
        g.set_solver(cb.SOLVE_FIXED, 1)
    else:
        g.set_solver(cb.SOLVE_FP64, 1, 1e-8, 100)
        g.set_krylov(True)
        g.set_coarse_solve(coarse)
    g.set_coarse_cells(cells)
    g.set_coarse_cluster(cs)
    g.step(steps)
    g.synchronize()
    out = (cb.field_hash(g), g.read_p64().tobytes() if mode != "fixed" else b"", g.info()["last_cycles"])
    g.close()
    return out


@pytest.mark.parametrize("nx,ny,kind,cells", [(256, 384, 0, 24576), (256, 384, 0, 1536), (96, 144, 2, 6144),
                                              (64, 96, 1, 1536)])
@pytest.mark.parametrize("cs", [4, 16])
def test_cluster_matches_the_one_cta_block(nx, ny, kind, cells, cs):
    ref = run(nx, ny, kind, 0, cells, "fp64", 3, "pipelined")
    got = run(nx, ny, kind, cs, cells, "fp64", 3, "pipelined")
    assert got == ref


@pytest.mark.parametrize("cs", [2, 8])
def test_cluster_matches_with_the_reference_sweeps(cs):
    # one fixed V-cycle per step: the coarsest by 120 sweeps on one CTA of the cluster
    ref = run(128, 192, 0, 0, 24576, "fixed", 4, False)
    got = run(128, 192, 0, cs, 24576, "fixed", 4, False)
    assert got == ref


def test_cluster_size_is_checked():
    sc = cb.generate_scene(0, 64, 96, 0.8, 1)
    g = cb.FluidSim(0, {"nx": 64, "ny": 96, "dt": sc["dt"]}, width=0.8).init()
    with pytest.raises(cb.CampfireError, match="INVAL"):
        g.set_coarse_cluster(3)
    g.set_coarse_cluster(8)
    g.set_coarse_cluster(0)
    g.close()
