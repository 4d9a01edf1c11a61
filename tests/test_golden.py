"""The CPU oracle against the golden fixtures.

The fixtures (tests/golden/*.npz, written by tests/golden/make_golden.py) hold
outputs of the reference's own WGSL kernels, translated mechanically to C++ and
run in FluidSim's dispatch order (js/fluid.js:225-253). The restatement used as
the parity oracle must reproduce every one of them bit for bit: geometry, every
stage of a step, the acc readback of each step, the state after several steps
and the radiation pass.
"""
import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "*.npz")))
STATE = ("T", "Y", "U", "V", "T2", "Y2", "U2", "V2", "SQ", "p")
STAGES = ("advect", "diffuse", "sources", "forces", "coef_rhs", "pressure", "project")


def load(path):
    with np.load(path) as z:
        return {k: z[k] for k in z.files}


def apply_inputs(sim, d):
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


def new_sim(om, d, impl="restatement"):
    nx, ny = (int(v) for v in d["meta_dims"])
    s = om.OracleSim(nx, ny, float(d["meta_width"]), float(d["meta_dt"]), impl=impl)
    apply_inputs(s, d)
    return s


def check_fixture(s, d):
    assert int(s.info()["levels"]) == int(d["meta_levels"])
    assert int(s.info()["diffSub"]) == int(d["meta_diffsub"])
    cg = s.read("cellG").reshape(-1, 2)
    np.testing.assert_array_equal(cg[:, 0].astype(np.float32), d["geo_cellG_sdf"])
    np.testing.assert_array_equal(cg[:, 1].astype(np.uint32), d["geo_cellG_id"])
    np.testing.assert_array_equal(s.read("fx").astype(np.float32), d["geo_fx"])
    np.testing.assert_array_equal(s.read("fy").astype(np.float32), d["geo_fy"])
    np.testing.assert_array_equal(s.readback()["faceW"], d["geo_faceW"])
    for i in range(int(d["meta_steps"])):
        s.set_frame(i)
        s.write_params()
        s.step()
        np.testing.assert_array_equal(s.readback()["acc"], d["acc"][i], err_msg=f"acc of step {i}")
    for k in d:
        if k.startswith("fin_"):
            np.testing.assert_array_equal(s.read(k[4:]).astype(np.float32), d[k], err_msg=k)
    s.set_frame(int(d["meta_steps"]))
    s.write_params()
    for st in STAGES:
        s.stage(st)
        for k in d:
            if k.startswith(f"st_{st}_"):
                np.testing.assert_array_equal(s.read(k[len(st) + 4:]).astype(np.float32), d[k], err_msg=k)
    np.testing.assert_array_equal(s.readback()["acc"], d["st_acc"])
    s.radiation()
    np.testing.assert_array_equal(s.readback()["rad"], d["rad"])


def test_fixtures_present():
    assert len(FIXTURES) >= 3
    for f in FIXTURES:
        d = load(f)
        assert d["acc"].shape == (int(d["meta_steps"]), 528)
        # the scenes are not at rest: the fixtures exercise flow, reaction and radiation
        assert np.abs(d["fin_V"]).max() > 0.1
        assert d["fin_T"].max() > float(d["in_T"].min()) + 100
        assert np.abs(d["rad"]).max() > 0


@pytest.mark.parametrize("path", FIXTURES, ids=[os.path.basename(f)[:-4] for f in FIXTURES])
def test_restatement_reproduces_reference(oracle_mod, path):
    d = load(path)
    s = new_sim(oracle_mod, d)
    try:
        check_fixture(s, d)
    finally:
        s.close()


@pytest.mark.parametrize("path", FIXTURES[:1], ids=[os.path.basename(f)[:-4] for f in FIXTURES[:1]])
def test_translated_reference_reproduces_fixture(oracle_mod, path):
    """Where oracle/_ref is built, the translated WGSL still writes the committed fixture."""
    if not os.path.exists(oracle_mod.REF_LIB_PATH):
        pytest.skip("oracle/_ref not built (needs the reference checkout)")
    d = load(path)
    s = new_sim(oracle_mod, d, impl="wgsl")
    try:
        check_fixture(s, d)
    finally:
        s.close()
