"""The serving loop (cfg_server_*): continuous batching of jobs of several sizes.

Each job's final state must not depend on the other jobs in the batch: the same
job alone, in a mix, under a budget that serialises the jobs, and through the
plain single-scene FluidSim gives bit-identical fields (equal FNV-1a hashes of
T, Y, U, V).
"""
import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu
CLASSES = [(64, 96), (96, 144)]
SOLVER = dict(mode=cb.SOLVE_FP64, ncycles=1, tol=1e-8, max_cycles=60, coarse_direct=True)


def jobs():
    rng = np.random.default_rng(7)
    out, t = [], 0.0
    for k in range(7):
        t += float(rng.exponential(0.01))
        out.append({"size_class": int(rng.integers(0, 2)), "kind": int(rng.integers(1, 3)), "seed": 9000 + k,
                    "nsteps": int(rng.integers(2, 7)), "arrival_s": t})
    return out


def serve(js, slots=(2, 2), budget=64e9):
    s = cb.Server(CLASSES, list(slots), budget)
    s.set_solver(**SOLVER)
    res, wall, cu = s.run(js)
    s.close()
    return res, wall, cu


def test_results_do_not_depend_on_the_mix():
    js = jobs()
    mixed, wall, cu = serve(js)
    assert cu == sum(CLASSES[j["size_class"]][0] * CLASSES[j["size_class"]][1] * j["nsteps"] for j in js)
    for j, r in zip(js, mixed):
        assert r["steps"] == j["nsteps"] and r["done_s"] >= r["admit_s"] >= r["arrival_s"] - 1e-9
        assert r["last_rel"] <= 1e-8
    for j, r in zip(js, mixed):
        alone, _, _ = serve([dict(j, arrival_s=0.0)])
        assert alone[0]["hash"] == r["hash"], j


def test_budget_admission_serialises_jobs_without_changing_results():
    js = jobs()
    mixed, _, _ = serve(js)
    s = cb.Server(CLASSES, [2, 2], 1e9)
    nbytes = [s.slot_bytes(0), s.slot_bytes(1)]
    s.close()
    budget = max(nbytes)   # the largest job alone
    tight, _, _ = serve(js, budget=budget)
    # at every admission, the resident jobs' slots fit in the budget
    for r in tight:
        t = r["admit_s"]
        resident = sum(nbytes[j["size_class"]] for j, q in zip(js, tight) if q["admit_s"] <= t < q["done_s"])
        assert resident <= budget
    assert [r["hash"] for r in tight] == [r["hash"] for r in mixed]


def test_server_matches_the_plain_step():
    j = {"size_class": 1, "kind": 1, "seed": 9100, "nsteps": 4, "arrival_s": 0.0}
    res, _, _ = serve([j])
    nx, ny = CLASSES[1]
    sc = cb.generate_scene(1, nx, ny, 0.8, 9100)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    g.set_solver(SOLVER["mode"], 1, SOLVER["tol"], SOLVER["max_cycles"])
    g.set_coarse_solve(True)
    g.step(4)
    assert cb.field_hash(g) == res[0]["hash"]
    g.close()


def test_bad_jobs_are_rejected():
    s = cb.Server(CLASSES, [1, 1], 64e9)
    with pytest.raises(cb.CampfireError):
        s.run([{"size_class": 5, "seed": 1, "nsteps": 2, "arrival_s": 0.0}])
    with pytest.raises(cb.CampfireError):
        s.run([{"size_class": 0, "seed": 1, "nsteps": 0, "arrival_s": 0.0}])
    s.close()
    small = cb.Server(CLASSES, [1, 1], 1e3)   # no slot fits the budget
    with pytest.raises(cb.CampfireError) as e:
        small.run([{"size_class": 0, "seed": 1, "nsteps": 2, "arrival_s": 0.0}])
    assert e.value.code == -34
    small.close()


def fnv(arrays):
    h = 1469598103934665603
    for a in arrays:
        for b in np.ascontiguousarray(a, np.float32).tobytes():
            h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def test_submitted_jobs_match_the_batch_run():
    """The service thread (cfg_server_submit / poll / wait / fetch): jobs handed over one at a
    time while others run give the same results as the list run, and kept fields hash to the
    reported hash."""
    import threading
    import time
    js = jobs()
    ref, _, _ = serve(js)
    s = cb.Server(CLASSES, [2, 2], 64e9)
    s.set_solver(**SOLVER)
    tickets = [None] * len(js)

    def client():   # a second host thread submits while the first polls
        for k, j in enumerate(js):
            tickets[k] = s.submit(j["size_class"], j["kind"], j["seed"], j["nsteps"], keep_fields=(k == 0))
            time.sleep(0.005)
    th = threading.Thread(target=client)
    th.start()
    th.join()
    got = {}
    deadline = time.time() + 120
    while len(got) < len(js) and time.time() < deadline:
        for k, t in enumerate(tickets):
            if k not in got:
                r = s.poll(t)
                if r is not None:
                    got[k] = r
        time.sleep(0.002)
    assert len(got) == len(js)
    for k, j in enumerate(js):
        assert got[k]["hash"] == ref[k]["hash"], j
        assert got[k]["steps"] == j["nsteps"] and got[k]["done_s"] >= got[k]["admit_s"] >= got[k]["arrival_s"]
    nx, ny = CLASSES[js[0]["size_class"]]
    fields = [s.fetch(tickets[0], "T", nx * ny), s.fetch(tickets[0], "Y", 4 * nx * ny),
              s.fetch(tickets[0], "U", (nx + 1) * ny), s.fetch(tickets[0], "V", nx * (ny + 1))]
    assert fnv(fields) == got[0]["hash"]
    s.release(tickets[0])
    with pytest.raises(cb.CampfireError, match="NOENT"):
        s.fetch(tickets[0], "T", nx * ny)
    with pytest.raises(cb.CampfireError, match="NOENT"):
        s.poll(tickets[1])               # already taken
    # wait() on a fresh job, then drain; a new submission restarts the service
    t = s.submit(0, 1, 4242, 3)
    r = s.wait(t, 60.0)
    assert r["steps"] == 3
    s.drain()
    t = s.submit(1, 2, 4243, 2)
    assert s.wait(t, 60.0)["steps"] == 2
    with pytest.raises(cb.CampfireError, match="BUSY"):
        s.submit(0, 1, 1, 400)
        s.set_solver(**SOLVER)
    s.close()


@pytest.mark.parametrize("krylov", [1, 2])
def test_krylov_results_do_not_depend_on_the_mix(krylov):
    """The FP64 loop by flexible CG, with its update as its own kernel (1) or folded into the
    level-0 kernels (2): each scene still decides its own solve, so a job's bits do not depend
    on the jobs beside it."""
    js = jobs()[:4]
    s = cb.Server(CLASSES, [2, 2], 64e9)
    s.set_solver(**dict(SOLVER, coarse_direct="pipelined", coarse_cells=1536, krylov=krylov))
    mixed, _, _ = s.run(js)
    alone = []
    for j in js:
        r, _, _ = s.run([dict(j, arrival_s=0.0)])
        alone.append(r[0]["hash"])
    s.close()
    assert [r["hash"] for r in mixed] == alone


def test_pipelined_coarse_solve_keeps_results_independent_of_the_mix():
    """With the pipelined coarsest inverse a slot's inverse belongs to its own scene: a job
    admitted into a used slot starts without one (reset), so mixes and reuse change nothing."""
    js = jobs()[:4]
    s = cb.Server(CLASSES, [1, 1], 64e9)
    s.set_solver(**dict(SOLVER, coarse_direct="pipelined"))
    mixed, _, _ = s.run(js)
    alone = []
    for j in js:
        r, _, _ = s.run([dict(j, arrival_s=0.0)])
        alone.append(r[0]["hash"])
    s.close()
    assert [r["hash"] for r in mixed] == alone
