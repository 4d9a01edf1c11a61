"""The asynchronous readback ring (encodeReadback + afterSubmit, js/fluid.js:315-342) through the
C ABI: three pinned staging slots filled on the stream, handed out oldest first with their tags,
and the reference's skip (no copy, acc keeps accumulating) while the next slot is still pending."""
import numpy as np
import pytest

import campfire_b200 as cb
from campfire_b200.fluid import load_scene

pytestmark = pytest.mark.gpu


def _sim(nx=128, ny=192):
    sc = cb.generate_scene(0, nx, ny, 0.8, 1234)
    g = cb.FluidSim(0, {"nx": nx, "ny": ny, "dt": sc["dt"]}, width=0.8).init()
    load_scene(g, sc)
    g.set_solver(cb.SOLVE_FIXED, 2)
    return g


def _same(a, b):
    return all(np.array_equal(a[k], b[k]) for k in ("acc", "rad", "faceW"))


def test_ring_gives_the_synchronous_readbacks_in_order():
    a, b = _sim(), _sim()
    want, got = [], []
    for k in range(5):
        a.step(1)
        want.append(a.readback())
        b.step(1)
        assert b.encodeReadback(tag=100 + k) is not None
        if k % 2 == 1:                       # collect two at a time: the ring holds them meanwhile
            while (r := b.pollReadback(wait=True)) is not None:
                got.append(r)
    while (r := b.pollReadback(wait=True)) is not None:
        got.append(r)
    assert [t for _, t in got] == [100 + k for k in range(5)]
    for k in range(5):
        assert _same(got[k][0], want[k]), k
    assert any(np.any(w["acc"] != 0) for w in want)   # the steps did accumulate something
    a.close(); b.close()


def test_busy_slot_skips_the_readback_and_acc_keeps_accumulating():
    a, b = _sim(), _sim()
    for k in range(3):                      # three readbacks in flight fill the ring
        a.step(1); a.readback()
        b.step(1)
        assert b.encodeReadback(tag=k) == k % 3
    a.step(1)                               # frame 4: the reference skips its readback
    b.step(1)
    assert b.encodeReadback(tag=3) is None
    tags = []
    while (r := b.pollReadback(wait=True)) is not None:
        tags.append(r[1])
    assert tags == [0, 1, 2]
    a.step(1)                               # frame 5: its readback holds steps 4 and 5
    want = a.readback()
    b.step(1)
    assert b.encodeReadback(tag=4) is not None
    got, tag = b.pollReadback(wait=True)
    assert tag == 4 and _same(got, want)
    a.close(); b.close()


def test_frames_receive_their_readbacks_late():
    """The app's pattern: each frame enqueues its step and its readback, then takes whatever has
    arrived (js/main.js:283 with the callback of :210). A frame never waits for its own step, so
    results arrive frames later, in order; a frame whose slot is still pending skips its readback."""
    g = _sim(256, 384)
    arrived, order, skipped = {}, [], set()
    for frame in range(12):
        g.step(1)
        if g.encodeReadback(tag=frame) is None:
            skipped.add(frame)
        while (r := g.pollReadback()) is not None:
            arrived[r[1]] = frame
            order.append(r[1])
    while (r := g.pollReadback(wait=True)) is not None:
        arrived[r[1]] = 12
        order.append(r[1])
    assert order == sorted(order) and len(order) == len(set(order))
    assert set(arrived) | skipped == set(range(12)) and not (set(arrived) & skipped)
    assert all(arrived[t] >= t for t in arrived)
    assert max(arrived[t] - t for t in arrived) >= 1    # collected frames after its own
    g.close()
