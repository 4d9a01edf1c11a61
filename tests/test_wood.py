"""The wood model of js/wood.js in the library (C++, through the C ABI) against the
oracle's independent Python restatement, on the scenarios of the reference's own
wood test (tests/wood_test.mjs: a 2.5 cm stick and a 5 cm log under 30 kW/m2 and
1100 K gas, a stick in cold air), with its crude char oxidation. CPU only.
"""
import math

import pytest

from campfire_b200.wood import WoodPiece
from oracle.wood_ref import WoodPiece as RefPiece

SIG = 5.670374e-8


def run(cls, side, qFlux, Tgas, h, seconds, charOx=0.0):
    w = cls(side, 500)
    dt = 1 / 60
    t, tign, peak, trace = 0.0, None, 0.0, []
    while t < seconds and not w.dead:
        s = w.side
        Ts = list(w.Ts)
        qConv = [h * s * (Tgas - T) for T in Ts]
        qInc = [qFlux + SIG * 293.15 ** 4] * 4
        cc = list(w.charCov)
        burnt = [charOx * cc[f] * 470 * math.exp(-12000 / Ts[f]) * 0.27 * s * dt / 2.667 for f in range(4)]
        w.step(dt, qConv, qInc, burnt, 0.25, 1.0)
        mf = sum(w.mflux) / 4
        peak = max(peak, mf)
        if tign is None and mf > 0.0025:
            tign = t
        trace.append((w.side, w.mv, w.mc, w.Tc, *w.Ts, *w.Tp, *w.d, *w.mflux))
        t += dt
    return tign, peak, trace


@pytest.mark.parametrize("side,q,Tg,h,secs,ox", [(0.025, 30000, 1100, 25, 120, 0.0), (0.05, 30000, 1100, 25, 60, 0.0),
                                                 (0.025, 0, 293, 10, 30, 0.0), (0.025, 30000, 1100, 25, 90, 1.0)])
def test_library_matches_restatement(side, q, Tg, h, secs, ox):
    a = run(WoodPiece, side, q, Tg, h, secs, ox)
    b = run(RefPiece, side, q, Tg, h, secs, ox)
    assert (a[0] is None) == (b[0] is None)
    if a[0] is not None:
        assert abs(a[0] - b[0]) < 1e-9
    assert len(a[2]) == len(b[2])
    for ra, rb in zip(a[2], b[2]):
        for x, y in zip(ra, rb):
            assert abs(x - y) <= 1e-9 * max(abs(y), 1e-3), (x, y)


def test_stick_ignites_under_flux_and_not_in_cold_air():
    tign, peak, _ = run(WoodPiece, 0.025, 30000, 1100, 25, 120)
    assert tign is not None and 5 < tign < 120 and peak > 0.0025
    tcold, _, trace = run(WoodPiece, 0.025, 0, 293, 10, 30)
    assert tcold is None and abs(trace[-1][4] - 293.15) < 1.0


def test_preheat_makes_a_charred_hot_piece():
    w = WoodPiece(0.05, 500)
    r = RefPiece(0.05, 500)
    w.preheat(900, 0.004, 500, 0.25)
    r.preheat(900, 0.004, 500, 0.25)
    assert w.Ts == r.Ts and w.d == r.d and abs(w.side - r.side) == 0.0
    assert w.mc > 0 and w.side < 0.05
