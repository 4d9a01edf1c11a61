"""ORACLE — test infrastructure, not product code.

Python restatement of the reference's wood model (js/wood.js: WOOD :12-31,
WoodPiece :33-182) and of the frame coupling of js/main.js (addPiece :103-119,
uploadPieces :190-207, onReadback :209-230, stepWood :232-243, the gas part of
frame() :247-283) driving the CPU gas-step oracle. Python floats are IEEE
doubles evaluated left to right, as JS numbers are.
"""
from __future__ import annotations

import math

import numpy as np

from .rigid_ref import exchange_contacts

WOOD = dict(cv=1500, kv=0.15, cc=1000, kc=0.08, pore=0.001, charDensityRatio=0.3, eps=0.9, pyroA=2.0e7,
            pyroTa=12000, dHpyro=3.0e5, dHchar=32.8e6, cpGas=1150, deltaS=0.0015, deltaP=0.002, minDepth=0.0004,
            sigma=5.670374e-8, minHalf=0.0015)
E_SCALE, M_SCALE, G_SCALE = 1e6, 1e12, 1e3          # js/fluid.js:9
ACC_GLOBAL = 512
TAMB, SIGMA = 293.15, 5.670374e-8                   # js/config.js PHYS


class WoodPiece:
    def __init__(self, side, rhoV, T0=293.15):
        self.rhoV = rhoV
        self.rhoC = rhoV * WOOD["charDensityRatio"]
        self.mv = rhoV * side * side
        self.mc = 0.0
        self.Ts = [T0] * 4
        self.Tp = [T0] * 4
        self.d = [0.0] * 4
        self.Tc = T0
        self.mflux = [0.0] * 4
        self.charCov = [0.0] * 4
        self.gasRate = 0.0
        self.exposure = [1.0] * 4
        self.dead = False
        self.side = side

    @property
    def half(self):
        return 0.5 * self.side

    def updateSide(self):
        self.side = math.sqrt(self.mv / self.rhoV + self.mc / self.rhoC)

    def preheat(self, Tsurf, charDepth, Tcore, charYield):
        s = self.side
        dv = min(charDepth, 0.45 * s)
        vVol = 4 * dv * s - 4 * dv * dv
        consumed = min(self.mv * 0.98, vVol * self.rhoV)
        self.mv -= consumed
        self.mc += consumed * charYield
        self.d = [dv] * 4
        self.Ts = [Tsurf] * 4
        self.Tp = [0.5 * (t + Tcore) for t in self.Ts]
        self.Tc = Tcore
        self.updateSide()

    def step(self, dt, qConv, qInc, charBurnt, charYield=0.25, pyroMult=1.0):
        if self.dead:
            return
        W, Yc = WOOD, charYield
        qChar = [0.0] * 4
        for f in range(4):
            m = min(charBurnt[f], self.mc)
            self.mc -= m
            qChar[f] = m * W["dHchar"] / dt
            self.d[f] = max(0.0, self.d[f] - m / (self.rhoC * max(self.side, 1e-3)))
        self.updateSide()
        nsub = max(1, math.ceil(dt / 0.004))
        h = dt / nsub
        gasTotal = 0.0
        gasFace = [0.0] * 4
        for _ in range(nsub):
            s = self.side
            dS, dP = min(W["deltaS"], s / 8), min(W["deltaP"], s / 8)
            allChar = self.mv <= 1e-9
            rcv, rcc = self.rhoV * W["cv"], self.rhoC * W["cc"]
            Cs, Cp, Csum = [0.0] * 4, [0.0] * 4, 0.0
            for f in range(4):
                phi = 1 if allChar else min(1, self.d[f] / dS)
                Cs[f] = (rcv * (1 - phi) + rcc * phi) * dS * s
                Cp[f] = (rcc if allChar else rcv) * dP * s
                Csum += Cs[f] + Cp[f]
            Ctot = self.mv * W["cv"] + self.mc * W["cc"]
            Cc = max(0.1 * Ctot, Ctot - Csum)
            A = W["pyroA"] * pyroMult
            mFrontCap = self.rhoV * dP * s
            mFrontSum = 0.0
            rf = [0.0] * 4
            for f in range(4):
                mFront = min(mFrontCap, self.mv / 5)
                mFrontSum += mFront
                rf[f] = A * math.exp(-W["pyroTa"] / self.Tp[f]) * mFront
            rCore = A * math.exp(-W["pyroTa"] / self.Tc) * max(0.0, self.mv - mFrontSum)
            rTot = rf[0] + rf[1] + rf[2] + rf[3] + rCore
            if rTot * h > self.mv:
                k = self.mv / (rTot * h)
                rf = [r * k for r in rf]
                rTot *= k
            rC = rTot - (rf[0] + rf[1] + rf[2] + rf[3])
            kv = W["kc"] if allChar else W["kv"]
            coreIn = 0.0
            for f in range(4):
                d = self.d[f]
                Tm = 0.5 * (self.Ts[f] + self.Tp[f])
                kcEff = W["kc"] + 4 * W["eps"] * W["sigma"] * Tm * Tm * Tm * W["pore"]
                Gsp = s / (d / kcEff + (dS + dP) / (2 * kv))
                Lpc = max(0.5 * (0.5 * s - d), 0.001)
                Gpc = kv * s / Lpc
                gas = (1 - Yc) * (rf[f] + 0.25 * rC)
                gasFace[f] += gas * h
                Ts, Tp = self.Ts[f], self.Tp[f]
                eps, ex = W["eps"], self.exposure[f]
                qRad = eps * s * ex * (qInc[f] - W["sigma"] * Ts * Ts * Ts * Ts)
                dRad = 4 * eps * W["sigma"] * Ts * Ts * Ts * s * ex
                qs = qConv[f] + qRad + qChar[f] - Gsp * (Ts - Tp) - gas * W["cpGas"] * (Ts - Tp)
                self.Ts[f] = Ts + h * qs / (Cs[f] + h * (dRad + Gsp))
                qp = Gsp * (Ts - Tp) - Gpc * (Tp - self.Tc) - W["dHpyro"] * rf[f]
                self.Tp[f] = Tp + h * qp / (Cp[f] + h * (Gsp + Gpc))
                coreIn += Gpc * (Tp - self.Tc)
                if not allChar:
                    self.d[f] = min(0.5 * s, self.d[f] + rf[f] * h / (self.rhoV * s))
            self.Tc += h * (coreIn - W["dHpyro"] * rC) / Cc
            self.mv -= rTot * h
            self.mc += Yc * rTot * h
            if self.mv < 1e-9:
                self.mv = 0.0
            gasTotal += (1 - Yc) * rTot * h
            self.updateSide()
        self.gasRate = gasTotal / dt
        s = max(self.side, 1e-4)
        ex = self.exposure
        exSum = ex[0] + ex[1] + ex[2] + ex[3]
        blocked = 0.0
        for f in range(4):
            blocked += gasFace[f] * (1 - ex[f])
        for f in range(4):
            g = gasFace[f] * ex[f] + (blocked * ex[f] / exSum if exSum > 0.05 else 0)
            self.mflux[f] = g / dt / s if ex[f] > 0.02 else 0.0
            self.charCov[f] = 1 if self.mv <= 0 else min(1, self.d[f] / WOOD["minDepth"])
        if self.half < WOOD["minHalf"] or (self.mv + self.mc) < 1e-7:
            self.dead = True


class WoodScene:
    """The frame loop of js/main.js for frozen pieces, over an OracleSim."""

    def __init__(self, sim, charYield=0.25, pyroMult=1.0, world=None, lag=0):
        """world: an oracle.rigid_ref.RigidWorld for moving pieces (None: frozen).
        lag: 0 applies each frame's readback at its end; 1..3 applies it at the start of the frame `lag`
        frames later, before the wood steps, with its own frame's gas time and only to the pieces that
        held the slots then (afterSubmit's tag and onReadback, js/fluid.js:327-342, js/main.js:210-230,
        with a fixed delay instead of the GPU's timing)."""
        self.sim, self.charYield, self.pyroMult, self.world = sim, charYield, pyroMult, world
        self.slots = [None] * 64
        self.simAcc = 0.0
        self.frame_no = 0
        self.hrr = self.rad = self.tmax = 0.0
        self.lag, self.queue = lag, []

    def add(self, x, y, angle, side, density, preheat=None, faceT=None):
        s = self.slots.index(None)
        w = WoodPiece(side, density)
        if preheat:
            w.preheat(*preheat, self.charYield)
        if faceT:
            for f, T in enumerate(faceT):
                if T:
                    w.Ts[f] = T
                    w.Tp[f] = max(w.Tp[f], 0.5 * (T + w.Tc))
        qa = SIGMA * TAMB ** 4
        self.slots[s] = dict(x=x, y=y, angle=angle, wood=w, qConv=[0.0] * 4, qInc=[qa] * 4, vis=[0.0] * 4,
                             charPending=[0.0] * 4, body=None)
        if self.world is not None:   # new Body(x, y, half, (mv + mc) / side^2, angle), js/main.js:109-110
            b = self.world.add(x, y, w.half, (w.mv + w.mc) / (w.side * w.side), angle)
            b.user = w
            self.slots[s]["body"] = b
        return s

    def upload(self):
        data = np.zeros(64 * 20, np.float32)
        n = 0
        for s, p in enumerate(self.slots):
            if p is None:
                continue
            w, b = p["wood"], p["body"]
            if b is not None:
                data[s * 20:s * 20 + 8] = [b.x, b.y, b.a, b.half, b.vx, b.vy, b.w, 1]
            else:
                data[s * 20:s * 20 + 8] = [p["x"], p["y"], p["angle"], w.half, 0, 0, 0, 1]
            data[s * 20 + 8:s * 20 + 12] = w.Ts
            data[s * 20 + 12:s * 20 + 16] = w.mflux
            data[s * 20 + 16:s * 20 + 20] = w.charCov
            n = s + 1
        self.sim.upload_pieces(data, n)

    def frame(self, sim_dt):
        dt = self.sim.info()["dt"]
        self.simAcc += sim_dt
        maxSteps = math.ceil(0.034 / dt)
        n = math.floor(self.simAcc / dt)
        if n > maxSteps:
            n, self.simAcc = maxSteps, 0.0
        else:
            self.simAcc -= n * dt
        simDt = n * dt
        while self.lag and len(self.queue) >= self.lag:   # the readback of the frame `lag` frames back
            rb_, simDt_, owners_ = self.queue.pop(0)
            self.apply(rb_, simDt_, owners_)
        if self.world is not None:   # js/main.js:262-263
            self.world.advance(simDt)
            exchange_contacts(self.world, simDt)
        if simDt > 0:
            for s, p in enumerate(self.slots):
                if p is None:
                    continue
                w = p["wood"]
                w.step(simDt, p["qConv"], p["qInc"], p["charPending"], self.charYield, self.pyroMult)
                p["charPending"] = [0.0] * 4
                if w.dead:
                    if p["body"] is not None:
                        self.world.remove(p["body"])
                    self.slots[s] = None
                    continue
                if p["body"] is not None:   # stepWood, js/main.js:239-241
                    p["body"].density = (w.mv + w.mc) / (w.side * w.side)
                    self.world.resize(p["body"], w.half)
        self.upload()
        self.sim.set_frame(self.frame_no)
        self.sim.write_params()
        self.sim.clear_geometry()
        self.sim.geometry()
        if n:
            self.sim.step(n)
        self.sim.radiation()
        self.frame_no += 1
        rb = self.sim.readback()
        if self.lag:
            self.queue.append((rb, simDt, list(self.slots)))
        else:
            self.apply(rb, simDt, None)
        return n

    def apply(self, rb, simDt, owners):
        """onReadback (js/main.js:210-230); owners: the slot contents when the readback's frame ran."""
        if simDt <= 0:
            return
        acc, rad, faceW = rb["acc"], rb["rad"], rb["faceW"]
        for s, p in enumerate(self.slots):
            if p is None or (owners is not None and owners[s] is not p):
                continue
            w = p["wood"]
            for f in range(4):
                w.exposure[f] = min(1.0, int(faceW[s * 4 + f]) / 1e8 / max(w.side, 1e-4))
                k = (s * 4 + f) * 2
                p["qConv"][f] = int(acc[k]) / E_SCALE / simDt
                p["charPending"][f] += int(acc[k + 1]) / M_SCALE
                p["qInc"][f] = float(rad[(s * 4 + f) * 4])
                p["vis"][f] = float(rad[(s * 4 + f) * 4 + 1])
        self.hrr = int(acc[ACC_GLOBAL]) / G_SCALE / simDt
        self.rad = int(acc[ACC_GLOBAL + 1]) / G_SCALE / simDt
        self.tmax = float(acc[ACC_GLOBAL + 2])


def default_scene(scene, charYield=0.25, density=500.0):
    """defaultScene, js/main.js:132-155, on a WoodScene of this module (SCENE_WIDTH 0.7 m)."""
    cx, S = 0.7 / 2, 0.0125

    def coal(x, y, sz, T):
        p = scene.slots[scene.add(x, y, 0.0, sz, density, preheat=(T, sz, T - 30))]
        w = p["wood"]
        w.mv = 0
        w.mc = w.rhoC * sz * sz
        w.updateSide()
        w.d = [sz / 2, sz / 2, sz / 2, sz / 2]
        w.charCov = [1, 1, 1, 1]
        w.Tp = [T - 20, T - 20, T - 20, T - 20]
        if p["body"] is not None:
            p["body"].density = w.mc / (sz * sz)
            scene.world.resize(p["body"], w.half)

    def lit(x, y, sz):
        w = scene.slots[scene.add(x, y, 0.0, sz, density, preheat=(880, 0.003 if sz > 0.03 else 0.002, 380))]["wood"]
        w.Tp = [590, 590, 590, 590]

    x = cx - 0.06
    for sz in (0.016, 0.02, 0.015, 0.018, 0.02, 0.016, 0.017):
        coal(x + sz / 2, sz / 2, sz, 1050)
        x += sz + 0.0015
    lit(cx - 0.093, 0.025, 0.05)
    lit(cx + 0.093, 0.025, 0.05)
    y1 = 0.02 + S + 0.001
    for dx in (-0.045, -0.016, 0.013, 0.042):
        lit(cx + dx, y1, 0.025)
    for dx in (-0.03, 0.0, 0.028):
        lit(cx + dx, y1 + 2 * S + 0.002, 0.025)
