"""ORACLE — test infrastructure, not product code.

Python restatement of the campfire app's rigid bodies (js/rigid.js) and of the
contact heat exchange (js/contact.js), used to check the C++ world bit for bit.
Python floats are IEEE doubles evaluated left to right, as JS numbers are;
math.cos/sin/exp/pow are the C library's, as in the C++ world. The JS built-ins
whose results are engine-defined are restated: Math.hypot as V8 evaluates it
(magnitudes normalised by the largest, Kahan-summed squares, sqrt times the
largest), Math.round (halves toward +inf) and Math.min/Math.max (NaN wins,
+0 above -0).
"""
from __future__ import annotations

import math

TAU = math.pi * 2                                                   # rigid.js:10
RIGID_DEFAULTS = dict(gravity=(0.0, -9.81), width=0.7, dt=1 / 480, substeps=4, slop=0.0002, contactHertz=240,
                      contactDamping=10, maxPushout=0.25, muStatic=0.7, muKinetic=0.5, stickSpeed=0.002, maxSpeed=8,
                      dragHertz=8, dragStrength=2.5)               # rigid.js:12-27


def js_hypot(x, y):
    if math.isinf(x) or math.isinf(y):
        return math.inf
    if math.isnan(x) or math.isnan(y):
        return math.nan
    vals = (abs(x), abs(y))
    mx = 0.0
    for v in vals:
        if v > mx:
            mx = v
    if mx == 0:
        return 0.0
    s = comp = 0.0
    for v in vals:
        n = v / mx
        summand = n * n - comp
        pre = s + summand
        comp = (pre - s) - summand
        s = pre
    return math.sqrt(s) * mx


def js_round(x):
    if not math.isfinite(x):
        return x
    r = float(math.ceil(x))
    if r - 0.5 > x:
        r -= 1.0
    if r == 0 and math.copysign(1.0, x) < 0:
        return -0.0
    return r


def js_max(a, b):
    if math.isnan(a) or math.isnan(b):
        return math.nan
    if a == b:
        return b if math.copysign(1.0, a) < 0 else a
    return a if a > b else b


def js_min(a, b):
    if math.isnan(a) or math.isnan(b):
        return math.nan
    if a == b:
        return a if math.copysign(1.0, a) < 0 else b
    return a if a < b else b


def make_soft(hertz, zeta, h):                                      # rigid.js:29-36
    if hertz == 0:
        return (0.0, 1.0, 0.0)
    omega = TAU * hertz
    a1 = 2 * zeta + h * omega
    a2 = h * omega * a1
    a3 = 1 / (1 + a2)
    return (omega / a1, a2 * a3, a3)


class Body:                                                          # rigid.js:40-59
    def __init__(self, bid, x, y, half, density, angle=0.0):
        self.id = bid
        self.x, self.y, self.a = x, y, angle
        self.vx = self.vy = self.w = 0.0
        self.density = density
        self.half = 0.0
        self.drag = None
        self.user = None
        self.set_half(half)

    def set_half(self, half):
        s = 2 * half
        self.half = half
        self.mass = self.density * s * s
        self.invMass = 1 / self.mass
        self.I = self.mass * s * s / 6
        self.invI = 1 / self.I


class _Static:
    id = 0
    x = y = a = 0.0
    half = 0.0
    invMass = invI = 0.0
    user = None

    def __init__(self):
        self.vx = self.vy = self.w = 0.0


LV = ((-1, -1), (1, -1), (1, 1), (-1, 1))
LN = ((0, -1), (1, 0), (0, 1), (-1, 0))


def box_geom(b):                                                     # rigid.js:65-76
    c, s, h = math.cos(b.a), math.sin(b.a), b.half
    v, n = [], []
    for i in range(4):
        lx, ly = LV[i][0] * h, LV[i][1] * h
        v.append((b.x + c * lx - s * ly, b.y + s * lx + c * ly))
        nx, ny = LN[i]
        n.append((c * nx - s * ny, s * nx + c * ny))
    return v, n


def max_separation(ga, gb):                                          # rigid.js:80-93
    best, edge = -math.inf, 0
    for i in range(4):
        nx, ny = ga[1][i]
        ox, oy = ga[0][i]
        m = math.inf
        for j in range(4):
            d = nx * (gb[0][j][0] - ox) + ny * (gb[0][j][1] - oy)
            if d < m:
                m = d
        if m > best:
            best, edge = m, i
    return best, edge


def clip_segment(pts, nx, ny, off, clip_id):                         # rigid.js:96-108
    if len(pts) < 2:
        return pts
    p0, p1 = pts[0], pts[1]
    d0 = nx * p0[0] + ny * p0[1] - off
    d1 = nx * p1[0] + ny * p1[1] - off
    out = []
    if d0 <= 0:
        out.append(p0)
    if d1 <= 0:
        out.append(p1)
    if d0 * d1 < 0:
        t = d0 / (d0 - d1)
        out.append((p0[0] + t * (p1[0] - p0[0]), p0[1] + t * (p1[1] - p0[1]), clip_id))
    return out


def collide_boxes(A, B, spec, slop):                                 # rigid.js:111-145
    GA, GB = box_geom(A), box_geom(B)
    sepA, eA = max_separation(GA, GB)
    if sepA > spec:
        return None
    sepB, eB = max_separation(GB, GA)
    if sepB > spec:
        return None
    if sepB > sepA + 0.1 * slop:
        flip, R, I, e = 1, GB, GA, eB
    else:
        flip, R, I, e = 0, GA, GB, eA
    nx, ny = R[1][e]
    j, md = 0, math.inf
    for k in range(4):
        d = I[1][k][0] * nx + I[1][k][1] * ny
        if d < md:
            md, j = d, k
    j2 = (j + 1) & 3
    r1, r2 = R[0][e], R[0][(e + 1) & 3]
    tx, ty = r2[0] - r1[0], r2[1] - r1[1]
    tl = js_hypot(tx, ty)
    tx /= tl
    ty /= tl
    base = (flip << 6) | (e << 3)
    pts = [(I[0][j][0], I[0][j][1], base | j), (I[0][j2][0], I[0][j2][1], base | j2)]
    pts = clip_segment(pts, -tx, -ty, -(tx * r1[0] + ty * r1[1]), base | 4)
    pts = clip_segment(pts, tx, ty, tx * r2[0] + ty * r2[1], base | 5)
    out = []
    for p in pts:
        sep = nx * (p[0] - r1[0]) + ny * (p[1] - r1[1])
        if sep <= spec:
            out.append({"x": p[0] - 0.5 * sep * nx, "y": p[1] - 0.5 * sep * ny, "sep": sep, "id": p[2]})
    if not out:
        return None
    return {"nx": -nx if flip else nx, "ny": -ny if flip else ny, "points": out}


def collide_plane(B, nx, ny, off, spec):                             # rigid.js:148-157
    v, _ = box_geom(B)
    out = []
    for i in range(4):
        x, y = v[i]
        sep = nx * x + ny * y - off
        if sep <= spec:
            out.append({"x": x - 0.5 * sep * nx, "y": y - 0.5 * sep * ny, "sep": sep, "id": i})
    return {"nx": nx, "ny": ny, "points": out} if out else None


def apply_impulse(A, B, c, Px, Py):                                  # rigid.js:471-476
    A.vx -= A.invMass * Px
    A.vy -= A.invMass * Py
    A.w -= A.invI * (c["rAx"] * Py - c["rAy"] * Px)
    B.vx += B.invMass * Px
    B.vy += B.invMass * Py
    B.w += B.invI * (c["rBx"] * Py - c["rBy"] * Px)


class RigidWorld:                                                    # rigid.js:159-468
    def __init__(self, **opts):
        self.p = dict(RIGID_DEFAULTS, **opts)
        self.bodies = []
        self.manifolds = {}    # insertion-ordered, as a JS Map
        self.time = 0.0
        self.accum = 0.0
        self.static = _Static()
        self.next_id = 1

    def add(self, x, y, half, density, angle=0.0):
        b = Body(self.next_id, x, y, half, density, angle)
        self.next_id += 1
        self.bodies.append(b)
        return b

    def remove(self, body):
        self.bodies.remove(body)
        self.manifolds = {k: m for k, m in self.manifolds.items() if m["A"] is not body and m["B"] is not body}

    def resize(self, body, half):
        f = half / body.half
        if f == 1:
            return
        for m in self.manifolds.values():
            if m["A"] is body:
                m["aAx"] *= f
                m["aAy"] *= f
            if m["B"] is body:
                m["aBx"] *= f
                m["aBy"] *= f
        body.set_half(half)

    def advance(self, dt):
        self.accum += dt
        h = self.p["dt"]
        n = 0
        while self.accum >= h and n < 64:
            self.step(h)
            self.accum -= h
            n += 1
        if n == 64:
            self.accum = 0.0

    def collide(self, dt):
        P, old, fresh = self.p, self.manifolds, {}
        spec0 = 4 * P["slop"]

        def take(key, A, Bb, man):
            prev = old.get(key)
            m = {"A": A, "B": Bb, "nx": man["nx"], "ny": man["ny"], "points": [], "cx": 0.0, "cy": 0.0, "Pt": 0.0,
                 "sticking": True, "aAx": 0.0, "aAy": 0.0, "aBx": 0.0, "aBy": 0.0}
            used = []
            n = len(man["points"])
            for p in man["points"]:
                c = {"id": p["id"], "x": p["x"], "y": p["y"], "sep": p["sep"], "Pn": 0.0}
                if prev:
                    q = next((q for q in prev["points"] if q["id"] == p["id"] and not any(q is u for u in used)), None)
                    if q is None:
                        best = 0.25 * js_min(A.half if A.half else Bb.half, Bb.half)
                        for r in prev["points"]:
                            d = js_hypot(r["x"] - p["x"], r["y"] - p["y"])
                            if d < best and not any(r is u for u in used):
                                best, q = d, r
                    if q is not None:
                        c["Pn"] = q["Pn"]
                        used.append(q)
                m["points"].append(c)
                m["cx"] += p["x"] / n
                m["cy"] += p["y"] / n
            if prev and prev["nx"] * m["nx"] + prev["ny"] * m["ny"] > 0.99:
                for k in ("Pt", "sticking", "aAx", "aAy", "aBx", "aBy"):
                    m[k] = prev[k]
            else:
                self.set_anchors(A, Bb, m, m["cx"], m["cy"])
            fresh[key] = m

        W = P["width"]
        for b in self.bodies:
            speed = js_hypot(b.vx, b.vy) + abs(b.w) * b.half * 1.5
            spec = spec0 + speed * dt
            m = collide_plane(b, 0, 1, 0, spec)
            if m:
                take(("f", b.id), self.static, b, m)
            m = collide_plane(b, 1, 0, 0, spec)
            if m:
                take(("l", b.id), self.static, b, m)
            m = collide_plane(b, -1, 0, -W, spec)
            if m:
                take(("r", b.id), self.static, b, m)
        B = self.bodies
        for i in range(len(B)):
            for j in range(i + 1, len(B)):
                a, b = B[i], B[j]
                if a.id > b.id:
                    a, b = b, a
                rel = js_hypot(b.vx - a.vx, b.vy - a.vy) + (abs(a.w) * a.half + abs(b.w) * b.half) * 1.5
                spec = spec0 + rel * dt
                reach = (a.half + b.half) * 1.4143 + spec
                if abs(a.x - b.x) > reach or abs(a.y - b.y) > reach:
                    continue
                m = collide_boxes(a, b, spec, P["slop"])
                if m:
                    take((a.id, b.id), a, b, m)
        self.manifolds = fresh

    @staticmethod
    def set_anchors(A, B, c, px, py):
        dx, dy, ca, sa = px - A.x, py - A.y, math.cos(A.a), math.sin(A.a)
        c["aAx"] = ca * dx + sa * dy
        c["aAy"] = -sa * dx + ca * dy
        dx, dy, ca, sa = px - B.x, py - B.y, math.cos(B.a), math.sin(B.a)
        c["aBx"] = ca * dx + sa * dy
        c["aBy"] = -sa * dx + ca * dy

    def step(self, dt):                                              # rigid.js:271-346
        P = self.p
        self.collide(dt)
        ns = P["substeps"]
        h = dt / ns
        inv_h = 1 / h
        soft = make_soft(js_min(P["contactHertz"], 0.25 / h), P["contactDamping"], h)
        drag_soft = make_soft(P["dragHertz"], 1, h)
        gx, gy = P["gravity"]
        cons = list(self.manifolds.values())
        for m in cons:
            A, B, nx, ny = m["A"], m["B"], m["nx"], m["ny"]
            tx, ty = ny, -nx
            mA, mB, iA, iB = A.invMass, B.invMass, A.invI, B.invI
            for c in m["points"]:
                rAx, rAy, rBx, rBy = c["x"] - A.x, c["y"] - A.y, c["x"] - B.x, c["y"] - B.y
                ca, sa, cb, sb = math.cos(A.a), math.sin(A.a), math.cos(B.a), math.sin(B.a)
                c["lAx"] = ca * rAx + sa * rAy
                c["lAy"] = -sa * rAx + ca * rAy
                c["lBx"] = cb * rBx + sb * rBy
                c["lBy"] = -sb * rBx + cb * rBy
                c["rAx"], c["rAy"], c["rBx"], c["rBy"] = rAx, rAy, rBx, rBy
                rnA, rnB = rAx * ny - rAy * nx, rBx * ny - rBy * nx
                c["nMass"] = 1 / (mA + mB + iA * rnA * rnA + iB * rnB * rnB)
            m["rAx"], m["rAy"] = m["cx"] - A.x, m["cy"] - A.y
            m["rBx"], m["rBy"] = m["cx"] - B.x, m["cy"] - B.y
            rtA = m["rAx"] * ty - m["rAy"] * tx
            rtB = m["rBx"] * ty - m["rBy"] * tx
            m["tMass"] = 1 / (mA + mB + iA * rtA * rtA + iB * rtB * rtB)
        dragged = [b for b in self.bodies if b.drag]
        for _ in range(ns):
            for b in self.bodies:
                if b.drag:
                    continue
                b.vx += gx * h
                b.vy += gy * h
            for m in cons:
                A, B = m["A"], m["B"]
                tx, ty = m["ny"], -m["nx"]
                for c in m["points"]:
                    apply_impulse(A, B, c, c["Pn"] * m["nx"], c["Pn"] * m["ny"])
                apply_impulse(A, B, m, m["Pt"] * tx, m["Pt"] * ty)
            self.solve_drag(dragged, drag_soft, h)
            self.solve_contacts(cons, soft, inv_h, True)
            vmax = P["maxSpeed"]
            for b in self.bodies:
                sp = js_hypot(b.vx, b.vy)
                if sp > vmax:
                    b.vx *= vmax / sp
                    b.vy *= vmax / sp
                b.x += b.vx * h
                b.y += b.vy * h
                b.a += b.w * h
            self.solve_contacts(cons, soft, inv_h, False)
        for m in cons:
            A, B = m["A"], m["B"]
            tx, ty = m["ny"], -m["nx"]
            Pn = 0.0
            for c in m["points"]:
                Pn += c["Pn"]
            if m["sticking"]:
                if Pn > 0 and abs(m["Pt"]) >= 0.999 * P["muStatic"] * Pn:
                    m["sticking"] = False
                continue
            dvx = B.vx - B.w * m["rBy"] - A.vx + A.w * m["rAy"]
            dvy = B.vy + B.w * m["rBx"] - A.vy - A.w * m["rAx"]
            if abs(dvx * tx + dvy * ty) < P["stickSpeed"]:
                m["sticking"] = True
                self.set_anchors(A, B, m, m["cx"], m["cy"])
        self.time += dt

    def solve_drag(self, dragged, soft, h):                          # rigid.js:351-371
        bias_rate, mscale, _ = soft
        for b in dragged:
            d = b.drag
            mi, ii = b.invMass, b.invI
            Cx, Cy = b.x - d["cx"], b.y - d["cy"]
            ix = -mscale * b.mass * (b.vx + bias_rate * Cx)
            iy = -mscale * b.mass * (b.vy + bias_rate * Cy)
            maxI, L = d["maxForce"] * h, js_hypot(ix, iy)
            if L > maxI:
                ix *= maxI / L
                iy *= maxI / L
            b.vx += mi * ix
            b.vy += mi * iy
            da = b.a - d["a0"]
            da -= 2 * math.pi * js_round(da / (2 * math.pi))
            ia = -mscale * b.I * (b.w + bias_rate * da)
            maxA = d["maxTorque"] * h
            ia = js_max(-maxA, js_min(maxA, ia))
            b.w += ii * ia

    def solve_contacts(self, cons, soft, inv_h, use_bias):           # rigid.js:373-416
        P = self.p
        bias_rate, mscale, iscale = soft
        for m in cons:
            A, B, nx, ny = m["A"], m["B"], m["nx"], m["ny"]
            tx, ty = ny, -nx
            cA, sA, cB, sB = math.cos(A.a), math.sin(A.a), math.cos(B.a), math.sin(B.a)
            Pn = 0.0
            for c in m["points"]:
                Pn += c["Pn"]
            dvx = B.vx - B.w * m["rBy"] - A.vx + A.w * m["rAy"]
            dvy = B.vy + B.w * m["rBx"] - A.vy - A.w * m["rAx"]
            vt = dvx * tx + dvy * ty
            if m["sticking"]:
                bias, ms, is_ = 0.0, 1.0, 0.0
                if use_bias:
                    pAx = A.x + cA * m["aAx"] - sA * m["aAy"]
                    pAy = A.y + sA * m["aAx"] + cA * m["aAy"]
                    pBx = B.x + cB * m["aBx"] - sB * m["aBy"]
                    pBy = B.y + sB * m["aBx"] + cB * m["aBy"]
                    drift = (pBx - pAx) * tx + (pBy - pAy) * ty
                    bias = js_max(-P["maxPushout"], js_min(P["maxPushout"], bias_rate * drift))
                    ms, is_ = mscale, iscale
                maxS = P["muStatic"] * Pn
                newP = m["Pt"] - m["tMass"] * ms * (vt + bias) - is_ * m["Pt"]
                newP = js_max(-maxS, js_min(maxS, newP))
            else:
                maxK = P["muKinetic"] * Pn
                newP = js_max(-maxK, js_min(maxK, m["Pt"] - m["tMass"] * vt))
            imp = newP - m["Pt"]
            m["Pt"] = newP
            apply_impulse(A, B, m, imp * tx, imp * ty)
            for c in m["points"]:
                pAx = A.x + cA * c["lAx"] - sA * c["lAy"]
                pAy = A.y + sA * c["lAx"] + cA * c["lAy"]
                pBx = B.x + cB * c["lBx"] - sB * c["lBy"]
                pBy = B.y + sB * c["lBx"] + cB * c["lBy"]
                sep = (pBx - pAx) * nx + (pBy - pAy) * ny + c["sep"]
                bias, ms, is_ = 0.0, 1.0, 0.0
                if sep > 0:
                    bias = sep * inv_h
                elif use_bias:
                    bias = js_max(bias_rate * sep, -P["maxPushout"])
                    ms, is_ = mscale, iscale
                dvx = B.vx - B.w * c["rBy"] - A.vx + A.w * c["rAy"]
                dvy = B.vy + B.w * c["rBx"] - A.vy - A.w * c["rAx"]
                vn = dvx * nx + dvy * ny
                imp = -c["nMass"] * ms * (vn + bias) - is_ * c["Pn"]
                newP = js_max(c["Pn"] + imp, 0.0)
                imp = newP - c["Pn"]
                c["Pn"] = newP
                apply_impulse(A, B, c, imp * nx, imp * ny)

    def pick(self, x, y):                                            # rigid.js:419-428
        for b in reversed(self.bodies):
            dx, dy, c, s = x - b.x, y - b.y, math.cos(b.a), math.sin(b.a)
            lx, ly = c * dx + s * dy, -s * dx + c * dy
            if abs(lx) <= b.half and abs(ly) <= b.half:
                return b, lx, ly
        return None

    def start_drag(self, b, lx, ly, tx, ty):                         # rigid.js:431-439
        gy = self.p["gravity"][1]
        g = abs(gy) if (gy != 0 and not math.isnan(gy)) else 9.81
        b.drag = {"lx": lx, "ly": ly, "a0": b.a, "cx": b.x, "cy": b.y,
                  "maxForce": self.p["dragStrength"] * b.mass * g,
                  "maxTorque": self.p["dragStrength"] * b.mass * g * b.half}
        self.move_drag(b, tx, ty)

    def move_drag(self, b, tx, ty):                                  # rigid.js:440-449
        d = b.drag
        if not d:
            return
        c, s = math.cos(d["a0"]), math.sin(d["a0"])
        ox, oy = c * d["lx"] - s * d["ly"], s * d["lx"] + c * d["ly"]
        h, W = b.half * 1.42, self.p["width"]
        d["cx"] = js_min(W - h, js_max(h, tx - ox))
        d["cy"] = js_max(h, ty - oy)

    def end_drag(self, b):                                           # rigid.js:451-455
        if not b.drag:
            return
        b.drag = None
        b.vx = b.vy = b.w = 0.0

    def max_penetration(self):
        m = 0.0
        for man in self.manifolds.values():
            for c in man["points"]:
                m = js_max(m, -c["sep"])
        return m


# ---------------------------------------------------------------- js/contact.js
CONTACT = dict(gap=0.0005, pointLength=0.001, maxSep=0.0005)
WOOD_EPS, WOOD_SIGMA = 0.9, 5.670374e-8


def face_toward(a, nx, ny):
    c, s = math.cos(a), math.sin(a)
    lx, ly = c * nx + s * ny, -s * nx + c * ny
    if abs(lx) > abs(ly):
        return 0 if lx > 0 else 2
    return 1 if ly > 0 else 3


def contact_conductance(T):
    kGas = 0.0241 * math.pow(T / 273.15, 0.8)
    return kGas / CONTACT["gap"] + 4 * WOOD_SIGMA * T * T * T / (2 / WOOD_EPS - 1)


def surface_cap(w, f):                                               # js/wood.js:53-58
    s = w.side
    dS = min(0.0015, s / 8)
    phi = 1 if w.mv <= 1e-9 else min(1, w.d[f] / dS)
    return (w.rhoV * 1500 * (1 - phi) + w.rhoC * 1000 * phi) * dS * s


def exchange_contacts(world, dt):
    """Body.user holds the WoodPiece of a wood body (None: no heat exchange)."""
    moved = 0.0
    if dt <= 0:
        return moved
    for m in world.manifolds.values():
        wa, wb = m["A"].user, m["B"].user
        if wa is None or wb is None:
            continue
        pts = [c for c in m["points"] if c["sep"] < CONTACT["maxSep"]]
        if not pts:
            continue
        L = js_hypot(pts[0]["x"] - pts[1]["x"], pts[0]["y"] - pts[1]["y"]) if len(pts) >= 2 else CONTACT["pointLength"]
        if L <= 0:
            continue
        fa = face_toward(m["A"].a, m["nx"], m["ny"])
        fb = face_toward(m["B"].a, -m["nx"], -m["ny"])
        Ta, Tb = wa.Ts[fa], wb.Ts[fb]
        G = contact_conductance(0.5 * (Ta + Tb)) * L
        Ca, Cb = surface_cap(wa, fa), surface_cap(wb, fb)
        inv = 1 / Ca + 1 / Cb
        E = (Ta - Tb) * (1 - math.exp(-G * inv * dt)) / inv
        wa.Ts[fa] -= E / Ca
        wb.Ts[fb] += E / Cb
        moved += abs(E)
    return moved
