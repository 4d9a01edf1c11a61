// 2D rigid bodies of the campfire app (js/rigid.js) and the contact heat
// exchange (js/contact.js). Double precision with the reference's order of
// operations; see rigid.h.
#include "rigid.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace cfg {

namespace {

constexpr double kTau = 3.141592653589793 * 2;   // rigid.js:10

// Math.max / Math.min of two numbers: NaN wins, and +0 is above -0
double js_max(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return std::numeric_limits<double>::quiet_NaN();
  if (a == b) return std::signbit(a) ? b : a;
  return a > b ? a : b;
}
double js_min(double a, double b) {
  if (std::isnan(a) || std::isnan(b)) return std::numeric_limits<double>::quiet_NaN();
  if (a == b) return std::signbit(a) ? a : b;
  return a < b ? a : b;
}

struct Soft { double biasRate, massScale, impulseScale; };
Soft make_soft(double hertz, double zeta, double h) {   // rigid.js:29-36
  if (hertz == 0) return {0, 1, 0};
  const double omega = kTau * hertz;
  const double a1 = 2 * zeta + h * omega;
  const double a2 = h * omega * a1;
  const double a3 = 1 / (1 + a2);
  return {omega / a1, a2 * a3, a3};
}

// corners counter-clockwise and the outward normal of edge i (v[i] -> v[i+1])
constexpr double kLV[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
constexpr double kLN[4][2] = {{0, -1}, {1, 0}, {0, 1}, {-1, 0}};

struct Geom { double v[4][2], n[4][2]; };
void box_geom(const Body& b, Geom& g) {   // rigid.js:65-76
  const double c = std::cos(b.a), s = std::sin(b.a), h = b.half;
  for (int i = 0; i < 4; i++) {
    const double lx = kLV[i][0] * h, ly = kLV[i][1] * h;
    g.v[i][0] = b.x + c * lx - s * ly;
    g.v[i][1] = b.y + s * lx + c * ly;
    const double nx = kLN[i][0], ny = kLN[i][1];
    g.n[i][0] = c * nx - s * ny;
    g.n[i][1] = s * nx + c * ny;
  }
}

// the largest over edges of A of the smallest separation of B's corners (rigid.js:80-93)
void max_separation(const Geom& ga, const Geom& gb, double* best, int* edge) {
  *best = -std::numeric_limits<double>::infinity();
  *edge = 0;
  for (int i = 0; i < 4; i++) {
    const double nx = ga.n[i][0], ny = ga.n[i][1], ox = ga.v[i][0], oy = ga.v[i][1];
    double m = std::numeric_limits<double>::infinity();
    for (int j = 0; j < 4; j++) {
      const double d = nx * (gb.v[j][0] - ox) + ny * (gb.v[j][1] - oy);
      if (d < m) m = d;
    }
    if (m > *best) { *best = m; *edge = i; }
  }
}

struct Pt { double x, y; int id; };
// keeps the part of a two-point segment with n.p <= off (rigid.js:96-108)
int clip_segment(Pt* pts, int n, double nx, double ny, double off, int clip_id) {
  if (n < 2) return n;
  const Pt p0 = pts[0], p1 = pts[1];
  const double d0 = nx * p0.x + ny * p0.y - off;
  const double d1 = nx * p1.x + ny * p1.y - off;
  int k = 0;
  Pt out[3];
  if (d0 <= 0) out[k++] = p0;
  if (d1 <= 0) out[k++] = p1;
  if (d0 * d1 < 0) {
    const double t = d0 / (d0 - d1);
    out[k++] = {p0.x + t * (p1.x - p0.x), p0.y + t * (p1.y - p0.y), clip_id};
  }
  for (int i = 0; i < k; i++) pts[i] = out[i];
  return k;
}

// box-box manifold, normal from A to B (rigid.js:111-145); false: no contact
bool collide_boxes(const Body& A, const Body& B, double spec, double slop, Manifold& m) {
  Geom ga, gb;
  box_geom(A, ga);
  box_geom(B, gb);
  double sepA, sepB;
  int eA, eB;
  max_separation(ga, gb, &sepA, &eA);
  if (sepA > spec) return false;
  max_separation(gb, ga, &sepB, &eB);
  if (sepB > spec) return false;
  const bool flip = sepB > sepA + 0.1 * slop;
  const Geom& R = flip ? gb : ga;
  const Geom& I = flip ? ga : gb;
  const int e = flip ? eB : eA;
  const double nx = R.n[e][0], ny = R.n[e][1];
  int j = 0;
  double md = std::numeric_limits<double>::infinity();
  for (int k = 0; k < 4; k++) {   // incident edge: the most anti-parallel normal
    const double d = I.n[k][0] * nx + I.n[k][1] * ny;
    if (d < md) { md = d; j = k; }
  }
  const int j2 = (j + 1) & 3;
  const double* r1 = R.v[e];
  const double* r2 = R.v[(e + 1) & 3];
  double tx = r2[0] - r1[0], ty = r2[1] - r1[1];
  const double tl = js_hypot(tx, ty);
  tx /= tl;
  ty /= tl;
  const int base = ((flip ? 1 : 0) << 6) | (e << 3);
  Pt pts[3] = {{I.v[j][0], I.v[j][1], base | j}, {I.v[j2][0], I.v[j2][1], base | j2}, {}};
  int n = 2;
  n = clip_segment(pts, n, -tx, -ty, -(tx * r1[0] + ty * r1[1]), base | 4);
  n = clip_segment(pts, n, tx, ty, tx * r2[0] + ty * r2[1], base | 5);
  m.npts = 0;
  for (int i = 0; i < n; i++) {
    const Pt& p = pts[i];
    const double sep = nx * (p.x - r1[0]) + ny * (p.y - r1[1]);
    if (sep <= spec) {
      ContactPoint& c = m.pts[m.npts++];
      c = ContactPoint{};
      c.x = p.x - 0.5 * sep * nx;
      c.y = p.y - 0.5 * sep * ny;
      c.sep = sep;
      c.id = p.id;
    }
  }
  if (!m.npts) return false;
  m.nx = flip ? -nx : nx;
  m.ny = flip ? -ny : ny;
  return true;
}

// box against the half-plane n.p >= off, normal from the plane to the box (rigid.js:148-157)
bool collide_plane(const Body& B, double nx, double ny, double off, double spec, Manifold& m) {
  Geom g;
  box_geom(B, g);
  m.npts = 0;
  for (int i = 0; i < 4; i++) {
    const double x = g.v[i][0], y = g.v[i][1];
    const double sep = nx * x + ny * y - off;
    if (sep <= spec) {
      ContactPoint& c = m.pts[m.npts++];
      c = ContactPoint{};
      c.x = x - 0.5 * sep * nx;
      c.y = y - 0.5 * sep * ny;
      c.sep = sep;
      c.id = i;
    }
  }
  if (!m.npts) return false;
  m.nx = nx;
  m.ny = ny;
  return true;
}

template <class C>
void apply_impulse(Body* A, Body* B, const C& c, double Px, double Py) {   // rigid.js:471-476
  A->vx -= A->invMass * Px; A->vy -= A->invMass * Py;
  A->w -= A->invI * (c.rAx * Py - c.rAy * Px);
  B->vx += B->invMass * Px; B->vy += B->invMass * Py;
  B->w += B->invI * (c.rBx * Py - c.rBy * Px);
}

// manifold keys: 'f'/'l'/'r' + body id for the floor and walls, a.id '_' b.id for pairs
uint64_t plane_key(int kind, int id) { return ((uint64_t)kind << 60) | (uint64_t)(uint32_t)id; }
uint64_t pair_key(int a, int b) { return ((uint64_t)4 << 60) | ((uint64_t)(uint32_t)a << 30) | (uint64_t)(uint32_t)b; }

}  // namespace

// Math.hypot as V8 evaluates it: the magnitudes normalised by the largest, their
// squares Kahan-summed, sqrt times the largest
double js_hypot(double x, double y) {
  if (std::isinf(x) || std::isinf(y)) return std::numeric_limits<double>::infinity();
  if (std::isnan(x) || std::isnan(y)) return std::numeric_limits<double>::quiet_NaN();
  const double ax = std::fabs(x), ay = std::fabs(y);
  double mx = 0;
  if (ax > mx) mx = ax;
  if (ay > mx) mx = ay;
  if (mx == 0) return 0;
  double sum = 0, comp = 0;
  for (double v : {ax, ay}) {
    const double n = v / mx;
    const double summand = n * n - comp;
    const double prelim = sum + summand;
    comp = (prelim - sum) - summand;
    sum = prelim;
  }
  return std::sqrt(sum) * mx;
}

// Math.round: the nearest integer, halves toward +infinity
double js_round(double x) {
  if (!std::isfinite(x)) return x;
  double r = std::ceil(x);
  if (r - 0.5 > x) r -= 1.0;
  if (r == 0 && std::signbit(x)) return -0.0;
  return r;
}

void Body::set_half(double h) {
  const double s = 2 * h;
  half = h;
  mass = density * s * s;
  invMass = 1 / mass;
  I = mass * s * s / 6;
  invI = 1 / I;
}

Body* RigidWorld::add(double x, double y, double half, double density, double angle) {
  auto b = std::make_unique<Body>();
  b->id = next_id_++;
  b->x = x; b->y = y; b->a = angle;
  b->density = density;
  b->set_half(half);
  bodies_.push_back(std::move(b));
  return bodies_.back().get();
}

Body* RigidWorld::find(int id) {
  for (auto& b : bodies_) if (b->id == id) return b.get();
  return nullptr;
}

int RigidWorld::remove(int id) {
  auto it = std::find_if(bodies_.begin(), bodies_.end(), [&](const std::unique_ptr<Body>& b) { return b->id == id; });
  if (it == bodies_.end()) return CFG_ERR_NOENT;
  const Body* b = it->get();
  manifolds_.erase(std::remove_if(manifolds_.begin(), manifolds_.end(),
                                  [&](const Manifold& m) { return m.A == b || m.B == b; }),
                   manifolds_.end());
  bodies_.erase(it);
  return CFG_OK;
}

void RigidWorld::resize(Body* b, double half) {
  const double f = half / b->half;
  if (f == 1) return;
  for (auto& m : manifolds_) {
    if (m.A == b) { m.aAx *= f; m.aAy *= f; }
    if (m.B == b) { m.aBx *= f; m.aBy *= f; }
  }
  b->set_half(half);
}

void RigidWorld::advance(double dt) {
  accum += dt;
  const double h = p.dt;
  int n = 0;
  while (accum >= h && n < 64) { step(h); accum -= h; n++; }
  if (n == 64) accum = 0;
}

void RigidWorld::set_anchors(const Body* A, const Body* B, Manifold& c, double px, double py) {
  double dx = px - A->x, dy = py - A->y, ca = std::cos(A->a), sa = std::sin(A->a);
  c.aAx = ca * dx + sa * dy; c.aAy = -sa * dx + ca * dy;
  dx = px - B->x; dy = py - B->y; ca = std::cos(B->a); sa = std::sin(B->a);
  c.aBx = ca * dx + sa * dy; c.aBy = -sa * dx + ca * dy;
}

void RigidWorld::take(uint64_t key, Body* A, Body* B, const Manifold& man, const std::vector<Manifold>& old,
                      const std::unordered_map<uint64_t, int>& old_index) {
  auto it = old_index.find(key);
  const Manifold* prev = it == old_index.end() ? nullptr : &old[it->second];
  Manifold m;
  m.key = key; m.A = A; m.B = B; m.nx = man.nx; m.ny = man.ny;
  bool used[4] = {false, false, false, false};
  for (int i = 0; i < man.npts; i++) {
    const ContactPoint& p = man.pts[i];
    ContactPoint& c = m.pts[m.npts++];
    c = ContactPoint{};
    c.id = p.id; c.x = p.x; c.y = p.y; c.sep = p.sep; c.Pn = 0;
    if (prev) {
      // warm start from the same feature, else from the nearest unused previous point
      int q = -1;
      for (int k = 0; k < prev->npts; k++)
        if (prev->pts[k].id == p.id && !used[k]) { q = k; break; }
      if (q < 0) {
        double best = 0.25 * js_min(A->half != 0 ? A->half : B->half, B->half);
        for (int k = 0; k < prev->npts; k++) {
          const double d = js_hypot(prev->pts[k].x - p.x, prev->pts[k].y - p.y);
          if (d < best && !used[k]) { best = d; q = k; }
        }
      }
      if (q >= 0) { c.Pn = prev->pts[q].Pn; used[q] = true; }
    }
    m.cx += p.x / man.npts;
    m.cy += p.y / man.npts;
  }
  if (prev && prev->nx * m.nx + prev->ny * m.ny > 0.99) {
    m.Pt = prev->Pt; m.sticking = prev->sticking;
    m.aAx = prev->aAx; m.aAy = prev->aAy; m.aBx = prev->aBx; m.aBy = prev->aBy;
  } else {
    set_anchors(A, B, m, m.cx, m.cy);
  }
  manifolds_.push_back(m);
}

void RigidWorld::collide(double dt) {
  std::vector<Manifold> old;
  old.swap(manifolds_);
  std::unordered_map<uint64_t, int> old_index;
  old_index.reserve(old.size() * 2 + 1);
  for (int i = 0; i < (int)old.size(); i++) old_index.emplace(old[i].key, i);
  const double spec0 = 4 * p.slop, W = p.width;
  Manifold man;
  for (auto& bp : bodies_) {
    Body* b = bp.get();
    const double speed = js_hypot(b->vx, b->vy) + std::fabs(b->w) * b->half * 1.5;
    const double spec = spec0 + speed * dt;
    if (collide_plane(*b, 0, 1, 0, spec, man)) take(plane_key(1, b->id), &static_, b, man, old, old_index);
    if (collide_plane(*b, 1, 0, 0, spec, man)) take(plane_key(2, b->id), &static_, b, man, old, old_index);
    if (collide_plane(*b, -1, 0, -W, spec, man)) take(plane_key(3, b->id), &static_, b, man, old, old_index);
  }
  const int nb = (int)bodies_.size();
  for (int i = 0; i < nb; i++)
    for (int j = i + 1; j < nb; j++) {
      Body* a = bodies_[i].get();
      Body* b = bodies_[j].get();
      if (a->id > b->id) std::swap(a, b);
      const double rel = js_hypot(b->vx - a->vx, b->vy - a->vy) +
                         (std::fabs(a->w) * a->half + std::fabs(b->w) * b->half) * 1.5;
      const double spec = spec0 + rel * dt;
      const double reach = (a->half + b->half) * 1.4143 + spec;
      if (std::fabs(a->x - b->x) > reach || std::fabs(a->y - b->y) > reach) continue;
      if (collide_boxes(*a, *b, spec, p.slop, man)) take(pair_key(a->id, b->id), a, b, man, old, old_index);
    }
}

void RigidWorld::step(double dt) {
  collide(dt);
  const int ns = p.substeps;
  const double h = dt / ns, inv_h = 1 / h;
  const Soft soft = make_soft(js_min(p.contactHertz, 0.25 / h), p.contactDamping, h);
  const Soft drag_soft = make_soft(p.dragHertz, 1, h);
  // prepare: contact arms, anchors in body frames, effective masses
  for (auto& m : manifolds_) {
    Body *A = m.A, *B = m.B;
    const double nx = m.nx, ny = m.ny, tx = ny, ty = -nx;
    const double mA = A->invMass, mB = B->invMass, iA = A->invI, iB = B->invI;
    for (int k = 0; k < m.npts; k++) {
      ContactPoint& c = m.pts[k];
      const double rAx = c.x - A->x, rAy = c.y - A->y, rBx = c.x - B->x, rBy = c.y - B->y;
      const double ca = std::cos(A->a), sa = std::sin(A->a), cb = std::cos(B->a), sb = std::sin(B->a);
      c.lAx = ca * rAx + sa * rAy; c.lAy = -sa * rAx + ca * rAy;
      c.lBx = cb * rBx + sb * rBy; c.lBy = -sb * rBx + cb * rBy;
      c.rAx = rAx; c.rAy = rAy; c.rBx = rBx; c.rBy = rBy;
      const double rnA = rAx * ny - rAy * nx, rnB = rBx * ny - rBy * nx;
      c.nMass = 1 / (mA + mB + iA * rnA * rnA + iB * rnB * rnB);
    }
    m.rAx = m.cx - A->x; m.rAy = m.cy - A->y; m.rBx = m.cx - B->x; m.rBy = m.cy - B->y;
    const double rtA = m.rAx * ty - m.rAy * tx, rtB = m.rBx * ty - m.rBy * tx;
    m.tMass = 1 / (mA + mB + iA * rtA * rtA + iB * rtB * rtB);
  }
  for (int s = 0; s < ns; s++) {
    for (auto& b : bodies_) {   // gravity on every body the grip does not hold up
      if (b->dragging) continue;
      b->vx += p.gx * h; b->vy += p.gy * h;
    }
    for (auto& m : manifolds_) {   // apply the impulses kept from the last collision step
      const double tx = m.ny, ty = -m.nx;
      for (int k = 0; k < m.npts; k++) apply_impulse(m.A, m.B, m.pts[k], m.pts[k].Pn * m.nx, m.pts[k].Pn * m.ny);
      apply_impulse(m.A, m.B, m, m.Pt * tx, m.Pt * ty);
    }
    solve_drag(drag_soft.massScale, drag_soft.biasRate, h);
    solve_contacts(soft.biasRate, soft.massScale, soft.impulseScale, inv_h, true);
    const double vmax = p.maxSpeed;
    for (auto& b : bodies_) {
      const double sp = js_hypot(b->vx, b->vy);
      if (sp > vmax) { b->vx *= vmax / sp; b->vy *= vmax / sp; }
      b->x += b->vx * h; b->y += b->vy * h; b->a += b->w * h;
    }
    solve_contacts(soft.biasRate, soft.massScale, soft.impulseScale, inv_h, false);   // final velocity pass without position bias
  }
  // stick / slip state and anchor maintenance
  for (auto& m : manifolds_) {
    Body *A = m.A, *B = m.B;
    const double tx = m.ny, ty = -m.nx;
    double Pn = 0;
    for (int k = 0; k < m.npts; k++) Pn += m.pts[k].Pn;
    if (m.sticking) {
      if (Pn > 0 && std::fabs(m.Pt) >= 0.999 * p.muStatic * Pn) m.sticking = false;
      continue;
    }
    const double dvx = B->vx - B->w * m.rBy - A->vx + A->w * m.rAy;
    const double dvy = B->vy + B->w * m.rBx - A->vy - A->w * m.rAx;
    if (std::fabs(dvx * tx + dvy * ty) < p.stickSpeed) {
      m.sticking = true;
      set_anchors(A, B, m, m.cx, m.cy);
    }
  }
  time += dt;
}

void RigidWorld::solve_drag(double mscale, double bias_rate, double h) {   // rigid.js:351-371
  for (auto& bp : bodies_) {
    Body* b = bp.get();
    if (!b->dragging) continue;
    const double mi = b->invMass, ii = b->invI;
    const double Cx = b->x - b->dcx, Cy = b->y - b->dcy;
    double ix = -mscale * b->mass * (b->vx + bias_rate * Cx);
    double iy = -mscale * b->mass * (b->vy + bias_rate * Cy);
    const double maxI = b->maxForce * h, L = js_hypot(ix, iy);
    if (L > maxI) { ix *= maxI / L; iy *= maxI / L; }
    b->vx += mi * ix; b->vy += mi * iy;
    double da = b->a - b->da0;
    da -= 2 * 3.141592653589793 * js_round(da / (2 * 3.141592653589793));
    double ia = -mscale * b->I * (b->w + bias_rate * da);
    const double maxA = b->maxTorque * h;
    ia = js_max(-maxA, js_min(maxA, ia));
    b->w += ii * ia;
  }
}

void RigidWorld::solve_contacts(double bias_rate, double mscale, double iscale, double inv_h, bool use_bias) {
  for (auto& m : manifolds_) {   // rigid.js:373-416
    Body *A = m.A, *B = m.B;
    const double nx = m.nx, ny = m.ny, tx = ny, ty = -nx;
    const double cA = std::cos(A->a), sA = std::sin(A->a), cB = std::cos(B->a), sB = std::sin(B->a);
    {   // friction on the whole face (previous normal impulses), then non-penetration
      double Pn = 0;
      for (int k = 0; k < m.npts; k++) Pn += m.pts[k].Pn;
      const double dvx = B->vx - B->w * m.rBy - A->vx + A->w * m.rAy;
      const double dvy = B->vy + B->w * m.rBx - A->vy - A->w * m.rAx;
      const double vt = dvx * tx + dvy * ty;
      double newP;
      if (m.sticking) {
        double bias = 0, ms = 1, is = 0;
        if (use_bias) {
          const double pAx = A->x + cA * m.aAx - sA * m.aAy, pAy = A->y + sA * m.aAx + cA * m.aAy;
          const double pBx = B->x + cB * m.aBx - sB * m.aBy, pBy = B->y + sB * m.aBx + cB * m.aBy;
          const double drift = (pBx - pAx) * tx + (pBy - pAy) * ty;
          bias = js_max(-p.maxPushout, js_min(p.maxPushout, bias_rate * drift));
          ms = mscale; is = iscale;
        }
        const double maxS = p.muStatic * Pn;
        newP = m.Pt - m.tMass * ms * (vt + bias) - is * m.Pt;
        newP = js_max(-maxS, js_min(maxS, newP));
      } else {
        const double maxK = p.muKinetic * Pn;
        newP = js_max(-maxK, js_min(maxK, m.Pt - m.tMass * vt));
      }
      const double imp = newP - m.Pt;
      m.Pt = newP;
      apply_impulse(A, B, m, imp * tx, imp * ty);
    }
    for (int k = 0; k < m.npts; k++) {
      ContactPoint& c = m.pts[k];
      const double pAx = A->x + cA * c.lAx - sA * c.lAy, pAy = A->y + sA * c.lAx + cA * c.lAy;
      const double pBx = B->x + cB * c.lBx - sB * c.lBy, pBy = B->y + sB * c.lBx + cB * c.lBy;
      const double sep = (pBx - pAx) * nx + (pBy - pAy) * ny + c.sep;
      double bias = 0, ms = 1, is = 0;
      if (sep > 0) bias = sep * inv_h;
      else if (use_bias) {
        bias = js_max(bias_rate * sep, -p.maxPushout);
        ms = mscale; is = iscale;
      }
      const double dvx = B->vx - B->w * c.rBy - A->vx + A->w * c.rAy;
      const double dvy = B->vy + B->w * c.rBx - A->vy - A->w * c.rAx;
      const double vn = dvx * nx + dvy * ny;
      double imp = -c.nMass * ms * (vn + bias) - is * c.Pn;
      const double newP = js_max(c.Pn + imp, 0);
      imp = newP - c.Pn;
      c.Pn = newP;
      apply_impulse(A, B, c, imp * nx, imp * ny);
    }
  }
}

Body* RigidWorld::pick(double x, double y, double* lx, double* ly) {
  for (int i = (int)bodies_.size() - 1; i >= 0; i--) {
    Body* b = bodies_[i].get();
    const double dx = x - b->x, dy = y - b->y, c = std::cos(b->a), s = std::sin(b->a);
    const double px = c * dx + s * dy, py = -s * dx + c * dy;
    if (std::fabs(px) <= b->half && std::fabs(py) <= b->half) {
      if (lx) *lx = px;
      if (ly) *ly = py;
      return b;
    }
  }
  return nullptr;
}

void RigidWorld::start_drag(Body* b, double lx, double ly, double tx, double ty) {
  const double g = (p.gy != 0 && !std::isnan(p.gy)) ? std::fabs(p.gy) : 9.81;
  b->dragging = true;
  b->dlx = lx; b->dly = ly; b->da0 = b->a; b->dcx = b->x; b->dcy = b->y;
  b->maxForce = p.dragStrength * b->mass * g;
  b->maxTorque = p.dragStrength * b->mass * g * b->half;
  move_drag(b, tx, ty);
}

void RigidWorld::move_drag(Body* b, double tx, double ty) {
  if (!b->dragging) return;
  const double c = std::cos(b->da0), s = std::sin(b->da0);
  const double ox = c * b->dlx - s * b->dly, oy = s * b->dlx + c * b->dly;
  const double h = b->half * 1.42, W = p.width;
  b->dcx = js_min(W - h, js_max(h, tx - ox));
  b->dcy = js_max(h, ty - oy);
}

void RigidWorld::end_drag(Body* b) {
  if (!b->dragging) return;
  b->dragging = false;
  b->vx = 0; b->vy = 0; b->w = 0;
}

double RigidWorld::max_penetration() const {
  double m = 0;
  for (const auto& man : manifolds_)
    for (int k = 0; k < man.npts; k++) m = js_max(m, -man.pts[k].sep);
  return m;
}

// ------------------------------------------------------------------ js/contact.js
namespace {
constexpr double kGap = 0.0005, kPointLength = 0.001, kMaxSep = 0.0005;   // CONTACT, contact.js:12-16
constexpr double kEps = 0.9, kSigmaW = 5.670374e-8;                        // WOOD.eps, WOOD.sigma

int face_toward(double a, double nx, double ny) {   // contact.js:19-24
  const double c = std::cos(a), s = std::sin(a);
  const double lx = c * nx + s * ny, ly = -s * nx + c * ny;
  if (std::fabs(lx) > std::fabs(ly)) return lx > 0 ? 0 : 2;
  return ly > 0 ? 1 : 3;
}
}  // namespace

double contact_conductance(double T) {   // contact.js:26-30
  const double kGas = 0.0241 * std::pow(T / 273.15, 0.8);
  return kGas / kGap + 4 * kSigmaW * T * T * T / (2 / kEps - 1);
}

double exchange_contacts(const RigidWorld& world, double dt, ContactWood& wood) {   // contact.js:33-56
  double moved = 0;
  if (dt <= 0) return moved;
  for (const auto& m : world.manifolds()) {
    const int pa = m.A->user, pb = m.B->user;
    if (pa < 0 || pb < 0) continue;   // floor and walls are adiabatic
    const ContactPoint* pts[4];
    int n = 0;
    for (int k = 0; k < m.npts; k++)
      if (m.pts[k].sep < kMaxSep) pts[n++] = &m.pts[k];
    if (!n) continue;
    const double L = n >= 2 ? js_hypot(pts[0]->x - pts[1]->x, pts[0]->y - pts[1]->y) : kPointLength;
    if (L <= 0) continue;
    const int fa = face_toward(m.A->a, m.nx, m.ny);
    const int fb = face_toward(m.B->a, -m.nx, -m.ny);
    const double Ta = wood.Ts(pa, fa), Tb = wood.Ts(pb, fb);
    const double G = contact_conductance(0.5 * (Ta + Tb)) * L;
    const double Ca = wood.surface_cap(pa, fa), Cb = wood.surface_cap(pb, fb);
    const double inv = 1 / Ca + 1 / Cb;
    const double E = (Ta - Tb) * (1 - std::exp(-G * inv * dt)) / inv;
    wood.Ts(pa, fa) -= E / Ca;
    wood.Ts(pb, fb) += E / Cb;
    moved += std::fabs(E);
  }
  return moved;
}

}  // namespace cfg
