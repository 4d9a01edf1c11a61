// 2D rigid bodies of the campfire app: square wood pieces per unit depth, their
// contacts with the floor, the side walls and each other, and the hand grip.
//
// Restates js/rigid.js (RIGID_DEFAULTS :12-27, makeSoft :29-36, Body :40-59,
// box geometry and SAT manifolds :61-156, RigidWorld :159-468, applyImpulse
// :471-476) in double precision with the reference's order of operations, and
// js/contact.js (heat exchange across wood-wood contacts) for the wood scene.
// JavaScript semantics that matter for bit-for-bit results are kept: Map
// iteration in insertion order (manifolds), Math.round (ties toward +inf) and
// Math.hypot as V8 computes it (normalise by the largest magnitude, Kahan-summed
// squares).
#pragma once
#include <cstdint>
#include <memory>
#include <unordered_map>
#include <vector>

#include "../../include/campfire_gas.h"

namespace cfg {

double js_hypot(double x, double y);
double js_round(double x);

struct RigidParams {                // RIGID_DEFAULTS, js/rigid.js:12-27
  double gx = 0, gy = -9.81;
  double width = 0.7;               // walls that keep the pieces in [0, width]
  double dt = 1.0 / 480;            // step of the collision solver (s)
  int substeps = 4;
  double slop = 0.0002;
  double contactHertz = 240, contactDamping = 10, maxPushout = 0.25;
  double muStatic = 0.7, muKinetic = 0.5, stickSpeed = 0.002, maxSpeed = 8;
  double dragHertz = 8, dragStrength = 2.5;
};

struct Body {
  int id = 0;                       // 0: the static floor/walls
  double x = 0, y = 0, a = 0, vx = 0, vy = 0, w = 0;
  double density = 0, half = 0, mass = 0, invMass = 0, I = 0, invI = 0;
  bool dragging = false;
  double dlx = 0, dly = 0, da0 = 0, dcx = 0, dcy = 0, maxForce = 0, maxTorque = 0;   // the hand grip
  int user = -1;                    // owner tag (the wood scene's slot)
  void set_half(double h);          // :50-58
};

struct ContactPoint {
  int id = 0;
  double x = 0, y = 0, sep = 0, Pn = 0;
  double lAx = 0, lAy = 0, lBx = 0, lBy = 0, rAx = 0, rAy = 0, rBx = 0, rBy = 0, nMass = 0;
};

struct Manifold {
  uint64_t key = 0;
  Body *A = nullptr, *B = nullptr;
  double nx = 0, ny = 0;
  ContactPoint pts[4];
  int npts = 0;
  double cx = 0, cy = 0, Pt = 0;
  bool sticking = true;
  double aAx = 0, aAy = 0, aBx = 0, aBy = 0;   // friction anchors (material points)
  double rAx = 0, rAy = 0, rBx = 0, rBy = 0, tMass = 0;
};

class RigidWorld {
 public:
  explicit RigidWorld(const RigidParams& p) : p(p) {}
  RigidParams p;

  Body* add(double x, double y, double half, double density, double angle);   // new Body + add
  int remove(int id);                                                         // :168-172
  void resize(Body* b, double half);                                          // :176-184
  void advance(double dt);                                                    // :187-193
  void step(double dt);                                                       // :271-346
  Body* find(int id);
  Body* pick(double x, double y, double* lx, double* ly);                    // :419-428
  void start_drag(Body* b, double lx, double ly, double tx, double ty);      // :431-439
  void move_drag(Body* b, double tx, double ty);                              // :440-449
  void end_drag(Body* b);                                                     // :451-455
  double max_penetration() const;                                             // :458-462
  const std::vector<std::unique_ptr<Body>>& bodies() const { return bodies_; }
  const std::vector<Manifold>& manifolds() const { return manifolds_; }
  double time = 0, accum = 0;

 private:
  void collide(double dt);                                                    // :195-259
  void take(uint64_t key, Body* A, Body* B, const Manifold& man, const std::vector<Manifold>& old,
            const std::unordered_map<uint64_t, int>& old_index);
  static void set_anchors(const Body* A, const Body* B, Manifold& m, double px, double py);
  void solve_drag(double mscale, double bias_rate, double h);
  void solve_contacts(double bias_rate, double mscale, double iscale, double inv_h, bool use_bias);
  std::vector<std::unique_ptr<Body>> bodies_;
  std::vector<Manifold> manifolds_;   // insertion order, as the reference's Map
  Body static_{};
  int next_id_ = 1;
};

// js/contact.js: heat exchange over dt across the wood-wood contacts of a world.
// face_T(user, f) / cap(user, f) give a piece's surface temperature and capacity.
struct ContactWood {
  virtual double& Ts(int user, int f) = 0;
  virtual double surface_cap(int user, int f) = 0;
  virtual ~ContactWood() = default;
};
double exchange_contacts(const RigidWorld& w, double dt, ContactWood& wood);
double contact_conductance(double T);

}  // namespace cfg
