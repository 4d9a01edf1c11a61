// Host-side wood model and the per-frame wood <-> gas coupling of the campfire
// app, around the GPU gas step.
//
// WoodPiece restates js/wood.js (WOOD constants :12-31, the class :33-182) in
// double precision, as the reference computes it in JS numbers. WoodScene
// restates the frame loop of js/main.js for frozen bodies (the rigid-body world
// and contacts are out of this path): addPiece :103-119 (slots, per-piece
// qConv/qInc/vis/charPending), uploadPieces :190-207, onReadback :209-230,
// stepWood :232-243 and the gas part of frame() :247-283.
#pragma once
#include <array>
#include <cstdint>
#include <memory>
#include <vector>

#include "rigid.h"

namespace cfg {

class Engine;

struct WoodCtl {
  double charYield = 0.25, pyroMult = 1.0;   // js/config.js:55-57 CONTROL_DEFAULTS
};

struct WoodPiece {
  double rhoV = 500, rhoC = 150, mv = 0, mc = 0, Tc = 293.15, gasRate = 0, side = 0;
  std::array<double, 4> Ts{}, Tp{}, d{}, mflux{}, charCov{}, exposure{1, 1, 1, 1};
  bool dead = false;

  WoodPiece() = default;
  WoodPiece(double side, double rhoV, double T0 = 293.15);   // js/wood.js:34-49
  double half() const { return 0.5 * side; }
  void updateSide();                                          // :60
  double surfaceCap(int f) const;                             // :53-58
  double charFraction() const;                                // :61
  void preheat(double Tsurf, double charDepth, double Tcore, double charYield);   // :64-76
  // :82-181: heat inputs per face (qConv W/m, qInc W/m^2, char burnt kg/m)
  void step(double dt, const std::array<double, 4>& qConv, const std::array<double, 4>& qInc,
            const std::array<double, 4>& charBurnt, const WoodCtl& ctl);
};

// A piece of the scene: its body (frozen: position and angle fixed, size from the
// wood; moving: a body of the scene's rigid world)
struct WoodSlot {
  bool used = false;
  uint64_t serial = 0;              // which piece holds the slot (a readback applies only to it)
  double x = 0, y = 0, angle = 0;
  int body = 0;                     // rigid body id (moving pieces), 0 when frozen
  WoodPiece wood;
  std::array<double, 4> qConv{}, qInc{}, vis{}, charPending{};
};

class WoodScene {
 public:
  WoodScene(Engine* eng, int scene, WoodCtl ctl) : eng_(eng), scene_(scene), ctl_(ctl) {}
  // moving pieces: a rigid world (js/main.js:61, friction from the controls :93-94) that
  // the frame advances before the wood step; only while the scene has no pieces
  int set_rigid(const RigidParams* p);
  RigidWorld* world() { return world_.get(); }
  // :103-119 (returns the slot, or a negative status when all 64 are taken)
  int add(double x, double y, double angle, double side, double density, const double* preheat3,
          const double* faceT4);
  int remove(int slot);
  // replace a piece's wood state (the app's defaultScene sets coal state directly, main.js:135-142)
  int set(int slot, const WoodPiece& w);
  // one frame of main.js frame() with `sim_dt` of gas time: the wood steps on the
  // last readback, pieces are uploaded, geometry rebuilt, floor(sim_dt/dt) gas steps
  // (at most ceil(0.034/dt)) and radiation run, and the readback applied
  int frame(double sim_dt, int* nsteps);
  const WoodSlot* slot(int s) const { return (s >= 0 && s < (int)slots_.size() && slots_[s].used) ? &slots_[s] : nullptr; }
  double hrr = 0, rad = 0, tmax = 0;   // stats of the last readback (main.js:225-229, before smoothing)
  // the renderer's wood buffer built with the last upload (main.js:188-207): 64 x {Tp[4], d[4],
  // char fraction, Tcore, mean visible irradiance, has virgin wood}
  const std::vector<float>& render_wood() const { return render_wood_; }
  // How a frame's readback reaches the wood. lag 0 (default): synchronously at the end of the
  // frame. Otherwise the reference's way (encodeReadback + afterSubmit, js/fluid.js:315-342, with
  // onReadback's tag, js/main.js:210-230): the frame enqueues its readback on the ring with a tag
  // holding its gas time and the pieces that held the slots, and readbacks are applied at the
  // start of later frames, before the wood steps, to those pieces only. lag < 0: whatever has
  // arrived, never waiting (the reference; a frame whose ring slot is still pending skips its
  // readback, and acc keeps accumulating); lag 1..3: the readback of the frame `lag` frames back,
  // waited for (a fixed pipeline depth, the same from run to run; the ring never fills).
  int set_readback_lag(int lag);
  int readback_lag() const { return lag_; }
  uint64_t applied = 0, skipped = 0;   // readbacks applied and skipped (lag != 0)

 private:
  int upload();
  int readback(double sim_dt);
  // one readback's data applied with its frame's gas time to the pieces that still hold their slots
  void apply(const int32_t* acc, const float* radv, const int32_t* faceW, double sim_dt, const uint64_t* owners);
  // apply the readbacks that have arrived (wait_upto > 0: wait for every tag <= wait_upto first)
  int collect(uint64_t wait_upto);
  struct Pending { double simDt; std::array<uint64_t, 64> owners; };
  int lag_ = 0;
  uint64_t next_serial_ = 1, next_tag_ = 1;
  std::vector<std::pair<uint64_t, Pending>> pending_;   // tags in flight on the ring
  Engine* eng_;
  int scene_;
  WoodCtl ctl_;
  std::vector<WoodSlot> slots_ = std::vector<WoodSlot>(64);
  double sim_acc_ = 0;
  std::vector<float> render_wood_ = std::vector<float>(64 * 12, 0.f);
  std::unique_ptr<RigidWorld> world_;
  friend struct SlotWood;
};

}  // namespace cfg
