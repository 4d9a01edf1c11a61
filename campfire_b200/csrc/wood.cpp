// Wood model (js/wood.js) and the frame coupling with the gas step (js/main.js);
// see wood.h. Expressions keep the reference's operation order (JS evaluates
// left to right in double precision); the library's host code is built without
// floating-point contraction.
#include "wood.h"

#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.h"

namespace cfg {

namespace {
// js/wood.js:12-31
struct WoodK {
  static constexpr double cv = 1500, kv = 0.15, cc = 1000, kc = 0.08, pore = 0.001, charDensityRatio = 0.3, eps = 0.9;
  static constexpr double pyroA = 2.0e7, pyroTa = 12000, dHpyro = 3.0e5, dHchar = 32.8e6, cpGas = 1150;
  static constexpr double deltaS = 0.0015, deltaP = 0.002, minDepth = 0.0004, sigma = 5.670374e-8, minHalf = 0.0015;
};
// js/fluid.js:9 fixed-point scales of the acc readback
constexpr double E_SCALE = 1e6, M_SCALE = 1e12, G_SCALE = 1e3;
constexpr double kTamb = 293.15, kSigma = 5.670374e-8;   // js/config.js PHYS
}  // namespace

WoodPiece::WoodPiece(double side_, double rhoV_, double T0) {
  rhoV = rhoV_;
  rhoC = rhoV_ * WoodK::charDensityRatio;
  mv = rhoV_ * side_ * side_;
  mc = 0;
  Ts = {T0, T0, T0, T0};
  Tp = {T0, T0, T0, T0};
  d = {0, 0, 0, 0};
  Tc = T0;
  mflux = {0, 0, 0, 0};
  charCov = {0, 0, 0, 0};
  gasRate = 0;
  exposure = {1, 1, 1, 1};
  dead = false;
  side = side_;
}

void WoodPiece::updateSide() { side = std::sqrt(mv / rhoV + mc / rhoC); }

double WoodPiece::surfaceCap(int f) const {
  const double s = side;
  const double dS = std::min(WoodK::deltaS, s / 8);
  const double phi = mv <= 1e-9 ? 1 : std::min(1.0, d[f] / dS);
  return (rhoV * WoodK::cv * (1 - phi) + rhoC * WoodK::cc * phi) * dS * s;
}

double WoodPiece::charFraction() const { return mc / rhoC / (mv / rhoV + mc / rhoC + 1e-12); }

void WoodPiece::preheat(double Tsurf, double charDepth, double Tcore, double charYield) {
  const double s = side;
  const double dv = std::min(charDepth, 0.45 * s);
  const double vVol = 4 * dv * s - 4 * dv * dv;
  const double consumed = std::min(mv * 0.98, vVol * rhoV);
  mv -= consumed;
  mc += consumed * charYield;
  d = {dv, dv, dv, dv};
  Ts = {Tsurf, Tsurf, Tsurf, Tsurf};
  for (int f = 0; f < 4; f++) Tp[f] = 0.5 * (Ts[f] + Tcore);
  Tc = Tcore;
  updateSide();
}

void WoodPiece::step(double dt, const std::array<double, 4>& qConv, const std::array<double, 4>& qInc,
                     const std::array<double, 4>& charBurnt, const WoodCtl& ctl) {
  if (dead) return;
  using W = WoodK;
  const double Yc = ctl.charYield;
  // burning char: its mass leaves the piece and its heat goes to the face
  std::array<double, 4> qChar{0, 0, 0, 0};
  for (int f = 0; f < 4; f++) {
    const double m = std::min(charBurnt[f], mc);
    mc -= m;
    qChar[f] = m * W::dHchar / dt;
    d[f] = std::max(0.0, d[f] - m / (rhoC * std::max(side, 1e-3)));
  }
  updateSide();
  const int nsub = std::max(1, (int)std::ceil(dt / 0.004));
  const double h = dt / nsub;
  double gasTotal = 0;
  std::array<double, 4> gasFace{0, 0, 0, 0};
  for (int n = 0; n < nsub; n++) {
    const double s = side;
    const double dS = std::min(W::deltaS, s / 8), dP = std::min(W::deltaP, s / 8);
    const bool allChar = mv <= 1e-9;
    // heat capacity of each layer, J/K per m of depth
    const double rcv = rhoV * W::cv, rcc = rhoC * W::cc;
    std::array<double, 4> Cs{}, Cp{};
    double Csum = 0;
    for (int f = 0; f < 4; f++) {
      const double phi = allChar ? 1 : std::min(1.0, d[f] / dS);
      Cs[f] = (rcv * (1 - phi) + rcc * phi) * dS * s;
      Cp[f] = (allChar ? rcc : rcv) * dP * s;
      Csum += Cs[f] + Cp[f];
    }
    const double Ctot = mv * W::cv + mc * W::cc;
    const double Cc = std::max(0.1 * Ctot, Ctot - Csum);
    // virgin wood turning into gas and char
    const double A = W::pyroA * ctl.pyroMult;
    const double mFrontCap = rhoV * dP * s;
    double mFrontSum = 0;
    std::array<double, 4> rf{0, 0, 0, 0};
    for (int f = 0; f < 4; f++) {
      const double mFront = std::min(mFrontCap, mv / 5);
      mFrontSum += mFront;
      rf[f] = A * std::exp(-W::pyroTa / Tp[f]) * mFront;
    }
    const double rCore = A * std::exp(-W::pyroTa / Tc) * std::max(0.0, mv - mFrontSum);
    double rTot = rf[0] + rf[1] + rf[2] + rf[3] + rCore;
    if (rTot * h > mv) {   // cap the step's loss at the virgin mass left
      const double k = mv / (rTot * h);
      for (int f = 0; f < 4; f++) rf[f] *= k;
      rTot *= k;
    }
    const double rC = rTot - (rf[0] + rf[1] + rf[2] + rf[3]);
    // conductances
    const double kvv = allChar ? W::kc : W::kv;
    double coreIn = 0;
    for (int f = 0; f < 4; f++) {
      const double df = d[f];
      // the char layer conducts by its solid and by radiation through its pores
      const double Tm = 0.5 * (Ts[f] + Tp[f]);
      const double kcEff = W::kc + 4 * W::eps * W::sigma * Tm * Tm * Tm * W::pore;
      const double Gsp = s / (df / kcEff + (dS + dP) / (2 * kvv));
      const double Lpc = std::max(0.5 * (0.5 * s - df), 0.001);
      const double Gpc = kvv * s / Lpc;
      const double gas = (1 - Yc) * (rf[f] + 0.25 * rC);   // gas mass per second and m of depth through this face
      gasFace[f] += gas * h;
      const double Tsf = Ts[f], Tpf = Tp[f];
      const double eps = W::eps;
      const double ex = exposure[f];
      const double qRad = eps * s * ex * (qInc[f] - W::sigma * Tsf * Tsf * Tsf * Tsf);
      const double dRad = 4 * eps * W::sigma * Tsf * Tsf * Tsf * s * ex;
      const double qs = qConv[f] + qRad + qChar[f] - Gsp * (Tsf - Tpf) - gas * W::cpGas * (Tsf - Tpf);
      Ts[f] = Tsf + h * qs / (Cs[f] + h * (dRad + Gsp));
      const double qp = Gsp * (Tsf - Tpf) - Gpc * (Tpf - Tc) - W::dHpyro * rf[f];
      Tp[f] = Tpf + h * qp / (Cp[f] + h * (Gsp + Gpc));
      coreIn += Gpc * (Tpf - Tc);
      // the charred depth advances by the char this face has made
      if (!allChar) d[f] = std::min(0.5 * s, d[f] + rf[f] * h / (rhoV * s));
    }
    Tc += h * (coreIn - W::dHpyro * rC) / Cc;
    mv -= rTot * h;
    mc += Yc * rTot * h;
    if (mv < 1e-9) mv = 0;
    gasTotal += (1 - Yc) * rTot * h;
    updateSide();
  }
  gasRate = gasTotal / dt;
  const double s = std::max(side, 1e-4);
  // volatiles leave through the open faces; gas from covered faces goes to the exposed ones
  const double exSum = exposure[0] + exposure[1] + exposure[2] + exposure[3];
  double blocked = 0;
  for (int f = 0; f < 4; f++) blocked += gasFace[f] * (1 - exposure[f]);
  for (int f = 0; f < 4; f++) {
    const double g = gasFace[f] * exposure[f] + (exSum > 0.05 ? blocked * exposure[f] / exSum : 0);
    mflux[f] = exposure[f] > 0.02 ? g / dt / s : 0;
    charCov[f] = mv <= 0 ? 1 : std::min(1.0, d[f] / W::minDepth);
  }
  if (half() < W::minHalf || (mv + mc) < 1e-7) dead = true;
}

// ------------------------------------------------------------------ the frame loop
int WoodScene::add(double x, double y, double angle, double side, double density, const double* preheat3,
                   const double* faceT4) {
  if (!(side > 0) || !(density > 0)) return fail(CFG_ERR_INVAL, "piece side and density must be positive");
  int slot = -1;
  for (int s = 0; s < (int)slots_.size(); s++)
    if (!slots_[s].used) { slot = s; break; }
  if (slot < 0) return fail(CFG_ERR_RANGE, "all 64 piece slots are in use");
  WoodSlot& p = slots_[slot];
  p = WoodSlot{};
  p.used = true;
  p.serial = next_serial_++;
  p.x = x; p.y = y; p.angle = angle;
  p.wood = WoodPiece(side, density);
  if (preheat3) p.wood.preheat(preheat3[0], preheat3[1], preheat3[2], ctl_.charYield);
  if (faceT4)
    for (int f = 0; f < 4; f++)
      if (faceT4[f] != 0) {
        p.wood.Ts[f] = faceT4[f];
        p.wood.Tp[f] = std::max(p.wood.Tp[f], 0.5 * (faceT4[f] + p.wood.Tc));
      }
  const double qa = kSigma * std::pow(kTamb, 4);
  p.qInc = {qa, qa, qa, qa};
  if (world_) {   // new Body(x, y, half, (mv + mc) / side^2, angle) (main.js:109-110)
    Body* b = world_->add(x, y, p.wood.half(), (p.wood.mv + p.wood.mc) / (p.wood.side * p.wood.side), angle);
    b->user = slot;
    p.body = b->id;
  }
  return slot;
}

int WoodScene::set_rigid(const RigidParams* rp) {
  for (const auto& p : slots_)
    if (p.used) return fail(CFG_ERR_BUSY, "the rigid world can be switched only while the scene has no pieces");
  if (rp) world_ = std::make_unique<RigidWorld>(*rp);
  else world_.reset();
  return CFG_OK;
}

// the wood side of js/contact.js: a slot's surface temperatures and capacities
struct SlotWood : ContactWood {
  std::vector<WoodSlot>& slots;
  explicit SlotWood(std::vector<WoodSlot>& s) : slots(s) {}
  double& Ts(int user, int f) override { return slots[user].wood.Ts[f]; }
  double surface_cap(int user, int f) override { return slots[user].wood.surfaceCap(f); }
};

int WoodScene::set(int slot, const WoodPiece& w) {
  if (slot < 0 || slot >= (int)slots_.size() || !slots_[slot].used) return fail(CFG_ERR_NOENT, "no piece in this slot");
  if (!(w.side > 0) || !(w.rhoV > 0) || !(w.rhoC > 0)) return fail(CFG_ERR_INVAL, "piece side and densities must be positive");
  slots_[slot].wood = w;
  return CFG_OK;
}

int WoodScene::remove(int slot) {
  if (slot < 0 || slot >= (int)slots_.size() || !slots_[slot].used) return fail(CFG_ERR_NOENT, "no piece in this slot");
  if (world_ && slots_[slot].body) world_->remove(slots_[slot].body);
  slots_[slot] = WoodSlot{};
  return CFG_OK;
}

int WoodScene::upload() {
  std::vector<float> data((size_t)MAX_PIECES * PIECE_FLOATS, 0.f);
  std::fill(render_wood_.begin(), render_wood_.end(), 0.f);
  int n = 0;
  for (int s = 0; s < (int)slots_.size(); s++) {
    const WoodSlot& p = slots_[s];
    if (!p.used) continue;
    // the renderer's wood buffer (main.js:200-203)
    float* r = render_wood_.data() + (size_t)s * 12;
    for (int f = 0; f < 4; f++) {
      r[f] = (float)p.wood.Tp[f];
      r[4 + f] = (float)p.wood.d[f];
    }
    r[8] = (float)p.wood.charFraction();
    r[9] = (float)p.wood.Tc;
    r[10] = (float)((p.vis[0] + p.vis[1] + p.vis[2] + p.vis[3]) / 4);
    r[11] = p.wood.mv > 0 ? 1.f : 0.f;
    float* o = data.data() + (size_t)s * PIECE_FLOATS;
    const Body* b = world_ && p.body ? world_->find(p.body) : nullptr;
    const float body[8] = {(float)(b ? b->x : p.x), (float)(b ? b->y : p.y), (float)(b ? b->a : p.angle),
                           (float)(b ? b->half : p.wood.half()), (float)(b ? b->vx : 0.0), (float)(b ? b->vy : 0.0),
                           (float)(b ? b->w : 0.0), 1.f};
    std::memcpy(o, body, sizeof body);
    for (int f = 0; f < 4; f++) {
      o[8 + f] = (float)p.wood.Ts[f];
      o[12 + f] = (float)p.wood.mflux[f];
      o[16 + f] = (float)p.wood.charCov[f];
    }
    n = std::max(n, s + 1);
  }
  return eng_->upload_pieces(scene_, data.data(), n);
}

int WoodScene::readback(double sim_dt) {
  if (lag_ != 0) {
    // encodeReadback + afterSubmit with the frame's tag {simDt, owners} (js/main.js:281-283)
    Pending pd;
    pd.simDt = sim_dt;
    for (int s = 0; s < (int)slots_.size(); s++) pd.owners[s] = slots_[s].used ? slots_[s].serial : 0;
    const uint64_t tag = next_tag_++;
    const int rc = eng_->readback_begin(scene_, tag, nullptr);
    if (rc == CFG_ERR_BUSY) { skipped++; return CFG_OK; }
    CFG_TRY(rc);
    pending_.emplace_back(tag, pd);
    return CFG_OK;
  }
  std::vector<int32_t> acc(ACC_LEN), faceW(MAX_PIECES * 4);
  std::vector<float> radv((size_t)RAD_LEN * 4);
  CFG_TRY(eng_->readback(scene_, acc.data(), radv.data(), faceW.data()));
  apply(acc.data(), radv.data(), faceW.data(), sim_dt, nullptr);
  return CFG_OK;
}

// the readbacks in flight, oldest first: those with tags <= wait_upto are waited for, the
// rest taken only if they have arrived (never, for a fixed lag: they wait their turn)
int WoodScene::collect(uint64_t wait_upto) {
  std::vector<int32_t> acc(ACC_LEN), faceW(MAX_PIECES * 4);
  std::vector<float> radv((size_t)RAD_LEN * 4);
  while (!pending_.empty()) {
    const bool wait = pending_.front().first <= wait_upto;
    if (!wait && lag_ > 0) return CFG_OK;
    uint64_t tag = 0;
    int ready = 0;
    CFG_TRY(eng_->readback_collect(scene_, wait, acc.data(), radv.data(), faceW.data(), &tag, &ready));
    if (!ready) return CFG_OK;
    auto it = pending_.begin();
    while (it != pending_.end() && it->first != tag) ++it;
    if (it == pending_.end()) return fail(CFG_ERR_INVAL, "a readback arrived with an unknown tag");
    const Pending pd = it->second;
    pending_.erase(it);
    apply(acc.data(), radv.data(), faceW.data(), pd.simDt, pd.owners.data());
    applied++;
  }
  return CFG_OK;
}

int WoodScene::set_readback_lag(int lag) {
  if (lag > 3) return fail(CFG_ERR_INVAL, "readback lag must be at most 3 frames (the ring's slots)");
  if (!pending_.empty()) CFG_TRY(collect(~0ull));   // deliver what is in flight before switching
  lag_ = lag < 0 ? -1 : lag;
  return CFG_OK;
}

// onReadback (js/main.js:210-230): owners = the serials of the pieces that held the slots when
// the readback's frame ran (null: the current ones)
void WoodScene::apply(const int32_t* acc, const float* radv, const int32_t* faceW, double sim_dt,
                      const uint64_t* owners) {
  if (sim_dt <= 0) return;
  for (int s = 0; s < (int)slots_.size(); s++) {
    WoodSlot& p = slots_[s];
    if (!p.used || (owners && owners[s] != p.serial)) continue;
    for (int f = 0; f < 4; f++) {
      // share of the face that touches gas: none where it rests on the floor or another piece
      p.wood.exposure[f] = std::min(1.0, faceW[s * 4 + f] / 1e8 / std::max(p.wood.side, 1e-4));
      const int k = (s * 4 + f) * 2;
      p.qConv[f] = acc[k] / E_SCALE / sim_dt;
      p.charPending[f] += acc[k + 1] / M_SCALE;
      p.qInc[f] = radv[(s * 4 + f) * 4];
      p.vis[f] = radv[(s * 4 + f) * 4 + 1];
    }
  }
  hrr = acc[ACC_GLOBAL] / G_SCALE / sim_dt;
  rad = acc[ACC_GLOBAL + 1] / G_SCALE / sim_dt;
  tmax = acc[ACC_GLOBAL + 2];
}

int WoodScene::frame(double sim_dt, int* nsteps) {
  if (!(sim_dt >= 0)) return fail(CFG_ERR_INVAL, "frame time must be >= 0");
  // dt and the frame counter from the host side: a frame does not wait for the device
  const double dt = eng_->host_dt(scene_);
  const uint32_t frame_no = eng_->host_frame(scene_);
  // gas steps for this frame, capped at ceil(0.034 / dt) (js/main.js:252-257)
  sim_acc_ += sim_dt;
  const int maxSteps = (int)std::ceil(0.034 / dt);
  int n = (int)std::floor(sim_acc_ / dt);
  if (n > maxSteps) { n = maxSteps; sim_acc_ = 0; } else sim_acc_ -= n * dt;
  const double simDt = n * dt;
  // readbacks of earlier frames, applied before this frame starts (the reference's callbacks run
  // between frames; the tag of frame f is f + 1): with a fixed lag the one of the frame `lag`
  // back, waited for; otherwise whatever has arrived
  if (lag_ != 0) CFG_TRY(collect(lag_ > 0 && next_tag_ > (uint64_t)lag_ ? next_tag_ - (uint64_t)lag_ : 0));
  // the bodies move and touching pieces exchange heat (:262-263; the simulation runs, so
  // the rigid world advances by the frame's gas time)
  if (world_) {
    world_->advance(simDt);
    SlotWood sw(slots_);
    exchange_contacts(*world_, simDt, sw);
  }
  // stepWood (:232-243): the wood advances on the last readback's heat inputs
  if (simDt > 0)
    for (auto& p : slots_) {
      if (!p.used) continue;
      p.wood.step(simDt, p.qConv, p.qInc, p.charPending, ctl_);
      p.charPending = {0, 0, 0, 0};
      if (p.wood.dead) {
        if (world_ && p.body) world_->remove(p.body);
        p = WoodSlot{};
        continue;
      }
      if (world_ && p.body) {
        Body* b = world_->find(p.body);
        b->density = (p.wood.mv + p.wood.mc) / (p.wood.side * p.wood.side);
        world_->resize(b, p.wood.half());
      }
    }
  CFG_TRY(upload());
  CFG_TRY(eng_->write_params(scene_));
  CFG_TRY(eng_->clear_geometry(scene_));
  CFG_TRY(eng_->geometry(scene_));
  CFG_TRY(eng_->step(n));
  CFG_TRY(eng_->radiation(scene_));
  CFG_TRY(eng_->set_frame(scene_, frame_no + 1));
  if (nsteps) *nsteps = n;
  return readback(simDt);
}

}  // namespace cfg
