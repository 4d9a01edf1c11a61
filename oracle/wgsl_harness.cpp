// ORACLE — test infrastructure, not product code.
// Runs the reference's WGSL kernels, mechanically translated to C++ by
// oracle/wgsl2cpp.py (oracle/_ref/wgsl_gen.hpp), with the buffers, bind groups
// and dispatch order of FluidSim (js/fluid.js): init :49-91 (six-level cap as in
// the reference), reset :162-176, writeParams :180-199, uploadPieces :201-204,
// clearGeometry/encodeGeometry :213-218, encodeRadiation :220-222, encodeStep
// :225-253 (one V-cycle, vcycle :294-312), encodeReadback :315-324. Exposes the
// wref_* C surface, argument for argument the orc_* surface of oracle_capi.cpp.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "wgsl_gen.hpp"
#include "wgsl_rt.hpp"

namespace {
thread_local std::string g_err;

const char* kParamNames[40] = {
  "nx", "ny", "dx", "dt", "Tamb", "rhoAmb", "YOamb", "grav", "cp", "Pr", "viscMult", "diffMult",
  "reactB", "reactTa", "dHc", "sO2", "sootFormA", "sootFormTa", "sootOxA", "sootOxTa",
  "kappaSootC", "kappaGas", "exchAlpha", "depth", "charA", "charTa", "nPieces", "frame",
  "heaterX0", "heaterX1", "heaterY1", "heaterT", "burnerX0", "burnerX1", "burnerFlux", "burnerT",
  "sootDensity", "sigma", "charO2", "time"};
int param_index(const char* n) { for (int i = 0; i < 40; i++) if (!std::strcmp(kParamNames[i], n)) return i; return -1; }

// js/config.js PHYS (the reference computes rhoAmb and sO2 in JS doubles)
const double kTamb = 293.15, kRhoAmb = 101325 * 0.0289 / (8.314462 * 293.15), kPr = 0.7;

struct Uni { int32_t nx, ny; float h2; int32_t color; };   // pressure.wgsl:7 Level uniform

struct Lv {
  int nx, ny; double h;
  std::vector<float> p, rhs, ax, ay;
  Uni u[2];
};

struct RefSim {
  int nx, ny; double dx, dt, time = 0; uint32_t frame = 0;
  uint32_t P[40];        // the uploaded uniform (raw words)
  uint32_t host[40];     // FluidSim.params
  std::vector<float> U, Uh, U2, V, Vh, V2, T, Th, T2, Y, Yh, Y2, SQ, cellG, fx, fy, pieces, rad;
  std::vector<int32_t> acc, faceW;
  std::vector<Lv> lv;
  float diffU[4] = {0, 0, 0, 0};
  int diffSub = 1;

  void setf(int i, double v) { float f = (float)v; std::memcpy(&host[i], &f, 4); }
  void seti(int i, int32_t v) { std::memcpy(&host[i], &v, 4); }
  float getf(int i) const { float f; std::memcpy(&f, &host[i], 4); return f; }

  RefSim(int nx_, int ny_, double width, double dt_) : nx(nx_), ny(ny_), dx(width / nx_), dt(dt_) {
    std::memset(host, 0, sizeof host);
    // js/fluid.js:35-45
    setf(4, kTamb); setf(5, kRhoAmb); setf(6, 0.232); setf(7, 9.81); setf(8, 1300); setf(9, kPr); setf(10, 1); setf(11, 1);
    setf(12, 2.0e10); setf(13, 15000); setf(14, 15.0e6); setf(15, 15.0e6 / 13.1e6); setf(16, 6.0e6); setf(17, 25000);
    setf(18, 5.4e8); setf(19, 19800); setf(20, 1862); setf(21, 0.8); setf(22, 0.05); setf(23, 0.8); setf(24, 6.6);
    setf(25, 5800); seti(26, 0); setf(35, 600); setf(36, 1800); setf(37, 5.670374e-8); setf(38, 2.667);
    const size_t nC = (size_t)nx * ny, nU = (size_t)(nx + 1) * ny, nV = (size_t)nx * (ny + 1);
    for (auto* a : {&U, &Uh, &U2}) a->assign(nU, 0.f);
    for (auto* a : {&V, &Vh, &V2}) a->assign(nV, 0.f);
    for (auto* a : {&T, &Th, &T2}) a->assign(nC, 0.f);
    for (auto* a : {&Y, &Yh, &Y2}) a->assign(nC * 4, 0.f);
    SQ.assign(nC * 2, 0.f); cellG.assign(nC * 2, 0.f); fx.assign(nU, 0.f); fy.assign(nV, 0.f);
    pieces.assign(64 * 20, 0.f); acc.assign(528, 0); rad.assign(320 * 4, 0.f); faceW.assign(256, 0);
    int lx = nx, ly = ny; double h = dx;
    for (int l = 0; l < 6; l++) {
      Lv L; L.nx = lx; L.ny = ly; L.h = h;
      L.p.assign((size_t)lx * ly, 0.f); L.rhs.assign((size_t)lx * ly, 0.f);
      L.ax.assign((size_t)(lx + 1) * ly, 0.f); L.ay.assign((size_t)lx * (ly + 1), 0.f);
      for (int c = 0; c < 2; c++) L.u[c] = Uni{lx, ly, (float)(h * h), c};
      lv.push_back(L);
      if (lx % 2 || ly % 2 || lx * ly <= 256) break;
      lx /= 2; ly /= 2; h *= 2;
    }
    if (lv.back().nx * lv.back().ny > 256) throw std::runtime_error("coarsest level too large");
    write_params();
    reset();
  }
  void reset() {
    std::fill(T.begin(), T.end(), (float)kTamb); T2 = T; Th = T;
    for (auto* a : {&Y, &Y2, &Yh})
      for (size_t k = 0; k < a->size() / 4; k++) { (*a)[4 * k] = 0; (*a)[4 * k + 1] = getf(6); (*a)[4 * k + 2] = 0; (*a)[4 * k + 3] = 0; }
    for (auto* a : {&U, &Uh, &U2, &V, &Vh, &V2, &SQ, &rad}) std::fill(a->begin(), a->end(), 0.f);
    std::fill(acc.begin(), acc.end(), 0);
    for (auto& L : lv) std::fill(L.p.begin(), L.p.end(), 0.f);
    time = 0;
  }
  void write_params() {
    seti(0, nx); seti(1, ny); setf(2, dx); setf(3, dt); setf(39, time); std::memcpy(&host[27], &frame, 4);
    std::memcpy(P, host, sizeof P);
    const double Tmax = 2200, mu = 1.716e-5 * std::pow(Tmax / 273.15, 1.5) * 383.55 / (Tmax + 110.4);
    const double alpha = mu / kPr * (double)getf(11) / (kRhoAmb * kTamb / Tmax);
    int n = (int)std::ceil(dt / (dx * dx / (4.5 * alpha)));
    n = std::min(5, n % 2 ? n : n + 1);
    diffSub = n;
    diffU[0] = (float)(dt / n);
  }
  int npieces() const { int32_t n; std::memcpy(&n, &P[26], 4); return n; }

  // ---------------------------------------------------------------- dispatches
  static uint32_t cdiv(int a, int b) { return (uint32_t)((a + b - 1) / b); }
  void bind_base_advect() {
    using namespace wgsl_advect;
    bind("P", P); bind("U", U.data()); bind("V", V.data()); bind("Uh", Uh.data()); bind("Vh", Vh.data());
    bind("U2", U2.data()); bind("V2", V2.data()); bind("T", T.data()); bind("Y", Y.data()); bind("Th", Th.data());
    bind("Yh", Yh.data()); bind("T2", T2.data()); bind("Y2", Y2.data());
  }
  void diffuse(std::vector<float>& Tin, std::vector<float>& Yin, std::vector<float>& Tout, std::vector<float>& Yout) {
    using namespace wgsl_diffuse;
    bind("P", P); bind("D", diffU); bind("Tin", Tin.data()); bind("Yin", Yin.data()); bind("Tout", Tout.data());
    bind("Yout", Yout.data()); bind("fx", fx.data()); bind("fy", fy.data());
    dispatch_main_(cdiv(nx, 8), cdiv(ny, 8), 1);
  }
  void bind_pressure(Lv& L, Lv* C, int color) {
    using namespace wgsl_pressure;
    bind("P", P); bind("U", U.data()); bind("V", V.data()); bind("T", T.data()); bind("fx", fx.data());
    bind("fy", fy.data()); bind("SQ", SQ.data()); bind("p", L.p.data()); bind("rhs", L.rhs.data());
    bind("ax", L.ax.data()); bind("ay", L.ay.data()); bind("L", &L.u[color]);
    if (C) { bind("pc", C->p.data()); bind("rhsc", C->rhs.data()); bind("axc", C->ax.data()); bind("ayc", C->ay.data()); }
  }
  void stage(const std::string& st) {
    const uint32_t gFx = cdiv(nx + 1, 8), gFy = cdiv(ny + 1, 8), gCx = cdiv(nx, 8), gCy = cdiv(ny, 8);
    if (st == "advect") {
      bind_base_advect();
      wgsl_advect::dispatch_scalForward(gCx, gCy, 1);
      wgsl_advect::dispatch_scalCorrect(gCx, gCy, 1);
      wgsl_advect::dispatch_velForward(gFx, gFy, 1);
      wgsl_advect::dispatch_velCorrect(gFx, gFy, 1);
    } else if (st == "diffuse") {
      diffuse(T2, Y2, T, Y);
      for (int s = 1; s < diffSub; s += 2) { diffuse(T, Y, Th, Yh); diffuse(Th, Yh, T, Y); }
    } else if (st == "sources") {
      using namespace wgsl_sources;
      bind("P", P); bind("T", T.data()); bind("Y", Y.data()); bind("Tadv", T2.data()); bind("U", U.data());
      bind("V", V.data()); bind("cellG", cellG.data()); bind("pieces", pieces.data()); bind("SQ", SQ.data());
      bind("acc", acc.data()); bind("faceW", faceW.data());
      dispatch_main_(gCx, gCy, 1);
    } else if (st == "forces") {
      using namespace wgsl_forces;
      bind("P", P); bind("U2", U2.data()); bind("V2", V2.data()); bind("T", T.data()); bind("fx", fx.data());
      bind("fy", fy.data()); bind("U", U.data()); bind("V", V.data());
      dispatch_main_(gFx, gFy, 1);
    } else if (st == "coef_rhs") {
      bind_pressure(lv[0], nullptr, 0);
      wgsl_pressure::dispatch_coef(gFx, gFy, 1);
      wgsl_pressure::dispatch_rhs0(gCx, gCy, 1);
      for (size_t l = 0; l + 1 < lv.size(); l++) {
        bind_pressure(lv[l], &lv[l + 1], 0);
        wgsl_pressure::dispatch_coefRestrict(cdiv(lv[l].nx / 2 + 1, 8), cdiv(lv[l].ny / 2 + 1, 8), 1);
      }
    } else if (st == "pressure" || st == "vcycle") {
      vcycle();
    } else if (st == "project") {
      bind_pressure(lv[0], nullptr, 0);
      wgsl_pressure::dispatch_project(gFx, gFy, 1);
    } else throw std::runtime_error("unknown stage " + st);
  }
  void vcycle() {   // js/fluid.js:294-312, nu = 2
    const int NL = (int)lv.size();
    auto g = [&](const Lv& L, uint32_t& x, uint32_t& y) { x = cdiv(L.nx, 8); y = cdiv(L.ny, 8); };
    uint32_t x, y;
    for (int l = 0; l < NL - 1; l++) {
      g(lv[l], x, y);
      for (int s = 0; s < 2; s++) {
        bind_pressure(lv[l], &lv[l + 1], 0); wgsl_pressure::dispatch_relax(x, y, 1);
        bind_pressure(lv[l], &lv[l + 1], 1); wgsl_pressure::dispatch_relax(x, y, 1);
      }
      g(lv[l + 1], x, y);
      bind_pressure(lv[l], &lv[l + 1], 0); wgsl_pressure::dispatch_restrictRes(x, y, 1);
    }
    bind_pressure(lv[NL - 1], nullptr, 0); wgsl_pressure::dispatch_coarsest(1, 1, 1);
    for (int l = NL - 2; l >= 0; l--) {
      g(lv[l], x, y);
      bind_pressure(lv[l], &lv[l + 1], 0); wgsl_pressure::dispatch_prolong(x, y, 1);
      for (int s = 0; s < 2; s++) {
        bind_pressure(lv[l], &lv[l + 1], 1); wgsl_pressure::dispatch_relax(x, y, 1);
        bind_pressure(lv[l], &lv[l + 1], 0); wgsl_pressure::dispatch_relax(x, y, 1);
      }
    }
  }
  void step() {   // js/fluid.js:225-253
    for (const char* s : {"advect", "diffuse", "sources", "forces", "coef_rhs", "vcycle", "project"}) stage(s);
    time += dt;
  }
  void geometry() {
    using namespace wgsl_geometry;
    bind("P", P); bind("pieces", pieces.data()); bind("cellG", cellG.data()); bind("fx", fx.data());
    bind("fy", fy.data()); bind("faceW", faceW.data());
    dispatch_main_(cdiv(nx + 1, 8), cdiv(ny + 1, 8), 1);
  }
  void radiation() {
    using namespace wgsl_radiation;
    bind("P", P); bind("T", T.data()); bind("Y", Y.data()); bind("pieces", pieces.data()); bind("rad", rad.data());
    dispatch_main_((uint32_t)(npieces() * 4 + 64), 1, 1);
  }
  // Renderer.encode (js/render.js:57-70): the fragment stage at every pixel centre,
  // row 0 at the top (uv.y = 1 - (y + 0.5) / H)
  void render(const void* rp, const float* wood, int W, int H, float* out) {
    using namespace wgsl_render;
    std::vector<float> zero(64 * 12, 0.f);
    bind("P", P); bind("R", const_cast<void*>(rp)); bind("T", T.data()); bind("Y", Y.data()); bind("SQ", SQ.data());
    bind("pieces", pieces.data()); bind("U", U.data()); bind("V", V.data());
    bind("wood", const_cast<float*>(wood ? wood : zero.data())); bind("rad", rad.data());
    for (int y = 0; y < H; y++)
      for (int x = 0; x < W; x++) {
        VSOut in;
        in.pos = vec4f((float)x + 0.5f, (float)y + 0.5f, 0.f, 1.f);
        in.uv = vec2f(((float)x + 0.5f) / (float)W, 1.0f - ((float)y + 0.5f) / (float)H);
        const vec4f c = fs(in);
        float* o = out + ((size_t)y * W + x) * 4;
        o[0] = c.x; o[1] = c.y; o[2] = c.z; o[3] = c.w;
      }
  }
  std::vector<float>* field(const std::string& nm, int* lvl) {
    *lvl = -1;
    if (nm == "U") return &U; if (nm == "Uh") return &Uh; if (nm == "U2") return &U2;
    if (nm == "V") return &V; if (nm == "Vh") return &Vh; if (nm == "V2") return &V2;
    if (nm == "T") return &T; if (nm == "Th") return &Th; if (nm == "T2") return &T2;
    if (nm == "Y") return &Y; if (nm == "Yh") return &Yh; if (nm == "Y2") return &Y2;
    if (nm == "SQ") return &SQ; if (nm == "fx") return &fx; if (nm == "fy") return &fy;
    if (nm == "rad") return &rad;
    std::string b = nm; int l = 0;
    const size_t dot = nm.find('.');
    if (dot != std::string::npos) { b = nm.substr(0, dot); l = std::atoi(nm.c_str() + dot + 1); }
    if (l < 0 || l >= (int)lv.size()) return nullptr;
    *lvl = l;
    if (b == "p") return &lv[l].p; if (b == "rhs") return &lv[l].rhs; if (b == "ax") return &lv[l].ax; if (b == "ay") return &lv[l].ay;
    return nullptr;
  }
};

template <class F> int guard(F&& f) {
  try { return f(); } catch (const std::exception& e) { g_err = e.what(); return -22; }
}
RefSim* S(void* h) { return static_cast<RefSim*>(h); }
}  // namespace

extern "C" {
const char* wref_error() { return g_err.c_str(); }
void* wref_create(int nx, int ny, double width, double dt, int /*fp64*/) {
  try { return new RefSim(nx, ny, width, dt); } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}
int wref_destroy(void* h) { delete S(h); return 0; }
int wref_reset(void* h) { return guard([&] { S(h)->reset(); return 0; }); }
int wref_write_params(void* h) { return guard([&] { S(h)->write_params(); return 0; }); }
int wref_set_param(void* h, const char* name, double v) {
  const int i = param_index(name);
  if (i < 0) { g_err = std::string("unknown param ") + name; return -2; }
  if (i == 0 || i == 1 || i == 26) S(h)->seti(i, (int32_t)v);
  else if (i == 27) { uint32_t x = (uint32_t)v; std::memcpy(&S(h)->host[27], &x, 4); }
  else S(h)->setf(i, v);
  return 0;
}
int wref_set_frame(void* h, unsigned f) { S(h)->frame = f; return 0; }
int wref_upload_pieces(void* h, const float* data, int n) {
  S(h)->seti(26, n);
  std::memcpy(S(h)->pieces.data(), data, 64 * 20 * 4);
  return 0;
}
int wref_clear_geometry(void* h) { std::fill(S(h)->faceW.begin(), S(h)->faceW.end(), 0); return 0; }
int wref_geometry(void* h) { return guard([&] { S(h)->geometry(); return 0; }); }
int wref_radiation(void* h) { return guard([&] { S(h)->radiation(); return 0; }); }
int wref_render(void* h, const void* rp, const float* wood, int W, int H, float* out) {
  return guard([&] { S(h)->render(rp, wood, W, H, out); return 0; });
}
int wref_step(void* h, int n) { return guard([&] { for (int i = 0; i < n; i++) S(h)->step(); return 0; }); }
int wref_vcycle(void* h, int) { return guard([&] { S(h)->vcycle(); return 0; }); }
int wref_stage(void* h, const char* st) { return guard([&] { S(h)->stage(st); return 0; }); }
int wref_read_field(void* h, const char* name, double* out, size_t n) {
  RefSim* s = S(h);
  const std::string nm(name);
  if (nm == "cellG") {   // (sdf, id as an integer value)
    if (n != s->cellG.size()) { g_err = "bad size"; return -22; }
    for (size_t k = 0; k < n / 2; k++) {
      uint32_t id; std::memcpy(&id, &s->cellG[2 * k + 1], 4);
      out[2 * k] = s->cellG[2 * k]; out[2 * k + 1] = (double)id;
    }
    return 0;
  }
  int l; std::vector<float>* a = s->field(nm, &l);
  if (!a) { g_err = "unknown field " + nm; return -2; }
  if (n != a->size()) { g_err = "field " + nm + ": expected " + std::to_string(a->size()); return -22; }
  for (size_t k = 0; k < n; k++) out[k] = (*a)[k];
  return 0;
}
int wref_write_field(void* h, const char* name, const double* in, size_t n) {
  RefSim* s = S(h);
  int l; std::vector<float>* a = s->field(name, &l);
  if (!a) { g_err = std::string("unknown field ") + name; return -2; }
  if (n != a->size()) { g_err = "bad size"; return -22; }
  for (size_t k = 0; k < n; k++) (*a)[k] = (float)in[k];
  return 0;
}
int wref_readback(void* h, int32_t* acc, float* rad, int32_t* faceW) {
  RefSim* s = S(h);
  if (acc) std::memcpy(acc, s->acc.data(), 528 * 4);
  if (rad) std::memcpy(rad, s->rad.data(), 320 * 16);
  if (faceW) std::memcpy(faceW, s->faceW.data(), 256 * 4);
  std::fill(s->acc.begin(), s->acc.end(), 0);
  return 0;
}
int wref_info(void* h, double* o) {
  RefSim* s = S(h);
  for (int i = 0; i < 12; i++) o[i] = 0;
  o[0] = s->nx; o[1] = s->ny; o[2] = s->dx; o[3] = s->dt; o[4] = s->time; o[5] = s->frame; o[6] = s->diffSub;
  o[7] = (double)s->lv.size(); o[8] = 1; o[10] = s->dx * s->ny;
  return 0;
}
int wref_level_dims(void* h, int l, int* d) {
  RefSim* s = S(h);
  if (l < 0 || l >= (int)s->lv.size()) return -2;
  d[0] = s->lv[l].nx; d[1] = s->lv[l].ny; return 0;
}
}  // extern "C"
