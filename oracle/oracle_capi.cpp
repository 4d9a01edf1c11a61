// ORACLE — test infrastructure, not product code.
// extern "C" entry points over cforc::Sim<float> / Sim<double> for the Python
// test harness (ctypes). The surface mirrors the product C ABI
// (include/campfire_gas.h) so that tests drive both through one wrapper; fields
// cross the boundary as doubles in the dense row-major layouts of
// js/fluid.js:51-68.
#include "gas_ref.hpp"

#include <cstdio>
#include <memory>
#include <string>

using namespace cforc;

namespace {
thread_local std::string g_err;

// Param names in upload order (js/fluid.js:13-24)
const char* kParamNames[40] = {
  "nx", "ny", "dx", "dt", "Tamb", "rhoAmb", "YOamb", "grav", "cp", "Pr", "viscMult", "diffMult",
  "reactB", "reactTa", "dHc", "sO2", "sootFormA", "sootFormTa", "sootOxA", "sootOxTa",
  "kappaSootC", "kappaGas", "exchAlpha", "depth", "charA", "charTa", "nPieces", "frame",
  "heaterX0", "heaterX1", "heaterY1", "heaterT", "burnerX0", "burnerX1", "burnerFlux", "burnerT",
  "sootDensity", "sigma", "charO2", "time"};

int param_index(const char* name) {
  for (int i = 0; i < 40; i++) if (std::strcmp(kParamNames[i], name) == 0) return i;
  return -1;
}

struct ISim {
  virtual ~ISim() = default;
};

template <class R> struct Box : ISim {
  Sim<R> s;
};

template <class R> Sim<R>* as(void* h) { return &static_cast<Box<R>*>(static_cast<ISim*>(h))->s; }

struct Handle { int fp64; ISim* impl; };

// field access in the dense reference layouts; comps = components per element
template <class R> int field(Sim<R>& s, const std::string& nm, double* out, const double* in, size_t n) {
  auto scal = [&](std::vector<R>& a) -> int {
    if (n != a.size()) { g_err = "field " + nm + ": expected " + std::to_string(a.size()) + " values"; return -22; }
    for (size_t k = 0; k < n; k++) { if (out) out[k] = (double)a[k]; else a[k] = R(in[k]); }
    return 0;
  };
  auto vec4 = [&](std::vector<Vec4<R>>& a) -> int {
    if (n != a.size() * 4) { g_err = "field " + nm + ": expected " + std::to_string(a.size() * 4) + " values"; return -22; }
    for (size_t k = 0; k < a.size(); k++) {
      if (out) { out[4 * k] = a[k].x; out[4 * k + 1] = a[k].y; out[4 * k + 2] = a[k].z; out[4 * k + 3] = a[k].w; }
      else a[k] = Vec4<R>{R(in[4 * k]), R(in[4 * k + 1]), R(in[4 * k + 2]), R(in[4 * k + 3])};
    }
    return 0;
  };
  if (nm == "U") return scal(s.U); if (nm == "Uh") return scal(s.Uh); if (nm == "U2") return scal(s.U2);
  if (nm == "V") return scal(s.V); if (nm == "Vh") return scal(s.Vh); if (nm == "V2") return scal(s.V2);
  if (nm == "T") return scal(s.T); if (nm == "Th") return scal(s.Th); if (nm == "T2") return scal(s.T2);
  if (nm == "fx") return scal(s.fx); if (nm == "fy") return scal(s.fy);
  if (nm == "Y") return vec4(s.Y); if (nm == "Yh") return vec4(s.Yh); if (nm == "Y2") return vec4(s.Y2);
  if (nm == "SQ") {
    if (n != s.SQ.size() * 2) { g_err = "field SQ: bad size"; return -22; }
    for (size_t k = 0; k < s.SQ.size(); k++) {
      if (out) { out[2 * k] = s.SQ[k].x; out[2 * k + 1] = s.SQ[k].y; }
      else s.SQ[k] = Vec2<R>{R(in[2 * k]), R(in[2 * k + 1])};
    }
    return 0;
  }
  if (nm == "cellG") {   // (sdf, piece*4+face as an integer value; 4294967295 = none)
    if (n != s.gsdf.size() * 2) { g_err = "field cellG: bad size"; return -22; }
    for (size_t k = 0; k < s.gsdf.size(); k++) {
      if (out) { out[2 * k] = s.gsdf[k]; out[2 * k + 1] = (double)s.gid[k]; }
      else { s.gsdf[k] = R(in[2 * k]); s.gid[k] = (uint32_t)in[2 * k + 1]; }
    }
    return 0;
  }
  if (nm == "p64") {
    if (n != s.p64.size()) { g_err = "field p64: bad size"; return -22; }
    for (size_t k = 0; k < n; k++) { if (out) out[k] = s.p64[k]; else s.p64[k] = in[k]; }
    return 0;
  }
  // multigrid level fields: p, rhs, ax, ay (level 0) or p.L, rhs.L, ax.L, ay.L
  std::string base = nm; int l = 0;
  const size_t dot = nm.find('.');
  if (dot != std::string::npos) { base = nm.substr(0, dot); l = std::atoi(nm.c_str() + dot + 1); }
  if (l < 0 || l >= (int)s.lv.size()) { g_err = "no level in " + nm; return -2; }
  auto& L = s.lv[l];
  if (base == "p") return scal(L.p); if (base == "rhs") return scal(L.rhs);
  if (base == "ax") return scal(L.ax); if (base == "ay") return scal(L.ay);
  g_err = "unknown field " + nm;
  return -2;
}

template <class F> int guard(F&& f) {
  try { return f(); } catch (const std::exception& e) { g_err = e.what(); return -22; }
}
}  // namespace

#define DISPATCH(h, expr)                                                   \
  do {                                                                      \
    Handle* H_ = static_cast<Handle*>(h);                                   \
    if (!H_) { g_err = "null handle"; return -22; }                         \
    if (H_->fp64) { auto& s = *as<double>(H_->impl); return guard([&] { expr; }); } \
    else { auto& s = *as<float>(H_->impl); return guard([&] { expr; }); }   \
  } while (0)

extern "C" {

const char* orc_error() { return g_err.c_str(); }

void* orc_create(int nx, int ny, double width, double dt, int fp64) {
  try {
    Handle* h = new Handle{fp64 ? 1 : 0, nullptr};
    if (fp64) { auto* b = new Box<double>; b->s.create(nx, ny, width, dt); h->impl = b; }
    else { auto* b = new Box<float>; b->s.create(nx, ny, width, dt); h->impl = b; }
    return h;
  } catch (const std::exception& e) { g_err = e.what(); return nullptr; }
}

int orc_destroy(void* h) {
  Handle* H = static_cast<Handle*>(h);
  if (!H) return 0;
  delete H->impl; delete H; return 0;
}

int orc_reset(void* h) { DISPATCH(h, s.reset(); return 0); }
int orc_write_params(void* h) { DISPATCH(h, s.write_params(); return 0); }
int orc_set_param(void* h, const char* name, double v) {
  DISPATCH(h, {
    const int i = param_index(name);
    if (i < 0) { g_err = std::string("unknown param ") + name; return -2; }
    char* base = reinterpret_cast<char*>(&s.host) + 4 * i;
    if (i == 0 || i == 1 || i == 26) { int32_t x = (int32_t)v; std::memcpy(base, &x, 4); }
    else if (i == 27) { uint32_t x = (uint32_t)v; std::memcpy(base, &x, 4); }
    else { float x = (float)v; std::memcpy(base, &x, 4); }
    return 0;
  });
}
int orc_get_param(void* h, const char* name, double* v) {
  DISPATCH(h, {
    const int i = param_index(name);
    if (i < 0) { g_err = std::string("unknown param ") + name; return -2; }
    const char* base = reinterpret_cast<const char*>(&s.host) + 4 * i;
    if (i == 0 || i == 1 || i == 26) { int32_t x; std::memcpy(&x, base, 4); *v = x; }
    else if (i == 27) { uint32_t x; std::memcpy(&x, base, 4); *v = x; }
    else { float x; std::memcpy(&x, base, 4); *v = x; }
    return 0;
  });
}
int orc_set_dt(void* h, double dt) { DISPATCH(h, s.dtd = dt; s.dt_cap = dt; return 0); }
int orc_set_cfl(void* h, double cfl, double dt_cap) { DISPATCH(h, s.cfl = cfl; s.dt_cap = dt_cap; return 0); }
int orc_set_frame(void* h, unsigned frame) { DISPATCH(h, s.frame = frame; return 0); }
int orc_set_nray(void* h, int nray) {
  DISPATCH(h, {
    if (nray < 1 || nray > 1024 || (nray & (nray - 1))) { g_err = "nray must be a power of two in [1, 1024]"; return -22; }
    s.nray = nray; return 0;
  });
}
int orc_set_solver(void* h, int mode, int ncycles, double tol, int max_cycles) {
  DISPATCH(h, s.mode = mode; s.ncycles = ncycles; s.tol = tol; s.max_cycles = max_cycles; return 0);
}
int orc_set_coarse_solve(void* h, int direct) { DISPATCH(h, s.coarse_direct = direct; return 0); }
int orc_set_krylov(void* h, int on) { DISPATCH(h, s.krylov = on; return 0); }
int orc_set_coarse_w(void* h, int cells) { DISPATCH(h, s.w_cells = cells; return 0); }
int orc_upload_pieces(void* h, const float* data, int n) {
  DISPATCH(h, {
    if (n < 0 || n > MAX_PIECES) { g_err = "piece count out of range"; return -22; }
    s.upload_pieces(data, n); return 0;
  });
}
int orc_clear_geometry(void* h) { DISPATCH(h, s.clear_geometry(); return 0); }
int orc_geometry(void* h) { DISPATCH(h, s.geometry(); return 0); }
int orc_radiation(void* h) { DISPATCH(h, s.radiation(); return 0); }
int orc_step(void* h, int n) { DISPATCH(h, for (int i = 0; i < n; i++) s.step(); return 0); }
int orc_vcycle(void* h, int nu) { DISPATCH(h, s.vcycle(nu); return 0); }

// one stage of encodeStepProfiled (js/fluid.js:256-292) or a single reference dispatch
int orc_stage(void* h, const char* stage) {
  DISPATCH(h, {
    const std::string st(stage);
    if (st == "advect") s.stage_advect();
    else if (st == "scalForward") s.scalForward();
    else if (st == "scalCorrect") s.scalCorrect();
    else if (st == "velForward") s.velForward();
    else if (st == "velCorrect") s.velCorrect();
    else if (st == "diffuse") s.stage_diffuse();
    else if (st == "sources") s.sources();
    else if (st == "forces") s.forces();
    else if (st == "coef_rhs") s.stage_coef_rhs();
    else if (st == "pressure") s.pressure_solve();
    else if (st == "project") s.stage_project();
    else if (st == "update_dt") s.update_dt();
    else { g_err = "unknown stage " + st; return -2; }
    return 0;
  });
}

int orc_read_field(void* h, const char* name, double* out, size_t n) { DISPATCH(h, return field(s, name, out, nullptr, n)); }
int orc_write_field(void* h, const char* name, const double* in, size_t n) { DISPATCH(h, return field(s, name, nullptr, in, n)); }
int orc_readback(void* h, int32_t* acc, float* rad, int32_t* faceW) { DISPATCH(h, s.readback(acc, rad, faceW); return 0); }
int orc_budgets(void* h, double* out) { DISPATCH(h, s.budgets(out); return 0); }

// info: nx, ny, dx, dt, time, frame, diffSub, levels, last_cycles, last_rel, height, last_rel0, pressure rel residual now
int orc_info(void* h, double* o) {
  DISPATCH(h, {
    o[0] = s.nx; o[1] = s.ny; o[2] = s.dxd; o[3] = s.dtd; o[4] = s.time; o[5] = s.frame; o[6] = s.diffSub;
    o[7] = (double)s.lv.size(); o[8] = s.last_cycles; o[9] = s.last_rel; o[10] = s.dxd * s.ny; o[11] = s.last_rel0;
    return 0;
  });
}
int orc_level_dims(void* h, int l, int* dims) {
  DISPATCH(h, {
    if (l < 0 || l >= (int)s.lv.size()) return -2;
    dims[0] = s.lv[l].nx; dims[1] = s.lv[l].ny; return 0;
  });
}
int orc_pressure_residual(void* h, double* rel) {
  DISPATCH(h, { const double b = s.rhs_norm(); *rel = b > 0 ? s.res_norm() / b : 0.0; return 0; });
}

}  // extern "C"
