// extern "C" surface of libcampfire_gas.so (include/campfire_gas.h): thin
// wrappers over cfg::Engine that validate handles and translate exceptions and
// CUDA failures into status codes.
#include <algorithm>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/campfire_gas.h"
#include "engine.h"
#include "wood.h"

struct cfg_sim {
  cfg::Engine* eng;
  int scene;
  bool owner;     // a single-scene FluidSim owns its engine; batch views do not
};
struct cfg_batch {
  cfg::Engine* eng;
  std::vector<std::unique_ptr<cfg_sim>> views;
};

namespace {
template <class F> int guarded(F&& f) {
  try { return f(); }
  catch (const std::bad_alloc&) { return cfg::fail(CFG_ERR_NOMEM, "host allocation failed"); }
  catch (const std::exception& e) { return cfg::fail(CFG_ERR_INVAL, e.what()); }
}
#define SIM_OK(sim) do { if (!(sim) || !(sim)->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_sim handle"); } while (0)
#define OWNER_OK(sim) do { if (!(sim)->owner) return cfg::fail(CFG_ERR_INVAL, "this call steps a whole batch: use the cfg_batch_* entry point"); } while (0)
}  // namespace

extern "C" {

int cfg_version(void) { return 10000; }

int cfg_last_error(char* buf, size_t len) {
  const std::string& e = cfg::last_error();
  if (buf && len) { std::strncpy(buf, e.c_str(), len - 1); buf[len - 1] = 0; }
  return (int)e.size();
}

int cfg_default_params(cfg_params* out) {
  if (!out) return cfg::fail(CFG_ERR_INVAL, "null output");
  cfg::default_params(out);
  return CFG_OK;
}

int cfg_device_count(int* count) {
  if (!count) return cfg::fail(CFG_ERR_INVAL, "null output");
  int n = 0;
  const cudaError_t e = cudaGetDeviceCount(&n);
  *count = e == cudaSuccess ? n : 0;
  return CFG_OK;
}

int cfg_create(int nx, int ny, double width, double dt, int device, cfg_sim** out) {
  if (!out) return cfg::fail(CFG_ERR_INVAL, "null output");
  *out = nullptr;
  return guarded([&] {
    auto eng = std::make_unique<cfg::Engine>();
    CFG_TRY(eng->init(device, 1, &nx, &ny, &width, &dt));
    *out = new cfg_sim{eng.release(), 0, true};
    return CFG_OK;
  });
}

int cfg_destroy(cfg_sim* sim) {
  if (!sim) return CFG_OK;
  if (!sim->owner) return cfg::fail(CFG_ERR_INVAL, "batch views are released with cfg_batch_destroy");
  delete sim->eng;
  delete sim;
  return CFG_OK;
}

#define SCENE_CALL(sim, expr) SIM_OK(sim); return guarded([&] { return sim->eng->expr; })

int cfg_reset(cfg_sim* sim) { SCENE_CALL(sim, reset(sim->scene)); }
int cfg_set_param(cfg_sim* sim, const char* name, double v) { SCENE_CALL(sim, set_param(sim->scene, name, v)); }
int cfg_get_param(cfg_sim* sim, const char* name, double* v) { SCENE_CALL(sim, get_param(sim->scene, name, v)); }
int cfg_set_dt(cfg_sim* sim, double dt) { SCENE_CALL(sim, set_dt(sim->scene, dt)); }
int cfg_write_params(cfg_sim* sim) { SCENE_CALL(sim, write_params(sim->scene)); }
int cfg_upload_pieces(cfg_sim* sim, const float* data, int n) { SCENE_CALL(sim, upload_pieces(sim->scene, data, n)); }
int cfg_clear_geometry(cfg_sim* sim) { SCENE_CALL(sim, clear_geometry(sim->scene)); }
int cfg_geometry(cfg_sim* sim) { SCENE_CALL(sim, geometry(sim->scene)); }
int cfg_radiation(cfg_sim* sim) { SCENE_CALL(sim, radiation(sim->scene)); }
int cfg_set_frame(cfg_sim* sim, uint32_t frame) { SCENE_CALL(sim, set_frame(sim->scene, frame)); }
int cfg_readback(cfg_sim* sim, int32_t* acc, float* rad, int32_t* faceW) { SCENE_CALL(sim, readback(sim->scene, acc, rad, faceW)); }
int cfg_readback_begin(cfg_sim* sim, uint64_t tag, int* slot) { SCENE_CALL(sim, readback_begin(sim->scene, tag, slot)); }
int cfg_readback_poll(cfg_sim* sim, int32_t* acc, float* rad, int32_t* faceW, uint64_t* tag, int* ready) {
  SCENE_CALL(sim, readback_collect(sim->scene, false, acc, rad, faceW, tag, ready));
}
int cfg_readback_wait(cfg_sim* sim, int32_t* acc, float* rad, int32_t* faceW, uint64_t* tag) {
  int ready = 0;
  SCENE_CALL(sim, readback_collect(sim->scene, true, acc, rad, faceW, tag, &ready));
}
int cfg_render_defaults(cfg_sim* sim, cfg_render_params* rp) { SCENE_CALL(sim, render_defaults(sim->scene, rp)); }
int cfg_render(cfg_sim* sim, const cfg_render_params* rp, const float* wood, int width, int height, float* rgba) {
  SIM_OK(sim);
  if (!rp) return cfg::fail(CFG_ERR_INVAL, "rp is null");
  return guarded([&] { return sim->eng->render(sim->scene, *rp, wood, width, height, rgba); });
}
int cfg_render_device(cfg_sim* sim, const cfg_render_params* rp, const float* wood, int width, int height,
                      void* rgba_device) {
  SIM_OK(sim);
  if (!rp) return cfg::fail(CFG_ERR_INVAL, "rp is null");
  return guarded([&] { return sim->eng->render_device(sim->scene, *rp, wood, width, height, (float*)rgba_device); });
}
int cfg_field_size(cfg_sim* sim, const char* name, size_t* count) { SCENE_CALL(sim, field_size(sim->scene, name, count)); }
int cfg_read_field(cfg_sim* sim, const char* name, float* out, size_t count) { SCENE_CALL(sim, read_field(sim->scene, name, out, count)); }
int cfg_write_field(cfg_sim* sim, const char* name, const float* in, size_t count) { SCENE_CALL(sim, write_field(sim->scene, name, in, count)); }
int cfg_read_p64(cfg_sim* sim, double* out, size_t count) { SCENE_CALL(sim, read_p64(sim->scene, out, count)); }
int cfg_get_info(cfg_sim* sim, cfg_info* out) { SCENE_CALL(sim, info(sim->scene, out)); }
int cfg_set_cfl(cfg_sim* sim, double cfl, double dt_cap) { SCENE_CALL(sim, set_cfl(sim->scene, cfl, dt_cap)); }
int cfg_set_nray(cfg_sim* sim, int nray) { SCENE_CALL(sim, set_nray(sim->scene, nray)); }
int cfg_pressure_residual(cfg_sim* sim, double* rel) { SCENE_CALL(sim, pressure_residual(sim->scene, rel)); }
int cfg_budgets(cfg_sim* sim, double* out) { SCENE_CALL(sim, budgets(sim->scene, out)); }

int cfg_step(cfg_sim* sim, int nsteps) { SIM_OK(sim); OWNER_OK(sim); return guarded([&] { return sim->eng->step(nsteps); }); }
int cfg_step_profiled(cfg_sim* sim, float* ms) { SIM_OK(sim); OWNER_OK(sim); return guarded([&] { return sim->eng->step_profiled(ms); }); }
int cfg_run_stage(cfg_sim* sim, const char* stage) { SIM_OK(sim); OWNER_OK(sim); return guarded([&] { return sim->eng->run_stage(stage); }); }
int cfg_vcycle(cfg_sim* sim, int nu) { SIM_OK(sim); OWNER_OK(sim); return guarded([&] { return sim->eng->vcycle_once(nu); }); }
int cfg_set_solver(cfg_sim* sim, int mode, int ncycles, double tol, int max_cycles) {
  SIM_OK(sim); OWNER_OK(sim);
  return guarded([&] { return sim->eng->set_solver(mode, ncycles, tol, max_cycles); });
}
int cfg_set_stream(cfg_sim* sim, void* stream) { SIM_OK(sim); OWNER_OK(sim); return guarded([&] { return sim->eng->set_stream((cudaStream_t)stream); }); }
int cfg_synchronize(cfg_sim* sim) { SIM_OK(sim); return guarded([&] { return sim->eng->synchronize(); }); }
int cfg_set_graphs(cfg_sim* sim, int enable) { SIM_OK(sim); OWNER_OK(sim); return sim->eng->set_graphs(enable != 0); }
int cfg_launch_count(cfg_sim* sim, int* per_step) {
  SIM_OK(sim);
  if (!per_step) return cfg::fail(CFG_ERR_INVAL, "null output");
  *per_step = sim->eng->launches_per_step();
  return CFG_OK;
}

// ---- batches
int cfg_batch_create(int nscenes, const int* nx, const int* ny, const double* width, const double* dt, int device, cfg_batch** out) {
  if (!out || !nx || !ny || !width || !dt) return cfg::fail(CFG_ERR_INVAL, "null argument");
  *out = nullptr;
  return guarded([&] {
    auto eng = std::make_unique<cfg::Engine>();
    CFG_TRY(eng->init(device, nscenes, nx, ny, width, dt));
    auto b = std::make_unique<cfg_batch>();
    b->eng = eng.release();
    for (int s = 0; s < nscenes; s++) b->views.emplace_back(new cfg_sim{b->eng, s, false});
    *out = b.release();
    return CFG_OK;
  });
}
int cfg_batch_destroy(cfg_batch* b) {
  if (!b) return CFG_OK;
  delete b->eng;
  delete b;
  return CFG_OK;
}
#define BATCH_OK(b) do { if (!(b) || !(b)->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_batch handle"); } while (0)
int cfg_batch_scene(cfg_batch* b, int i, cfg_sim** view) {
  BATCH_OK(b);
  if (!view || i < 0 || i >= (int)b->views.size()) return cfg::fail(CFG_ERR_INVAL, "scene index out of range");
  *view = b->views[i].get();
  return CFG_OK;
}
int cfg_batch_set_solver(cfg_batch* b, int mode, int ncycles, double tol, int max_cycles) {
  BATCH_OK(b); return guarded([&] { return b->eng->set_solver(mode, ncycles, tol, max_cycles); });
}
int cfg_batch_set_active(cfg_batch* b, int i, int active) {
  BATCH_OK(b);
  if (i < 0 || i >= (int)b->views.size()) return cfg::fail(CFG_ERR_INVAL, "scene index out of range");
  return guarded([&] { return b->eng->set_active(i, active != 0); });
}
int cfg_batch_step(cfg_batch* b, int nsteps) { BATCH_OK(b); return guarded([&] { return b->eng->step(nsteps); }); }
int cfg_batch_set_stream(cfg_batch* b, void* stream) { BATCH_OK(b); return guarded([&] { return b->eng->set_stream((cudaStream_t)stream); }); }
int cfg_batch_synchronize(cfg_batch* b) { BATCH_OK(b); return guarded([&] { return b->eng->synchronize(); }); }
int cfg_batch_set_graphs(cfg_batch* b, int enable) {
  if (!b || !b->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_batch handle");
  return b->eng->set_graphs(enable != 0);
}
int cfg_batch_launch_count(cfg_batch* b, int* per_step) {
  BATCH_OK(b);
  if (!per_step) return cfg::fail(CFG_ERR_INVAL, "null output");
  *per_step = b->eng->launches_per_step();
  return CFG_OK;
}
int cfg_batch_write_params(cfg_batch* b) { BATCH_OK(b); return guarded([&] { return b->eng->write_params_all(); }); }
int cfg_batch_geometry(cfg_batch* b) { BATCH_OK(b); return guarded([&] { return b->eng->geometry_all(); }); }

}  // extern "C"

extern "C" int cfg_time_kernel(cfg_sim* sim, const char* kernel, int iters, double* mean_ms, double* bytes_per_launch,
                               double* launches_per_step) {
  SIM_OK(sim); OWNER_OK(sim);
  return guarded([&] { return sim->eng->time_kernel(kernel, iters, mean_ms, bytes_per_launch, launches_per_step); });
}

extern "C" int cfg_set_coarse_cells(cfg_sim* sim, int cells) {
  SIM_OK(sim); OWNER_OK(sim);
  return guarded([&] { return sim->eng->set_coarse_cells(cells); });
}
extern "C" int cfg_batch_set_coarse_cells(cfg_batch* b, int cells) {
  if (!b || !b->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_batch handle");
  return guarded([&] { return b->eng->set_coarse_cells(cells); });
}
extern "C" int cfg_set_coarse_w(cfg_sim* sim, int cells) {
  SIM_OK(sim); OWNER_OK(sim);
  return guarded([&] { return sim->eng->set_coarse_w(cells); });
}
extern "C" int cfg_batch_set_coarse_w(cfg_batch* b, int cells) {
  if (!b || !b->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_batch handle");
  return guarded([&] { return b->eng->set_coarse_w(cells); });
}
extern "C" int cfg_set_coarse_cluster(cfg_sim* sim, int cs) {
  SIM_OK(sim); OWNER_OK(sim);
  return guarded([&] { return sim->eng->set_coarse_cluster(cs); });
}
extern "C" int cfg_batch_set_coarse_cluster(cfg_batch* b, int cs) {
  if (!b || !b->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_batch handle");
  return guarded([&] { return b->eng->set_coarse_cluster(cs); });
}

int cfg::load_generated_scene(cfg::Engine& eng, int s, int kind, double width, uint64_t seed) {
  const int nx = eng.scene_nx(s), ny = eng.scene_ny(s);
  const size_t n = (size_t)nx * ny;
  std::vector<float> T(n), Y(4 * n), U((size_t)(nx + 1) * ny), V((size_t)nx * (ny + 1)),
      pieces((size_t)CFG_MAX_PIECES * CFG_PIECE_FLOATS);
  int np = 0;
  cfg_params P;
  double dt = 0;
  CFG_TRY(cfg_scene_generate(kind, nx, ny, width, seed, T.data(), Y.data(), U.data(), V.data(), pieces.data(), &np, &P,
                             &dt));
  for (const char* k : {"Tamb", "rhoAmb", "YOamb", "reactB", "reactTa", "dHc", "Pr", "exchAlpha", "depth"}) {
    float f;
    std::memcpy(&f, reinterpret_cast<const char*>(&P) + 4 * cfg::param_index(k), 4);
    CFG_TRY(eng.set_param(s, k, f));
  }
  CFG_TRY(eng.set_dt(s, dt));
  CFG_TRY(eng.set_frame(s, 0));
  // reset before writeParams so that a reused batch slot uploads time 0, as a fresh one does
  CFG_TRY(eng.reset(s));
  CFG_TRY(eng.upload_pieces(s, pieces.data(), np));
  CFG_TRY(eng.write_params(s));
  CFG_TRY(eng.write_field(s, "T", T.data(), T.size()));
  CFG_TRY(eng.write_field(s, "Y", Y.data(), Y.size()));
  CFG_TRY(eng.write_field(s, "U", U.data(), U.size()));
  CFG_TRY(eng.write_field(s, "V", V.data(), V.size()));
  CFG_TRY(eng.write_field(s, "T2", T.data(), T.size()));
  CFG_TRY(eng.write_field(s, "Y2", Y.data(), Y.size()));
  CFG_TRY(eng.clear_geometry(s));
  return eng.geometry(s);
}

extern "C" int cfg_autotune(int device, int nscenes, const int* nx, const int* ny, int coarse_direct, int iters,
                            int* best_cells, int* cand_cells, double* cand_ms, int* ncand) {
  if (nscenes < 1 || !nx || !ny || iters < 1 || !best_cells || !cand_cells || !cand_ms || !ncand || *ncand < 1)
    return cfg::fail(CFG_ERR_INVAL, "bad argument");
  return guarded([&] {
    std::vector<double> width(nscenes, 0.8), dt(nscenes, 0.002);
    cfg::Engine eng;
    CFG_TRY(eng.init(device, nscenes, nx, ny, width.data(), dt.data()));
    for (int s = 0; s < nscenes; s++) CFG_TRY(cfg::load_generated_scene(eng, s, 0, 0.8, 1234 + s));
    if (coarse_direct) {
      CFG_TRY(eng.set_solver(CFG_SOLVE_FP64, 1, 1e-6, 4));
      CFG_TRY(eng.set_coarse_solve(1));
    } else {
      CFG_TRY(eng.set_solver(CFG_SOLVE_FIXED, 1, 1e-6, 1));
    }
    CFG_TRY(eng.step(1));
    CFG_TRY(eng.synchronize());
    // candidate thresholds: the level sizes below level 0, largest first
    std::vector<int> cells;
    for (int s = 0; s < nscenes; s++) {
      cfg_info inf;
      CFG_TRY(eng.info(s, &inf));
      for (int l = 1; l < inf.levels; l++) cells.push_back(inf.level_nx[l] * inf.level_ny[l]);
    }
    std::sort(cells.begin(), cells.end(), [](int a, int b) { return a > b; });
    cells.erase(std::unique(cells.begin(), cells.end()), cells.end());
    int k = 0;
    double best = 1e300;
    *best_cells = 0;
    for (int c : cells) {
      if (k >= *ncand) break;
      if (eng.set_coarse_cells(c) != CFG_OK) continue;   // does not fit in shared memory
      double ms = 0, bytes = 0, per = 0;
      CFG_TRY(eng.time_kernel("vcycle", iters, &ms, &bytes, &per));
      cand_cells[k] = c; cand_ms[k] = ms; k++;
      if (ms < best) { best = ms; *best_cells = c; }
    }
    *ncand = k;
    if (k == 0) return cfg::fail(CFG_ERR_RANGE, "no smoother schedule fits these sizes");
    return CFG_OK;
  });
}

extern "C" int cfg_set_tiles(cfg_sim* sim, int advect, int diffuse_sources, int forces) {
  SIM_OK(sim); OWNER_OK(sim);
  return guarded([&] { return sim->eng->set_tiles(advect, diffuse_sources, forces); });
}
extern "C" int cfg_batch_set_tiles(cfg_batch* b, int advect, int diffuse_sources, int forces) {
  if (!b || !b->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_batch handle");
  return guarded([&] { return b->eng->set_tiles(advect, diffuse_sources, forces); });
}
extern "C" int cfg_autotune_tiles(int device, int nscenes, const int* nx, const int* ny, int iters, int* best,
                                  double* ms) {
  if (nscenes < 1 || !nx || !ny || iters < 1 || !best) return cfg::fail(CFG_ERR_INVAL, "bad argument");
  return guarded([&] {
    std::vector<double> width(nscenes, 0.8), dt(nscenes, 0.002);
    cfg::Engine eng;
    CFG_TRY(eng.init(device, nscenes, nx, ny, width.data(), dt.data()));
    for (int s = 0; s < nscenes; s++) CFG_TRY(cfg::load_generated_scene(eng, s, 0, 0.8, 1234 + s));
    CFG_TRY(eng.set_solver(CFG_SOLVE_FP64, 1, 1e-6, 4));
    CFG_TRY(eng.step(1));
    CFG_TRY(eng.synchronize());
    return eng.autotune_tiles(iters, best, ms);
  });
}

extern "C" int cfg_set_coarse_solve(cfg_sim* sim, int direct) {
  SIM_OK(sim); OWNER_OK(sim);
  return guarded([&] { return sim->eng->set_coarse_solve(direct); });
}
extern "C" int cfg_batch_set_coarse_solve(cfg_batch* b, int direct) {
  if (!b || !b->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_batch handle");
  return guarded([&] { return b->eng->set_coarse_solve(direct); });
}

extern "C" int cfg_checkpoint_save(cfg_sim* sim, const char* path) {
  SIM_OK(sim);
  return guarded([&] { return sim->eng->checkpoint_save(sim->scene, path); });
}
extern "C" int cfg_checkpoint_load(cfg_sim* sim, const char* path) {
  SIM_OK(sim);
  return guarded([&] { return sim->eng->checkpoint_load(sim->scene, path); });
}

extern "C" int cfg_set_krylov(cfg_sim* sim, int on) {
  SIM_OK(sim); OWNER_OK(sim);
  return guarded([&] { return sim->eng->set_krylov(on); });
}
extern "C" int cfg_batch_set_krylov(cfg_batch* b, int on) {
  if (!b || !b->eng) return cfg::fail(CFG_ERR_INVAL, "null cfg_batch handle");
  return guarded([&] { return b->eng->set_krylov(on); });
}
extern "C" int cfg_krylov_folded(cfg_sim* sim, int* folded) {
  SIM_OK(sim);
  if (!folded) return cfg::fail(CFG_ERR_INVAL, "null output");
  *folded = sim->eng->krylov_folded() ? 1 : 0;
  return CFG_OK;
}
extern "C" int cfg_batch_krylov_folded(cfg_batch* b, int* folded) {
  if (!b || !b->eng || !folded) return cfg::fail(CFG_ERR_INVAL, "null argument");
  *folded = b->eng->krylov_folded() ? 1 : 0;
  return CFG_OK;
}

// ------------------------------------------------------------------ wood
struct cfg_rigid {
  cfg::RigidWorld* world;                   // owned (cfg_rigid_create) or a wood scene's (cfg_wood_rigid)
  std::unique_ptr<cfg::RigidWorld> own;
};
struct cfg_wood {
  cfg::Engine* eng;
  std::unique_ptr<cfg::WoodScene> scene;
  cfg_rigid view{nullptr, nullptr};
};

namespace {
void to_c(const cfg::RigidParams& r, cfg_rigid_params* o) {
  o->gravity[0] = r.gx; o->gravity[1] = r.gy; o->width = r.width; o->dt = r.dt;
  o->substeps = r.substeps; o->pad = 0;
  o->slop = r.slop; o->contact_hertz = r.contactHertz; o->contact_damping = r.contactDamping;
  o->max_pushout = r.maxPushout; o->mu_static = r.muStatic; o->mu_kinetic = r.muKinetic;
  o->stick_speed = r.stickSpeed; o->max_speed = r.maxSpeed; o->drag_hertz = r.dragHertz;
  o->drag_strength = r.dragStrength;
}
int from_c(const cfg_rigid_params* o, cfg::RigidParams* r) {
  if (!(o->dt > 0) || o->substeps < 1 || o->substeps > 64 || !(o->width > 0))
    return cfg::fail(CFG_ERR_INVAL, "rigid world: dt and width must be > 0, substeps in [1, 64]");
  r->gx = o->gravity[0]; r->gy = o->gravity[1]; r->width = o->width; r->dt = o->dt; r->substeps = o->substeps;
  r->slop = o->slop; r->contactHertz = o->contact_hertz; r->contactDamping = o->contact_damping;
  r->maxPushout = o->max_pushout; r->muStatic = o->mu_static; r->muKinetic = o->mu_kinetic;
  r->stickSpeed = o->stick_speed; r->maxSpeed = o->max_speed; r->dragHertz = o->drag_hertz;
  r->dragStrength = o->drag_strength;
  return CFG_OK;
}
void to_c(const cfg::WoodPiece& w, cfg_wood_piece* o) {
  o->side = w.side; o->rhoV = w.rhoV; o->rhoC = w.rhoC; o->mv = w.mv; o->mc = w.mc; o->Tc = w.Tc; o->gasRate = w.gasRate;
  for (int f = 0; f < 4; f++) {
    o->Ts[f] = w.Ts[f]; o->Tp[f] = w.Tp[f]; o->d[f] = w.d[f]; o->mflux[f] = w.mflux[f];
    o->charCov[f] = w.charCov[f]; o->exposure[f] = w.exposure[f];
  }
  o->dead = w.dead ? 1 : 0;
  o->pad = 0;
}
cfg::WoodPiece from_c(const cfg_wood_piece* o) {
  cfg::WoodPiece w;
  w.side = o->side; w.rhoV = o->rhoV; w.rhoC = o->rhoC; w.mv = o->mv; w.mc = o->mc; w.Tc = o->Tc; w.gasRate = o->gasRate;
  for (int f = 0; f < 4; f++) {
    w.Ts[f] = o->Ts[f]; w.Tp[f] = o->Tp[f]; w.d[f] = o->d[f]; w.mflux[f] = o->mflux[f];
    w.charCov[f] = o->charCov[f]; w.exposure[f] = o->exposure[f];
  }
  w.dead = o->dead != 0;
  return w;
}
std::array<double, 4> a4(const double* p) { return {p[0], p[1], p[2], p[3]}; }
}  // namespace

extern "C" {
int cfg_wood_piece_init(cfg_wood_piece* w, double side, double density, double T0) {
  if (!w || !(side > 0) || !(density > 0) || !(T0 > 0)) return cfg::fail(CFG_ERR_INVAL, "bad wood piece arguments");
  to_c(cfg::WoodPiece(side, density, T0), w);
  return CFG_OK;
}
int cfg_wood_piece_preheat(cfg_wood_piece* w, double Tsurf, double char_depth, double Tcore, double char_yield) {
  if (!w) return cfg::fail(CFG_ERR_INVAL, "null piece");
  cfg::WoodPiece p = from_c(w);
  p.preheat(Tsurf, char_depth, Tcore, char_yield);
  to_c(p, w);
  return CFG_OK;
}
int cfg_wood_piece_step(cfg_wood_piece* w, double dt, const double* qConv4, const double* qInc4,
                        const double* charBurnt4, double char_yield, double pyro_mult) {
  if (!w || !qConv4 || !qInc4 || !charBurnt4 || !(dt > 0)) return cfg::fail(CFG_ERR_INVAL, "bad wood step arguments");
  cfg::WoodPiece p = from_c(w);
  cfg::WoodCtl ctl;
  ctl.charYield = char_yield;
  ctl.pyroMult = pyro_mult;
  p.step(dt, a4(qConv4), a4(qInc4), a4(charBurnt4), ctl);
  to_c(p, w);
  return CFG_OK;
}
int cfg_wood_create(cfg_sim* sim, double char_yield, double pyro_mult, cfg_wood** out) {
  SIM_OK(sim); OWNER_OK(sim);
  if (!out) return cfg::fail(CFG_ERR_INVAL, "null output");
  return guarded([&] {
    cfg::WoodCtl ctl;
    ctl.charYield = char_yield;
    ctl.pyroMult = pyro_mult;
    auto* w = new cfg_wood{sim->eng, std::make_unique<cfg::WoodScene>(sim->eng, sim->scene, ctl)};
    *out = w;
    return CFG_OK;
  });
}
int cfg_wood_destroy(cfg_wood* w) {
  // readbacks still on the ring are collected first, so the scene's ring is free again
  const int rc = (w && w->scene) ? guarded([&] { return w->scene->set_readback_lag(0); }) : CFG_OK;
  delete w;
  return rc;
}
int cfg_wood_set_readback_lag(cfg_wood* w, int lag) {
  if (!w) return cfg::fail(CFG_ERR_INVAL, "null argument");
  return guarded([&] { return w->scene->set_readback_lag(lag); });
}
int cfg_wood_readbacks(cfg_wood* w, uint64_t* applied, uint64_t* skipped) {
  if (!w) return cfg::fail(CFG_ERR_INVAL, "null argument");
  if (applied) *applied = w->scene->applied;
  if (skipped) *skipped = w->scene->skipped;
  return CFG_OK;
}
int cfg_wood_add(cfg_wood* w, double x, double y, double angle, double side, double density, const double* preheat3,
                 const double* face_T4, int* slot) {
  if (!w || !slot) return cfg::fail(CFG_ERR_INVAL, "null argument");
  return guarded([&] {
    const int s = w->scene->add(x, y, angle, side, density, preheat3, face_T4);
    if (s < 0) return s;
    *slot = s;
    return CFG_OK;
  });
}
int cfg_wood_remove(cfg_wood* w, int slot) {
  if (!w) return cfg::fail(CFG_ERR_INVAL, "null argument");
  return guarded([&] { return w->scene->remove(slot); });
}
int cfg_wood_frame(cfg_wood* w, double sim_dt, int* nsteps) {
  if (!w) return cfg::fail(CFG_ERR_INVAL, "null argument");
  return guarded([&] { return w->scene->frame(sim_dt, nsteps); });
}
int cfg_wood_get(cfg_wood* w, int slot, cfg_wood_piece* out, double* qConv4, double* qInc4) {
  if (!w || !out) return cfg::fail(CFG_ERR_INVAL, "null argument");
  const cfg::WoodSlot* p = w->scene->slot(slot);
  if (!p) return cfg::fail(CFG_ERR_NOENT, "no piece in this slot");
  to_c(p->wood, out);
  if (qConv4) for (int f = 0; f < 4; f++) qConv4[f] = p->qConv[f];
  if (qInc4) for (int f = 0; f < 4; f++) qInc4[f] = p->qInc[f];
  return CFG_OK;
}
int cfg_wood_set_rigid(cfg_wood* w, const cfg_rigid_params* p) {
  if (!w) return cfg::fail(CFG_ERR_INVAL, "null argument");
  if (!p) return w->scene->set_rigid(nullptr);
  cfg::RigidParams rp;
  CFG_TRY(from_c(p, &rp));
  return w->scene->set_rigid(&rp);
}
int cfg_wood_rigid(cfg_wood* w, cfg_rigid** world) {
  if (!w || !world) return cfg::fail(CFG_ERR_INVAL, "null argument");
  if (!w->scene->world()) return cfg::fail(CFG_ERR_NOENT, "the pieces of this scene are frozen (no rigid world)");
  w->view.world = w->scene->world();
  *world = &w->view;
  return CFG_OK;
}
int cfg_wood_body(cfg_wood* w, int slot, int* body_id) {
  if (!w || !body_id) return cfg::fail(CFG_ERR_INVAL, "null argument");
  const cfg::WoodSlot* p = w->scene->slot(slot);
  if (!p) return cfg::fail(CFG_ERR_NOENT, "no piece in this slot");
  *body_id = p->body;
  return CFG_OK;
}
int cfg_wood_set(cfg_wood* w, int slot, const cfg_wood_piece* state) {
  if (!w || !state) return cfg::fail(CFG_ERR_INVAL, "null argument");
  return w->scene->set(slot, from_c(state));
}
int cfg_wood_render_data(cfg_wood* w, float* wood) {
  if (!w || !wood) return cfg::fail(CFG_ERR_INVAL, "null argument");
  const auto& r = w->scene->render_wood();
  std::copy(r.begin(), r.end(), wood);
  return CFG_OK;
}
int cfg_wood_stats(cfg_wood* w, double* hrr, double* rad, double* tmax) {
  if (!w) return cfg::fail(CFG_ERR_INVAL, "null argument");
  if (hrr) *hrr = w->scene->hrr;
  if (rad) *rad = w->scene->rad;
  if (tmax) *tmax = w->scene->tmax;
  return CFG_OK;
}

// ------------------------------------------------------------------ rigid bodies (js/rigid.js)
#define RIGID_OK(w) do { if (!(w) || !(w)->world) return cfg::fail(CFG_ERR_INVAL, "null cfg_rigid handle"); } while (0)
int cfg_rigid_defaults(cfg_rigid_params* p) {
  if (!p) return cfg::fail(CFG_ERR_INVAL, "null argument");
  to_c(cfg::RigidParams{}, p);
  return CFG_OK;
}
int cfg_rigid_create(const cfg_rigid_params* p, cfg_rigid** out) {
  if (!out) return cfg::fail(CFG_ERR_INVAL, "null output");
  cfg::RigidParams rp;
  if (p) CFG_TRY(from_c(p, &rp));
  return guarded([&] {
    auto* r = new cfg_rigid{nullptr, std::make_unique<cfg::RigidWorld>(rp)};
    r->world = r->own.get();
    *out = r;
    return CFG_OK;
  });
}
int cfg_rigid_destroy(cfg_rigid* w) {
  if (!w) return CFG_OK;
  if (!w->own) return cfg::fail(CFG_ERR_INVAL, "a wood scene's rigid world is destroyed with the scene");
  delete w;
  return CFG_OK;
}
int cfg_rigid_get_params(cfg_rigid* w, cfg_rigid_params* p) {
  RIGID_OK(w);
  if (!p) return cfg::fail(CFG_ERR_INVAL, "null argument");
  to_c(w->world->p, p);
  return CFG_OK;
}
int cfg_rigid_set_params(cfg_rigid* w, const cfg_rigid_params* p) {
  RIGID_OK(w);
  if (!p) return cfg::fail(CFG_ERR_INVAL, "null argument");
  return from_c(p, &w->world->p);
}
int cfg_rigid_add(cfg_rigid* w, double x, double y, double half, double density, double angle, int* id) {
  RIGID_OK(w);
  if (!(half > 0) || !(density > 0)) return cfg::fail(CFG_ERR_INVAL, "half side and density must be positive");
  return guarded([&] {
    cfg::Body* b = w->world->add(x, y, half, density, angle);
    if (id) *id = b->id;
    return CFG_OK;
  });
}
int cfg_rigid_remove(cfg_rigid* w, int id) {
  RIGID_OK(w);
  if (w->world->remove(id) != CFG_OK) return cfg::fail(CFG_ERR_NOENT, "no body with this id");
  return CFG_OK;
}
static cfg::Body* rigid_body(cfg_rigid* w, int id) { return w->world->find(id); }
int cfg_rigid_resize(cfg_rigid* w, int id, double half) {
  RIGID_OK(w);
  cfg::Body* b = rigid_body(w, id);
  if (!b) return cfg::fail(CFG_ERR_NOENT, "no body with this id");
  if (!(half > 0)) return cfg::fail(CFG_ERR_INVAL, "half side must be positive");
  w->world->resize(b, half);
  return CFG_OK;
}
int cfg_rigid_set_density(cfg_rigid* w, int id, double density) {
  RIGID_OK(w);
  cfg::Body* b = rigid_body(w, id);
  if (!b) return cfg::fail(CFG_ERR_NOENT, "no body with this id");
  if (!(density > 0)) return cfg::fail(CFG_ERR_INVAL, "density must be positive");
  b->density = density;
  return CFG_OK;
}
int cfg_rigid_step(cfg_rigid* w, double dt, int nsteps) {
  RIGID_OK(w);
  if (!(dt > 0) || nsteps < 0) return cfg::fail(CFG_ERR_INVAL, "dt must be > 0 and nsteps >= 0");
  return guarded([&] { for (int i = 0; i < nsteps; i++) w->world->step(dt); return CFG_OK; });
}
int cfg_rigid_advance(cfg_rigid* w, double dt) {
  RIGID_OK(w);
  if (!(dt >= 0)) return cfg::fail(CFG_ERR_INVAL, "dt must be >= 0");
  return guarded([&] { w->world->advance(dt); return CFG_OK; });
}
static void body_to_c(const cfg::Body& b, cfg_rigid_body* o) {
  o->id = b.id; o->dragging = b.dragging ? 1 : 0;
  o->x = b.x; o->y = b.y; o->a = b.a; o->vx = b.vx; o->vy = b.vy; o->w = b.w;
  o->half = b.half; o->density = b.density; o->mass = b.mass;
}
int cfg_rigid_bodies(cfg_rigid* w, cfg_rigid_body* out, int capacity, int* count) {
  RIGID_OK(w);
  if (!count || (capacity > 0 && !out)) return cfg::fail(CFG_ERR_INVAL, "null argument");
  const auto& bs = w->world->bodies();
  *count = (int)bs.size();
  for (int i = 0; i < capacity && i < (int)bs.size(); i++) body_to_c(*bs[i], &out[i]);
  return CFG_OK;
}
int cfg_rigid_get(cfg_rigid* w, int id, cfg_rigid_body* out) {
  RIGID_OK(w);
  if (!out) return cfg::fail(CFG_ERR_INVAL, "null argument");
  const cfg::Body* b = rigid_body(w, id);
  if (!b) return cfg::fail(CFG_ERR_NOENT, "no body with this id");
  body_to_c(*b, out);
  return CFG_OK;
}
int cfg_rigid_pick(cfg_rigid* w, double x, double y, int* id, double* lx, double* ly) {
  RIGID_OK(w);
  if (!id) return cfg::fail(CFG_ERR_INVAL, "null argument");
  const cfg::Body* b = w->world->pick(x, y, lx, ly);
  *id = b ? b->id : 0;
  return CFG_OK;
}
int cfg_rigid_drag_start(cfg_rigid* w, int id, double lx, double ly, double tx, double ty) {
  RIGID_OK(w);
  cfg::Body* b = rigid_body(w, id);
  if (!b) return cfg::fail(CFG_ERR_NOENT, "no body with this id");
  w->world->start_drag(b, lx, ly, tx, ty);
  return CFG_OK;
}
int cfg_rigid_drag_move(cfg_rigid* w, int id, double tx, double ty) {
  RIGID_OK(w);
  cfg::Body* b = rigid_body(w, id);
  if (!b) return cfg::fail(CFG_ERR_NOENT, "no body with this id");
  w->world->move_drag(b, tx, ty);
  return CFG_OK;
}
int cfg_rigid_drag_end(cfg_rigid* w, int id) {
  RIGID_OK(w);
  cfg::Body* b = rigid_body(w, id);
  if (!b) return cfg::fail(CFG_ERR_NOENT, "no body with this id");
  w->world->end_drag(b);
  return CFG_OK;
}
int cfg_rigid_max_penetration(cfg_rigid* w, double* pen) {
  RIGID_OK(w);
  if (!pen) return cfg::fail(CFG_ERR_INVAL, "null argument");
  *pen = w->world->max_penetration();
  return CFG_OK;
}
int cfg_rigid_contacts(cfg_rigid* w, int* manifolds, int* points) {
  RIGID_OK(w);
  int np = 0;
  for (const auto& m : w->world->manifolds()) np += m.npts;
  if (manifolds) *manifolds = (int)w->world->manifolds().size();
  if (points) *points = np;
  return CFG_OK;
}
}  // extern "C"
