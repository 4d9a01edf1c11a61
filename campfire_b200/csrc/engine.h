// Host side of the B200 gas step: the FluidSim state of each scene, the batch
// engine that owns device memory, work lists, streams and the CUDA graph of one
// step, and the status/error plumbing of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <string>
#include <vector>

#include "gas_dev.cuh"
#include "kernels.h"

namespace cfg {

void set_error(const std::string& msg);
const std::string& last_error();

// Status helper: CFG_OK or a negative CFG_ERR_*, with the message recorded.
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define CFG_CUDA(call)                                             \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return ::cfg::cuda_fail(e_, #call);     \
  } while (0)
#define CFG_TRY(call)                 \
  do {                                \
    int rc_ = (call);                 \
    if (rc_ != CFG_OK) return rc_;    \
  } while (0)

// js/config.js:12-47 constants used on the host
struct PhysConst {
  static constexpr double Tamb = 293.15, p0 = 101325, Wmix = 0.0289, R = 8.314462, Pr = 0.7;
  static double rhoAmb() { return p0 * Wmix / (R * Tamb); }
};

void default_params(cfg_params* p);
int param_index(const char* name);   // -1 if unknown

class Engine;
// A seeded synthetic scene (cfg_scene_generate) loaded into scene s of an engine in
// FluidSim's set-up order (params, pieces, writeParams, reset, fields, geometry),
// with the scene's own dt; frame 0.
int load_generated_scene(Engine& eng, int s, int kind, double width, uint64_t seed);

// One scene: FluidSim's host fields (js/fluid.js:27-47) and its device arrays.
struct Scene {
  int nx = 0, ny = 0, nlev = 0;
  double width = 0, dxd = 0, dtd = 0, time = 0;
  uint32_t frame = 0;
  double cfl = 0, dt_cap = 0;
  int nray = 64;
  cfg_params host{};             // FluidSim.params (applied by write_params)
  cfg_params P{};                // the uploaded uniform
  float pieces[MAX_PIECES * PIECE_FLOATS] = {};
  int diff_sub = 1;
  float diff_dt = 0;
  double alpha = 0;              // alpha(2200 K) of the diffusion sub-step rule
  int lnx[MAX_LEVELS] = {}, lny[MAX_LEVELS] = {};
  int lc = 0;                    // first level of the one-CTA coarse block
  int lw = MAX_LEVELS;           // nlev - 3 with the W tail, else MAX_LEVELS
  // the dx and diffusion alpha last copied to the device (write_params copies them only when
  // they change; nothing on the device writes them)
  double up_dxd = -1.0, up_alpha = -1.0;
  void* arena = nullptr;
  size_t arena_bytes = 0;
  SceneDesc desc{};              // host mirror of the device descriptor
  bool enabled = true;
  // CFL step: a step has set this scene's dt on the device since the host last set it
  // (reset, set_dt, set_cfl, checkpoint load): write_params then leaves dt to the device
  bool dt_on_device = false;
  // the arena's arrays in allocation order; `state`: part of a checkpoint (not the
  // tensor maps, which hold this arena's addresses, nor per-step scratch)
  struct Item { void* ptr; size_t bytes; bool state; };
  std::vector<Item> items;
  // The asynchronous readback ring (js/fluid.js:315-342): three pinned staging slots of
  // acc, rad and faceW, each filled by copies on the stream and completed by its event,
  // handed out oldest first. Allocated on the first cfg_readback_begin.
  struct Ring {
    char* host = nullptr;              // kRingSlots x kRingBytes, pinned and mapped
    char* dev = nullptr;               // the same memory in the device's address space
    cudaEvent_t ev[3] = {};
    uint64_t tag[3] = {}, seq[3] = {};
    bool busy[3] = {};                 // copies enqueued, not yet handed out (stageBusy)
    int idx = 0;                       // the next slot to fill (stageIdx)
    uint64_t next = 0;                 // sequence number of the next fill
  } ring;
};

constexpr int kRingSlots = 3;
// One readback is one copy: acc, rad and faceW sit next to each other in the scene arena (each
// array's start rounded up to 256 bytes), and a ring slot mirrors that layout.
constexpr size_t kRbRadOff = (ACC_LEN * 4 + 255) / 256 * 256;
constexpr size_t kRbFaceWOff = kRbRadOff + (RAD_LEN * 16 + 255) / 256 * 256;
constexpr size_t kRingBytes = kRbFaceWOff + MAX_PIECES * 16;

// Bytes of SceneDesc that cfg_write_params uploads: the uniform and the step
// controls up to (not including) the tile counts and device pointers.
constexpr size_t kDescParamBytes = offsetof(SceneDesc, nt_fr);

// Work lists: per-kernel tiles of every scene. MGV/MGC: single-pass multigrid
// tiles of level l / l+1 for scenes where l is not the coarsest level; MGD:
// fused smoother tiles of level l for scenes where l is below the coarse block.
enum WL { WL_ADV = 0, WL_DS, WL_FR, WL_PR, WL_GEO, WL_MG0, WL_MGV0, WL_MGC0 = WL_MGV0 + MAX_LEVELS,
          WL_MGD0 = WL_MGC0 + MAX_LEVELS, WL_COUNT = WL_MGD0 + MAX_LEVELS };

class Engine {
 public:
  ~Engine();
  int init(int device, int nscenes, const int* nx, const int* ny, const double* width, const double* dt);

  // per-scene FluidSim surface
  int reset(int s);
  int set_param(int s, const char* name, double v);
  int get_param(int s, const char* name, double* v);
  int set_dt(int s, double dt);
  int write_params(int s);
  int upload_pieces(int s, const float* data, int n);
  int clear_geometry(int s);
  int geometry(int s);
  int radiation(int s);
  int set_frame(int s, uint32_t f);
  int set_cfl(int s, double cfl, double dt_cap);
  int set_nray(int s, int nray);
  int readback(int s, int32_t* acc, float* rad, int32_t* faceW);
  // encodeReadback + afterSubmit (js/fluid.js:315-342): CFG_ERR_BUSY when the next slot is still pending
  int readback_begin(int s, uint64_t tag, int* slot);
  // the oldest pending slot: *ready = 1 and its data once its copies have completed (wait: block for them)
  int readback_collect(int s, bool wait, int32_t* acc, float* rad, int32_t* faceW, uint64_t* tag, int* ready);
  // render.wgsl's fragment stage into a host RGBA float image (wood: MAX_PIECES x 12 floats or null)
  int render(int s, const cfg_render_params& rp, const float* wood, int width, int height, float* rgba);
  int render_defaults(int s, cfg_render_params* rp);
  int render_device(int s, const cfg_render_params& rp, const float* wood, int width, int height, float* rgba_dev);
  int field_size(int s, const char* name, size_t* count);
  int read_field(int s, const char* name, float* out, size_t count);
  int write_field(int s, const char* name, const float* in, size_t count);
  int read_p64(int s, double* out, size_t count);
  int info(int s, cfg_info* out);
  int pressure_residual(int s, double* rel);
  int budgets(int s, double* out);
  int set_active(int s, bool on);
  // the scene's state to / from a file (same grid size on load)
  int checkpoint_save(int s, const char* path);
  int checkpoint_load(int s, const char* path);

  // whole-batch operations
  int set_solver(int mode, int ncycles, double tol, int max_cycles);
  int step(int nsteps);
  int step_profiled(float* stage_ms);
  int run_stage(const char* stage);
  int vcycle_once(int nu);
  int set_stream(cudaStream_t s);
  int synchronize();
  int set_graphs(bool on) { use_graphs_ = on; graph_dirty_ = true; return CFG_OK; }
  int launches_per_step() const { return launches_per_step_; }
  int write_params_all();
  int geometry_all();
  int time_kernel(const char* name, int iters, double* ms, double* bytes, double* per_step);
  // smoother schedule: the one-CTA coarse block starts at the first level with at
  // most `cells` cells (levels above it run as tiled down/up kernels)
  int set_coarse_cells(int cells);
  int coarse_cells() const { return coarse_cells_; }
  // cycle shape of the pressure loop: with cells > 0, the level two above the coarsest visits
  // its coarser level twice per cycle (the W tail) when it has at most `cells` cells; that
  // level always runs inside the one-CTA coarse block
  int set_coarse_w(int cells);
  int coarse_w() const { return w_cells_; }
  bool any_wtail() const;       // some scene's coarse block runs the W tail
  bool any_block_level0() const;   // some scene's coarse block covers level 0
  bool krylov_folded() const { return pcg_fused(); }   // the loop folds the Krylov update
  // the coarse phase on one CTA (0) or on a cluster of cs CTAs per scene (2..16, from level 1)
  int set_coarse_cluster(int cs);
  int coarse_cluster() const { return coarse_cluster_; }
  // coarsest level of the TOL/FP64 modes: 0 the reference's 120 sweeps, 1 its inverse,
  // 2 its inverse factored beside the pressure loop and used from the next step on
  int set_coarse_solve(int direct);
  // FP64 mode: flexible preconditioned CG around the V-cycle (1) or plain defect correction (0)
  int set_krylov(int on);
  // tile shapes of the advection, diffusion + sources and forces kernels (TILE_TX/TILE_TY index)
  int set_tiles(int advect, int diffsrc, int forces);
  int tiles(int k) const { return tiles_[k]; }
  // times every shape of the three kernels on the current state and keeps the fastest
  int autotune_tiles(int iters, int* best, double* ms);
  int scene_lc(int s) const { return scenes_[s].lc; }
  size_t arena_bytes(int s) const { return scenes_[s].arena_bytes; }
  int scene_nx(int s) const { return scenes_[s].nx; }
  // the host's dt and frame counter of a scene, read without touching the device (a CFL scene's
  // dt is the last one the host has seen)
  double host_dt(int s) const { return scenes_[s].dtd; }
  uint32_t host_frame(int s) const { return scenes_[s].frame; }
  int scene_ny(int s) const { return scenes_[s].ny; }
  cudaStream_t stream() const { return st(); }
  int nscenes() const { return (int)scenes_.size(); }

 private:
  static int choose_lc(const Scene& sc, int cells, int cs);
  int alloc_scene(Scene& sc);
  int build_tmaps(Scene& sc);
  int upload_desc(int s);
  int upload_descs();
  int upload_ctl();
  int build_worklists();
  int ensure_graph();
  void destroy_graph();
  cudaStream_t st() const { return user_stream_ ? user_stream_ : stream_; }
  int activate() const;
  int field_ptr(int s, const std::string& name, char** base, size_t* elem, int* width, int* height, size_t* pitch);
  int max_sub() const;
  int max_levels() const;
  bool any_fp64() const { return mode_ == CFG_SOLVE_FP64; }

  // step pieces; launches counted in launches_
  void enqueue_pre_solve(cudaStream_t s, unsigned long long h, int use_cond);
  // fused kernels (the step's cycle); tail as k_mg_up; count_iter: the first kernel opens a graph iteration
  void enqueue_vcycle(cudaStream_t s, int tail, int count_iter);
  void enqueue_vcycle_ref(cudaStream_t s);   // one kernel per reference dispatch (cfg_vcycle)
  int max_lc() const;
  bool direct_coarse() const { return mode_ != CFG_SOLVE_FIXED && coarse_direct_ != 0; }
  bool pipelined_coarse() const { return direct_coarse() && coarse_direct_ == 2; }
  void enqueue_factor(cudaStream_t s);
  void enqueue_factor_join(cudaStream_t s);
  bool krylov() const { return mode_ == CFG_SOLVE_FP64 && krylov_ != 0; }
  // Krylov mode with the update folded into the level-0 smoother kernels (krylov 1: one scene,
  // 2: any engine), when every scene's coarse block starts below level 0
  bool pcg_fused() const;
  bool any_cfl() const;
  // after a step's launch: every enabled CFL scene's dt now lives on the device
  void mark_device_dt() { for (auto& sc : scenes_) if (sc.enabled && sc.cfl > 0) sc.dt_on_device = true; }
  int cycle_tail() const { return any_fp64() ? (krylov() ? (pcg_fused() ? 4 : 3) : 2) : 1; }
  void enqueue_loop_end(cudaStream_t s);
  void enqueue_fp64_tail(cudaStream_t s);
  void enqueue_cycle_tail(cudaStream_t s, unsigned long long h, int use_cond);
  cudaError_t enqueue_post_solve(cudaStream_t s);
  int host_pressure_loop(bool started);
  void enqueue_bnorm(cudaStream_t s);

  int device_ = 0;
  cudaStream_t stream_ = nullptr, user_stream_ = nullptr, body_stream_ = nullptr;
  cudaStream_t side_stream_ = nullptr;           // the pipelined coarse factorisation's branch
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  std::vector<Scene> scenes_;
  SceneDesc* d_scenes_ = nullptr;
  SolveState* d_solve_ = nullptr;
  SolveCtl* d_ctl_ = nullptr;
  SolveCtl* h_ctl_pinned_ = nullptr;
  // CFL steps: the projection writes each scene's next dt into pinned host memory mapped into
  // the device's address space (d_dtv_ is its device address) and the step records ev_dt_, so
  // cfg_write_params reads it once that event has passed instead of reading the descriptor back
  // (dt_from_step_: no descriptor upload since that step)
  float *h_dt_pinned_ = nullptr, *d_dtv_ = nullptr;
  cudaEvent_t ev_dt_ = nullptr;
  bool dt_from_step_ = false;
  double* d_dxd_ = nullptr;
  double* d_alpha_ = nullptr;
  double* d_scratch_ = nullptr;   // small FP64 outputs (budgets, norms)
  float* d_rwood_ = nullptr;      // the renderer's wood buffer (MAX_PIECES x 12 floats)
  float* d_image_ = nullptr;      // the renderer's output image
  size_t image_bytes_ = 0;
  Work* d_wl_[WL_COUNT] = {};
  int nwl_[WL_COUNT] = {};
  int mode_ = CFG_SOLVE_FIXED, ncycles_ = 1, max_cycles_ = 50;
  double tol_ = 1e-6;
  bool use_graphs_ = true, graph_dirty_ = true;
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t exec_ = nullptr;
  int graph_sub_ = -1;
  int launches_ = 0, launches_per_step_ = 0;
  int last_cycles_ = 1;        // V-cycles of scene 0's last step, recorded by synchronize()
  int vcycle_launches_ = 0;
  size_t coarse_smem_ = 0;
  size_t cf_smem_ = 0;          // k_coarse_factor's dynamic shared memory (largest coarsest level)
  int coarse_cluster_ = 0;      // 0: one-CTA coarse block; cs: the cluster coarse phase
  size_t cluster_smem_ = 0;
  int cf_bw_ = 0;               // the widest coarsest level (k_coarse_factor's register window)
  int coarse_cells_ = COARSE_CELLS;
  int w_cells_ = 0;             // set_coarse_w
  int coarse_direct_ = 0;
  int krylov_ = 0;
  int tiles_[TK_COUNT] = {0, 0, 0};       // tile shape of advection, diffusion + sources, forces
  unsigned long long cond_handle_ = 0;   // the step graph's WHILE-node handle
  int ctl_use_cond_ = 0;                 // SolveCtl::use_cond on the device (-1: stale)
  int set_cond_mode(bool graph);
};

}  // namespace cfg
