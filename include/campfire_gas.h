/*
 * campfire_gas.h — C ABI of the B200 gas step (libcampfire_gas.so).
 *
 * Drop-in for the gas solver host of BoccheseGiacomo/campfire: `class FluidSim`
 * in js/fluid.js:26-356, whose step runs the WGSL kernels of shaders/*.wgsl.
 * Each entry point below names the FluidSim member (or WGSL entry point) it
 * replaces. A JS host binds these through an N-API addon; any other host binds
 * them through its FFI (ctypes, cgo, JNI).
 *
 * Conventions
 *  - Every call returns an int status: CFG_OK (0) or a negative CFG_ERR_*.
 *    cfg_last_error() gives the message of the calling thread's last failure.
 *  - Handles are opaque. A handle is thread-compatible, not thread-safe: calls
 *    on one handle must not overlap. Work is ordered on the handle's CUDA
 *    stream; calls that return host data synchronise that stream.
 *  - Host arrays use the reference's dense row-major layouts (js/fluid.js:51-68):
 *    cells nx*ny (index j*nx+i), U faces (nx+1)*ny, V faces nx*(ny+1), Y 4 floats
 *    per cell (fuel, O2, products, soot), SQ 2 floats per cell (S, heat release),
 *    cellG 2 floats per cell (sdf, bitcast<f32>(piece*4+face)).
 *  - There is no CPU fallback: every entry point that computes needs a CUDA
 *    device and fails with CFG_ERR_NODEV / CFG_ERR_CUDA otherwise.
 */
#ifndef CAMPFIRE_GAS_H
#define CAMPFIRE_GAS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Module constants, js/fluid.js:5-11 */
#define CFG_MAX_PIECES 64
#define CFG_PIECE_FLOATS 20
#define CFG_ACC_GLOBAL 512
#define CFG_ACC_LEN (CFG_ACC_GLOBAL + 16)
#define CFG_E_SCALE 1e6
#define CFG_M_SCALE 1e12
#define CFG_G_SCALE 1e3
#define CFG_N_FLOOR 64
#define CFG_RAD_LEN (CFG_MAX_PIECES * 4 + CFG_N_FLOOR)
#define CFG_MAX_LEVELS 7

/* Status codes */
#define CFG_OK 0
#define CFG_ERR_NOENT (-2)     /* unknown parameter, field or stage name */
#define CFG_ERR_IO (-5)        /* a CUDA call failed */
#define CFG_ERR_NOMEM (-12)    /* device allocation failed or over the memory budget */
#define CFG_ERR_BUSY (-16)     /* readback ring slot still pending (js/fluid.js:317); server busy */
#define CFG_ERR_NODEV (-19)    /* no CUDA device */
#define CFG_ERR_INVAL (-22)    /* bad argument */
#define CFG_ERR_RANGE (-34)    /* 'coarsest level too large' (js/fluid.js:91) */
#define CFG_ERR_TIMEDOUT (-110) /* a bounded device wait ran out */

/* Pressure solve modes (extension; the reference runs one V(2,2) cycle, js/fluid.js:250) */
#define CFG_SOLVE_FIXED 0      /* exactly ncycles V(2,2) cycles */
#define CFG_SOLVE_TOL 1        /* V(2,2) cycles until ||r||2/||rhs||2 <= tol */
#define CFG_SOLVE_FP64 2       /* FP32 V-cycles inside an FP64 defect-correction loop */

/* The 40-field uniform of shaders/common.wgsl:4-15, in the upload order of js/fluid.js:13-24 */
typedef struct cfg_params {
  int32_t nx, ny; float dx, dt;
  float Tamb, rhoAmb, YOamb, grav;
  float cp, Pr, viscMult, diffMult;
  float reactB, reactTa, dHc, sO2;
  float sootFormA, sootFormTa, sootOxA, sootOxTa;
  float kappaSootC, kappaGas, exchAlpha, depth;
  float charA, charTa; int32_t nPieces; uint32_t frame;
  float heaterX0, heaterX1, heaterY1, heaterT;
  float burnerX0, burnerX1, burnerFlux, burnerT;
  float sootDensity, sigma, charO2, time;
} cfg_params;

/* Read-only view of FluidSim's public scalars (js/fluid.js:29-46, 70-91) */
typedef struct cfg_info {
  int32_t nx, ny, levels, diff_sub;
  double dx, dt, height, time;
  uint32_t frame;
  int32_t last_cycles;      /* V-cycles run by the last pressure solve */
  double last_rel;          /* its final ||r||2/||rhs||2 (FP64 mode: of the FP64 defect) */
  int32_t level_nx[CFG_MAX_LEVELS], level_ny[CFG_MAX_LEVELS];
} cfg_info;

typedef struct cfg_sim cfg_sim;
typedef struct cfg_batch cfg_batch;

int cfg_version(void);
int cfg_last_error(char* buf, size_t len);
/* FluidSim's default params (js/fluid.js:35-45 from js/config.js PHYS) */
int cfg_default_params(cfg_params* out);
int cfg_device_count(int* count);

/* new FluidSim(device, {nx, ny, dt}) + await init()  (js/fluid.js:27-47, 49-160).
 * dx = width/nx (the reference fixes width = SCENE_WIDTH = 0.7, js/config.js:3).
 * Fails with CFG_ERR_RANGE when the coarsest multigrid level keeps more than 256
 * cells after 7 halvings (the reference throws after 6, js/fluid.js:72, 91). */
int cfg_create(int nx, int ny, double width, double dt, int device, cfg_sim** out);
int cfg_destroy(cfg_sim* sim);
/* reset(): ambient state, zero velocity/pressure/accumulators  (js/fluid.js:162-176) */
int cfg_reset(cfg_sim* sim);
/* setParam(k, v): stored, applied by the next cfg_write_params  (js/fluid.js:178) */
int cfg_set_param(cfg_sim* sim, const char* name, double value);
int cfg_get_param(cfg_sim* sim, const char* name, double* value);
/* sim.dt = dt (public field; applied by the next cfg_write_params) */
int cfg_set_dt(cfg_sim* sim, double dt);
/* writeParams(): upload the 40-field uniform, recompute the diffusion sub-steps  (js/fluid.js:180-199);
   ordered on the stream (with a CFL step it first reads the device's dt back) */
int cfg_write_params(cfg_sim* sim);
/* uploadPieces(Float32Array(64*20), n)  (js/fluid.js:201-204; packing js/main.js:190-199);
   ordered on the stream, `data` may be reused as soon as the call returns */
int cfg_upload_pieces(cfg_sim* sim, const float* data, int n);
/* clearGeometry(enc)  (js/fluid.js:213): zero the per-face band weights */
int cfg_clear_geometry(cfg_sim* sim);
/* encodeGeometry(pass)  (js/fluid.js:215-218; shaders/geometry.wgsl) */
int cfg_geometry(cfg_sim* sim);
/* nsteps x encodeStep(pass)  (js/fluid.js:225-253), time += dt per step */
int cfg_step(cfg_sim* sim, int nsteps);
/* encodeStepProfiled: one step, per-stage device ms for the 7 stages
 * 'advect','diffuse','sources','forces','coef/rhs','vcycle','project'  (js/fluid.js:256-292).
 * Here 'diffuse' and 'sources' run fused; the fused time is reported under 'sources'. */
int cfg_step_profiled(cfg_sim* sim, float* stage_ms);
/* One stage of the step on the current state: "advect", "diffuse", "sources",
 * "forces", "coef_rhs", "pressure", "project", "diffuse_sources" */
int cfg_run_stage(cfg_sim* sim, const char* stage);
/* vcycle(pass, nu): one V(nu,nu) cycle on the current level-0 rhs/p  (js/fluid.js:294-312); nu = 2 */
int cfg_vcycle(cfg_sim* sim, int nu);
/* encodeRadiation(pass)  (js/fluid.js:220-222; shaders/radiation.wgsl) */
int cfg_radiation(cfg_sim* sim);
/* sim.frame++ (js/main.js:282): the frame counter of the radiation jitter */
int cfg_set_frame(cfg_sim* sim, uint32_t frame);
/* encodeReadback + afterSubmit (js/fluid.js:315-342), synchronous: copies
 * acc[528] (i32), rad[320*4] (f32), faceW[256] (i32), then clears acc. Any pointer may be NULL. */
int cfg_readback(cfg_sim* sim, int32_t* acc, float* rad, int32_t* faceW);
/* encodeReadback(enc) + afterSubmit(cb, tag) (js/fluid.js:315-342), asynchronous: enqueues on the
 * stream the copy of acc[528], rad[320*4] and faceW[256] into the next of three pinned staging
 * slots, then clears acc, and returns at once; *slot (may be NULL) receives the slot. When that
 * slot still holds a readback not yet collected (three pending), it copies nothing, leaves acc
 * accumulating and returns CFG_ERR_BUSY, as the reference skips a frame's readback while its
 * staging buffer is mapped (:317). `tag` comes back with the data (the reference's tag). */
int cfg_readback_begin(cfg_sim* sim, uint64_t tag, int* slot);
/* afterSubmit's callback, polled: the oldest pending readback. *ready = 1 and acc/rad/faceW/tag
 * filled (any pointer may be NULL) once its copies have completed, freeing its slot; *ready = 0
 * if none is pending or the oldest is still in flight. Never waits. */
int cfg_readback_poll(cfg_sim* sim, int32_t* acc, float* rad, int32_t* faceW, uint64_t* tag, int* ready);
/* the same, waiting for the oldest pending readback's copies; CFG_ERR_NOENT if none is pending */
int cfg_readback_wait(cfg_sim* sim, int32_t* acc, float* rad, int32_t* faceW, uint64_t* tag);
/* readBuffer(name) (js/fluid.js:345-355) and its inverse. Names: U V T Y SQ cellG fx fy
 * U2 V2 T2 Y2 p rhs ax ay, and p.L rhs.L ax.L ay.L for multigrid level L.
 * Uh Vh Th Yh are not kept by the fused kernels and read as CFG_ERR_NOENT. */
int cfg_field_size(cfg_sim* sim, const char* name, size_t* count);
int cfg_read_field(cfg_sim* sim, const char* name, float* out, size_t count);
int cfg_write_field(cfg_sim* sim, const char* name, const float* in, size_t count);
/* FP64 level-0 pressure of CFG_SOLVE_FP64 (nx*ny doubles) */
int cfg_read_p64(cfg_sim* sim, double* out, size_t count);
int cfg_get_info(cfg_sim* sim, cfg_info* out);

/* ---- extensions (no counterpart in the reference) ---- */
/* Pressure solve mode; see CFG_SOLVE_*. Defaults: CFG_SOLVE_FIXED, 1 cycle (the reference). */
int cfg_set_solver(cfg_sim* sim, int mode, int ncycles, double tol, int max_cycles);
/* CFL step: after each step dt = min(dt_cap, cfl*dx/max|u|); cfl = 0 keeps dt fixed. Takes effect
 * from the next step. While it is on, the device owns dt: cfg_write_params leaves it as the last
 * step set it (without waiting for the GPU) and cfg_get_info reads dt and the clock from the device. */
int cfg_set_cfl(cfg_sim* sim, double cfl, double dt_cap);
/* Rays per wood face / floor probe of the radiation pass (radiation.wgsl:22 fixes 64) */
int cfg_set_nray(cfg_sim* sim, int nray);
/* ||r||2/||rhs||2 of the level-0 pressure equation now (FP64 sums) */
int cfg_pressure_residual(cfg_sim* sim, double* rel);
/* ||r||2/||rhs||2 of a level-0 pressure field the caller owns, with no device allocation
 * (no counterpart in the reference). For callers that cannot allocate at this point: a frame
 * or serving loop whose device memory is already committed, or that must not stall on the
 * device-wide synchronisation cudaMalloc/cudaFree can cause. Device arrays in the dense
 * layouts of js/fluid.js:75-78: p, rhs nx*ny; ax (nx+1)*ny; ay nx*(ny+1); h2 = (cell size)^2,
 * rounded to f32 as the level uniform. Per-block partial sums go to a fixed 64 KiB
 * __device__ array held by every GPU that loads the library: at most 1,048,576 cells, larger
 * grids fail with CFG_ERR_RANGE. The first call on each device looks up that array's device
 * address; make it before any stream capture. All calls share the array: calls that overlap
 * on the GPU race. Runs on `stream` (NULL: the legacy default stream) and waits for it. */
int cfg_pressure_residual_noalloc(const float* p, const float* rhs, const float* ax, const float* ay, int nx, int ny,
                                  double h2, void* stream, double* rel);
/* FP64 sums over gas cells, per m of depth: mass, energy (rho cp T), fuel, O2, products,
 * soot masses, heat release rate, max T  (8 doubles) */
int cfg_budgets(cfg_sim* sim, double* out);
/* Run the handle's work on a caller-owned cudaStream_t (NULL: the handle's own stream) */
int cfg_set_stream(cfg_sim* sim, void* cuda_stream);
int cfg_synchronize(cfg_sim* sim);
/* Capture each step in a CUDA graph (default on); off launches kernel by kernel */
int cfg_set_graphs(cfg_sim* sim, int enable);
/* Kernels launched by the last cfg_step (per step) */
int cfg_launch_count(cfg_sim* sim, int* per_step);
/* Measurement: launch one kernel of the step `iters` times back to back on the
 * current state and report its mean device time (CUDA events on the handle's
 * stream), its algorithmic bytes per launch and its launches per step.
 * Kernels: "advect", "diffuse_sources", "forces", "relax0", "restrict0",
 * "prolong0", "coarsest", "resnorm", "mg_down0", "mg_up0", "mg_coarse", "vcycle"
 * (one fused V-cycle), "defect64", "project", "mg_downL" / "mg_upL" (level L below the coarse
 * block), "mg_down0_krylov" / "mg_up0_krylov" (the level-0 kernels with the Krylov update folded
 * in, as the step runs them when it is), "pcg_decide" (that mode's per-scene sums and loop decision),
 * "pcg_step", "coarse_factor". The state changes as the kernel runs. */
int cfg_time_kernel(cfg_sim* sim, const char* kernel, int iters, double* mean_ms, double* bytes_per_launch,
                    double* launches_per_step);

/* Smoother schedule (no counterpart in the reference, whose schedule is fixed): the levels
 * from the first one with at most `cells` cells down to the coarsest run in one CTA per
 * scene, the levels above as tiled down/up kernels. Results are bit-identical for every
 * choice; only the time changes. Default 6144. Batch views: use cfg_batch_set_coarse_cells. */
int cfg_set_coarse_cells(cfg_sim* sim, int cells);
/* Where that coarse phase runs: 0 (default) one CTA per scene; 2, 4, 8 or 16: a thread-block
 * cluster of that many CTAs per scene, each owning a share of every level's rows (from level 1
 * at the earliest; level 0 stays tiled). Results are bit-identical for every choice. */
int cfg_set_coarse_cluster(cfg_sim* sim, int cs);
int cfg_batch_set_coarse_cluster(cfg_batch* b, int cs);
/* Cycle shape of the pressure loop (no counterpart in the reference, whose V(2,2) cycle of
 * js/fluid.js:294-312 is the default, cells = 0): the W tail. When the level two above the
 * coarsest has at most `cells` cells, it visits the level below it twice per cycle: after the
 * first visit has come back up, that level is smoothed on from its result and restricted
 * again, and the coarsest is solved again. The level runs inside the one-CTA coarse block,
 * which then starts there at the latest; results do not depend on cfg_set_coarse_cells. A
 * better coarse correction per cycle for the FP64 loop's preconditioner (fewer cycles to the
 * same tolerance on scenes whose coarse levels limit the convergence) for a few block phases.
 * CFG_ERR_INVAL with a cluster coarse phase; CFG_ERR_RANGE if that level does not fit in one
 * CTA's shared memory. */
int cfg_set_coarse_w(cfg_sim* sim, int cells);
int cfg_batch_set_coarse_w(cfg_batch* b, int cells);
/* Coarsest-level solve of the TOL and FP64 modes (no counterpart in the reference, which runs
 * one fixed cycle): 0 (default) the reference's 120 red-black sweeps; 1 the level's operator
 * inverted once per step (f32 banded Cholesky and column solves, after the coefficients are
 * built) and applied in every cycle; 2 (pipelined) the same inverse factored beside the step's
 * pressure loop and applied from the next step on, so the factorisation leaves the critical
 * path (each step's cycles use the previous step's coarsest operator inverse; the first step
 * after a reset or load keeps the sweeps). Scenes whose coarsest level is wider than 32 cells,
 * or has a sealed gas pocket (no open boundary in reach: singular operator), keep the sweeps.
 * FIXED mode ignores it. */
int cfg_set_coarse_solve(cfg_sim* sim, int direct);
int cfg_batch_set_coarse_solve(cfg_batch* b, int direct);
/* FP64 mode outer loop (no counterpart in the reference): 0 (default) plain defect correction
 * (p64 += V-cycle(f32(r)) per cycle); 1 flexible preconditioned conjugate gradients on the
 * level-0 operator in FP64 with the same FP32 V-cycle as preconditioner (Polak-Ribiere
 * direction update), which needs about half the cycles for the same tolerance. With 1 the
 * direction update is folded into the level-0 smoother kernels for one scene and runs as its
 * own kernel for a batch; 2 folds it and 3 keeps the kernel whatever the engine (the folded
 * form reads more bytes per cycle and ends each cycle with a one-CTA decision kernel in place
 * of the update kernel; the same iteration up to rounding). The fold needs every scene's
 * coarse block below level 0, else the update kernel runs (cfg_krylov_folded says which). */
int cfg_set_krylov(cfg_sim* sim, int on);
int cfg_batch_set_krylov(cfg_batch* b, int on);
/* *folded = 1 when the pressure loop runs the Krylov update folded into the level-0 smoother
 * kernels (with a per-scene decision kernel after them): the mode asks for it and every
 * scene's coarse block starts below level 0 (cfg_set_coarse_cells); 0 otherwise */
int cfg_krylov_folded(cfg_sim* sim, int* folded);
int cfg_batch_krylov_folded(cfg_batch* b, int* folded);
/* Autotuner of that schedule (no counterpart in the reference): builds a scratch batch of
 * these sizes on `device` with generated scenes, runs one step to build the coefficients
 * (and, with coarse_direct, the coarsest inverse), then times `iters` fused V-cycles for
 * every threshold that fits (the level sizes). On entry *ncand is the capacity of
 * cand_cells/cand_ms; on return, the candidates timed (ms per cycle) and *best_cells the
 * fastest. */
int cfg_autotune(int device, int nscenes, const int* nx, const int* ny, int coarse_direct, int iters,
                 int* best_cells, int* cand_cells, double* cand_ms, int* ncand);

/* Tile shapes of the advection, diffusion + sources and forces kernels (no counterpart in the
 * reference, whose workgroups are 8x8): 0 = 32x8 cells (default), 1 = 64x8, 2 = 32x16. Every
 * shape gives the same bits; only the time changes. Batch views: use cfg_batch_set_tiles. */
int cfg_set_tiles(cfg_sim* sim, int advect, int diffuse_sources, int forces);
int cfg_batch_set_tiles(cfg_batch* b, int advect, int diffuse_sources, int forces);
/* Autotuner of those shapes (no counterpart in the reference): builds a scratch batch of these
 * sizes on `device` with generated scenes, runs one step, then times `iters` launches of each
 * kernel under each shape; best[3] receives the fastest shape of advection, diffusion + sources
 * and forces, ms[k * 3 + s] (may be NULL) kernel k's mean time under shape s. */
int cfg_autotune_tiles(int device, int nscenes, const int* nx, const int* ny, int iters, int* best, double* ms);

/* Checkpoint / resume of one scene (no counterpart in the reference, which only resets,
 * js/fluid.js:162-176): every state array of the scene (fields, advected copies, sources,
 * geometry, pressure levels, FP64 pressure, accumulators, pieces), its host clock, dt and
 * parameters, the device's parameter block (the CFL step) and its solve state, with an
 * FNV-1a checksum. Loading needs a scene of the same grid size (batch views included);
 * a step after loading continues bit for bit as the saved scene would have. */
int cfg_checkpoint_save(cfg_sim* sim, const char* path);
int cfg_checkpoint_load(cfg_sim* sim, const char* path);

/* Synthetic scenes for the benchmark workloads (seeded, deterministic).
 * kind 0: three square logs of half 0.025 at (0.35,0.025) (0.45,0.025) (0.40,0.068),
 *         flux 5e-3 kg/m2/s at 600 K;  kind 1: five logs of half 0.05 in a seeded tepee,
 *         flux 8e-3;  kind 2: 2-6 seeded floor logs of half 0.025 or 0.05 with B scaled
 *         by log-uniform [0.5,2] and YOamb uniform in [0.18,0.233].
 * Writes the initial T[nx*ny], Y[4*nx*ny], U[(nx+1)*ny], V[nx*(ny+1)], pieces[64*20],
 * the piece count, the params and the CFL-limited dt. */
int cfg_scene_generate(int kind, int nx, int ny, double width, uint64_t seed,
                       float* T, float* Y, float* U, float* V, float* pieces, int* npieces,
                       cfg_params* params, double* dt);

/* ---- batches: many independent scenes of uneven size stepped together ---- */
int cfg_batch_create(int nscenes, const int* nx, const int* ny, const double* width,
                     const double* dt, int device, cfg_batch** out);
int cfg_batch_destroy(cfg_batch* b);
/* A non-owning cfg_sim view of scene i: every single-scene call above except
 * cfg_step / cfg_step_profiled / cfg_vcycle / cfg_run_stage applies to that scene. */
int cfg_batch_scene(cfg_batch* b, int i, cfg_sim** view);
int cfg_batch_set_solver(cfg_batch* b, int mode, int ncycles, double tol, int max_cycles);
int cfg_batch_set_active(cfg_batch* b, int i, int active);
int cfg_batch_step(cfg_batch* b, int nsteps);
int cfg_batch_set_stream(cfg_batch* b, void* cuda_stream);
int cfg_batch_synchronize(cfg_batch* b);
int cfg_batch_launch_count(cfg_batch* b, int* per_step);
/* as cfg_set_graphs, for the whole batch (off: kernel by kernel, e.g. for a profiler's launch list) */
int cfg_batch_set_graphs(cfg_batch* b, int enable);
int cfg_batch_write_params(cfg_batch* b);
int cfg_batch_geometry(cfg_batch* b);
int cfg_batch_set_coarse_cells(cfg_batch* b, int cells);

/* ---- wood: the CPU wood model (js/wood.js WoodPiece) and the per-frame coupling of the
 * campfire app (js/main.js frame(): stepWood, uploadPieces, geometry, gas steps, radiation,
 * readback) around the GPU gas step, for pieces frozen in place (no rigid-body motion). */
typedef struct cfg_wood_piece {
  double side, rhoV, rhoC, mv, mc, Tc, gasRate;
  double Ts[4], Tp[4], d[4], mflux[4], charCov[4], exposure[4];
  int32_t dead, pad;
} cfg_wood_piece;
/* new WoodPiece(side, rhoV, T0) (js/wood.js:34-49) */
int cfg_wood_piece_init(cfg_wood_piece* w, double side, double density, double T0);
/* WoodPiece.preheat (js/wood.js:64-76) */
int cfg_wood_piece_preheat(cfg_wood_piece* w, double Tsurf, double char_depth, double Tcore, double char_yield);
/* WoodPiece.step (js/wood.js:82-181): per face qConv (W/m), qInc (W/m^2), char burnt (kg/m) */
int cfg_wood_piece_step(cfg_wood_piece* w, double dt, const double* qConv4, const double* qInc4,
                        const double* charBurnt4, double char_yield, double pyro_mult);
typedef struct cfg_wood cfg_wood;
/* the pieces of a single-scene handle (not a batch view) and their coupling state */
int cfg_wood_create(cfg_sim* sim, double char_yield, double pyro_mult, cfg_wood** out);
int cfg_wood_destroy(cfg_wood* w);
/* addPiece (js/main.js:103-119): optional preheat {Tsurf, char depth, Tcore} and face
 * temperatures (0: keep); *slot receives the piece slot (0..63) */
int cfg_wood_add(cfg_wood* w, double x, double y, double angle, double side, double density, const double* preheat3,
                 const double* face_T4, int* slot);
int cfg_wood_remove(cfg_wood* w, int slot);
/* one frame with `sim_dt` seconds of gas time (js/main.js:247-283); *nsteps gas steps run */
int cfg_wood_frame(cfg_wood* w, double sim_dt, int* nsteps);
/* How each frame's readback reaches the wood. lag 0 (default): synchronously at the end of the
 * frame. Otherwise as the reference does it (encodeReadback + afterSubmit, js/fluid.js:315-342,
 * and onReadback's tag, js/main.js:210-230): enqueued on the readback ring with the frame's gas
 * time and the pieces that held the slots, and applied at the start of a later frame, before the
 * wood steps, only to those pieces. lag < 0: whatever has arrived, never waiting (a frame whose
 * ring slot is still pending skips its readback); lag 1..3: exactly the readback of the frame
 * `lag` frames back, waited for (the same result from run to run). Pending readbacks are applied
 * before the mode changes. */
int cfg_wood_set_readback_lag(cfg_wood* w, int lag);
/* readbacks applied and skipped (busy ring slot) in the lagged modes so far */
int cfg_wood_readbacks(cfg_wood* w, uint64_t* applied, uint64_t* skipped);
/* a piece's state and its last heat inputs (qConv W/m, qInc W/m^2); CFG_ERR_NOENT if the slot is empty */
int cfg_wood_get(cfg_wood* w, int slot, cfg_wood_piece* out, double* qConv4, double* qInc4);
/* heat release rate and radiative loss (W per m depth) and max T of the last frame (js/main.js:225-229) */
int cfg_wood_stats(cfg_wood* w, double* hrr, double* rad, double* tmax);

/* ---- rigid bodies: the campfire app's 2D rigid-body world (js/rigid.js) on the host in double
 * precision: square pieces per unit depth on a floor between two side walls, soft contacts with
 * warm starting, Coulomb friction with static anchors, and the hand grip. */
typedef struct cfg_rigid cfg_rigid;
typedef struct cfg_rigid_params {    /* RIGID_DEFAULTS, js/rigid.js:12-27 */
  double gravity[2];                 /* m/s^2 */
  double width;                      /* side walls at x = 0 and x = width */
  double dt;                         /* collision step (s) */
  int32_t substeps, pad;
  double slop, contact_hertz, contact_damping, max_pushout;
  double mu_static, mu_kinetic, stick_speed, max_speed;
  double drag_hertz, drag_strength;
} cfg_rigid_params;
typedef struct cfg_rigid_body {
  int32_t id, dragging;
  double x, y, a, vx, vy, w;         /* centre (m), angle (rad), velocities */
  double half, density, mass;        /* half side (m), kg/m^3, kg per m depth */
} cfg_rigid_body;
int cfg_rigid_defaults(cfg_rigid_params* p);
/* new RigidWorld(opts) (js/rigid.js:160-166); p NULL: the defaults */
int cfg_rigid_create(const cfg_rigid_params* p, cfg_rigid** out);
int cfg_rigid_destroy(cfg_rigid* w);
int cfg_rigid_get_params(cfg_rigid* w, cfg_rigid_params* p);
/* world.p = ... (js/main.js:93-94 sets the friction coefficients) */
int cfg_rigid_set_params(cfg_rigid* w, const cfg_rigid_params* p);
/* add(new Body(x, y, half, density, angle)) (:40-49, :167); *id > 0 */
int cfg_rigid_add(cfg_rigid* w, double x, double y, double half, double density, double angle, int* id);
int cfg_rigid_remove(cfg_rigid* w, int id);                                   /* :168-172 */
int cfg_rigid_resize(cfg_rigid* w, int id, double half);                      /* :176-184 */
int cfg_rigid_set_density(cfg_rigid* w, int id, double density);             /* body.density = ... */
int cfg_rigid_step(cfg_rigid* w, double dt, int nsteps);                      /* step(dt) x nsteps, :271-346 */
int cfg_rigid_advance(cfg_rigid* w, double dt);                               /* fixed steps of p.dt, :187-193 */
/* the bodies in world order; *count = all of them, at most `capacity` written */
int cfg_rigid_bodies(cfg_rigid* w, cfg_rigid_body* out, int capacity, int* count);
int cfg_rigid_get(cfg_rigid* w, int id, cfg_rigid_body* out);
/* the topmost body under (x, y) and the point in its frame; *id = 0 if none (:419-428) */
int cfg_rigid_pick(cfg_rigid* w, double x, double y, int* id, double* lx, double* ly);
int cfg_rigid_drag_start(cfg_rigid* w, int id, double lx, double ly, double tx, double ty);   /* :431-439 */
int cfg_rigid_drag_move(cfg_rigid* w, int id, double tx, double ty);                          /* :440-449 */
int cfg_rigid_drag_end(cfg_rigid* w, int id);                                                 /* :451-455 */
int cfg_rigid_max_penetration(cfg_rigid* w, double* pen);                     /* :458-462 */
int cfg_rigid_contacts(cfg_rigid* w, int* manifolds, int* points);
/* Moving pieces in a wood scene: a rigid world (p, or NULL for frozen pieces; only while the scene
 * has no pieces). Each frame then advances the bodies by the frame's gas time and exchanges heat
 * across wood-wood contacts (js/contact.js) before the wood step, the bodies follow the wood's
 * size and density, and the geometry pass rasterises the moved pieces. */
int cfg_wood_set_rigid(cfg_wood* w, const cfg_rigid_params* p);
/* the scene's rigid world (owned by the scene: not for cfg_rigid_destroy), and a piece's body */
int cfg_wood_rigid(cfg_wood* w, cfg_rigid** world);
int cfg_wood_body(cfg_wood* w, int slot, int* body_id);

/* ---- headless renderer: the fragment stage of shaders/render.wgsl (fs :189-273) for one
 * scene into an RGBA float image, in place of Renderer.encode's swapchain pass (js/render.js:
 * 57-70). Pixel (x, y), row 0 at the top, is shaded at uv = ((x + 0.5) / W, 1 - (y + 0.5) / H);
 * the values are the fragment output (sRGB-encoded in view 0) before 8-bit quantisation. */
typedef struct cfg_render_params {    /* the uniform RP (render.wgsl:13-17, js/render.js:41-53) */
  int32_t view;                       /* VIEWS (js/render.js:5): 0 photo, 1 temperature, 2 reaction,
                                         3 oxygen, 4 fuel, 5 velocity, 6 soot */
  int32_t nPieces;                    /* pieces scanned (0..64) */
  float exposure, width, height, ground, time, tmax, chemi, camX, camY, zoom;
} cfg_render_params;
/* Renderer.writeParams's values for this scene (js/render.js:41-53, js/main.js:268-271): view 0,
 * the scene's nPieces, exposure 1, width/height the domain, ground 0.03 m, time the scene's
 * clock, tmax 1800 K, chemi 3e-7, camera (0, -ground), zoom 1 */
int cfg_render_defaults(cfg_sim* sim, cfg_render_params* rp);
/* Renders into rgba (width * height * 4 floats, host). wood: the renderer's wood buffer
 * (64 pieces x 12 floats: Tp[4], d[4], char fraction, Tcore, mean visible irradiance,
 * has virgin wood; js/main.js:200-203), or NULL for zeros. */
int cfg_render(cfg_sim* sim, const cfg_render_params* rp, const float* wood, int width, int height, float* rgba);
/* The same into device memory of the scene's GPU (width * height * 4 floats, 16-byte aligned),
 * enqueued on the handle's stream without waiting (the wood buffer is copied before return). */
int cfg_render_device(cfg_sim* sim, const cfg_render_params* rp, const float* wood, int width, int height,
                      void* rgba_device);
/* Replace the wood state of a piece (js/main.js:135-142 sets a coal's state this way) */
int cfg_wood_set(cfg_wood* w, int slot, const cfg_wood_piece* state);
/* The wood buffer of a wood scene's pieces as uploadPieces builds it (js/main.js:188-207) */
int cfg_wood_render_data(cfg_wood* w, float* wood);

/* ---- serving: jobs of several grid sizes in resident batch slots (no counterpart in the
 * reference). One batch holds slots[c] scenes of size class c (nx[c] x ny[c]); a job is
 * admitted into a free slot of its class once it has arrived and the bytes of the slots in
 * use plus its own fit in budget_bytes. Admitted jobs advance together, one batched step per
 * loop iteration, and leave after their own step count (continuous batching). */
typedef struct cfg_server cfg_server;
typedef struct cfg_job {
  int32_t size_class;       /* index into the server's classes */
  int32_t kind;             /* scene generator kind (cfg_scene_generate) */
  uint64_t seed;            /* scene seed */
  int32_t nsteps;           /* gas steps to run */
  int32_t flags;            /* CFG_JOB_KEEP_FIELDS (cfg_server_submit) */
  double arrival_s;         /* arrival time, seconds after cfg_server_run starts (cfg_server_run only) */
} cfg_job;
#define CFG_JOB_KEEP_FIELDS 1   /* keep the final T, Y, U, V on the host for cfg_server_fetch */
typedef struct cfg_job_result {
  double arrival_s, admit_s, done_s;   /* seconds after cfg_server_run starts */
  int32_t slot, steps, last_cycles, pad;
  double last_rel;          /* final relative residual of the last pressure solve */
  uint64_t hash;            /* FNV-1a 64 of the final dense T, Y, U, V bytes */
  double t_sum;             /* sum of the final T */
} cfg_job_result;
int cfg_server_create(int device, int nclasses, const int* nx, const int* ny, const int* slots, double budget_bytes,
                      double width, cfg_server** out);
int cfg_server_destroy(cfg_server* s);
/* solver of every slot (as cfg_set_solver, cfg_set_coarse_solve, cfg_set_coarse_cells (cells <= 0
 * keeps it) and cfg_set_krylov, whose 0-3 it takes) */
int cfg_server_set_solver(cfg_server* s, int mode, int ncycles, double tol, int max_cycles, int coarse_direct,
                          int coarse_cells, int krylov);
/* cycle shape of every slot (as cfg_set_coarse_w); CFG_ERR_BUSY while jobs run */
int cfg_server_set_coarse_w(cfg_server* s, int cells);
/* device bytes of one slot of a size class */
int cfg_server_slot_bytes(cfg_server* s, int size_class, size_t* bytes);
/* run the jobs to completion in real time (arrivals are honoured by the host clock);
 * results[j] for jobs[j]; *wall_s the run's duration, *cell_updates the cells stepped */
int cfg_server_run(cfg_server* s, const cfg_job* jobs, int njobs, cfg_job_result* results, double* wall_s,
                   double* cell_updates);
/* Asynchronous service: a host thread (started by the first submission) runs the same loop on
 * jobs handed over one at a time; a job arrives when it is submitted. Times in the results are
 * seconds after cfg_server_create. */
int cfg_server_submit(cfg_server* s, const cfg_job* job, uint64_t* ticket);
/* *done = 1 and *out filled (the result is then released) once the job has finished, else 0 */
int cfg_server_poll(cfg_server* s, uint64_t ticket, cfg_job_result* out, int* done);
/* waits up to timeout_s for the job; CFG_ERR_TIMEDOUT if it has not finished */
int cfg_server_wait(cfg_server* s, uint64_t ticket, double timeout_s, cfg_job_result* out);
/* runs every submitted job to completion and stops the service thread (destroy does the same) */
int cfg_server_drain(cfg_server* s);
/* a finished CFG_JOB_KEEP_FIELDS job's final field ("T", "Y", "U", "V"; dense, count floats) */
int cfg_server_fetch(cfg_server* s, uint64_t ticket, const char* name, float* out, size_t count);
/* frees a job's kept fields */
int cfg_server_release(cfg_server* s, uint64_t ticket);

#ifdef __cplusplus
}
#endif
#endif /* CAMPFIRE_GAS_H */
