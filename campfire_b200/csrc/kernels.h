// Kernel launchers of the B200 gas step (host-callable, stream-ordered).
#pragma once
#include <cuda_runtime.h>

#include "gas_dev.cuh"

namespace cfg {

// Tile shapes (cells) of the level-0 kernels. Tiles are aligned to multiples of
// 8 cells so the 8x8 blocks of the heat-release reduction match the WGSL
// workgroups of sources.wgsl:34 exactly.
constexpr int ADV_TX = 32, ADV_TY = 8, ADV_H = 2;    // advection (halo for |displacement| < 2 cells)
constexpr int DS_TX = 32, DS_TY = 8;                 // diffusion + sources
constexpr int FR_TX = 32, FR_TY = 8;                 // forces + coef + rhs0 (+ coefficient hierarchy)
// Tile shapes the advection, diffusion + sources and forces kernels can run with (the
// defaults above are shape 0). Every shape gives the same bits: each cell's arithmetic does
// not depend on its tile, and the 8x8 blocks of the heat-release reduction stay whole.
constexpr int kTileShapes = 3;
constexpr int TILE_TX[kTileShapes] = {32, 64, 32}, TILE_TY[kTileShapes] = {8, 8, 16};
enum TileKernel { TK_ADVECT = 0, TK_DIFFSRC, TK_FORCES, TK_COUNT };
// diffusion + sources keeps its tile and halo state in dynamic shared memory (up to ~53 KB):
// allowed once per device before the first launch
cudaError_t prepare_diffuse_sources();
constexpr int FR_KMAX = 3;                           // coarse coefficient levels built inside FR tiles
constexpr int MG_TX = 32, MG_TY = 8;                 // single-pass multigrid kernels
constexpr int MGF_TX = 32, MGF_TY = 16;              // fused (temporally blocked) multigrid kernels
constexpr int MGF_H = 5;                             // their halo: 4 colour passes + the residual's neighbours
// The fused kernels stage their tiles with TMA tensor copies. A box starts MGF_SX
// cells left of the tile so that its x coordinate stays 16-byte aligned, and the
// level's boundary is zero-filled by the copy.
constexpr int MGF_SX = 8;
constexpr int MGF_BW = MGF_TX + 2 * MGF_SX, MGF_BH = MGF_TY + 2 * MGF_H;   // p, pb, rhs, ax box (ay: one more row)
constexpr int MGF_CBW = MGF_TX / 2 + 16, MGF_CBH = MGF_TY / 2 + 8;        // coarse p box of the up kernel
// tensor maps per level, in the scene arena (CUtensorMap: 128 bytes, 64-byte aligned)
enum TmapKind { TM_P = 0, TM_PB, TM_RHS, TM_AX, TM_AY, TM_PC, TM_PER_LEVEL };
constexpr int TMAP_BYTES = 128;
constexpr int COARSE_CELLS = 6144;                   // default: largest level handled by the one-CTA coarse block
constexpr size_t kCoarseSmemMax = 232448 - 2048;     // dynamic shared memory of the coarse block (227 KB less static)
constexpr int PR_TX = 32, PR_TY = 8;                 // projection
static_assert(PR_TX == MG_TX && PR_TY == MG_TY, "the projection's tiles are counted as the level-0 multigrid tiles");
constexpr int GEO_TX = 32, GEO_TY = 8;               // geometry

// Launch with programmatic stream serialization (the kernel must call pdl_wait()
// before it touches data an earlier kernel of the step writes) when `pdl`, else an
// ordinary launch.
template <typename... KArgs, typename... Args>
inline void launch_pdl(bool pdl, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = pdl ? 1 : 0;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}
// programmatic dependent launch for the pressure-loop kernels (set by the engine)
void set_pdl(bool on);
bool pdl_enabled();

// Work-list kinds (tiles per scene are built by the engine)
enum WorkKind { WK_ADV, WK_DS, WK_FR, WK_PR, WK_GEO, WK_MG0 };

// shape: an index into TILE_TX/TILE_TY, the shape the work list was built with
void launch_advect(const SceneDesc* scenes, const Work* work, int ntiles, int shape, cudaStream_t st);
// diffusion sub-steps (diff_sub of each scene) fused with the sources pass
void launch_diffuse_sources(const SceneDesc* scenes, const Work* work, int ntiles, int max_sub,
                            bool with_sources, bool with_diffusion, int shape, cudaStream_t st);
// forces (+ coef + rhs0 + coefficient levels 1..FR_KMAX + ||rhs|| reduction)
void launch_forces(const SceneDesc* scenes, const Work* work, int ntiles, SolveCtl* ctl, bool forces,
                   bool coef_rhs, bool fp64, int shape, cudaStream_t st);
// coefficient restriction of level l -> l+1 for levels the FR tiles did not build
void launch_coef_restrict(const SceneDesc* scenes, const Work* work, int ntiles, int level, cudaStream_t st);
// single-pass multigrid (pressure.wgsl:87-129)
void launch_relax(const SceneDesc* scenes, const Work* work, int ntiles, int level, int color, cudaStream_t st);
void launch_restrict_res(const SceneDesc* scenes, const Work* work, int ntiles, int level, cudaStream_t st);
void launch_prolong(const SceneDesc* scenes, const Work* work, int ntiles, int level, cudaStream_t st);
void launch_coarsest(const SceneDesc* scenes, int nscenes, cudaStream_t st);
// level-0 residual norm + per-scene loop decision
void launch_resnorm(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, SolveCtl* ctl,
                    cudaStream_t st);
// FP64 defect: r64 = rhs64 - A p64, rhs0 = f32(r64), p0 = 0, ||r64|| + loop decision
void launch_defect64(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, SolveCtl* ctl,
                     int first, cudaStream_t st);
// Krylov FP64 mode: direction + L d + alpha; then p64/r update + ||r|| + loop decision
void launch_pcg_step(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, SolveCtl* ctl,
                     cudaStream_t st);
// fused Krylov mode, after the loop: the last cycle's d and p64 update
void launch_pcg_finish(const SceneDesc* scenes, const Work* work, int ntiles, cudaStream_t st);
// end of a loop iteration: count it and set the WHILE node's condition (bounded by SolveCtl::hard_cap)
void launch_loop_guard(SolveCtl* ctl, unsigned long long cond_handle, int use_cond, cudaStream_t st);
// a scene's parameter block (the leading PARAM_WORDS words of SceneDesc) and its pieces, passed by value
constexpr int PARAM_WORDS = 51;
struct ParamWords { uint32_t w[PARAM_WORDS]; };
struct PieceFloats { float f[MAX_PIECES * PIECE_FLOATS]; };
// dst[k] = b.w[k] except word `skip` and words [s0, s1) (-1: none)
void launch_write_params(uint32_t* dst, const ParamWords& b, int skip, int s0, int s1, cudaStream_t st);
void launch_write_pieces(float* dst, const PieceFloats& b, cudaStream_t st);
// nwords words of src to mapped pinned host memory, then the first nzero cleared on the device
void launch_readback(uint32_t* src, uint32_t* host, int nwords, int nzero, cudaStream_t st);
// fused V(2,2) cycle: per fine level a down kernel (4 passes + restriction) and an
// up kernel (prolongation + 4 passes; level 0 tail: 1 residual norm + decision,
// 2 p64 += p, 3 the Krylov dot products, 4 the fused Krylov mode's), and one CTA per
// scene for levels lc..coarsest
// count_iter: the kernel opens a graph loop iteration (loop_count); pcg: level 0 of the
// fused Krylov mode (applies the previous cycle's update); nscenes: the engine's scenes
// (with one, tiles are requested before the scene's active flag is read: it only stops the loop)
void launch_mg_down(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, int level, SolveCtl* ctl,
                    int count_iter, int pcg, cudaStream_t st);
void launch_mg_up(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, int level, int tail, SolveCtl* ctl,
                  cudaStream_t st);
// after the level-0 up kernel with tail 4: each scene's dot products summed, the coefficients
// and the loop decision (one CTA per scene)
void launch_pcg_decide(const SceneDesc* scenes, int nscenes, SolveCtl* ctl, cudaStream_t st);
// wtail: some scene has the W tail (SceneDesc::lw), else the V-cycle's instance; level0: some
// scene's block covers level 0 (the cycle's level-0 ends: warm start, `tail`), else an instance
// without them
void launch_mg_coarse(const SceneDesc* scenes, int nscenes, SolveCtl* ctl, int tail, int count_iter, size_t smem,
                      int wtail, int level0, cudaStream_t st);
size_t coarse_smem_bytes(const int* lnx, const int* lny, int lc, int nlev);
// the cluster coarse phase (k_mgc.cu): levels lc..coarsest of each scene on a cluster of cs CTAs
constexpr size_t kClusterSmemMax = 232448 - 2048;
size_t cluster_smem_bytes(const int* lnx, const int* lny, int lc, int nlev, int cs);
cudaError_t prepare_mg_cluster();
void launch_mg_cluster(const SceneDesc* scenes, int nscenes, SolveCtl* ctl, int cs, int count_iter, size_t smem,
                       cudaStream_t st);
cudaError_t prepare_mg_coarse(size_t smem);
// direct coarse solve: the inverse of each scene's coarsest operator (scenes whose
// coarsest level is wider than 32 cells keep the sweeps)
// pipelined: factor this step's operator into the half the next step uses (see k_cinv_swap)
void launch_coarse_factor(const SceneDesc* scenes, int nscenes, size_t smem, int bw, int pipelined, cudaStream_t st);
// pipelined coarse solve: switch every enabled scene to the inverse factored during the step
void launch_cinv_swap(const SceneDesc* scenes, int nscenes, cudaStream_t st);
// Row stride (floats) of the coarsest inverse of n unknowns: the smallest ld >= n with ld = 8
// (mod 32), so that the four rows a warp reads at once in the coarse block's product fall in
// different shared-memory banks (ld * 4 bytes stays a multiple of 16 for the bulk copies)
__host__ __device__ constexpr int cinv_ld(int n) { return n <= 8 ? 8 : (n - 8 + 31) / 32 * 32 + 8; }
// dynamic shared memory of k_coarse_factor for a coarsest level of n cells and band width bw
size_t coarse_factor_smem(int n, int bw);
cudaError_t prepare_coarse_factor(size_t smem);
// ||rhs||^2 (FP64 mode: ||rhs64||^2) of level 0; arms the pressure loop
void launch_bnorm(const SceneDesc* scenes, const Work* work, int ntiles, SolveCtl* ctl, bool fp64, cudaStream_t st);
// FP64: p64 += p0
void launch_accum64(const SceneDesc* scenes, const Work* work, int ntiles, cudaStream_t st);
// projection (+ max|u| and the CFL step for the next step)
// post: bit 0 swaps the scenes' coarsest inverse halves, bit 1 sets the CFL scenes' next dt
// (what k_cinv_swap and k_cfl_update do on their own), both after the projection's work
// the coefficient restriction of every level from `level` down, one CTA per scene
void launch_coef_restrict_tail(const SceneDesc* scenes, int nscenes, int level, cudaStream_t st);
// (bit 1 also stores each CFL scene's next dt in dtv[scene] when dtv is given)
void launch_project(SceneDesc* scenes, const Work* work, int ntiles, bool fp64, cudaStream_t st, int nscenes = 0,
                    int post = 0, const double* dxd = nullptr, const double* alpha = nullptr, float* dtv = nullptr);
void launch_cfl_update(SceneDesc* scenes, int nscenes, const double* dxd, const double* alpha, cudaStream_t st);
void launch_geometry(const SceneDesc* scenes, const Work* work, int ntiles, cudaStream_t st);
void launch_radiation(const SceneDesc* scenes, int scene, int ntargets, int nray, cudaStream_t st);
// FP64 budgets of one scene into out[8] (device)
void launch_budgets(const SceneDesc* scenes, int scene, double* out, cudaStream_t st);
// ||r||2 and ||rhs||2 of level 0 of one scene into out[2] (device, FP64)
void launch_residual_norms(const SceneDesc* scenes, int scene, double* out, cudaStream_t st);
// render.wgsl's fragment stage of one scene: W x H float4 pixels, row 0 at the top
void launch_render(const SceneDesc* scenes, int scene, const cfg_render_params& rp, const float* wood, int width,
                   int height, float* out, cudaStream_t st);

}  // namespace cfg
