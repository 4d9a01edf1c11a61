// Fused multigrid V(2,2) cycle of shaders/pressure.wgsl (schedule of
// js/fluid.js:294-312) with temporal blocking.
//
// Each fine level l < lc is handled by two kernels per cycle:
//   down: stage p, rhs, ax, ay of the tile plus a 5-cell halo into shared
//         memory with TMA tensor copies, run the 4 colour passes (red, black,
//         red, black), each one cell narrower than the last, then the residual
//         of the tile's cells and its restriction to the coarse rhs (coarse p = 0);
//   up:   the same staging (and the coarse p under the tile), bilinear
//         prolongation of the coarse correction, 4 colour passes (black, red,
//         black, red); on level 0 also the residual norm (FP32 modes) or
//         p64 += p (FP64 defect correction).
// A cell update reads exactly the neighbour values the separate dispatches
// would read, so the result equals the reference schedule bit for bit.
// Down kernels read p and write pb; up kernels read pb and write p, so no CTA
// reads a halo another CTA is rewriting.
// Levels lc..coarsest run in one CTA per scene (coarse block): every level's
// arrays staged into shared memory by TMA bulk copies, __syncthreads between
// passes, and the coarsest level's 120 red-black sweeps (pressure.wgsl:132-156)
// on one thread per red/black cell pair with a named barrier.
#include "gas_dev.cuh"
#include "kernels.h"
#include "reduce.cuh"
#include "mg_common.cuh"
#include "tma.cuh"

#include <algorithm>

namespace cfg {

namespace {

// Shared tile of the fused kernels: every array staged as an MGF_BW-wide box whose
// column 0 is level column sx and row 0 is level row sy (ay has one more row).
struct Tile {
  float *p, *rhs, *ax, *ay;
  int sx, sy;
  __device__ __forceinline__ int c(int i, int j) const { return (j - sy) * MGF_BW + (i - sx); }
};

// pressure.wgsl:77-85 on the shared tile (i, j in level coordinates); ax[c] is the
// west face of cell c, ay[c] its south face
__device__ __forceinline__ void stencil_s(const Tile& t, int nx, int ny, int i, int j, float& off, float& diag) {
  off = 0.f; diag = 0.f;
  const int k = t.c(i, j);
  const float w = t.ax[k], e = t.ax[k + 1], s = t.ay[k], n = t.ay[k + MGF_BW];
  if (i > 0) { off += w * t.p[k - 1]; diag += w; } else { diag += 2.f * w; }
  if (i < nx - 1) { off += e * t.p[k + 1]; diag += e; } else { diag += 2.f * e; }
  if (j > 0) { off += s * t.p[k - MGF_BW]; diag += s; }
  if (j < ny - 1) { off += n * t.p[k + MGF_BW]; diag += n; } else { diag += 2.f * n; }
}
// (L z)_ij in FP64 from the tile's f32 z and coefficients (pressure.wgsl:77-85 promoted,
// as the FP64 defect: (off - diag z) / h2, 0 in closed cells). The products of two f32 values
// are exact in FP64, so the fused multiply-adds round as the separate products and sums
// would; the division is a product with rh2 = 1 / h2 (FP64, one rounding more: the Krylov
// loop's own operator, the same in every kernel that forms it)
__device__ __forceinline__ double lap_tile64(const Tile& t, const LevelDesc& L, int i, int j, double rh2) {
  const int k = t.c(i, j);
  const double w = t.ax[k], e = t.ax[k + 1], s = t.ay[k], n = t.ay[k + MGF_BW];
  double off = 0.0, diag = 0.0;
  if (i > 0) { off = __fma_rn(w, (double)t.p[k - 1], off); diag += w; } else diag += 2.0 * w;
  if (i < L.nx - 1) { off = __fma_rn(e, (double)t.p[k + 1], off); diag += e; } else diag += 2.0 * e;
  if (j > 0) { off = __fma_rn(s, (double)t.p[k - MGF_BW], off); diag += s; }
  if (j < L.ny - 1) { off = __fma_rn(n, (double)t.p[k + MGF_BW], off); diag += n; } else diag += 2.0 * n;
  return diag > 0.0 ? __fma_rn(-diag, (double)t.p[k], off) * rh2 : 0.0;
}
__device__ __forceinline__ float diag_s(const Tile& t, int nx, int ny, int i, int j) {
  const int k = t.c(i, j);
  const float w = t.ax[k], e = t.ax[k + 1], s = t.ay[k], n = t.ay[k + MGF_BW];
  float diag = 0.f;
  if (i > 0) diag += w; else diag += 2.f * w;
  if (i < nx - 1) diag += e; else diag += 2.f * e;
  if (j > 0) diag += s;
  if (j < ny - 1) diag += n; else diag += 2.f * n;
  return diag;
}

constexpr uint32_t BOX_BYTES = MGF_BW * MGF_BH * 4, BOX_AY_BYTES = MGF_BW * (MGF_BH + 1) * 4;
constexpr uint32_t CBOX_BYTES = MGF_CBW * MGF_CBH * 4;

__device__ __forceinline__ const void* tmap_of(const SceneDesc& S, int level, int kind) {
  return S.tmap + (size_t)(level * TM_PER_LEVEL + kind) * TMAP_BYTES;
}

// Tile staging on two barriers around the wait on the previous kernel. stage_coef
// (before the wait in a one-scene engine, which also waits for them and builds the stencils
// before the wait, with the state copies' tensor maps prefetched; else once the scene's flag
// says it still cycles): one thread initialises both barriers and requests the coefficients
// ax, ay on bar[0]; they are built before the pressure loop and written by no loop kernel
// (the loop is entered through a full dependency: a graph node or a memset). stage_state
// (after the wait): p from map `pkind`, rhs and the coarse p under the tile on bar[1]; with
// `copy` false nothing is requested and bar[1] completes on its arrival; with `pload` false p
// is not copied (the caller zero-fills its box). The copies are
// issued whether or not the scene still cycles, so the read of its `active` flag overlaps
// them. tile_wait: all threads wait for one barrier (bounded); false in every thread if a
// wait ran out, after recording the error and waiting once more for the copies in flight.
__device__ __forceinline__ void stage_coef(const SceneDesc& S, int level, const Tile& t, uint64_t* bar) {
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_arrive_expect_tx(&bar[0], BOX_BYTES + BOX_AY_BYTES);
    tma_load_2d(t.ax, tmap_of(S, level, TM_AX), t.sx, t.sy, &bar[0]);
    tma_load_2d(t.ay, tmap_of(S, level, TM_AY), t.sx, t.sy, &bar[0]);
  }
}
// the tensor maps of stage_state's copies into the descriptor cache (before the wait)
__device__ __forceinline__ void prefetch_state_maps(const SceneDesc& S, int level, int pkind, bool coarse) {
  if (threadIdx.x == 0) {
    tmap_prefetch(tmap_of(S, level, pkind));
    tmap_prefetch(tmap_of(S, level, TM_RHS));
    if (coarse) tmap_prefetch(tmap_of(S, level + 1, TM_PC));
  }
}
__device__ __forceinline__ void stage_state(const SceneDesc& S, int level, int pkind, const Tile& t, bool copy,
                                            float* cp, int cx, int cy, uint64_t* bar, bool pload = true) {
  if (threadIdx.x == 0) {
    mbar_arrive_expect_tx(&bar[1], copy ? (pload ? 2 : 1) * BOX_BYTES + (cp ? CBOX_BYTES : 0u) : 0u);
    if (copy) {
      if (pload) tma_load_2d(t.p, tmap_of(S, level, pkind), t.sx, t.sy, &bar[1]);
      tma_load_2d(t.rhs, tmap_of(S, level, TM_RHS), t.sx, t.sy, &bar[1]);
      if (cp) tma_load_2d(cp, tmap_of(S, level + 1, TM_PC), cx, cy, &bar[1]);
    }
  }
}
__device__ __forceinline__ bool tile_wait(uint64_t* bar, SolveCtl* ctl) {
  const bool ok = mbar_wait(bar, 0);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(&ctl->err, 1);
    mbar_wait(bar, 0);
    return false;
  }
  return true;
}
// both barriers of a tile: the coefficients (then `between`, e.g. the stencils), the state
template <class F>
__device__ __forceinline__ bool tile_wait2(uint64_t* bar, SolveCtl* ctl, F&& between) {
  if (!tile_wait(&bar[0], ctl)) {
    mbar_wait(&bar[1], 0);
    return false;
  }
  between();
  return tile_wait(&bar[1], ctl);
}


// The four colour passes of a fused kernel with every cell's stencil in registers. Pass k
// (1..4) covers [x0-H+k, x0+TX+H-k) x [y0-H+k, y0+TY+H-k) clipped to the level, with colour
// (first + k - 1) & 1; thread t owns slots t and t + 256 of each colour in pass 1's region
// (the largest; 20 cells of a colour per row). tile_stencils builds their stencils from the
// coefficients alone (the four coefficients, zero for a neighbour outside the level, the
// diagonal, its correctly rounded reciprocal, the passes that include the cell, whether it
// is a tile cell); tile_passes adds rhs h2 once the state has landed and updates the cells
// by pressure.wgsl:87-94, dividing by div_by_rcp.
struct TCell { float w, e, s, n, rh, diag, rcp; int kp, fl; };   // fl: 1 a tile cell; 16 << k: pass k
constexpr int SM_W1 = MGF_TX + 2 * MGF_H - 2, SM_H1 = MGF_TY + 2 * MGF_H - 2;   // pass 1's region
__device__ __forceinline__ void tile_stencils(const Tile& t, const LevelDesc& L, int x0, int y0, int first,
                                              TCell (&c)[2][2]) {
  constexpr int HALF = SM_W1 / 2;
  static_assert(SM_W1 % 2 == 0 && HALF * SM_H1 <= 2 * 256, "two slots of a colour per thread");
  const int ib = x0 - MGF_H + 1, jb = y0 - MGF_H + 1;
  #pragma unroll
  for (int col = 0; col < 2; col++)
    #pragma unroll
    for (int m = 0; m < 2; m++) {
      TCell& q = c[col][m];
      q.fl = 0;
      const int sl = threadIdx.x + 256 * m;
      if (sl >= HALF * SM_H1) continue;
      const int r = sl / HALF, j = jb + r, i = ib + ((ib + j + col) & 1) + 2 * (sl - r * HALF);
      if (i < 0 || i >= L.nx || j < 0 || j >= L.ny) continue;
      // pass k (1..4) covers the cells at distance >= k from the edge of the region
      // [x0-H, x0+TX+H) x [y0-H, y0+TY+H), and has colour (first + k - 1) & 1: passes 1, 3
      // or 2, 4 for this cell's colour, up to its distance; distance >= H: a tile cell
      const int d = min(min(i - (x0 - MGF_H), x0 + MGF_TX + MGF_H - 1 - i),
                        min(j - (y0 - MGF_H), y0 + MGF_TY + MGF_H - 1 - j));
      const int pm = (((first ^ col) & 1) ? (64 | 256) : (32 | 128)) & (((2 << min(d, 4)) - 2) << 4);
      if (!pm) continue;
      const int k = t.c(i, j);
      q.kp = k;
      const float w = t.ax[k], e = t.ax[k + 1], s = t.ay[k], n = t.ay[k + MGF_BW];
      float diag = 0.f;
      if (i > 0) diag += w; else diag += 2.f * w;
      if (i < L.nx - 1) diag += e; else diag += 2.f * e;
      if (j > 0) diag += s;
      if (j < L.ny - 1) diag += n; else diag += 2.f * n;
      q.diag = diag;
      q.rcp = diag > 0.f ? __frcp_rn(diag) : 0.f;
      // a neighbour outside the level contributes nothing (pressure.wgsl:77-85): its
      // coefficient is zero in the passes' sums, whose values outside the level are zero
      q.w = i > 0 ? w : 0.f;
      q.e = i < L.nx - 1 ? e : 0.f;
      q.s = j > 0 ? s : 0.f;
      q.n = j < L.ny - 1 ? n : 0.f;
      q.fl = pm | (d >= MGF_H ? 1 : 0);
    }
}
// off of pressure.wgsl:77-85 from the slot's stencil: every neighbour's term is added in the
// reference's order (west, east, south, north); a missing neighbour's term is an exact zero,
// and adding it to a sum that started at +0 leaves the sum's bits unchanged
__device__ __forceinline__ float tcell_off(const Tile& t, const TCell& q) {
  float off = 0.f;
  off += q.w * t.p[q.kp - 1];
  off += q.e * t.p[q.kp + 1];
  off += q.s * t.p[q.kp - MGF_BW];
  off += q.n * t.p[q.kp + MGF_BW];
  return off;
}
__device__ __forceinline__ void tile_passes(const Tile& t, const LevelDesc& L, int first, TCell (&c)[2][2]) {
  #pragma unroll
  for (int col = 0; col < 2; col++)
    #pragma unroll
    for (int m = 0; m < 2; m++)
      if (c[col][m].fl) c[col][m].rh = t.rhs[c[col][m].kp] * L.h2;
  #pragma unroll
  for (int k = 1; k <= 4; k++) {
    const int col = (first + k - 1) & 1;
    float v[2];
    #pragma unroll
    for (int m = 0; m < 2; m++) {
      const TCell& q = c[col][m];
      if (!(q.fl & (16 << k))) continue;
      const float off = tcell_off(t, q);
      v[m] = q.diag > 0.f ? mgc::div_by_rcp(off - q.rh, q.diag, q.rcp) : 0.f;
    }
    #pragma unroll
    for (int m = 0; m < 2; m++)
      if (c[col][m].fl & (16 << k)) t.p[c[col][m].kp] = v[m];
    __syncthreads();
  }
}

// The up kernel's prolongation (pressure.wgsl:116-129) over the region [x0-H, x0+TX+H) x
// [y0-H, y0+TY+H); with one scene split in two. prolong_plan (from the coefficients and the level
// sizes alone, beside the stencils before the wait) packs for element e = threadIdx.x + 256 m: the fine cell's box index
// (bits 0-10), the index in the coarse box of its own coarse cell (11-19), the steps to the other
// coarse column and row of its bilinear stencil plus one (20-21, 22-23), whether the cell is open
// (24) and whether it lies in the level (25). prolong_apply adds the interpolated correction once
// the coarse box has landed: a closed cell adds +0, as pressure.wgsl:129 has it.
constexpr int PR_W = MGF_TX + 2 * MGF_H, PR_H = MGF_TY + 2 * MGF_H, PR_N = (PR_W * PR_H + 255) / 256;
static_assert(MGF_BW * MGF_BH <= 2048 && MGF_CBW * MGF_CBH <= 512, "plan fields");
__device__ __forceinline__ void prolong_plan(const Tile& t, const LevelDesc& L, const LevelDesc& C, int x0, int y0,
                                             int cx, int cy, uint32_t (&pl)[PR_N]) {
  #pragma unroll
  for (int m = 0; m < PR_N; m++) {
    const int e = threadIdx.x + 256 * m;
    const int i = x0 - MGF_H + e % PR_W, j = y0 - MGF_H + e / PR_W;
    pl[m] = 0u;
    if (e >= PR_W * PR_H || i < 0 || i >= L.nx || j < 0 || j >= L.ny) continue;
    const int I = i / 2, J = j / 2;
    const int dI = min(max(I + ((i & 1) == 1 ? 1 : -1), 0), C.nx - 1) - I;
    const int dJ = min(max(J + ((j & 1) == 1 ? 1 : -1), 0), C.ny - 1) - J;
    const int a = (J - cy) * MGF_CBW + I - cx;
    pl[m] = (uint32_t)t.c(i, j) | (uint32_t)a << 11 | (uint32_t)(dI + 1) << 20 | (uint32_t)(dJ + 1) << 22 |
            (diag_s(t, L.nx, L.ny, i, j) > 0.f ? 1u << 24 : 0u) | 1u << 25;
  }
}
// the same additions computed in one pass after the coarse box has landed (several scenes: the
// plan would only add instructions after the wait)
__device__ __forceinline__ void prolong_direct(const Tile& t, const LevelDesc& L, const LevelDesc& C, int x0, int y0,
                                               int cx, int cy, const float* scp) {
  for (int e = threadIdx.x; e < PR_W * PR_H; e += 256) {
    const int i = x0 - MGF_H + e % PR_W, j = y0 - MGF_H + e / PR_W;
    if (i < 0 || i >= L.nx || j < 0 || j >= L.ny) continue;
    const int I = i / 2, J = j / 2;
    const int I2 = min(max(I + ((i & 1) == 1 ? 1 : -1), 0), C.nx - 1);
    const int J2 = min(max(J + ((j & 1) == 1 ? 1 : -1), 0), C.ny - 1);
    const int r0 = (J - cy) * MGF_CBW, r1 = (J2 - cy) * MGF_CBW;
    const float c_ = 0.5625f * scp[r0 + I - cx] + 0.1875f * (scp[r0 + I2 - cx] + scp[r1 + I - cx]) +
                     0.0625f * scp[r1 + I2 - cx];
    t.p[t.c(i, j)] += diag_s(t, L.nx, L.ny, i, j) > 0.f ? c_ : 0.f;
  }
}
__device__ __forceinline__ void prolong_apply(const Tile& t, const float* scp, const uint32_t (&pl)[PR_N]) {
  #pragma unroll
  for (int m = 0; m < PR_N; m++) {
    const uint32_t q = pl[m];
    if (!(q & (1u << 25))) continue;
    const int a = (q >> 11) & 511, dI = (int)((q >> 20) & 3) - 1, dJ = ((int)((q >> 22) & 3) - 1) * MGF_CBW;
    const float c_ = 0.5625f * scp[a] + 0.1875f * (scp[a + dI] + scp[a + dJ]) + 0.0625f * scp[a + dI + dJ];
    t.p[q & 2047] += (q & (1u << 24)) ? c_ : 0.f;
  }
}

// Fused Krylov mode on level 0 (all scenes' coarse blocks start below it). The update of
// cycle c (d = z + beta d, q = Lz + beta q, p64 += alpha d, r -= alpha q with cycle c's
// alpha, beta) is split: the next cycle's down kernel forms d and p64 on its tile and the
// new rhs0 = f32(r - alpha q) on pass 1's region from the stored r, q, Lz (read only
// there, so no CTA reads a value another rewrites); the next up kernel rewrites r and q on
// its tile before its dot products; the update of the last cycle is applied by
// k_pcg_finish after the loop. The up kernel's tiles leave their nine dot products as
// partials; k_pcg_decide (one CTA per scene, the next kernel) sums them, forms the cycle's
// alpha and beta, and ||r_c||^2 = r.r - 2 alpha r.q_c + alpha^2 q_c.q_c (q_c = Lz + beta q)
// for the loop decision.
// This thread's share of the down kernel's update: up to 4 cells of pass 1's region and
// 2 tile cells, with their stored values loaded right after the wait.
struct PcgDown {
  double r[4], q[4], lz[4], dA[2], p64[2];
  float z[2];
};
__device__ __forceinline__ void pcg_down_load(const SceneDesc& S, const LevelDesc& L, int x0, int y0, PcgDown& u) {
  constexpr int N1 = SM_W1 * SM_H1;
  #pragma unroll
  for (int m = 0; m < 4; m++) {
    const int e = threadIdx.x + 256 * m;
    const int i = x0 - MGF_H + 1 + e % SM_W1, j = y0 - MGF_H + 1 + e / SM_W1;
    if (e < N1 && i >= 0 && i < L.nx && j >= 0 && j < L.ny) {
      const int k = j * L.nx + i;
      u.r[m] = __ldcg(S.r64 + k); u.q[m] = __ldcg(S.q64 + k); u.lz[m] = __ldcg(S.dB + k);
    }
  }
  #pragma unroll
  for (int m = 0; m < 2; m++) {
    const int e = threadIdx.x + 256 * m;
    const int i = x0 + e % MGF_TX, j = y0 + e / MGF_TX;
    if (i < L.nx && j < L.ny) {
      u.dA[m] = __ldcg(S.dA + j * L.nx + i); u.p64[m] = __ldcg(S.p64 + j * L.nx + i);
      u.z[m] = __ldcg(L.p + j * L.pc + i);
    }
  }
}
// after the state barrier: p = 0 on the whole box, rhs0 on pass 1's region, d and p64 on the
// tile (rhs0 of the tile to global for the up kernel's staging once the block has synced)
__device__ __forceinline__ void pcg_down_apply(const SceneDesc& S, const LevelDesc& L, const Tile& t, int x0, int y0,
                                               const PcgPrev& pv, const PcgDown& u) {
  constexpr int N1 = SM_W1 * SM_H1;
  const bool first = pv.cycles == 1;
  for (int e = threadIdx.x; e < MGF_BW * MGF_BH; e += 256) t.p[e] = 0.f;
  #pragma unroll
  for (int m = 0; m < 4; m++) {
    const int e = threadIdx.x + 256 * m;
    const int i = x0 - MGF_H + 1 + e % SM_W1, j = y0 - MGF_H + 1 + e / SM_W1;
    if (e < N1 && i >= 0 && i < L.nx && j >= 0 && j < L.ny) {
      const double q = first ? u.lz[m] : u.lz[m] + pv.beta * u.q[m];
      const double r = u.r[m] - pv.alpha * q;
      t.rhs[t.c(i, j)] = (float)r;
    }
  }
  #pragma unroll
  for (int m = 0; m < 2; m++) {
    const int e = threadIdx.x + 256 * m;
    const int i = x0 + e % MGF_TX, j = y0 + e / MGF_TX;
    if (i < L.nx && j < L.ny) {
      const double z = (double)u.z[m];
      const double d = first ? z : z + pv.beta * u.dA[m];
      S.dA[j * L.nx + i] = d;
      S.p64[j * L.nx + i] = u.p64[m] + pv.alpha * d;
    }
  }
}

}  // namespace

// ------------------------------------------------------------------ down: 4 passes + restrict
// PCG: the fused Krylov update on level 0 (above)
// ONE: compiled for an engine of one scene (nscenes == 1), whose flag only ends the loop
// MINB: resident CTAs per SM the registers are sized for (3; 2 for a level-0 Krylov kernel whose
// tiles fit in one wave at two per SM: no spill)
template <int TX, int TY, bool PCG, bool ONE, int MINB = 3>
// three CTAs per SM (at most 85 registers a thread; 44 bytes of spill in the fused Krylov
// variant): 512x768's 768 level-0 tiles run in two waves instead of three (measured: -5% per
// Krylov cycle at 512x768). Four for the plain variants (62 registers) was measured 3-4% slower
// per step at 256x384 and 512x768 and no faster for the batch.
__global__ void __launch_bounds__(256, MINB) k_mg_down(const SceneDesc* __restrict__ scenes, int nscenes, const Work* __restrict__ work,
                                                 int level, SolveCtl* ctl, int count_iter) {
  static_assert(TX == MGF_TX && TY == MGF_TY, "the tensor-map boxes are built for the MGF tile");
  __shared__ __align__(128) float sp[MGF_BH * MGF_BW];
  __shared__ __align__(128) float srhs[MGF_BH * MGF_BW];
  __shared__ __align__(128) float sax[MGF_BH * MGF_BW];
  __shared__ __align__(128) float say[(MGF_BH + 1) * MGF_BW];
  __shared__ float sr[TY * TX];
  __shared__ __align__(8) uint64_t bar[2];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  pdl_trigger();
  const LevelDesc L = S.lev[level], C = S.lev[level + 1];
  const int x0 = w.tx * TX, y0 = w.ty * TY;
  const Tile t{sp, srhs, sax, say, x0 - MGF_SX, y0 - MGF_H};
  const bool on = S.enabled;   // host-written, constant during the step
  SolveState* ss = S.solve;
  // one scene: its flag only ends the loop, so the tile is requested before it is read;
  // several: a scene that stopped loads nothing
  constexpr bool spec = ONE;
  if (on && spec) {
    stage_coef(S, level, t, bar);
    prefetch_state_maps(S, level, TM_P, false);
  }
  // below level 0 the level's p is zero on entry (the restriction above zeroes it): with one
  // scene its box is zero-filled before the wait instead of copied after it
  const bool pz = spec && level > 0;
  if (pz)
    for (int e = threadIdx.x; e < MGF_BW * MGF_BH; e += 256) t.p[e] = 0.f;
  __syncthreads();
  // one scene: the stencils, which depend on the coefficients alone, are built before the wait
  TCell c[2][2];
  bool ok = true;
  if (on && spec && (ok = tile_wait(&bar[0], ctl))) tile_stencils(t, L, x0, y0, 0, c);
  pdl_wait();
  if (count_iter && blockIdx.x == 0 && threadIdx.x == 0) loop_count(ctl);
  if (!on || !ok) return;
  if (!spec) {
    if (*(volatile int*)&ss->active == 0) return;
    stage_coef(S, level, t, bar);
    __syncthreads();
  }
  PcgPrev pv{};
  PcgDown u;
  if (PCG) {
    pv = pcg_load(ss);
    pcg_down_load(S, L, x0, y0, u);
  }
  const bool live = *(volatile int*)&ss->active != 0;
  const bool upd = PCG && pv.cycles >= 1;   // an update of the previous cycle is pending
  stage_state(S, level, TM_P, t, !upd, nullptr, 0, 0, bar, !pz);
  if (!(spec ? tile_wait(&bar[1], ctl) : tile_wait2(bar, ctl, [&] { tile_stencils(t, L, x0, y0, 0, c); })) || !live)
    return;
  if (upd) {
    pcg_down_apply(S, L, t, x0, y0, pv, u);
    __syncthreads();
    for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
      const int i = x0 + e % TX, j = y0 + e / TX;
      if (i < L.nx && j < L.ny) L.rhs[j * L.pc + i] = t.rhs[t.c(i, j)];
    }
  }
  tile_passes(t, L, 0, c);   // colours 0, 1, 0, 1 (js/fluid.js:298-301)
  // residual of the tile cells (pressure.wgsl:96-101) from the slots' stencils (every tile cell
  // of the level is a slot of some thread); the quotient by h2 from RN(1/h2), the IEEE one
  const float rh2 = __frcp_rn(L.h2);
  #pragma unroll
  for (int col = 0; col < 2; col++)
    #pragma unroll
    for (int m = 0; m < 2; m++) {
      const TCell& q = c[col][m];
      if (!(q.fl & 1)) continue;
      const int bj = q.kp / MGF_BW, bi = q.kp - bj * MGF_BW;   // box row and column
      const float off = tcell_off(t, q);
      sr[(bj - MGF_H) * TX + (bi - MGF_SX)] =
          q.diag <= 0.f ? 0.f : t.rhs[q.kp] - mgc::div_by_rcp(off - q.diag * t.p[q.kp], L.h2, rh2);
    }
  // the smoothed p
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    const int i = x0 + e % TX, j = y0 + e / TX;
    if (i < L.nx && j < L.ny) L.pb[j * L.pc + i] = t.p[t.c(i, j)];
  }
  __syncthreads();
  // restriction (pressure.wgsl:104-113)
  constexpr int CX = TX / 2, CY = TY / 2;
  for (int e = threadIdx.x; e < CX * CY; e += blockDim.x) {
    const int a = e % CX, b = e / CX, I = x0 / 2 + a, J = y0 / 2 + b;
    if (I >= C.nx || J >= C.ny) continue;
    const float r = sr[(2 * b) * TX + 2 * a] + sr[(2 * b) * TX + 2 * a + 1] + sr[(2 * b + 1) * TX + 2 * a] +
                    sr[(2 * b + 1) * TX + 2 * a + 1];
    C.rhs[J * C.pc + I] = 0.25f * r;
    C.p[J * C.pc + I] = 0.f;
  }
}

// ------------------------------------------------------------------ up: prolong + 4 passes (+ level-0 tail)
// tail: 0 none, 1 residual norm + loop decision (FP32 modes), 2 p64 += p (FP64 defect correction),
// 3 r.z, q.z, z.Lz -> the direction update (Krylov FP64 mode), 4 the same in the fused Krylov
// mode (the pending r, q update first; the loop decision from the recurrence for ||r||); one
// instance per tail (levels below 0: tail 0)
template <int TX, int TY, int TAIL, bool ONE, int MINB = 3>   // ONE, MINB: as in k_mg_down
__global__ void __launch_bounds__(256, MINB) k_mg_up(const SceneDesc* __restrict__ scenes, int nscenes, const Work* __restrict__ work,
                                               int level, SolveCtl* ctl) {
  static_assert(TX == MGF_TX && TY == MGF_TY, "the tensor-map boxes are built for the MGF tile");
  static_assert(TAIL >= 0 && TAIL <= 4, "tails 0-4");
  constexpr bool KRY = TAIL == 4;
  constexpr int tail = TAIL;
  __shared__ __align__(128) float sp[MGF_BH * MGF_BW];
  __shared__ __align__(128) float srhs[MGF_BH * MGF_BW];
  __shared__ __align__(128) float sax[MGF_BH * MGF_BW];
  __shared__ __align__(128) float say[(MGF_BH + 1) * MGF_BW];
  __shared__ __align__(128) float scp[MGF_CBH * MGF_CBW];
  __shared__ double red[32];
  __shared__ __align__(8) uint64_t bar[2];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  pdl_trigger();
  const LevelDesc L = S.lev[level], C = S.lev[level + 1];
  const int x0 = w.tx * TX, y0 = w.ty * TY;
  const Tile t{sp, srhs, sax, say, x0 - MGF_SX, y0 - MGF_H};
  // coarse p under the region: columns x0/2-4 .. x0/2+TX/2+3, rows y0/2-4 .. y0/2+TY/2+3
  const int cx = x0 / 2 - 8, cy = y0 / 2 - 4;
  const bool on = S.enabled;   // host-written, constant during the step
  SolveState* ss = S.solve;
  constexpr bool spec = ONE;   // as in k_mg_down
  if (on && spec) {
    stage_coef(S, level, t, bar);
    prefetch_state_maps(S, level, TM_PB, true);
  }
  __shared__ double s_rh2;   // the FP64 operator's 1 / h2 (tails 3 and 4)
  if (threadIdx.x == 0) s_rh2 = 1.0 / (double)L.h2;
  __syncthreads();
  const double rh2 = s_rh2;
  TCell c[2][2];
  uint32_t pl[PR_N];
  bool ok = true;
  if (on && spec && (ok = tile_wait(&bar[0], ctl))) {
    tile_stencils(t, L, x0, y0, 1, c);
    prolong_plan(t, L, C, x0, y0, cx, cy, pl);
  }
  pdl_wait();
  if (!on || !ok) return;
  if (!spec) {
    if (*(volatile int*)&ss->active == 0) return;
    stage_coef(S, level, t, bar);
    __syncthreads();
  }
  stage_state(S, level, TM_PB, t, true, scp, cx, cy, bar);
  const bool live = *(volatile int*)&ss->active != 0;
  // fused Krylov mode: the solve state and this thread's stored r, q, Lz, read beside the copies
  PcgPrev pv{};
  double r0[2] = {0.0, 0.0}, q0[2] = {0.0, 0.0}, lz0[2] = {0.0, 0.0};
  if (KRY) {
    pv = pcg_load(ss);
    #pragma unroll
    for (int m = 0; m < 2; m++) {
      const int e = threadIdx.x + 256 * m;
      const int i = x0 + e % TX, j = y0 + e / TX;
      if (i < L.nx && j < L.ny) {
        const int kk = j * L.nx + i;
        r0[m] = __ldcg(S.r64 + kk); q0[m] = __ldcg(S.q64 + kk); lz0[m] = __ldcg(S.dB + kk);
      }
    }
  }
  if (!(spec ? tile_wait(&bar[1], ctl) : tile_wait2(bar, ctl, [&] { tile_stencils(t, L, x0, y0, 1, c); })) || !live)
    return;
  // prolongation (pressure.wgsl:116-129) on the whole region
  if (spec)
    prolong_apply(t, scp, pl);
  else
    prolong_direct(t, L, C, x0, y0, cx, cy, scp);
  __syncthreads();
  tile_passes(t, L, 1, c);   // colours 1, 0, 1, 0 (js/fluid.js:307-310)
  if (KRY) {
    // the pending r, q update (cycles >= 1), then r.z, q.z, z.Lz and the recurrence's r.r,
    // r.Lz, r.q, Lz.Lz, Lz.q, q.q on the tile
    const bool upd = pv.cycles >= 1, first = pv.cycles == 1;
    double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    #pragma unroll
    for (int m = 0; m < 2; m++) {
      const int e = threadIdx.x + 256 * m;
      const int i = x0 + e % TX, j = y0 + e / TX;
      if (i >= L.nx || j >= L.ny) continue;
      const int k = t.c(i, j), kk = j * L.nx + i;
      L.p[j * L.pc + i] = t.p[k];
      double r = r0[m], q = q0[m];
      if (upd) {
        q = first ? lz0[m] : lz0[m] + pv.beta * q;
        r = r - pv.alpha * q;
        S.q64[kk] = q;
        S.r64[kk] = r;
      }
      const double z = (double)t.p[k];
      const double lz = lap_tile64(t, L, i, j, rh2);
      S.dB[kk] = lz;
      v[0] = __fma_rn(r, z, v[0]); v[1] = __fma_rn(q, z, v[1]); v[2] = __fma_rn(z, lz, v[2]);
      v[3] = __fma_rn(r, r, v[3]); v[4] = __fma_rn(r, lz, v[4]); v[5] = __fma_rn(r, q, v[5]);
      v[6] = __fma_rn(lz, lz, v[6]); v[7] = __fma_rn(lz, q, v[7]); v[8] = __fma_rn(q, q, v[8]);
    }
    // the tile's nine partials, quantity-major (part[m * nt_up0 + tile]); k_pcg_decide sums
    // them once this kernel has completed (no arrival, no fence in these CTAs)
    __shared__ double redt[9 * 256 + 9];
    block_sum_t<9>(v, redt);
    if (threadIdx.x == 0)
      #pragma unroll
      for (int m = 0; m < 9; m++) S.part[m * S.nt_up0 + w.tile] = v[m];
    return;
  }
  double part = 0.0, part2 = 0.0, part3 = 0.0;
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    const int i = x0 + e % TX, j = y0 + e / TX;
    if (i >= L.nx || j >= L.ny) continue;
    const int k = t.c(i, j);
    L.p[j * L.pc + i] = t.p[k];
    if (tail == 1) {
      float off, diag; stencil_s(t, L.nx, L.ny, i, j, off, diag);
      const double r = diag <= 0.f ? 0.0 : (double)(t.rhs[k] - (off - diag * t.p[k]) / L.h2);
      part += r * r;
    } else if (tail == 2) {
      S.p64[j * L.nx + i] += (double)t.p[k];
    } else if (tail == 3) {
      // z = the cycle's p; Lz from the tile (its ring is exact after the fourth pass), in FP64
      const int kk = j * L.nx + i;
      const double z = (double)t.p[k];
      const double lz = lap_tile64(t, L, i, j, rh2);
      S.dB[kk] = lz;
      part += S.r64[kk] * z;
      part2 += S.q64[kk] * z;
      part3 += z * lz;
    }
  }
  if (tail == 3) {
    const double pa = block_sum(part, red);
    const double pb = block_sum(part2, red);
    const double pz = block_sum(part3, red);
    double ta = 0.0, tb = 0.0, tz = 0.0;
    if (scene_reduce3(S, w.tile, S.nt_up0, pa, pb, pz, red, &ta, &tb, &tz) && threadIdx.x == 0) pcg_coef(S, ta, tb, tz);
    return;
  }
  if (tail != 1) return;
  const double bp = block_sum(part, red);
  double total = 0.0;
  if (scene_reduce(S, w.tile, S.nt_up0, bp, red, &total) && threadIdx.x == 0) solve_decide(ctl, ss, total, true);
}

// ------------------------------------------------------------------ fused Krylov mode: the loop decision
// One CTA per scene, after the level-0 up kernel has completed: the nine sums over the scene's
// tiles (thread t adds tiles t, t + 256, ... in that order, four tiles' loads in flight at a
// time; then block_sum_t's fixed order), the cycle's coefficients and the decision. A scene
// that is disabled or no longer cycles wrote no partials and does not decide.
__global__ void __launch_bounds__(256) k_pcg_decide(const SceneDesc* __restrict__ scenes, SolveCtl* ctl) {
  const SceneDesc& S = scenes[blockIdx.x];
  pdl_trigger();
  const bool on = S.enabled;   // host-written, constant during the step
  const int nt = S.nt_up0;
  SolveState* ss = S.solve;
  pdl_wait();
  // the flag, the solve state and the partials are read together (the partial array is always
  // allocated; a scene that stopped leaves stale values, which are loaded but not used)
  const int act = *(volatile int*)&ss->active;
  PcgPrev pv{};
  DecideIn din{};
  if (threadIdx.x == 0) {
    pv = pcg_load(ss);
    din = decide_load(ctl, ss);
  }
  double v[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int k0 = threadIdx.x; k0 < nt; k0 += 4 * 256) {
    double a[4][9];
    #pragma unroll
    for (int j = 0; j < 4; j++)
      #pragma unroll
      for (int m = 0; m < 9; m++) a[j][m] = k0 + 256 * j < nt ? __ldcg(S.part + (size_t)m * nt + k0 + 256 * j) : 0.0;
    #pragma unroll
    for (int j = 0; j < 4; j++)
      if (k0 + 256 * j < nt)
        #pragma unroll
        for (int m = 0; m < 9; m++) v[m] += a[j][m];
  }
  if (!on || act == 0) return;   // the same in every thread of the CTA
  __shared__ double redt[9 * 256 + 9];
  block_sum_t<9>(v, redt);
  if (threadIdx.x == 0) {
    double alpha, beta;
    pcg_coef(ss, pv, v[0], v[1], v[2], &alpha, &beta);
    // ||r - alpha (Lz + beta q)||^2 from the dot products
    const double rq = v[4] + beta * v[5];
    const double qq = v[6] + 2.0 * beta * v[7] + beta * beta * v[8];
    const double r2 = v[3] - 2.0 * alpha * rq + alpha * alpha * qq;
    solve_decide(ctl, ss, din, r2 > 0.0 ? r2 : 0.0, true);
  }
}

// ------------------------------------------------------------------ coarse block: levels lc..coarsest in one CTA
// Shared memory holds every level >= lc with the global row pitches (pc for p,
// rhs, ay; pu for ax), so each array arrives by one TMA bulk copy; then a
// residual scratch of level lc's size.
namespace {
constexpr int CB_THREADS = 512;
constexpr int kStagedInverseMax = 128;   // coarsest unknowns whose inverse (<= 64 KB) is staged in shared memory
constexpr int CB_WARPS = CB_THREADS / 32;
constexpr int COARSEST_SCRATCH = 0;     // the coarsest keeps its stencils in registers
using namespace mgc;


// Cells of a level mapped linearly onto the block: thread t takes column t % w of rows
// t / w, t / w + R, ... (R = rows per round of the block), so every lane works whatever the
// level's width and warps beyond the level's cells skip at once. w > CB_THREADS: the block
// strides along each row instead.
struct LinMap {
  int i0, j0, R;   // first column and row of this thread, rows per round (0: the thread idles)
  __device__ __forceinline__ LinMap(int w, unsigned long long mw) {   // mw = fdiv_magic(w)
    if (w >= CB_THREADS) { i0 = threadIdx.x; j0 = 0; R = 1; }
    else {
      R = fdiv(CB_THREADS, mw);
      j0 = fdiv(threadIdx.x, mw);
      i0 = threadIdx.x - j0 * w;
      if (j0 >= R) R = 0;
    }
  }
  __device__ __forceinline__ int di(int w) const { return w >= CB_THREADS ? CB_THREADS : w; }   // column stride
};
// one colour pass over the cells of one colour: slot q of row j is cell i = 2q + ((j + color) & 1).
// A pass reads only cells of the other colour: up to 4 rows of a thread are computed before
// any is stored, so their shared-memory loads overlap.
__device__ __forceinline__ void pass_d(const LvS& L, int color, const LinMap& mp) {
  const int half = (L.nx + 1) >> 1;
  if (!mp.R) return;
  for (int q = mp.i0; q < half; q += mp.di(half))
    for (int jb = mp.j0; jb < L.ny; jb += 4 * mp.R) {
      float v[4];
      int kk[4];
      #pragma unroll
      for (int m = 0; m < 4; m++) {
        const int j = jb + m * mp.R, i = 2 * q + ((j + color) & 1);
        kk[m] = -1;
        if (j < L.ny && i < L.nx) {
          float off, diag; stencil_d(L, i, j, off, diag);
          const int k = j * L.pc + i;
          v[m] = diag > 0.f ? (off - L.rhs[k] * L.h2) / diag : 0.f;
          kk[m] = k;
        }
      }
      #pragma unroll
      for (int m = 0; m < 4; m++)
        if (kk[m] >= 0) L.p[kk[m]] = v[m];
    }
}
// A level visit's smoothing with every cell's stencil in registers: thread t owns colour
// slots t, t + CB_THREADS, ... (slot -> row slot / half, cell 2 (slot % half) + parity) of
// each colour, and builds their stencils once (coefficients, neighbour flags, rhs h2, the
// diagonal and its correctly rounded reciprocal) for the visit's two sweeps. The update is
// pass_d's, with the division by the diagonal as div_by_rcp: the same quotient.
// one cell's stencil in 9 registers: fl bit 0..3 = west, east, south, north neighbour present
struct RCell { float w, e, s, n, rh, diag, rcp; int kp, fl; };
// the diagonal's reciprocal comes from the block's table (L.rc, built once per kernel)
__device__ __forceinline__ RCell rcell_of(const LvS& L, int i, int j) {
  RCell c;
  c.kp = j * L.pc + i;
  c.w = L.ax[j * L.pu + i]; c.e = L.ax[j * L.pu + i + 1];
  c.s = L.ay[c.kp]; c.n = L.ay[c.kp + L.pc];
  float diag = 0.f;
  if (i > 0) diag += c.w; else diag += 2.f * c.w;
  if (i < L.nx - 1) diag += c.e; else diag += 2.f * c.e;
  if (j > 0) diag += c.s;
  if (j < L.ny - 1) diag += c.n; else diag += 2.f * c.n;
  c.diag = diag;
  c.rcp = L.rc[j * L.nx + i];
  c.rh = L.rhs[c.kp] * L.h2;
  c.fl = (i > 0 ? 1 : 0) | (i < L.nx - 1 ? 2 : 0) | (j > 0 ? 4 : 0) | (j < L.ny - 1 ? 8 : 0);
  return c;
}
// res (the down visit's residuals, or null): after the sweeps, each thread writes the residual
// of its cells (pressure.wgsl:96-101, with the stencils it holds) to res[j * pc + i]
template <int NPER>
__device__ __forceinline__ void smooth_regs(const LvS& L, int first, float* res = nullptr) {
  const int half = (L.nx + 1) >> 1;
  RCell c[2][NPER];
  bool act[2][NPER];
  #pragma unroll
  for (int col = 0; col < 2; col++)
    #pragma unroll
    for (int m = 0; m < NPER; m++) {
      const int t = threadIdx.x + m * CB_THREADS;
      const int j = fdiv(t, L.mhalf), i = 2 * (t - j * half) + ((j + col) & 1);
      act[col][m] = j < L.ny && i < L.nx;
      if (act[col][m]) c[col][m] = rcell_of(L, i, j);
    }
  #pragma unroll 1
  for (int k = 0; k < 2; k++)
    #pragma unroll
    for (int h = 0; h < 2; h++) {
      const int col = h == 0 ? first : 1 - first;
      float v[NPER];
      #pragma unroll
      for (int m = 0; m < NPER; m++) {
        if (!act[col][m]) continue;
        const RCell& q = c[col][m];
        float off = 0.f;
        if (q.fl & 1) off += q.w * L.p[q.kp - 1];
        if (q.fl & 2) off += q.e * L.p[q.kp + 1];
        if (q.fl & 4) off += q.s * L.p[q.kp - L.pc];
        if (q.fl & 8) off += q.n * L.p[q.kp + L.pc];
        v[m] = q.diag > 0.f ? div_by_rcp(off - q.rh, q.diag, q.rcp) : 0.f;
      }
      #pragma unroll
      for (int m = 0; m < NPER; m++)
        if (act[col][m]) L.p[c[col][m].kp] = v[m];
      __syncthreads();
    }
  if (!res) return;
  #pragma unroll
  for (int col = 0; col < 2; col++)
    #pragma unroll
    for (int m = 0; m < NPER; m++) {
      if (!act[col][m]) continue;
      const RCell& q = c[col][m];
      float off = 0.f;
      if (q.fl & 1) off += q.w * L.p[q.kp - 1];
      if (q.fl & 2) off += q.e * L.p[q.kp + 1];
      if (q.fl & 4) off += q.s * L.p[q.kp - L.pc];
      if (q.fl & 8) off += q.n * L.p[q.kp + L.pc];
      res[q.kp] = q.diag <= 0.f ? 0.f : L.rhs[q.kp] - div_by_rcp(off - q.diag * L.p[q.kp], L.h2, L.rh2);
    }
  __syncthreads();
}
// both sweeps of a level visit (colour `first` first in each sweep, a block barrier after
// every pass): in registers when each thread owns at most two cells of a colour. With res
// (a down visit), true when the residuals were also written there (the register path)
__device__ __forceinline__ bool smooth_visit(const LvS& L, int first, float* res = nullptr) {
  const int half = (L.nx + 1) >> 1, nslot = half * L.ny;
  if (nslot <= CB_THREADS) { smooth_regs<1>(L, first, res); return res != nullptr; }
  if (nslot <= 2 * CB_THREADS) { smooth_regs<2>(L, first, res); return res != nullptr; }
  const LinMap mh(half, L.mhalf);
  for (int k = 0; k < 2; k++) { pass_d(L, first, mh); __syncthreads(); pass_d(L, 1 - first, mh); __syncthreads(); }
  return false;
}
// The coarse block's level visits (k_mg_coarse), and what they read beside the block's shared
// memory.
struct CbCtx {
  float* smem;
  const LvO* lvo;     // level offsets in smem (shared)
  float* sres;        // residual scratch (level lc size)
  const SceneDesc* S;
  int nl, s_dir, s_inv, s_A;
};
// level l's visit on the way down: smoothing, then per coarse cell the residuals of its four
// fine cells summed in the restriction's order
__device__ __forceinline__ void cb_down(const CbCtx c, int l) {
  float* const smem = c.smem;
  const LvO* const lvo = c.lvo;
  const LvS F = lvs_at(smem, lvo[l]), Cc = lvs_at(smem, lvo[l + 1]);
  const LinMap mc(Cc.nx, Cc.mnx);
  // the residuals from the smoothing's register stencils (pitched like F in the scratch), or
  // recomputed per coarse cell on the shared-memory path of large levels
  if (smooth_visit(F, 0, c.sres)) {
    const float* r = c.sres;
    if (mc.R)
    for (int J = mc.j0; J < Cc.ny; J += mc.R)
      for (int I = mc.i0; I < Cc.nx; I += mc.di(Cc.nx)) {
        const int e = 2 * J * F.pc + 2 * I;
        Cc.rhs[J * Cc.pc + I] = 0.25f * (r[e] + r[e + 1] + r[e + F.pc] + r[e + F.pc + 1]);
        Cc.p[J * Cc.pc + I] = 0.f;
      }
    __syncthreads();
    return;
  }
  auto res = [&](int i, int j) {
    float off, diag; stencil_d(F, i, j, off, diag);
    const int e = j * F.pc + i;
    return diag <= 0.f ? 0.f : F.rhs[e] - div_by_rcp(off - diag * F.p[e], F.h2, F.rh2);
  };
  if (mc.R)
  for (int J = mc.j0; J < Cc.ny; J += mc.R)
    for (int I = mc.i0; I < Cc.nx; I += mc.di(Cc.nx)) {
      const float r = res(2 * I, 2 * J) + res(2 * I + 1, 2 * J) + res(2 * I, 2 * J + 1) + res(2 * I + 1, 2 * J + 1);
      Cc.rhs[J * Cc.pc + I] = 0.25f * r;
      Cc.p[J * Cc.pc + I] = 0.f;
    }
  __syncthreads();
}
// the coarsest level's solve (its p overwritten: the inverse's product, or sweeps from zero)
__device__ __forceinline__ void cb_coarsest(const CbCtx c) {
  float* const smem = c.smem;
  const LvO* const lvo = c.lvo;
  float* const sres = c.sres;
  const SceneDesc& S = *c.S;
  const int nl = c.nl, s_dir = c.s_dir, s_inv = c.s_inv, s_A = c.s_A;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // ---- coarsest (pressure.wgsl:132-156): 120 red-black sweeps from zero. Row-major
    // cells 2t and 2t+1 have opposite colours for any nx (even nx: same row, adjacent;
    // odd nx: colour = index parity), so thread t owns one cell of each colour and every
    // thread works in every pass; the ceil(n/2) threads (<= 128, rounded up to warps)
    // sync on a named barrier while the other warps wait at the block barrier below.
    // Stencils, diagonals and their reciprocals stay in registers for all sweeps.
    if (s_dir) {
      // direct coarse solve (TOL/FP64 modes): p = A^-1 b with b = -rhs h2 (0 in closed cells),
      // each row's dot product as 8 strided partial sums combined pairwise (the oracle's order)
      const LvS L = lvs_at(smem, lvo[nl - 1]);
      const int n = L.nx * L.ny;
      for (int k = threadIdx.x; k < n; k += CB_THREADS) {
        const int j = fdiv(k, L.mnx), i = k - j * L.nx;
        sres[k] = L.rc[k] > 0.f ? -(L.rhs[j * L.pc + i] * L.h2) : 0.f;
      }
      __syncthreads();
      const int q = lane & 7;
      const bool staged = s_inv != 0;
      // the global copy is addressed only when the inverse is not staged
      const int ld = cinv_ld(n);
      const float* Ag = staged ? nullptr : S.cinv + (size_t)S.solve->cinv_cur * n * ld;
      const float* As = smem + s_A;
      for (int base = warp * 4; base < n; base += CB_WARPS * 4) {
        const int k = base + (lane >> 3);
        float sum = 0.f;
        if (k < n) {
          if (staged) {
            #pragma unroll 4
            for (int m = q; m < n; m += 8) sum = __fmaf_rn(As[k * ld + m], sres[m], sum);
          } else {
            #pragma unroll 4
            for (int m = q; m < n; m += 8) sum = __fmaf_rn(__ldg(Ag + (size_t)k * ld + m), sres[m], sum);
          }
        }
        sum += __shfl_xor_sync(0xffffffffu, sum, 1);
        sum += __shfl_xor_sync(0xffffffffu, sum, 2);
        sum += __shfl_xor_sync(0xffffffffu, sum, 4);
        if (k < n && q == 0) { const int j = fdiv(k, L.mnx); L.p[j * L.pc + k - j * L.nx] = sum; }
      }
    } else {
      const LvS L = lvs_at(smem, lvo[nl - 1]);
      const int npair = (L.nx * L.ny + 1) >> 1;
      const int nthr = (npair + 31) & ~31;
      if ((int)threadIdx.x < nthr) {
        const CCell a = coarsest_cell(L, 2 * threadIdx.x), b = coarsest_cell(L, 2 * threadIdx.x + 1);
        if (a.act) L.p[a.kp] = 0.f;
        if (b.act) L.p[b.kp] = 0.f;
        // colour of cell 2t: (i + j) & 1
        const int k0 = 2 * threadIdx.x;
        const int j0 = fdiv(k0, L.mnx);
        const bool a_red = ((k0 - j0 * L.nx + j0) & 1) == 0;
        const CCell c0 = a_red ? a : b, c1 = a_red ? b : a;
        float* p = L.p;
        bar_coarsest(nthr);
        #pragma unroll 1
        for (int it = 0; it < 120; it++) {
          coarsest_update(p, L.pc, c0);
          bar_coarsest(nthr);
          coarsest_update(p, L.pc, c1);
          bar_coarsest(nthr);
        }
      }
    }
    __syncthreads();
}
// level l's visit on the way up: prolongation of level l + 1's p, then smoothing
__device__ __forceinline__ void cb_up(const CbCtx c, int l) {
  float* const smem = c.smem;
  const LvO* const lvo = c.lvo;
    const LvS F = lvs_at(smem, lvo[l]), Cc = lvs_at(smem, lvo[l + 1]);
    const LinMap mp(F.nx, F.mnx);
    if (mp.R)
    for (int j = mp.j0; j < F.ny; j += mp.R)
      for (int i = mp.i0; i < F.nx; i += mp.di(F.nx)) {
        const int I = i / 2, J = j / 2;
        const int I2 = min(max(I + ((i & 1) == 1 ? 1 : -1), 0), Cc.nx - 1);
        const int J2 = min(max(J + ((j & 1) == 1 ? 1 : -1), 0), Cc.ny - 1);
        const float c = 0.5625f * Cc.p[J * Cc.pc + I] + 0.1875f * (Cc.p[J * Cc.pc + I2] + Cc.p[J2 * Cc.pc + I]) +
                        0.0625f * Cc.p[J2 * Cc.pc + I2];
        F.p[j * F.pc + i] += F.rc[j * F.nx + i] > 0.f ? c : 0.f;
      }
    __syncthreads();
    smooth_visit(F, 1);
}
}  // namespace

// smem_floats: the launch's dynamic shared memory in floats; past the levels and the residual
// scratch, the coarsest inverse of the direct solve is staged there when it fits
// WT: compiled with the W tail (an engine whose scenes have one); without it the V-cycle's code alone
// L0: compiled with the level-0 ends of the cycle (an engine where some scene's block covers level 0)
template <bool WT, bool L0>
__global__ void __launch_bounds__(CB_THREADS) k_mg_coarse(const SceneDesc* __restrict__ scenes, int nscenes, SolveCtl* ctl, int tail,
                                                         int count_iter, int smem_floats) {
  extern __shared__ __align__(128) float smem[];
  __shared__ double red[32];
  __shared__ LvO lvo[MAX_LEVELS];
  __shared__ __align__(8) uint64_t bar;    // the coefficients (+ inverse)
  __shared__ int s_inv, s_res, s_A, s_dir, s_gpc;   // offsets: residual scratch, inverse
  __shared__ float* s_gp;                         // level lc's p in global memory
  const SceneDesc& S = scenes[blockIdx.x];
  pdl_trigger();
  const int lc = S.lc, nl = S.nlev;
  if (threadIdx.x == 0) {
    int q = 0;
    for (int l = lc; l < nl; l++) {
      const LevelDesc& G = S.lev[l];
      LvS v;
      v.nx = G.nx; v.h2 = G.h2; lvs_derive(v);
      LvO o;
      o.nx = G.nx; o.ny = G.ny; o.pc = G.pc; o.pu = G.pu; o.h2 = G.h2; o.rh2 = v.rh2; o.mnx = v.mnx; o.mhalf = v.mhalf;
      o.po = q; q += G.ny * G.pc;
      o.ro = q; q += G.ny * G.pc;
      o.ao = q; q += G.ny * G.pu;
      o.yo = q; q += (G.ny + 1) * G.pc;
      lvo[l] = o;
    }
    s_res = q;
    const int nres = S.lev[lc].ny * S.lev[lc].pc;   // the largest level's pitched size
    q += round_up(nres > COARSEST_SCRATCH ? nres : COARSEST_SCRATCH, 32);   // residual scratch
    for (int l = lc; l < nl; l++) { lvo[l].to = q; q += S.lev[l].nx * S.lev[l].ny; }
    q = round_up(q, 32);
    s_A = q;
    s_gp = S.lev[lc].p; s_gpc = S.lev[lc].pc;
    mbar_init(&bar, 1);
  }
  __syncthreads();
  // ---- stage the arrays. The coefficients are built before the pressure loop and no loop
  // kernel writes them; the direct solve's inverse (the half cinv_cur of S.cinv) is factored
  // before the loop or, pipelined, during the previous step (this step's side branch writes
  // the other half). Both arrive by TMA bulk copies (sizes multiples of 16 bytes; the
  // inverse when it fits, n even) before the wait on the previous kernel, and the reciprocal
  // of each cell's diagonal (pressure.wgsl:77-86; 0 marks a closed cell) is tabled then too,
  // beside the previous kernel. After the wait only level lc's rhs (and p when lc = 0) is
  // read, with plain loads from L2.
  const bool on = S.enabled;   // host-written, constant during the step
  const volatile int* act = &S.solve->active;
  if (threadIdx.x == 0) {
    s_inv = 0;
    s_dir = 0;
    if (on) {
      uint32_t bytes = 0;
      for (int l = lc; l < nl; l++) bytes += (S.lev[l].ny * S.lev[l].pu + (S.lev[l].ny + 1) * S.lev[l].pc) * 4;
      const int n = S.lev[nl - 1].nx * S.lev[nl - 1].ny;
      s_dir = ctl->coarse_direct && S.solve->direct_ok;   // both fixed for the loop
      const int ld = cinv_ld(n);
      const bool inv = s_dir && (n % 2) == 0 && n <= kStagedInverseMax && s_A + n * ld <= smem_floats;
      if (inv) bytes += (uint32_t)(n * ld * 4);
      mbar_arrive_expect_tx(&bar, bytes);
      for (int l = lc; l < nl; l++) {
        const LevelDesc& G = S.lev[l];
        bulk_g2s(smem + lvo[l].ao, G.ax, G.ny * G.pu * 4, &bar);
        bulk_g2s(smem + lvo[l].yo, G.ay, (G.ny + 1) * G.pc * 4, &bar);
      }
      if (inv) {
        bulk_g2s(smem + s_A, S.cinv + (size_t)S.solve->cinv_cur * n * ld, (uint32_t)(n * ld * 4), &bar);
        s_inv = 1;
      }
    }
  }
  const LvS V0 = lvs_at(smem, lvo[lc]);
  const float* grhs = S.lev[lc].rhs;
  bool okc = true;
  if (on) {
    okc = mbar_wait(&bar, 0);
    if (okc)
      for (int l = lc; l < nl; l++) {
        const LvS L = lvs_at(smem, lvo[l]);
        float* rc = smem + lvo[l].to;
        for (int e = threadIdx.x; e < L.nx * L.ny; e += CB_THREADS) {
          const int j = fdiv(e, L.mnx), i = e - j * L.nx;
          const float d = diag_d(L, i, j);
          rc[e] = d > 0.f ? __frcp_rn(d) : 0.f;
        }
      }
    // level lc's p is zero after the restriction into it (pressure.wgsl:112)
    if (lc > 0)
      for (int e = threadIdx.x; e < V0.ny * V0.pc; e += CB_THREADS) V0.p[e] = 0.f;
  }
  pdl_wait();
  if (count_iter && blockIdx.x == 0 && threadIdx.x == 0) loop_count(ctl);
  if (!on) return;
  if (__syncthreads_or(!okc)) {
    // the copies did not land in time: record it and leave once they have (bounded)
    if (threadIdx.x == 0) atomicExch(&ctl->err, 1);
    mbar_wait(&bar, 0);
    return;
  }
  // the scene's flag and level lc's rhs are read together (two L2 round trips overlapped): the
  // loads land in shared memory whether or not the scene still cycles, then every thread leaves
  // together if it does not
  const int still = *act;
  float* sres = smem + s_res;   // residual scratch (level lc size)
  for (int e = threadIdx.x; e < V0.ny * V0.pc; e += CB_THREADS) V0.rhs[e] = __ldcg(grhs + e);
  if (L0 && lc == 0)   // warm start
    for (int e = threadIdx.x; e < V0.ny * V0.pc; e += CB_THREADS) V0.p[e] = __ldcg(s_gp + e);
  if (still == 0) return;
  __syncthreads();
  const CbCtx cbx{smem, lvo, sres, &S, nl, s_dir, s_inv, s_A};
  // The cycle over levels lc..nl-1: the V(2,2) cycle of js/fluid.js:294-312, straight down, the
  // coarsest, straight up. With the W tail (S.lw = nl - 3) level nl - 3 visits level nl - 2
  // twice: after the first visit has come back up through level nl - 2, that level is smoothed
  // from its p and restricted again (its rhs stays) and the coarsest solved again. Straight-line
  // code: the visits keep their registers to themselves.
  for (int l = lc; l < nl - 1; l++) cb_down(cbx, l);
  cb_coarsest(cbx);
  if (WT && S.lw == nl - 3 && nl - 3 >= lc) {
    cb_up(cbx, nl - 2);
    cb_down(cbx, nl - 2);
    cb_coarsest(cbx);
  }
  for (int l = nl - 2; l >= lc; l--) cb_up(cbx, l);
  // ---- write level lc back; when the block covers level 0, finish the cycle here
  float* const gp = s_gp;
  const int gpc = s_gpc, gnx = V0.nx;
  if (!L0 || lc > 0) {
    // the shared copy of level lc's p has the global pitch: one bulk copy (the last visit ended
    // with a block barrier); the next kernel reads it after this grid has completed
    if (threadIdx.x == 0) {
      proxy_fence_shared();
      bulk_s2g(gp, V0.p, (uint32_t)(V0.ny * gpc * 4));
      bulk_wait_read();
    }
    return;
  }
  double part = 0.0, part2 = 0.0, part3 = 0.0;
  const LinMap mw(V0.nx, V0.mnx);
  if (mw.R)
  for (int j = mw.j0; j < V0.ny; j += mw.R)
    for (int i = mw.i0; i < V0.nx; i += mw.di(V0.nx)) {
      const int e = j * V0.pc + i;
      gp[j * gpc + i] = V0.p[e];
      if (lc == 0 && tail == 1) {
        float off, diag; stencil_d(V0, i, j, off, diag);
        const double r = diag <= 0.f ? 0.0 : (double)(V0.rhs[e] - (off - diag * V0.p[e]) / V0.h2);
        part += r * r;
      } else if (lc == 0 && tail == 2) {
        S.p64[j * gnx + i] += (double)V0.p[e];
      } else if (lc == 0 && tail == 3) {
        const double z = (double)V0.p[e];
        const double lz = lap_block64(V0, i, j);
        S.dB[j * gnx + i] = lz;
        part += S.r64[j * gnx + i] * z;
        part2 += S.q64[j * gnx + i] * z;
        part3 += z * lz;
      }
    }
  if (lc == 0 && tail == 1) {
    const double t = block_sum(part, red);
    if (threadIdx.x == 0) solve_decide(ctl, S.solve, t, true);
  } else if (lc == 0 && tail == 3) {
    const double ta = block_sum(part, red);
    const double tb = block_sum(part2, red);
    const double tz = block_sum(part3, red);
    if (threadIdx.x == 0) pcg_coef(S, ta, tb, tz);
  }
}

// ------------------------------------------------------------------ direct coarse solve: the coarsest inverse
// The coarsest operator A (A_kk = the stencil's diagonal, A_km = -face coefficient;
// a closed cell gets the row dmax e_k) is symmetric with half-bandwidth nx in
// row-major cell order. Once per step: banded Cholesky A = L L^T (right-looking,
// one warp: per column jc, L_jcjc = sqrt(a_jcjc), L_ijc = a_ijc / L_jcjc, then
// a_ik = fma(-L_ijc, L_kjc, a_ik) for jc < k <= i <= jc + nx), then column c of
// A^-1 by forward and back substitution on thread c (y_i = (e_ic - sum L_ik y_k) *
// (1/L_ii) with k ascending, then x_i = (y_i - sum L_ki x_k) * (1/L_ii), k ascending).
// A pivot a_jcjc <= 1e-6 dmax (a sealed gas pocket: singular) or a level wider than
// CF_MAXBW cells leaves direct_ok = 0, and the coarse block keeps the 120 sweeps.
namespace {
constexpr int CF_THREADS = 256;   // the coarsest level has at most 256 cells
constexpr int CF_MAXBW = 32;
constexpr size_t CF_SMEM_BUDGET = 200 * 1024;
}

// Columns of the inverse solved per pass: all n when the working columns fit the
// shared-memory budget beside the band, else 128 per pass.
__host__ __device__ inline int coarse_factor_cols(int n) {
  const size_t W = CF_MAXBW + 1;   // the widest band
  return ((size_t)n * n + (size_t)n * W + n) * sizeof(float) <= CF_SMEM_BUDGET ? n : 128;
}
size_t coarse_factor_smem(int n, int bw) {
  const int C = coarse_factor_cols(n);
  return ((size_t)n * (bw + 1) + n + (size_t)n * C) * sizeof(float);
}

// The inverse of the coarsest operator of each scene: the banded matrix is
// factored L L^T by one warp (right-looking; lane l owns row jc + 1 + l of the
// trailing band, takes the new column's l_kj from the lanes that computed them
// by shuffle and updates its row from registers), then each thread solves
// L L^T x = e_c for its column c with the band's sliding window in registers
// (BWM = the band width bound, a compile-time size so the window stays in
// registers); the forward result is kept in shared memory (Y[i * C + t]).
// pipelined = 0: the inverse of this step's operator into the half the cycles use (direct_ok);
// pipelined = 1: into the other half for the next step (direct_ok_next), while this step's
// cycles use the current half.
template <int BWM>
__global__ void __launch_bounds__(CF_THREADS) k_coarse_factor(const SceneDesc* __restrict__ scenes, int pipelined) {
  extern __shared__ float cf_smem[];
  __shared__ float s_dmax;
  __shared__ int s_ok;
  const SceneDesc& S = scenes[blockIdx.x];
  if (!S.enabled) return;
  const LevelDesc L = S.lev[S.nlev - 1];
  const int n = L.nx * L.ny, bw = L.nx, W = bw + 1;
  int* ok_flag = pipelined ? &S.solve->direct_ok_next : &S.solve->direct_ok;
  const int ld = cinv_ld(n);
  float* cinv = S.cinv + (size_t)(pipelined ? 1 - S.solve->cinv_cur : S.solve->cinv_cur) * n * ld;
  if (n > CF_THREADS || bw > BWM) {
    if (threadIdx.x == 0) *ok_flag = 0;
    return;
  }
  float* band = cf_smem;                 // n * W
  float* rinv = band + (size_t)n * W;    // n
  float* Y = rinv + n;                   // n * C
  const int C = coarse_factor_cols(n);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < n * W; e += CF_THREADS) band[e] = 0.f;
  __syncthreads();
  // lower band: band[k*W + d] = A[k][k-d]; the diagonal is kept in rinv[] until dmax is known
  for (int k = tid; k < n; k += CF_THREADS) {
    const int i = k % L.nx, j = k / L.nx;
    const float w = L.ax[j * L.pu + i], e = L.ax[j * L.pu + i + 1];
    const float so = L.ay[j * L.pc + i], no = L.ay[(j + 1) * L.pc + i];
    float diag = 0.f;
    if (i > 0) diag += w; else diag += 2.f * w;
    if (i < L.nx - 1) diag += e; else diag += 2.f * e;
    if (j > 0) diag += so;
    if (j < L.ny - 1) diag += no; else diag += 2.f * no;
    rinv[k] = diag;
    if (diag > 0.f) {
      band[k * W] = diag;
      if (i > 0) band[k * W + 1] = -w;
      if (j > 0) band[k * W + bw] = -so;
    }
  }
  __syncthreads();
  if (tid == 0) {
    float m = 0.f;
    for (int k = 0; k < n; k++) m = fmaxf(m, rinv[k]);
    s_dmax = m;
    s_ok = m > 0.f ? 1 : 0;
  }
  __syncthreads();
  const float dmax = s_dmax, thr = 1e-6f * dmax;
  for (int k = tid; k < n; k += CF_THREADS)
    if (!(rinv[k] > 0.f)) band[k * W] = dmax;
  __syncthreads();
  if (warp == 0 && s_ok) {
    for (int jc = 0; jc < n; jc++) {
      const float piv = band[jc * W];
      if (!(piv > thr)) {   // every lane read the same pivot
        if (lane == 0) s_ok = 0;
        break;
      }
      const float ljj = sqrtf(piv);
      const int i = jc + 1 + lane;
      const bool mine = lane < bw && i < n;
      float lij = 0.f;
      if (mine) lij = band[i * W + (i - jc)] / ljj;
      // A[i][k] -= l_ij l_kj for k = jc + 1 + m <= i: l_kj from lane m, A[i][k] at band[i*W + lane - m]
      float lk[BWM], tg[BWM];
#pragma unroll
      for (int m = 0; m < BWM; m++) lk[m] = __shfl_sync(0xffffffffu, lij, m);
#pragma unroll
      for (int m = 0; m < BWM; m++) tg[m] = (mine && m <= lane) ? band[i * W + (lane - m)] : 0.f;
      __syncwarp();
      if (lane == 0) band[jc * W] = ljj;
      if (mine) band[i * W + (i - jc)] = lij;
#pragma unroll
      for (int m = 0; m < BWM; m++)
        if (mine && m <= lane) band[i * W + (lane - m)] = __fmaf_rn(-lij, lk[m], tg[m]);
      __syncwarp();
    }
  }
  __syncthreads();
  if (!s_ok) {
    if (tid == 0) *ok_flag = 0;
    return;
  }
  for (int k = tid; k < n; k += CF_THREADS) rinv[k] = 1.0f / band[k * W];
  __syncthreads();
  for (int c0 = 0; c0 < n; c0 += C) {
    const int t = tid, c = c0 + tid;
    if (t < C && c < n) {
      float* y = Y + t;   // y[i * C]
      for (int i = 0; i < c; i++) y[i * C] = 0.f;
      // forward: y_i = (e_c[i] - sum_{k = max(c, i-bw)}^{i-1} L[i][k] y_k) / L[i][i], k ascending;
      // win[m] = y_{i-1-m}
      float win[BWM];
#pragma unroll
      for (int m = 0; m < BWM; m++) win[m] = 0.f;
      for (int i = c; i < n; i++) {
        float sum = i == c ? 1.f : 0.f;
#pragma unroll
        for (int m = BWM - 1; m >= 0; m--)
          if (m < bw && i - 1 - m >= c) sum = __fmaf_rn(-band[i * W + (m + 1)], win[m], sum);
        const float yi = sum * rinv[i];
        y[i * C] = yi;
#pragma unroll
        for (int m = BWM - 1; m > 0; m--) win[m] = win[m - 1];
        win[0] = yi;
      }
      // backward: x_i = (y_i - sum_{k = i+1}^{min(n-1, i+bw)} L[k][i] x_k) / L[i][i], k ascending;
      // win[m] = x_{i+1+m}
#pragma unroll
      for (int m = 0; m < BWM; m++) win[m] = 0.f;
      for (int i = n - 1; i >= 0; i--) {
        float sum = y[i * C];
#pragma unroll
        for (int m = 0; m < BWM; m++)
          if (m < bw && i + 1 + m <= n - 1) sum = __fmaf_rn(-band[(i + 1 + m) * W + (m + 1)], win[m], sum);
        const float xi = sum * rinv[i];
        cinv[(size_t)i * ld + c] = xi;
#pragma unroll
        for (int m = BWM - 1; m > 0; m--) win[m] = win[m - 1];
        win[0] = xi;
      }
    }
    __syncthreads();
  }
  if (tid == 0) *ok_flag = 1;
}

// Pipelined coarse solve, after the step's pressure loop and the factorisation have both
// finished: the next step's cycles use the inverse just factored.
__global__ void k_cinv_swap(const SceneDesc* __restrict__ scenes, int nscenes) {
  for (int s = threadIdx.x; s < nscenes; s += blockDim.x) {
    const SceneDesc& S = scenes[s];
    if (!S.enabled) continue;
    SolveState* ss = S.solve;
    ss->cinv_cur ^= 1;
    ss->direct_ok = ss->direct_ok_next;
    ss->direct_ok_next = 0;
  }
}

// shared bytes of the coarse block for one scene (the layout built by k_mg_coarse)
size_t coarse_smem_bytes(const int* lnx, const int* lny, int lc, int nlev) {
  size_t f = 0;
  for (int l = lc; l < nlev; l++) {
    const size_t pc = (size_t)round_up(lnx[l], 32), pu = (size_t)round_up(lnx[l] + 1, 32);
    f += 2 * lny[l] * pc + lny[l] * pu + (lny[l] + 1) * pc;
  }
  f += (size_t)round_up(std::max(round_up(lnx[lc], 32) * lny[lc], COARSEST_SCRATCH), 32);
  size_t cells = 0;   // the 1/diag table of every level
  for (int l = lc; l < nlev; l++) cells += (size_t)lnx[l] * lny[l];
  f += (size_t)round_up((int)cells, 32);
  // room for the coarsest inverse of the direct solve when it fits
  const size_t n = (size_t)lnx[nlev - 1] * lny[nlev - 1];
  const size_t ld = (size_t)cinv_ld((int)n);
  if (n % 2 == 0 && n <= (size_t)kStagedInverseMax && (f + n * ld) * 4 <= kCoarseSmemMax) f += n * ld;
  return f * 4;
}

using UpKernel = void (*)(const SceneDesc*, int, const Work*, int, SolveCtl*);
template <bool ONE>
static UpKernel up_kernel(int tail) {
  switch (tail) {
    case 1: return k_mg_up<MGF_TX, MGF_TY, 1, ONE>;
    case 2: return k_mg_up<MGF_TX, MGF_TY, 2, ONE>;
    case 3: return k_mg_up<MGF_TX, MGF_TY, 3, ONE>;
    case 4: return k_mg_up<MGF_TX, MGF_TY, 4, ONE>;
    default: return k_mg_up<MGF_TX, MGF_TY, 0, ONE>;
  }
}
// whether `ntiles` CTAs fit in one wave at two per SM (this process's device)
static bool one_wave_at_two(int ntiles) {
  static const int sms = [] {
    int d = 0, n = 0;
    if (cudaGetDevice(&d) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, d) != cudaSuccess)
      n = 0;
    return n;
  }();
  return ntiles <= 2 * sms;
}
void launch_mg_down(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, int level, SolveCtl* ctl,
                    int count_iter, int pcg, cudaStream_t st) {
  if (ntiles <= 0) return;
  const auto k = nscenes == 1
                     ? (pcg ? (one_wave_at_two(ntiles) ? k_mg_down<MGF_TX, MGF_TY, true, true, 2>
                                                       : k_mg_down<MGF_TX, MGF_TY, true, true>)
                            : k_mg_down<MGF_TX, MGF_TY, false, true>)
                     : (pcg ? k_mg_down<MGF_TX, MGF_TY, true, false> : k_mg_down<MGF_TX, MGF_TY, false, false>);
  launch_pdl(pdl_enabled(), k, dim3(ntiles), dim3(256), 0, st, scenes, nscenes, work, level, ctl, count_iter);
}
void launch_mg_up(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, int level, int tail, SolveCtl* ctl,
                  cudaStream_t st) {
  if (ntiles <= 0) return;
  const UpKernel k = nscenes != 1 ? up_kernel<false>(tail)
                     : tail == 4 && one_wave_at_two(ntiles) ? k_mg_up<MGF_TX, MGF_TY, 4, true, 2>
                                                            : up_kernel<true>(tail);
  launch_pdl(pdl_enabled(), k, dim3(ntiles), dim3(256), 0, st, scenes, nscenes, work, level, ctl);
}
void launch_pcg_decide(const SceneDesc* scenes, int nscenes, SolveCtl* ctl, cudaStream_t st) {
  if (nscenes > 0) launch_pdl(pdl_enabled(), k_pcg_decide, dim3(nscenes), dim3(256), 0, st, scenes, ctl);
}
void launch_mg_coarse(const SceneDesc* scenes, int nscenes, SolveCtl* ctl, int tail, int count_iter, size_t smem,
                      int wtail, int level0, cudaStream_t st) {
  if (nscenes > 0)
    launch_pdl(pdl_enabled(),
               wtail ? (level0 ? k_mg_coarse<true, true> : k_mg_coarse<true, false>)
                     : (level0 ? k_mg_coarse<false, true> : k_mg_coarse<false, false>),
               dim3(nscenes), dim3(CB_THREADS), smem, st, scenes, nscenes, ctl, tail, count_iter, (int)(smem / 4));
}
// bw: the widest coarsest level of the batch (the register window's bound)
void launch_coarse_factor(const SceneDesc* scenes, int nscenes, size_t smem, int bw, int pipelined, cudaStream_t st) {
  if (nscenes <= 0) return;
  if (bw <= 8) k_coarse_factor<8><<<nscenes, CF_THREADS, smem, st>>>(scenes, pipelined);
  else if (bw <= 16) k_coarse_factor<16><<<nscenes, CF_THREADS, smem, st>>>(scenes, pipelined);
  else k_coarse_factor<32><<<nscenes, CF_THREADS, smem, st>>>(scenes, pipelined);
}
void launch_cinv_swap(const SceneDesc* scenes, int nscenes, cudaStream_t st) {
  if (nscenes > 0) k_cinv_swap<<<1, 128, 0, st>>>(scenes, nscenes);
}
// The attribute belongs to the kernel, not to an engine: it is set to the largest size any
// coarsest level can ask for, so engines of different sizes never lower it under each other.
cudaError_t prepare_coarse_factor(size_t smem) {
  const int cap = (int)std::max(smem, CF_SMEM_BUDGET);   // every level that fits: the columns' budget bounds it
  cudaError_t e = cudaFuncSetAttribute(k_coarse_factor<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_coarse_factor<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_coarse_factor<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, cap);
  return e;
}
cudaError_t prepare_mg_coarse(size_t smem) {
  // the kernel's attribute, shared by every engine: the largest size any schedule can ask for
  const int bytes = (int)std::max(smem, kCoarseSmemMax);
  cudaError_t e = cudaFuncSetAttribute(k_mg_coarse<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mg_coarse<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mg_coarse<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_mg_coarse<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  return e;
}

}  // namespace cfg
