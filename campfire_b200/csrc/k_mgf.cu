// Fused multigrid V(2,2) cycle of shaders/pressure.wgsl (schedule of
// js/fluid.js:294-312) with temporal blocking.
//
// Each fine level l < lc is handled by two kernels per cycle:
//   down: load p, rhs, ax, ay on the tile plus a 5-cell halo into shared
//         memory, run the 4 colour passes (red, black, red, black), each one
//         cell narrower than the last, then the residual of the tile's cells
//         and its restriction to the coarse rhs (coarse p = 0);
//   up:   the same halo load, bilinear prolongation of the coarse correction,
//         4 colour passes (black, red, black, red); on level 0 also the
//         residual norm (FP32 modes) or p64 += p (FP64 defect correction).
// A cell update reads exactly the neighbour values the separate dispatches
// would read, so the result equals the reference schedule bit for bit.
// Down kernels read p and write pb; up kernels read pb and write p, so no CTA
// reads a halo another CTA is rewriting.
// Levels lc..coarsest run in one CTA per scene (coarse block): every level's
// arrays staged into shared memory by TMA bulk copies, __syncthreads between
// passes, and the coarsest level's 120 red-black sweeps (pressure.wgsl:132-156)
// on 256 threads (one cell each) with a named barrier.
#include "gas_dev.cuh"
#include "kernels.h"
#include "reduce.cuh"
#include "tma.cuh"

#include <algorithm>

namespace cfg {

namespace {

constexpr int H_DOWN = 5;   // 4 passes + the residual's neighbours
constexpr int H_UP = 5;     // 4 passes + the level-0 residual's neighbours

struct Tile {
  // shared arrays of a (RW x RH) cell region at origin (rx0, ry0)
  float *p, *rhs, *ax, *ay;
  int RW, RH, rx0, ry0;
  __device__ __forceinline__ int c(int i, int j) const { return (j - ry0) * RW + (i - rx0); }
  __device__ __forceinline__ int u(int i, int j) const { return (j - ry0) * (RW + 1) + (i - rx0); }
};

// pressure.wgsl:77-85 on the shared tile (i, j in level coordinates)
__device__ __forceinline__ void stencil_s(const Tile& t, int nx, int ny, int i, int j, float& off, float& diag) {
  off = 0.f; diag = 0.f;
  const int k = t.c(i, j), ku = t.u(i, j);
  const float w = t.ax[ku], e = t.ax[ku + 1], s = t.ay[k], n = t.ay[k + t.RW];
  if (i > 0) { off += w * t.p[k - 1]; diag += w; } else { diag += 2.f * w; }
  if (i < nx - 1) { off += e * t.p[k + 1]; diag += e; } else { diag += 2.f * e; }
  if (j > 0) { off += s * t.p[k - t.RW]; diag += s; }
  if (j < ny - 1) { off += n * t.p[k + t.RW]; diag += n; } else { diag += 2.f * n; }
}
__device__ __forceinline__ float diag_s(const Tile& t, int nx, int ny, int i, int j) {
  const int k = t.c(i, j), ku = t.u(i, j);
  const float w = t.ax[ku], e = t.ax[ku + 1], s = t.ay[k], n = t.ay[k + t.RW];
  float diag = 0.f;
  if (i > 0) diag += w; else diag += 2.f * w;
  if (i < nx - 1) diag += e; else diag += 2.f * e;
  if (j > 0) diag += s;
  if (j < ny - 1) diag += n; else diag += 2.f * n;
  return diag;
}

// load p (from src), rhs, ax, ay of the region, clipped to the level
__device__ __forceinline__ void load_tile(const Tile& t, const LevelDesc& L, const float* src) {
  const int RW = t.RW, RH = t.RH;
  for (int e = threadIdx.x; e < RH * RW; e += blockDim.x) {
    const int i = t.rx0 + e % RW, j = t.ry0 + e / RW;
    if (i < 0 || i >= L.nx || j < 0 || j >= L.ny) continue;
    t.p[e] = src[j * L.pc + i];
    t.rhs[e] = __ldg(L.rhs + j * L.pc + i);
  }
  for (int e = threadIdx.x; e < RH * (RW + 1); e += blockDim.x) {
    const int i = t.rx0 + e % (RW + 1), j = t.ry0 + e / (RW + 1);
    if (i < 0 || i > L.nx || j < 0 || j >= L.ny) continue;
    t.ax[e] = __ldg(L.ax + j * L.pu + i);
  }
  for (int e = threadIdx.x; e < (RH + 1) * RW; e += blockDim.x) {
    const int i = t.rx0 + e % RW, j = t.ry0 + e / RW;
    if (i < 0 || i >= L.nx || j < 0 || j > L.ny) continue;
    t.ay[e] = __ldg(L.ay + j * L.pc + i);
  }
}

// one red-black colour pass (pressure.wgsl:87-94) over cells [xa,xb) x [ya,yb) of colour
// `color`: warps take rows, lanes every other cell (the region is at most 64 cells wide)
__device__ __forceinline__ void colour_pass(const Tile& t, const LevelDesc& L, int xa, int xb, int ya, int yb, int color) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j = ya + warp; j < yb; j += nw) {
    const int i = xa + ((xa + j + color) & 1) + 2 * lane;
    if (i >= xb) continue;
    float off, diag; stencil_s(t, L.nx, L.ny, i, j, off, diag);
    const int k = t.c(i, j);
    t.p[k] = diag > 0.f ? (off - t.rhs[k] * L.h2) / diag : 0.f;
  }
}

__device__ __forceinline__ bool scene_live(const SceneDesc& S) { return S.enabled && S.solve->active; }

}  // namespace

// ------------------------------------------------------------------ down: 4 passes + restrict
template <int TX, int TY>
__global__ void __launch_bounds__(256) k_mg_down(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work, int level) {
  constexpr int RW = TX + 2 * H_DOWN, RH = TY + 2 * H_DOWN;
  __shared__ float sp[RH * RW], srhs[RH * RW], sax[RH * (RW + 1)], say[(RH + 1) * RW];
  __shared__ float sr[TY * TX];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!scene_live(S)) return;
  const LevelDesc L = S.lev[level], C = S.lev[level + 1];
  const int x0 = w.tx * TX, y0 = w.ty * TY;
  const Tile t{sp, srhs, sax, say, RW, RH, x0 - H_DOWN, y0 - H_DOWN};
  load_tile(t, L, L.p);
  __syncthreads();
  #pragma unroll 1
  for (int k = 1; k <= 4; k++) {   // colours 0, 1, 0, 1 (js/fluid.js:298-301)
    colour_pass(t, L, max(x0 - H_DOWN + k, 0), min(x0 + TX + H_DOWN - k, L.nx), max(y0 - H_DOWN + k, 0),
                min(y0 + TY + H_DOWN - k, L.ny), (k - 1) & 1);
    __syncthreads();
  }
  // residual of the tile cells (pressure.wgsl:96-101) and the smoothed p
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    const int i = x0 + e % TX, j = y0 + e / TX;
    if (i >= L.nx || j >= L.ny) continue;
    float off, diag; stencil_s(t, L.nx, L.ny, i, j, off, diag);
    const int k = t.c(i, j);
    sr[e] = diag <= 0.f ? 0.f : t.rhs[k] - (off - diag * t.p[k]) / L.h2;
    L.pb[j * L.pc + i] = t.p[k];
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
// tail: 0 none, 1 residual norm + loop decision (FP32 modes), 2 p64 += p (FP64 defect correction)
template <int TX, int TY>
__global__ void __launch_bounds__(256) k_mg_up(const SceneDesc* __restrict__ scenes, int nscenes, const Work* __restrict__ work,
                                               int level, int tail, SolveCtl* ctl);

namespace {
__device__ void solve_decide_f(const SceneDesc* scenes, int nscenes, const SceneDesc& S, SolveCtl* ctl, double r2) {
  SolveState* ss = S.solve;
  ss->cycles += 1;
  ss->rnorm2 = r2;
  const double b2 = ss->bnorm2;
  const double rel = b2 > 0.0 ? sqrt(r2 / b2) : 0.0;
  ss->rel = rel;
  const int act = ctl->mode == CFG_SOLVE_FIXED ? (ss->cycles < ctl->ncycles)
                                               : ((rel > ctl->tol) && (ss->cycles < ctl->max_cycles));
  ss->active = act;
  __threadfence();
  const unsigned d = atomicAdd(&ctl->scenes_done, 1u);
  if (d == (unsigned)ctl->nactive - 1u) {
    __threadfence();
    int na = 0;
    for (int s = 0; s < nscenes; s++)
      if (scenes[s].enabled && *((volatile int*)&scenes[s].solve->active)) na++;
    ctl->scenes_done = 0u;
    ctl->nactive = na;
    ctl->any_active = na > 0 ? 1 : 0;
  }
}
}  // namespace

template <int TX, int TY>
__global__ void __launch_bounds__(256) k_mg_up(const SceneDesc* __restrict__ scenes, int nscenes, const Work* __restrict__ work,
                                               int level, int tail, SolveCtl* ctl) {
  constexpr int RW = TX + 2 * H_UP, RH = TY + 2 * H_UP;
  __shared__ float sp[RH * RW], srhs[RH * RW], sax[RH * (RW + 1)], say[(RH + 1) * RW];
  __shared__ double red[32];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!scene_live(S)) return;
  const LevelDesc L = S.lev[level], C = S.lev[level + 1];
  const int x0 = w.tx * TX, y0 = w.ty * TY;
  const Tile t{sp, srhs, sax, say, RW, RH, x0 - H_UP, y0 - H_UP};
  load_tile(t, L, L.pb);
  __syncthreads();
  // prolongation (pressure.wgsl:116-129) on the whole region
  for (int e = threadIdx.x; e < RH * RW; e += blockDim.x) {
    const int i = t.rx0 + e % RW, j = t.ry0 + e / RW;
    if (i < 0 || i >= L.nx || j < 0 || j >= L.ny) continue;
    const int I = i / 2, J = j / 2;
    const int I2 = min(max(I + ((i & 1) == 1 ? 1 : -1), 0), C.nx - 1);
    const int J2 = min(max(J + ((j & 1) == 1 ? 1 : -1), 0), C.ny - 1);
    const float* cp = C.p;
    const float c = 0.5625f * cp[J * C.pc + I] + 0.1875f * (cp[J * C.pc + I2] + cp[J2 * C.pc + I]) + 0.0625f * cp[J2 * C.pc + I2];
    t.p[e] += diag_s(t, L.nx, L.ny, i, j) > 0.f ? c : 0.f;
  }
  __syncthreads();
  #pragma unroll 1
  for (int k = 1; k <= 4; k++) {   // colours 1, 0, 1, 0 (js/fluid.js:307-310)
    colour_pass(t, L, max(x0 - H_UP + k, 0), min(x0 + TX + H_UP - k, L.nx), max(y0 - H_UP + k, 0),
                min(y0 + TY + H_UP - k, L.ny), k & 1);
    __syncthreads();
  }
  double part = 0.0;
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
    }
  }
  if (tail != 1) return;
  const double bp = block_sum(part, red);
  double total = 0.0;
  if (scene_reduce(S, w.tile, S.nt_up0, bp, red, &total) && threadIdx.x == 0)
    solve_decide_f(scenes, nscenes, S, ctl, total);
}

// ------------------------------------------------------------------ coarse block: levels lc..coarsest in one CTA
// Shared memory holds every level >= lc with the global row pitches (pc for p,
// rhs, ay; pu for ax), so each array arrives by one TMA bulk copy; then a
// residual scratch of level lc's size.
namespace {
constexpr int CB_THREADS = 1024;
constexpr int CB_WARPS = CB_THREADS / 32;
constexpr int COARSEST_THREADS = 256;   // the coarsest level has at most 256 cells
constexpr int COARSEST_SCRATCH = 0;     // the coarsest keeps its stencils in registers

struct LvS { float *p, *rhs, *ax, *ay; int nx, ny, pc, pu; float h2; int pad; };

__device__ __forceinline__ void stencil_d(const LvS& L, int i, int j, float& off, float& diag) {
  off = 0.f; diag = 0.f;
  const float w = L.ax[j * L.pu + i], e = L.ax[j * L.pu + i + 1];
  const float s = L.ay[j * L.pc + i], n = L.ay[(j + 1) * L.pc + i];
  const float* p = L.p;
  if (i > 0) { off += w * p[j * L.pc + i - 1]; diag += w; } else { diag += 2.f * w; }
  if (i < L.nx - 1) { off += e * p[j * L.pc + i + 1]; diag += e; } else { diag += 2.f * e; }
  if (j > 0) { off += s * p[(j - 1) * L.pc + i]; diag += s; }
  if (j < L.ny - 1) { off += n * p[(j + 1) * L.pc + i]; diag += n; } else { diag += 2.f * n; }
}
// one colour pass: warps take rows, lanes take every other cell of the row
__device__ __forceinline__ void pass_d(const LvS& L, int color) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int j = warp; j < L.ny; j += CB_WARPS)
    for (int i = 2 * lane + ((j + color) & 1); i < L.nx; i += 64) {
      float off, diag; stencil_d(L, i, j, off, diag);
      const int k = j * L.pc + i;
      L.p[k] = diag > 0.f ? (off - L.rhs[k] * L.h2) / diag : 0.f;
    }
}
__device__ __forceinline__ void bar_coarsest() { asm volatile("bar.sync 1, %0;" ::"r"(COARSEST_THREADS) : "memory"); }
}  // namespace

__global__ void __launch_bounds__(CB_THREADS) k_mg_coarse(const SceneDesc* __restrict__ scenes, int nscenes, SolveCtl* ctl, int tail) {
  extern __shared__ __align__(128) float smem[];
  __shared__ double red[32];
  __shared__ LvS lv[MAX_LEVELS];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  const SceneDesc& S = scenes[blockIdx.x];
  if (!scene_live(S)) return;
  const int lc = S.lc, nl = S.nlev;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    float* q = smem;
    for (int l = lc; l < nl; l++) {
      const LevelDesc& G = S.lev[l];
      LvS v;
      v.nx = G.nx; v.ny = G.ny; v.pc = G.pc; v.pu = G.pu; v.h2 = G.h2; v.pad = 0;
      v.p = q; q += G.ny * G.pc;
      v.rhs = q; q += G.ny * G.pc;
      v.ax = q; q += G.ny * G.pu;
      v.ay = q; q += (G.ny + 1) * G.pc;
      lv[l] = v;
    }
    mbar_init(&bar, 1);
  }
  __syncthreads();
  const LvS V0 = lv[lc];
  float* sres = lv[nl - 1].ay + (lv[nl - 1].ny + 1) * lv[nl - 1].pc;   // residual scratch (level lc size)
  // ---- stage the arrays with TMA bulk copies (one per array; sizes are multiples of 128 bytes)
  if (threadIdx.x == 0) {
    uint32_t bytes = 0;
    const LevelDesc& G0 = S.lev[lc];
    bytes += G0.ny * G0.pc * 4 * (lc == 0 ? 2 : 1);
    for (int l = lc; l < nl; l++) bytes += (S.lev[l].ny * S.lev[l].pu + (S.lev[l].ny + 1) * S.lev[l].pc) * 4;
    mbar_arrive_expect_tx(&bar, bytes);
    bulk_g2s(V0.rhs, G0.rhs, G0.ny * G0.pc * 4, &bar);
    if (lc == 0) bulk_g2s(V0.p, G0.p, G0.ny * G0.pc * 4, &bar);   // warm start
    for (int l = lc; l < nl; l++) {
      const LevelDesc& G = S.lev[l];
      bulk_g2s(lv[l].ax, G.ax, G.ny * G.pu * 4, &bar);
      bulk_g2s(lv[l].ay, G.ay, (G.ny + 1) * G.pc * 4, &bar);
    }
  }
  // level lc's p is zero after the restriction into it (pressure.wgsl:112)
  if (lc > 0)
    for (int e = threadIdx.x; e < V0.ny * V0.pc; e += CB_THREADS) V0.p[e] = 0.f;
  const bool ok = mbar_wait(&bar, 0);
  if (threadIdx.x == 0) s_ok = ok ? 1 : 0;
  __syncthreads();
  if (!s_ok) {
    // the copies did not land in time: record it and leave once they have (bounded)
    if (threadIdx.x == 0) atomicExch(&ctl->err, 1);
    mbar_wait(&bar, 0);
    return;
  }
  // ---- down
  for (int l = lc; l < nl - 1; l++) {
    const LvS F = lv[l], Cc = lv[l + 1];
    for (int k = 0; k < 2; k++) { pass_d(F, 0); __syncthreads(); pass_d(F, 1); __syncthreads(); }
    for (int j = warp; j < F.ny; j += CB_WARPS)
      for (int i = lane; i < F.nx; i += 32) {
        float off, diag; stencil_d(F, i, j, off, diag);
        const int e = j * F.pc + i;
        sres[j * F.nx + i] = diag <= 0.f ? 0.f : F.rhs[e] - (off - diag * F.p[e]) / F.h2;
      }
    __syncthreads();
    for (int J = warp; J < Cc.ny; J += CB_WARPS)
      for (int I = lane; I < Cc.nx; I += 32) {
        const float r = sres[(2 * J) * F.nx + 2 * I] + sres[(2 * J) * F.nx + 2 * I + 1] + sres[(2 * J + 1) * F.nx + 2 * I] +
                        sres[(2 * J + 1) * F.nx + 2 * I + 1];
        Cc.rhs[J * Cc.pc + I] = 0.25f * r;
        Cc.p[J * Cc.pc + I] = 0.f;
      }
    __syncthreads();
  }
  // ---- coarsest (pressure.wgsl:132-156): 120 red-black sweeps from zero, one cell per thread
  // of the first 256 (a named barrier keeps the other warps out); each thread's stencil is
  // fixed during the sweeps and held in registers
  if (threadIdx.x < COARSEST_THREADS) {
    const LvS L = lv[nl - 1];
    const int k = threadIdx.x, n = L.nx * L.ny;
    const int i = k % L.nx, j = k / L.nx;
    const bool act = k < n;
    const int kp = j * L.pc + i;
    float w = 0.f, e = 0.f, s = 0.f, nn = 0.f, diag = 0.f, rh = 0.f;
    int col = -1;
    if (act) {
      w = L.ax[j * L.pu + i]; e = L.ax[j * L.pu + i + 1];
      s = L.ay[j * L.pc + i]; nn = L.ay[(j + 1) * L.pc + i];
      if (i > 0) diag += w; else diag += 2.f * w;
      if (i < L.nx - 1) diag += e; else diag += 2.f * e;
      if (j > 0) diag += s;
      if (j < L.ny - 1) diag += nn; else diag += 2.f * nn;
      rh = L.rhs[kp] * L.h2;
      col = (i + j) & 1;
      L.p[kp] = 0.f;
    }
    const bool hw = act && i > 0, he = act && i < L.nx - 1, hs = act && j > 0, hn = act && j < L.ny - 1;
    float* p = L.p;
    bar_coarsest();
    #pragma unroll 1
    for (int it = 0; it < 120; it++) {
      #pragma unroll
      for (int c = 0; c < 2; c++) {
        if (col == c) {
          float off = 0.f;
          if (hw) off += w * p[kp - 1];
          if (he) off += e * p[kp + 1];
          if (hs) off += s * p[kp - L.pc];
          if (hn) off += nn * p[kp + L.pc];
          p[kp] = diag > 0.f ? (off - rh) / diag : 0.f;
        }
        bar_coarsest();
      }
    }
  }
  __syncthreads();
  // ---- up
  for (int l = nl - 2; l >= lc; l--) {
    const LvS F = lv[l], Cc = lv[l + 1];
    for (int j = warp; j < F.ny; j += CB_WARPS)
      for (int i = lane; i < F.nx; i += 32) {
        const int I = i / 2, J = j / 2;
        const int I2 = min(max(I + ((i & 1) == 1 ? 1 : -1), 0), Cc.nx - 1);
        const int J2 = min(max(J + ((j & 1) == 1 ? 1 : -1), 0), Cc.ny - 1);
        const float c = 0.5625f * Cc.p[J * Cc.pc + I] + 0.1875f * (Cc.p[J * Cc.pc + I2] + Cc.p[J2 * Cc.pc + I]) +
                        0.0625f * Cc.p[J2 * Cc.pc + I2];
        float off, diag; stencil_d(F, i, j, off, diag);
        F.p[j * F.pc + i] += diag > 0.f ? c : 0.f;
      }
    __syncthreads();
    for (int k = 0; k < 2; k++) { pass_d(F, 1); __syncthreads(); pass_d(F, 0); __syncthreads(); }
  }
  // ---- write level lc back; when the block covers level 0, finish the cycle here
  const LevelDesc& G = S.lev[lc];
  double part = 0.0;
  for (int j = warp; j < G.ny; j += CB_WARPS)
    for (int i = lane; i < G.nx; i += 32) {
      const int e = j * V0.pc + i;
      G.p[j * G.pc + i] = V0.p[e];
      if (lc == 0 && tail == 1) {
        float off, diag; stencil_d(V0, i, j, off, diag);
        const double r = diag <= 0.f ? 0.0 : (double)(V0.rhs[e] - (off - diag * V0.p[e]) / V0.h2);
        part += r * r;
      } else if (lc == 0 && tail == 2) {
        S.p64[j * G.nx + i] += (double)V0.p[e];
      }
    }
  if (lc == 0 && tail == 1) {
    const double t = block_sum(part, red);
    if (threadIdx.x == 0) solve_decide_f(scenes, nscenes, S, ctl, t);
  }
}

// shared bytes of the coarse block for one scene (the layout built by k_mg_coarse)
size_t coarse_smem_bytes(const int* lnx, const int* lny, int lc, int nlev) {
  size_t f = 0;
  for (int l = lc; l < nlev; l++) {
    const size_t pc = (size_t)round_up(lnx[l], 32), pu = (size_t)round_up(lnx[l] + 1, 32);
    f += 2 * lny[l] * pc + lny[l] * pu + (lny[l] + 1) * pc;
  }
  f += std::max((size_t)lnx[lc] * lny[lc], (size_t)COARSEST_SCRATCH);
  return f * 4;
}

void launch_mg_down(const SceneDesc* scenes, const Work* work, int ntiles, int level, cudaStream_t st) {
  if (ntiles > 0) k_mg_down<MGF_TX, MGF_TY><<<ntiles, 256, 0, st>>>(scenes, work, level);
}
void launch_mg_up(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, int level, int tail, SolveCtl* ctl,
                  cudaStream_t st) {
  if (ntiles > 0) k_mg_up<MGF_TX, MGF_TY><<<ntiles, 256, 0, st>>>(scenes, nscenes, work, level, tail, ctl);
}
void launch_mg_coarse(const SceneDesc* scenes, int nscenes, SolveCtl* ctl, int tail, size_t smem, cudaStream_t st) {
  if (nscenes > 0) k_mg_coarse<<<nscenes, CB_THREADS, smem, st>>>(scenes, nscenes, ctl, tail);
}
cudaError_t prepare_mg_coarse(size_t smem) {
  return cudaFuncSetAttribute(k_mg_coarse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

}  // namespace cfg
