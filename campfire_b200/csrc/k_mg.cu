// Cut-cell multigrid of shaders/pressure.wgsl: one red-black colour pass,
// residual restriction, prolongation and the coarsest solve, one dispatch each
// as in FluidSim.vcycle (js/fluid.js:294-312); plus the loop control of the
// pressure solve (residual norms, FP64 defect correction) that decides, per
// scene, whether another V-cycle runs.
#include <atomic>

#include "gas_dev.cuh"
#include "kernels.h"
#include "reduce.cuh"

namespace cfg {

namespace {

// pressure.wgsl:77-85: sum a*p_nb and the diagonal (Dirichlet p = 0 at open domain faces: ghost = -p)
__device__ __forceinline__ void stencil(const LevelDesc& L, const float* p, int i, int j, float& off, float& diag) {
  off = 0.f; diag = 0.f;
  const float w = __ldg(L.ax + j * L.pu + i), e = __ldg(L.ax + j * L.pu + i + 1);
  const float s = __ldg(L.ay + j * L.pc + i), n = __ldg(L.ay + (j + 1) * L.pc + i);
  if (i > 0) { off += w * p[j * L.pc + i - 1]; diag += w; } else { diag += 2.f * w; }
  if (i < L.nx - 1) { off += e * p[j * L.pc + i + 1]; diag += e; } else { diag += 2.f * e; }
  if (j > 0) { off += s * p[(j - 1) * L.pc + i]; diag += s; }
  if (j < L.ny - 1) { off += n * p[(j + 1) * L.pc + i]; diag += n; } else { diag += 2.f * n; }
}
__device__ __forceinline__ float diag_of(const LevelDesc& L, int i, int j) {
  const float w = __ldg(L.ax + j * L.pu + i), e = __ldg(L.ax + j * L.pu + i + 1);
  const float s = __ldg(L.ay + j * L.pc + i), n = __ldg(L.ay + (j + 1) * L.pc + i);
  float diag = 0.f;
  if (i > 0) diag += w; else diag += 2.f * w;
  if (i < L.nx - 1) diag += e; else diag += 2.f * e;
  if (j > 0) diag += s;
  if (j < L.ny - 1) diag += n; else diag += 2.f * n;
  return diag;
}
// pressure.wgsl:96-101
__device__ __forceinline__ float residual(const LevelDesc& L, int i, int j) {
  float off, diag; stencil(L, L.p, i, j, off, diag);
  if (diag <= 0.f) return 0.f;
  return L.rhs[j * L.pc + i] - (off - diag * L.p[j * L.pc + i]) / L.h2;
}

__device__ __forceinline__ bool scene_live(const SceneDesc& S) { return S.enabled && S.solve->active; }

}  // namespace

// Last kernel of each iteration of the host-driven loop (launches outside a graph):
// count the cycle and fold in the hard cap.
__global__ void k_loop_guard(SolveCtl* ctl, unsigned long long h, int use_cond) {
  pdl_wait();
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int it = ctl->iter + 1;
  ctl->iter = it;
  const int go = (ctl->any_active && it < ctl->hard_cap) ? 1 : 0;
  ctl->any_active = go;
  if (use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)h, (unsigned)go);
}

// pressure.wgsl:87-94 (in place: a colour pass reads only the other colour)
__global__ void __launch_bounds__(256) k_relax(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work, int level, int color) {
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!scene_live(S)) return;
  const LevelDesc L = S.lev[level];
  const int i = w.tx * MG_TX + (threadIdx.x % MG_TX), j = w.ty * MG_TY + (threadIdx.x / MG_TX);
  if (i >= L.nx || j >= L.ny || ((i + j) & 1) != color) return;
  float off, diag; stencil(L, L.p, i, j, off, diag);
  const int k = j * L.pc + i;
  L.p[k] = diag > 0.f ? (off - L.rhs[k] * L.h2) / diag : 0.f;
}

// pressure.wgsl:104-113 (work tiles over the coarse level l+1)
__global__ void __launch_bounds__(256) k_restrict_res(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work, int level) {
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!scene_live(S)) return;
  const LevelDesc F = S.lev[level], C = S.lev[level + 1];
  const int I = w.tx * MG_TX + (threadIdx.x % MG_TX), J = w.ty * MG_TY + (threadIdx.x / MG_TX);
  if (I >= C.nx || J >= C.ny) return;
  const float r = residual(F, 2 * I, 2 * J) + residual(F, 2 * I + 1, 2 * J) + residual(F, 2 * I, 2 * J + 1) +
                  residual(F, 2 * I + 1, 2 * J + 1);
  C.rhs[J * C.pc + I] = 0.25f * r;
  C.p[J * C.pc + I] = 0.f;
}

// pressure.wgsl:116-129 (work tiles over the fine level l)
__global__ void __launch_bounds__(256) k_prolong(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work, int level) {
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!scene_live(S)) return;
  const LevelDesc F = S.lev[level], C = S.lev[level + 1];
  const int i = w.tx * MG_TX + (threadIdx.x % MG_TX), j = w.ty * MG_TY + (threadIdx.x / MG_TX);
  if (i >= F.nx || j >= F.ny) return;
  const int nxc = C.nx, nyc = C.ny;
  const int I = i / 2, J = j / 2;
  const int I2 = min(max(I + ((i & 1) == 1 ? 1 : -1), 0), nxc - 1);
  const int J2 = min(max(J + ((j & 1) == 1 ? 1 : -1), 0), nyc - 1);
  const float c = 0.5625f * C.p[J * C.pc + I] + 0.1875f * (C.p[J * C.pc + I2] + C.p[J2 * C.pc + I]) + 0.0625f * C.p[J2 * C.pc + I2];
  const int k = j * F.pc + i;
  F.p[k] += diag_of(F, i, j) > 0.f ? c : 0.f;
}

// pressure.wgsl:132-156: 120 red-black sweeps from zero on the coarsest level, one CTA per scene
__global__ void __launch_bounds__(256) k_coarsest(const SceneDesc* __restrict__ scenes) {
  __shared__ float wp[256], srhs[256], sw[256], se[256], ss[256], sn[256];
  const SceneDesc& S = scenes[blockIdx.x];
  if (!scene_live(S)) return;
  const LevelDesc L = S.lev[S.nlev - 1];
  const int n = L.nx * L.ny;
  const int k = threadIdx.x;
  const int i = k % L.nx, j = k / L.nx;
  if (k < n) {
    wp[k] = 0.f;
    srhs[k] = L.rhs[j * L.pc + i];
    sw[k] = L.ax[j * L.pu + i]; se[k] = L.ax[j * L.pu + i + 1];
    ss[k] = L.ay[j * L.pc + i]; sn[k] = L.ay[(j + 1) * L.pc + i];
  }
  __syncthreads();
  for (int it = 0; it < 120; it++) {
    for (int c = 0; c < 2; c++) {
      if (k < n && ((i + j) & 1) == c) {
        float off = 0.f, diag = 0.f;
        const float w = sw[k], e = se[k], s = ss[k], nn = sn[k];
        if (i > 0) { off += w * wp[k - 1]; diag += w; } else { diag += 2.f * w; }
        if (i < L.nx - 1) { off += e * wp[k + 1]; diag += e; } else { diag += 2.f * e; }
        if (j > 0) { off += s * wp[k - L.nx]; diag += s; }
        if (j < L.ny - 1) { off += nn * wp[k + L.nx]; diag += nn; } else { diag += 2.f * nn; }
        wp[k] = diag > 0.f ? (off - srhs[k] * L.h2) / diag : 0.f;
      }
      __syncthreads();
    }
  }
  if (k < n) L.p[j * L.pc + i] = wp[k];
}

// pressure.wgsl:57-67 for level l -> l+1 (work tiles over level l+1 cells; the last
// tile column/row also writes the east/north boundary faces)
__global__ void __launch_bounds__(256) k_coef_restrict(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work, int level) {
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!S.enabled) return;
  const LevelDesc F = S.lev[level], C = S.lev[level + 1];
  const int I = w.tx * MG_TX + (threadIdx.x % MG_TX), J = w.ty * MG_TY + (threadIdx.x / MG_TX);
  const int nxc = C.nx, nyc = C.ny;
  auto ax = [&](int a, int b) {
    C.ax[b * C.pu + a] = 0.5f * (F.ax[(2 * b) * F.pu + 2 * a] + F.ax[(2 * b + 1) * F.pu + 2 * a]);
  };
  auto ay = [&](int a, int b) {
    C.ay[b * C.pc + a] = 0.5f * (F.ay[(2 * b) * F.pc + 2 * a] + F.ay[(2 * b) * F.pc + 2 * a + 1]);
  };
  if (I < nxc && J < nyc) { ax(I, J); ay(I, J); }
  if (I == nxc - 1 && J < nyc) ax(nxc, J);
  if (J == nyc - 1 && I < nxc) ay(I, nyc);
}

// pressure.wgsl:57-67 for every level from `level` down, one CTA per scene (the levels
// below the forces kernel's in-tile restriction are small): level by level, a block
// barrier between them (each level reads the one just written by the same block)
__global__ void __launch_bounds__(512) k_coef_restrict_tail(const SceneDesc* __restrict__ scenes, int level) {
  const SceneDesc& S = scenes[blockIdx.x];
  if (!S.enabled) return;
  for (int l = level; l + 1 < S.nlev; l++) {
    const LevelDesc F = S.lev[l], C = S.lev[l + 1];
    const int nxc = C.nx, nyc = C.ny;
    for (int e = threadIdx.x; e < nxc * nyc; e += blockDim.x) {
      const int J = e / nxc, I = e - J * nxc;
      C.ax[J * C.pu + I] = 0.5f * (F.ax[(2 * J) * F.pu + 2 * I] + F.ax[(2 * J + 1) * F.pu + 2 * I]);
      C.ay[J * C.pc + I] = 0.5f * (F.ay[(2 * J) * F.pc + 2 * I] + F.ay[(2 * J) * F.pc + 2 * I + 1]);
      if (I == nxc - 1) C.ax[J * C.pu + nxc] = 0.5f * (F.ax[(2 * J) * F.pu + 2 * nxc] + F.ax[(2 * J + 1) * F.pu + 2 * nxc]);
      if (J == nyc - 1) C.ay[nyc * C.pc + I] = 0.5f * (F.ay[(2 * nyc) * F.pc + 2 * I] + F.ay[(2 * nyc) * F.pc + 2 * I + 1]);
    }
    __syncthreads();
  }
}

// ||r||^2 of level 0 after a V-cycle -> per-scene decision -> loop condition
__global__ void __launch_bounds__(256) k_resnorm(const SceneDesc* __restrict__ scenes, int nscenes, const Work* __restrict__ work,
                                                 SolveCtl* ctl) {
  __shared__ double red[32];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!scene_live(S)) return;
  const LevelDesc L = S.lev[0];
  const int i = w.tx * MG_TX + (threadIdx.x % MG_TX), j = w.ty * MG_TY + (threadIdx.x / MG_TX);
  double v = 0.0;
  if (i < L.nx && j < L.ny) { const double r = (double)residual(L, i, j); v = r * r; }
  const double bp = block_sum(v, red);
  double total = 0.0;
  if (scene_reduce(S, w.tile, S.nt_mg0, bp, red, &total) && threadIdx.x == 0)
    solve_decide(ctl, S.solve, total, true);
}

// FP64 defect: r64 = rhs64 - A p64 (f32 coefficients promoted), rhs0 = f32(r64), p0 = 0
__global__ void __launch_bounds__(256) k_defect64(const SceneDesc* __restrict__ scenes, int nscenes, const Work* __restrict__ work,
                                                  SolveCtl* ctl, int first) {
  __shared__ double red[32];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  pdl_trigger();
  const LevelDesc L = S.lev[0];
  pdl_wait();
  if (!scene_live(S)) return;
  const int nx = L.nx;
  const int i = w.tx * MG_TX + (threadIdx.x % MG_TX), j = w.ty * MG_TY + (threadIdx.x / MG_TX);
  double v = 0.0;
  if (i < L.nx && j < L.ny) {
    const double* p = S.p64;
    const double wv = __ldg(L.ax + j * L.pu + i), e = __ldg(L.ax + j * L.pu + i + 1);
    const double so = __ldg(L.ay + j * L.pc + i), n = __ldg(L.ay + (j + 1) * L.pc + i);
    double off = 0.0, diag = 0.0;
    if (i > 0) { off += wv * p[j * nx + i - 1]; diag += wv; } else diag += 2.0 * wv;
    if (i < L.nx - 1) { off += e * p[j * nx + i + 1]; diag += e; } else diag += 2.0 * e;
    if (j > 0) { off += so * p[(j - 1) * nx + i]; diag += so; }
    if (j < L.ny - 1) { off += n * p[(j + 1) * nx + i]; diag += n; } else diag += 2.0 * n;
    const int k = j * nx + i;
    const double r = diag > 0.0 ? S.rhs64[k] - (off - diag * p[k]) / (double)L.h2 : 0.0;
    L.rhs[j * L.pc + i] = (float)r;
    L.p[j * L.pc + i] = 0.f;
    if (first && ctl->krylov) {   // the Krylov loop starts from this residual with no direction
      S.r64[k] = r;
      S.dA[k] = 0.0; S.dB[k] = 0.0; S.q64[k] = 0.0;
    }
    v = r * r;
  }
  const double bp = block_sum(v, red);
  double total = 0.0;
  if (scene_reduce(S, w.tile, S.nt_mg0, bp, red, &total) && threadIdx.x == 0) {
    if (first) {
      S.solve->rel0 = S.solve->bnorm2 > 0.0 ? sqrt(total / S.solve->bnorm2) : 0.0;
      S.solve->alpha = 0.0; S.solve->beta = 0.0; S.solve->delta = 0.0;
    }
    solve_decide(ctl, S.solve, total, !first);
  }
}

// Krylov FP64 mode (flexible preconditioned CG on the level-0 operator L, the V-cycle's
// z ~ L^-1 r as preconditioner), after the V-cycle (beta, alpha from the level-0 up
// kernel): d = z + beta d, q = Lz + beta q (= L d, L symmetric; z the cycle's level-0 p,
// Lz from the up kernel), p64 += alpha d, r -= alpha q, rhs0 = f32(r), p0 = 0, ||r|| ->
// the loop decision. The scene's solve state is read in one round after the wait.
__global__ void __launch_bounds__(256) k_pcg_step(const SceneDesc* __restrict__ scenes, int nscenes,
                                                  const Work* __restrict__ work, SolveCtl* ctl) {
  __shared__ double red[32];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  pdl_trigger();
  const LevelDesc L = S.lev[0];
  const bool on = S.enabled;   // host-written, constant during the step
  SolveState* ss = S.solve;
  pdl_wait();
  if (!on) return;
  const int live = ss->active;
  const double alpha = ss->alpha, beta = ss->beta;
  const DecideIn din = decide_load(ctl, ss);
  if (!live) return;
  const int cyc = din.cycles;
  const int nx = L.nx;
  const bool first = cyc == 0;
  const int i = w.tx * MG_TX + (threadIdx.x % MG_TX), j = w.ty * MG_TY + (threadIdx.x / MG_TX);
  double v = 0.0;
  if (i < L.nx && j < L.ny) {
    const int k = j * nx + i;
    const double z = (double)L.p[j * L.pc + i], lz = S.dB[k];
    const double d = first ? z : z + beta * S.dA[k];
    const double q = first ? lz : lz + beta * S.q64[k];
    S.dA[k] = d;
    S.q64[k] = q;
    S.p64[k] += alpha * d;
    const double r = S.r64[k] - alpha * q;
    S.r64[k] = r;
    L.rhs[j * L.pc + i] = (float)r;
    L.p[j * L.pc + i] = 0.f;
    v = r * r;
  }
  const double bp = block_sum(v, red);
  double total = 0.0;
  if (scene_reduce(S, w.tile, S.nt_mg0, bp, red, &total) && threadIdx.x == 0) solve_decide(ctl, ss, din, total, true);
}

// Fused Krylov mode, after the loop: the update of each scene's last cycle (cycles >= 1),
// d = z + beta d (z on the first cycle), p64 += alpha d; r and q are not needed again
__global__ void __launch_bounds__(256) k_pcg_finish(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work) {
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  pdl_trigger();
  const LevelDesc L = S.lev[0];
  const bool on = S.enabled;   // host-written, constant during the step
  SolveState* ss = S.solve;
  pdl_wait();
  if (!on) return;
  const int cyc = ss->cycles;
  const double alpha = ss->alpha, beta = ss->beta;
  if (cyc < 1) return;
  const int i = w.tx * MG_TX + (threadIdx.x % MG_TX), j = w.ty * MG_TY + (threadIdx.x / MG_TX);
  if (i >= L.nx || j >= L.ny) return;
  const int k = j * L.nx + i;
  const double z = (double)L.p[j * L.pc + i];
  const double d = cyc == 1 ? z : z + beta * S.dA[k];
  S.dA[k] = d;
  S.p64[k] += alpha * d;
}

// FP64: p64 += p0 after a V-cycle on the defect
__global__ void __launch_bounds__(256) k_accum64(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work) {
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!scene_live(S)) return;
  const LevelDesc L = S.lev[0];
  const int i = w.tx * MG_TX + (threadIdx.x % MG_TX), j = w.ty * MG_TY + (threadIdx.x / MG_TX);
  if (i >= L.nx || j >= L.ny) return;
  S.p64[j * L.nx + i] += (double)L.p[j * L.pc + i];
}

// ||r||2 and ||rhs||2 of level 0 for one scene (diagnostic, one CTA)
__global__ void __launch_bounds__(1024) k_residual_norms(const SceneDesc* __restrict__ scenes, int scene, double* out) {
  __shared__ double red[32];
  const SceneDesc& S = scenes[scene];
  const LevelDesc L = S.lev[0];
  double vr = 0.0, vb = 0.0;
  for (int e = threadIdx.x; e < L.nx * L.ny; e += blockDim.x) {
    const int i = e % L.nx, j = e / L.nx;
    const double r = (double)residual(L, i, j);
    const double b = (double)L.rhs[j * L.pc + i];
    vr += r * r; vb += b * b;
  }
  const double tr = block_sum(vr, red);
  const double tb = block_sum(vb, red);
  if (threadIdx.x == 0) { out[0] = tr; out[1] = tb; }
}

// ||rhs||^2 of level 0 (FP64 mode: of rhs64); arms the pressure loop of every scene
__global__ void __launch_bounds__(256) k_bnorm(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work, SolveCtl* ctl, int fp64) {
  __shared__ double red[32];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!S.enabled) return;
  const LevelDesc L = S.lev[0];
  const int i = w.tx * MG_TX + (threadIdx.x % MG_TX), j = w.ty * MG_TY + (threadIdx.x / MG_TX);
  double v = 0.0;
  if (i < L.nx && j < L.ny) {
    const double b = fp64 ? S.rhs64[j * L.nx + i] : (double)L.rhs[j * L.pc + i];
    v = b * b;
  }
  const double bp = block_sum(v, red);
  double total = 0.0;
  if (scene_reduce(S, w.tile, S.nt_mg0, bp, red, &total) && threadIdx.x == 0) {
    S.solve->bnorm2 = total; S.solve->cycles = 0; S.solve->active = 1;
    const unsigned d = arrive_acq_rel(&ctl->scenes_done);
    if (d == (unsigned)ctl->nscenes - 1u) { ctl->scenes_done = 0u; ctl->nactive = ctl->nscenes; ctl->any_active = 1; }
  }
}

void launch_coef_restrict_tail(const SceneDesc* scenes, int nscenes, int level, cudaStream_t st) {
  if (nscenes > 0) k_coef_restrict_tail<<<nscenes, 512, 0, st>>>(scenes, level);
}
void launch_bnorm(const SceneDesc* scenes, const Work* work, int ntiles, SolveCtl* ctl, bool fp64, cudaStream_t st) {
  if (ntiles > 0) k_bnorm<<<ntiles, MG_TX * MG_TY, 0, st>>>(scenes, work, ctl, fp64 ? 1 : 0);
}
void launch_relax(const SceneDesc* scenes, const Work* work, int ntiles, int level, int color, cudaStream_t st) {
  if (ntiles > 0) k_relax<<<ntiles, MG_TX * MG_TY, 0, st>>>(scenes, work, level, color);
}
void launch_restrict_res(const SceneDesc* scenes, const Work* work, int ntiles, int level, cudaStream_t st) {
  if (ntiles > 0) k_restrict_res<<<ntiles, MG_TX * MG_TY, 0, st>>>(scenes, work, level);
}
void launch_prolong(const SceneDesc* scenes, const Work* work, int ntiles, int level, cudaStream_t st) {
  if (ntiles > 0) k_prolong<<<ntiles, MG_TX * MG_TY, 0, st>>>(scenes, work, level);
}
void launch_coarsest(const SceneDesc* scenes, int nscenes, cudaStream_t st) {
  if (nscenes > 0) k_coarsest<<<nscenes, 256, 0, st>>>(scenes);
}
void launch_coef_restrict(const SceneDesc* scenes, const Work* work, int ntiles, int level, cudaStream_t st) {
  if (ntiles > 0) k_coef_restrict<<<ntiles, MG_TX * MG_TY, 0, st>>>(scenes, work, level);
}
void launch_resnorm(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, SolveCtl* ctl,
                    cudaStream_t st) {
  if (ntiles > 0) k_resnorm<<<ntiles, MG_TX * MG_TY, 0, st>>>(scenes, nscenes, work, ctl);
}
void launch_defect64(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, SolveCtl* ctl,
                     int first, cudaStream_t st) {
  if (ntiles > 0)
    launch_pdl(pdl_enabled(), k_defect64, dim3(ntiles), dim3(MG_TX * MG_TY), 0, st, scenes, nscenes, work, ctl, first);
}
void launch_pcg_finish(const SceneDesc* scenes, const Work* work, int ntiles, cudaStream_t st) {
  // after the loop node (or the host loop's copy-back): an ordinary launch
  if (ntiles > 0) k_pcg_finish<<<ntiles, MG_TX * MG_TY, 0, st>>>(scenes, work);
}
void launch_pcg_step(const SceneDesc* scenes, int nscenes, const Work* work, int ntiles, SolveCtl* ctl,
                     cudaStream_t st) {
  if (ntiles > 0)
    launch_pdl(pdl_enabled(), k_pcg_step, dim3(ntiles), dim3(MG_TX * MG_TY), 0, st, scenes, nscenes, work, ctl);
}
void launch_loop_guard(SolveCtl* ctl, unsigned long long cond_handle, int use_cond, cudaStream_t st) {
  launch_pdl(pdl_enabled(), k_loop_guard, dim3(1), dim3(32), 0, st, ctl, cond_handle, use_cond);
}

namespace {
std::atomic<bool> g_pdl{true};
}
void set_pdl(bool on) { g_pdl.store(on); }
bool pdl_enabled() { return g_pdl.load(); }
void launch_accum64(const SceneDesc* scenes, const Work* work, int ntiles, cudaStream_t st) {
  if (ntiles > 0) k_accum64<<<ntiles, MG_TX * MG_TY, 0, st>>>(scenes, work);
}
void launch_residual_norms(const SceneDesc* scenes, int scene, double* out, cudaStream_t st) {
  k_residual_norms<<<1, 1024, 0, st>>>(scenes, scene, out);
}

}  // namespace cfg
