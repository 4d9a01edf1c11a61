// Momentum forces (shaders/forces.wgsl:34-101) fused with the level-0 face
// coefficients (pressure.wgsl:30-43), the right-hand side (pressure.wgsl:46-54),
// the coefficient restriction to levels 1..FR_KMAX (pressure.wgsl:57-67) and the
// ||rhs||2 reduction that the pressure loop divides by.
//
// A CTA computes the new U/V of its tile's faces (including the east and north
// boundary faces, which neighbouring tiles also compute and own), keeps them in
// shared memory for the divergence of its cells, and writes the faces it owns.
// Coefficient levels 1..FR_KMAX are averaged inside the tile from the level
// below, in the same order as the reference's per-level dispatches.
#include "gas_dev.cuh"
#include "kernels.h"
#include "reduce.cuh"

namespace cfg {

namespace {

// forces.wgsl:30-32 entrained air arrives with no momentum
__device__ __forceinline__ float exchange(const cfg_params& P, float spd, float Tf) {
  return expf(-2.f * P.exchAlpha * spd * (Tf / P.Tamb) / P.depth * P.dt);
}

__device__ __forceinline__ float invRho(const cfg_params& P, float T) { return T / (P.rhoAmb * P.Tamb); }  // pressure.wgsl:27

}  // namespace

template <int TX, int TY, bool FORCES, bool COEF>
__global__ void __launch_bounds__(256) k_forces(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work,
                                               SolveCtl* ctl, int fp64) {
  constexpr int AXW = TX + 1, AYH = TY + 1;
  constexpr int MW = TX + 2, MH = TY + 2;   // cell viscosities of the tile and a one-cell ring
  __shared__ float sU[TY * AXW], sV[AYH * TX];
  __shared__ float sMu[FORCES ? MH * MW : 1];
  __shared__ float sAx[2][TY * AXW], sAy[2][AYH * TX];
  __shared__ double red[32];

  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!S.enabled) return;
  const cfg_params& P = S.P;
  const int nx = S.nx, ny = S.ny, pc = S.pc, pu = S.pu;
  const int x0 = w.tx * TX, y0 = w.ty * TY;
  const float dt = P.dt, dx = P.dx;
  const float idx2 = 1.f / (dx * dx);
  const float* __restrict__ T = S.T;
  const float* __restrict__ U2 = S.U2;
  const float* __restrict__ V2 = S.V2;
  const float* __restrict__ fxa = S.fx;
  const float* __restrict__ fya = S.fy;
  auto Tc = [&](int i, int j) { return __ldg(T + min(max(j, 0), ny - 1) * pc + min(max(i, 0), nx - 1)); };
  auto u2 = [&](int i, int j) { const int k = j * pu + i; return __ldg(fxa + k) > 0.f ? __ldg(U2 + k) : 0.f; };
  auto v2 = [&](int i, int j) { const int k = j * pc + i; return __ldg(fya + k) > 0.f ? __ldg(V2 + k) : 0.f; };
  const LevelDesc L0 = S.lev[0];

  // each cell's viscosity once (a cell's mu enters the two U faces and the two V faces beside
  // it); the ring's indices clamp as Tc's do
  if (FORCES) {
    for (int e = threadIdx.x; e < MH * MW; e += blockDim.x)
      sMu[e] = muOf(P, Tc(x0 - 1 + e % MW, y0 - 1 + e / MW));
    __syncthreads();
  }
  auto muC = [&](int i, int j) { return sMu[(j - y0 + 1) * MW + (i - x0 + 1)]; };

  // ---- U faces: x in [x0, x0+TX], y in [y0, y0+TY)
  for (int e = threadIdx.x; e < TY * AXW; e += blockDim.x) {
    const int i = x0 + e % AXW, j = y0 + e / AXW;
    if (i > nx || j >= ny) continue;
    const int k = j * pu + i;
    const bool own = (i < x0 + TX) || (i == nx);
    float unew;
    if (FORCES) {
      if (__ldg(fxa + k) <= 0.f) unew = 0.f;
      else if (i == 0) unew = fminf(__ldg(U2 + j * pu + 1), 0.f);
      else if (i == nx) unew = fmaxf(__ldg(U2 + j * pu + nx - 1), 0.f);
      else {
        const float u = __ldg(U2 + k);
        const float TL = Tc(i - 1, j), TR = Tc(i, j);
        const float rhoF = rhoOf(P, 0.5f * (TL + TR));
        const float muE = muC(i, j), muW = muC(i - 1, j);
        float uN = u, muN, uS = -u, muS;
        if (j < ny - 1) { uN = u2(i, j + 1); muN = muOf(P, 0.25f * (TL + TR + Tc(i - 1, j + 1) + Tc(i, j + 1))); }
        else muN = muOf(P, 0.5f * (TL + TR));
        if (j > 0) { uS = u2(i, j - 1); muS = muOf(P, 0.25f * (TL + TR + Tc(i - 1, j - 1) + Tc(i, j - 1))); }
        else muS = muOf(P, 0.5f * (TL + TR));
        const float visc = (muE * (u2(i + 1, j) - u) + muW * (u2(i - 1, j) - u) + muN * (uN - u) + muS * (uS - u)) * idx2 / rhoF;
        const float vAvg = 0.25f * (__ldg(V2 + j * pc + i - 1) + __ldg(V2 + j * pc + i) + __ldg(V2 + (j + 1) * pc + i - 1) +
                                    __ldg(V2 + (j + 1) * pc + i));
        unew = (u + dt * visc) * exchange(P, sqrtf(u * u + vAvg * vAvg), 0.5f * (TL + TR));
      }
      if (own) S.U[k] = unew;
    } else {
      unew = __ldg(S.U + k);
    }
    sU[e] = unew;
    if (COEF) {
      const float Tf = 0.5f * (__ldg(T + j * pc + min(max(i - 1, 0), nx - 1)) + __ldg(T + j * pc + min(i, nx - 1)));
      const float a = __ldg(fxa + k) * invRho(P, Tf);
      sAx[0][e] = a;
      if (own) L0.ax[j * L0.pu + i] = a;
    }
  }
  // ---- V faces: x in [x0, x0+TX), y in [y0, y0+TY]
  for (int e = threadIdx.x; e < AYH * TX; e += blockDim.x) {
    const int i = x0 + e % TX, j = y0 + e / TX;
    if (i >= nx || j > ny) continue;
    const int k = j * pc + i;
    const bool own = (j < y0 + TY) || (j == ny);
    float vnew;
    if (FORCES) {
      if (j == 0 || __ldg(fya + k) <= 0.f) vnew = 0.f;
      else if (j == ny) vnew = fmaxf(__ldg(V2 + (ny - 1) * pc + i), 0.f);
      else {
        const float v = __ldg(V2 + k);
        const float TB = Tc(i, j - 1), TT = Tc(i, j);
        const float Tf = 0.5f * (TB + TT);
        const float rhoF = rhoOf(P, Tf);
        const float muN = muC(i, j), muS = muC(i, j - 1);
        float vE = v, muE, vW = v, muW;
        if (i < nx - 1) { vE = v2(i + 1, j); muE = muOf(P, 0.25f * (TB + TT + Tc(i + 1, j - 1) + Tc(i + 1, j))); }
        else muE = muOf(P, Tf);
        if (i > 0) { vW = v2(i - 1, j); muW = muOf(P, 0.25f * (TB + TT + Tc(i - 1, j - 1) + Tc(i - 1, j))); }
        else muW = muOf(P, Tf);
        const float visc = (muN * (v2(i, j + 1) - v) + muS * (v2(i, j - 1) - v) + muE * (vE - v) + muW * (vW - v)) * idx2 / rhoF;
        const float buoy = P.grav * (Tf / P.Tamb - 1.f);
        const float uAvg = 0.25f * (__ldg(U2 + (j - 1) * pu + i) + __ldg(U2 + (j - 1) * pu + i + 1) + __ldg(U2 + j * pu + i) +
                                    __ldg(U2 + j * pu + i + 1));
        vnew = (v + dt * (visc + buoy)) * exchange(P, sqrtf(uAvg * uAvg + v * v), Tf);
      }
      if (own) S.V[k] = vnew;
    } else {
      vnew = __ldg(S.V + k);
    }
    sV[e] = vnew;
    if (COEF) {
      const float Tf = 0.5f * (__ldg(T + min(max(j - 1, 0), ny - 1) * pc + i) + __ldg(T + min(j, ny - 1) * pc + i));
      const float a = __ldg(fya + k) * invRho(P, Tf);
      sAy[0][e] = a;
      if (own) L0.ay[j * L0.pc + i] = a;
    }
  }
  if (!COEF) return;
  __syncthreads();

  // ---- rhs0 (pressure.wgsl:46-54) for the tile cells; FP64 mode also assembles rhs64
  double part = 0.0;
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    const int ci = e % TX, cj = e / TX, i = x0 + ci, j = y0 + cj;
    if (i >= nx || j >= ny) continue;
    const float fE = __ldg(fxa + j * pu + i + 1), fW = __ldg(fxa + j * pu + i);
    const float fN = __ldg(fya + (j + 1) * pc + i), fS = __ldg(fya + j * pc + i);
    const float uE = sU[cj * AXW + ci + 1], uW = sU[cj * AXW + ci];
    const float vN = sV[(cj + 1) * TX + ci], vS = sV[cj * TX + ci];
    const float div = (fE * uE - fW * uW + fN * vN - fS * vS) / dx;
    const float open = fE + fW + fN + fS;
    const float sq = __ldg(&S.SQ[j * pc + i].x);
    const float r = open > 0.f ? (div - sq) / dt : 0.f;
    L0.rhs[j * L0.pc + i] = r;
    if (fp64) {
      const double a = (double)fE * (double)uE, b = (double)fW * (double)uW;
      const double c = (double)fN * (double)vN, d = (double)fS * (double)vS;
      const double op = (double)fE + (double)fW + (double)fN + (double)fS;
      const double r64 = op > 0.0 ? (((a - b) + c - d) / (double)dx - (double)sq) / (double)dt : 0.0;
      S.rhs64[j * nx + i] = r64;
      part += r64 * r64;
    } else {
      part += (double)r * (double)r;
    }
  }

  // ---- coefficient levels 1..FR_KMAX inside the tile (pressure.wgsl:57-67)
  int cur = 0;
  for (int l = 1; l <= FR_KMAX && l < S.nlev; l++) {
    const int tw = TX >> l, th = TY >> l;             // tile size at level l
    if (tw < 1 || th < 1) break;
    const int fw = TX >> (l - 1);                       // tile width at level l-1
    const LevelDesc C = S.lev[l];
    const int I0 = x0 >> l, J0 = y0 >> l;
    const float* Ax = sAx[cur]; const float* Ay = sAy[cur];
    float* Axn = sAx[cur ^ 1]; float* Ayn = sAy[cur ^ 1];
    __syncthreads();
    for (int e = threadIdx.x; e < th * (tw + 1); e += blockDim.x) {
      const int a = e % (tw + 1), b = e / (tw + 1), I = I0 + a, J = J0 + b;
      if (I > C.nx || J >= C.ny) continue;
      const float v = 0.5f * (Ax[(2 * b) * (fw + 1) + 2 * a] + Ax[(2 * b + 1) * (fw + 1) + 2 * a]);
      Axn[b * (tw + 1) + a] = v;
      if (a < tw || I == C.nx) C.ax[J * C.pu + I] = v;
    }
    for (int e = threadIdx.x; e < (th + 1) * tw; e += blockDim.x) {
      const int a = e % tw, b = e / tw, I = I0 + a, J = J0 + b;
      if (I >= C.nx || J > C.ny) continue;
      const float v = 0.5f * (Ay[(2 * b) * fw + 2 * a] + Ay[(2 * b) * fw + 2 * a + 1]);
      Ayn[b * tw + a] = v;
      if (b < th || J == C.ny) C.ay[J * C.pc + I] = v;
    }
    cur ^= 1;
  }

  // ---- ||rhs||^2: per-scene deterministic reduction; the finishing CTA arms the pressure loop
  const double bp = block_sum(part, red);
  double total = 0.0;
  if (scene_reduce(S, w.tile, S.nt_fr, bp, red, &total) && threadIdx.x == 0) {
    SolveState* ss = S.solve;
    ss->bnorm2 = total;
    ss->cycles = 0;
    ss->active = 1;
    const unsigned d = arrive_acq_rel(&ctl->scenes_done);
    if (d == (unsigned)ctl->nscenes - 1u) {
      ctl->scenes_done = 0u;
      ctl->nactive = ctl->nscenes;
      ctl->any_active = 1;
    }
  }
}

template <int TX, int TY>
static void launch_forces_t(const SceneDesc* scenes, const Work* work, int ntiles, SolveCtl* ctl, bool forces,
                            bool coef_rhs, bool fp64, cudaStream_t st) {
  if (forces && coef_rhs) k_forces<TX, TY, true, true><<<ntiles, 256, 0, st>>>(scenes, work, ctl, fp64 ? 1 : 0);
  else if (forces) k_forces<TX, TY, true, false><<<ntiles, 256, 0, st>>>(scenes, work, ctl, fp64 ? 1 : 0);
  else if (coef_rhs) k_forces<TX, TY, false, true><<<ntiles, 256, 0, st>>>(scenes, work, ctl, fp64 ? 1 : 0);
}
void launch_forces(const SceneDesc* scenes, const Work* work, int ntiles, SolveCtl* ctl, bool forces, bool coef_rhs,
                   bool fp64, int shape, cudaStream_t st) {
  if (ntiles <= 0) return;
  static_assert(TILE_TX[0] == FR_TX && TILE_TY[0] == FR_TY, "shape 0 is the default tile");
  if (shape == 1) launch_forces_t<TILE_TX[1], TILE_TY[1]>(scenes, work, ntiles, ctl, forces, coef_rhs, fp64, st);
  else if (shape == 2) launch_forces_t<TILE_TX[2], TILE_TY[2]>(scenes, work, ntiles, ctl, forces, coef_rhs, fp64, st);
  else launch_forces_t<FR_TX, FR_TY>(scenes, work, ntiles, ctl, forces, coef_rhs, fp64, st);
}

}  // namespace cfg
