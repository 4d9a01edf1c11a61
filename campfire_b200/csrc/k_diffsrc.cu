// Diffusion sub-steps (shaders/diffuse.wgsl:18-50, count from js/fluid.js:190-198)
// fused with the pointwise sources pass (shaders/sources.wgsl:34-173).
//
// A CTA loads T2/Y2 on its tile plus a halo of n = diff_sub cells into shared
// memory, runs the n explicit sub-steps there (each shrinks the valid region by
// one cell, so the result equals n separate dispatches), then applies the
// sources to its own cells and writes T, Y, SQ. The heat-release and radiative
// totals are tree-reduced per 8x8 block in the order of sources.wgsl:160-167
// and rounded to fixed point per block, so acc[512..514] reproduce the
// reference's per-workgroup atomics.
#include "gas_dev.cuh"
#include "kernels.h"

namespace cfg {

namespace {

// sources.wgsl:34-157 for one gas cell; returns false for a cell inside wood
struct SrcOut { float T; float4 Y; float S, qrel, qrad, tpeak; bool solid; };

// Tamb4 = powf(P.Tamb, 4) (the radiation's ambient term, the same for every cell of the scene)
__device__ __forceinline__ SrcOut sources_cell(const SceneDesc& S, const cfg_params& P, int i, int j, float Tc, float4 Yc,
                                               float Tadv, float Tamb4) {
  SrcOut o; o.qrel = 0.f; o.qrad = 0.f; o.tpeak = 0.f; o.solid = false; o.S = 0.f;
  const int k = j * S.pc + i;
  const float2 g = __ldg(S.cellG + k);
  const float sdf = g.x;
  const uint32_t sid = __float_as_uint(g.y);
  float massSrc = 0.f;
  const float dx = P.dx, dt = P.dt;
  const float cellA = dx * dx;
  const Piece* pieces = reinterpret_cast<const Piece*>(S.pieces);
  if (sdf < 0.f && sid != SOLID_NONE) {
    // :50-54 inside wood: hold the surface temperature (Y untouched, SQ = 0)
    o.solid = true;
    o.T = __ldg(&pieces[sid >> 2u].Ts[sid & 3u]);
    o.Y = Yc;
    return o;
  }
  if (sid != SOLID_NONE && sdf < 2.f * dx) {   // :57-94 wood coupling
    const uint32_t pi = sid >> 2u, fi = sid & 3u;
    const Piece& pc = pieces[pi];
    const float Ts = __ldg(&pc.Ts[fi]);
    const float half = __ldg(&pc.half);
    const float band = (float)__ldg(S.faceW + sid) / 1.0e8f;
    const float w = fmaxf(0.f, 1.f - fabsf(sdf - dx) / dx) / dx * (2.f * half) / fmaxf(band, 1e-6f);
    const float rho = rhoOf(P, Tc);
    const float kg = rhoDOf(P, 0.5f * (Tc + Ts)) * P.cp;
    const float dist = fmaxf(sdf, 0.5f * dx);
    const float rate = kg * w / (dist * rho * P.cp);
    const float dTc = (Ts - Tc) * (1.f - expf(-rate * dt));
    Tc += dTc;
    const float toWood = -rho * P.cp * dTc * cellA;
    atomicAdd(S.acc + (pi * 4u + fi) * 2u, wgsl_i32_round(toWood * 1.0e6f));
    const float mf = __ldg(&pc.mflux[fi]) * w;
    if (mf > 0.f) {
      const float madd = mf * dt;
      const float r = rhoOf(P, Tc);
      Yc = make_float4((r * Yc.x + madd) / (r + madd), (r * Yc.y + 0.f) / (r + madd),
                       (r * Yc.z + 0.f) / (r + madd), (r * Yc.w + 0.f) / (r + madd));
      Tc = (r * Tc + madd * Ts) / (r + madd);
      massSrc += mf;
    }
    const float cov = __ldg(&pc.charCov[fi]);
    if (cov > 0.f && Yc.y > 0.f) {
      const float r = rhoOf(P, Tc);
      const float kc = P.charA * expf(-P.charTa / Ts) * cov;
      const float mO2 = fminf(kc * r * Yc.y * w * dt, 0.9f * r * Yc.y);
      const float mC = mO2 / P.charO2;
      Yc = make_float4((r * Yc.x + 0.f) / (r + mC), (r * Yc.y + -mO2) / (r + mC),
                       (r * Yc.z + (mC + mO2)) / (r + mC), (r * Yc.w + 0.f) / (r + mC));
      Tc = (r * Tc + mC * Ts) / (r + mC);
      massSrc += mC / dt;
      atomicAdd(S.acc + (pi * 4u + fi) * 2u + 1u, wgsl_i32_round(mC * cellA * 1.0e12f));
    }
  }
  // :96-107 test sources
  const float x = ((float)i + 0.5f) * dx, y = ((float)j + 0.5f) * dx;
  if (P.heaterT > 0.f && x > P.heaterX0 && x < P.heaterX1 && y < P.heaterY1) Tc = P.heaterT;
  if (P.burnerFlux > 0.f && j == 0 && x > P.burnerX0 && x < P.burnerX1) {
    const float mf = P.burnerFlux / dx;
    const float madd = mf * dt;
    const float r = rhoOf(P, Tc);
    Yc = make_float4((r * Yc.x + madd) / (r + madd), (r * Yc.y + 0.f) / (r + madd),
                     (r * Yc.z + 0.f) / (r + madd), (r * Yc.w + 0.f) / (r + madd));
    Tc = (r * Tc + madd * P.burnerT) / (r + madd);
    massSrc += mf;
  }
  // :109-120 gas-phase combustion, 8 sub-steps
  const float rho0 = rhoOf(P, Tc);
  const float h = dt / 8.f;
  float burned = 0.f;
  #pragma unroll 1
  for (int s = 0; s < 8; s++) {
    const float wr = P.reactB * rho0 * Yc.x * Yc.y * expf(-P.reactTa / Tc);
    const float dF = fminf(wr * h, fminf(Yc.x, Yc.y / P.sO2));
    Yc = make_float4(Yc.x + -dF, Yc.y + -P.sO2 * dF, Yc.z + (1.f + P.sO2) * dF, Yc.w + 0.f);
    Tc += dF * P.dHc / P.cp;
    burned += dF;
  }
  // :122-128 soot formation and oxidation
  const float dSf = fminf(P.sootFormA * expf(-P.sootFormTa / Tc) * Yc.x * dt, Yc.x);
  Yc = make_float4(Yc.x + -dSf, Yc.y + 0.f, Yc.z + 0.f, Yc.w + dSf);
  const float dSo = fminf(P.sootOxA * Yc.w * Yc.y * expf(-P.sootOxTa / Tc) * dt, fminf(Yc.w, Yc.y / P.sO2));
  Yc = make_float4(Yc.x + 0.f, Yc.y + -P.sO2 * dSo, Yc.z + (1.f + P.sO2) * dSo, Yc.w + -dSo);
  Tc += dSo * P.dHc / P.cp;
  burned += dSo;
  o.qrel = rho0 * burned * P.dHc / dt;
  // :130-136 optically thin radiation, linearised implicit
  const float r1 = rhoOf(P, Tc);
  const float fv = r1 * Yc.w / P.sootDensity;
  const float kap = P.kappaSootC * fv * Tc + P.kappaGas * Yc.z;
  const float T3 = Tc * Tc * Tc;
  o.qrad = 4.f * kap * P.sigma * (T3 * Tc - Tamb4);
  const float dTr = o.qrad * dt / (r1 * P.cp) / (1.f + 16.f * kap * P.sigma * T3 * dt / (r1 * P.cp));
  Tc -= dTr;
  // :140-148 entrainment of ambient air through the front/back faces
  const float ucx = 0.5f * (__ldg(S.U + j * S.pu + i) + __ldg(S.U + j * S.pu + i + 1));
  const float ucy = 0.5f * (__ldg(S.V + j * S.pc + i) + __ldg(S.V + (j + 1) * S.pc + i));
  const float me = 2.f * P.exchAlpha * sqrtf(ucx * ucx + ucy * ucy) * P.rhoAmb / P.depth;
  if (me > 0.f) {
    const float madd = me * dt;
    const float r = rhoOf(P, Tc);
    const float4 a = ambY(P);
    Yc = make_float4((r * Yc.x + madd * a.x) / (r + madd), (r * Yc.y + madd * a.y) / (r + madd),
                     (r * Yc.z + madd * a.z) / (r + madd), (r * Yc.w + madd * a.w) / (r + madd));
    Tc = (r * Tc + madd * P.Tamb) / (r + madd);
    massSrc += me;
  }
  // :150-156
  Tc = fmaxf(Tc, 0.5f * P.Tamb);
  Yc = max4(Yc, make_float4(0.f, 0.f, 0.f, 0.f));
  o.S = massSrc / rhoOf(P, Tc) + logf(Tc / Tadv) / dt;
  o.T = Tc; o.Y = Yc; o.tpeak = Tc;
  return o;
}

}  // namespace

// NMAX: largest diffusion sub-step count this instantiation handles (halo NMAX)
template <int TX, int TY, int NMAX, bool SOURCES, bool DIFFUSION>
__global__ void __launch_bounds__(256) k_diffuse_sources(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work) {
  constexpr int RW = TX + 2 * NMAX, RH = TY + 2 * NMAX;
  // the ping-pong state of tile + halo in dynamic shared memory (ds_smem_bytes: above 48 KB for
  // the larger tiles at 5 sub-steps)
  extern __shared__ __align__(16) unsigned char ds_smem[];
  float4 (*sY)[RH * RW] = reinterpret_cast<float4 (*)[RH * RW]>(ds_smem);
  float (*sT)[RH * RW] = reinterpret_cast<float (*)[RH * RW]>(ds_smem + 2 * RH * RW * sizeof(float4));
  __shared__ float rq[TY * TX], rr[TY * TX], rt[TY * TX];

  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!S.enabled) return;
  const cfg_params& P = S.P;
  const int nx = S.nx, ny = S.ny, pc = S.pc, pu = S.pu;
  const int n = DIFFUSION ? min(S.diff_sub, NMAX) : 0;
  const int x0 = w.tx * TX, y0 = w.ty * TY;
  const int rx0 = x0 - NMAX, ry0 = y0 - NMAX;

  // ---- load the diffusion input on tile + n (T2/Y2: the advected state; or T/Y without diffusion)
  const float* Tin = DIFFUSION ? S.T2 : S.T;
  const float4* Yin = DIFFUSION ? S.Y2 : S.Y;
  for (int e = threadIdx.x; e < RH * RW; e += blockDim.x) {
    const int i = rx0 + e % RW, j = ry0 + e / RW;
    if (i < 0 || i >= nx || j < 0 || j >= ny) continue;
    if (i < x0 - n || i >= x0 + TX + n || j < y0 - n || j >= y0 + TY + n) continue;
    sT[0][e] = __ldg(Tin + j * pc + i);
    sY[0][e] = __ldg(Yin + j * pc + i);
  }
  __syncthreads();

  // ---- diffusion sub-steps (diffuse.wgsl:18-50), buffer ping-pong in shared memory
  const float c0 = S.diff_dt;
  int cur = 0;
  for (int s = 1; s <= n; s++) {
    const int xa = max(x0 - n + s, 0), xb = min(x0 + TX + n - s, nx);
    const int ya = max(y0 - n + s, 0), yb = min(y0 + TY + n - s, ny);
    const int W = xb - xa, Hh = yb - ya;
    const float* Ti = sT[cur]; const float4* Yi = sY[cur];
    float* To = sT[cur ^ 1]; float4* Yo = sY[cur ^ 1];
    for (int e = threadIdx.x; e < W * Hh; e += blockDim.x) {
      const int i = xa + e % W, j = ya + e / W;
      const int r = (j - ry0) * RW + (i - rx0);
      const float T0 = Ti[r]; const float4 Y0 = Yi[r];
      float sTa = 0.f; float sYx = 0.f, sYy = 0.f, sYz = 0.f;
      #define CFG_DIFF_FACE(fval, roff)                                          \
        {                                                                       \
          const float f = (fval);                                               \
          if (f > 0.f) {                                                        \
            const float Tn = Ti[r + (roff)]; const float4 Yn = Yi[r + (roff)];  \
            const float a = f * rhoDOf(P, 0.5f * (T0 + Tn));                    \
            sTa += a * (Tn - T0);                                               \
            sYx += a * (Yn.x - Y0.x); sYy += a * (Yn.y - Y0.y); sYz += a * (Yn.z - Y0.z); \
          }                                                                     \
        }
      if (i > 0) CFG_DIFF_FACE(__ldg(S.fx + j * pu + i), -1)
      if (i < nx - 1) CFG_DIFF_FACE(__ldg(S.fx + j * pu + i + 1), 1)
      if (j > 0) CFG_DIFF_FACE(__ldg(S.fy + j * pc + i), -RW)
      if (j < ny - 1) CFG_DIFF_FACE(__ldg(S.fy + (j + 1) * pc + i), RW)
      #undef CFG_DIFF_FACE
      const float c = c0 / (rhoOf(P, T0) * P.dx * P.dx);
      To[r] = T0 + c * sTa;
      Yo[r] = make_float4(fmaxf(Y0.x + c * sYx, 0.f), fmaxf(Y0.y + c * sYy, 0.f), fmaxf(Y0.z + c * sYz, 0.f), fmaxf(Y0.w, 0.f));
    }
    cur ^= 1;
    __syncthreads();
  }

  // ---- sources on the tile cells (or write the diffused state)
  const float Tamb4 = powf(P.Tamb, 4.f);
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    const int i = x0 + e % TX, j = y0 + e / TX;
    float q = 0.f, qr = 0.f, tp = 0.f;
    if (i < nx && j < ny) {
      const int r = (j - ry0) * RW + (i - rx0);
      const int k = j * pc + i;
      const float Tc = sT[cur][r]; const float4 Yc = sY[cur][r];
      if (SOURCES) {
        const SrcOut o = sources_cell(S, P, i, j, Tc, Yc, __ldg(S.T2 + k), Tamb4);
        S.T[k] = o.T; S.Y[k] = o.Y;
        S.SQ[k] = o.solid ? make_float2(0.f, 0.f) : make_float2(o.S, o.qrel);
        q = o.qrel; qr = o.qrad; tp = o.tpeak;
      } else {
        S.T[k] = Tc; S.Y[k] = Yc;
      }
    }
    if (SOURCES) { rq[e] = q * P.dx * P.dx * P.dt; rr[e] = qr * P.dx * P.dx * P.dt; rt[e] = tp; }
  }
  if (!SOURCES) return;
  __syncthreads();
  // ---- per-8x8-block tree reduction in the order of sources.wgsl:160-167 (one warp per block)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int NBX = TX / 8, NBY = TY / 8;
  for (int b = warp; b < NBX * NBY; b += blockDim.x >> 5) {
    const int bx = (b % NBX) * 8, by = (b / NBX) * 8;
    const int e1 = (by + (lane >> 3)) * TX + bx + (lane & 7);       // li = lane
    const int e2 = (by + 4 + (lane >> 3)) * TX + bx + (lane & 7);   // li = lane + 32
    float vq = rq[e1] + rq[e2], vr = rr[e1] + rr[e2], vt = fmaxf(rt[e1], rt[e2]);
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vq = vq + __shfl_down_sync(0xffffffffu, vq, o);
      vr = vr + __shfl_down_sync(0xffffffffu, vr, o);
      vt = fmaxf(vt, __shfl_down_sync(0xffffffffu, vt, o));
    }
    // a block entirely outside the domain still adds round(0) = 0, as the WGSL does
    if (lane == 0) {
      atomicAdd(S.acc + ACC_GLOBAL, wgsl_i32_round(vq * 1.0e3f));
      atomicAdd(S.acc + ACC_GLOBAL + 1, wgsl_i32_round(vr * 1.0e3f));
      atomicMax(S.acc + ACC_GLOBAL + 2, wgsl_i32(vt));
    }
  }
}

template <int TX, int TY, int NMAX>
constexpr size_t ds_smem_bytes() { return (size_t)2 * (TX + 2 * NMAX) * (TY + 2 * NMAX) * (sizeof(float4) + sizeof(float)); }

template <int TX, int TY, int NMAX, bool SRC, bool DIF>
static void ds_launch(const SceneDesc* scenes, const Work* work, int ntiles, cudaStream_t st) {
  k_diffuse_sources<TX, TY, NMAX, SRC, DIF><<<ntiles, 256, ds_smem_bytes<TX, TY, NMAX>(), st>>>(scenes, work);
}
template <int TX, int TY>
static void ds_launch_shape(const SceneDesc* scenes, const Work* work, int ntiles, int max_sub, bool with_sources,
                            bool with_diffusion, cudaStream_t st) {
  if (!with_diffusion) { ds_launch<TX, TY, 1, true, false>(scenes, work, ntiles, st); return; }
  if (with_sources) {
    if (max_sub <= 1) ds_launch<TX, TY, 1, true, true>(scenes, work, ntiles, st);
    else if (max_sub <= 3) ds_launch<TX, TY, 3, true, true>(scenes, work, ntiles, st);
    else ds_launch<TX, TY, 5, true, true>(scenes, work, ntiles, st);
  } else {
    if (max_sub <= 1) ds_launch<TX, TY, 1, false, true>(scenes, work, ntiles, st);
    else if (max_sub <= 3) ds_launch<TX, TY, 3, false, true>(scenes, work, ntiles, st);
    else ds_launch<TX, TY, 5, false, true>(scenes, work, ntiles, st);
  }
}
template <int TX, int TY, int NMAX>
static cudaError_t ds_allow_smem() {
  const int b = (int)ds_smem_bytes<TX, TY, NMAX>();
  cudaError_t e = cudaSuccess;
  for (cudaError_t x : {cudaFuncSetAttribute(k_diffuse_sources<TX, TY, NMAX, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b),
                        cudaFuncSetAttribute(k_diffuse_sources<TX, TY, NMAX, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b),
                        cudaFuncSetAttribute(k_diffuse_sources<TX, TY, NMAX, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b)})
    if (x != cudaSuccess && e == cudaSuccess) e = x;
  return e;
}
template <int TX, int TY>
static cudaError_t ds_allow_shape() {
  cudaError_t e = ds_allow_smem<TX, TY, 1>();
  if (e == cudaSuccess) e = ds_allow_smem<TX, TY, 3>();
  if (e == cudaSuccess) e = ds_allow_smem<TX, TY, 5>();
  return e;
}

// the dynamic shared memory every instantiation may use (once per device, before any launch)
cudaError_t prepare_diffuse_sources() {
  static_assert(TILE_TX[0] == DS_TX && TILE_TY[0] == DS_TY, "shape 0 is the default tile");
  cudaError_t e = ds_allow_shape<TILE_TX[0], TILE_TY[0]>();
  if (e == cudaSuccess) e = ds_allow_shape<TILE_TX[1], TILE_TY[1]>();
  if (e == cudaSuccess) e = ds_allow_shape<TILE_TX[2], TILE_TY[2]>();
  return e;
}

void launch_diffuse_sources(const SceneDesc* scenes, const Work* work, int ntiles, int max_sub, bool with_sources,
                            bool with_diffusion, int shape, cudaStream_t st) {
  if (ntiles <= 0) return;
  if (shape == 1) ds_launch_shape<TILE_TX[1], TILE_TY[1]>(scenes, work, ntiles, max_sub, with_sources, with_diffusion, st);
  else if (shape == 2) ds_launch_shape<TILE_TX[2], TILE_TY[2]>(scenes, work, ntiles, max_sub, with_sources, with_diffusion, st);
  else ds_launch_shape<DS_TX, DS_TY>(scenes, work, ntiles, max_sub, with_sources, with_diffusion, st);
}

}  // namespace cfg
