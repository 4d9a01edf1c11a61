// Advection stage: scalForward + scalCorrect + velForward + velCorrect of
// shaders/advect.wgsl:36-103 in one kernel per tile.
//
// The first-order values Th, Yh, Uh, Vh (advect.wgsl:68-76, 36-47) exist only
// in shared memory: each CTA computes them on its tile plus a halo of H cells,
// then applies the MacCormack correction (:78-103, :49-66) to its own cells and
// faces. A forward-trace sample that lands outside the halo (a displacement of
// H cells or more) recomputes the first-order value from global memory, so the
// result does not depend on the time step. Global traffic per cell: U, V, T, Y
// read (through L1), T2, Y2, U2, V2 written; the 40 bytes/cell of Th/Yh and
// 8 bytes/face of Uh/Vh of the reference schedule never reach HBM.
#include "gas_dev.cuh"
#include "kernels.h"

namespace cfg {

namespace {

// at(i, j): the first-order value from shared memory, recomputed from global memory outside
// the staged region; quad(i, j, ...): the 2x2 block straight from shared memory when all four
// corners are inside the level (no boundary rule applies) and inside the staged region
__device__ __forceinline__ bool staged_block(int i, int j, int nx1, int ny1, int rx0, int ry0, int RW, int RH) {
  return (unsigned)i < (unsigned)nx1 && (unsigned)j < (unsigned)ny1 && (unsigned)(i - rx0) < (unsigned)(RW - 1) &&
         (unsigned)(j - ry0) < (unsigned)(RH - 1);
}
struct ThLookup {
  const float* sm; int rx0, ry0, RW, RH; const VelSampler* vs; const CField* T; float dt;
  __device__ __forceinline__ bool quad(int i, int j, float& A, float& C, float& D, float& E) const {
    if (!staged_block(i, j, T->nx - 1, T->ny - 1, rx0, ry0, RW, RH)) return false;
    const float* q = sm + (j - ry0) * RW + (i - rx0);
    A = q[0]; C = q[1]; D = q[RW]; E = q[RW + 1];
    return true;
  }
  __device__ __forceinline__ float at(int i, int j) const {
    if (i < 0 || i >= T->nx || j >= T->ny) return T->amb;
    j = max(j, 0);
    const int ri = i - rx0, rj = j - ry0;
    if (ri >= 0 && ri < RW && rj >= 0 && rj < RH) return sm[rj * RW + ri];
    float ox, oy; vs->trace((float)i + 0.5f, (float)j + 0.5f, dt, ox, oy);
    return sample(*T, ox, oy, 0.5f, 0.5f);
  }
};
struct YhLookup {
  const float4* sm; int rx0, ry0, RW, RH; const VelSampler* vs; const C4Field* Y; float dt;
  __device__ __forceinline__ bool quad(int i, int j, float4& A, float4& C, float4& D, float4& E) const {
    if (!staged_block(i, j, Y->nx - 1, Y->ny - 1, rx0, ry0, RW, RH)) return false;
    const float4* q = sm + (j - ry0) * RW + (i - rx0);
    A = q[0]; C = q[1]; D = q[RW]; E = q[RW + 1];
    return true;
  }
  __device__ __forceinline__ float4 at(int i, int j) const {
    if (i < 0 || i >= Y->nx || j >= Y->ny) return Y->amb;
    j = max(j, 0);
    const int ri = i - rx0, rj = j - ry0;
    if (ri >= 0 && ri < RW && rj >= 0 && rj < RH) return sm[rj * RW + ri];
    float ox, oy; vs->trace((float)i + 0.5f, (float)j + 0.5f, dt, ox, oy);
    return sample4(*Y, ox, oy);
  }
};
struct UhLookup {
  const float* sm; int rx0, ry0, RW, RH; const VelSampler* vs; float dt;
  __device__ __forceinline__ bool quad(int i, int j, float& A, float& C, float& D, float& E) const {
    if (!staged_block(i, j, vs->u.nx, vs->u.ny - 1, rx0, ry0, RW, RH)) return false;
    const float* q = sm + (j - ry0) * RW + (i - rx0);
    A = q[0]; C = q[1]; D = q[RW]; E = q[RW + 1];
    return true;
  }
  __device__ __forceinline__ float at(int i, int j) const {
    const UField& u = vs->u;
    if (i < 0 || i > u.nx || j >= u.ny) return 0.f;
    float sgn = 1.f;
    if (j < 0) { j = 0; sgn = -1.f; }
    const int ri = i - rx0, rj = j - ry0;
    float v;
    if (ri >= 0 && ri < RW && rj >= 0 && rj < RH) v = sm[rj * RW + ri];
    else { float ox, oy; vs->trace((float)i, (float)j + 0.5f, dt, ox, oy); v = sample(u, ox, oy, 0.f, 0.5f); }
    return sgn < 0.f ? -v : v;
  }
};
struct VhLookup {
  const float* sm; int rx0, ry0, RW, RH; const VelSampler* vs; float dt;
  __device__ __forceinline__ bool quad(int i, int j, float& A, float& C, float& D, float& E) const {
    if (!staged_block(i, j, vs->v.nx - 1, vs->v.ny, rx0, ry0, RW, RH)) return false;
    const float* q = sm + (j - ry0) * RW + (i - rx0);
    A = q[0]; C = q[1]; D = q[RW]; E = q[RW + 1];
    return true;
  }
  __device__ __forceinline__ float at(int i, int j) const {
    const VField& v = vs->v;
    if (i < 0 || i >= v.nx || j > v.ny) return 0.f;
    j = max(j, 0);
    const int ri = i - rx0, rj = j - ry0;
    if (ri >= 0 && ri < RW && rj >= 0 && rj < RH) return sm[rj * RW + ri];
    float ox, oy; vs->trace((float)i + 0.5f, (float)j, dt, ox, oy);
    return sample(v, ox, oy, 0.5f, 0.f);
  }
};

}  // namespace

// four CTAs per SM (64 registers, 20 bytes of spill; 80 registers and three CTAs without the
// bound): 512x768 -0.7% per step, the 64-scene batch -0.3%, 256x384 (one wave either way) unchanged
template <int TX, int TY, int H>
__global__ void __launch_bounds__(256, 4) k_advect(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work) {
  constexpr int RW = TX + 2 * H, RH = TY + 2 * H;            // cell region
  constexpr int UW = RW + 1, UH = RH;                          // U-face region
  constexpr int VW = RW, VH = RH + 1;                          // V-face region
  __shared__ float sTh[RH * RW];
  __shared__ float4 sYh[RH * RW];
  __shared__ float2 sDc[RH * RW];
  __shared__ float sUh[UH * UW];
  __shared__ float2 sDu[UH * UW];
  __shared__ float sVh[VH * VW];
  __shared__ float2 sDv[VH * VW];

  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!S.enabled) return;
  const int nx = S.nx, ny = S.ny, pc = S.pc, pu = S.pu;
  const float dt = S.P.dt, dx = S.P.dx;
  const int x0 = w.tx * TX, y0 = w.ty * TY;
  const int rx0 = x0 - H, ry0 = y0 - H;

  VelSampler vs;
  vs.u = UField{S.U, nx, ny, pu};
  vs.v = VField{S.V, nx, ny, pc};
  vs.dx = dx;
  vs.rdx = __frcp_rn(dx);
  const CField Tf{S.T, nx, ny, pc, S.P.Tamb};
  const C4Field Yf{S.Y, nx, ny, pc, ambY(S.P)};

  // ---- first-order (forward) values on tile + halo (advect.wgsl:36-47, 68-76)
  for (int e = threadIdx.x; e < RH * RW; e += blockDim.x) {
    const int ri = e % RW, rj = e / RW, i = rx0 + ri, j = ry0 + rj;
    if (i < 0 || i >= nx || j < 0 || j >= ny) continue;
    float ox, oy; vs.trace((float)i + 0.5f, (float)j + 0.5f, dt, ox, oy);
    sTh[e] = sample(Tf, ox, oy, 0.5f, 0.5f);
    sYh[e] = sample4(Yf, ox, oy);
    sDc[e] = make_float2(ox, oy);
  }
  for (int e = threadIdx.x; e < UH * UW; e += blockDim.x) {
    const int ri = e % UW, rj = e / UW, i = rx0 + ri, j = ry0 + rj;
    if (i < 0 || i > nx || j < 0 || j >= ny) continue;
    float ox, oy; vs.trace((float)i, (float)j + 0.5f, dt, ox, oy);
    sUh[e] = sample(vs.u, ox, oy, 0.f, 0.5f);
    sDu[e] = make_float2(ox, oy);
  }
  for (int e = threadIdx.x; e < VH * VW; e += blockDim.x) {
    const int ri = e % VW, rj = e / VW, i = rx0 + ri, j = ry0 + rj;
    if (i < 0 || i >= nx || j < 0 || j > ny) continue;
    float ox, oy; vs.trace((float)i + 0.5f, (float)j, dt, ox, oy);
    sVh[e] = sample(vs.v, ox, oy, 0.5f, 0.f);
    sDv[e] = make_float2(ox, oy);
  }
  __syncthreads();

  const ThLookup Th{sTh, rx0, ry0, RW, RH, &vs, &Tf, dt};
  const YhLookup Yh{sYh, rx0, ry0, RW, RH, &vs, &Yf, dt};
  const UhLookup Uh{sUh, rx0, ry0, UW, UH, &vs, dt};
  const VhLookup Vh{sVh, rx0, ry0, VW, VH, &vs, dt};
  const float sO2 = S.P.sO2;

  // ---- scalCorrect (advect.wgsl:78-103)
  for (int e = threadIdx.x; e < TX * TY; e += blockDim.x) {
    const int i = x0 + e % TX, j = y0 + e / TX;
    if (i >= nx || j >= ny) continue;
    const int r = (j - ry0) * RW + (i - rx0);
    const int k = j * pc + i;
    const float gx = (float)i + 0.5f, gy = (float)j + 0.5f;
    const float2 d = sDc[r];
    float fx_, fy_; vs.trace(gx, gy, -dt, fx_, fy_);
    float tlo, thi; minmax(Tf, d.x, d.y, 0.5f, 0.5f, tlo, thi);
    float4 ylo, yhi; minmax4(Yf, d.x, d.y, ylo, yhi);
    const float th = sTh[r]; const float4 yh = sYh[r];
    const float Tc = th + 0.5f * (__ldg(S.T + k) - sample(Th, fx_, fy_, 0.5f, 0.5f));
    const float4 y0v = __ldg(S.Y + k);
    const float4 sb = sample4(Yh, fx_, fy_);
    const float4 Yc = make_float4(yh.x + 0.5f * (y0v.x - sb.x), yh.y + 0.5f * (y0v.y - sb.y),
                                  yh.z + 0.5f * (y0v.z - sb.z), yh.w + 0.5f * (y0v.w - sb.w));
    const bool inT = Tc >= tlo && Tc <= thi;
    const bool inY = Yc.x >= ylo.x && Yc.y >= ylo.y && Yc.z >= ylo.z && Yc.w >= ylo.w &&
                     Yc.x <= yhi.x && Yc.y <= yhi.y && Yc.z <= yhi.z && Yc.w <= yhi.w;
    const float mixC = fminf(Yc.x, Yc.y / sO2);
    const float mixL = fminf(yh.x, yh.y / sO2);
    if (inT && inY && mixC <= mixL + 1e-5f) { S.T2[k] = Tc; S.Y2[k] = Yc; }
    else { S.T2[k] = th; S.Y2[k] = yh; }
  }
  // ---- velCorrect, U faces (advect.wgsl:52-58): this tile owns x in [x0, x0+TX), plus x = nx at the east edge
  const int uxe = (x0 + TX >= nx) ? nx + 1 : x0 + TX;
  const int UTW = uxe - x0;
  for (int e = threadIdx.x; e < UTW * TY; e += blockDim.x) {
    const int i = x0 + e % UTW, j = y0 + e / UTW;
    if (j >= ny) continue;
    const int r = (j - ry0) * UW + (i - rx0);
    const int k = j * pu + i;
    const float gx = (float)i, gy = (float)j + 0.5f;
    float bx_, by_; vs.trace(gx, gy, -dt, bx_, by_);
    const float back = sample(Uh, bx_, by_, 0.f, 0.5f);
    const float2 d = sDu[r];
    float lo, hi; minmax(vs.u, d.x, d.y, 0.f, 0.5f, lo, hi);
    S.U2[k] = clampf(sUh[r] + 0.5f * (__ldg(S.U + k) - back), lo, hi);
  }
  // ---- velCorrect, V faces (advect.wgsl:59-65): y in [y0, y0+TY), plus y = ny at the top edge
  const int vye = (y0 + TY >= ny) ? ny + 1 : y0 + TY;
  const int VTH = vye - y0;
  for (int e = threadIdx.x; e < TX * VTH; e += blockDim.x) {
    const int i = x0 + e % TX, j = y0 + e / TX;
    if (i >= nx) continue;
    const int r = (j - ry0) * VW + (i - rx0);
    const int k = j * pc + i;
    const float gx = (float)i + 0.5f, gy = (float)j;
    float bx_, by_; vs.trace(gx, gy, -dt, bx_, by_);
    const float back = sample(Vh, bx_, by_, 0.5f, 0.f);
    const float2 d = sDv[r];
    float lo, hi; minmax(vs.v, d.x, d.y, 0.5f, 0.f, lo, hi);
    S.V2[k] = clampf(sVh[r] + 0.5f * (__ldg(S.V + k) - back), lo, hi);
  }
}

void launch_advect(const SceneDesc* scenes, const Work* work, int ntiles, int shape, cudaStream_t st) {
  if (ntiles <= 0) return;
  static_assert(TILE_TX[0] == ADV_TX && TILE_TY[0] == ADV_TY, "shape 0 is the default tile");
  if (shape == 1) k_advect<TILE_TX[1], TILE_TY[1], ADV_H><<<ntiles, 256, 0, st>>>(scenes, work);
  else if (shape == 2) k_advect<TILE_TX[2], TILE_TY[2], ADV_H><<<ntiles, 256, 0, st>>>(scenes, work);
  else k_advect<ADV_TX, ADV_TY, ADV_H><<<ntiles, 256, 0, st>>>(scenes, work);
}

}  // namespace cfg
