// Projection (pressure.wgsl:159-180), the CFL step update, geometry
// rasterisation (geometry.wgsl), radiation to wood faces (radiation.wgsl) and
// the FP64 budget sums.
#include "gas_dev.cuh"
#include "kernels.h"
#include "reduce.cuh"

namespace cfg {

// u -= dt (1/rho_f) grad p; ghost -p at the open sides/top, closed faces 0.
// FP64: the FP64 pressure of the defect-correction loop, rounded once to f32.
// CFL step for the next step: dt = min(dt_cap, cfl*dx/max|u|) and the diffusion
// sub-step count of js/fluid.js:190-198 for that dt (one thread, after max|u| is complete)
// advance_clock: the step's own dt (P.dt, before it is replaced) is added to the scene's clock
__device__ __forceinline__ void cfl_next_dt(SceneDesc& S, double h, double alpha, bool advance_clock) {
  if (advance_clock) S.solve->time += (double)S.P.dt;
  const float m = __uint_as_float(S.solve->maxu);
  const float cand = m > 0.f ? S.cfl * S.P.dx / m : S.dt_cap;
  const float dt = fminf(S.dt_cap, cand);
  S.P.dt = dt;
  int n = (int)ceil((double)dt / (h * h / (4.5 * alpha)));
  n = min(5, n % 2 ? n : n + 1);
  S.diff_sub = n;
  S.diff_dt = (float)((double)dt / n);
  S.solve->maxu = 0u;
}

// post (the step's tail folded into the projection): bit 0 swaps every scene's coarsest
// inverse halves (after the factorisation's branch has joined), bit 1 sets each CFL scene's
// next dt in the scene's last CTA (arrival on the scene's counter after its max|u|).
template <bool FP64>
__global__ void __launch_bounds__(256) k_project(SceneDesc* __restrict__ scenes, const Work* __restrict__ work, int nscenes,
                                                 int post, const double* dxd, const double* alpha, float* dtv) {
  __shared__ float redm[32];
  __shared__ int s_last;
  const Work w = work[blockIdx.x];
  if ((post & 1) && blockIdx.x == 0)
    for (int s = threadIdx.x; s < nscenes; s += blockDim.x) {
      const SceneDesc& Q = scenes[s];
      if (!Q.enabled) continue;
      SolveState* ss = Q.solve;
      ss->cinv_cur ^= 1;
      ss->direct_ok = ss->direct_ok_next;
      ss->direct_ok_next = 0;
    }
  SceneDesc& S = scenes[w.scene];
  if (!S.enabled) return;
  const cfg_params& P = S.P;
  const int nx = S.nx, ny = S.ny, pc = S.pc, pu = S.pu;
  const LevelDesc L0 = S.lev[0];
  const float* p = L0.p;
  const double* p64 = S.p64;
  const float dt = P.dt, dx = P.dx, rT = P.rhoAmb * P.Tamb;
  const int i = w.tx * PR_TX + (threadIdx.x % PR_TX), j = w.ty * PR_TY + (threadIdx.x / PR_TX);
  auto pf = [&](int a, int b) { return p[b * L0.pc + a]; };
  auto pd = [&](int a, int b) { return p64[b * nx + a]; };
  auto Tat = [&](int a, int b) { return __ldg(S.T + b * pc + a); };
  float m = 0.f;
  auto uface = [&](int a, int b) {
    const int k = b * pu + a;
    float u;
    if (__ldg(S.fx + k) > 0.f) {
      if (FP64) {
        const double Tf = 0.5 * ((double)Tat(min(max(a - 1, 0), nx - 1), b) + (double)Tat(min(a, nx - 1), b));
        const double pl = a > 0 ? pd(a - 1, b) : -pd(0, b);
        const double pr = a < nx ? pd(min(a, nx - 1), b) : -pd(nx - 1, b);
        u = (float)((double)S.U[k] - (double)dt * (Tf / (double)rT) * (pr - pl) / (double)dx);
      } else {
        const float Tf = 0.5f * (Tat(min(max(a - 1, 0), nx - 1), b) + Tat(min(a, nx - 1), b));
        const float pl = a > 0 ? pf(max(a - 1, 0), b) : -pf(0, b);
        const float pr = a < nx ? pf(min(a, nx - 1), b) : -pf(nx - 1, b);
        u = S.U[k] - dt * (Tf / rT) * (pr - pl) / dx;
      }
    } else u = 0.f;
    S.U[k] = u;
    m = fmaxf(m, fabsf(u));
  };
  auto vface = [&](int a, int b) {
    const int k = b * pc + a;
    float v;
    if (b > 0 && __ldg(S.fy + k) > 0.f) {
      if (FP64) {
        const double Tf = 0.5 * ((double)Tat(a, b - 1) + (double)Tat(a, min(b, ny - 1)));
        const double pb = pd(a, b - 1);
        const double pt = b < ny ? pd(a, min(b, ny - 1)) : -pd(a, ny - 1);
        v = (float)((double)S.V[k] - (double)dt * (Tf / (double)rT) * (pt - pb) / (double)dx);
      } else {
        const float Tf = 0.5f * (Tat(a, b - 1) + Tat(a, min(b, ny - 1)));
        const float pb = pf(a, b - 1);
        const float pt = b < ny ? pf(a, min(b, ny - 1)) : -pf(a, ny - 1);
        v = S.V[k] - dt * (Tf / rT) * (pt - pb) / dx;
      }
    } else v = 0.f;
    S.V[k] = v;
    m = fmaxf(m, fabsf(v));
  };
  if (i < nx && j < ny) {
    uface(i, j);
    vface(i, j);
    if (i == nx - 1) uface(nx, j);
    if (j == ny - 1) vface(i, ny);
  }
  const float bm = block_max(m, redm);
  if (threadIdx.x == 0 && S.cfl > 0.f) atomicMax(&S.solve->maxu, __float_as_uint(bm));
  if (!(post & 2) || !(S.cfl > 0.f)) return;
  // every CTA of the scene has read P.dt and added its max|u| before it arrives
  if (threadIdx.x == 0) s_last = arrive_acq_rel(&S.solve->counter) == (unsigned)S.nt_mg0 - 1u;
  __syncthreads();
  if (s_last && threadIdx.x == 0) {
    S.solve->counter = 0u;
    cfl_next_dt(S, dxd[w.scene], alpha[w.scene], true);
    if (dtv) {   // pinned host memory: visible to the host once the step's event has passed
      dtv[w.scene] = S.P.dt;
      __threadfence_system();
    }
  }
}

// the CFL update on its own (one thread per scene)
__global__ void k_cfl_update(SceneDesc* scenes, int nscenes, const double* dxd, const double* alpha) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nscenes) return;
  SceneDesc& S = scenes[s];
  if (!S.enabled || !(S.cfl > 0.f)) return;
  cfl_next_dt(S, dxd[s], alpha[s], false);
}

// geometry.wgsl:121-153: per cell the nearest piece (sdf, piece*4+face) and the
// band weight; per face the open fraction. Tiles cover (nx+1) x (ny+1) sites.
__global__ void __launch_bounds__(256) k_geometry(const SceneDesc* __restrict__ scenes, const Work* __restrict__ work) {
  __shared__ Piece sp[MAX_PIECES];
  const Work w = work[blockIdx.x];
  const SceneDesc& S = scenes[w.scene];
  if (!S.enabled) return;
  const cfg_params& P = S.P;
  const int np = min(max(P.nPieces, 0), MAX_PIECES);
  for (int e = threadIdx.x; e < np * PIECE_FLOATS; e += blockDim.x)
    reinterpret_cast<float*>(sp)[e] = S.pieces[e];
  __syncthreads();
  const int nx = S.nx, ny = S.ny;
  const float dx = P.dx;
  const int i = w.tx * GEO_TX + (threadIdx.x % GEO_TX), j = w.ty * GEO_TY + (threadIdx.x / GEO_TX);
  auto nearest = [&](float px, float py, float& best, uint32_t& bid) {
    best = 1e9f; bid = SOLID_NONE;
    for (int n = 0; n < np; n++) {
      const Piece& pc = sp[n];
      if (pc.alive <= 0.f) continue;
      const float d = sdBox(px, py, pc);
      if (d < best) { best = d; bid = (uint32_t)n * 4u + faceOf(px, py, pc); }
    }
  };
  if (i < nx && j < ny) {
    float best; uint32_t bid;
    nearest(((float)i + 0.5f) * dx, ((float)j + 0.5f) * dx, best, bid);
    S.cellG[j * S.pc + i] = make_float2(best, __uint_as_float(bid));
    if (bid != SOLID_NONE && best >= 0.f && best < 2.f * dx) {
      const float wgt = fmaxf(0.f, 1.f - fabsf(best - dx) / dx) / dx;
      atomicAdd(S.faceW + bid, wgsl_i32_round(wgt * dx * dx * 1.0e8f));
    }
  }
  if (i <= nx && j < ny) {
    float d; uint32_t b; nearest((float)i * dx, ((float)j + 0.5f) * dx, d, b);
    S.fx[j * S.pu + i] = clampf(0.5f + d / dx, 0.f, 1.f);
  }
  if (i < nx && j <= ny) {
    float d; uint32_t b; nearest(((float)i + 0.5f) * dx, (float)j * dx, d, b);
    S.fy[j * S.pc + i] = j == 0 ? 0.f : clampf(0.5f + d / dx, 0.f, 1.f);
  }
}

// ---------------------------------------------------------------- radiation.wgsl
namespace {
__device__ __forceinline__ float planck580(float t) {   // :28-33
  const float l = 580e-9f;
  const float x = 1.438777e-2f / (l * t);
  if (x > 80.f) return 0.f;
  return 1.191042e-16f / (l * l * l * l * l) / (expf(x) - 1.f) * 1e-9f;
}
// :36-51 ray vs rotated box: t_enter (or < 0) and the face hit
__device__ __forceinline__ void hitBox(float ox, float oy, float dxr, float dyr, const Piece& pc, float& tn_out, float& face) {
  const float c = cosf(pc.angle), s = sinf(pc.angle);
  const float qx = ox - pc.pos[0], qy = oy - pc.pos[1];
  const float lox = c * qx + s * qy, loy = -s * qx + c * qy;
  const float ldx = c * dxr + s * dyr, ldy = -s * dxr + c * dyr;
  const float h = pc.half;
  const float invx = 1.f / (fabsf(ldx) < 1e-9f ? 1e-9f : ldx);
  const float invy = 1.f / (fabsf(ldy) < 1e-9f ? 1e-9f : ldy);
  const float t1x = (-h - lox) * invx, t1y = (-h - loy) * invy;
  const float t2x = (h - lox) * invx, t2y = (h - loy) * invy;
  const float tminx = fminf(t1x, t2x), tminy = fminf(t1y, t2y);
  const float tmaxx = fmaxf(t1x, t2x), tmaxy = fmaxf(t1y, t2y);
  const float tn = fmaxf(tminx, tminy), tf = fminf(tmaxx, tmaxy);
  if (tf < 0.f || tn > tf || tn < 1e-5f) { tn_out = -1.f; face = 0.f; return; }
  if (tminx > tminy) face = ldx < 0.f ? 0.f : 2.f; else face = ldy < 0.f ? 1.f : 3.f;
  tn_out = tn;
}
__device__ __forceinline__ float fractf(float x) { return x - floorf(x); }
}  // namespace

// :64-158 one CTA of nray rays per wood face or floor probe
__global__ void __launch_bounds__(1024) k_radiation(const SceneDesc* __restrict__ scenes, int scene) {
  __shared__ Piece sp[MAX_PIECES];
  __shared__ float sq[1024], sv[1024];
  const SceneDesc& S = scenes[scene];
  const cfg_params& P = S.P;
  const int np = min(max(P.nPieces, 0), MAX_PIECES);
  for (int e = threadIdx.x; e < np * PIECE_FLOATS; e += blockDim.x)
    reinterpret_cast<float*>(sp)[e] = S.pieces[e];
  __syncthreads();
  const float PI = 3.14159265f;
  const int NRAY = blockDim.x;
  const uint32_t tgt = blockIdx.x, li = threadIdx.x;
  const uint32_t nFaces = (uint32_t)np * 4u;
  const int nx = S.nx, ny = S.ny, pcw = S.pc;
  const float dx = P.dx;
  float ox0 = 0.f, oy0 = 0.f, nrx = 0.f, nry = 1.f;
  bool valid = false;
  if (tgt < nFaces) {
    const Piece& pc = sp[tgt / 4u];
    const uint32_t f = tgt % 4u;
    if (pc.alive > 0.f) {
      const float c = cosf(pc.angle), s = sinf(pc.angle);
      float lnx = 1.f, lny = 0.f;
      if (f == 1u) { lnx = 0.f; lny = 1.f; } else if (f == 2u) { lnx = -1.f; lny = 0.f; } else if (f == 3u) { lnx = 0.f; lny = -1.f; }
      nrx = c * lnx - s * lny; nry = s * lnx + c * lny;
      const float tx = -nry, ty = nrx;
      const float u = (fractf((float)li * 0.618034f + (float)P.frame * 0.1234f) - 0.5f) * 1.6f * pc.half;
      const float hh = pc.half + 1e-4f;
      ox0 = pc.pos[0] + nrx * hh + tx * u; oy0 = pc.pos[1] + nry * hh + ty * u;
      valid = true;
    }
  } else {
    const uint32_t fi = tgt - nFaces;
    if (fi < (uint32_t)N_FLOOR) {
      ox0 = ((float)fi + 0.5f) / (float)N_FLOOR * (float)P.nx * dx; oy0 = 1e-4f;
      nrx = 0.f; nry = 1.f; valid = true;
    }
  }
  float dq = 0.f, dv = 0.f;
  if (valid) {
    const float jit = fractf((float)P.frame * 0.7548777f + (float)tgt * 0.5698403f);
    const float a = (((float)li + jit) / (float)NRAY - 0.5f) * PI;
    const float cosn = cosf(a);
    const float base = atan2f(nry, nrx);
    float ddx = cosf(base + a), ddy = sinf(base + a);
    float ox = ox0, oy = oy0;
    float J = 0.f, Jv = 0.f, Twall = P.Tamb;
    bool bounced = false;
    const float ds = dx;
    const float T4a = powf(P.Tamb, 4.f);
    for (int step = 0; step < 4096; step++) {
      float tHit = 1e9f, hitT = 0.f;
      for (int n = 0; n < np; n++) {
        const Piece& pc = sp[n];
        if (pc.alive <= 0.f) continue;
        float hx, hy; hitBox(ox, oy, ddx, ddy, pc, hx, hy);
        if (hx > 0.f && hx < tHit) { tHit = hx; hitT = pc.Ts[(uint32_t)hy]; }
      }
      float tFloor = 1e9f;
      if (ddy < -1e-6f) tFloor = -oy / ddy;
      const float tEnd = fminf(tHit, tFloor);
      const float W = (float)P.nx * dx, H = (float)P.ny * dx;
      float tx = 1e9f, ty = 1e9f;
      if (ddx > 1e-6f) tx = (W - ox) / ddx; else if (ddx < -1e-6f) tx = -ox / ddx;
      if (ddy > 1e-6f) ty = (H - oy) / ddy;
      const float tOut = fminf(fminf(tx, ty), tEnd);
      const int ns = wgsl_i32(ceilf(tOut / ds));
      for (int m = 0; m < ns; m++) {
        const float t = ((float)m + 0.5f) * tOut / (float)ns;
        const float px = ox + ddx * t, py = oy + ddy * t;
        const int gi = wgsl_i32(px / dx), gj = wgsl_i32(py / dx);
        float gx = 0.f, gy = 0.f;
        if (!(gi < 0 || gj < 0 || gi >= nx || gj >= ny)) {   // gasAt (:53-62)
          const int k = gj * pcw + gi;
          const float Tg = __ldg(S.T + k); const float4 Yg = __ldg(S.Y + k);
          const float fv = rhoOf(P, Tg) * Yg.w / P.sootDensity;
          const float kap = P.kappaSootC * fv * Tg + P.kappaGas * Yg.z;
          const float T2v = Tg * Tg;
          gx = kap * P.sigma * (T2v * T2v - T4a) / 3.14159265f;
          gy = 6.3f * fv / 580e-9f * planck580(Tg);
        }
        J += gx * tOut / (float)ns;
        Jv += gy * tOut / (float)ns;
      }
      if (tHit < tFloor && tHit < 1e8f) { Twall = hitT; break; }
      if (tFloor < 1e8f && tFloor <= tHit && !bounced) {
        ox = ox + ddx * tFloor; oy = oy + ddy * tFloor + 1e-5f;
        ddy = -ddy;
        bounced = true;
        continue;
      }
      Twall = P.Tamb;
      break;
    }
    const float wgt = PI / (float)NRAY * cosn;
    const float T2v = Twall * Twall;
    dq = wgt * (0.5f * P.sigma * T2v * T2v + 2.f * J);
    dv = wgt * (2.f * Jv);
  }
  sq[li] = dq; sv[li] = dv;
  __syncthreads();
  for (int s = NRAY / 2; s > 0; s >>= 1) {
    if ((int)li < s) { sq[li] += sq[li + s]; sv[li] += sv[li + s]; }
    __syncthreads();
  }
  if (li == 0 && valid) {
    const float4 old = S.rad[tgt];
    const float al = old.x <= 0.f ? 1.f : 0.35f;
    S.rad[tgt] = make_float4(mixf(old.x, sq[0], al), mixf(old.y, sv[0], al), 0.f, 0.f);
  }
}

// FP64 budgets over gas cells of one scene
__global__ void __launch_bounds__(1024) k_budgets(const SceneDesc* __restrict__ scenes, int scene, double* out) {
  __shared__ double red[32];
  __shared__ float redm[32];
  const SceneDesc& S = scenes[scene];
  const cfg_params& P = S.P;
  const double cellA = (double)P.dx * (double)P.dx;
  double v[7] = {0, 0, 0, 0, 0, 0, 0};
  float tmax = 0.f;
  for (int e = threadIdx.x; e < S.nx * S.ny; e += blockDim.x) {
    const int i = e % S.nx, j = e / S.nx, k = j * S.pc + i;
    const float2 g = S.cellG[k];
    if (g.x < 0.f && __float_as_uint(g.y) != SOLID_NONE) continue;
    const double t = (double)S.T[k];
    const double rho = (double)P.rhoAmb * (double)P.Tamb / t;
    const float4 y = S.Y[k];
    v[0] += rho * cellA; v[1] += rho * (double)P.cp * t * cellA;
    v[2] += rho * (double)y.x * cellA; v[3] += rho * (double)y.y * cellA;
    v[4] += rho * (double)y.z * cellA; v[5] += rho * (double)y.w * cellA;
    v[6] += (double)S.SQ[k].y * cellA;
    tmax = fmaxf(tmax, S.T[k]);
  }
  for (int q = 0; q < 7; q++) {
    const double t = block_sum(v[q], red);
    if (threadIdx.x == 0) out[q] = t;
  }
  const float tm = block_max(tmax, redm);
  if (threadIdx.x == 0) out[7] = (double)tm;
}

// ------------------------------------------------------------------ host blocks by value, readback
// A scene's parameter block (writeParams, js/fluid.js:180-199) and its pieces (uploadPieces,
// js/fluid.js:201-204) arrive as kernel parameters: one launch each instead of copy-engine
// transfers beside the compute stream, and the host's copy is free again once the launch returns.
// k_write_params leaves out word `skip` and words [s0, s1) (the step-owned dt and diffusion
// sub-steps of a CFL scene; -1: none).
__global__ void k_write_params(uint32_t* __restrict__ dst, const ParamWords b, int skip, int s0, int s1) {
  for (int k = threadIdx.x; k < PARAM_WORDS; k += blockDim.x)
    if (k != skip && (k < s0 || k >= s1)) dst[k] = b.w[k];
}
__global__ void k_write_pieces(float* __restrict__ dst, const PieceFloats b) {
  for (int k = threadIdx.x; k < MAX_PIECES * PIECE_FLOATS; k += blockDim.x) dst[k] = b.f[k];
}
// The readback (js/fluid.js:315-342): nwords words from src into pinned host memory mapped into the
// device's address space, then the first nzero of them (the accumulators) cleared on the device;
// each thread clears only words it has read. The host reads the slot after the event that follows.
__global__ void k_readback(uint32_t* __restrict__ src, uint32_t* __restrict__ host, int nwords, int nzero) {
  for (int k = threadIdx.x; k < nwords; k += blockDim.x) {
    host[k] = src[k];
    if (k < nzero) src[k] = 0u;
  }
  __threadfence_system();
}

void launch_write_params(uint32_t* dst, const ParamWords& b, int skip, int s0, int s1, cudaStream_t st) {
  k_write_params<<<1, 64, 0, st>>>(dst, b, skip, s0, s1);
}
void launch_write_pieces(float* dst, const PieceFloats& b, cudaStream_t st) {
  k_write_pieces<<<1, 256, 0, st>>>(dst, b);
}
void launch_readback(uint32_t* src, uint32_t* host, int nwords, int nzero, cudaStream_t st) {
  k_readback<<<1, 512, 0, st>>>(src, host, nwords, nzero);
}
void launch_project(SceneDesc* scenes, const Work* work, int ntiles, bool fp64, cudaStream_t st, int nscenes, int post,
                    const double* dxd, const double* alpha, float* dtv) {
  if (ntiles <= 0) return;
  if (fp64) k_project<true><<<ntiles, PR_TX * PR_TY, 0, st>>>(scenes, work, nscenes, post, dxd, alpha, dtv);
  else k_project<false><<<ntiles, PR_TX * PR_TY, 0, st>>>(scenes, work, nscenes, post, dxd, alpha, dtv);
}
void launch_cfl_update(SceneDesc* scenes, int nscenes, const double* dxd, const double* alpha, cudaStream_t st) {
  if (nscenes > 0) k_cfl_update<<<(nscenes + 127) / 128, 128, 0, st>>>(scenes, nscenes, dxd, alpha);
}
void launch_geometry(const SceneDesc* scenes, const Work* work, int ntiles, cudaStream_t st) {
  if (ntiles > 0) k_geometry<<<ntiles, GEO_TX * GEO_TY, 0, st>>>(scenes, work);
}
void launch_radiation(const SceneDesc* scenes, int scene, int ntargets, int nray, cudaStream_t st) {
  if (ntargets > 0) k_radiation<<<ntargets, nray, 0, st>>>(scenes, scene);
}
void launch_budgets(const SceneDesc* scenes, int scene, double* out, cudaStream_t st) {
  k_budgets<<<1, 1024, 0, st>>>(scenes, scene, out);
}

}  // namespace cfg
