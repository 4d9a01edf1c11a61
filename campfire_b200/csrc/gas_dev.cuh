// Shared device/host definitions of the B200 gas step.
//
// Every kernel is batched over scenes: it receives the device array of
// SceneDesc and a work list of tiles (scene, tile x, tile y). A single
// FluidSim is a batch of one. Field arrays are row-pitched (pitches rounded up
// to 32 elements so each row starts on a 128-byte boundary):
//   cells  T, T2, Y, Y2, SQ, cellG      [ny][pc]       pc = roundup(nx, 32)
//   U faces U, U2, fx, ax0              [ny][pu]       pu = roundup(nx+1, 32)
//   V faces V, V2, fy, ay0              [ny+1][pc]
// Arithmetic follows the WGSL expressions operation by operation (the library
// is compiled with -fmad=false) so that the CPU restatement of the reference
// reproduces it to a few ulp; each helper cites the WGSL it restates.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/campfire_gas.h"

namespace cfg {

constexpr int MAX_PIECES = CFG_MAX_PIECES;
constexpr int PIECE_FLOATS = CFG_PIECE_FLOATS;
constexpr int ACC_GLOBAL = CFG_ACC_GLOBAL;
constexpr int ACC_LEN = CFG_ACC_LEN;
constexpr int N_FLOOR = CFG_N_FLOOR;
constexpr int RAD_LEN = CFG_RAD_LEN;
constexpr int MAX_LEVELS = CFG_MAX_LEVELS;
constexpr uint32_t SOLID_NONE = 0xffffffffu;   // common.wgsl:27

struct LevelDesc {
  int nx, ny, pc, pu;       // dims and pitches (pc: cells and ay; pu: ax)
  float h2;                 // f32((dx * 2^l)^2), js/fluid.js:82
  float *p, *pb, *rhs, *ax, *ay;   // pb: second pressure buffer of the fused smoothers
};

// Per-scene state of the pressure solve loop and its reductions (device-owned)
struct SolveState {
  double bnorm2;            // ||rhs||^2 (FP32 modes) or ||rhs64||^2 (FP64 mode)
  double rnorm2;            // last ||r||^2
  double rel;               // last ||r||/||rhs||
  double rel0;              // FP64 mode: relative defect before the first cycle of the step
  int cycles;               // V-cycles run in this step
  int active;               // 1 while this scene keeps cycling
  unsigned int counter;     // CTAs finished in the current reduction
  unsigned int maxu;        // max |u| over faces after projection (f32 bits; CFL step)
  int direct_ok;            // the coarsest inverse in half cinv_cur of SceneDesc::cinv is valid (direct coarse solve)
  int cinv_cur;             // the half of the double-buffered inverse the cycles use
  int direct_ok_next;       // pipelined coarse solve: the other half, factored from this step's operator, is valid
  int pad;
  double delta, alpha, beta;   // Krylov FP64 mode: r.z of this cycle, the step length, the direction update
  double pi;                // Krylov FP64 mode: d.q of this cycle
  double time;              // CFL step: the scene's clock, advanced on the device by each step's own dt
};

struct SceneDesc {
  cfg_params P;             // the uniform (common.wgsl:4-15); P.dt is rewritten on device in CFL mode
  int nx, ny, pc, pu;
  int nlev, diff_sub;       // multigrid levels; diffusion sub-steps (js/fluid.js:190-198)
  float diff_dt;            // dt / diff_sub as f32 (the DiffParams uniform)
  float cfl, dt_cap;        // CFL step (extension); cfl = 0 keeps dt fixed
  int nray;                 // rays per target of the radiation pass
  int enabled;              // 0: scene skipped by every kernel (batch slot not in use)
  int nt_fr, nt_mg0;        // tiles of this scene in the forces and level-0 multigrid work lists
  int nt_up0;               // tiles of this scene in the level-0 fused up-smoother work list
  int lc;                   // first level of the one-CTA coarse block (levels lc..nlev-1)
  int lw;                   // nlev - 3: the coarse block's W tail (that level visits the next twice); nlev: none
  float *U, *V, *U2, *V2, *T, *T2, *Tw;   // Tw: diffusion ping-pong buffer
  float4 *Y, *Y2, *Yw;
  float2 *SQ, *cellG;
  float *fx, *fy;
  int32_t *acc, *faceW;
  float *pieces;
  float4 *rad;
  double *p64, *rhs64, *part;   // FP64 pressure, FP64 rhs, per-CTA partial sums (3 per tile)
  double *r64, *dA, *dB, *q64;  // Krylov FP64 mode: residual, search direction d, L z of the cycle, q = L d
  SolveState* solve;
  const char* tmap;         // TMA tensor maps of the levels (TM_PER_LEVEL per level, 128 bytes each)
  float* cinv;              // inverses of the coarsest operator, two halves of n x n (n = its cells), direct coarse solve
  LevelDesc lev[MAX_LEVELS];
};

// Pressure-solve control shared by all scenes of a batch (device-owned)
struct SolveCtl {
  int mode, ncycles, max_cycles, min_cycles;
  double tol;
  unsigned int scenes_done;   // arrivals of the current reduction (decisions: arrivals << 16 | scenes cycling on)
  int nscenes;                // enabled scenes taking part in this solve
  int nactive;                // scenes cycling in the current V-cycle
  int any_active;             // the loop decision of the last cycle
  int iter;                   // cycles run by the loop in this step (reset before the loop)
  int hard_cap;               // the loop stops after this many cycles whatever any_active says
  int err;                    // set by a kernel whose bounded wait ran out (reported as CFG_ERR_TIMEDOUT)
  int coarse_direct;          // TOL/FP64 modes: solve the coarsest level with its inverse instead of 120 sweeps
  int use_cond;               // 1 while the step runs as a graph: the loop decision sets the WHILE node's condition
  int krylov;                 // FP64 mode: preconditioned (flexible) CG around the V-cycle instead of plain correction
  unsigned long long cond;    // that node's cudaGraphConditionalHandle
};

// One tile of a work list
struct Work { int scene, tx, ty, tile; };

__host__ __device__ inline int round_up(int x, int m) { return (x + m - 1) / m * m; }

#ifdef __CUDACC__
// Programmatic dependent launch (kernels of the pressure loop): a kernel launched
// with programmatic stream serialization may start while its predecessor is still
// running. pdl_wait() blocks until the predecessor grid has completed and its
// writes are visible; everything before it may read only data no kernel of the
// step writes (descriptors, work lists, tensor maps). pdl_trigger() lets the
// successor begin launching. Both are no-ops for an ordinary launch.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Arrival on a gpu-scope counter (atomic add of v with acquire-release semantics): the
// calling thread's earlier writes are visible to any thread that later observes the
// count, and the thread that makes the last arrival sees every earlier arriver's writes
// (the counter's release sequence). Returns the count before this arrival.
__device__ __forceinline__ unsigned arrive_acq_rel(unsigned* counter, unsigned v = 1u) {
  unsigned old;
  asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(counter), "r"(v) : "memory");
  return old;
}

// Pressure loop as a graph WHILE node: the first kernel of each iteration counts it
// (one thread; at the hard cap the loop ends after this iteration even if no
// decision is ever recorded), and the last scene's decision of the iteration sets
// the node's condition. Outside a graph (use_cond = 0) the host reads any_active.
__device__ __forceinline__ void loop_count(SolveCtl* ctl) {
  const int it = ctl->iter + 1;
  ctl->iter = it;
  if (it >= ctl->hard_cap && ctl->use_cond) cudaGraphSetConditional((cudaGraphConditionalHandle)ctl->cond, 0u);
}


// ------------------------------------------------------------- common.wgsl
__device__ __forceinline__ float rhoOf(const cfg_params& P, float T) { return P.rhoAmb * P.Tamb / T; }   // :33
// :36-38 Sutherland viscosity
__device__ __forceinline__ float muOf(const cfg_params& P, float T) {
  return 1.716e-5f * powf(T / 273.15f, 1.5f) * (float)(273.15 + 110.4) / (T + 110.4f) * P.viscMult;
}
// :40-42 rho*D = k/cp
__device__ __forceinline__ float rhoDOf(const cfg_params& P, float T) {
  return 1.716e-5f * powf(T / 273.15f, 1.5f) * (float)(273.15 + 110.4) / (T + 110.4f) / P.Pr * P.diffMult;
}
__device__ __forceinline__ float4 ambY(const cfg_params& P) { return make_float4(0.f, P.YOamb, 0.f, 0.f); }  // :44
// WGSL mix(a, b, t) = a * (1 - t) + b * t
__device__ __forceinline__ float mixf(float a, float b, float t) { return a * (1.f - t) + b * t; }
__device__ __forceinline__ float4 mix4(float4 a, float4 b, float t) {
  return make_float4(mixf(a.x, b.x, t), mixf(a.y, b.y, t), mixf(a.z, b.z, t), mixf(a.w, b.w, t));
}
__device__ __forceinline__ float clampf(float e, float lo, float hi) { return fminf(fmaxf(e, lo), hi); }
__device__ __forceinline__ float4 min4(float4 a, float4 b) { return make_float4(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z), fminf(a.w, b.w)); }
__device__ __forceinline__ float4 max4(float4 a, float4 b) { return make_float4(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z), fmaxf(a.w, b.w)); }
// WGSL i32(f32): truncation toward zero, saturating; i32(round(x)): ties to even, saturating
__device__ __forceinline__ int32_t wgsl_i32(float v) { return __float2int_rz(v); }
__device__ __forceinline__ int32_t wgsl_i32_round(float v) { return __float2int_rn(v); }

// Piece as laid out in the storage buffer (common.wgsl:17-23)
struct Piece { float pos[2], angle, half, vel[2], omega, alive, Ts[4], mflux[4], charCov[4]; };
static_assert(sizeof(Piece) == PIECE_FLOATS * 4, "Piece is 20 floats");

// :47-53 signed distance to a rotated square (negative inside)
__device__ __forceinline__ float sdBox(float px, float py, const Piece& pc) {
  const float c = cosf(pc.angle), s = sinf(pc.angle);
  const float dxp = px - pc.pos[0], dyp = py - pc.pos[1];
  const float lx = c * dxp + s * dyp, ly = -s * dxp + c * dyp;
  const float qx = fabsf(lx) - pc.half, qy = fabsf(ly) - pc.half;
  const float mx = fmaxf(qx, 0.f), my = fmaxf(qy, 0.f);
  return sqrtf(mx * mx + my * my) + fminf(fmaxf(qx, qy), 0.f);
}
// :56-62 local face index nearest to p: 0:+x 1:+y 2:-x 3:-y
__device__ __forceinline__ uint32_t faceOf(float px, float py, const Piece& pc) {
  const float c = cosf(pc.angle), s = sinf(pc.angle);
  const float dxp = px - pc.pos[0], dyp = py - pc.pos[1];
  const float lx = c * dxp + s * dyp, ly = -s * dxp + c * dyp;
  if (fabsf(lx) > fabsf(ly)) return lx > 0.f ? 0u : 2u;
  return ly > 0.f ? 1u : 3u;
}

// ------------------------------------------------------------- samplers (js/gpu.js:16-65)
// at(i, j) applies the boundary rules; quad(i, j, ...) reads the 2x2 block (i..i+1, j..j+1)
// directly when every corner of it is an ordinary value (the same values at() returns) and
// says whether it did
// C fields: open sides/top sample the ambient, the floor is zero-gradient (:32-35)
struct CField {
  const float* a; int nx, ny, pc; float amb;
  __device__ __forceinline__ float at(int i, int j) const {
    if (i < 0 || i >= nx || j >= ny) return amb;
    return __ldg(a + max(j, 0) * pc + i);
  }
  __device__ __forceinline__ bool quad(int i, int j, float& A, float& C, float& D, float& E) const {
    if ((unsigned)i >= (unsigned)(nx - 1) || (unsigned)j >= (unsigned)(ny - 1)) return false;
    const float* q = a + j * pc + i;
    A = __ldg(q); C = __ldg(q + 1); D = __ldg(q + pc); E = __ldg(q + pc + 1);
    return true;
  }
};
struct C4Field {
  const float4* a; int nx, ny, pc; float4 amb;
  __device__ __forceinline__ float4 at(int i, int j) const {
    if (i < 0 || i >= nx || j >= ny) return amb;
    return __ldg(a + max(j, 0) * pc + i);
  }
  __device__ __forceinline__ bool quad(int i, int j, float4& A, float4& C, float4& D, float4& E) const {
    if ((unsigned)i >= (unsigned)(nx - 1) || (unsigned)j >= (unsigned)(ny - 1)) return false;
    const float4* q = a + j * pc + i;
    A = __ldg(q); C = __ldg(q + 1); D = __ldg(q + pc); E = __ldg(q + pc + 1);
    return true;
  }
};
// U: still air outside, no-slip floor ghost -U(i,0) (:44-46)
struct UField {
  const float* a; int nx, ny, pu;
  __device__ __forceinline__ float at(int i, int j) const {
    if (i < 0 || i > nx || j >= ny) return 0.f;
    if (j < 0) return -__ldg(a + i);
    return __ldg(a + j * pu + i);
  }
  __device__ __forceinline__ bool quad(int i, int j, float& A, float& C, float& D, float& E) const {
    if ((unsigned)i >= (unsigned)nx || (unsigned)j >= (unsigned)(ny - 1)) return false;
    const float* q = a + j * pu + i;
    A = __ldg(q); C = __ldg(q + 1); D = __ldg(q + pu); E = __ldg(q + pu + 1);
    return true;
  }
};
// V: still air outside, clamp at the floor (:47-48)
struct VField {
  const float* a; int nx, ny, pc;
  __device__ __forceinline__ float at(int i, int j) const {
    if (i < 0 || i >= nx || j > ny) return 0.f;
    return __ldg(a + max(j, 0) * pc + i);
  }
  __device__ __forceinline__ bool quad(int i, int j, float& A, float& C, float& D, float& E) const {
    if ((unsigned)i >= (unsigned)(nx - 1) || (unsigned)j >= (unsigned)ny) return false;
    const float* q = a + j * pc + i;
    A = __ldg(q); C = __ldg(q + 1); D = __ldg(q + pc); E = __ldg(q + pc + 1);
    return true;
  }
};

// s_<name>: bilinear at g - off (cell units); off = (0.5,0.5) C, (0,0.5) U, (0.5,0) V
// the four corners of the 2x2 block at (i, j), directly when the field allows it
template <class F, class T>
__device__ __forceinline__ void corners(const F& f, int i, int j, T& A, T& C, T& D, T& E) {
  if (f.quad(i, j, A, C, D, E)) return;
  A = f.at(i, j); C = f.at(i + 1, j); D = f.at(i, j + 1); E = f.at(i + 1, j + 1);
}
template <class F>
__device__ __forceinline__ float sample(const F& f, float gx, float gy, float ox, float oy) {
  const float fxp = gx - ox, fyp = gy - oy;
  const float bx = floorf(fxp), by = floorf(fyp), tx = fxp - bx, ty = fyp - by;
  const int i = wgsl_i32(bx), j = wgsl_i32(by);
  float A, C, D, E;
  corners(f, i, j, A, C, D, E);
  return mixf(mixf(A, C, tx), mixf(D, E, tx), ty);
}
template <class F>
__device__ __forceinline__ float4 sample4(const F& f, float gx, float gy) {
  const float fxp = gx - 0.5f, fyp = gy - 0.5f;
  const float bx = floorf(fxp), by = floorf(fyp), tx = fxp - bx, ty = fyp - by;
  const int i = wgsl_i32(bx), j = wgsl_i32(by);
  float4 A, C, D, E;
  corners(f, i, j, A, C, D, E);
  return mix4(mix4(A, C, tx), mix4(D, E, tx), ty);
}
// mm_<name>: min/max of the 4 corners
template <class F>
__device__ __forceinline__ void minmax(const F& f, float gx, float gy, float ox, float oy, float& lo, float& hi) {
  const int i = wgsl_i32(floorf(gx - ox)), j = wgsl_i32(floorf(gy - oy));
  float A, C, D, E;
  corners(f, i, j, A, C, D, E);
  lo = fminf(fminf(A, C), fminf(D, E)); hi = fmaxf(fmaxf(A, C), fmaxf(D, E));
}
template <class F>
__device__ __forceinline__ void minmax4(const F& f, float gx, float gy, float4& lo, float4& hi) {
  const int i = wgsl_i32(floorf(gx - 0.5f)), j = wgsl_i32(floorf(gy - 0.5f));
  float4 A, C, D, E;
  corners(f, i, j, A, C, D, E);
  lo = min4(min4(A, C), min4(D, E)); hi = max4(max4(A, C), max4(D, E));
}

// x / d rounded to nearest from r = RN(1/d): q0 = RN(x r), q = RN(q0 + r (x - d q0)),
// the residual x - d q0 exact by FMA (Markstein, IBM J. Res. Dev. 34(1), 1990). Equal
// to the IEEE quotient for quotients in the normal range (and for x = +0); for x = -0 it
// gives +0. It replaces the division subroutine where the divisor is fixed for many
// quotients (smoother diagonals, h2, dx).
__device__ __forceinline__ float div_by_rcp(float x, float d, float r) {
  const float q0 = __fmul_rn(x, r);
  const float e = __fmaf_rn(-q0, d, x);
  return __fmaf_rn(e, r, q0);
}

// advect.wgsl:28-34: vel = (s_U, s_V)/dx; RK2 midpoint back-trace (dt < 0 traces forward).
// The quotient by dx from rdx = RN(1/dx): the IEEE one, except that a velocity of -0 comes
// out +0, which moves no trace point (g - h * (+-0) = g)
struct VelSampler {
  UField u; VField v; float dx, rdx;
  __device__ __forceinline__ void vel(float gx, float gy, float& vx, float& vy) const {
    vx = div_by_rcp(sample(u, gx, gy, 0.f, 0.5f), dx, rdx);
    vy = div_by_rcp(sample(v, gx, gy, 0.5f, 0.f), dx, rdx);
  }
  __device__ __forceinline__ void trace(float gx, float gy, float tdt, float& ox, float& oy) const {
    float vx, vy; vel(gx, gy, vx, vy);
    const float hd = 0.5f * tdt;
    const float mx = gx - hd * vx, my = gy - hd * vy;
    vel(mx, my, vx, vy);
    ox = gx - tdt * vx; oy = gy - tdt * vy;
  }
};

#endif  // __CUDACC__

}  // namespace cfg
