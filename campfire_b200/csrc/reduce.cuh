// Deterministic FP64 block reductions and the per-scene "last CTA finishes"
// protocol used by the norm reductions of the pressure solve.
//
// A reduction over the tiles of one scene: every CTA writes its partial to
// scene.part[tile] and arrives on scene.solve->counter (release); the CTA that
// makes the last arrival (acquire) sums the partials in tile order (so the total
// does not depend on CTA scheduling) and resets the counter. Its other threads read
// the partials after the block barrier that follows thread 0's acquire, from L2.
#pragma once
#include "gas_dev.cuh"

namespace cfg {

// Sum over the block; the result is valid in thread 0. blockDim.x must be a
// multiple of 32 and at most 1024. Fixed combination order -> deterministic.
__device__ __forceinline__ double block_sum(double v, double* sh /* >= 32 doubles */) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (warp == 0) {
    t = lane < nw ? sh[lane] : 0.0;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;
}

__device__ __forceinline__ float block_max(float v, float* sh /* >= 32 floats */) {
  #pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  float t = 0.f;
  if (warp == 0) {
    t = lane < nw ? sh[lane] : 0.f;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) t = fmaxf(t, __shfl_down_sync(0xffffffffu, t, o));
  }
  return t;
}

// Publish this CTA's partial; returns true (in every thread) in the CTA that
// completes the scene's reduction, which then holds the total in *total.
__device__ __forceinline__ bool scene_reduce(const SceneDesc& S, int tile, int ntiles, double partial,
                                             double* sh, double* total) {
  __shared__ int s_last;
  if (threadIdx.x == 0) {
    S.part[tile] = partial;
    const unsigned prev = arrive_acq_rel(&S.solve->counter);
    s_last = (prev == (unsigned)ntiles - 1u) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last) return false;
  double v = 0.0;
  // each thread sums a fixed strided subset in order, then the fixed block tree
  for (int k = threadIdx.x; k < ntiles; k += blockDim.x) v += __ldcg(S.part + k);
  const double t = block_sum(v, sh);
  if (threadIdx.x == 0) { *total = t; S.solve->counter = 0u; }
  return true;
}

// Two sums at once (partials at part[2 tile], part[2 tile + 1]); same protocol.
__device__ __forceinline__ bool scene_reduce2(const SceneDesc& S, int tile, int ntiles, double a, double b,
                                              double* sh, double* ta, double* tb) {
  __shared__ int s_last2;
  if (threadIdx.x == 0) {
    S.part[2 * tile] = a;
    S.part[2 * tile + 1] = b;
    const unsigned prev = arrive_acq_rel(&S.solve->counter);
    s_last2 = (prev == (unsigned)ntiles - 1u) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last2) return false;
  double va = 0.0, vb = 0.0;
  for (int k = threadIdx.x; k < ntiles; k += blockDim.x) {
    va += __ldcg(S.part + 2 * k);
    vb += __ldcg(S.part + 2 * k + 1);
  }
  const double sa = block_sum(va, sh);
  const double sb = block_sum(vb, sh);
  if (threadIdx.x == 0) { *ta = sa; *tb = sb; S.solve->counter = 0u; }
  return true;
}

// Three sums at once (partials at part[3 tile + 0..2]); same protocol.
__device__ __forceinline__ bool scene_reduce3(const SceneDesc& S, int tile, int ntiles, double a, double b, double c,
                                              double* sh, double* ta, double* tb, double* tc) {
  __shared__ int s_last3;
  if (threadIdx.x == 0) {
    S.part[3 * tile] = a;
    S.part[3 * tile + 1] = b;
    S.part[3 * tile + 2] = c;
    const unsigned prev = arrive_acq_rel(&S.solve->counter);
    s_last3 = (prev == (unsigned)ntiles - 1u) ? 1 : 0;
  }
  __syncthreads();
  if (!s_last3) return false;
  double va = 0.0, vb = 0.0, vc = 0.0;
  for (int k = threadIdx.x; k < ntiles; k += blockDim.x) {
    va += __ldcg(S.part + 3 * k);
    vb += __ldcg(S.part + 3 * k + 1);
    vc += __ldcg(S.part + 3 * k + 2);
  }
  const double sa = block_sum(va, sh);
  const double sb = block_sum(vb, sh);
  const double sc = block_sum(vc, sh);
  if (threadIdx.x == 0) { *ta = sa; *tb = sb; *tc = sc; S.solve->counter = 0u; }
  return true;
}

// N sums over a block of 256 threads at once, in a fixed order: every thread's values go to
// shared memory; warp w sums quantities w, w + 8, ...: lane l adds threads l, l + 32, ...,
// l + 224 in that order, then the warp's shuffle tree. The totals are valid in thread 0.
// sh holds at least 256 N + N doubles.
template <int N>
__device__ __forceinline__ void block_sum_t(double (&v)[N], double* sh) {
  #pragma unroll
  for (int m = 0; m < N; m++) sh[m * 256 + threadIdx.x] = v[m];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int m = warp; m < N; m += 8) {
    double t = 0.0;
    #pragma unroll
    for (int k = 0; k < 8; k++) t += sh[m * 256 + lane + 32 * k];
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sh[N * 256 + m] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0)
    #pragma unroll
    for (int m = 0; m < N; m++) v[m] = sh[N * 256 + m];
}

// N sums of one scene at once (partials at part[N tile + m]); the scene_reduce protocol.
// On return true (the CTA that completed the scene), v holds the totals in thread 0.
// 256 threads; sh as for block_sum_t.
template <int N>
__device__ __forceinline__ bool scene_reduce_n(const SceneDesc& S, int tile, int ntiles, double (&v)[N], double* sh) {
  __shared__ int s_lastn;
  if (threadIdx.x == 0) {
    #pragma unroll
    for (int m = 0; m < N; m++) S.part[N * tile + m] = v[m];
    const unsigned prev = arrive_acq_rel(&S.solve->counter);
    s_lastn = (prev == (unsigned)ntiles - 1u) ? 1 : 0;
  }
  __syncthreads();
  if (!s_lastn) return false;
  #pragma unroll
  for (int m = 0; m < N; m++) v[m] = 0.0;
  // two tiles' partials loaded before either is added (their L2 round trips overlap); the sums
  // keep the order of one tile after the other
  const int stride = blockDim.x;
  for (int k = threadIdx.x; k < ntiles; k += 2 * stride) {
    double a[N], b[N];
    const bool two = k + stride < ntiles;
    #pragma unroll
    for (int m = 0; m < N; m++) {
      a[m] = __ldcg(S.part + N * k + m);
      b[m] = two ? __ldcg(S.part + N * (k + stride) + m) : 0.0;
    }
    #pragma unroll
    for (int m = 0; m < N; m++) {
      v[m] += a[m];
      if (two) v[m] += b[m];
    }
  }
  block_sum_t<N>(v, sh);
  if (threadIdx.x == 0) S.solve->counter = 0u;
  return true;
}

// The Krylov state a cycle's coefficients start from (read after the wait on the previous kernel)
struct PcgPrev {
  double alpha, beta, delta, pi;
  int cycles;
};
__device__ __forceinline__ PcgPrev pcg_load(const SolveState* ss) {
  PcgPrev p;
  p.alpha = ss->alpha; p.beta = ss->beta; p.delta = ss->delta; p.pi = ss->pi; p.cycles = ss->cycles;
  return p;
}

// Krylov FP64 mode, after the V-cycle, from delta = r.z, eta = q_prev.z and zeta = z.Lz:
// the direction update beta = -alpha_prev eta / delta_prev (0 in the first cycle), the
// direction's d.q = zeta + 2 beta eta + beta^2 (d.q)_prev (d = z + beta d_prev and
// q = L d = Lz + beta q_prev, L symmetric), and the step length alpha = delta / d.q.
__device__ __forceinline__ void pcg_coef(SolveState* ss, const PcgPrev& pv, double delta, double eta, double zeta,
                                         double* alpha_out, double* beta_out) {
  const double prev = pv.delta;
  const bool more = pv.cycles > 0 && prev != 0.0;
  const double beta = more ? -pv.alpha * eta / prev : 0.0;
  const double pi = more ? zeta + 2.0 * beta * eta + beta * beta * pv.pi : zeta;
  const double alpha = pi != 0.0 ? delta / pi : 0.0;
  ss->beta = beta;
  ss->delta = delta;
  ss->pi = pi;
  ss->alpha = alpha;
  *alpha_out = alpha;
  *beta_out = beta;
}
__device__ __forceinline__ void pcg_coef(const SceneDesc& S, double delta, double eta, double zeta) {
  double a, b;
  pcg_coef(S.solve, pcg_load(S.solve), delta, eta, zeta, &a, &b);
}

// What a scene's loop decision reads: its cycle count and ||rhs||^2, and the loop's
// control values. Kernels that decide load it after their wait on the previous kernel,
// beside their other reads, so the decision itself waits on no load.
struct DecideIn {
  double b2, tol;
  unsigned long long cond;
  int cycles, mode, ncycles, max_cycles, nactive, iter, hard_cap, use_cond;
};
__device__ __forceinline__ DecideIn decide_load(const SolveCtl* ctl, const SolveState* ss) {
  DecideIn d;
  d.b2 = ss->bnorm2; d.tol = ctl->tol;
  d.cycles = ss->cycles; d.mode = ctl->mode; d.ncycles = ctl->ncycles; d.max_cycles = ctl->max_cycles;
  d.nactive = ctl->nactive; d.iter = ctl->iter; d.hard_cap = ctl->hard_cap; d.use_cond = ctl->use_cond;
  d.cond = ctl->cond;
  return d;
}

// The loop decision of one scene after a norm reduction (thread 0 of the CTA that
// finished it): count the cycle, record ||r|| / ||rhs||, keep cycling while rel > tol
// (TOL/FP64) or cycles < n (FIXED), and cycles < max. Every scene deciding in this
// cycle arrives on ctl->scenes_done with 1 << 16 | (cycles on), so the last one knows
// how many scenes cycle on without reading them; it records that and, in a graph, sets
// the loop's condition.
__device__ __forceinline__ void solve_decide(SolveCtl* ctl, SolveState* ss, const DecideIn& in, double r2,
                                             bool count_cycle) {
  const int cyc = in.cycles + (count_cycle ? 1 : 0);
  const double rel = in.b2 > 0.0 ? sqrt(r2 / in.b2) : 0.0;
  const int act = in.mode == CFG_SOLVE_FIXED ? (cyc < in.ncycles) : ((rel > in.tol) && (cyc < in.max_cycles));
  ss->cycles = cyc;
  ss->rnorm2 = r2;
  ss->rel = rel;
  ss->active = act;
  // one scene cycling: it is the last to decide, with no arrival to count
  const unsigned old = in.nactive == 1 ? 0u : arrive_acq_rel(&ctl->scenes_done, (1u << 16) | (unsigned)act);
  if ((int)(old >> 16) + 1 == in.nactive) {
    const int na = (int)(old & 0xffffu) + act;
    ctl->scenes_done = 0u;
    ctl->nactive = na;
    const int go = (na > 0 && in.iter < in.hard_cap) ? 1 : 0;
    ctl->any_active = go;
    // the condition starts every launch of the step graph at 1 (cudaGraphCondAssignDefault)
    // and only this decision or the hard cap clears it, so it is written only to stop
    if (in.use_cond && !go) cudaGraphSetConditional((cudaGraphConditionalHandle)in.cond, 0u);
  }
}
__device__ __forceinline__ void solve_decide(SolveCtl* ctl, SolveState* ss, double r2, bool count_cycle) {
  solve_decide(ctl, ss, decide_load(ctl, ss), r2, count_cycle);
}


}  // namespace cfg
