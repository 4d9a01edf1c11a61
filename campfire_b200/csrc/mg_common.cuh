// Pieces of the multigrid level solves shared by the one-CTA coarse block (k_mgf.cu)
// and the cluster coarse phase (k_mgc.cu): a level held in shared memory with the
// global row pitches, its 5-point stencil (pressure.wgsl:77-86), and the coarsest
// level's red-black sweeps with fixed stencils (pressure.wgsl:132-156).
#pragma once
#include "gas_dev.cuh"

namespace cfg {
namespace mgc {

struct LvS {
  float *p, *rhs, *ax, *ay;
  const float* rc;                    // the coarse block's RN(1/diag) per cell (0: closed), row-major
  int nx, ny, pc, pu;
  float h2, rh2;                      // rh2 = RN(1 / h2)
  unsigned long long mnx, mhalf;      // fdiv multipliers of nx and (nx + 1) / 2
};

// t / d without a division instruction for 0 <= t < 2^16 and 1 <= d < 2^16, from
// m = floor(2^32 / d) + 1 = (2^32 + e) / d with 0 < e <= d: t m / 2^32 = t / d + t e / (d 2^32)
// and t e < 2^32, so the excess stays below 1/d and the floor is t / d (the invariant-divisor
// multiplication of Granlund & Montgomery, PLDI 1994). The coarse levels in shared memory
// and the block's thread indices are far below 2^16.
__device__ __forceinline__ unsigned long long fdiv_magic(int d) { return 0x100000000ull / (unsigned)d + 1ull; }
__device__ __forceinline__ int fdiv(int t, unsigned long long m) {
  return (int)(((unsigned long long)(unsigned)t * m) >> 32);
}
// A level of a block's shared-memory layout as offsets from the block's dynamic shared
// array; lvs_at rebuilds the pointers from that array inside the kernel, so the compiler
// sees shared-memory addresses (shared loads and stores, 32-bit addresses).
struct LvO {
  int po, ro, ao, yo, to;             // p, rhs, ax, ay; to: the 1/diag table
  int nx, ny, pc, pu;
  float h2, rh2;
  unsigned long long mnx, mhalf;
};
__device__ __forceinline__ LvS lvs_at(float* base, const LvO& o) {
  LvS v;
  v.p = base + o.po; v.rhs = base + o.ro; v.ax = base + o.ao; v.ay = base + o.yo;
  v.rc = base + o.to;
  v.nx = o.nx; v.ny = o.ny; v.pc = o.pc; v.pu = o.pu; v.h2 = o.h2; v.rh2 = o.rh2; v.mnx = o.mnx; v.mhalf = o.mhalf;
  return v;
}
// the derived constants of a level (one thread, once per kernel)
__device__ __forceinline__ void lvs_derive(LvS& v) {
  v.rh2 = __frcp_rn(v.h2);
  v.mnx = fdiv_magic(v.nx);
  v.mhalf = fdiv_magic((v.nx + 1) >> 1);
}

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
// the diagonal of stencil_d alone (the same sums in the same order)
__device__ __forceinline__ float diag_d(const LvS& L, int i, int j) {
  const float w = L.ax[j * L.pu + i], e = L.ax[j * L.pu + i + 1];
  const float s = L.ay[j * L.pc + i], n = L.ay[(j + 1) * L.pc + i];
  float diag = 0.f;
  if (i > 0) diag += w; else diag += 2.f * w;
  if (i < L.nx - 1) diag += e; else diag += 2.f * e;
  if (j > 0) diag += s;
  if (j < L.ny - 1) diag += n; else diag += 2.f * n;
  return diag;
}
// (L z)_ij in FP64 from a level in shared memory (the FP64 defect's form)
__device__ __forceinline__ double lap_block64(const LvS& L, int i, int j) {
  const int k = j * L.pc + i;
  const double w = L.ax[j * L.pu + i], e = L.ax[j * L.pu + i + 1];
  const double s = L.ay[j * L.pc + i], n = L.ay[(j + 1) * L.pc + i];
  double off = 0.0, diag = 0.0;
  if (i > 0) { off += w * (double)L.p[k - 1]; diag += w; } else diag += 2.0 * w;
  if (i < L.nx - 1) { off += e * (double)L.p[k + 1]; diag += e; } else diag += 2.0 * e;
  if (j > 0) { off += s * (double)L.p[k - L.pc]; diag += s; }
  if (j < L.ny - 1) { off += n * (double)L.p[k + L.pc]; diag += n; } else diag += 2.0 * n;
  return diag > 0.0 ? (off - diag * (double)L.p[k]) / (double)L.h2 : 0.0;
}
__device__ __forceinline__ void bar_coarsest(int nthreads) { asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory"); }

using cfg::div_by_rcp;   // gas_dev.cuh

// One coarsest-level cell with its fixed stencil (pressure.wgsl:132-156).
struct CCell {
  float w, e, s, n, rh, diag, rcp;
  int kp;
  bool act, hw, he, hs, hn;
};
__device__ __forceinline__ CCell coarsest_cell(const LvS& L, int k) {
  CCell c{};
  c.act = k < L.nx * L.ny;
  if (!c.act) return c;
  const int j = fdiv(k, L.mnx), i = k - j * L.nx;
  c.kp = j * L.pc + i;
  c.w = L.ax[j * L.pu + i]; c.e = L.ax[j * L.pu + i + 1];
  c.s = L.ay[j * L.pc + i]; c.n = L.ay[(j + 1) * L.pc + i];
  float diag = 0.f;
  if (i > 0) diag += c.w; else diag += 2.f * c.w;
  if (i < L.nx - 1) diag += c.e; else diag += 2.f * c.e;
  if (j > 0) diag += c.s;
  if (j < L.ny - 1) diag += c.n; else diag += 2.f * c.n;
  c.diag = diag;
  c.rcp = diag > 0.f ? __frcp_rn(diag) : 0.f;
  c.rh = L.rhs[c.kp] * L.h2;
  c.hw = i > 0; c.he = i < L.nx - 1; c.hs = j > 0; c.hn = j < L.ny - 1;
  return c;
}
__device__ __forceinline__ void coarsest_update(float* p, int pc, const CCell& c) {
  if (!c.act) return;
  float off = 0.f;
  if (c.hw) off += c.w * p[c.kp - 1];
  if (c.he) off += c.e * p[c.kp + 1];
  if (c.hs) off += c.s * p[c.kp - pc];
  if (c.hn) off += c.n * p[c.kp + pc];
  p[c.kp] = c.diag > 0.f ? div_by_rcp(off - c.rh, c.diag, c.rcp) : 0.f;
}

}  // namespace mgc
}  // namespace cfg
