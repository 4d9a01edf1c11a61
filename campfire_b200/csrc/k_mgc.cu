// Cluster coarse phase of the fused V(2,2) cycle (pressure.wgsl:77-156, the levels of
// js/fluid.js:294-312 from level lc down): levels lc .. coarsest of one scene on a
// thread-block cluster of CS CTAs instead of tiled kernels per level or one CTA.
//
// Each level's rows are shared out over the cluster: CTA r owns rows
// [r ny / CS, (r + 1) ny / CS). Its shared memory holds, for every level, its rows of
// p with one halo row on each side, rhs, ax, the ay rows of their south and north
// faces, and the owned rows' residuals. A colour pass updates the owned cells of one
// colour and writes the updated cells of its first and last row straight into the halo
// rows of the CTAs owning the rows next to them (distributed shared memory); one cluster
// barrier then makes them visible. A pass reads only cells of the other colour, so the
// writes race with no read. Restriction reads the fine residuals of rows owned by other
// CTAs, prolongation their coarse p, both through distributed shared memory. The
// coarsest level is solved by its inverse, each CTA taking the rows of its own cells
// (b gathered from every CTA), or, without a valid inverse, by the reference's 120
// sweeps on one CTA over a gathered copy of the level.
//
// Per cell the arithmetic is that of the one-CTA coarse block (k_mgf.cu), in the same
// order: results are bit-identical whichever form runs.
#include <cooperative_groups.h>

#include <algorithm>

#include "gas_dev.cuh"
#include "kernels.h"
#include "mg_common.cuh"
#include "tma.cuh"

namespace cg = cooperative_groups;

namespace cfg {

namespace {

constexpr int CC_THREADS = 512;
using namespace mgc;

__host__ __device__ inline int share0(int r, int ny, int cs) { return (int)(((long long)r * ny) / cs); }
// the CTA owning row j: the largest r with share0(r) <= j
__host__ __device__ inline int owner_of(int j, int ny, int cs) { return (int)((((long long)j + 1) * cs - 1) / ny); }
__host__ __device__ inline int rows_max(int ny, int cs) { return (ny + cs - 1) / cs; }
__host__ __device__ inline int up32(int n) { return (n + 31) & ~31; }

// One level in the cluster layout (offsets identical on every CTA of the cluster).
struct LvC {
  float *p, *rhs, *ax, *ay, *res;   // p rows r0-1 .. r1; rhs, ax, res rows r0 .. r1-1; ay rows r0 .. r1
  int nx, ny, pc, pu, r0, r1;
  float h2;
  int pad;
};

// floats of one level's arrays on one CTA
__host__ __device__ inline int level_floats(int nx, int ny, int cs) {
  const int pc = up32(nx), pu = up32(nx + 1), rm = rows_max(ny, cs);
  return (rm + 2) * pc + rm * pc + rm * pu + (rm + 1) * pc + up32(rm * nx);
}

// Cells of an owned block of rows mapped linearly onto the CTA: thread t takes column
// t % w of the block's rows t / w, t / w + R, ... (R = CC_THREADS / w); w >= CC_THREADS:
// the CTA strides along each row.
struct LinMap {
  int i0, j0, R, di;
  __device__ __forceinline__ explicit LinMap(int w) {
    if (w >= CC_THREADS) { i0 = threadIdx.x; j0 = 0; R = 1; di = CC_THREADS; }
    else { R = CC_THREADS / w; i0 = threadIdx.x % w; j0 = threadIdx.x / w; di = w; if (j0 >= R) R = 0; }
  }
};

// the stencil of an owned cell (the order of stencil_d: w, e, s, n)
__device__ __forceinline__ void stencil_c(const LvC& L, int i, int j, float& off, float& diag) {
  const int lr = j - L.r0;
  const float* pr = L.p + (lr + 1) * L.pc;
  const float w = L.ax[lr * L.pu + i], e = L.ax[lr * L.pu + i + 1];
  const float s = L.ay[lr * L.pc + i], n = L.ay[(lr + 1) * L.pc + i];
  off = 0.f; diag = 0.f;
  if (i > 0) { off += w * pr[i - 1]; diag += w; } else { diag += 2.f * w; }
  if (i < L.nx - 1) { off += e * pr[i + 1]; diag += e; } else { diag += 2.f * e; }
  if (j > 0) { off += s * pr[i - L.pc]; diag += s; }
  if (j < L.ny - 1) { off += n * pr[i + L.pc]; diag += n; } else { diag += 2.f * n; }
}

// the diagonal alone (prolongation reads no p), in stencil_c's order
__device__ __forceinline__ float diag_c(const LvC& L, int i, int j) {
  const int lr = j - L.r0;
  const float w = L.ax[lr * L.pu + i], e = L.ax[lr * L.pu + i + 1];
  const float s = L.ay[lr * L.pc + i], n = L.ay[(lr + 1) * L.pc + i];
  float diag = 0.f;
  if (i > 0) diag += w; else diag += 2.f * w;
  if (i < L.nx - 1) diag += e; else diag += 2.f * e;
  if (j > 0) diag += s;
  if (j < L.ny - 1) diag += n; else diag += 2.f * n;
  return diag;
}

// Halo rows of the neighbours: the CTA owning row r0 - 1 keeps row r0 as its halo below,
// the CTA owning row r1 keeps row r1 - 1 as its halo above (null at the domain's edges).
struct Halos {
  float* up;   // where row r0 goes (the owner of r0 - 1)
  float* dn;   // where row r1 - 1 goes (the owner of r1)
};
__device__ __forceinline__ Halos halos_of(const LvC& L, cg::cluster_group& cl, int cs) {
  Halos h{nullptr, nullptr};
  if (L.r1 <= L.r0) return h;
  if (L.r0 > 0) {
    const int q = owner_of(L.r0 - 1, L.ny, cs), a0 = share0(q, L.ny, cs);
    h.up = cl.map_shared_rank(L.p + (L.r0 - a0 + 1) * L.pc, q);   // q's rows a0 .. r0-1, then its halo below
  }
  if (L.r1 < L.ny) {
    const int q = owner_of(L.r1, L.ny, cs);
    h.dn = cl.map_shared_rank(L.p, q);                             // q's halo above is its local row 0
  }
  return h;
}

__device__ __forceinline__ void store_p(const LvC& L, const Halos& h, int i, int j, float v) {
  L.p[(j - L.r0 + 1) * L.pc + i] = v;
  if (j == L.r0 && h.up) h.up[i] = v;
  if (j == L.r1 - 1 && h.dn) h.dn[i] = v;
}

// one colour pass over the owned cells of `color` (pressure.wgsl:87-94); up to 4 rows of a
// thread are computed before any is stored (their loads overlap)
__device__ __forceinline__ void pass_c(const LvC& L, const Halos& h, const LinMap& mp, int color) {
  const int half = (L.nx + 1) >> 1;
  if (!mp.R) return;
  for (int q = mp.i0; q < half; q += mp.di)
    for (int jb = L.r0 + mp.j0; jb < L.r1; jb += 4 * mp.R) {
      float v[4];
      int jj[4], ii[4];
      #pragma unroll
      for (int m = 0; m < 4; m++) {
        const int j = jb + m * mp.R, i = 2 * q + ((j + color) & 1);
        jj[m] = -1;
        if (j < L.r1 && i < L.nx) {
          float off, diag; stencil_c(L, i, j, off, diag);
          v[m] = diag > 0.f ? (off - L.rhs[(j - L.r0) * L.pc + i] * L.h2) / diag : 0.f;
          jj[m] = j; ii[m] = i;
        }
      }
      #pragma unroll
      for (int m = 0; m < 4; m++)
        if (jj[m] >= 0) store_p(L, h, ii[m], jj[m], v[m]);
    }
}

}  // namespace

// One cluster per scene: blockIdx.x / cs is the scene, the CTA's rank in the cluster its
// share of the rows. Launched with cluster dimension cs (8 or 16).
__global__ void __launch_bounds__(CC_THREADS) k_mg_cluster(const SceneDesc* __restrict__ scenes, SolveCtl* ctl,
                                                           int cs, int count_iter) {
  extern __shared__ __align__(128) float smem[];
  __shared__ LvC lv[MAX_LEVELS];
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_ok;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const SceneDesc& S = scenes[blockIdx.x / cs];
  pdl_trigger();
  const int lc = S.lc, nl = S.nlev;
  const LevelDesc& Gc = S.lev[nl - 1];
  const int ncs = Gc.nx * Gc.ny;
  float* bfull = nullptr;   // the coarsest b, gathered
  float* arow = nullptr;    // this CTA's rows of the coarsest inverse
  float* dense = nullptr;   // the coarsest level gathered on rank 0 (sweeps)
  {
    float* q = smem;
    for (int l = lc; l < nl; l++) {
      const LevelDesc& G = S.lev[l];
      const int pc = up32(G.nx), pu = up32(G.nx + 1), rm = rows_max(G.ny, cs);
      if (threadIdx.x == 0) {
        LvC v;
        v.nx = G.nx; v.ny = G.ny; v.pc = pc; v.pu = pu; v.h2 = G.h2; v.pad = 0;
        v.r0 = share0(rank, G.ny, cs); v.r1 = share0(rank + 1, G.ny, cs);
        v.p = q; v.rhs = q + (rm + 2) * pc; v.ax = v.rhs + rm * pc; v.ay = v.ax + rm * pu; v.res = v.ay + (rm + 1) * pc;
        lv[l] = v;
      }
      q += level_floats(G.nx, G.ny, cs);
    }
    bfull = q; q += up32(ncs);
    arow = q; q += up32(rows_max(Gc.ny, cs) * Gc.nx * ncs);
    dense = q;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
  }
  __syncthreads();
  pdl_wait();
  if (count_iter && blockIdx.x == 0 && threadIdx.x == 0) loop_count(ctl);
  if (!(S.enabled && S.solve->active)) return;   // the same for every CTA of the cluster
  const bool direct = ctl->coarse_direct && S.solve->direct_ok;
  const LvC V0 = lv[lc];
  // ---- stage the owned rows of level lc's rhs and every level's coefficients
  if (threadIdx.x == 0) {
    uint32_t bytes = 0;
    const LevelDesc& G0 = S.lev[lc];
    const int n0 = V0.r1 - V0.r0;
    if (n0 > 0) bytes += n0 * G0.pc * 4;
    for (int l = lc; l < nl; l++) {
      const int nr = lv[l].r1 - lv[l].r0;
      if (nr > 0) bytes += (nr * S.lev[l].pu + (nr + 1) * S.lev[l].pc) * 4;
    }
    mbar_arrive_expect_tx(&bar, bytes);
    if (n0 > 0) bulk_g2s(V0.rhs, G0.rhs + (size_t)V0.r0 * G0.pc, n0 * G0.pc * 4, &bar);
    for (int l = lc; l < nl; l++) {
      const LevelDesc& G = S.lev[l];
      const int nr = lv[l].r1 - lv[l].r0;
      if (nr <= 0) continue;
      bulk_g2s(lv[l].ax, G.ax + (size_t)lv[l].r0 * G.pu, nr * G.pu * 4, &bar);
      bulk_g2s(lv[l].ay, G.ay + (size_t)lv[l].r0 * G.pc, (nr + 1) * G.pc * 4, &bar);
    }
  }
  // level lc's p is zero after the restriction into it (pressure.wgsl:112), halos included
  for (int e = threadIdx.x; e < (V0.r1 - V0.r0 + 2) * V0.pc; e += CC_THREADS) V0.p[e] = 0.f;
  // this CTA's rows of the coarsest inverse (constant during the step)
  if (direct) {
    const LvC& C = lv[nl - 1];
    const int ld = cinv_ld(ncs);   // the inverse's row stride in global memory
    const float* A = S.cinv + (size_t)S.solve->cinv_cur * ncs * ld + (size_t)C.r0 * C.nx * ld;
    const int na = (C.r1 - C.r0) * C.nx * ncs;
    for (int e = threadIdx.x; e < na; e += CC_THREADS) arow[e] = __ldg(A + (size_t)(e / ncs) * ld + e % ncs);
  }
  const bool ok = mbar_wait(&bar, 0);
  if (threadIdx.x == 0) s_ok = ok ? 1 : 0;
  __syncthreads();
  // every CTA leaves together if any copy failed to land (bounded waits only)
  cl.sync();
  int all_ok = 1;
  for (int r = 0; r < cs; r++) all_ok &= *cl.map_shared_rank(&s_ok, r);
  cl.sync();
  if (!all_ok) {
    if (threadIdx.x == 0 && rank == 0) atomicExch(&ctl->err, 1);
    if (!s_ok) mbar_wait(&bar, 0);
    return;
  }
  // ---- down
  for (int l = lc; l < nl - 1; l++) {
    const LvC F = lv[l], Cc = lv[l + 1];
    const Halos h = halos_of(F, cl, cs);
    const LinMap mh((F.nx + 1) >> 1);
    for (int k = 0; k < 2; k++) { pass_c(F, h, mh, 0); cl.sync(); pass_c(F, h, mh, 1); cl.sync(); }
    {
      const LinMap mp(F.nx);
      if (mp.R)
        for (int j = F.r0 + mp.j0; j < F.r1; j += mp.R)
          for (int i = mp.i0; i < F.nx; i += mp.di) {
            float off, diag; stencil_c(F, i, j, off, diag);
            const int lr = j - F.r0;
            F.res[lr * F.nx + i] =
                diag <= 0.f ? 0.f : F.rhs[lr * F.pc + i] - (off - diag * F.p[(lr + 1) * F.pc + i]) / F.h2;
          }
    }
    cl.sync();
    // restriction into the owned coarse rows; the coarse p starts at zero (halos included)
    for (int e = threadIdx.x; e < (Cc.r1 - Cc.r0 + 2) * Cc.pc; e += CC_THREADS) Cc.p[e] = 0.f;
    {
      const LinMap mc(Cc.nx);
      if (mc.R)
        for (int J = Cc.r0 + mc.j0; J < Cc.r1; J += mc.R) {
          const int ja = 2 * J, jb = 2 * J + 1;
          const int qa = owner_of(ja, F.ny, cs), qb = owner_of(jb, F.ny, cs);
          const float* ra = cl.map_shared_rank(F.res, qa) + (ja - share0(qa, F.ny, cs)) * F.nx;
          const float* rb = cl.map_shared_rank(F.res, qb) + (jb - share0(qb, F.ny, cs)) * F.nx;
          for (int I = mc.i0; I < Cc.nx; I += mc.di) {
            const float r = ra[2 * I] + ra[2 * I + 1] + rb[2 * I] + rb[2 * I + 1];
            Cc.rhs[(J - Cc.r0) * Cc.pc + I] = 0.25f * r;
          }
        }
    }
    cl.sync();
  }
  // ---- coarsest
  {
    const LvC L = lv[nl - 1];
    if (direct) {
      // b = -rhs h2 (0 in closed cells) of the owned cells, gathered by every CTA; x = A^-1 b
      // row by row, 8 strided partial sums combined pairwise (the one-CTA block's order)
      const LinMap mp(L.nx);
      if (mp.R)
        for (int j = L.r0 + mp.j0; j < L.r1; j += mp.R)
          for (int i = mp.i0; i < L.nx; i += mp.di) {
            float off, diag; stencil_c(L, i, j, off, diag);
            L.res[(j - L.r0) * L.nx + i] = diag > 0.f ? -(L.rhs[(j - L.r0) * L.pc + i] * L.h2) : 0.f;
          }
      cl.sync();
      for (int m = threadIdx.x; m < ncs; m += CC_THREADS) {
        const int j = m / L.nx, i = m - j * L.nx, q = owner_of(j, L.ny, cs);
        bfull[m] = cl.map_shared_rank(L.res, q)[(j - share0(q, L.ny, cs)) * L.nx + i];
      }
      __syncthreads();
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q8 = lane & 7;
      const int nown = (L.r1 - L.r0) * L.nx;
      for (int base = warp * 4; base < nown; base += (CC_THREADS / 32) * 4) {
        const int k = base + (lane >> 3);
        float sum = 0.f;
        if (k < nown)
          for (int m = q8; m < ncs; m += 8) sum = __fmaf_rn(arow[(size_t)k * ncs + m], bfull[m], sum);
        sum += __shfl_xor_sync(0xffffffffu, sum, 1);
        sum += __shfl_xor_sync(0xffffffffu, sum, 2);
        sum += __shfl_xor_sync(0xffffffffu, sum, 4);
        if (k < nown && q8 == 0) L.p[(k / L.nx + 1) * L.pc + k % L.nx] = sum;
      }
    } else {
      // the reference's 120 sweeps from zero on rank 0 over a gathered copy of the level
      LvS D;
      D.nx = L.nx; D.ny = L.ny; D.pc = L.pc; D.pu = L.pu; D.h2 = L.h2; D.rc = nullptr; lvs_derive(D);
      D.p = dense; D.rhs = D.p + L.ny * L.pc; D.ax = D.rhs + L.ny * L.pc; D.ay = D.ax + L.ny * L.pu;
      cl.sync();   // the owners' coarsest rhs is complete
      if (rank == 0) {
        for (int e = threadIdx.x; e < L.ny * L.pc; e += CC_THREADS) {
          const int j = e / L.pc, i = e - j * L.pc, q = owner_of(j, L.ny, cs), lr = j - share0(q, L.ny, cs);
          D.rhs[e] = i < L.nx ? cl.map_shared_rank(L.rhs, q)[lr * L.pc + i] : 0.f;
          D.p[e] = 0.f;
        }
        for (int e = threadIdx.x; e < L.ny * L.pu; e += CC_THREADS) {
          const int j = e / L.pu, i = e - j * L.pu, q = owner_of(j, L.ny, cs), lr = j - share0(q, L.ny, cs);
          D.ax[e] = cl.map_shared_rank(L.ax, q)[lr * L.pu + i];
        }
        for (int e = threadIdx.x; e < (L.ny + 1) * L.pc; e += CC_THREADS) {
          const int j = e / L.pc, i = e - j * L.pc;
          const int q = owner_of(j < L.ny ? j : L.ny - 1, L.ny, cs), lr = j - share0(q, L.ny, cs);
          D.ay[e] = cl.map_shared_rank(L.ay, q)[lr * L.pc + i];
        }
        __syncthreads();
        const int npair = (L.nx * L.ny + 1) >> 1;
        const int nthr = (npair + 31) & ~31;
        if ((int)threadIdx.x < nthr) {
          const CCell a = coarsest_cell(D, 2 * threadIdx.x), b = coarsest_cell(D, 2 * threadIdx.x + 1);
          const int k0 = 2 * threadIdx.x;
          const bool a_red = ((k0 % L.nx + k0 / L.nx) & 1) == 0;
          const CCell c0 = a_red ? a : b, c1 = a_red ? b : a;
          bar_coarsest(nthr);
          #pragma unroll 1
          for (int it = 0; it < 120; it++) {
            coarsest_update(D.p, L.pc, c0);
            bar_coarsest(nthr);
            coarsest_update(D.p, L.pc, c1);
            bar_coarsest(nthr);
          }
        }
        __syncthreads();
        // scatter p back to the owners' rows
        for (int e = threadIdx.x; e < L.ny * L.nx; e += CC_THREADS) {
          const int j = e / L.nx, i = e - j * L.nx, q = owner_of(j, L.ny, cs), lr = j - share0(q, L.ny, cs);
          cl.map_shared_rank(L.p, q)[(lr + 1) * L.pc + i] = D.p[j * L.pc + i];
        }
      }
    }
    cl.sync();
  }
  // ---- up
  for (int l = nl - 2; l >= lc; l--) {
    const LvC F = lv[l], Cc = lv[l + 1];
    const Halos h = halos_of(F, cl, cs);
    {
      const LinMap mp(F.nx);
      if (mp.R)
        for (int j = F.r0 + mp.j0; j < F.r1; j += mp.R) {
          const int J = j / 2, J2 = min(max(J + ((j & 1) == 1 ? 1 : -1), 0), Cc.ny - 1);
          const int qa = owner_of(J, Cc.ny, cs), qb = owner_of(J2, Cc.ny, cs);
          const float* pa = cl.map_shared_rank(Cc.p, qa) + (J - share0(qa, Cc.ny, cs) + 1) * Cc.pc;
          const float* pb = cl.map_shared_rank(Cc.p, qb) + (J2 - share0(qb, Cc.ny, cs) + 1) * Cc.pc;
          for (int i = mp.i0; i < F.nx; i += mp.di) {
            const int I = i / 2, I2 = min(max(I + ((i & 1) == 1 ? 1 : -1), 0), Cc.nx - 1);
            const float c = 0.5625f * pa[I] + 0.1875f * (pa[I2] + pb[I]) + 0.0625f * pb[I2];
            const float diag = diag_c(F, i, j);
            const int k = (j - F.r0 + 1) * F.pc + i;
            store_p(F, h, i, j, F.p[k] + (diag > 0.f ? c : 0.f));
          }
        }
    }
    cl.sync();
    const LinMap mh((F.nx + 1) >> 1);
    for (int k = 0; k < 2; k++) { pass_c(F, h, mh, 1); cl.sync(); pass_c(F, h, mh, 0); cl.sync(); }
  }
  // ---- level lc's owned rows back to global memory for the tiled level above
  const LevelDesc& G = S.lev[lc];
  for (int e = threadIdx.x; e < (V0.r1 - V0.r0) * G.nx; e += CC_THREADS) {
    const int lr = e / G.nx, i = e - lr * G.nx;
    G.p[(size_t)(V0.r0 + lr) * G.pc + i] = V0.p[(lr + 1) * V0.pc + i];
  }
}

// shared bytes of the cluster coarse phase on one CTA for one scene
size_t cluster_smem_bytes(const int* lnx, const int* lny, int lc, int nlev, int cs) {
  size_t f = 0;
  for (int l = lc; l < nlev; l++) f += level_floats(lnx[l], lny[l], cs);
  const int nc = lnx[nlev - 1] * lny[nlev - 1];
  f += up32(nc) + up32(rows_max(lny[nlev - 1], cs) * lnx[nlev - 1] * nc);
  const int pc = up32(lnx[nlev - 1]), pu = up32(lnx[nlev - 1] + 1);
  f += 2 * lny[nlev - 1] * pc + lny[nlev - 1] * pu + (lny[nlev - 1] + 1) * pc;   // the gathered coarsest
  return f * 4;
}

cudaError_t prepare_mg_cluster() {
  cudaError_t e = cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_mg_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClusterSmemMax);
  return e;
}

void launch_mg_cluster(const SceneDesc* scenes, int nscenes, SolveCtl* ctl, int cs, int count_iter, size_t smem,
                       cudaStream_t st) {
  if (nscenes <= 0) return;
  cudaLaunchConfig_t c = {};
  c.gridDim = dim3(nscenes * cs);
  c.blockDim = dim3(CC_THREADS);
  c.dynamicSmemBytes = smem;
  c.stream = st;
  cudaLaunchAttribute at[2];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = cs; at[0].val.clusterDim.y = 1; at[0].val.clusterDim.z = 1;
  at[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[1].val.programmaticStreamSerializationAllowed = pdl_enabled() ? 1 : 0;
  c.attrs = at;
  c.numAttrs = 2;
  cudaLaunchKernelEx(&c, k_mg_cluster, scenes, ctl, cs, count_iter);
}

}  // namespace cfg
