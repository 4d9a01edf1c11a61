// Host engine of the B200 gas step. See engine.h.
//
// One step (FluidSim.encodeStep, js/fluid.js:225-253) is enqueued as
//   advect -> diffuse+sources -> forces+coef+rhs0 (+ coarse coefficients)
//   -> [pressure loop: V(2,2) cycle -> residual norm / FP64 defect] -> project
// and captured once in a CUDA graph whose pressure loop is a conditional WHILE
// node: the kernel that finishes each residual reduction decides, per scene,
// whether another cycle runs and sets the node's condition on the device, so a
// step never waits on the host.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "kernels.h"

namespace cfg {

// bench.py counts these bytes as the per-step parameter upload of cfg_write_params
static_assert(kDescParamBytes == 204, "parameter block of SceneDesc");
static_assert(kDescParamBytes == 4 * PARAM_WORDS && sizeof(ParamWords) == kDescParamBytes, "parameter words");
static_assert(sizeof(PieceFloats) == sizeof(Scene::pieces), "piece block");
static_assert(kRingBytes % 4 == 0, "readback words");

namespace {
thread_local std::string g_err;

const char* kParamNames[40] = {
  "nx", "ny", "dx", "dt", "Tamb", "rhoAmb", "YOamb", "grav", "cp", "Pr", "viscMult", "diffMult",
  "reactB", "reactTa", "dHc", "sO2", "sootFormA", "sootFormTa", "sootOxA", "sootOxTa",
  "kappaSootC", "kappaGas", "exchAlpha", "depth", "charA", "charTa", "nPieces", "frame",
  "heaterX0", "heaterX1", "heaterY1", "heaterT", "burnerX0", "burnerX1", "burnerFlux", "burnerT",
  "sootDensity", "sigma", "charO2", "time"};

__global__ void k_fill_f32(float* a, int pitch, int w, int h, float v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i < w && j < h) a[(size_t)j * pitch + i] = v;
}
__global__ void k_fill_f4(float4* a, int pitch, int w, int h, float4 v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
  if (i < w && j < h) a[(size_t)j * pitch + i] = v;
}
}  // namespace

void set_error(const std::string& msg) { g_err = msg; }
const std::string& last_error() { return g_err; }
int fail(int code, const std::string& msg) { g_err = msg; return code; }
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorInvalidDevice) return CFG_ERR_NODEV;
  if (e == cudaErrorMemoryAllocation) return CFG_ERR_NOMEM;
  return CFG_ERR_IO;
}

// FluidSim defaults (js/fluid.js:35-45) from PHYS (js/config.js:12-47)
void default_params(cfg_params* p) {
  std::memset(p, 0, sizeof *p);
  const double rhoAmb = PhysConst::rhoAmb();
  p->Tamb = (float)293.15; p->rhoAmb = (float)rhoAmb; p->YOamb = 0.232f; p->grav = 9.81f;
  p->cp = 1300.f; p->Pr = 0.7f; p->viscMult = 1.f; p->diffMult = 1.f;
  p->reactB = 2.0e10f; p->reactTa = 15000.f; p->dHc = 15.0e6f; p->sO2 = (float)(15.0e6 / 13.1e6);
  p->sootFormA = 6.0e6f; p->sootFormTa = 25000.f; p->sootOxA = 5.4e8f; p->sootOxTa = 19800.f;
  p->kappaSootC = 1862.f; p->kappaGas = 0.8f; p->exchAlpha = 0.05f; p->depth = 0.8f;
  p->charA = 6.6f; p->charTa = 5800.f; p->burnerT = 600.f;
  p->sootDensity = 1800.f; p->sigma = (float)5.670374e-8; p->charO2 = 2.667f;
}

int param_index(const char* name) {
  if (!name) return -1;
  for (int i = 0; i < 40; i++) if (std::strcmp(kParamNames[i], name) == 0) return i;
  return -1;
}

// ------------------------------------------------------------------ lifetime
Engine::~Engine() {
  // nothing was allocated before the streams; keep the caller's error message intact
  if (!stream_ || cudaSetDevice(device_) != cudaSuccess) return;
  destroy_graph();
  if (stream_) cudaStreamSynchronize(stream_);
  for (auto& sc : scenes_) if (sc.arena) cudaFree(sc.arena);
  for (auto& sc : scenes_) {
    if (sc.ring.host) cudaFreeHost(sc.ring.host);
    for (auto& e : sc.ring.ev) if (e) cudaEventDestroy(e);
  }
  for (auto& w : d_wl_) if (w) cudaFree(w);
  if (d_scenes_) cudaFree(d_scenes_);
  if (d_solve_) cudaFree(d_solve_);
  if (d_ctl_) cudaFree(d_ctl_);
  if (d_dxd_) cudaFree(d_dxd_);
  if (d_alpha_) cudaFree(d_alpha_);
  if (d_scratch_) cudaFree(d_scratch_);
  if (d_rwood_) cudaFree(d_rwood_);
  if (d_image_) cudaFree(d_image_);
  if (h_ctl_pinned_) cudaFreeHost(h_ctl_pinned_);
  if (h_dt_pinned_) cudaFreeHost(h_dt_pinned_);   // d_dtv_ is its device address
  if (ev_dt_) cudaEventDestroy(ev_dt_);
  if (stream_) cudaStreamDestroy(stream_);
  if (body_stream_) cudaStreamDestroy(body_stream_);
  if (side_stream_) { cudaStreamSynchronize(side_stream_); cudaStreamDestroy(side_stream_); }
  if (ev_fork_) cudaEventDestroy(ev_fork_);
  if (ev_join_) cudaEventDestroy(ev_join_);
}

int Engine::activate() const {
  CFG_CUDA(cudaSetDevice(device_));
  return CFG_OK;
}

// The coarse block starts at the first level with at most `cells` cells whose
// arrays fit in one CTA's shared memory (else at the coarsest level).
// cs > 0: the cluster coarse phase, which starts at level 1 at the earliest (level 0
// always runs as tiled kernels) and fits each CTA's share of the levels
int Engine::choose_lc(const Scene& sc, int cells, int cs) {
  if (cs > 0) {
    for (int l = std::min(1, sc.nlev - 1); l < sc.nlev; l++)
      if (sc.lnx[l] * sc.lny[l] <= cells && cluster_smem_bytes(sc.lnx, sc.lny, l, sc.nlev, cs) <= kClusterSmemMax)
        return l;
    return sc.nlev - 1;
  }
  for (int l = 0; l < sc.nlev; l++)
    if (sc.lnx[l] * sc.lny[l] <= cells && coarse_smem_bytes(sc.lnx, sc.lny, l, sc.nlev) <= kCoarseSmemMax) return l;
  return sc.nlev - 1;
}

int Engine::init(int device, int n, const int* nx, const int* ny, const double* width, const double* dt) {
  if (n <= 0) return fail(CFG_ERR_INVAL, "scene count must be positive");
  scenes_.resize(n);
  for (int s = 0; s < n; s++) {
    Scene& sc = scenes_[s];
    if (nx[s] < 2 || ny[s] < 2 || nx[s] > 16384 || ny[s] > 16384) return fail(CFG_ERR_INVAL, "grid size out of range");
    if (!(width[s] > 0) || !(dt[s] > 0)) return fail(CFG_ERR_INVAL, "width and dt must be positive");
    sc.nx = nx[s]; sc.ny = ny[s]; sc.width = width[s];
    sc.dxd = width[s] / nx[s]; sc.dtd = dt[s]; sc.dt_cap = dt[s];
    default_params(&sc.host);
    // multigrid hierarchy (js/fluid.js:70-91), at most MAX_LEVELS levels
    int lx = sc.nx, ly = sc.ny, L = 0;
    for (int l = 0; l < MAX_LEVELS; l++) {
      sc.lnx[l] = lx; sc.lny[l] = ly; L = l + 1;
      if (lx % 2 || ly % 2 || lx * ly <= 256) break;
      lx /= 2; ly /= 2;
    }
    sc.nlev = L;
    if (sc.lnx[L - 1] * sc.lny[L - 1] > 256) return fail(CFG_ERR_RANGE, "coarsest level too large");
    sc.lc = choose_lc(sc, coarse_cells_, 0);
    coarse_smem_ = std::max(coarse_smem_, coarse_smem_bytes(sc.lnx, sc.lny, sc.lc, sc.nlev));
    const int cn = sc.lnx[L - 1] * sc.lny[L - 1], cbw = sc.lnx[L - 1];
    if (cbw <= 32) { cf_smem_ = std::max(cf_smem_, coarse_factor_smem(cn, cbw)); cf_bw_ = std::max(cf_bw_, cbw); }
  }
  int ndev = 0;
  const cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return fail(CFG_ERR_NODEV, "no CUDA device: the gas step has no CPU fallback");
  if (device < 0 || device >= ndev) return fail(CFG_ERR_INVAL, "device index out of range");
  device_ = device;
  CFG_TRY(activate());
  // CAMPFIRE_PDL=0 launches the pressure-loop kernels without programmatic dependent launch
  if (const char* v = std::getenv("CAMPFIRE_PDL")) set_pdl(v[0] != '0');
  CFG_CUDA(prepare_mg_coarse(coarse_smem_));
  CFG_CUDA(prepare_coarse_factor(cf_smem_));
  CFG_CUDA(prepare_diffuse_sources());
  CFG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  CFG_CUDA(cudaStreamCreateWithFlags(&body_stream_, cudaStreamNonBlocking));
  CFG_CUDA(cudaStreamCreateWithFlags(&side_stream_, cudaStreamNonBlocking));
  CFG_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
  CFG_CUDA(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
  CFG_CUDA(cudaEventCreateWithFlags(&ev_dt_, cudaEventDisableTiming));
  CFG_CUDA(cudaMalloc(&d_scenes_, sizeof(SceneDesc) * n));
  CFG_CUDA(cudaMalloc(&d_solve_, sizeof(SolveState) * n));
  CFG_CUDA(cudaMemset(d_solve_, 0, sizeof(SolveState) * n));
  CFG_CUDA(cudaMalloc(&d_ctl_, sizeof(SolveCtl)));
  CFG_CUDA(cudaMallocHost(&h_ctl_pinned_, sizeof(SolveCtl)));
  CFG_CUDA(cudaHostAlloc(&h_dt_pinned_, sizeof(float) * n, cudaHostAllocMapped | cudaHostAllocPortable));
  std::memset(h_dt_pinned_, 0, sizeof(float) * n);   // 0: no step has set a scene's dt yet
  CFG_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&d_dtv_), h_dt_pinned_, 0));
  CFG_CUDA(cudaMalloc(&d_dxd_, sizeof(double) * n));
  CFG_CUDA(cudaMalloc(&d_alpha_, sizeof(double) * n));
  CFG_CUDA(cudaMalloc(&d_scratch_, sizeof(double) * 64));
  for (int s = 0; s < n; s++) CFG_TRY(alloc_scene(scenes_[s]));
  CFG_TRY(build_worklists());
  for (int s = 0; s < n; s++) {
    scenes_[s].desc.solve = d_solve_ + s;
    CFG_TRY(upload_desc(s));
    CFG_TRY(write_params(s));
    CFG_TRY(reset(s));
  }
  CFG_TRY(upload_ctl());
  CFG_CUDA(cudaStreamSynchronize(st()));
  return CFG_OK;
}

// One arena per scene; every array 256-byte aligned, rows pitched to 32 elements.
namespace {
// cuTensorMapEncodeTiled from the driver (through the runtime's entry-point query,
// so the library links against cudart only)
PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

// 2D f32 map of a pitched array (w x h elements, rows `pitch` elements apart) with a
// bw x bh box; out-of-range elements read as zero
int encode_map(CUtensorMap* m, const float* base, int w, int h, int pitch, int bw, int bh) {
  auto fn = tmap_encoder();
  if (!fn) return fail(CFG_ERR_NODEV, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t dims[2] = {(cuuint64_t)w, (cuuint64_t)h};
  const cuuint64_t strides[1] = {(cuuint64_t)pitch * 4};
  const cuuint32_t box[2] = {(cuuint32_t)bw, (cuuint32_t)bh};
  const cuuint32_t es[2] = {1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(CFG_ERR_INVAL, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return CFG_OK;
}
}  // namespace

// Tensor maps of every level for the fused smoother kernels, copied into the arena.
int Engine::build_tmaps(Scene& sc) {
  static_assert(sizeof(CUtensorMap) == TMAP_BYTES, "CUtensorMap is 128 bytes");
  const SceneDesc& d = sc.desc;
  std::vector<CUtensorMap> maps((size_t)MAX_LEVELS * TM_PER_LEVEL);
  std::memset(maps.data(), 0, maps.size() * sizeof(CUtensorMap));
  for (int l = 0; l < sc.nlev; l++) {
    const LevelDesc& L = d.lev[l];
    CUtensorMap* m = &maps[(size_t)l * TM_PER_LEVEL];
    CFG_TRY(encode_map(&m[TM_P], L.p, L.nx, L.ny, L.pc, MGF_BW, MGF_BH));
    CFG_TRY(encode_map(&m[TM_PB], L.pb, L.nx, L.ny, L.pc, MGF_BW, MGF_BH));
    CFG_TRY(encode_map(&m[TM_RHS], L.rhs, L.nx, L.ny, L.pc, MGF_BW, MGF_BH));
    CFG_TRY(encode_map(&m[TM_AX], L.ax, L.nx + 1, L.ny, L.pu, MGF_BW, MGF_BH));
    CFG_TRY(encode_map(&m[TM_AY], L.ay, L.nx, L.ny + 1, L.pc, MGF_BW, MGF_BH + 1));
    CFG_TRY(encode_map(&m[TM_PC], L.p, L.nx, L.ny, L.pc, MGF_CBW, MGF_CBH));
  }
  CFG_CUDA(cudaMemcpy(const_cast<char*>(d.tmap), maps.data(), maps.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice));
  return CFG_OK;
}

int Engine::alloc_scene(Scene& sc) {
  SceneDesc& d = sc.desc;
  std::memset(&d, 0, sizeof d);
  d.nx = sc.nx; d.ny = sc.ny;
  d.pc = round_up(sc.nx, 32); d.pu = round_up(sc.nx + 1, 32);
  d.nlev = sc.nlev; d.nray = sc.nray; d.enabled = 1;
  const size_t C = (size_t)sc.ny * d.pc, Uf = (size_t)sc.ny * d.pu, Vf = (size_t)(sc.ny + 1) * d.pc;
  const int nt_fr = ((sc.nx + FR_TX - 1) / FR_TX) * ((sc.ny + FR_TY - 1) / FR_TY);
  const int nt_mg0 = ((sc.nx + MG_TX - 1) / MG_TX) * ((sc.ny + MG_TY - 1) / MG_TY);
  const int nt_up0 = ((sc.nx + MGF_TX - 1) / MGF_TX) * ((sc.ny + MGF_TY - 1) / MGF_TY);
  d.nt_fr = nt_fr; d.nt_mg0 = nt_mg0; d.nt_up0 = nt_up0; d.lc = sc.lc; d.lw = std::min(sc.lw, sc.nlev);
  struct Item { void** ptr; size_t bytes; };
  std::vector<Item> items = {
    {(void**)&d.U, Uf * 4}, {(void**)&d.U2, Uf * 4}, {(void**)&d.fx, Uf * 4},
    {(void**)&d.V, Vf * 4}, {(void**)&d.V2, Vf * 4}, {(void**)&d.fy, Vf * 4},
    {(void**)&d.T, C * 4}, {(void**)&d.T2, C * 4}, {(void**)&d.Tw, C * 4},
    {(void**)&d.Y, C * 16}, {(void**)&d.Y2, C * 16}, {(void**)&d.Yw, C * 16},
    {(void**)&d.SQ, C * 8}, {(void**)&d.cellG, C * 8},
    // acc, rad, faceW in this order: the readback ring copies them in one piece (kRingBytes)
    {(void**)&d.acc, ACC_LEN * 4}, {(void**)&d.rad, RAD_LEN * 16}, {(void**)&d.faceW, MAX_PIECES * 4 * 4},
    {(void**)&d.pieces, MAX_PIECES * PIECE_FLOATS * 4},
    {(void**)&d.p64, (size_t)sc.nx * sc.ny * 8}, {(void**)&d.rhs64, (size_t)sc.nx * sc.ny * 8},
    {(void**)&d.part, (size_t)std::max(std::max(nt_fr, nt_mg0), nt_up0) * 72},   // up to 9 sums per tile
    {(void**)&d.r64, (size_t)sc.nx * sc.ny * 8}, {(void**)&d.dA, (size_t)sc.nx * sc.ny * 8},
    {(void**)&d.dB, (size_t)sc.nx * sc.ny * 8}, {(void**)&d.q64, (size_t)sc.nx * sc.ny * 8},
    {(void**)&d.tmap, (size_t)MAX_LEVELS * TM_PER_LEVEL * TMAP_BYTES},
    {(void**)&d.cinv, (size_t)2 * sc.lnx[sc.nlev - 1] * sc.lny[sc.nlev - 1] * cinv_ld(sc.lnx[sc.nlev - 1] * sc.lny[sc.nlev - 1]) * 4},
  };
  double h = sc.dxd;
  for (int l = 0; l < sc.nlev; l++) {
    LevelDesc& L = d.lev[l];
    L.nx = sc.lnx[l]; L.ny = sc.lny[l];
    L.pc = round_up(L.nx, 32); L.pu = round_up(L.nx + 1, 32);
    L.h2 = (float)(h * h);
    h *= 2;
    const size_t lc = (size_t)L.ny * L.pc;
    items.push_back({(void**)&L.p, lc * 4});
    items.push_back({(void**)&L.pb, lc * 4});
    items.push_back({(void**)&L.rhs, lc * 4});
    items.push_back({(void**)&L.ax, (size_t)L.ny * L.pu * 4});
    items.push_back({(void**)&L.ay, (size_t)(L.ny + 1) * L.pc * 4});
  }
  size_t total = 0;
  for (auto& it : items) total += (it.bytes + 255) / 256 * 256;
  void* arena = nullptr;
  cudaError_t e = cudaMalloc(&arena, total);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(scene arena)");
  CFG_CUDA(cudaMemset(arena, 0, total));
  sc.arena = arena; sc.arena_bytes = total;
  size_t off = 0;
  sc.items.clear();
  for (auto& it : items) {
    *it.ptr = (char*)arena + off;
    off += (it.bytes + 255) / 256 * 256;
    // the coarsest inverses are state: with the pipelined coarse solve the next step uses the
    // one factored during the last step
    const bool scratch = it.ptr == (void**)&d.tmap || it.ptr == (void**)&d.part;
    sc.items.push_back({*it.ptr, it.bytes, !scratch});
  }
  if ((char*)d.rad != (char*)d.acc + kRbRadOff || (char*)d.faceW != (char*)d.acc + kRbFaceWOff)
    return fail(CFG_ERR_INVAL, "readback arrays not laid out as the ring expects");
  return build_tmaps(sc);
}

// ------------------------------------------------------------------ checkpoints
// File: "CFGCKPT1", u32 version 2, nx, ny, nlev, nitems; f64 time, dt, dt_cap, cfl,
// width; u32 frame, nray; the host params (cfg_params); the host pieces
// (64 x 20 f32); the device's parameter block (the uniform and step controls,
// which the CFL step updates on the device); the scene's SolveState; then per
// state array of the arena (allocation order, pitched as allocated) u64 bytes +
// the bytes; last u64 FNV-1a of everything after the magic.
namespace {
constexpr char kCkptMagic[8] = {'C', 'F', 'G', 'C', 'K', 'P', 'T', '1'};
// 2: the solve state carries the device clock; acc, rad, faceW adjacent in the arena
constexpr uint32_t kCkptVersion = 2u;
struct CkptHead {
  uint32_t version, nx, ny, nlev, nitems, frame, nray, pad;
  double time, dt, dt_cap, cfl, width;
};
struct Fnv64 {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
  }
};
struct File {
  FILE* f = nullptr;
  ~File() { if (f) std::fclose(f); }
};
}  // namespace

int Engine::checkpoint_save(int s, const char* path) {
  if (!path) return fail(CFG_ERR_INVAL, "null path");
  CFG_TRY(activate());
  CFG_CUDA(cudaStreamSynchronize(st()));
  const Scene& sc = scenes_[s];
  int nstate = 0;
  for (auto& it : sc.items) nstate += it.state ? 1 : 0;
  std::vector<char> dparams(kDescParamBytes);
  SolveState ss{};
  CFG_CUDA(cudaMemcpy(dparams.data(), d_scenes_ + s, kDescParamBytes, cudaMemcpyDeviceToHost));
  CFG_CUDA(cudaMemcpy(&ss, sc.desc.solve, sizeof ss, cudaMemcpyDeviceToHost));
  CkptHead h{kCkptVersion, (uint32_t)sc.nx, (uint32_t)sc.ny, (uint32_t)sc.nlev, (uint32_t)nstate, sc.frame, (uint32_t)sc.nray, 0u,
             sc.cfl > 0 ? ss.time : sc.time, sc.dtd, sc.dt_cap, sc.cfl, sc.width};
  File out;
  out.f = std::fopen(path, "wb");
  if (!out.f) return fail(CFG_ERR_IO, std::string("cannot write ") + path);
  Fnv64 sum;
  auto put = [&](const void* p, size_t n) {
    sum.add(p, n);
    return std::fwrite(p, 1, n, out.f) == n;
  };
  bool ok = std::fwrite(kCkptMagic, 1, 8, out.f) == 8;
  ok = ok && put(&h, sizeof h) && put(&sc.host, sizeof sc.host) && put(sc.pieces, sizeof sc.pieces) &&
       put(dparams.data(), dparams.size()) && put(&ss, sizeof ss);
  std::vector<char> buf;
  for (auto& it : sc.items) {
    if (!ok) break;
    if (!it.state) continue;
    buf.resize(it.bytes);
    CFG_CUDA(cudaMemcpy(buf.data(), it.ptr, it.bytes, cudaMemcpyDeviceToHost));
    const uint64_t n = it.bytes;
    ok = put(&n, 8) && put(buf.data(), it.bytes);
  }
  const uint64_t digest = sum.h;
  ok = ok && std::fwrite(&digest, 1, 8, out.f) == 8;
  if (!ok) return fail(CFG_ERR_IO, std::string("short write to ") + path);
  return CFG_OK;
}

int Engine::checkpoint_load(int s, const char* path) {
  if (!path) return fail(CFG_ERR_INVAL, "null path");
  CFG_TRY(activate());
  CFG_CUDA(cudaStreamSynchronize(st()));
  Scene& sc = scenes_[s];
  File in;
  in.f = std::fopen(path, "rb");
  if (!in.f) return fail(CFG_ERR_NOENT, std::string("cannot read ") + path);
  Fnv64 sum;
  auto get = [&](void* p, size_t n) {
    if (std::fread(p, 1, n, in.f) != n) return false;
    sum.add(p, n);
    return true;
  };
  char magic[8];
  if (std::fread(magic, 1, 8, in.f) != 8 || std::memcmp(magic, kCkptMagic, 8) != 0)
    return fail(CFG_ERR_INVAL, std::string(path) + " is not a gas-step checkpoint");
  CkptHead h;
  cfg_params host;
  float pieces[MAX_PIECES * PIECE_FLOATS];
  std::vector<char> dparams(kDescParamBytes);
  SolveState ss;
  if (!get(&h, sizeof h) || !get(&host, sizeof host) || !get(pieces, sizeof pieces) ||
      !get(dparams.data(), dparams.size()) || !get(&ss, sizeof ss))
    return fail(CFG_ERR_IO, std::string("truncated checkpoint ") + path);
  int nstate = 0;
  for (auto& it : sc.items) nstate += it.state ? 1 : 0;
  if (h.version != kCkptVersion) return fail(CFG_ERR_INVAL, "unsupported checkpoint version");
  if ((int)h.nx != sc.nx || (int)h.ny != sc.ny || (int)h.nlev != sc.nlev || (int)h.nitems != nstate)
    return fail(CFG_ERR_RANGE, "checkpoint grid " + std::to_string(h.nx) + "x" + std::to_string(h.ny) +
                                   " does not match this scene");
  // read every array before touching the scene, so a bad file leaves it unchanged
  std::vector<std::vector<char>> arrays;
  for (auto& it : sc.items) {
    if (!it.state) continue;
    uint64_t n = 0;
    if (!get(&n, 8) || n != it.bytes) return fail(CFG_ERR_INVAL, "checkpoint array sizes do not match this scene");
    arrays.emplace_back(it.bytes);
    if (!get(arrays.back().data(), it.bytes)) return fail(CFG_ERR_IO, std::string("truncated checkpoint ") + path);
  }
  uint64_t digest = 0;
  const uint64_t expect = sum.h;
  if (std::fread(&digest, 1, 8, in.f) != 8 || digest != expect)
    return fail(CFG_ERR_INVAL, std::string("checkpoint checksum mismatch in ") + path);
  // the handle's stream does not order against the legacy stream of the blocking copies
  // below: let its queued work finish before the arrays are replaced
  CFG_CUDA(cudaStreamSynchronize(st()));
  size_t k = 0;
  for (auto& it : sc.items) {
    if (!it.state) continue;
    CFG_CUDA(cudaMemcpy(it.ptr, arrays[k].data(), it.bytes, cudaMemcpyHostToDevice));
    k++;
  }
  sc.host = host;
  std::memcpy(sc.pieces, pieces, sizeof pieces);
  sc.time = h.time; sc.dtd = h.dt; sc.dt_cap = h.dt_cap; sc.cfl = h.cfl; sc.frame = h.frame; sc.nray = (int)h.nray;
  const double cfl = sc.cfl;
  sc.cfl = 0;   // write_params must not read the device's step back: it is restored below
  sc.dt_on_device = false;
  CFG_TRY(write_params(s));
  // write_params enqueues its parameter upload on the stream; it must land before the
  // saved block is restored below (a blocking copy on the legacy stream)
  CFG_CUDA(cudaStreamSynchronize(st()));
  sc.cfl = cfl;
  // the device's parameter block as saved (CFL step included); this slot's enabled flag kept
  SceneDesc tmp = sc.desc;
  std::memcpy(&tmp, dparams.data(), kDescParamBytes);
  tmp.enabled = sc.enabled ? 1 : 0;
  std::memcpy(&sc.desc, &tmp, kDescParamBytes);
  sc.P = sc.desc.P;
  sc.diff_sub = sc.desc.diff_sub;
  sc.diff_dt = sc.desc.diff_dt;
  dt_from_step_ = false;
  CFG_CUDA(cudaMemcpy(d_scenes_ + s, &sc.desc, kDescParamBytes, cudaMemcpyHostToDevice));
  CFG_CUDA(cudaMemcpy(sc.desc.solve, &ss, sizeof ss, cudaMemcpyHostToDevice));
  graph_dirty_ = true;
  return CFG_OK;
}

int Engine::build_worklists() {
  std::vector<Work> lists[WL_COUNT];
  const int n = (int)scenes_.size();
  auto tiles = [&](std::vector<Work>& v, int s, int w, int h, int TX, int TY) {
    int t = 0;
    for (int ty = 0; ty < (h + TY - 1) / TY; ty++)
      for (int tx = 0; tx < (w + TX - 1) / TX; tx++) v.push_back(Work{s, tx, ty, t++});
  };
  for (int s = 0; s < n; s++) {
    const Scene& sc = scenes_[s];
    tiles(lists[WL_ADV], s, sc.nx, sc.ny, TILE_TX[tiles_[TK_ADVECT]], TILE_TY[tiles_[TK_ADVECT]]);
    tiles(lists[WL_DS], s, sc.nx, sc.ny, TILE_TX[tiles_[TK_DIFFSRC]], TILE_TY[tiles_[TK_DIFFSRC]]);
    tiles(lists[WL_FR], s, sc.nx, sc.ny, TILE_TX[tiles_[TK_FORCES]], TILE_TY[tiles_[TK_FORCES]]);
    tiles(lists[WL_PR], s, sc.nx, sc.ny, PR_TX, PR_TY);
    tiles(lists[WL_GEO], s, sc.nx + 1, sc.ny + 1, GEO_TX, GEO_TY);
    tiles(lists[WL_MG0], s, sc.nx, sc.ny, MG_TX, MG_TY);
    for (int l = 0; l + 1 < sc.nlev; l++) {
      tiles(lists[WL_MGV0 + l], s, sc.lnx[l], sc.lny[l], MG_TX, MG_TY);
      tiles(lists[WL_MGC0 + l], s, sc.lnx[l + 1], sc.lny[l + 1], MG_TX, MG_TY);
    }
    for (int l = 0; l < sc.lc; l++) tiles(lists[WL_MGD0 + l], s, sc.lnx[l], sc.lny[l], MGF_TX, MGF_TY);
  }
  for (int k = 0; k < WL_COUNT; k++) {
    nwl_[k] = (int)lists[k].size();
    if (nwl_[k] == 0) continue;
    CFG_CUDA(cudaMalloc(&d_wl_[k], sizeof(Work) * lists[k].size()));
    CFG_CUDA(cudaMemcpy(d_wl_[k], lists[k].data(), sizeof(Work) * lists[k].size(), cudaMemcpyHostToDevice));
  }
  return CFG_OK;
}

int Engine::set_coarse_cluster(int cs) {
  if (cs != 0 && cs != 2 && cs != 4 && cs != 8 && cs != 16)
    return fail(CFG_ERR_INVAL, "the coarse cluster size must be 0 (one CTA), 2, 4, 8 or 16");
  for (const auto& sc : scenes_)
    if (cs > 0 && sc.nlev < 2) return fail(CFG_ERR_INVAL, "the cluster coarse phase needs two levels or more in every scene");
  const int prev = coarse_cluster_;
  coarse_cluster_ = cs;
  const int rc = set_coarse_cells(coarse_cells_);
  if (rc != CFG_OK) coarse_cluster_ = prev;
  return rc;
}

int Engine::set_coarse_cells(int cells) {
  if (cells < 1) return fail(CFG_ERR_INVAL, "coarse cells must be >= 1");
  CFG_TRY(activate());
  CFG_CUDA(cudaStreamSynchronize(st()));
  const int cs = coarse_cluster_;
  if (cs > 0 && w_cells_ > 0) return fail(CFG_ERR_INVAL, "the W tail runs in the one-CTA coarse block only");
  size_t smem = 0;
  std::vector<int> lcs(scenes_.size()), lws(scenes_.size());
  for (size_t s = 0; s < scenes_.size(); s++) {
    const Scene& sc = scenes_[s];
    // the W tail: level nlev - 3 (two above the coarsest) visits level nlev - 2 twice when it has
    // at most w_cells_ cells; it starts the coarse block at the latest
    int lw = MAX_LEVELS;
    if (w_cells_ > 0 && sc.nlev >= 3 && sc.lnx[sc.nlev - 3] * sc.lny[sc.nlev - 3] <= w_cells_) lw = sc.nlev - 3;
    lws[s] = lw;
    lcs[s] = choose_lc(sc, std::max(cells, lw < sc.nlev ? sc.lnx[lw] * sc.lny[lw] : 0), cs);
    if (lw < sc.nlev && lcs[s] > lw)
      return fail(CFG_ERR_RANGE, "the W tail's levels do not fit in the coarse block's shared memory");
    smem = std::max(smem, cs > 0 ? cluster_smem_bytes(sc.lnx, sc.lny, lcs[s], sc.nlev, cs)
                                 : coarse_smem_bytes(sc.lnx, sc.lny, lcs[s], sc.nlev));
  }
  if (cs > 0) {
    if (smem > kClusterSmemMax) return fail(CFG_ERR_RANGE, "the coarse levels do not fit in the cluster's shared memory");
    CFG_CUDA(prepare_mg_cluster());
    cluster_smem_ = smem;
  } else {
    if (smem > kCoarseSmemMax) return fail(CFG_ERR_RANGE, "the coarsest level does not fit in one CTA's shared memory");
    CFG_CUDA(prepare_mg_coarse(smem));
    coarse_smem_ = smem;
  }
  coarse_cells_ = cells;
  for (size_t s = 0; s < scenes_.size(); s++) {
    scenes_[s].lc = lcs[s];
    scenes_[s].desc.lc = lcs[s];
    scenes_[s].lw = lws[s];
    scenes_[s].desc.lw = std::min(lws[s], scenes_[s].nlev);
    CFG_TRY(upload_desc((int)s));
  }
  for (int k = 0; k < WL_COUNT; k++) {
    if (d_wl_[k]) cudaFree(d_wl_[k]);
    d_wl_[k] = nullptr;
    nwl_[k] = 0;
  }
  CFG_TRY(build_worklists());
  graph_dirty_ = true;
  CFG_CUDA(cudaStreamSynchronize(st()));
  return CFG_OK;
}

// The pressure loop's cycle shape: the W tail when the level two above the coarsest has at most
// `cells` cells (0: the V-cycle). The coarse block is re-chosen so that it holds that level.
int Engine::set_coarse_w(int cells) {
  if (cells < 0) return fail(CFG_ERR_INVAL, "W cells must be >= 0");
  if (cells > 0 && coarse_cluster_ > 0) return fail(CFG_ERR_INVAL, "the W tail runs in the one-CTA coarse block only");
  const int prev = w_cells_;
  w_cells_ = cells;
  const int rc = set_coarse_cells(coarse_cells_);
  if (rc != CFG_OK) {
    w_cells_ = prev;
    set_coarse_cells(coarse_cells_);
  }
  return rc;
}

// Tile shapes of the advection, diffusion + sources and forces kernels (indices into
// TILE_TX/TILE_TY): the work lists are rebuilt, and each scene's forces tile count (its
// reduction's arrivals) follows. Every shape gives the same bits.
int Engine::set_tiles(int advect, int diffsrc, int forces) {
  for (int v : {advect, diffsrc, forces})
    if (v < 0 || v >= kTileShapes) return fail(CFG_ERR_INVAL, "tile shape must be 0 (32x8), 1 (64x8) or 2 (32x16)");
  CFG_TRY(activate());
  CFG_CUDA(cudaStreamSynchronize(st()));
  tiles_[TK_ADVECT] = advect; tiles_[TK_DIFFSRC] = diffsrc; tiles_[TK_FORCES] = forces;
  const int tx = TILE_TX[forces], ty = TILE_TY[forces];
  for (int s = 0; s < nscenes(); s++) {
    Scene& sc = scenes_[s];
    sc.desc.nt_fr = ((sc.nx + tx - 1) / tx) * ((sc.ny + ty - 1) / ty);
    // only the tile count changes: the device's parameter block (a CFL step's dt) stays
    CFG_CUDA(cudaMemcpyAsync(&d_scenes_[s].nt_fr, &sc.desc.nt_fr, sizeof(int), cudaMemcpyHostToDevice, st()));
  }
  for (int k = 0; k < WL_COUNT; k++) {
    if (d_wl_[k]) cudaFree(d_wl_[k]);
    d_wl_[k] = nullptr;
    nwl_[k] = 0;
  }
  CFG_TRY(build_worklists());
  graph_dirty_ = true;
  CFG_CUDA(cudaStreamSynchronize(st()));
  return CFG_OK;
}

// The autotuner of the tile shapes: each of the three kernels is timed (`iters` launches
// back to back, CUDA events on the stream) under every shape on the current state, and the
// fastest shapes are kept. The kernels rewrite their outputs as they run, so the state
// changes (use a scratch scene); ms[k * kTileShapes + s]: kernel k, shape s.
int Engine::autotune_tiles(int iters, int* best, double* ms) {
  if (iters < 1 || !best) return fail(CFG_ERR_INVAL, "bad argument");
  const int keep[TK_COUNT] = {tiles_[0], tiles_[1], tiles_[2]};
  const char* names[TK_COUNT] = {"advect", "diffuse_sources", "forces"};
  double tbest[TK_COUNT] = {1e300, 1e300, 1e300};
  for (int k = 0; k < TK_COUNT; k++) best[k] = keep[k];
  for (int shape = 0; shape < kTileShapes; shape++) {
    CFG_TRY(set_tiles(shape, shape, shape));
    for (int k = 0; k < TK_COUNT; k++) {
      double t = 0, b = 0, n = 0;
      CFG_TRY(time_kernel(names[k], iters, &t, &b, &n));
      if (ms) ms[k * kTileShapes + shape] = t;
      if (t < tbest[k]) { tbest[k] = t; best[k] = shape; }
    }
  }
  return set_tiles(best[0], best[1], best[2]);
}

int Engine::upload_desc(int s) {
  // a CFL step the device owns survives a full descriptor upload
  Scene& sc = scenes_[s];
  if (sc.dt_on_device && sc.cfl > 0) {
    SceneDesc dev;
    CFG_CUDA(cudaMemcpyAsync(&dev, d_scenes_ + s, kDescParamBytes, cudaMemcpyDeviceToHost, st()));
    CFG_CUDA(cudaStreamSynchronize(st()));
    sc.desc.P.dt = dev.P.dt; sc.desc.diff_sub = dev.diff_sub; sc.desc.diff_dt = dev.diff_dt;
    sc.P.dt = dev.P.dt; sc.diff_sub = dev.diff_sub; sc.diff_dt = dev.diff_dt;
    sc.dtd = (double)dev.P.dt;
  }
  dt_from_step_ = false;
  CFG_CUDA(cudaMemcpyAsync(d_scenes_ + s, &scenes_[s].desc, sizeof(SceneDesc), cudaMemcpyHostToDevice, st()));
  return CFG_OK;
}
int Engine::upload_descs() {
  for (int s = 0; s < (int)scenes_.size(); s++) CFG_TRY(upload_desc(s));
  return CFG_OK;
}
int Engine::upload_ctl() {
  SolveCtl c{};
  c.mode = mode_; c.ncycles = ncycles_; c.max_cycles = max_cycles_; c.min_cycles = 1; c.tol = tol_;
  int en = 0;
  for (auto& sc : scenes_) en += sc.enabled ? 1 : 0;
  c.nscenes = en; c.nactive = en; c.any_active = 1; c.scenes_done = 0;
  c.iter = 0; c.hard_cap = std::max(ncycles_, max_cycles_) + 1;
  c.coarse_direct = (mode_ != CFG_SOLVE_FIXED && coarse_direct_) ? 1 : 0;
  c.use_cond = ctl_use_cond_ == 1 ? 1 : 0;
  c.krylov = krylov() ? 1 : 0;
  c.cond = cond_handle_;
  *h_ctl_pinned_ = c;
  CFG_CUDA(cudaMemcpyAsync(d_ctl_, h_ctl_pinned_, sizeof(SolveCtl), cudaMemcpyHostToDevice, st()));
  CFG_CUDA(cudaStreamSynchronize(st()));
  return CFG_OK;
}

// Diffusion sub-steps for dt (js/fluid.js:190-198, JS double arithmetic)
static int substeps(double dt, double dx, double alpha) {
  int n = (int)std::ceil(dt / (dx * dx / (4.5 * alpha)));
  n = std::min(5, n % 2 ? n : n + 1);
  return n < 1 ? 1 : n;
}

// The largest diffusion sub-step count of the enabled scenes (the step graph's diffusion
// kernel is instantiated for it). A CFL scene's device may move dt anywhere up to dt_cap
// without the host seeing it, so its count at dt_cap counts too.
int Engine::max_sub() const {
  int m = 1;
  for (auto& sc : scenes_) {
    if (!sc.enabled) continue;
    m = std::max(m, sc.diff_sub);
    if (sc.cfl > 0 && sc.alpha > 0) m = std::max(m, substeps(sc.dt_cap, sc.dxd, sc.alpha));
  }
  return m;
}
int Engine::max_levels() const {
  int m = 1;
  for (auto& sc : scenes_) m = std::max(m, sc.nlev);
  return m;
}

// ------------------------------------------------------------------ FluidSim surface
// reset() (js/fluid.js:162-176)
int Engine::reset(int s) {
  CFG_TRY(activate());
  Scene& sc = scenes_[s];
  SceneDesc& d = sc.desc;
  cudaStream_t q = st();
  const float Tamb = (float)PhysConst::Tamb;
  auto fill = [&](float* a, int pitch, int w, int h, float v) {
    k_fill_f32<<<dim3((w + 255) / 256, h), 256, 0, q>>>(a, pitch, w, h, v);
  };
  auto fill4 = [&](float4* a, int pitch, int w, int h, float4 v) {
    k_fill_f4<<<dim3((w + 255) / 256, h), 256, 0, q>>>(a, pitch, w, h, v);
  };
  for (float* a : {d.T, d.T2, d.Tw}) fill(a, d.pc, sc.nx, sc.ny, Tamb);
  const float4 y0 = make_float4(0.f, sc.host.YOamb, 0.f, 0.f);
  for (float4* a : {d.Y, d.Y2, d.Yw}) fill4(a, d.pc, sc.nx, sc.ny, y0);
  for (float* a : {d.U, d.U2}) fill(a, d.pu, sc.nx + 1, sc.ny, 0.f);
  for (float* a : {d.V, d.V2}) fill(a, d.pc, sc.nx, sc.ny + 1, 0.f);
  CFG_CUDA(cudaMemsetAsync(d.SQ, 0, (size_t)sc.ny * d.pc * 8, q));
  CFG_CUDA(cudaMemsetAsync(d.acc, 0, ACC_LEN * 4, q));
  CFG_CUDA(cudaMemsetAsync(d.rad, 0, RAD_LEN * 16, q));
  for (int l = 0; l < sc.nlev; l++) {
    CFG_CUDA(cudaMemsetAsync(d.lev[l].p, 0, (size_t)d.lev[l].ny * d.lev[l].pc * 4, q));
    CFG_CUDA(cudaMemsetAsync(d.lev[l].pb, 0, (size_t)d.lev[l].ny * d.lev[l].pc * 4, q));
  }
  CFG_CUDA(cudaMemsetAsync(d.p64, 0, (size_t)sc.nx * sc.ny * 8, q));
  // no coarsest inverse of an earlier state survives a reset (direct_ok, cinv_cur, direct_ok_next)
  CFG_CUDA(cudaMemsetAsync(&d_solve_[s].direct_ok, 0, 3 * sizeof(int), q));
  CFG_CUDA(cudaMemsetAsync(&d_solve_[s].time, 0, sizeof(double), q));   // the CFL step's device clock
  CFG_CUDA(cudaGetLastError());
  sc.time = 0;
  sc.dt_on_device = false;
  return CFG_OK;
}

int Engine::set_param(int s, const char* name, double v) {
  const int i = param_index(name);
  if (i < 0) return fail(CFG_ERR_NOENT, std::string("unknown param ") + (name ? name : "(null)"));
  char* base = reinterpret_cast<char*>(&scenes_[s].host) + 4 * i;
  if (i == 0 || i == 1 || i == 26) { int32_t x = (int32_t)v; std::memcpy(base, &x, 4); }
  else if (i == 27) { uint32_t x = (uint32_t)v; std::memcpy(base, &x, 4); }
  else { float x = (float)v; std::memcpy(base, &x, 4); }
  return CFG_OK;
}
int Engine::get_param(int s, const char* name, double* v) {
  const int i = param_index(name);
  if (i < 0) return fail(CFG_ERR_NOENT, std::string("unknown param ") + (name ? name : "(null)"));
  if (!v) return fail(CFG_ERR_INVAL, "null output");
  const char* base = reinterpret_cast<const char*>(&scenes_[s].host) + 4 * i;
  if (i == 0 || i == 1 || i == 26) { int32_t x; std::memcpy(&x, base, 4); *v = x; }
  else if (i == 27) { uint32_t x; std::memcpy(&x, base, 4); *v = x; }
  else { float x; std::memcpy(&x, base, 4); *v = x; }
  return CFG_OK;
}
int Engine::set_dt(int s, double dt) {
  if (!(dt > 0)) return fail(CFG_ERR_INVAL, "dt must be positive");
  scenes_[s].dtd = dt; scenes_[s].dt_cap = dt;
  scenes_[s].dt_on_device = false;
  return CFG_OK;
}

// writeParams() (js/fluid.js:180-199)
int Engine::write_params(int s) {
  CFG_TRY(activate());
  Scene& sc = scenes_[s];
  // With a CFL step that a step of this scene has already taken, the device owns dt: the
  // upload below leaves dt and the diffusion sub-steps as that step set them, so nothing
  // here waits for the GPU. The host's copy of dt follows the step's pinned copy once it
  // has landed. Otherwise (no step since set_cfl, a staged update) the device's dt is read
  // back before the upload.
  const bool device_dt = sc.cfl > 0 && sc.desc.solve && sc.dt_on_device && sc.enabled;
  if (device_dt && dt_from_step_) {
    const cudaError_t q = cudaEventQuery(ev_dt_);
    if (q == cudaSuccess) {
      if (h_dt_pinned_[s] > 0.f) sc.dtd = (double)h_dt_pinned_[s];
    } else if (q != cudaErrorNotReady) {
      return cuda_fail(q, "cudaEventQuery(step dt)");
    }
  } else if (!device_dt && sc.cfl > 0 && sc.desc.solve) {
    float dt = 0.f;
    CFG_CUDA(cudaMemcpyAsync(&dt, (char*)(d_scenes_ + s) + offsetof(SceneDesc, P) + offsetof(cfg_params, dt), 4,
                             cudaMemcpyDeviceToHost, st()));
    CFG_CUDA(cudaStreamSynchronize(st()));
    if (dt > 0.f) sc.dtd = (double)dt;
  }
  sc.host.nx = sc.nx; sc.host.ny = sc.ny; sc.host.dx = (float)sc.dxd; sc.host.dt = (float)sc.dtd;
  sc.host.time = (float)sc.time; sc.host.frame = sc.frame;
  sc.P = sc.host;
  const double Tmax = 2200, mu = 1.716e-5 * std::pow(Tmax / 273.15, 1.5) * 383.55 / (Tmax + 110.4);
  sc.alpha = mu / PhysConst::Pr * (double)sc.host.diffMult / (PhysConst::rhoAmb() * PhysConst::Tamb / Tmax);
  const int n = substeps(sc.dtd, sc.dxd, sc.alpha);
  sc.diff_sub = n;
  sc.diff_dt = (float)(sc.dtd / n);
  SceneDesc& d = sc.desc;
  d.P = sc.P; d.diff_sub = n; d.diff_dt = sc.diff_dt;
  d.cfl = (float)sc.cfl; d.dt_cap = (float)sc.dt_cap; d.nray = sc.nray; d.enabled = sc.enabled ? 1 : 0;
  // only the leading scalar block changes here (the uniform and the step controls): one kernel
  // on the stream with the block as its parameter (no copy engine, nothing to wait for), which
  // with a step-owned dt leaves P.dt and (diff_sub, diff_dt) as the step set them
  {
    ParamWords b;
    std::memcpy(b.w, &d, kDescParamBytes);
    int skip = -1, s0 = -1, s1 = -1;
    if (device_dt) {
      skip = (int)((offsetof(SceneDesc, P) + offsetof(cfg_params, dt)) / 4);
      s0 = (int)(offsetof(SceneDesc, diff_sub) / 4);
      s1 = (int)(offsetof(SceneDesc, cfl) / 4);
    }
    launch_write_params(reinterpret_cast<uint32_t*>(d_scenes_ + s), b, skip, s0, s1, st());
    CFG_CUDA(cudaGetLastError());
  }
  if (sc.dxd != sc.up_dxd) {
    CFG_CUDA(cudaMemcpyAsync(d_dxd_ + s, &sc.dxd, 8, cudaMemcpyHostToDevice, st()));
    sc.up_dxd = sc.dxd;
  }
  if (sc.alpha != sc.up_alpha) {
    CFG_CUDA(cudaMemcpyAsync(d_alpha_ + s, &sc.alpha, 8, cudaMemcpyHostToDevice, st()));
    sc.up_alpha = sc.alpha;
  }
  if (graph_sub_ >= 0 && max_sub() > graph_sub_) graph_dirty_ = true;
  return CFG_OK;
}
int Engine::write_params_all() {
  for (int s = 0; s < (int)scenes_.size(); s++) CFG_TRY(write_params(s));
  return CFG_OK;
}

// uploadPieces(data, n) (js/fluid.js:201-204)
int Engine::upload_pieces(int s, const float* data, int n) {
  if (n < 0 || n > MAX_PIECES) return fail(CFG_ERR_INVAL, "piece count out of range");
  if (!data && n > 0) return fail(CFG_ERR_INVAL, "null piece data");
  CFG_TRY(activate());
  Scene& sc = scenes_[s];
  sc.host.nPieces = n;
  std::memset(sc.pieces, 0, sizeof sc.pieces);
  if (data) std::memcpy(sc.pieces, data, sizeof sc.pieces);
  // the block as the parameter of one kernel on the stream (no copy engine, no wait)
  PieceFloats b;
  std::memcpy(b.f, sc.pieces, sizeof sc.pieces);
  launch_write_pieces(sc.desc.pieces, b, st());
  CFG_CUDA(cudaGetLastError());
  return CFG_OK;
}

int Engine::clear_geometry(int s) {
  CFG_TRY(activate());
  CFG_CUDA(cudaMemsetAsync(scenes_[s].desc.faceW, 0, MAX_PIECES * 4 * 4, st()));
  return CFG_OK;
}

int Engine::geometry(int s) {
  CFG_TRY(activate());
  // this scene's tiles are a contiguous run of the geometry work list
  int off = 0;
  for (int q = 0; q < s; q++) off += ((scenes_[q].nx + 1 + GEO_TX - 1) / GEO_TX) * ((scenes_[q].ny + 1 + GEO_TY - 1) / GEO_TY);
  const int cnt = ((scenes_[s].nx + 1 + GEO_TX - 1) / GEO_TX) * ((scenes_[s].ny + 1 + GEO_TY - 1) / GEO_TY);
  launch_geometry(d_scenes_, d_wl_[WL_GEO] + off, cnt, st());
  CFG_CUDA(cudaGetLastError());
  return CFG_OK;
}
int Engine::geometry_all() {
  CFG_TRY(activate());
  for (int s = 0; s < (int)scenes_.size(); s++) CFG_TRY(clear_geometry(s));
  launch_geometry(d_scenes_, d_wl_[WL_GEO], nwl_[WL_GEO], st());
  CFG_CUDA(cudaGetLastError());
  return CFG_OK;
}

int Engine::radiation(int s) {
  CFG_TRY(activate());
  const Scene& sc = scenes_[s];
  const int np = std::min(std::max(sc.desc.P.nPieces, 0), MAX_PIECES);
  launch_radiation(d_scenes_, s, np * 4 + N_FLOOR, sc.nray, st());
  CFG_CUDA(cudaGetLastError());
  return CFG_OK;
}
int Engine::set_frame(int s, uint32_t f) { scenes_[s].frame = f; return CFG_OK; }
int Engine::set_cfl(int s, double cfl, double dt_cap) {
  if (cfl < 0 || !(dt_cap > 0)) return fail(CFG_ERR_INVAL, "cfl must be >= 0 and dt_cap > 0");
  CFG_TRY(activate());
  Scene& sc = scenes_[s];
  if (cfl > 0 && !(sc.cfl > 0) && sc.desc.solve)   // the device clock starts from the host's
    CFG_CUDA(cudaMemcpyAsync(&d_solve_[s].time, &sc.time, sizeof(double), cudaMemcpyHostToDevice, st()));
  if (!(cfl > 0) && sc.cfl > 0 && sc.desc.solve) {  // and the host's clock and dt from the device's
    double t = 0;
    float dt = 0.f;
    CFG_CUDA(cudaMemcpyAsync(&t, &d_solve_[s].time, sizeof t, cudaMemcpyDeviceToHost, st()));
    CFG_CUDA(cudaMemcpyAsync(&dt, (char*)(d_scenes_ + s) + offsetof(SceneDesc, P) + offsetof(cfg_params, dt), 4,
                             cudaMemcpyDeviceToHost, st()));
    CFG_CUDA(cudaStreamSynchronize(st()));
    sc.time = t;
    if (dt > 0.f) sc.dtd = (double)dt;
  }
  sc.cfl = cfl; sc.dt_cap = dt_cap;
  sc.dt_on_device = false;
  // the step controls take effect with the next step, as the solver settings do (not at the
  // next cfg_write_params): the descriptor's cfl and dt_cap are updated on the device now
  sc.desc.cfl = (float)cfl; sc.desc.dt_cap = (float)dt_cap;
  static_assert(offsetof(SceneDesc, dt_cap) == offsetof(SceneDesc, cfl) + sizeof(float), "cfl, dt_cap adjacent");
  CFG_CUDA(cudaMemcpyAsync(&d_scenes_[s].cfl, &sc.desc.cfl, 2 * sizeof(float), cudaMemcpyHostToDevice, st()));
  graph_dirty_ = true;
  dt_from_step_ = false;
  return CFG_OK;
}
int Engine::set_nray(int s, int nray) {
  if (nray < 1 || nray > 1024 || (nray & (nray - 1))) return fail(CFG_ERR_INVAL, "nray must be a power of two in [1, 1024]");
  scenes_[s].nray = nray;
  return CFG_OK;
}

// encodeReadback + afterSubmit (js/fluid.js:315-342), synchronous
int Engine::readback(int s, int32_t* acc, float* rad, int32_t* faceW) {
  CFG_TRY(activate());
  const SceneDesc& d = scenes_[s].desc;
  cudaStream_t q = st();
  if (acc) CFG_CUDA(cudaMemcpyAsync(acc, d.acc, ACC_LEN * 4, cudaMemcpyDeviceToHost, q));
  if (rad) CFG_CUDA(cudaMemcpyAsync(rad, d.rad, RAD_LEN * 16, cudaMemcpyDeviceToHost, q));
  if (faceW) CFG_CUDA(cudaMemcpyAsync(faceW, d.faceW, MAX_PIECES * 16, cudaMemcpyDeviceToHost, q));
  CFG_CUDA(cudaMemsetAsync(d.acc, 0, ACC_LEN * 4, q));
  CFG_CUDA(cudaStreamSynchronize(q));
  return CFG_OK;
}

// encodeReadback (js/fluid.js:315-324) + afterSubmit (:327-342): the accumulators, the radiation
// output and the face weights are copied on the stream into the ring's next pinned slot, then
// acc is cleared; the slot's event marks the copies complete. When that slot still holds a
// readback nobody has collected (three in flight), nothing is copied and acc keeps
// accumulating (the reference's stageBusy skip): CFG_ERR_BUSY.
int Engine::readback_begin(int s, uint64_t tag, int* slot) {
  CFG_TRY(activate());
  Scene& sc = scenes_[s];
  Scene::Ring& R = sc.ring;
  if (!R.host) {
    CFG_CUDA(cudaHostAlloc(&R.host, kRingSlots * kRingBytes, cudaHostAllocMapped | cudaHostAllocPortable));
    CFG_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&R.dev), R.host, 0));
    for (auto& e : R.ev) CFG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  const int i = R.idx;
  if (R.busy[i]) return fail(CFG_ERR_BUSY, "readback ring slot still pending (three readbacks not collected)");
  const SceneDesc& d = sc.desc;
  cudaStream_t q = st();
  // acc, rad, faceW (contiguous on the device) written into the slot by one kernel, which then
  // clears the accumulators
  launch_readback(reinterpret_cast<uint32_t*>(d.acc), reinterpret_cast<uint32_t*>(R.dev + (size_t)i * kRingBytes),
                  (int)(kRingBytes / 4), ACC_LEN, q);
  CFG_CUDA(cudaGetLastError());
  CFG_CUDA(cudaEventRecord(R.ev[i], q));
  R.busy[i] = true;
  R.tag[i] = tag;
  R.seq[i] = R.next++;
  R.idx = (i + 1) % kRingSlots;
  if (slot) *slot = i;
  return CFG_OK;
}

int Engine::readback_collect(int s, bool wait, int32_t* acc, float* rad, int32_t* faceW, uint64_t* tag, int* ready) {
  if (!ready) return fail(CFG_ERR_INVAL, "null ready flag");
  *ready = 0;
  CFG_TRY(activate());
  Scene::Ring& R = scenes_[s].ring;
  int i = -1;
  for (int k = 0; k < kRingSlots; k++)
    if (R.busy[k] && (i < 0 || R.seq[k] < R.seq[i])) i = k;
  if (i < 0) return wait ? fail(CFG_ERR_NOENT, "no readback pending") : CFG_OK;
  if (wait) {
    CFG_CUDA(cudaEventSynchronize(R.ev[i]));
  } else {
    const cudaError_t e = cudaEventQuery(R.ev[i]);
    if (e == cudaErrorNotReady) return CFG_OK;
    CFG_CUDA(e);
  }
  const char* h = R.host + (size_t)i * kRingBytes;
  if (acc) std::memcpy(acc, h, ACC_LEN * 4);
  if (rad) std::memcpy(rad, h + kRbRadOff, RAD_LEN * 16);
  if (faceW) std::memcpy(faceW, h + kRbFaceWOff, MAX_PIECES * 16);
  if (tag) *tag = R.tag[i];
  R.busy[i] = false;
  *ready = 1;
  return CFG_OK;
}

// Renderer.encode (js/render.js:57-70) into a device image instead of the canvas:
// the wood buffer (Renderer.writeWood, :55) is uploaded, one thread per pixel runs
// the fragment stage, and the image is copied back.
int Engine::render_device(int s, const cfg_render_params& rp, const float* wood, int width, int height,
                          float* rgba_dev) {
  if (width < 1 || height < 1 || width > 16384 || height > 16384)
    return fail(CFG_ERR_INVAL, "image size must be in [1, 16384] x [1, 16384]");
  if (rp.nPieces < 0 || rp.nPieces > MAX_PIECES) return fail(CFG_ERR_INVAL, "nPieces must be in [0, 64]");
  if (!rgba_dev || ((uintptr_t)rgba_dev & 15)) return fail(CFG_ERR_INVAL, "rgba must be a 16-byte aligned device pointer");
  CFG_TRY(activate());
  cudaStream_t q = st();
  const size_t wood_bytes = sizeof(float) * MAX_PIECES * 12;
  if (!d_rwood_) CFG_CUDA(cudaMalloc(&d_rwood_, wood_bytes));
  if (wood) CFG_CUDA(cudaMemcpyAsync(d_rwood_, wood, wood_bytes, cudaMemcpyHostToDevice, q));
  else CFG_CUDA(cudaMemsetAsync(d_rwood_, 0, wood_bytes, q));
  launch_render(d_scenes_, s, rp, d_rwood_, width, height, rgba_dev, q);
  CFG_CUDA(cudaGetLastError());
  return CFG_OK;
}

int Engine::render(int s, const cfg_render_params& rp, const float* wood, int width, int height, float* rgba) {
  if (width < 1 || height < 1 || width > 16384 || height > 16384)
    return fail(CFG_ERR_INVAL, "image size must be in [1, 16384] x [1, 16384]");
  if (!rgba) return fail(CFG_ERR_INVAL, "rgba is null");
  CFG_TRY(activate());
  cudaStream_t q = st();
  const size_t bytes = sizeof(float) * 4 * (size_t)width * height;
  if (bytes > image_bytes_) {
    CFG_CUDA(cudaStreamSynchronize(q));
    if (d_image_) CFG_CUDA(cudaFree(d_image_));
    d_image_ = nullptr; image_bytes_ = 0;
    CFG_CUDA(cudaMalloc(&d_image_, bytes));
    image_bytes_ = bytes;
  }
  CFG_TRY(render_device(s, rp, wood, width, height, d_image_));
  CFG_CUDA(cudaMemcpyAsync(rgba, d_image_, bytes, cudaMemcpyDeviceToHost, q));
  CFG_CUDA(cudaStreamSynchronize(q));
  return CFG_OK;
}

// Renderer.writeParams as the app calls it (js/render.js:41-53, js/main.js:268-271)
int Engine::render_defaults(int s, cfg_render_params* rp) {
  if (!rp) return fail(CFG_ERR_INVAL, "rp is null");
  const Scene& sc = scenes_[s];
  const double ground = 0.03;   // GROUND, js/render.js:6
  rp->view = 0;
  rp->nPieces = std::min(std::max(sc.host.nPieces, 0), MAX_PIECES);
  rp->exposure = 1.0f;          // Math.pow(2, 0)
  rp->width = (float)(sc.nx * sc.dxd);
  rp->height = (float)(sc.ny * sc.dxd);
  rp->ground = (float)ground;
  rp->time = (float)sc.time;
  rp->tmax = 1800.0f;
  rp->chemi = (float)3e-7;
  rp->camX = 0.0f;
  rp->camY = (float)(-ground);
  rp->zoom = 1.0f;
  return CFG_OK;
}

int Engine::field_ptr(int s, const std::string& nm, char** base, size_t* elem, int* w, int* h, size_t* pitch) {
  const Scene& sc = scenes_[s];
  const SceneDesc& d = sc.desc;
  auto set = [&](void* b, size_t e, int ww, int hh, int pe) { *base = (char*)b; *elem = e; *w = ww; *h = hh; *pitch = (size_t)pe * e; return CFG_OK; };
  if (nm == "U") return set(d.U, 4, sc.nx + 1, sc.ny, d.pu);
  if (nm == "U2") return set(d.U2, 4, sc.nx + 1, sc.ny, d.pu);
  if (nm == "fx") return set(d.fx, 4, sc.nx + 1, sc.ny, d.pu);
  if (nm == "V") return set(d.V, 4, sc.nx, sc.ny + 1, d.pc);
  if (nm == "V2") return set(d.V2, 4, sc.nx, sc.ny + 1, d.pc);
  if (nm == "fy") return set(d.fy, 4, sc.nx, sc.ny + 1, d.pc);
  if (nm == "T") return set(d.T, 4, sc.nx, sc.ny, d.pc);
  if (nm == "T2") return set(d.T2, 4, sc.nx, sc.ny, d.pc);
  if (nm == "Y") return set(d.Y, 16, sc.nx, sc.ny, d.pc);
  if (nm == "Y2") return set(d.Y2, 16, sc.nx, sc.ny, d.pc);
  if (nm == "SQ") return set(d.SQ, 8, sc.nx, sc.ny, d.pc);
  if (nm == "cellG") return set(d.cellG, 8, sc.nx, sc.ny, d.pc);
  if (nm == "rad") return set(d.rad, 16, RAD_LEN, 1, RAD_LEN);   // encodeRadiation's output (vec4f per target)
  if (nm == "Uh" || nm == "Vh" || nm == "Th" || nm == "Yh")
    return fail(CFG_ERR_NOENT, "field " + nm + " is not kept: the first-order advection values live in shared memory only");
  std::string b = nm; int l = 0;
  const size_t dot = nm.find('.');
  if (dot != std::string::npos) { b = nm.substr(0, dot); l = std::atoi(nm.c_str() + dot + 1); }
  if (l < 0 || l >= sc.nlev) return fail(CFG_ERR_NOENT, "no multigrid level in " + nm);
  const LevelDesc& L = d.lev[l];
  if (b == "p") return set(L.p, 4, L.nx, L.ny, L.pc);
  if (b == "rhs") return set(L.rhs, 4, L.nx, L.ny, L.pc);
  if (b == "ax") return set(L.ax, 4, L.nx + 1, L.ny, L.pu);
  if (b == "ay") return set(L.ay, 4, L.nx, L.ny + 1, L.pc);
  return fail(CFG_ERR_NOENT, "unknown field " + nm);
}

int Engine::field_size(int s, const char* name, size_t* count) {
  if (!name || !count) return fail(CFG_ERR_INVAL, "null argument");
  char* b; size_t e, p; int w, h;
  CFG_TRY(field_ptr(s, name, &b, &e, &w, &h, &p));
  *count = (size_t)w * h * (e / 4);
  return CFG_OK;
}

// readBuffer(name) (js/fluid.js:345-355): dense copy of a field
int Engine::read_field(int s, const char* name, float* out, size_t count) {
  if (!name || !out) return fail(CFG_ERR_INVAL, "null argument");
  CFG_TRY(activate());
  char* b; size_t e, p; int w, h;
  CFG_TRY(field_ptr(s, name, &b, &e, &w, &h, &p));
  if (count != (size_t)w * h * (e / 4)) return fail(CFG_ERR_INVAL, std::string("field ") + name + ": expected " + std::to_string((size_t)w * h * (e / 4)) + " floats");
  CFG_CUDA(cudaMemcpy2DAsync(out, (size_t)w * e, b, p, (size_t)w * e, h, cudaMemcpyDeviceToHost, st()));
  CFG_CUDA(cudaStreamSynchronize(st()));
  return CFG_OK;
}
int Engine::write_field(int s, const char* name, const float* in, size_t count) {
  if (!name || !in) return fail(CFG_ERR_INVAL, "null argument");
  CFG_TRY(activate());
  char* b; size_t e, p; int w, h;
  CFG_TRY(field_ptr(s, name, &b, &e, &w, &h, &p));
  if (count != (size_t)w * h * (e / 4)) return fail(CFG_ERR_INVAL, std::string("field ") + name + ": expected " + std::to_string((size_t)w * h * (e / 4)) + " floats");
  CFG_CUDA(cudaMemcpy2DAsync(b, p, in, (size_t)w * e, (size_t)w * e, h, cudaMemcpyHostToDevice, st()));
  CFG_CUDA(cudaStreamSynchronize(st()));
  return CFG_OK;
}
int Engine::read_p64(int s, double* out, size_t count) {
  const Scene& sc = scenes_[s];
  if (!out || count != (size_t)sc.nx * sc.ny) return fail(CFG_ERR_INVAL, "p64: expected nx*ny doubles");
  CFG_TRY(activate());
  CFG_CUDA(cudaMemcpyAsync(out, sc.desc.p64, count * 8, cudaMemcpyDeviceToHost, st()));
  CFG_CUDA(cudaStreamSynchronize(st()));
  return CFG_OK;
}

int Engine::info(int s, cfg_info* o) {
  if (!o) return fail(CFG_ERR_INVAL, "null output");
  CFG_TRY(activate());
  const Scene& sc = scenes_[s];
  SolveState ss{};
  float dt = 0.f;
  CFG_CUDA(cudaMemcpyAsync(&ss, d_solve_ + s, sizeof ss, cudaMemcpyDeviceToHost, st()));
  CFG_CUDA(cudaMemcpyAsync(&dt, (char*)(d_scenes_ + s) + offsetof(SceneDesc, P) + offsetof(cfg_params, dt), 4,
                           cudaMemcpyDeviceToHost, st()));
  CFG_CUDA(cudaStreamSynchronize(st()));
  std::memset(o, 0, sizeof *o);
  o->nx = sc.nx; o->ny = sc.ny; o->levels = sc.nlev; o->diff_sub = sc.diff_sub;
  o->dx = sc.dxd; o->dt = sc.cfl > 0 ? (double)dt : sc.dtd; o->height = sc.dxd * sc.ny;
  o->time = sc.cfl > 0 ? ss.time : sc.time;   // a CFL scene's clock runs on the device
  o->frame = sc.frame; o->last_cycles = ss.cycles; o->last_rel = ss.rel;
  for (int l = 0; l < MAX_LEVELS; l++) { o->level_nx[l] = l < sc.nlev ? sc.lnx[l] : 0; o->level_ny[l] = l < sc.nlev ? sc.lny[l] : 0; }
  return CFG_OK;
}

int Engine::pressure_residual(int s, double* rel) {
  if (!rel) return fail(CFG_ERR_INVAL, "null output");
  CFG_TRY(activate());
  launch_residual_norms(d_scenes_, s, d_scratch_, st());
  double o[2];
  CFG_CUDA(cudaMemcpyAsync(o, d_scratch_, 16, cudaMemcpyDeviceToHost, st()));
  CFG_CUDA(cudaStreamSynchronize(st()));
  *rel = o[1] > 0 ? std::sqrt(o[0] / o[1]) : 0.0;
  return CFG_OK;
}
int Engine::budgets(int s, double* out) {
  if (!out) return fail(CFG_ERR_INVAL, "null output");
  CFG_TRY(activate());
  launch_budgets(d_scenes_, s, d_scratch_, st());
  CFG_CUDA(cudaMemcpyAsync(out, d_scratch_, 64, cudaMemcpyDeviceToHost, st()));
  CFG_CUDA(cudaStreamSynchronize(st()));
  return CFG_OK;
}
int Engine::set_active(int s, bool on) {
  CFG_TRY(activate());
  scenes_[s].enabled = on;
  scenes_[s].desc.enabled = on ? 1 : 0;
  const int v = on ? 1 : 0;
  CFG_CUDA(cudaMemcpyAsync((char*)(d_scenes_ + s) + offsetof(SceneDesc, enabled), &v, 4, cudaMemcpyHostToDevice, st()));
  CFG_CUDA(cudaStreamSynchronize(st()));
  return upload_ctl();
}

// ------------------------------------------------------------------ the step
int Engine::set_solver(int mode, int ncycles, double tol, int max_cycles) {
  if (mode < CFG_SOLVE_FIXED || mode > CFG_SOLVE_FP64) return fail(CFG_ERR_INVAL, "unknown solver mode");
  if (mode == CFG_SOLVE_FIXED && ncycles < 1) return fail(CFG_ERR_INVAL, "ncycles must be >= 1");
  if (mode != CFG_SOLVE_FIXED && (!(tol > 0) || max_cycles < 1)) return fail(CFG_ERR_INVAL, "tol must be > 0 and max_cycles >= 1");
  CFG_TRY(activate());
  mode_ = mode; ncycles_ = ncycles; tol_ = tol; max_cycles_ = max_cycles;
  graph_dirty_ = true;
  return upload_ctl();
}

void Engine::enqueue_pre_solve(cudaStream_t s, unsigned long long h, int use_cond) {
  const bool fp64 = any_fp64();
  launch_advect(d_scenes_, d_wl_[WL_ADV], nwl_[WL_ADV], tiles_[TK_ADVECT], s); launches_++;
  launch_diffuse_sources(d_scenes_, d_wl_[WL_DS], nwl_[WL_DS], max_sub(), true, true, tiles_[TK_DIFFSRC], s); launches_++;
  launch_forces(d_scenes_, d_wl_[WL_FR], nwl_[WL_FR], d_ctl_, true, true, fp64, tiles_[TK_FORCES], s); launches_++;
  // the levels below the forces kernel's in-tile restriction, one block per scene
  if (FR_KMAX + 1 < max_levels()) { launch_coef_restrict_tail(d_scenes_, nscenes(), FR_KMAX, s); launches_++; }
  enqueue_factor(s);
  if (fp64) { launch_defect64(d_scenes_, nscenes(), d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, 1, s); launches_++; }
  // the loop's cycle counter starts at zero in every step
  cudaMemsetAsync(&d_ctl_->iter, 0, sizeof(int), s);
  (void)h; (void)use_cond;
}

// The loop decision sets the graph's WHILE condition only while steps run as that
// graph; every launch outside it (host loop, stages, timing) runs with use_cond = 0.
int Engine::set_cond_mode(bool graph) {
  const int want = graph ? 1 : 0;
  if (ctl_use_cond_ == want) return CFG_OK;
  ctl_use_cond_ = want;
  return upload_ctl();
}

int Engine::set_krylov(int on) {
  if (on < 0 || on > 3) return fail(CFG_ERR_INVAL, "krylov must be 0 (off), 1 (on), 2 (on, update folded) or 3 (on, update kernel)");
  CFG_TRY(activate());
  krylov_ = on;
  graph_dirty_ = true;
  return upload_ctl();
}

int Engine::set_coarse_solve(int direct) {
  if (direct < 0 || direct > 2)
    return fail(CFG_ERR_INVAL, "coarse solve must be 0 (sweeps), 1 (direct) or 2 (direct, pipelined)");
  CFG_TRY(activate());
  coarse_direct_ = direct;
  graph_dirty_ = true;
  return upload_ctl();
}

int Engine::max_lc() const {
  int m = 0;
  for (auto& sc : scenes_) m = std::max(m, sc.lc);
  return m;
}

bool Engine::any_cfl() const {
  for (auto& sc : scenes_) if (sc.cfl > 0) return true;
  return false;
}

bool Engine::any_wtail() const {
  for (auto& sc : scenes_) if (sc.lw < sc.nlev) return true;
  return false;
}

bool Engine::any_block_level0() const {
  for (auto& sc : scenes_) if (sc.lc == 0) return true;
  return false;
}

bool Engine::pcg_fused() const {
  // krylov 1: one scene folds the update into the level-0 kernels (a shorter kernel chain); a
  // batch, bound by bandwidth, keeps the separate update kernel, which moves fewer bytes.
  // krylov 2 / 3 choose the fold / the kernel for any engine (the batch autotuner times both)
  if (!krylov() || krylov_ == 3 || (krylov_ == 1 && scenes_.size() != 1)) return false;
  for (auto& sc : scenes_)
    if (sc.lc < 1) return false;
  return true;
}

// after the pressure loop: the fused Krylov mode's last update
void Engine::enqueue_loop_end(cudaStream_t s) {
  if (!pcg_fused()) return;
  launch_pcg_finish(d_scenes_, d_wl_[WL_MG0], nwl_[WL_MG0], s);
  launches_++;
}

// The step's V(2,2) cycle with the fused kernels (k_mgf.cu); the level-0 up
// kernel (or the coarse block of scenes whose block starts at level 0) ends
// the cycle with the residual norm (FP32 modes) or p64 += p (FP64 mode).
void Engine::enqueue_vcycle(cudaStream_t s, int tail, int count_iter) {
  const int LD = max_lc();
  for (int l = 0; l < LD; l++) {
    if (nwl_[WL_MGD0 + l] == 0) continue;
    launch_mg_down(d_scenes_, nscenes(), d_wl_[WL_MGD0 + l], nwl_[WL_MGD0 + l], l, d_ctl_, count_iter, tail == 4 && l == 0, s);
    count_iter = 0;
    vcycle_launches_++;
  }
  if (coarse_cluster_ > 0)
    launch_mg_cluster(d_scenes_, nscenes(), d_ctl_, coarse_cluster_, count_iter, cluster_smem_, s);
  else
    launch_mg_coarse(d_scenes_, nscenes(), d_ctl_, tail, count_iter, coarse_smem_, any_wtail(), any_block_level0(), s);
  vcycle_launches_++;
  for (int l = LD - 1; l >= 0; l--) {
    if (nwl_[WL_MGD0 + l] == 0) continue;
    launch_mg_up(d_scenes_, nscenes(), d_wl_[WL_MGD0 + l], nwl_[WL_MGD0 + l], l, l == 0 ? tail : 0, d_ctl_, s);
    vcycle_launches_++;
  }
  if (tail == 4) {   // the fused Krylov mode's sums and decision
    launch_pcg_decide(d_scenes_, nscenes(), d_ctl_, s);
    vcycle_launches_++;
  }
}

// FluidSim.vcycle (js/fluid.js:294-312), nu = 2: one kernel per reference dispatch
void Engine::enqueue_vcycle_ref(cudaStream_t s) {
  const int L = max_levels();
  for (int l = 0; l + 1 < L; l++) {
    const int wv = WL_MGV0 + l;
    if (nwl_[wv] == 0) continue;
    for (int k = 0; k < 2; k++) {
      launch_relax(d_scenes_, d_wl_[wv], nwl_[wv], l, 0, s);
      launch_relax(d_scenes_, d_wl_[wv], nwl_[wv], l, 1, s);
      vcycle_launches_ += 2;
    }
    launch_restrict_res(d_scenes_, d_wl_[WL_MGC0 + l], nwl_[WL_MGC0 + l], l, s);
    vcycle_launches_++;
  }
  launch_coarsest(d_scenes_, nscenes(), s);
  vcycle_launches_++;
  for (int l = L - 2; l >= 0; l--) {
    const int wv = WL_MGV0 + l;
    if (nwl_[wv] == 0) continue;
    launch_prolong(d_scenes_, d_wl_[wv], nwl_[wv], l, s);
    vcycle_launches_++;
    for (int k = 0; k < 2; k++) {
      launch_relax(d_scenes_, d_wl_[wv], nwl_[wv], l, 1, s);
      launch_relax(d_scenes_, d_wl_[wv], nwl_[wv], l, 0, s);
      vcycle_launches_ += 2;
    }
  }
}

// FP64 mode after the fused cycle: the defect of the corrected p64 (plain correction),
// or the Krylov direction and update (the cycle ended with the direction update beta)
void Engine::enqueue_fp64_tail(cudaStream_t s) {
  if (!any_fp64()) return;
  if (krylov()) {
    if (pcg_fused()) return;   // the level-0 smoother kernels carry the update
    launch_pcg_step(d_scenes_, nscenes(), d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, s);
    vcycle_launches_++;
  } else {
    launch_defect64(d_scenes_, nscenes(), d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, 0, s);
    vcycle_launches_++;
  }
}

void Engine::enqueue_cycle_tail(cudaStream_t s, unsigned long long h, int use_cond) {
  // the fused cycle already ended with p64 += p / the direction update (FP64) or the residual norm
  enqueue_fp64_tail(s);
  launch_loop_guard(d_ctl_, h, use_cond, s);
  vcycle_launches_++;
}

// The coarsest inverse of the step's operator: before the loop on the step's stream
// (direct), or on a side branch that runs beside the whole pressure loop (pipelined)
void Engine::enqueue_factor(cudaStream_t s) {
  if (!direct_coarse()) return;
  if (!pipelined_coarse()) {
    launch_coarse_factor(d_scenes_, nscenes(), cf_smem_, cf_bw_, 0, s);
    launches_++;
    return;
  }
  cudaEventRecord(ev_fork_, s);
  cudaStreamWaitEvent(side_stream_, ev_fork_, 0);
  launch_coarse_factor(d_scenes_, nscenes(), cf_smem_, cf_bw_, 1, side_stream_);
  cudaEventRecord(ev_join_, side_stream_);
  launches_++;
}
void Engine::enqueue_factor_join(cudaStream_t s) {
  if (!pipelined_coarse()) return;
  cudaStreamWaitEvent(s, ev_join_, 0);
  launch_cinv_swap(d_scenes_, nscenes(), s);
  launches_++;
}

// The step's tail: the projection, which also swaps the pipelined coarsest inverse
// (after the factorisation's branch has joined) and sets the next CFL dt
// Returns the first failing CUDA call's status; on failure the pinned dt must not be
// trusted (the caller leaves dt_from_step_ unset).
cudaError_t Engine::enqueue_post_solve(cudaStream_t s) {
  const bool pipe = pipelined_coarse();
  if (pipe) {
    const cudaError_t e = cudaStreamWaitEvent(s, ev_join_, 0);
    if (e != cudaSuccess) return e;
  }
  const bool cfl = any_cfl();
  launch_project(d_scenes_, d_wl_[WL_PR], nwl_[WL_PR], any_fp64(), s, nscenes(), (pipe ? 1 : 0) | (cfl ? 2 : 0),
                 d_dxd_, d_alpha_, d_dtv_);
  launches_++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess || !cfl) return e;
  // the projection wrote the next dt to the host side (mapped pinned memory) for cfg_write_params
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return e;
  if (cap == cudaStreamCaptureStatusActive)
    return cudaEventRecordWithFlags(ev_dt_, s, cudaEventRecordExternal);   // a node of the step graph
  return cudaEventRecord(ev_dt_, s);
}

void Engine::enqueue_bnorm(cudaStream_t s) {
  launch_bnorm(d_scenes_, d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, any_fp64(), s);
}

// Pressure loop driven from the host (launches outside a graph): the device
// decides per cycle and mirrors the decision into SolveCtl::any_active.
// started: the step's pre-solve kernels already launched the first FP64 defect and reset the
// cycle counter (the stream-launched step); false for the staged calls that run the loop alone
int Engine::host_pressure_loop(bool started) {
  cudaStream_t s = st();
  int guard = 0;
  if (!started) {
    if (any_fp64()) launch_defect64(d_scenes_, nscenes(), d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, 1, s);
    CFG_CUDA(cudaMemsetAsync(&d_ctl_->iter, 0, sizeof(int), s));
  }
  CFG_CUDA(cudaMemcpyAsync(h_ctl_pinned_, d_ctl_, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s));
  CFG_CUDA(cudaStreamSynchronize(s));
  int any = any_fp64() ? h_ctl_pinned_->any_active : 1;
  while (any) {
    enqueue_vcycle(s, cycle_tail(), 0);
    enqueue_cycle_tail(s, 0ull, 0);
    CFG_CUDA(cudaMemcpyAsync(h_ctl_pinned_, d_ctl_, sizeof(SolveCtl), cudaMemcpyDeviceToHost, s));
    CFG_CUDA(cudaStreamSynchronize(s));
    any = h_ctl_pinned_->any_active;
    if (++guard > std::max(ncycles_, max_cycles_) + 2) return fail(CFG_ERR_TIMEDOUT, "pressure loop did not terminate");
  }
  enqueue_loop_end(s);
  return CFG_OK;
}

void Engine::destroy_graph() {
  if (exec_) { cudaGraphExecDestroy(exec_); exec_ = nullptr; }
  if (graph_) { cudaGraphDestroy(graph_); graph_ = nullptr; }
}

int Engine::ensure_graph() {
  if (!graph_dirty_ && exec_ && graph_sub_ >= max_sub()) return CFG_OK;
  destroy_graph();
  cudaStream_t s = stream_;
  CFG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  cudaStreamCaptureStatus status;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t ndeps = 0;
  auto abort_capture = [&](cudaError_t e, const char* what) {
    cudaGraph_t tmp = nullptr;
    cudaStreamEndCapture(s, &tmp);
    if (tmp) cudaGraphDestroy(tmp);
    return cuda_fail(e, what);
  };
  cudaError_t e = cudaStreamGetCaptureInfo(s, &status, nullptr, &g, nullptr, nullptr);
  if (e != cudaSuccess) return abort_capture(e, "cudaStreamGetCaptureInfo");
  cudaGraphConditionalHandle h = 0;
  e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) return abort_capture(e, "cudaGraphConditionalHandleCreate");
  launches_ = 0;
  enqueue_pre_solve(s, (unsigned long long)h, 1);
  e = cudaStreamGetCaptureInfo(s, &status, nullptr, &g, &deps, &ndeps);
  if (e != cudaSuccess) return abort_capture(e, "cudaStreamGetCaptureInfo");
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  e = cudaGraphAddNode(&cnode, g, deps, ndeps, &cp);
  if (e != cudaSuccess) return abort_capture(e, "cudaGraphAddNode(while)");
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  e = cudaStreamUpdateCaptureDependencies(s, &cnode, 1, cudaStreamSetCaptureDependencies);
  if (e != cudaSuccess) return abort_capture(e, "cudaStreamUpdateCaptureDependencies");
  e = cudaStreamBeginCaptureToGraph(body_stream_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return abort_capture(e, "cudaStreamBeginCaptureToGraph");
  vcycle_launches_ = 0;
  // the first kernel of the body counts the iteration and the cycle's decision sets the
  // condition (loop_count / solve_decide): no guard kernel in the body
  enqueue_vcycle(body_stream_, cycle_tail(), 1);
  enqueue_fp64_tail(body_stream_);
  e = cudaStreamEndCapture(body_stream_, &body);
  if (e != cudaSuccess) return abort_capture(e, "cudaStreamEndCapture(body)");
  enqueue_loop_end(s);
  e = enqueue_post_solve(s);
  if (e != cudaSuccess) return abort_capture(e, "enqueue_post_solve");
  e = cudaStreamEndCapture(s, &g);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
  graph_ = g;
  e = cudaGraphInstantiate(&exec_, graph_, 0);
  if (e != cudaSuccess) { destroy_graph(); return cuda_fail(e, "cudaGraphInstantiate"); }
  cond_handle_ = (unsigned long long)h;
  ctl_use_cond_ = -1;   // upload the new handle before the next launch
  graph_dirty_ = false;
  graph_sub_ = max_sub();
  return CFG_OK;
}

int Engine::step(int nsteps) {
  if (nsteps < 0) return fail(CFG_ERR_INVAL, "negative step count");
  CFG_TRY(activate());
  for (int k = 0; k < nsteps; k++) {
    if (use_graphs_) {
      if (ensure_graph() != CFG_OK) {
        // a driver that cannot capture programmatic launches into the loop body: capture without them
        if (!pdl_enabled()) return fail(CFG_ERR_INVAL, last_error());
        cudaGetLastError();
        set_pdl(false);
        graph_dirty_ = true;
        CFG_TRY(ensure_graph());
      }
      CFG_TRY(set_cond_mode(true));
      CFG_CUDA(cudaGraphLaunch(exec_, st()));
      dt_from_step_ = dt_from_step_ || any_cfl();
      mark_device_dt();
    } else {
      CFG_TRY(set_cond_mode(false));
      launches_ = 0; vcycle_launches_ = 0;
      enqueue_pre_solve(st(), 0ull, 0);
      CFG_CUDA(cudaGetLastError());
      CFG_TRY(host_pressure_loop(true));
      CFG_CUDA(enqueue_post_solve(st()));
      dt_from_step_ = dt_from_step_ || any_cfl();
      mark_device_dt();
    }
    for (auto& sc : scenes_) if (sc.enabled) sc.time += sc.dtd;
  }
  CFG_CUDA(cudaGetLastError());
  return CFG_OK;
}

int Engine::synchronize() {
  CFG_TRY(activate());
  CFG_CUDA(cudaStreamSynchronize(st()));
  // per-step launch count: kernels outside the loop + kernels per cycle x cycles (scene 0)
  SolveState ss{};
  CFG_CUDA(cudaMemcpy(&ss, d_solve_, sizeof ss, cudaMemcpyDeviceToHost));
  last_cycles_ = std::max(ss.cycles, 1);
  launches_per_step_ = launches_ + vcycle_launches_ * last_cycles_;
  int err = 0;
  CFG_CUDA(cudaMemcpy(&err, &d_ctl_->err, sizeof err, cudaMemcpyDeviceToHost));
  if (err) {
    CFG_CUDA(cudaMemset(&d_ctl_->err, 0, sizeof err));
    return fail(CFG_ERR_TIMEDOUT, "a bounded device wait ran out (TMA staging of the coarse multigrid levels)");
  }
  return CFG_OK;
}

int Engine::set_stream(cudaStream_t s) {
  CFG_TRY(activate());
  CFG_CUDA(cudaStreamSynchronize(st()));
  user_stream_ = s;
  return CFG_OK;
}

// encodeStepProfiled (js/fluid.js:256-292): the unfused stage kernels between events
int Engine::step_profiled(float* ms) {
  if (!ms) return fail(CFG_ERR_INVAL, "null output");
  CFG_TRY(activate());
  cudaStream_t s = st();
  cudaEvent_t ev[8];
  for (auto& e : ev) CFG_CUDA(cudaEventCreate(&e));
  CFG_CUDA(cudaEventRecord(ev[0], s));
  launch_advect(d_scenes_, d_wl_[WL_ADV], nwl_[WL_ADV], tiles_[TK_ADVECT], s);
  CFG_CUDA(cudaEventRecord(ev[1], s));
  launch_diffuse_sources(d_scenes_, d_wl_[WL_DS], nwl_[WL_DS], max_sub(), false, true, tiles_[TK_DIFFSRC], s);
  CFG_CUDA(cudaEventRecord(ev[2], s));
  launch_diffuse_sources(d_scenes_, d_wl_[WL_DS], nwl_[WL_DS], 1, true, false, tiles_[TK_DIFFSRC], s);
  CFG_CUDA(cudaEventRecord(ev[3], s));
  launch_forces(d_scenes_, d_wl_[WL_FR], nwl_[WL_FR], d_ctl_, true, false, any_fp64(), tiles_[TK_FORCES], s);
  CFG_CUDA(cudaEventRecord(ev[4], s));
  launch_forces(d_scenes_, d_wl_[WL_FR], nwl_[WL_FR], d_ctl_, false, true, any_fp64(), tiles_[TK_FORCES], s);
  for (int l = FR_KMAX; l + 1 < max_levels(); l++)
    launch_coef_restrict(d_scenes_, d_wl_[WL_MGC0 + l], nwl_[WL_MGC0 + l], l, s);
  CFG_CUDA(cudaEventRecord(ev[5], s));
  CFG_TRY(set_cond_mode(false));
  enqueue_factor(s);
  CFG_TRY(host_pressure_loop(false));
  CFG_CUDA(cudaEventRecord(ev[6], s));
  CFG_CUDA(enqueue_post_solve(s));
  dt_from_step_ = dt_from_step_ || any_cfl();
  mark_device_dt();
  CFG_CUDA(cudaEventRecord(ev[7], s));
  CFG_CUDA(cudaEventSynchronize(ev[7]));
  for (int k = 0; k < 7; k++) CFG_CUDA(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]));
  for (auto& e : ev) cudaEventDestroy(e);
  for (auto& sc : scenes_) if (sc.enabled) sc.time += sc.dtd;
  return CFG_OK;
}

int Engine::run_stage(const char* stage) {
  if (!stage) return fail(CFG_ERR_INVAL, "null stage");
  CFG_TRY(activate());
  dt_from_step_ = false;   // a stage may change the device's dt (update_dt) without the step's copy
  const std::string st_(stage);
  cudaStream_t s = st();
  const bool fp64 = any_fp64();
  if (st_ == "advect") launch_advect(d_scenes_, d_wl_[WL_ADV], nwl_[WL_ADV], tiles_[TK_ADVECT], s);
  else if (st_ == "diffuse") launch_diffuse_sources(d_scenes_, d_wl_[WL_DS], nwl_[WL_DS], max_sub(), false, true, tiles_[TK_DIFFSRC], s);
  else if (st_ == "sources") launch_diffuse_sources(d_scenes_, d_wl_[WL_DS], nwl_[WL_DS], 1, true, false, tiles_[TK_DIFFSRC], s);
  else if (st_ == "diffuse_sources") launch_diffuse_sources(d_scenes_, d_wl_[WL_DS], nwl_[WL_DS], max_sub(), true, true, tiles_[TK_DIFFSRC], s);
  else if (st_ == "forces") launch_forces(d_scenes_, d_wl_[WL_FR], nwl_[WL_FR], d_ctl_, true, false, fp64, tiles_[TK_FORCES], s);
  else if (st_ == "coef_rhs") {
    launch_forces(d_scenes_, d_wl_[WL_FR], nwl_[WL_FR], d_ctl_, false, true, fp64, tiles_[TK_FORCES], s);
    for (int l = FR_KMAX; l + 1 < max_levels(); l++)
      launch_coef_restrict(d_scenes_, d_wl_[WL_MGC0 + l], nwl_[WL_MGC0 + l], l, s);
  } else if (st_ == "pressure") {
    CFG_TRY(set_cond_mode(false));
    enqueue_factor(s);
    enqueue_bnorm(s);
    CFG_TRY(host_pressure_loop(false));
    enqueue_factor_join(s);
  } else if (st_ == "project") launch_project(d_scenes_, d_wl_[WL_PR], nwl_[WL_PR], fp64, s);
  else if (st_ == "update_dt") launch_cfl_update(d_scenes_, nscenes(), d_dxd_, d_alpha_, s);
  else return fail(CFG_ERR_NOENT, "unknown stage " + st_);
  CFG_CUDA(cudaGetLastError());
  CFG_CUDA(cudaStreamSynchronize(s));
  return CFG_OK;
}

// Mean device time of one kernel of the step on scene 0, with the algorithmic
// bytes per launch of the reference schedule (one read + one write per array
// element at storage width; the per-cell figures of each WGSL dispatch).
int Engine::time_kernel(const char* name, int iters, double* ms, double* bytes, double* per_step) {
  if (!name || !ms || !bytes || !per_step || iters < 1) return fail(CFG_ERR_INVAL, "bad argument");
  CFG_TRY(activate());
  const Scene& sc = scenes_[0];
  const double cells = (double)sc.nx * sc.ny;
  SolveState ss{};
  CFG_CUDA(cudaMemcpy(&ss, d_solve_, sizeof ss, cudaMemcpyDeviceToHost));
  const double cyc = std::max(std::max(ss.cycles, 1), last_cycles_);
  const bool fp64 = any_fp64();
  cudaStream_t s = st();
  const std::string n(name);
  std::function<void(int)> go;
  double b = 0, cnt = 1;
  if (n == "advect") { go = [&](int) { launch_advect(d_scenes_, d_wl_[WL_ADV], nwl_[WL_ADV], tiles_[TK_ADVECT], s); }; b = 156 * cells; }
  else if (n == "diffuse_sources") {
    go = [&](int) { launch_diffuse_sources(d_scenes_, d_wl_[WL_DS], nwl_[WL_DS], max_sub(), true, true, tiles_[TK_DIFFSRC], s); };
    b = (48.0 * sc.diff_sub + 68) * cells;
  } else if (n == "forces") {
    go = [&](int) { launch_forces(d_scenes_, d_wl_[WL_FR], nwl_[WL_FR], d_ctl_, true, true, fp64, tiles_[TK_FORCES], s); };
    b = (28 + 20 + 28 + 13.3) * cells;
  } else if (n == "relax0") {
    go = [&](int k) { launch_relax(d_scenes_, d_wl_[WL_MGV0], nwl_[WL_MGV0], 0, k & 1, s); };
    b = 16 * cells; cnt = 8 * cyc;
  } else if (n == "restrict0") {
    go = [&](int) { launch_restrict_res(d_scenes_, d_wl_[WL_MGC0], nwl_[WL_MGC0], 0, s); };
    b = 18 * cells; cnt = cyc;
  } else if (n == "prolong0") {
    go = [&](int) { launch_prolong(d_scenes_, d_wl_[WL_MGV0], nwl_[WL_MGV0], 0, s); };
    b = 17 * cells; cnt = cyc;
  } else if (n == "coarsest") {
    go = [&](int) { launch_coarsest(d_scenes_, nscenes(), s); };
    b = 0; cnt = cyc;
  } else if (n == "mg_down0") {
    go = [&](int) { launch_mg_down(d_scenes_, nscenes(), d_wl_[WL_MGD0], nwl_[WL_MGD0], 0, d_ctl_, 0, 0, s); };
    b = (4 * 16 + 18) * cells; cnt = cyc;   // 4 colour passes + residual restriction
  } else if (n == "mg_up0") {
    go = [&](int) { launch_mg_up(d_scenes_, nscenes(), d_wl_[WL_MGD0], nwl_[WL_MGD0], 0, 0, d_ctl_, s); };
    b = (17 + 4 * 16) * cells; cnt = cyc;   // prolongation + 4 colour passes
  } else if (n == "mg_down0_krylov" || n == "mg_up0_krylov") {
    // the level-0 kernels as the step runs them in the fused Krylov mode (the update folded in):
    // the V-cycle's bytes plus half of the FP64 iteration's 40 B per cell each
    if (!pcg_fused()) return fail(CFG_ERR_NOENT, n + ": the Krylov update is not folded in this engine");
    if (n == "mg_down0_krylov") {
      go = [&](int) { launch_mg_down(d_scenes_, nscenes(), d_wl_[WL_MGD0], nwl_[WL_MGD0], 0, d_ctl_, 0, 1, s); };
      b = (4 * 16 + 18 + 20) * cells;
    } else {
      go = [&](int) { launch_mg_up(d_scenes_, nscenes(), d_wl_[WL_MGD0], nwl_[WL_MGD0], 0, 4, d_ctl_, s); };
      b = (17 + 4 * 16 + 20) * cells;
    }
    cnt = cyc;
  } else if (n == "pcg_decide") {
    // the fused Krylov mode's per-scene sums and decision: nine partials per level-0 tile read
    if (!pcg_fused()) return fail(CFG_ERR_NOENT, n + ": the Krylov update is not folded in this engine");
    go = [&](int) { launch_pcg_decide(d_scenes_, nscenes(), d_ctl_, s); };
    b = 0;
    for (int k = 0; k < nscenes(); k++)
      b += 72.0 * ((scenes_[k].nx + MGF_TX - 1) / MGF_TX) * ((scenes_[k].ny + MGF_TY - 1) / MGF_TY);
    cnt = cyc;
  } else if (n == "mg_coarse") {
    go = [&](int) {
      if (coarse_cluster_ > 0) launch_mg_cluster(d_scenes_, nscenes(), d_ctl_, coarse_cluster_, 0, cluster_smem_, s);
      else launch_mg_coarse(d_scenes_, nscenes(), d_ctl_, 0, 0, coarse_smem_, any_wtail(), any_block_level0(), s);
    };
    // the reference schedule's V-cycle bytes of the levels the block covers (163 B per level cell)
    b = 0;
    for (int l = sc.lc; l < sc.nlev; l++) b += 163.0 * sc.lnx[l] * sc.lny[l];
    cnt = cyc;
  } else if (n == "vcycle") {
    // one fused V(2,2) cycle without its tail (the smoother schedule's cost)
    go = [&](int) { enqueue_vcycle(s, 0, 0); };
    b = 0;
    for (int l = 0; l + 1 < sc.nlev; l++) b += 163.0 * sc.lnx[l] * sc.lny[l];
    cnt = cyc;
  } else if (n == "defect64") {
    go = [&](int) { launch_defect64(d_scenes_, nscenes(), d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, 0, s); };
    b = 32 * cells; cnt = fp64 ? (krylov() ? 1 : cyc) : 0;   // the Krylov loop runs it once, to start
  } else if (n == "resnorm") {
    go = [&](int) { launch_resnorm(d_scenes_, nscenes(), d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, s); };
    b = (fp64 ? 32 : 16) * cells; cnt = cyc;
  } else if (n == "project") {
    go = [&](int) { launch_project(d_scenes_, d_wl_[WL_PR], nwl_[WL_PR], fp64, s); };
    b = 32 * cells;
  } else if (n == "coarse_factor") {
    go = [&](int) { launch_coarse_factor(d_scenes_, nscenes(), cf_smem_, cf_bw_, pipelined_coarse() ? 1 : 0, s); };
    b = 0; cnt = direct_coarse() ? 1 : 0;
  } else if (n == "pcg_step") {
    go = [&](int) { launch_pcg_step(d_scenes_, nscenes(), d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, s); };
    b = 84 * cells; cnt = krylov() && !pcg_fused() ? cyc : 0;   // z, Lz, d, q, p64, r read; d, q, p64, r, rhs0, p0 written
  } else if (n.size() == 8 && (n.compare(0, 7, "mg_down") == 0) && n[7] >= '1' && n[7] <= '6') {
    const int l = n[7] - '0';
    if (l >= sc.lc) return fail(CFG_ERR_NOENT, "level " + n.substr(7) + " is in the coarse block");
    go = [&, l](int) { launch_mg_down(d_scenes_, nscenes(), d_wl_[WL_MGD0 + l], nwl_[WL_MGD0 + l], l, d_ctl_, 0, 0, s); };
    b = (4 * 16 + 18) * (double)sc.lnx[l] * sc.lny[l]; cnt = cyc;
  } else if (n.size() == 6 && (n.compare(0, 5, "mg_up") == 0) && n[5] >= '1' && n[5] <= '6') {
    const int l = n[5] - '0';
    if (l >= sc.lc) return fail(CFG_ERR_NOENT, "level " + n.substr(5) + " is in the coarse block");
    go = [&, l](int) { launch_mg_up(d_scenes_, nscenes(), d_wl_[WL_MGD0 + l], nwl_[WL_MGD0 + l], l, 0, d_ctl_, s); };
    b = (17 + 4 * 16) * (double)sc.lnx[l] * sc.lny[l]; cnt = cyc;
  } else return fail(CFG_ERR_NOENT, "unknown kernel " + n);
  CFG_TRY(set_cond_mode(false));
  launch_bnorm(d_scenes_, d_wl_[WL_MG0], nwl_[WL_MG0], d_ctl_, false, s);   // arm the multigrid kernels
  cudaEvent_t e0, e1;
  CFG_CUDA(cudaEventCreate(&e0));
  CFG_CUDA(cudaEventCreate(&e1));
  go(0);   // warm-up
  CFG_CUDA(cudaEventRecord(e0, s));
  for (int k = 0; k < iters; k++) go(k);
  CFG_CUDA(cudaEventRecord(e1, s));
  CFG_CUDA(cudaEventSynchronize(e1));
  float t = 0.f;
  CFG_CUDA(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0); cudaEventDestroy(e1);
  CFG_CUDA(cudaGetLastError());
  *ms = (double)t / iters; *bytes = b; *per_step = cnt;
  return CFG_OK;
}

int Engine::vcycle_once(int nu) {
  if (nu != 2) return fail(CFG_ERR_INVAL, "only V(2,2) cycles are provided (js/fluid.js:294 default nu = 2)");
  CFG_TRY(activate());
  cudaStream_t s = st();
  CFG_TRY(set_cond_mode(false));
  enqueue_bnorm(s);   // arms every scene (active = 1)
  enqueue_vcycle_ref(s);
  CFG_CUDA(cudaGetLastError());
  CFG_CUDA(cudaStreamSynchronize(s));
  return CFG_OK;
}

}  // namespace cfg
