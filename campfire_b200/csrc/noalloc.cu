// Level-0 pressure residual norms with no device allocation.
//
// Some callers cannot allocate device memory when they need this check: a
// frame or serving loop that has already committed every GPU's memory to its
// scenes and jobs, or one that must not stall, since cudaMalloc and cudaFree
// can synchronise the whole device and hold up work on every other stream.
// cfg_pressure_residual_noalloc gives them the residual norms of a pressure
// field they own, using only the fixed scratch array below for its per-block
// partial sums.
//
// The scratch lives in a file-scope __device__ array of 8194 doubles (65,552
// bytes): every GPU that loads this library holds it until the process exits.
// It bounds the grid at 4096 blocks of 256 cells (1,048,576 cells). Host code
// cannot pass the array's name to a kernel (in host code it is a stand-in, not
// a device address), so on its first call on each device the entry point asks
// for the device address with cudaGetSymbolAddress, with that device current,
// and keeps it. Make that first call before any stream capture.
// All calls share the array and it keeps the last call's contents. Each call
// writes every slot it reads, so nothing has to start at zero, but calls that
// overlap on the GPU (other streams, other threads) race on it.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "../../include/campfire_gas.h"
#include "engine.h"
#include "reduce.cuh"

namespace cfg {

constexpr int NA_THREADS = 256;                 // cells per block
constexpr int NA_MAX_BLOCKS = 4096;             // -> at most 1,048,576 cells (1024 x 1024)
constexpr int NA_SLOTS = 2 * NA_MAX_BLOCKS + 2; // two partials per block, then the two totals
static __device__ __align__(256) double g_noalloc_scratch[NA_SLOTS];

namespace {

// pressure.wgsl:77-101 on the dense reference layouts (js/fluid.js:75-78):
// p, rhs [ny][nx], ax [ny][nx+1], ay [ny+1][nx]
__global__ void __launch_bounds__(NA_THREADS) k_na_partials(const float* __restrict__ p, const float* __restrict__ rhs,
                                                           const float* __restrict__ ax, const float* __restrict__ ay,
                                                           int nx, int ny, float h2, double* scratch) {
  __shared__ double red[32];
  const int cell = blockIdx.x * NA_THREADS + threadIdx.x;
  double vr = 0.0, vb = 0.0;
  if (cell < nx * ny) {
    const int i = cell % nx, j = cell / nx;
    const float w = ax[j * (nx + 1) + i], e = ax[j * (nx + 1) + i + 1];
    const float s = ay[j * nx + i], n = ay[(j + 1) * nx + i];
    float off = 0.f, diag = 0.f;
    if (i > 0) { off += w * p[j * nx + i - 1]; diag += w; } else { diag += 2.f * w; }
    if (i < nx - 1) { off += e * p[j * nx + i + 1]; diag += e; } else { diag += 2.f * e; }
    if (j > 0) { off += s * p[(j - 1) * nx + i]; diag += s; }
    if (j < ny - 1) { off += n * p[(j + 1) * nx + i]; diag += n; } else { diag += 2.f * n; }
    const float r = diag <= 0.f ? 0.f : rhs[cell] - (off - diag * p[cell]) / h2;
    vr = (double)r * (double)r;
    vb = (double)rhs[cell] * (double)rhs[cell];
  }
  const double tr = block_sum(vr, red);
  const double tb = block_sum(vb, red);
  if (threadIdx.x == 0) { scratch[2 * blockIdx.x] = tr; scratch[2 * blockIdx.x + 1] = tb; }
}

// sums the per-block partials in block order (deterministic) into the two total slots
__global__ void __launch_bounds__(1024) k_na_combine(double* scratch, int nblocks) {
  __shared__ double red[32];
  double vr = 0.0, vb = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) { vr += scratch[2 * b]; vb += scratch[2 * b + 1]; }
  const double tr = block_sum(vr, red);
  const double tb = block_sum(vb, red);
  if (threadIdx.x == 0) { scratch[2 * NA_MAX_BLOCKS] = tr; scratch[2 * NA_MAX_BLOCKS + 1] = tb; }
}

constexpr int NA_MAX_DEVICES = 64;
std::mutex g_na_mutex;
double* g_na_ptr[NA_MAX_DEVICES] = {};

// device address of the scratch on the current device, looked up once per device
int scratch_ptr(double** out) {
  int dev = -1;
  CFG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= NA_MAX_DEVICES) return fail(CFG_ERR_INVAL, "device index beyond the no-allocation table");
  std::lock_guard<std::mutex> lock(g_na_mutex);
  if (!g_na_ptr[dev]) {
    double* ptr = nullptr;
    CFG_CUDA(cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch));
    g_na_ptr[dev] = ptr;
  }
  *out = g_na_ptr[dev];
  return CFG_OK;
}

}  // namespace
}  // namespace cfg

extern "C" int cfg_pressure_residual_noalloc(const float* p, const float* rhs, const float* ax, const float* ay, int nx,
                                             int ny, double h2, void* stream, double* rel) {
  using namespace cfg;
  if (!p || !rhs || !ax || !ay || !rel) return fail(CFG_ERR_INVAL, "null argument");
  if (nx < 1 || ny < 1 || !(h2 > 0)) return fail(CFG_ERR_INVAL, "nx, ny and h2 must be positive");
  const long long cells = (long long)nx * ny;
  if (cells > (long long)NA_THREADS * NA_MAX_BLOCKS)
    return fail(CFG_ERR_RANGE, "grid larger than the no-allocation scratch allows (at most 1048576 cells)");
  double* scratch = nullptr;
  CFG_TRY(scratch_ptr(&scratch));
  cudaStream_t st = (cudaStream_t)stream;
  const int nblocks = (int)((cells + NA_THREADS - 1) / NA_THREADS);
  k_na_partials<<<nblocks, NA_THREADS, 0, st>>>(p, rhs, ax, ay, nx, ny, (float)h2, scratch);
  k_na_combine<<<1, 1024, 0, st>>>(scratch, nblocks);
  CFG_CUDA(cudaGetLastError());
  double tot[2] = {0.0, 0.0};
  CFG_CUDA(cudaMemcpyAsync(tot, scratch + 2 * NA_MAX_BLOCKS, sizeof tot, cudaMemcpyDeviceToHost, st));
  CFG_CUDA(cudaStreamSynchronize(st));
  *rel = tot[1] > 0.0 ? std::sqrt(tot[0] / tot[1]) : 0.0;
  return CFG_OK;
}
