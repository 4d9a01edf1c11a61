// Serving loop for gas-step jobs (no counterpart in the reference, which steps one
// scene per browser tab): jobs of several grid sizes arrive over time, are
// admitted into resident batch slots while the HBM budget allows, advance
// together one batched step at a time (continuous batching: a job joins at the
// next step after it is admitted and leaves after its last step), and report
// arrival, admission and completion times.
//
// Slots: one cfg::Engine holds `slots[c]` scenes of each size class c; every
// slot starts disabled. A job is admitted into a free slot of its class when the
// bytes of the slots in use plus its own stay within the budget. Its state is
// generated on the host (cfg_scene_generate with the job's seed), uploaded into
// the slot (FluidSim's set-up order) and the slot enabled. Each loop iteration
// launches one step of the whole batch; disabled slots leave every kernel at
// once. A job's fields are read back after its last step, hashed, and its slot
// disabled and freed. Every scene's solve decides for itself, so a job's result
// does not depend on the other jobs in the batch.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <deque>
#include <string>
#include <thread>
#include <vector>

#include "../../include/campfire_gas.h"
#include "engine.h"

static_assert(sizeof(cfg_job) == 32, "cfg_job layout");
static_assert(sizeof(cfg_job_result) == 64, "cfg_job_result layout");

struct cfg_server {
  cfg::Engine eng;
  std::vector<int> cls_nx, cls_ny;
  std::vector<int> slot_class;
  std::vector<size_t> slot_bytes;
  double budget = 0, width = 0.8;
};

namespace {

using Clock = std::chrono::steady_clock;

// FNV-1a (64-bit) over the bytes of the dense fields T, Y, U, V: equal hashes mean
// (with overwhelming likelihood) bit-identical states
struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
  }
};

int field_hash(cfg::Engine& eng, int s, uint64_t* hash, double* tsum) {
  Fnv f;
  double sum = 0;
  for (const char* name : {"T", "Y", "U", "V"}) {
    size_t n = 0;
    CFG_TRY(eng.field_size(s, name, &n));
    std::vector<float> buf(n);
    CFG_TRY(eng.read_field(s, name, buf.data(), n));
    f.add(buf.data(), n * sizeof(float));
    if (name[0] == 'T') for (float v : buf) sum += v;
  }
  *hash = f.h;
  *tsum = sum;
  return CFG_OK;
}

}  // namespace

extern "C" {

int cfg_server_create(int device, int nclasses, const int* nx, const int* ny, const int* slots, double budget_bytes,
                      double width, cfg_server** out) {
  if (!out) return cfg::fail(CFG_ERR_INVAL, "null output");
  *out = nullptr;
  if (nclasses < 1 || !nx || !ny || !slots || !(budget_bytes > 0) || !(width > 0))
    return cfg::fail(CFG_ERR_INVAL, "bad server configuration");
  std::vector<int> snx, sny, scls;
  for (int c = 0; c < nclasses; c++) {
    if (slots[c] < 0) return cfg::fail(CFG_ERR_INVAL, "negative slot count");
    for (int k = 0; k < slots[c]; k++) { snx.push_back(nx[c]); sny.push_back(ny[c]); scls.push_back(c); }
  }
  if (snx.empty()) return cfg::fail(CFG_ERR_INVAL, "the server has no slots");
  try {
    auto* s = new cfg_server;
    s->cls_nx.assign(nx, nx + nclasses);
    s->cls_ny.assign(ny, ny + nclasses);
    s->slot_class = scls;
    s->budget = budget_bytes;
    s->width = width;
    const int n = (int)snx.size();
    std::vector<double> w(n, width), dt(n, 0.002);
    int rc = s->eng.init(device, n, snx.data(), sny.data(), w.data(), dt.data());
    for (int k = 0; rc == CFG_OK && k < n; k++) rc = s->eng.set_active(k, false);
    if (rc != CFG_OK) { delete s; return rc; }
    for (int k = 0; k < n; k++) s->slot_bytes.push_back(s->eng.arena_bytes(k));
    *out = s;
    return CFG_OK;
  } catch (const std::bad_alloc&) {
    return cfg::fail(CFG_ERR_NOMEM, "host allocation failed");
  }
}

int cfg_server_destroy(cfg_server* s) {
  delete s;
  return CFG_OK;
}

int cfg_server_set_solver(cfg_server* s, int mode, int ncycles, double tol, int max_cycles, int coarse_direct,
                          int coarse_cells, int krylov) {
  if (!s) return cfg::fail(CFG_ERR_INVAL, "null cfg_server handle");
  CFG_TRY(s->eng.set_solver(mode, ncycles, tol, max_cycles));
  CFG_TRY(s->eng.set_coarse_solve(coarse_direct ? 1 : 0));
  CFG_TRY(s->eng.set_krylov(krylov ? 1 : 0));
  if (coarse_cells > 0) CFG_TRY(s->eng.set_coarse_cells(coarse_cells));
  return CFG_OK;
}

int cfg_server_slot_bytes(cfg_server* s, int size_class, size_t* bytes) {
  if (!s || !bytes) return cfg::fail(CFG_ERR_INVAL, "null argument");
  for (size_t k = 0; k < s->slot_class.size(); k++)
    if (s->slot_class[k] == size_class) { *bytes = s->slot_bytes[k]; return CFG_OK; }
  return cfg::fail(CFG_ERR_NOENT, "no slot of this size class");
}

int cfg_server_run(cfg_server* s, const cfg_job* jobs, int njobs, cfg_job_result* res, double* wall_s,
                   double* cell_updates) {
  if (!s || (!jobs && njobs > 0) || (!res && njobs > 0) || njobs < 0 || !wall_s || !cell_updates)
    return cfg::fail(CFG_ERR_INVAL, "bad argument");
  const int ncls = (int)s->cls_nx.size(), nslot = (int)s->slot_class.size();
  for (int j = 0; j < njobs; j++) {
    if (jobs[j].size_class < 0 || jobs[j].size_class >= ncls) return cfg::fail(CFG_ERR_INVAL, "job size class out of range");
    if (jobs[j].nsteps < 1) return cfg::fail(CFG_ERR_INVAL, "job step count must be >= 1");
    if (jobs[j].kind < 0 || jobs[j].kind > 2) return cfg::fail(CFG_ERR_INVAL, "job scene kind must be 0, 1 or 2");
    bool has_slot = false;
    for (int k = 0; k < nslot; k++)
      if (s->slot_class[k] == jobs[j].size_class && s->slot_bytes[k] <= s->budget) has_slot = true;
    if (!has_slot) return cfg::fail(CFG_ERR_RANGE, "a job's size class has no slot within the budget");
    std::memset(&res[j], 0, sizeof(cfg_job_result));
    res[j].slot = -1;
  }
  cfg::Engine& eng = s->eng;
  std::vector<int> order(njobs);
  for (int j = 0; j < njobs; j++) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a].arrival_s < jobs[b].arrival_s; });
  std::vector<std::deque<int>> waiting(ncls);
  std::vector<int> slot_job(nslot, -1), left(nslot, 0);
  size_t used = 0;
  double cu = 0;
  int next = 0, done = 0, active = 0;
  cudaEvent_t ev[4];
  for (auto& e : ev) CFG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  struct EvGuard { cudaEvent_t* e; ~EvGuard() { for (int k = 0; k < 4; k++) cudaEventDestroy(e[k]); } } guard{ev};
  long long nstep = 0;
  const auto t0 = Clock::now();
  auto now = [&] { return std::chrono::duration<double>(Clock::now() - t0).count(); };

  while (done < njobs) {
    const double t = now();
    while (next < njobs && jobs[order[next]].arrival_s <= t) {
      waiting[jobs[order[next]].size_class].push_back(order[next]);
      next++;
    }
    // admission: per class in arrival order, while a slot is free and the budget allows
    for (int c = 0; c < ncls; c++)
      while (!waiting[c].empty()) {
        int slot = -1;
        for (int k = 0; k < nslot; k++)
          if (s->slot_class[k] == c && slot_job[k] < 0 && used + s->slot_bytes[k] <= s->budget) { slot = k; break; }
        if (slot < 0) break;
        const int j = waiting[c].front();
        waiting[c].pop_front();
        if (nstep > 0) CFG_TRY(eng.synchronize());
        // enabled first: the geometry pass of the set-up skips disabled scenes
        CFG_TRY(eng.set_active(slot, true));
        CFG_TRY(cfg::load_generated_scene(eng, slot, jobs[j].kind, s->width, jobs[j].seed));
        slot_job[slot] = j;
        left[slot] = jobs[j].nsteps;
        used += s->slot_bytes[slot];
        active++;
        res[j].slot = slot;
        res[j].arrival_s = jobs[j].arrival_s;
        res[j].admit_s = now();
      }
    if (active == 0) {
      if (next >= njobs) return cfg::fail(CFG_ERR_RANGE, "waiting jobs can never be admitted");
      const double dtw = jobs[order[next]].arrival_s - now();
      if (dtw > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(dtw, 0.05)));
      continue;
    }
    // one batched step; the host runs at most two steps ahead of the device
    if (nstep >= 2) CFG_CUDA(cudaEventSynchronize(ev[(nstep - 2) % 4]));
    CFG_TRY(eng.step(1));
    CFG_CUDA(cudaEventRecord(ev[nstep % 4], eng.stream()));
    nstep++;
    for (int k = 0; k < nslot; k++) {
      if (slot_job[k] < 0) continue;
      cu += (double)s->cls_nx[s->slot_class[k]] * s->cls_ny[s->slot_class[k]];
      if (--left[k] > 0) continue;
      const int j = slot_job[k];
      CFG_TRY(eng.synchronize());
      cfg_info inf;
      CFG_TRY(eng.info(k, &inf));
      CFG_TRY(field_hash(eng, k, &res[j].hash, &res[j].t_sum));
      res[j].done_s = now();
      res[j].steps = jobs[j].nsteps;
      res[j].last_cycles = inf.last_cycles;
      res[j].last_rel = inf.last_rel;
      CFG_TRY(eng.set_active(k, false));
      slot_job[k] = -1;
      used -= s->slot_bytes[k];
      active--;
      done++;
    }
  }
  CFG_TRY(eng.synchronize());
  *wall_s = now();
  *cell_updates = cu;
  return CFG_OK;
}

}  // extern "C"
