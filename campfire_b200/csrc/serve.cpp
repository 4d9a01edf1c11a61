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
//
// Two fronts share the loop: cfg_server_run takes a list of jobs with arrival
// times and returns when all are done; cfg_server_submit hands jobs one at a
// time to a service thread (started on the first submission) whose results are
// collected with cfg_server_poll / cfg_server_wait.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/campfire_gas.h"
#include "engine.h"

static_assert(sizeof(cfg_job) == 32, "cfg_job layout");
static_assert(sizeof(cfg_job_result) == 64, "cfg_job_result layout");

using Clock = std::chrono::steady_clock;

struct cfg_server {
  cfg::Engine eng;
  std::vector<int> cls_nx, cls_ny;
  std::vector<int> slot_class;
  std::vector<size_t> slot_bytes;
  double budget = 0, width = 0.8;
  // the service thread (cfg_server_submit)
  struct Submitted { uint64_t ticket; cfg_job job; double arrival; };
  struct Kept { std::vector<float> T, Y, U, V; };
  std::mutex mu;
  std::condition_variable work_cv, done_cv;
  std::deque<Submitted> queue;                          // submitted, not yet taken by the loop
  std::unordered_map<uint64_t, cfg_job_result> finished;
  std::unordered_map<uint64_t, Kept> kept;              // CFG_JOB_KEEP_FIELDS
  std::unordered_map<uint64_t, int> in_flight;          // tickets taken by the loop
  uint64_t next_ticket = 1;
  std::thread worker;
  bool stopping = false, running = false, sync_busy = false;
  int worker_rc = CFG_OK;
  std::string worker_msg;
  Clock::time_point t0;
  ~cfg_server();
};

namespace {

// FNV-1a (64-bit) over the bytes of the dense fields T, Y, U, V: equal hashes mean
// (with overwhelming likelihood) bit-identical states
struct Fnv {
  uint64_t h = 1469598103934665603ull;
  void add(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= 1099511628211ull; }
  }
};

int read_dense(cfg::Engine& eng, int s, const char* name, std::vector<float>& buf) {
  size_t n = 0;
  CFG_TRY(eng.field_size(s, name, &n));
  buf.resize(n);
  return eng.read_field(s, name, buf.data(), n);
}

int field_hash(cfg::Engine& eng, int s, uint64_t* hash, double* tsum, cfg_server::Kept* keep) {
  Fnv f;
  double sum = 0;
  std::vector<float> local[4];
  const char* names[4] = {"T", "Y", "U", "V"};
  for (int k = 0; k < 4; k++) {
    std::vector<float>& buf = keep ? (k == 0 ? keep->T : k == 1 ? keep->Y : k == 2 ? keep->U : keep->V) : local[k];
    CFG_TRY(read_dense(eng, s, names[k], buf));
    f.add(buf.data(), buf.size() * sizeof(float));
    if (k == 0) for (float v : buf) sum += v;
  }
  *hash = f.h;
  *tsum = sum;
  return CFG_OK;
}

int check_job(const cfg_server* s, const cfg_job& j) {
  const int ncls = (int)s->cls_nx.size(), nslot = (int)s->slot_class.size();
  if (j.size_class < 0 || j.size_class >= ncls) return cfg::fail(CFG_ERR_INVAL, "job size class out of range");
  if (j.nsteps < 1) return cfg::fail(CFG_ERR_INVAL, "job step count must be >= 1");
  if (j.kind < 0 || j.kind > 2) return cfg::fail(CFG_ERR_INVAL, "job scene kind must be 0, 1 or 2");
  for (int k = 0; k < nslot; k++)
    if (s->slot_class[k] == j.size_class && s->slot_bytes[k] <= s->budget) return CFG_OK;
  return cfg::fail(CFG_ERR_RANGE, "a job's size class has no slot within the budget");
}

// The admission / continuous-batching loop over the server's slots. Jobs are
// identified by an index into `jobs` (the caller's list, or the service's
// growing list of taken submissions).
struct Loop {
  cfg_server* s;
  std::vector<std::deque<int>> waiting;
  std::vector<int> slot_job, left;
  size_t used = 0;
  double cu = 0;
  int active = 0;
  long long nstep = 0;
  cudaEvent_t ev[4] = {};
  explicit Loop(cfg_server* srv)
      : s(srv), waiting(srv->cls_nx.size()), slot_job(srv->slot_class.size(), -1), left(srv->slot_class.size(), 0) {}
  ~Loop() { for (auto& e : ev) if (e) cudaEventDestroy(e); }
  int init() {
    for (auto& e : ev) CFG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return CFG_OK;
  }
  double now() const { return std::chrono::duration<double>(Clock::now() - s->t0).count(); }
  // admission: per class in arrival order, while a slot is free and the budget allows
  int admit(const std::vector<cfg_job>& jobs, std::vector<cfg_job_result>& res) {
    cfg::Engine& eng = s->eng;
    const int nslot = (int)s->slot_class.size();
    for (size_t c = 0; c < waiting.size(); c++)
      while (!waiting[c].empty()) {
        int slot = -1;
        for (int k = 0; k < nslot; k++)
          if (s->slot_class[k] == (int)c && slot_job[k] < 0 && used + s->slot_bytes[k] <= s->budget) { slot = k; break; }
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
        res[j].admit_s = now();
      }
    return CFG_OK;
  }
  // one batched step; the host runs at most two steps ahead of the device. on_done(j, slot)
  // is called for each job that took its last step (the device is idle then).
  template <class F>
  int step(const std::vector<cfg_job>& jobs, std::vector<cfg_job_result>& res, F&& on_done) {
    cfg::Engine& eng = s->eng;
    if (nstep >= 2) CFG_CUDA(cudaEventSynchronize(ev[(nstep - 2) % 4]));
    CFG_TRY(eng.step(1));
    CFG_CUDA(cudaEventRecord(ev[nstep % 4], eng.stream()));
    nstep++;
    for (int k = 0; k < (int)slot_job.size(); k++) {
      if (slot_job[k] < 0) continue;
      cu += (double)s->cls_nx[s->slot_class[k]] * s->cls_ny[s->slot_class[k]];
      if (--left[k] > 0) continue;
      const int j = slot_job[k];
      CFG_TRY(eng.synchronize());
      cfg_info inf;
      CFG_TRY(eng.info(k, &inf));
      res[j].steps = jobs[j].nsteps;
      res[j].last_cycles = inf.last_cycles;
      res[j].last_rel = inf.last_rel;
      CFG_TRY(on_done(j, k));
      res[j].done_s = now();
      CFG_TRY(eng.set_active(k, false));
      slot_job[k] = -1;
      used -= s->slot_bytes[k];
      active--;
    }
    return CFG_OK;
  }
};

// the service thread: takes submissions, runs the loop, files results
void service(cfg_server* s) {
  std::vector<cfg_job> jobs;
  std::vector<cfg_job_result> res;
  std::vector<uint64_t> ticket;
  Loop loop(s);
  int rc = loop.init();
  auto fail_all = [&](int code) {
    std::lock_guard<std::mutex> g(s->mu);
    s->worker_rc = code;
    s->worker_msg = cfg::last_error();
    s->running = false;
    s->done_cv.notify_all();
  };
  if (rc != CFG_OK) { fail_all(rc); return; }
  for (;;) {
    {
      std::unique_lock<std::mutex> g(s->mu);
      if (loop.active == 0 && s->queue.empty()) {
        bool waiting = false;
        for (auto& w : loop.waiting) waiting = waiting || !w.empty();
        if (!waiting) {
          if (s->stopping) { s->running = false; s->done_cv.notify_all(); return; }
          s->work_cv.wait(g, [&] { return s->stopping || !s->queue.empty(); });
        }
      }
      while (!s->queue.empty()) {
        const cfg_server::Submitted sub = s->queue.front();
        s->queue.pop_front();
        const int j = (int)jobs.size();
        jobs.push_back(sub.job);
        cfg_job_result r;
        std::memset(&r, 0, sizeof r);
        r.slot = -1;
        r.arrival_s = sub.arrival;
        res.push_back(r);
        ticket.push_back(sub.ticket);
        s->in_flight[sub.ticket] = j;
        loop.waiting[sub.job.size_class].push_back(j);
      }
    }
    rc = loop.admit(jobs, res);
    if (rc != CFG_OK) { fail_all(rc); return; }
    if (loop.active == 0) continue;
    rc = loop.step(jobs, res, [&](int j, int slot) {
      cfg_server::Kept keep;
      const bool want = (jobs[j].flags & CFG_JOB_KEEP_FIELDS) != 0;
      CFG_TRY(field_hash(s->eng, slot, &res[j].hash, &res[j].t_sum, want ? &keep : nullptr));
      res[j].done_s = loop.now();
      std::lock_guard<std::mutex> g(s->mu);
      s->finished[ticket[j]] = res[j];
      if (want) s->kept[ticket[j]] = std::move(keep);
      s->in_flight.erase(ticket[j]);
      s->done_cv.notify_all();
      return CFG_OK;
    });
    if (rc != CFG_OK) { fail_all(rc); return; }
  }
}

void stop_service(cfg_server* s) {
  {
    std::lock_guard<std::mutex> g(s->mu);
    s->stopping = true;
  }
  s->work_cv.notify_all();
  if (s->worker.joinable()) s->worker.join();
  std::lock_guard<std::mutex> g(s->mu);
  s->stopping = false;
}

}  // namespace

cfg_server::~cfg_server() { stop_service(this); }

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
    s->t0 = Clock::now();
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

static bool server_busy(cfg_server* s) {
  std::lock_guard<std::mutex> g(s->mu);
  return s->running || s->sync_busy;
}

int cfg_server_set_solver(cfg_server* s, int mode, int ncycles, double tol, int max_cycles, int coarse_direct,
                          int coarse_cells, int krylov) {
  if (!s) return cfg::fail(CFG_ERR_INVAL, "null cfg_server handle");
  if (server_busy(s)) return cfg::fail(CFG_ERR_BUSY, "the server is running jobs: drain it first");
  CFG_TRY(s->eng.set_solver(mode, ncycles, tol, max_cycles));
  CFG_TRY(s->eng.set_coarse_solve(coarse_direct));
  CFG_TRY(s->eng.set_krylov(krylov));   // 0-3 as cfg_set_krylov
  if (coarse_cells > 0) CFG_TRY(s->eng.set_coarse_cells(coarse_cells));
  return CFG_OK;
}

int cfg_server_set_coarse_w(cfg_server* s, int cells) {
  if (!s) return cfg::fail(CFG_ERR_INVAL, "null cfg_server handle");
  if (server_busy(s)) return cfg::fail(CFG_ERR_BUSY, "the server is running jobs: drain it first");
  return s->eng.set_coarse_w(cells);
}

int cfg_server_slot_bytes(cfg_server* s, int size_class, size_t* bytes) {
  if (!s || !bytes) return cfg::fail(CFG_ERR_INVAL, "null argument");
  for (size_t k = 0; k < s->slot_class.size(); k++)
    if (s->slot_class[k] == size_class) { *bytes = s->slot_bytes[k]; return CFG_OK; }
  return cfg::fail(CFG_ERR_NOENT, "no slot of this size class");
}

int cfg_server_run(cfg_server* s, const cfg_job* jobs_in, int njobs, cfg_job_result* res_out, double* wall_s,
                   double* cell_updates) {
  if (!s || (!jobs_in && njobs > 0) || (!res_out && njobs > 0) || njobs < 0 || !wall_s || !cell_updates)
    return cfg::fail(CFG_ERR_INVAL, "bad argument");
  for (int j = 0; j < njobs; j++) CFG_TRY(check_job(s, jobs_in[j]));
  {
    std::lock_guard<std::mutex> g(s->mu);
    if (s->running || s->sync_busy) return cfg::fail(CFG_ERR_BUSY, "the server is running submitted jobs");
    s->sync_busy = true;
  }
  struct Busy { cfg_server* s; ~Busy() { std::lock_guard<std::mutex> g(s->mu); s->sync_busy = false; } } busy{s};
  std::vector<cfg_job> jobs(jobs_in, jobs_in + njobs);
  std::vector<cfg_job_result> res(njobs);
  for (auto& r : res) { std::memset(&r, 0, sizeof r); r.slot = -1; }
  std::vector<int> order(njobs);
  for (int j = 0; j < njobs; j++) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return jobs[a].arrival_s < jobs[b].arrival_s; });
  Loop loop(s);
  CFG_TRY(loop.init());
  const Clock::time_point saved_t0 = s->t0;
  s->t0 = Clock::now();
  struct T0 { cfg_server* s; Clock::time_point t; ~T0() { s->t0 = t; } } restore{s, saved_t0};
  int next = 0, done = 0;
  while (done < njobs) {
    const double t = loop.now();
    while (next < njobs && jobs[order[next]].arrival_s <= t) {
      res[order[next]].arrival_s = jobs[order[next]].arrival_s;
      loop.waiting[jobs[order[next]].size_class].push_back(order[next]);
      next++;
    }
    CFG_TRY(loop.admit(jobs, res));
    if (loop.active == 0) {
      if (next >= njobs) return cfg::fail(CFG_ERR_RANGE, "waiting jobs can never be admitted");
      const double dtw = jobs[order[next]].arrival_s - loop.now();
      if (dtw > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(dtw, 0.05)));
      continue;
    }
    CFG_TRY(loop.step(jobs, res, [&](int j, int slot) {
      done++;
      return field_hash(s->eng, slot, &res[j].hash, &res[j].t_sum, nullptr);
    }));
  }
  CFG_TRY(s->eng.synchronize());
  *wall_s = loop.now();
  *cell_updates = loop.cu;
  std::copy(res.begin(), res.end(), res_out);
  return CFG_OK;
}

int cfg_server_submit(cfg_server* s, const cfg_job* job, uint64_t* ticket) {
  if (!s || !job || !ticket) return cfg::fail(CFG_ERR_INVAL, "null argument");
  CFG_TRY(check_job(s, *job));
  std::lock_guard<std::mutex> g(s->mu);
  if (s->sync_busy) return cfg::fail(CFG_ERR_BUSY, "cfg_server_run is in progress");
  if (s->worker_rc != CFG_OK) return cfg::fail(s->worker_rc, "the service stopped: " + s->worker_msg);
  if (!s->running) {
    if (s->worker.joinable()) s->worker.join();   // a service that drained and exited
    s->running = true;
    s->worker = std::thread(service, s);
  }
  const uint64_t t = s->next_ticket++;
  s->queue.push_back({t, *job, std::chrono::duration<double>(Clock::now() - s->t0).count()});
  *ticket = t;
  s->work_cv.notify_all();
  return CFG_OK;
}

static int take_result(cfg_server* s, uint64_t ticket, cfg_job_result* out, bool* done) {
  auto it = s->finished.find(ticket);
  if (it != s->finished.end()) {
    if (out) *out = it->second;
    s->finished.erase(it);
    *done = true;
    return CFG_OK;
  }
  *done = false;
  if (s->worker_rc != CFG_OK) return cfg::fail(s->worker_rc, "the service stopped: " + s->worker_msg);
  bool queued = s->in_flight.count(ticket) != 0;
  for (const auto& q : s->queue) queued = queued || q.ticket == ticket;
  if (!queued) return cfg::fail(CFG_ERR_NOENT, "unknown ticket (or its result was already taken)");
  return CFG_OK;
}

int cfg_server_poll(cfg_server* s, uint64_t ticket, cfg_job_result* out, int* done) {
  if (!s || !done) return cfg::fail(CFG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> g(s->mu);
  bool d = false;
  const int rc = take_result(s, ticket, out, &d);
  *done = d ? 1 : 0;
  return rc;
}

int cfg_server_wait(cfg_server* s, uint64_t ticket, double timeout_s, cfg_job_result* out) {
  if (!s || !(timeout_s >= 0)) return cfg::fail(CFG_ERR_INVAL, "bad argument");
  const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(timeout_s));
  std::unique_lock<std::mutex> g(s->mu);
  for (;;) {
    bool d = false;
    CFG_TRY(take_result(s, ticket, out, &d));
    if (d) return CFG_OK;
    if (s->done_cv.wait_until(g, deadline) == std::cv_status::timeout) {
      CFG_TRY(take_result(s, ticket, out, &d));
      if (d) return CFG_OK;
      return cfg::fail(CFG_ERR_TIMEDOUT, "the job has not finished");
    }
  }
}

int cfg_server_drain(cfg_server* s) {
  if (!s) return cfg::fail(CFG_ERR_INVAL, "null cfg_server handle");
  stop_service(s);
  std::lock_guard<std::mutex> g(s->mu);
  if (s->worker_rc != CFG_OK) return cfg::fail(s->worker_rc, "the service stopped: " + s->worker_msg);
  return CFG_OK;
}

int cfg_server_fetch(cfg_server* s, uint64_t ticket, const char* name, float* out, size_t count) {
  if (!s || !name) return cfg::fail(CFG_ERR_INVAL, "null argument");
  std::lock_guard<std::mutex> g(s->mu);
  auto it = s->kept.find(ticket);
  if (it == s->kept.end()) return cfg::fail(CFG_ERR_NOENT, "no kept fields for this ticket (submit with CFG_JOB_KEEP_FIELDS)");
  const std::string n(name);
  const std::vector<float>* f = n == "T" ? &it->second.T : n == "Y" ? &it->second.Y : n == "U" ? &it->second.U
                              : n == "V" ? &it->second.V : nullptr;
  if (!f) return cfg::fail(CFG_ERR_NOENT, "kept fields are T, Y, U and V");
  if (!out) return cfg::fail(CFG_ERR_INVAL, "null output");
  if (count != f->size()) return cfg::fail(CFG_ERR_INVAL, "count must be " + std::to_string(f->size()));
  std::copy(f->begin(), f->end(), out);
  return CFG_OK;
}

int cfg_server_release(cfg_server* s, uint64_t ticket) {
  if (!s) return cfg::fail(CFG_ERR_INVAL, "null cfg_server handle");
  std::lock_guard<std::mutex> g(s->mu);
  if (!s->kept.erase(ticket)) return cfg::fail(CFG_ERR_NOENT, "no kept fields for this ticket");
  return CFG_OK;
}

}  // extern "C"
