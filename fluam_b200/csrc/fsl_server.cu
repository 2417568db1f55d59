// fsl_server.cu -- the serving loop (fsl_server_* C ABI): a scheduler thread
// that admits queued requests into slots of their size class under a device
// memory budget and steps every admitted request together (continuous
// batching).  The slot of a finished request is switched off in its group's
// instance table and handed to the next request of the class, so the
// captured step graph stays valid; only a group whose slot list grows or
// shrinks needs a new capture.
#include <algorithm>
#include <array>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "fsl_group.cuh"

namespace {

using fsl::errorf;

struct Request {
  int64_t id = 0;
  fsl_config cfg{};
  fsl::Params P{};
  std::vector<double> q;  // positions in, final positions out
  std::vector<double> F;  // final forces
  int64_t nsteps = 0, remaining = 0;
  int state = FSL_REQ_QUEUED;
  int error_bits = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
  struct SGroup* group = nullptr;
  int slot = -1;
  std::string msg;
};

// A size class: its group (shared plan and instance table) and its slots.
struct SGroup {
  fsl::Group g;
  std::vector<std::unique_ptr<fsl::Slot>> slots;
  std::vector<Request*> owner;  // per slot; nullptr = free
  int busy = 0;
  int idle_rounds = 0;  // rounds since a slot of this class was last busy
};

// Rounds a class without busy slots stays in the stepped set: a class that
// comes and goes costs a graph capture each time, a class that stays costs
// its (empty) launches every step.
constexpr int kKeepIdleRounds = 4;
// Longest round while no request waits for admission, in units of
// max_round_steps (fewer host round trips; a new arrival waits at most one
// round).
constexpr int kQuietRoundFactor = 4;

// particle capacity of a new slot: the next power of two, at least 64
int capacity_for(int64_t np) {
  int64_t c = 64;
  while (c < np) c <<= 1;
  return (int)c;
}

}  // namespace

struct fsl_server {
  fsl_server_config cfg{};
  std::mutex mu;
  std::condition_variable cv;     // scheduler: work arrived or stop
  std::condition_variable done;   // waiters: a request finished
  std::deque<Request*> queue;
  std::map<int64_t, std::unique_ptr<Request>> reqs;
  int64_t next_id = 1;
  bool stop = false;
  std::thread th;
  std::chrono::steady_clock::time_point t0;
  // scheduler-thread state
  std::map<fsl::ClassKey, std::unique_ptr<SGroup>> groups;
  fsl::Exec exec;
  int64_t bytes_held = 0;
  // statistics (under mu)
  fsl_server_stats st{};

  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
};

namespace {

int64_t count_slots(const fsl_server* s) {
  int64_t n = 0;
  for (const auto& kv : s->groups) n += (int64_t)kv.second->slots.size();
  return n;
}

// Frees idle slots (largest first) until `need` more bytes fit the budget.
// Scheduler thread only.
bool make_room(fsl_server* s, int64_t need) {
  while (s->bytes_held + need > s->cfg.hbm_budget) {
    SGroup* best = nullptr;
    int bi = -1;
    size_t bb = 0;
    for (auto& kv : s->groups) {
      SGroup& G = *kv.second;
      for (size_t i = 0; i < G.slots.size(); ++i)
        if (!G.owner[i] && G.slots[i]->bytes > bb) {
          best = &G;
          bi = (int)i;
          bb = G.slots[i]->bytes;
        }
    }
    if (!best) return false;
    cudaStreamSynchronize(s->exec.stream);
    s->bytes_held -= (int64_t)best->slots[bi]->bytes;
    fsl::slot_free(*best->slots[bi]);
    best->slots.erase(best->slots.begin() + bi);
    best->owner.erase(best->owner.begin() + bi);
    // owners of later slots move down one place
    for (size_t i = bi; i < best->owner.size(); ++i)
      if (best->owner[i]) best->owner[i]->slot = (int)i;
    best->g.slots.clear();
    for (auto& sl : best->slots) best->g.slots.push_back(sl.get());
    best->g.dirty = true;
  }
  return true;
}

// Puts request r into a slot of its class: a free slot with enough capacity
// (the smallest such), else a new slot if the budget allows.  Returns 1 if
// admitted, 0 if it must wait for memory, -1 if it can never fit (r failed).
int admit(fsl_server* s, Request* r) {
  fsl::ClassKey key = fsl::class_of(r->P);
  auto it = s->groups.find(key);
  if (it == s->groups.end()) {
    std::unique_ptr<SGroup> G(new SGroup());
    G->g.allow_one = false;  // slots change between captures
    if (fsl::group_init(G->g, r->P)) {
      r->msg = fsl::last_error();
      return -1;
    }
    it = s->groups.emplace(key, std::move(G)).first;
  }
  SGroup& G = *it->second;
  int pick = -1;
  for (size_t i = 0; i < G.slots.size(); ++i)
    if (!G.owner[i] && G.slots[i]->np_cap >= r->P.np &&
        (pick < 0 || G.slots[i]->np_cap < G.slots[pick]->np_cap))
      pick = (int)i;
  if (pick < 0) {
    const int cap = capacity_for(r->P.np);
    const int64_t need = (int64_t)fsl::slot_bytes(r->P, cap);
    if (need > s->cfg.hbm_budget) {
      r->msg = "request needs more device memory than the server's whole budget";
      return -1;
    }
    if (!make_room(s, need)) return 0;
    std::unique_ptr<fsl::Slot> sl(new fsl::Slot());
    if (fsl::slot_alloc(*sl, r->P, cap, s->exec.stream)) {
      r->msg = fsl::last_error();
      return -1;
    }
    s->bytes_held += (int64_t)sl->bytes;
    G.slots.push_back(std::move(sl));
    G.owner.push_back(nullptr);
    G.g.slots.push_back(G.slots.back().get());
    pick = (int)G.slots.size() - 1;
  }
  fsl::Slot& sl = *G.slots[pick];
  if (fsl::slot_reset(sl, r->P, r->q.data(), r->cfg, s->exec.stream)) {
    r->msg = fsl::last_error();
    return -1;
  }
  G.owner[pick] = r;
  G.busy++;
  G.g.dirty = true;
  r->group = &G;
  r->slot = pick;
  return 1;
}

}  // namespace

namespace {

// Releases r's slot (scheduler thread; caller holds mu).
void release_slot(Request* r) {
  if (!r->group) return;
  SGroup& G = *r->group;
  G.slots[r->slot]->r.active = 0;
  G.owner[r->slot] = nullptr;
  G.busy--;
  G.g.dirty = true;
  r->group = nullptr;
  r->slot = -1;
}

void fail_locked(fsl_server* s, Request* r, const std::string& msg) {
  release_slot(r);
  r->state = FSL_REQ_FAILED;
  r->msg = msg;
  r->t_done = s->now();
  s->st.failed++;
}

void scheduler(fsl_server* s) {
  cudaSetDevice(s->exec.device);
  std::vector<Request*> running;
  for (;;) {
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (running.empty()) s->cv.wait(lk, [&] { return s->stop || !s->queue.empty(); });
      if (s->stop) break;
    }
    // admission in arrival order; the head waits when memory is short
    for (;;) {
      Request* r = nullptr;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->queue.empty()) break;
        r = s->queue.front();
      }
      int a = r->nsteps == 0 ? 2 : admit(s, r);
      if (a == 0) break;
      std::lock_guard<std::mutex> lk(s->mu);
      s->queue.pop_front();
      if (a < 0) {
        fail_locked(s, r, r->msg);
        s->done.notify_all();
      } else if (a == 2) {  // nothing to step: the input is the result
        r->F.assign(r->q.size(), 0.0);
        r->state = FSL_REQ_DONE;
        r->t_start = r->t_done = s->now();
        s->st.completed++;
        s->done.notify_all();
      } else {
        r->state = FSL_REQ_RUNNING;
        r->t_start = s->now();
        r->remaining = r->nsteps;
        running.push_back(r);
      }
    }
    if (running.empty()) continue;
    // one round: the classes with busy slots plus those idle for fewer than
    // kKeepIdleRounds rounds (an idle class's kernels return at once, which
    // is cheaper than a new graph capture while classes come and go), as
    // many steps as the nearest completion, at most max_round_steps (or a
    // few times that while nothing waits for admission)
    std::vector<fsl::Group*> gl;
    for (auto& kv : s->groups) {
      SGroup& G = *kv.second;
      G.idle_rounds = G.busy > 0 ? 0 : G.idle_rounds + 1;
      if (!G.slots.empty() && G.idle_rounds <= kKeepIdleRounds) gl.push_back(&G.g);
    }
    if (gl != s->exec.groups) s->exec.groups = gl;
    bool waiting;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      waiting = !s->queue.empty();
    }
    int64_t n = s->cfg.max_round_steps * (waiting ? 1 : kQuietRoundFactor);
    for (Request* r : running) n = std::min(n, r->remaining);
    const double ta = s->now();
    int rc = fsl::exec_step(s->exec, n);
    std::vector<Request*> fin;
    std::vector<std::array<int, 4>> errs;
    if (rc == FSL_OK) {
      for (Request* r : running) {
        if (r->remaining > n) continue;
        const fsl::Rep& rep = r->group->slots[r->slot]->r;
        const size_t n3 = 3 * (size_t)r->P.np;
        r->F.resize(n3);
        fin.push_back(r);
        errs.push_back(std::array<int, 4>{});
        cudaMemcpyAsync(r->q.data(), rep.q, sizeof(double) * n3, cudaMemcpyDeviceToHost, s->exec.stream);
        cudaMemcpyAsync(r->F.data(), rep.F, sizeof(double) * n3, cudaMemcpyDeviceToHost, s->exec.stream);
        cudaMemcpyAsync(errs.back().data(), rep.err, sizeof(int) * 4, cudaMemcpyDeviceToHost,
                        s->exec.stream);
      }
      cudaError_t ce = cudaStreamSynchronize(s->exec.stream);
      if (ce != cudaSuccess) rc = fsl::cuda_fail(ce, "round");
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.busy_s += s->now() - ta;
    // the scheduler owns these; callers read the snapshot
    s->st.bytes_held = s->bytes_held;
    s->st.slots = count_slots(s);
    s->st.groups = (int64_t)s->groups.size();
    s->st.captures = s->exec.captures;
    if (rc != FSL_OK) {
      std::string m = fsl::last_error();
      for (Request* r : running) fail_locked(s, r, m);
      running.clear();
      s->done.notify_all();
      continue;
    }
    s->st.rounds++;
    for (Request* r : running) {
      r->remaining -= n;
      s->st.steps += n;
      s->st.particle_steps += n * (int64_t)r->P.np;
    }
    const double t = s->now();
    for (size_t k = 0; k < fin.size(); ++k) {
      Request* r = fin[k];
      release_slot(r);
      r->t_done = t;
      r->error_bits = errs[k][fsl::ERR_BITS];
      if (errs[k][fsl::ERR_ANY]) {
        r->state = FSL_REQ_FAILED;
        r->msg = "kernel error word set";
        s->st.failed++;
      } else {
        r->state = FSL_REQ_DONE;
        s->st.completed++;
      }
    }
    running.erase(std::remove_if(running.begin(), running.end(),
                                 [](const Request* r) { return r->remaining <= 0; }),
                  running.end());
    if (!fin.empty()) s->done.notify_all();
  }
  // stopping: whatever is left fails
  std::lock_guard<std::mutex> lk(s->mu);
  for (Request* r : running) fail_locked(s, r, "server stopped");
  for (Request* r : s->queue) fail_locked(s, r, "server stopped");
  s->queue.clear();
  s->done.notify_all();
}

void fill_info(const Request* r, fsl_request_info* info) {
  std::memset(info, 0, sizeof(*info));
  info->state = r->state;
  info->error_bits = r->error_bits;
  info->np = r->P.np;
  info->steps = r->nsteps;
  info->steps_done = r->state == FSL_REQ_QUEUED ? 0 : r->nsteps - std::max<int64_t>(r->remaining, 0);
  if (r->state == FSL_REQ_DONE) info->steps_done = r->nsteps;
  info->submit_s = r->t_submit;
  info->start_s = r->t_start;
  info->done_s = r->t_done;
}

}  // namespace

extern "C" {

void fsl_server_config_defaults(fsl_server_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->hbm_budget = (int64_t)150 * 1000 * 1000 * 1000;
  c->device = -1;
  c->max_round_steps = 8;
}

int fsl_server_create(const fsl_server_config* cfg, fsl_server** out) {
  if (!cfg || !out) return errorf(FSL_E_ARG, "null argument");
  *out = nullptr;
  if (cfg->hbm_budget <= 0) return errorf(FSL_E_ARG, "hbm_budget must be > 0");
  if (cfg->max_round_steps < 1) return errorf(FSL_E_ARG, "max_round_steps must be >= 1");
  int dev = cfg->device;
  if (dev < 0) FSL_TRY(cudaGetDevice(&dev));
  fsl_server* s = new fsl_server();
  s->cfg = *cfg;
  s->cfg.device = dev;
  s->t0 = std::chrono::steady_clock::now();
  int rc = fsl::exec_init(s->exec, dev);
  if (rc) {
    delete s;
    return rc;
  }
  s->th = std::thread(scheduler, s);
  *out = s;
  return FSL_OK;
}

void fsl_server_destroy(fsl_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv.notify_all();
  if (s->th.joinable()) s->th.join();
  cudaSetDevice(s->exec.device);
  fsl::exec_destroy(s->exec);
  for (auto& kv : s->groups) {
    fsl::group_destroy(kv.second->g);
    for (auto& sl : kv.second->slots) fsl::slot_free(*sl);
  }
  delete s;
}

int fsl_server_submit(fsl_server* s, const fsl_config* cfg, int64_t np, const double* q,
                      int64_t nsteps, int64_t* id) {
  if (!s || !cfg || !id) return errorf(FSL_E_ARG, "null argument");
  if (nsteps < 0) return errorf(FSL_E_ARG, "negative step count");
  std::unique_ptr<Request> r(new Request());
  int rc = fsl::make_params(*cfg, np, r->P);
  if (rc) return rc;
  if (np > 0 && !q) return errorf(FSL_E_ARG, "null positions");
  if (cfg->device >= 0 && cfg->device != s->cfg.device)
    return errorf(FSL_E_ARG, "request for device %d on a server of device %d", cfg->device,
                  s->cfg.device);
  r->cfg = *cfg;
  r->q.assign(q, q + 3 * (size_t)np);
  r->nsteps = nsteps;
  r->remaining = nsteps;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->stop) return errorf(FSL_E_ARG, "server stopped");
  r->id = s->next_id++;
  r->t_submit = s->now();
  *id = r->id;
  s->queue.push_back(r.get());
  s->reqs.emplace(r->id, std::move(r));
  s->st.submitted++;
  s->cv.notify_all();
  return FSL_OK;
}

int fsl_server_poll(fsl_server* s, int64_t id, fsl_request_info* info) {
  if (!s || !info) return errorf(FSL_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return errorf(FSL_E_ARG, "unknown request %lld", (long long)id);
  fill_info(it->second.get(), info);
  return FSL_OK;
}

int fsl_server_wait(fsl_server* s, int64_t id, double timeout_s, fsl_request_info* info) {
  if (!s || !info) return errorf(FSL_E_ARG, "null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return errorf(FSL_E_ARG, "unknown request %lld", (long long)id);
  Request* r = it->second.get();
  auto fin = [&] { return r->state == FSL_REQ_DONE || r->state == FSL_REQ_FAILED; };
  if (timeout_s < 0) s->done.wait(lk, fin);
  else s->done.wait_for(lk, std::chrono::duration<double>(timeout_s), fin);
  fill_info(r, info);
  return FSL_OK;
}

int fsl_server_result(fsl_server* s, int64_t id, double* q_out, double* F_out) {
  if (!s) return errorf(FSL_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return errorf(FSL_E_ARG, "unknown request %lld", (long long)id);
  Request* r = it->second.get();
  if (r->state == FSL_REQ_QUEUED || r->state == FSL_REQ_RUNNING)
    return errorf(FSL_E_ARG, "request %lld has not finished", (long long)id);
  int rc = FSL_OK;
  if (r->state == FSL_REQ_FAILED) {
    rc = errorf(r->error_bits ? FSL_E_KERNEL : FSL_E_CUDA, "request %lld failed: %s (bits 0x%x)",
                (long long)id, r->msg.c_str(), r->error_bits);
  } else {
    if (q_out) std::memcpy(q_out, r->q.data(), sizeof(double) * r->q.size());
    if (F_out) std::memcpy(F_out, r->F.data(), sizeof(double) * r->F.size());
  }
  s->reqs.erase(it);
  return rc;
}

int fsl_server_get_stats(fsl_server* s, fsl_server_stats* st) {
  if (!s || !st) return errorf(FSL_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *st = s->st;
  st->queued = (int64_t)s->queue.size();
  int64_t running = 0;
  for (const auto& kv : s->reqs)
    if (kv.second->state == FSL_REQ_RUNNING) running++;
  st->running = running;
  st->now_s = s->now();
  return FSL_OK;
}

}  // extern "C"
