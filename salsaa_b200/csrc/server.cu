// server.cu — continuous-batching proof service on one GPU.
//
// Parameter sets are registered with a number of proof slots (device
// workspace + stream each), preallocated inside an HBM budget so that no
// allocation happens while proofs run.  Submitted requests wait in a FIFO;
// salsaa_server_progress() retires finished proofs (CUDA events) and admits
// waiting requests whenever a slot of their parameter set is free, skipping
// past requests whose set is saturated so one busy set does not block the
// others.  Admitted proofs run concurrently on their slots' streams, with
// witnesses and all round state resident in HBM.
#include <chrono>
#include <deque>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/salsaa_gpu.h"
#include "kernels.cuh"

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Slot {
  salsaa_prover* pr = nullptr;
  cudaEvent_t done = nullptr;
  uint64_t ticket = 0;  // 0 = free
};

struct PSet {
  salsaa_ctx* ctx = nullptr;
  uint64_t workspace = 0;
  std::vector<Slot> slots;
};

enum ReqState { RQ_QUEUED = 1, RQ_RUNNING = 2, RQ_DONE = 3, RQ_FAILED = 4 };

struct Req {
  int set = 0;
  uint64_t seed = 0;
  const uint64_t* d_witness = nullptr;
  uint8_t* d_proof = nullptr;
  int state = RQ_QUEUED;
  int rc = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
  int slot = -1;
};

}  // namespace

struct salsaa_server {
  int device = 0;
  uint64_t budget = 0, used = 0;
  std::vector<PSet> sets;
  std::unordered_map<uint64_t, Req> reqs;
  std::deque<uint64_t> queue;
  uint64_t next_ticket = 1;
  uint32_t max_inflight = 0;  // 0 = as many as there are slots
  std::mutex mu;
};

extern "C" int salsaa_server_create(int device, uint64_t hbm_budget_bytes, salsaa_server** out) {
  if (!out) return salsaa_set_error(-1, "server_create: null output");
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "server_create: cudaSetDevice");
  salsaa_server* s = new (std::nothrow) salsaa_server;
  if (!s) return salsaa_set_error(-1, "server_create: out of host memory");
  s->device = device;
  s->budget = hbm_budget_bytes;
  *out = s;
  return 0;
}

extern "C" int salsaa_server_register(salsaa_server* s, const salsaa_params* p, uint64_t crs_seed, uint32_t slots,
                                      int* set_id) {
  if (!s || !p || !set_id || slots == 0) return salsaa_set_error(-1, "server_register: bad argument");
  std::lock_guard<std::mutex> lk(s->mu);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "server_register: cudaSetDevice");
  const uint64_t ws = salsaa_workspace_bytes(p);
  if (!ws) return salsaa_set_error(-1, "server_register: invalid parameter set");
  if (s->used + (uint64_t)slots * ws > s->budget)
    return salsaa_set_error(-5, "server_register: slots exceed the HBM budget");
  PSet ps;
  int rc = salsaa_ctx_create(p, crs_seed, s->device, &ps.ctx);
  if (rc) return rc;
  ps.workspace = ws;
  for (uint32_t i = 0; i < slots; i++) {
    Slot sl;
    rc = salsaa_prover_create(ps.ctx, &sl.pr);
    if (!rc && cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess)
      rc = salsaa_set_error(-1, "server_register: event");
    if (rc) {
      if (sl.pr) salsaa_prover_destroy(sl.pr);
      for (Slot& o : ps.slots) {
        salsaa_prover_destroy(o.pr);
        cudaEventDestroy(o.done);
      }
      salsaa_ctx_destroy(ps.ctx);
      return rc;
    }
    ps.slots.push_back(sl);
  }
  s->used += (uint64_t)slots * ws;
  s->sets.push_back(ps);
  *set_id = (int)s->sets.size() - 1;
  return 0;
}

extern "C" int salsaa_server_submit(salsaa_server* s, int set_id, uint64_t seed, const uint64_t* d_witness,
                                    uint8_t* d_proof, uint64_t* ticket) {
  if (!s || !d_proof || !ticket) return salsaa_set_error(-1, "server_submit: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  if (set_id < 0 || set_id >= (int)s->sets.size()) return salsaa_set_error(-1, "server_submit: unknown set");
  Req r;
  r.set = set_id;
  r.seed = seed;
  r.d_witness = d_witness;
  r.d_proof = d_proof;
  r.t_submit = now_ms();
  const uint64_t t = s->next_ticket++;
  s->reqs.emplace(t, r);
  s->queue.push_back(t);
  *ticket = t;
  return 0;
}

// Retire finished proofs, then admit queued requests onto free slots.
// Returns the number of requests still queued or running.
extern "C" int salsaa_server_progress(salsaa_server* s) {
  if (!s) return salsaa_set_error(-1, "server_progress: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return salsaa_set_cuda_error(e, "server_progress: cudaSetDevice");
  for (PSet& ps : s->sets)
    for (Slot& sl : ps.slots) {
      if (!sl.ticket) continue;
      e = cudaEventQuery(sl.done);
      if (e == cudaErrorNotReady) continue;
      Req& r = s->reqs[sl.ticket];
      if (e != cudaSuccess) {
        r.state = RQ_FAILED;
        r.rc = salsaa_set_cuda_error(e, "server: proof");
      } else {
        r.state = RQ_DONE;
      }
      r.t_done = now_ms();
      sl.ticket = 0;
    }
  uint32_t running = 0;
  for (PSet& ps : s->sets)
    for (Slot& sl : ps.slots)
      if (sl.ticket) running++;
  for (auto it = s->queue.begin(); it != s->queue.end();) {
    if (s->max_inflight && running >= s->max_inflight) break;
    Req& r = s->reqs[*it];
    PSet& ps = s->sets[r.set];
    int free_slot = -1;
    for (size_t i = 0; i < ps.slots.size(); i++)
      if (!ps.slots[i].ticket) {
        free_slot = (int)i;
        break;
      }
    if (free_slot < 0) {
      ++it;
      continue;
    }
    Slot& sl = ps.slots[free_slot];
    r.t_start = now_ms();
    int rc = salsaa_prover_enqueue(sl.pr, r.seed, r.d_witness, r.d_proof);
    if (!rc && cudaEventRecord(sl.done, (cudaStream_t)salsaa_prover_stream(sl.pr)) != cudaSuccess)
      rc = salsaa_set_error(-1, "server: event record");
    if (rc) {
      r.state = RQ_FAILED;
      r.rc = rc;
      r.t_done = now_ms();
    } else {
      r.state = RQ_RUNNING;
      r.slot = free_slot;
      sl.ticket = *it;
      running++;
    }
    it = s->queue.erase(it);
  }
  int pending = (int)s->queue.size();
  for (PSet& ps : s->sets)
    for (Slot& sl : ps.slots)
      if (sl.ticket) pending++;
  return pending;
}

// Cap on proofs running at once over all parameter sets (0 = no cap beyond
// the slots).  Every admitted proof shares the GPU with the others, so a
// small cap keeps completion close to arrival order (tail latency) while
// still overlapping one proof's short kernels with another's.
extern "C" int salsaa_server_limit(salsaa_server* s, uint32_t max_inflight) {
  if (!s) return salsaa_set_error(-1, "server_limit: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  s->max_inflight = max_inflight;
  return 0;
}

// 1 queued or running, 0 done (latencies in ms: from submit, and on the GPU
// from admission), negative on failure.  A finished ticket is forgotten.
extern "C" int salsaa_server_poll(salsaa_server* s, uint64_t ticket, double* latency_ms, double* run_ms) {
  if (!s) return salsaa_set_error(-1, "server_poll: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return salsaa_set_error(-1, "server_poll: unknown ticket");
  Req& r = it->second;
  if (r.state == RQ_QUEUED || r.state == RQ_RUNNING) return 1;
  const int rc = r.state == RQ_DONE ? 0 : (r.rc ? r.rc : -1);
  if (latency_ms) *latency_ms = r.t_done - r.t_submit;
  if (run_ms) *run_ms = r.t_done - r.t_start;
  s->reqs.erase(it);
  return rc;
}

// Withdraw a request that is still queued: it is forgotten (a later poll
// reports an unknown ticket) and its proof buffer is the caller's again.
// A request already admitted keeps running, since its kernels are in flight
// on the slot's stream; it is reported (1) and completes as usual.
extern "C" int salsaa_server_cancel(salsaa_server* s, uint64_t ticket) {
  if (!s) return salsaa_set_error(-1, "server_cancel: null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return salsaa_set_error(-1, "server_cancel: unknown ticket");
  if (it->second.state != RQ_QUEUED) return 1;
  for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
    if (*q == ticket) {
      s->queue.erase(q);
      break;
    }
  s->reqs.erase(it);
  return 0;
}

extern "C" void salsaa_server_destroy(salsaa_server* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  for (PSet& ps : s->sets) {
    for (Slot& sl : ps.slots) {
      salsaa_prover_destroy(sl.pr);
      cudaEventDestroy(sl.done);
    }
    salsaa_ctx_destroy(ps.ctx);
  }
  delete s;
}
