// Serving loop: continuous batching of verification requests over a
// resident reference (no counterpart in the reference, whose API verifies one
// caller-filled buffer per send).
//
// Threads:
//  * submitters (callers) copy each request into the server and queue it;
//  * the dispatcher takes every queued request that fits a free batch slot,
//    packs them into the slot's pinned buffers (query indices and PEQ entry
//    offsets rebased to the batch), and enqueues H2D copies, the kernels and
//    the D2H copy of the results on the slot's stream;
//  * the completer waits for the slots in dispatch order, hands the results
//    back to the requests and frees the slot.
// With K slots, K batches are in flight: while one runs, the next gathers
// whatever arrived meanwhile -- batches grow with the load and shrink to one
// request when the server is idle.
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/myers-interface.h"
#include "myers_internal.h"

using namespace myers;

namespace {

using Clock = std::chrono::steady_clock;

inline uint64_t now_ns() {
  return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now().time_since_epoch()).count();
}

enum { kPending = 0, kInFlight = 1, kDone = 2 };

struct Request {
  uint64_t ticket;
  uint32_t m;
  int state;
  int status;
  std::vector<qryEntry_t> peq;
  std::vector<uint64_t> pos;
  std::vector<resEntry_t> res;
  uint64_t t_done;
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  cudaGraphExec_t exec = nullptr;  // the last batch's copies + kernels, updated per batch
  myersContext* ctx = nullptr;
  qryEntry_t* h_peq = nullptr;
  qryInfo_t* h_qinfo = nullptr;
  candInfo_t* h_cands = nullptr;
  resEntry_t* h_res = nullptr;
  qryEntry_t* d_peq = nullptr;
  qryInfo_t* d_qinfo = nullptr;
  candInfo_t* d_cands = nullptr;
  resEntry_t* d_res = nullptr;
  std::vector<Request*> reqs;
  uint32_t ncands = 0;
  bool busy = false;
};

uint32_t entries_of(uint32_t m) { return (m + NUM_BASES_ENTRY - 1) / NUM_BASES_ENTRY; }

}  // namespace

struct myersServer {
  const myersReference* ref = nullptr;
  bool want_requests = false;        // the dispatcher sleeps for lack of requests
  std::vector<Request*> free_reqs;   // recycled requests (their vectors keep capacity)
  myersServerConfig_t cfg{};
  uint32_t cap_cands = 0, cap_queries = 0, cap_entries = 0;
  std::vector<Slot> slots;
  std::mutex mu;
  std::condition_variable cv_dispatch, cv_complete, cv_done;
  std::deque<Request*> pending;
  std::deque<int> inflight;
  std::unordered_map<uint64_t, Request*> live;
  std::thread dispatcher, completer;
  bool stop = false;
  int fatal = MYERS_SUCCESS;
  uint64_t next_ticket = 1;
  myersServerStats_t stats{};
};

static void slot_free(Slot& s) {
  if (s.stream) cudaStreamSynchronize(s.stream);
  cudaFreeHost(s.h_peq);
  cudaFreeHost(s.h_qinfo);
  cudaFreeHost(s.h_cands);
  cudaFreeHost(s.h_res);
  cudaFree(s.d_peq);
  cudaFree(s.d_qinfo);
  cudaFree(s.d_cands);
  cudaFree(s.d_res);
  if (s.exec) cudaGraphExecDestroy(s.exec);
  if (s.ctx) myersContextDestroy(s.ctx);
  if (s.done) cudaEventDestroy(s.done);
  if (s.stream) cudaStreamDestroy(s.stream);
  s = Slot();
}

static int slot_alloc(Slot& s, uint32_t nc, uint32_t nq, uint32_t ne) {
  if (cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) != cudaSuccess) return MYERS_E_CUDA;
  if (cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming) != cudaSuccess) return MYERS_E_CUDA;
  if (cudaHostAlloc((void**)&s.h_peq, (size_t)ne * sizeof(qryEntry_t), 0) != cudaSuccess ||
      cudaHostAlloc((void**)&s.h_qinfo, (size_t)nq * sizeof(qryInfo_t), 0) != cudaSuccess ||
      cudaHostAlloc((void**)&s.h_cands, (size_t)nc * sizeof(candInfo_t), 0) != cudaSuccess ||
      cudaHostAlloc((void**)&s.h_res, (size_t)nc * sizeof(resEntry_t), 0) != cudaSuccess)
    return MYERS_E_ALLOCATE_MEM;
  if (cudaMalloc((void**)&s.d_peq, (size_t)ne * sizeof(qryEntry_t)) != cudaSuccess ||
      cudaMalloc((void**)&s.d_qinfo, (size_t)nq * sizeof(qryInfo_t)) != cudaSuccess ||
      cudaMalloc((void**)&s.d_cands, (size_t)nc * sizeof(candInfo_t)) != cudaSuccess ||
      cudaMalloc((void**)&s.d_res, (size_t)nc * sizeof(resEntry_t)) != cudaSuccess)
    return MYERS_E_INSUFFICIENT_MEM_GPU;
  return myersContextCreate(&s.ctx, nc);
}

static int enqueue_batch(myersServer* srv, Slot& s, const PlanTable& plan, uint32_t ne, uint32_t nq, uint32_t nc);

// Pack the slot's requests, enqueue copies and kernels. Runs on the
// dispatcher thread without the lock (the slot and its requests are owned by
// the dispatcher until it is pushed on the in-flight queue).
static int dispatch_slot(myersServer* srv, Slot& s) {
  NvtxRange range("myers server: pack and launch a batch");
  uint8_t present[kMaxWords + 1];
  memset(present, 0, sizeof(present));
  uint32_t ne = 0, nq = 0, nc = 0;
  for (Request* r : s.reqs) {
    const uint32_t e = entries_of(r->m);
    memcpy(s.h_peq + ne, r->peq.data(), (size_t)e * sizeof(qryEntry_t));
    s.h_qinfo[nq].posEntry = ne;
    s.h_qinfo[nq].size = r->m;
    for (size_t k = 0; k < r->pos.size(); ++k) {
      s.h_cands[nc + k].query = nq;
      s.h_cands[nc + k].position = r->pos[k];
    }
    if (r->m > 0) present[(r->m + 31) / 32] = 1;
    ne += e;
    ++nq;
    nc += (uint32_t)r->pos.size();
  }
  s.ncands = nc;
  PlanTable plan;
  int st = build_plan(plan, present, srv->cfg.path == MYERS_PATH_BATCHED, srv->cfg.laneWords, nc, nq);
  if (st != MYERS_SUCCESS) return st;
  // With graphs, the batch's copies and kernels are captured and replayed as
  // one graph, updated in place from the slot's previous batch.
  if (srv->cfg.useGraphs != 0)
    st = launch_as_graph(s.stream, &s.exec, [&] { return enqueue_batch(srv, s, plan, ne, nq, nc); });
  else
    st = enqueue_batch(srv, s, plan, ne, nq, nc);
  if (st != MYERS_SUCCESS) return st;
  if (cudaEventRecord(s.done, s.stream) != cudaSuccess) return MYERS_E_CUDA;
  return MYERS_SUCCESS;
}

// Copies and kernels of one packed batch on the slot's stream.
static int enqueue_batch(myersServer* srv, Slot& s, const PlanTable& plan, uint32_t ne, uint32_t nq, uint32_t nc) {
  int st;
  if (cudaMemcpyAsync(s.d_peq, s.h_peq, (size_t)ne * sizeof(qryEntry_t), cudaMemcpyHostToDevice, s.stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(s.d_qinfo, s.h_qinfo, (size_t)nq * sizeof(qryInfo_t), cudaMemcpyHostToDevice, s.stream) !=
          cudaSuccess ||
      cudaMemcpyAsync(s.d_cands, s.h_cands, (size_t)nc * sizeof(candInfo_t), cudaMemcpyHostToDevice, s.stream) !=
          cudaSuccess)
    return MYERS_E_CUDA;
  DevInputs in;
  memset(&in, 0, sizeof(in));
  in.peq = reinterpret_cast<const uint32_t*>(s.d_peq);
  in.qinfo = reinterpret_cast<const uint2*>(s.d_qinfo);
  in.cands = reinterpret_cast<const Cand*>(s.d_cands);
  in.results = reinterpret_cast<uint2*>(s.d_res);
  in.num_cands = nc;
  in.num_queries = nq;
  in.num_entries = ne;
  in.distance = srv->cfg.distance;
  in.exact = srv->cfg.windowMode == MYERS_WINDOW_EXACT;
  st = verify_enqueue(s.ctx, srv->ref, in, plan, srv->cfg.path, s.stream);
  if (st != MYERS_SUCCESS) return st;
  if (cudaMemcpyAsync(s.h_res, s.d_res, (size_t)nc * sizeof(resEntry_t), cudaMemcpyDeviceToHost, s.stream) !=
      cudaSuccess)
    return MYERS_E_CUDA;
  return MYERS_SUCCESS;
}

static void dispatcher_main(myersServer* srv) {
  cudaSetDevice(srv->ref->device);
  std::unique_lock<std::mutex> lk(srv->mu);
  while (true) {
    int free_slot = -1;
    srv->cv_dispatch.wait(lk, [&] {
      if (srv->stop && srv->pending.empty()) return true;
      srv->want_requests = srv->pending.empty();
      if (srv->pending.empty()) return false;
      for (size_t i = 0; i < srv->slots.size(); ++i)
        if (!srv->slots[i].busy) {
          free_slot = (int)i;
          return true;
        }
      return false;
    });
    srv->want_requests = false;
    if (free_slot < 0) break;  // stopping, nothing left
    Slot& s = srv->slots[free_slot];
    s.reqs.clear();
    uint32_t ne = 0, nq = 0, nc = 0;
    while (!srv->pending.empty()) {
      Request* r = srv->pending.front();
      const uint32_t e = entries_of(r->m);
      if (ne + e > srv->cap_entries || nq + 1 > srv->cap_queries || nc + r->pos.size() > srv->cap_cands) break;
      srv->pending.pop_front();
      r->state = kInFlight;
      s.reqs.push_back(r);
      ne += e;
      ++nq;
      nc += (uint32_t)r->pos.size();
    }
    s.busy = true;
    lk.unlock();
    const int st = dispatch_slot(srv, s);
    lk.lock();
    if (st != MYERS_SUCCESS) {
      srv->fatal = st;
      for (Request* r : s.reqs) {
        r->status = st;
        r->state = kDone;
        r->t_done = now_ns();
      }
      s.reqs.clear();
      s.busy = false;
      srv->cv_done.notify_all();
      continue;
    }
    srv->stats.batches++;
    if (nc > srv->stats.batchCandidatesMax) srv->stats.batchCandidatesMax = nc;
    srv->inflight.push_back(free_slot);
    srv->cv_complete.notify_one();
  }
  srv->cv_complete.notify_one();
}

static void completer_main(myersServer* srv) {
  cudaSetDevice(srv->ref->device);
  std::unique_lock<std::mutex> lk(srv->mu);
  while (true) {
    srv->cv_complete.wait(lk, [&] {
      return !srv->inflight.empty() || (srv->stop && srv->pending.empty() && srv->inflight.empty());
    });
    if (srv->inflight.empty()) {
      bool any_busy = false;
      for (auto& s : srv->slots) any_busy |= s.busy;
      if (!any_busy) break;
      continue;
    }
    const int si = srv->inflight.front();
    srv->inflight.pop_front();
    Slot& s = srv->slots[si];
    lk.unlock();
    cudaError_t e;
    {
      NvtxRange range("myers server: wait for a batch");
      e = cudaEventSynchronize(s.done);
    }
    const uint64_t t = now_ns();
    uint32_t off = 0;
    {
      NvtxRange range("myers server: hand back results");
      for (Request* r : s.reqs) {
        const size_t n = r->pos.size();
        r->res.assign(s.h_res + off, s.h_res + off + n);
        off += (uint32_t)n;
      }
    }
    lk.lock();
    for (Request* r : s.reqs) {
      r->status = e == cudaSuccess ? MYERS_SUCCESS : MYERS_E_CUDA;
      r->state = kDone;
      r->t_done = t;
      srv->stats.completed++;
      srv->stats.candidatesCompleted += r->pos.size();
    }
    if (e != cudaSuccess) srv->fatal = MYERS_E_CUDA;
    s.reqs.clear();
    s.busy = false;
    srv->cv_done.notify_all();
    srv->cv_dispatch.notify_one();
  }
}

extern "C" int myersServerCreate(myersServer_t** out, const myersReference_t* ref, const myersServerConfig_t* cfg) {
  if (out == nullptr || ref == nullptr) return MYERS_E_INVALID_ARGUMENT;
  myersServer* srv = new myersServer();
  srv->ref = ref;
  if (cfg) srv->cfg = *cfg;
  myersServerConfig_t& c = srv->cfg;
  if (c.slots == 0) c.slots = 4;
  if (c.maxQueued == 0) c.maxQueued = 1u << 20;
  if (c.maxQuerySize == 0) c.maxQuerySize = 1024;
  if (c.distance == 0.0f && cfg == nullptr) c.distance = 0.2f;
  if (c.path != MYERS_PATH_PLAIN) c.path = MYERS_PATH_BATCHED;
  if (!(c.distance >= 0.0f) || c.maxQuerySize > kMaxWords * 32 ||
      (c.windowMode != MYERS_WINDOW_ALIGNED && c.windowMode != MYERS_WINDOW_EXACT)) {
    delete srv;
    return MYERS_E_INVALID_ARGUMENT;
  }
  if (cudaSetDevice(ref->device) != cudaSuccess) {
    delete srv;
    return MYERS_E_CUDA;
  }
  size_t freeb = 0, totalb = 0;
  cudaMemGetInfo(&freeb, &totalb);
  uint64_t budget = c.budgetBytes ? c.budgetBytes : (16ull << 30);
  if (budget > (uint64_t)(freeb * 0.8)) budget = (uint64_t)(freeb * 0.8);
  c.budgetBytes = budget;
  // device bytes per candidate slot: candidate 16 + result 8 + bucketing 5, and
  // room for one query of maxQuerySize per candidate (the worst case, one
  // candidate per read)
  const uint64_t per_query = (uint64_t)entries_of(c.maxQuerySize) * sizeof(qryEntry_t) + sizeof(qryInfo_t);
  const uint64_t per_slot = budget / c.slots;
  uint64_t nc = c.maxBatchCandidates ? c.maxBatchCandidates : (1u << 20);
  if (nc > (1u << 26)) nc = 1u << 26;
  if (nc * (29 + per_query) > per_slot) nc = per_slot / (29 + per_query);
  if (nc < 1) {
    delete srv;
    return MYERS_E_INSUFFICIENT_MEM_GPU;
  }
  srv->cap_cands = (uint32_t)nc;
  srv->cap_queries = (uint32_t)nc;
  srv->cap_entries = (uint32_t)(nc * entries_of(c.maxQuerySize));
  srv->slots.resize(c.slots);
  for (auto& s : srv->slots) {
    const int st = slot_alloc(s, srv->cap_cands, srv->cap_queries, srv->cap_entries);
    if (st != MYERS_SUCCESS) {
      for (auto& t : srv->slots) slot_free(t);
      delete srv;
      return st;
    }
  }
  srv->stats.slots = c.slots;
  srv->stats.maxBatchCandidates = srv->cap_cands;
  srv->stats.maxBatchQueries = srv->cap_queries;
  srv->stats.maxBatchEntries = srv->cap_entries;
  srv->dispatcher = std::thread(dispatcher_main, srv);
  srv->completer = std::thread(completer_main, srv);
  *out = srv;
  return MYERS_SUCCESS;
}

namespace {
struct SubmitItem {
  const qryEntry_t* peq;
  uint32_t m;
  const uint64_t* pos;
  uint32_t ncand;
};
}  // namespace

// Queue n requests under one lock round (the replay driver uses it when
// several requests are due at once). status[i] / ticket[i] per request.
static void submit_many(myersServer* srv, const SubmitItem* it, uint32_t n, int* status, uint64_t* ticket) {
  Request* reqs[256];
  uint32_t ok = 0;
  for (uint32_t i = 0; i < n; ++i) {
    status[i] = MYERS_SUCCESS;
    if (it[i].m > srv->cfg.maxQuerySize) status[i] = MYERS_E_QUERY_TOO_LONG;
    else if (it[i].ncand > srv->cap_cands || entries_of(it[i].m) > srv->cap_entries) status[i] = MYERS_E_CAPACITY;
  }
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    for (uint32_t i = 0; i < n; ++i) {
      reqs[i] = nullptr;
      if (status[i] != MYERS_SUCCESS) continue;
      if (srv->stop) status[i] = MYERS_E_INVALID_ARGUMENT;
      else if (srv->fatal != MYERS_SUCCESS) status[i] = srv->fatal;
      else if (srv->pending.size() + ok >= srv->cfg.maxQueued) {
        srv->stats.refused++;
        status[i] = MYERS_E_BUSY;
      } else {
        ++ok;
        if (!srv->free_reqs.empty()) {
          reqs[i] = srv->free_reqs.back();
          srv->free_reqs.pop_back();
        }
      }
    }
  }
  for (uint32_t i = 0; i < n; ++i) {
    if (status[i] != MYERS_SUCCESS) continue;
    Request* r = reqs[i] ? reqs[i] : new Request();
    r->m = it[i].m;
    r->state = kPending;
    r->status = MYERS_SUCCESS;
    r->peq.assign(it[i].peq, it[i].peq + entries_of(it[i].m));
    r->pos.assign(it[i].pos, it[i].pos + it[i].ncand);
    reqs[i] = r;
  }
  bool wake = false;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    for (uint32_t i = 0; i < n; ++i) {
      if (status[i] != MYERS_SUCCESS) continue;
      Request* r = reqs[i];
      r->ticket = srv->next_ticket++;
      srv->live[r->ticket] = r;
      srv->pending.push_back(r);
      srv->stats.submitted++;
      ticket[i] = r->ticket;
    }
    wake = srv->want_requests && ok > 0;
  }
  if (wake) srv->cv_dispatch.notify_one();
}

extern "C" int myersServerSubmit(myersServer_t* srv, const qryEntry_t* peq, uint32_t querySize,
                                 const uint64_t* positions, uint32_t numCandidates, uint64_t* ticket) {
  if (srv == nullptr || ticket == nullptr || (querySize > 0 && peq == nullptr) ||
      (numCandidates > 0 && positions == nullptr))
    return MYERS_E_INVALID_ARGUMENT;
  if (querySize > srv->cfg.maxQuerySize) return MYERS_E_QUERY_TOO_LONG;
  if (numCandidates > srv->cap_cands || entries_of(querySize) > srv->cap_entries) return MYERS_E_CAPACITY;
  Request* r = nullptr;
  bool wake = false;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stop) return MYERS_E_INVALID_ARGUMENT;
    if (srv->fatal != MYERS_SUCCESS) return srv->fatal;
    if (srv->pending.size() >= srv->cfg.maxQueued) {
      srv->stats.refused++;
      return MYERS_E_BUSY;
    }
    if (!srv->free_reqs.empty()) {
      r = srv->free_reqs.back();
      srv->free_reqs.pop_back();
    }
  }
  if (r == nullptr) r = new Request();
  r->m = querySize;
  r->state = kPending;
  r->status = MYERS_SUCCESS;
  r->peq.assign(peq, peq + entries_of(querySize));
  r->pos.assign(positions, positions + numCandidates);
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    r->ticket = srv->next_ticket++;
    srv->live[r->ticket] = r;
    srv->pending.push_back(r);
    srv->stats.submitted++;
    wake = srv->want_requests;  // a dispatcher waiting for a free slot is woken by the completer
  }
  if (wake) srv->cv_dispatch.notify_one();
  *ticket = r->ticket;
  return MYERS_SUCCESS;
}

static int take_result(myersServer* srv, uint64_t ticket, resEntry_t* results, bool wait, uint32_t timeout_ms) {
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->live.find(ticket);
  if (it == srv->live.end()) return MYERS_E_INVALID_ARGUMENT;
  Request* r = it->second;
  if (r->state != kDone) {
    if (!wait) return MYERS_E_NOT_READY;
    if (!srv->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->state == kDone; }))
      return MYERS_E_TIMEOUT;
  }
  const int st = r->status;
  if (results && !r->res.empty()) memcpy(results, r->res.data(), r->res.size() * sizeof(resEntry_t));
  srv->live.erase(it);
  srv->free_reqs.push_back(r);
  return st;
}

extern "C" int myersServerPoll(myersServer_t* srv, uint64_t ticket, resEntry_t* results) {
  if (srv == nullptr) return MYERS_E_INVALID_ARGUMENT;
  return take_result(srv, ticket, results, false, 0);
}

extern "C" int myersServerWait(myersServer_t* srv, uint64_t ticket, resEntry_t* results, uint32_t timeoutMs) {
  if (srv == nullptr) return MYERS_E_INVALID_ARGUMENT;
  return take_result(srv, ticket, results, true, timeoutMs);
}

extern "C" int myersServerStats(myersServer_t* srv, myersServerStats_t* st) {
  if (srv == nullptr || st == nullptr) return MYERS_E_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(srv->mu);
  *st = srv->stats;
  return MYERS_SUCCESS;
}

extern "C" int myersServerDestroy(myersServer_t* srv) {
  if (srv == nullptr) return MYERS_E_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->stop = true;
  }
  srv->cv_dispatch.notify_all();
  srv->cv_complete.notify_all();
  if (srv->dispatcher.joinable()) srv->dispatcher.join();
  srv->cv_complete.notify_all();
  if (srv->completer.joinable()) srv->completer.join();
  for (auto& kv : srv->live) delete kv.second;
  for (Request* r : srv->free_reqs) delete r;
  for (auto& s : srv->slots) slot_free(s);
  delete srv;
  return MYERS_SUCCESS;
}

extern "C" int myersServerReplay(myersServer_t* srv, const qryEntry_t* peq, const qryInfo_t* qinfo,
                                 const uint32_t* candOffset, const uint64_t* positions, uint32_t numRequests,
                                 const uint64_t* arrivalNs, uint64_t* latencyNs, resEntry_t* results,
                                 uint64_t* wallNs) {
  if (srv == nullptr || qinfo == nullptr || candOffset == nullptr || arrivalNs == nullptr || latencyNs == nullptr)
    return MYERS_E_INVALID_ARGUMENT;
  std::vector<uint64_t> tickets(numRequests, 0);
  std::vector<int> ok(numRequests, 0);
  {
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->live.reserve(srv->live.size() + numRequests);
  }
  const uint64_t t0 = now_ns() + 1000000;  // start 1 ms from now
  SubmitItem items[256];
  int st[256];
  for (uint32_t i = 0; i < numRequests;) {
    const uint64_t due = t0 + arrivalNs[i];
    uint64_t now = now_ns();
    while (now < due) now = now_ns();
    // every request already due goes in one round
    uint32_t n = 0;
    while (i + n < numRequests && n < 256 && t0 + arrivalNs[i + n] <= now) {
      const uint32_t q = i + n;
      items[n] = SubmitItem{peq + qinfo[q].posEntry, qinfo[q].size, positions + candOffset[q],
                            candOffset[q + 1] - candOffset[q]};
      ++n;
    }
    submit_many(srv, items, n, st, tickets.data() + i);
    for (uint32_t k = 0; k < n; ++k) ok[i + k] = st[k] == MYERS_SUCCESS;
    i += n;
  }
  uint64_t last = t0;
  int status = MYERS_SUCCESS;
  for (uint32_t i = 0; i < numRequests; ++i) {
    if (!ok[i]) {
      latencyNs[i] = UINT64_MAX;
      continue;
    }
    std::unique_lock<std::mutex> lk(srv->mu);
    Request* r = srv->live[tickets[i]];
    srv->cv_done.wait(lk, [&] { return r->state == kDone; });
    const uint64_t done = r->t_done;
    lk.unlock();
    latencyNs[i] = done - (t0 + arrivalNs[i]);
    if (done > last) last = done;
    const int st = take_result(srv, tickets[i], results ? results + candOffset[i] : nullptr, false, 0);
    if (st != MYERS_SUCCESS) status = st;
  }
  if (wallNs) *wallNs = last - (t0 + (numRequests ? arrivalNs[0] : 0));
  return status;
}
