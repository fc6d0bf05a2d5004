// Continuous-batching answer service over one server handle (via_service_* in
// include/via_gpu.h). The reference answers one query per Server::answer call
// (crates/via-server/src/answer.rs:534) or one VIA-B batch per answer_batch
// (srv/batch.rs:72-163); this layer is the serving loop around those calls.
//
// Requests queue on the host. A worker thread owns `lanes` device lanes, each a
// workspace, a stream and pinned staging buffers. Whenever a lane is free and
// requests are pending, the worker takes up to the lane's capacity of them
// (capacity = the largest batch whose workspace fits the HBM budget share of
// one lane, capped by max_batch) and enqueues upload, the batched answer (one
// database scan for the whole batch) and download on the lane's stream. Lanes
// run concurrently, so a batch admitted while others are on the GPU overlaps
// with them. Completion is polled with cudaEventQuery: no host thread blocks in
// the driver, and every wait the API offers has a time limit.
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

#include "server.cuh"

namespace via {

namespace {

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

struct Request {
  u64 ticket = 0;
  std::vector<u64> query;  // units of query_lwes(p) LWEs (one, or T for VIA-B)
  std::vector<u64> mask, body;
  double t_submit = 0, t_done = 0;
  int state = 0;  // 0 pending, 1 on the GPU, 2 done, 3 failed
  via_status status = VIA_OK;
  std::string error;
};

struct Lane {
  std::unique_ptr<Workspace, WorkspaceDeleter> ws;
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  u64* h_in = nullptr;   // pinned: cap units of queries
  u64* h_mask = nullptr;  // pinned: cap answers
  u64* h_body = nullptr;
  int* h_err = nullptr;  // pinned copy of the scan's error word
  std::unique_ptr<DevBuf> d_in;  // VIA-B requests larger than the workspace: their queries, answered in chunks
  int cap = 0;
  bool busy = false;
  std::vector<Request*> batch;
};

}  // namespace

struct Service {
  Server* s = nullptr;
  via_service_config cfg{};
  bool via_b = false;
  std::vector<via_scan_tuning> tuning;  // the autotuner's choices at creation
  size_t unit_len = 0;  // u64 per request (one query, or T queries)
  std::vector<Lane> lanes;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> pending;
  std::unordered_map<u64, std::unique_ptr<Request>> reqs;
  u64 next_ticket = 1;
  bool stop = false;
  std::thread worker;
  // Statistics.
  u64 submitted = 0, completed = 0, failed = 0, batches = 0, units = 0;
  uint32_t max_in_flight = 0;
  std::vector<double> latencies;
  double t_first = 0, t_last = 0;

  ~Service();
  void run();
  void launch(Lane& L);
  void finish(Lane& L, cudaError_t e);
};

Service::~Service() {
  {
    std::lock_guard<std::mutex> lk(mu);
    stop = true;
  }
  cv_work.notify_all();
  if (worker.joinable()) worker.join();
  for (auto& L : lanes) {
    if (L.stream) cudaStreamSynchronize(L.stream);
    if (L.done) cudaEventDestroy(L.done);
    if (L.stream) cudaStreamDestroy(L.stream);
    cudaFreeHost(L.h_in);
    cudaFreeHost(L.h_mask);
    cudaFreeHost(L.h_body);
    cudaFreeHost(L.h_err);
    L.ws.reset();
  }
}

// Called with mu held: moves up to cap pending requests onto lane L and enqueues them.
void Service::launch(Lane& L) {
  const via_params& p = s->prm;
  const int n = std::min<int>(L.cap, (int)pending.size());
  L.batch.clear();
  for (int i = 0; i < n; ++i) {
    Request* r = pending.front();
    pending.pop_front();
    r->state = 1;
    std::memcpy(L.h_in + (size_t)i * unit_len, r->query.data(), unit_len * 8);
    L.batch.push_back(r);
  }
  try {
    std::shared_lock<std::shared_mutex> plan(s->plan_mu);  // the scan tiles stay fixed while this batch is enqueued
    u64* d_in = L.d_in ? L.d_in->p : ws_query(*L.ws);
    VIA_CUDA(cudaMemcpyAsync(d_in, L.h_in, (size_t)n * unit_len * 8, cudaMemcpyHostToDevice, L.stream));
    if (via_b)
      answer_batch_device(*s, *L.ws, d_in, n, ws_answer_mask(*L.ws), ws_answer_body(*L.ws), L.stream);
    else
      answer_graph(*s, *L.ws, n, L.stream);
    VIA_CUDA(cudaMemcpyAsync(L.h_mask, ws_answer_mask(*L.ws), (size_t)n * p.n2 * 8, cudaMemcpyDeviceToHost, L.stream));
    VIA_CUDA(cudaMemcpyAsync(L.h_body, ws_answer_body(*L.ws), (size_t)n * p.n2 * 8, cudaMemcpyDeviceToHost, L.stream));
    if (s->fd_err.p) VIA_CUDA(cudaMemcpyAsync(L.h_err, s->fd_err.p, sizeof(int), cudaMemcpyDeviceToHost, L.stream));
    VIA_CUDA(cudaEventRecord(L.done, L.stream));
    L.busy = true;
    ++batches;
    units += (u64)n;
    uint32_t busy = 0;
    for (auto& o : lanes) busy += o.busy ? 1 : 0;
    max_in_flight = std::max(max_in_flight, busy);
  } catch (const std::exception& e) {
    for (Request* r : L.batch) {
      r->state = 3;
      r->status = VIA_ERR_CUDA;
      r->error = e.what();
      ++failed;
    }
    L.batch.clear();
    cv_done.notify_all();
  }
}

// Called with mu held once lane L's event has completed (or failed with e).
void Service::finish(Lane& L, cudaError_t e) {
  const via_params& p = s->prm;
  const double t = now_ms();
  const bool timeout = e == cudaSuccess && *L.h_err != 0;
  for (size_t i = 0; i < L.batch.size(); ++i) {
    Request* r = L.batch[i];
    if (e != cudaSuccess || timeout) {
      r->state = 3;
      r->status = timeout ? VIA_ERR_TIMEOUT : VIA_ERR_CUDA;
      r->error = timeout ? "FirstDim scan: a bounded device wait ran out" : cudaGetErrorString(e);
      ++failed;
      continue;
    }
    r->mask.assign(L.h_mask + i * p.n2, L.h_mask + (i + 1) * p.n2);
    r->body.assign(L.h_body + i * p.n2, L.h_body + (i + 1) * p.n2);
    r->t_done = t;
    r->state = 2;
    ++completed;
    latencies.push_back(t - r->t_submit);
    t_last = t;
  }
  L.batch.clear();
  L.busy = false;
  cv_done.notify_all();
}

void Service::run() {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lk(mu);
  while (true) {
    bool any_busy = false;
    for (auto& L : lanes) {
      if (!L.busy) continue;
      cudaError_t e = cudaEventQuery(L.done);
      if (e == cudaErrorNotReady) {
        any_busy = true;
        continue;
      }
      finish(L, e);
    }
    if (stop && !any_busy) break;
    if (!stop)
      for (auto& L : lanes)
        if (!L.busy && !pending.empty()) {
          launch(L);
          any_busy = any_busy || L.busy;
        }
    if (any_busy) {
      // Poll the in-flight lanes again shortly; a new request also wakes us.
      cv_work.wait_for(lk, std::chrono::microseconds(50));
    } else if (!stop) {
      cv_work.wait_for(lk, std::chrono::milliseconds(5), [&] { return stop || !pending.empty(); });
    }
  }
}

}  // namespace via

using namespace via;

struct via_service : via::Service {};

static via_status fail(via_status code, const std::string& msg) {
  set_last_error(msg);
  return code;
}

extern "C" {

via_status via_service_create(via_server* s, const via_service_config* cfg, via_service** out) {
  if (!s || !out) return fail(VIA_ERR_INVALID_ARGUMENT, "via_service_create: null argument");
  *out = nullptr;
  try {
    std::unique_ptr<via_service> v(new via_service());
    v->s = s;
    if (cfg) v->cfg = *cfg;
    via_service_config& c = v->cfg;
    if (c.lanes == 0) c.lanes = 2;
    if (c.max_batch == 0) c.max_batch = 64;
    if (c.max_pending == 0) c.max_pending = 1u << 20;
    if (c.lanes > 16 || c.max_batch > 4096)
      return fail(VIA_ERR_INVALID_ARGUMENT, "via_service_create: lanes must be <= 16 and max_batch <= 4096");
    const via_params& p = s->prm;
    if (!s->cascade_eval.p) return fail(VIA_ERR_SETUP_NOT_COMPLETE, "server has no public keys");
    v->via_b = via_b_batch(p) >= 2;
    const int T = v->via_b ? via_b_batch(p) : 1;
    v->unit_len = (size_t)T * query_lwes(p) * lwe_len(p);
    VIA_CUDA(cudaSetDevice(s->device));
    // Admission: each lane's workspace holds `qcap` queries, the most whose
    // device memory fits the lane's share of the HBM budget (up to max_batch
    // requests). A lane batch is cap = qcap / T requests; a VIA-B request
    // larger than the workspace (T > qcap) runs alone, its prefix in chunks of
    // qcap queries, with its T queries held in a separate device buffer.
    const size_t qbytes = (size_t)query_lwes(p) * lwe_len(p) * 8;
    auto lane_bytes = [&](int q) { return workspace_bytes(*s, q) + (q < T ? (size_t)T * qbytes : 0); };
    int qcap = (int)c.max_batch * T;
    if (v->via_b && !c.hbm_budget && T > VIA_B_CHUNK) qcap = VIA_B_CHUNK;
    if (c.hbm_budget) {
      const size_t share = c.hbm_budget / c.lanes;
      if (lane_bytes(1) > share)
        return fail(VIA_ERR_OUT_OF_MEMORY, "via_service_create: hbm_budget / lanes = " + std::to_string(share) +
                                               " bytes is below one query's workspace (" +
                                               std::to_string(lane_bytes(1)) + " bytes)");
      int lo = 1, hi = qcap;  // device bytes grow with the batch: largest fitting query count
      while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (lane_bytes(mid) <= share) lo = mid;
        else hi = mid - 1;
      }
      qcap = lo;
    }
    const int cap = std::max(1, qcap / T);
    if (qcap >= T) qcap = cap * T;
    v->lanes.resize(c.lanes);
    bool tuned = false;
    for (auto& L : v->lanes) {
      L.cap = cap;
      L.ws = workspace_make(*s, qcap);
      if (qcap < T) L.d_in.reset(new DevBuf((size_t)T * qbytes / 8));
      if (c.autotune && !tuned) {  // on the first lane's workspace, before any graph is captured
        std::vector<int> sizes;
        const int top = std::min(qcap, cap * T);
        for (int n = T; n < top; n *= 2) sizes.push_back(n);
        sizes.push_back(top);
        std::lock_guard<std::mutex> g(s->mu);
        autotune_scan(*s, *L.ws, sizes, c.tune_cache, &v->tuning);
        tuned = true;
      }
      VIA_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
      VIA_CUDA(cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming));
      VIA_CUDA(cudaHostAlloc((void**)&L.h_in, (size_t)cap * v->unit_len * 8, cudaHostAllocDefault));
      VIA_CUDA(cudaHostAlloc((void**)&L.h_mask, (size_t)cap * p.n2 * 8, cudaHostAllocDefault));
      VIA_CUDA(cudaHostAlloc((void**)&L.h_body, (size_t)cap * p.n2 * 8, cudaHostAllocDefault));
      VIA_CUDA(cudaHostAlloc((void**)&L.h_err, sizeof(int), cudaHostAllocDefault));
      *L.h_err = 0;
      if (c.warm && !v->via_b)  // capture the answer graph of every batch size now, not on first use
        for (int n = 1; n <= cap; ++n) answer_graph(*s, *L.ws, n, nullptr);
    }
    via_service* raw = v.get();
    v->worker = std::thread([raw] { raw->run(); });
    *out = v.release();
    return VIA_OK;
  } catch (const CudaError& e) {
    return fail(e.status == 101 ? VIA_ERR_OUT_OF_MEMORY : VIA_ERR_CUDA, e.what());
  } catch (const std::bad_alloc&) {
    return fail(VIA_ERR_OUT_OF_MEMORY, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(VIA_ERR_CUDA, e.what());
  }
}

uint64_t via_service_latencies(via_service* v, double* out, uint64_t cap) {
  if (!v) return 0;
  std::lock_guard<std::mutex> lk(v->mu);
  if (out)
    for (uint64_t i = 0; i < std::min<uint64_t>(cap, v->latencies.size()); ++i) out[i] = v->latencies[i];
  return v->latencies.size();
}

uint64_t via_service_tuning(via_service* v, via_scan_tuning* out, uint64_t cap) {
  if (!v) return 0;
  if (out)
    for (uint64_t i = 0; i < std::min<uint64_t>(cap, v->tuning.size()); ++i) out[i] = v->tuning[i];
  return v->tuning.size();
}

via_status via_service_submit(via_service* v, const uint64_t* query, uint64_t n_lwe, uint64_t* ticket) {
  if (!v || !query || !ticket) return fail(VIA_ERR_INVALID_ARGUMENT, "via_service_submit: null argument");
  const via_params& p = v->s->prm;
  if (n_lwe != query_lwes(p))
    return fail(VIA_ERR_QUERY_LENGTH_MISMATCH, "query length mismatch: expected " + std::to_string(query_lwes(p)) +
                                                   " ciphertexts, got " + std::to_string(n_lwe));
  auto r = std::make_unique<Request>();
  r->query.assign(query, query + v->unit_len);
  {
    std::lock_guard<std::mutex> lk(v->mu);
    if (v->pending.size() >= v->cfg.max_pending) return fail(VIA_ERR_BUSY, "via_service_submit: queue is full");
    r->ticket = v->next_ticket++;
    r->t_submit = now_ms();
    if (v->submitted == 0) v->t_first = r->t_submit;
    ++v->submitted;
    *ticket = r->ticket;
    v->pending.push_back(r.get());
    v->reqs.emplace(r->ticket, std::move(r));
  }
  v->cv_work.notify_one();
  return VIA_OK;
}

// Copies a finished request's answer out and forgets it.
static via_status take(via_service* v, std::unordered_map<u64, std::unique_ptr<Request>>::iterator it,
                       uint64_t* out_mask, uint64_t* out_body) {
  Request* r = it->second.get();
  via_status st = r->state == 2 ? VIA_OK : r->status;
  if (st != VIA_OK) set_last_error(r->error);
  if (r->state == 2) {
    std::memcpy(out_mask, r->mask.data(), r->mask.size() * 8);
    std::memcpy(out_body, r->body.data(), r->body.size() * 8);
  }
  v->reqs.erase(it);
  return st;
}

via_status via_service_poll(via_service* v, uint64_t ticket, uint64_t* out_mask, uint64_t* out_body, int* done) {
  if (!v || !out_mask || !out_body || !done) return VIA_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(v->mu);
  auto it = v->reqs.find(ticket);
  if (it == v->reqs.end()) return fail(VIA_ERR_INVALID_ARGUMENT, "unknown ticket");
  *done = it->second->state >= 2;
  if (!*done) return VIA_OK;
  return take(v, it, out_mask, out_body);
}

via_status via_service_wait(via_service* v, uint64_t ticket, uint64_t* out_mask, uint64_t* out_body,
                            uint32_t timeout_ms) {
  if (!v || !out_mask || !out_body) return VIA_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(v->mu);
  auto it = v->reqs.find(ticket);
  if (it == v->reqs.end()) return fail(VIA_ERR_INVALID_ARGUMENT, "unknown ticket");
  Request* r = it->second.get();
  if (!v->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return r->state >= 2; }))
    return fail(VIA_ERR_TIMEOUT, "via_service_wait: the request is not done yet");
  return take(v, v->reqs.find(ticket), out_mask, out_body);
}

via_status via_service_stats_get(via_service* v, via_service_stats* out) {
  if (!v || !out) return VIA_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(v->mu);
  std::memset(out, 0, sizeof(*out));
  out->submitted = v->submitted;
  out->completed = v->completed;
  out->failed = v->failed;
  out->batches = v->batches;
  out->units = v->units;
  out->lanes = (uint32_t)v->lanes.size();
  out->batch_cap = v->lanes.empty() ? 0 : (uint32_t)v->lanes[0].cap;
  out->max_in_flight = v->max_in_flight;
  out->mean_batch = v->batches ? (double)v->units / (double)v->batches : 0.0;
  if (!v->latencies.empty()) {
    std::vector<double> l = v->latencies;
    auto pct = [&](double q) {
      size_t k = (size_t)std::min<double>((double)l.size() - 1, q * (double)(l.size() - 1) + 0.5);
      std::nth_element(l.begin(), l.begin() + (long)k, l.end());
      return l[k];
    };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    const double span = v->t_last - v->t_first;
    out->answers_per_s = span > 0 ? (double)v->completed * 1e3 / span : 0.0;
  }
  return VIA_OK;
}

void via_service_destroy(via_service* v) { delete v; }

via_status via_service_stats_reset(via_service* v) {
  if (!v) return fail(VIA_ERR_INVALID_ARGUMENT, "null argument");
  std::lock_guard<std::mutex> lk(v->mu);
  v->submitted = v->completed = v->failed = v->batches = v->units = 0;
  v->max_in_flight = 0;
  v->latencies.clear();
  v->t_first = v->t_last = 0;
  return VIA_OK;
}

uint64_t via_server_workspace_bytes(via_server* s, uint64_t max_queries) {
  if (!s || max_queries == 0 || max_queries > (1u << 20)) return 0;
  return workspace_bytes(*s, (int)max_queries);
}

}  // extern "C"
