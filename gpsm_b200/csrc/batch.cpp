// Batched and served matching: several engine slots on one device, each
// with its own stream and workspace, fed from one queue, so that the
// kernels of different queries overlap on the GPU and one query's host-side
// waits (a sync per join step) hide behind another's work.
//
//   gpsm_match_batch_parallel  - a fixed batch, slots take the next query as
//                                soon as they finish one (continuous batching)
//   gpsm_server_*              - a request loop: requests arrive at any time,
//                                wait for a free slot, run their filter and
//                                planning, and are admitted to the joins only
//                                when their predicted join memory fits the
//                                server's budget; latency is recorded per
//                                request (submit, start, end).
// The reference has neither: main/run.cpp matches one query after another
// and re-uploads the data graph for each (match/Match.cu:1714).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <stdexcept>
#include <thread>

#include "engine.h"
#include "learned.h"

namespace gpsm {

// One set of slots per (device, count, arena size); kept for the process.
struct SlotPool {
  int device = 0;
  uint64_t arena = 0;
  std::vector<Workspace*> ws;
};

static std::mutex g_pool_mu;
static std::vector<SlotPool*> g_pools;

// Workspace bytes per slot: the caller's figure, else GPSM_ARENA_GB (the same
// override the default engine reads), else half the free memory shared out,
// at most 16 GiB each.
uint64_t slot_arena_bytes(uint32_t slots, uint64_t per_slot) {
  if (per_slot) return per_slot;
  if (const char* e = getenv("GPSM_ARENA_GB")) return (uint64_t)(atof(e) * (double)(1ull << 30));
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 2ull << 30;
  return std::min<uint64_t>(16ull << 30, (uint64_t)(free_b * 0.5 / std::max<uint32_t>(slots, 1)));
}

// arena == 0: any existing pool of that many slots (its size was chosen from
// the free memory when it was created; later calls must not size a second
// pool from what the first one left free).
SlotPool* slot_pool(int device, uint32_t slots, uint64_t arena) {
  std::lock_guard<std::mutex> lk(g_pool_mu);
  for (SlotPool* p : g_pools)
    if (p->device == device && p->ws.size() == slots && (arena == 0 || p->arena == arena)) return p;
  if (arena == 0) arena = slot_arena_bytes(slots, 0);
  SlotPool* p = new SlotPool();
  p->device = device;
  p->arena = arena;
  for (uint32_t i = 0; i < slots; ++i) p->ws.push_back(workspace_create(device, arena, 1u << 20));
  g_pools.push_back(p);
  return p;
}


struct BatchOut {
  std::vector<uint64_t> rows;
  std::vector<int32_t> capped;
  std::vector<double> query_ms;
  std::vector<int> status;
  double device_ms = 0;
  uint64_t launches = 0, expand_launches = 0, alg_bytes = 0, join_steps = 0;
  double expand_ms = 0, filter_ms = 0;
  std::string first_msg;  // error text of the first failing query (set on a worker thread)
};

// Runs queries [0, nq) on the pool's slots. Device time of the batch is the
// span from the earliest slot's start event to the latest slot's end event.
// Slots take the queries largest first (query edges, then vertices; ties in
// batch order): a long query starts while the others still run instead of
// running alone at the end (longest-processing-time-first dispatch).
// Results stay indexed by the query's place in the batch.
int run_batch_parallel(SlotPool& pool, const DeviceGraph& g, uint32_t nq, const uint32_t* q_voff,
                       const uint32_t* q_labels, const uint64_t* q_eoff, const uint32_t* q_edges,
                       const MatchOptions& base, const int32_t* orders, BatchOut& out) {
  const uint32_t S = (uint32_t)pool.ws.size();
  out.rows.assign(nq, 0);
  out.capped.assign(nq, 0);
  out.query_ms.assign(nq, 0);
  out.status.assign(nq, GPSM_OK);
  std::vector<uint32_t> dispatch(nq);
  for (uint32_t k = 0; k < nq; ++k) dispatch[k] = k;
  std::stable_sort(dispatch.begin(), dispatch.end(), [&](uint32_t a, uint32_t b) {
    const uint64_t ma = q_eoff[a + 1] - q_eoff[a], mb = q_eoff[b + 1] - q_eoff[b];
    if (ma != mb) return ma > mb;
    return q_voff[a + 1] - q_voff[a] > q_voff[b + 1] - q_voff[b];
  });
  std::atomic<uint32_t> next(0);
  std::atomic<int> first_error(GPSM_OK);
  std::mutex agg_mu;
  std::vector<cudaEvent_t> e0(S), e1(S);
  for (uint32_t s = 0; s < S; ++s) {
    GPSM_CUDA(cudaSetDevice(pool.device));
    GPSM_CUDA(cudaEventCreate(&e0[s]));
    GPSM_CUDA(cudaEventCreate(&e1[s]));
  }
  auto worker = [&](uint32_t s) {
    cudaSetDevice(pool.device);
    Workspace& ws = *pool.ws[s];
    cudaEventRecord(e0[s], ws.stream);
    for (;;) {
      const uint32_t slot_k = next.fetch_add(1);
      if (slot_k >= nq) break;
      const uint32_t k = dispatch[slot_k];
      const uint32_t qn = q_voff[k + 1] - q_voff[k];
      const uint32_t qm = (uint32_t)(q_eoff[k + 1] - q_eoff[k]);
      int rc;
      MatchResult R;
      try {
        QueryPlan Q;
        std::string err;
        rc = plan_query(g, qn, q_labels + q_voff[k], qm, q_edges + 2 * q_eoff[k], Q, err);
        if (rc == GPSM_OK) {
          MatchOptions mo = base;
          if (orders) {
            mo.order_mode = ORDER_GIVEN;
            mo.given_order.assign(orders + q_voff[k], orders + q_voff[k + 1]);
          }
          rc = run_query(ws, g, Q, mo, R);
        } else {
          set_last_error("query " + std::to_string(k) + ": " + err);
        }
      } catch (const CudaError& e) {
        rc = e.err == cudaErrorMemoryAllocation ? GPSM_ERR_NOMEM : GPSM_ERR_CUDA;
      } catch (const std::bad_alloc&) {
        set_last_error("batch slot: host allocation failed");
        rc = GPSM_ERR_NOMEM;
      } catch (const std::exception& e) {
        set_last_error(std::string("batch slot: ") + e.what());
        rc = GPSM_ERR_CUDA;
      }
      out.status[k] = rc;
      if (rc != GPSM_OK) {
        int expected = GPSM_OK;
        if (first_error.compare_exchange_strong(expected, rc)) {
          std::lock_guard<std::mutex> lk(agg_mu);
          out.first_msg = "query " + std::to_string(k) + ": " + last_error();
        }
        continue;
      }
      out.rows[k] = R.rows;
      out.capped[k] = R.capped ? 1 : (R.stats.aborted ? 2 : 0);
      out.query_ms[k] = R.stats.device_ms;
      std::lock_guard<std::mutex> lk(agg_mu);
      out.launches += R.stats.filter_launches + R.stats.expand_launches;
      out.expand_launches += R.stats.expand_launches;
      out.join_steps += R.stats.join_steps;
      out.alg_bytes += R.stats.alg_bytes_join;
      out.expand_ms += R.stats.expand_ms;
      out.filter_ms += R.stats.filter_ms;
    }
    cudaEventRecord(e1[s], ws.stream);
    cudaEventSynchronize(e1[s]);
  };
  std::vector<std::thread> th;
  for (uint32_t s = 0; s < S; ++s) th.emplace_back(worker, s);
  for (auto& t : th) t.join();
  float span = 0.f;
  for (uint32_t a = 0; a < S; ++a)
    for (uint32_t b = 0; b < S; ++b) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, e0[a], e1[b]) == cudaSuccess && ms > span) span = ms;
    }
  out.device_ms = span;
  for (uint32_t s = 0; s < S; ++s) {
    cudaEventDestroy(e0[s]);
    cudaEventDestroy(e1[s]);
  }
  return first_error.load();
}

// ---------------------------------------------------------------------------
// request server
// ---------------------------------------------------------------------------
struct Request {
  uint64_t id = 0;
  uint32_t qn = 0, qm = 0;
  std::vector<uint32_t> lab, edges;
  double t_submit = 0, t_start = 0, t_admit = 0, t_end = 0;
  int status = 1;  // 1 = pending
  std::string err;  // error text of a failed request (set on the slot's thread)
  uint64_t rows = 0;
  int capped = 0;
  double device_ms = 0;
  uint64_t admitted_bytes = 0;
  HostRows result;  // rows (table-column order) when collect is on
  std::vector<int32_t> id2pos;
};

struct Server {
  const DeviceGraph* g = nullptr;
  std::vector<Workspace*> ws;
  std::vector<std::thread> threads;
  std::thread completer;  // publishes requests whose rows are still being copied
  std::mutex mu;
  std::condition_variable cv_q, cv_done, cv_mem, cv_drain;
  std::deque<Request*> queue;
  // requests whose joins are done and whose last row copies are still
  // running, with the event recorded after those copies (completion order)
  std::deque<std::pair<Request*, cudaEvent_t>> draining;
  bool slots_done = false;
  std::map<uint64_t, Request*> all;
  std::deque<uint64_t> finished;  // tickets in completion order (for wait_any)
  uint64_t next_id = 1;
  bool stopping = false;
  uint64_t budget = 0, in_use = 0, peak_in_use = 0;
  uint32_t active = 0;
  MatchOptions base;
  bool collect = false;
  bool largest_first = false;  // GPSM_F_LARGEST_FIRST
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

  // The next request for a free slot (mu held, queue not empty): the oldest,
  // or with largest_first the one with the most query edges, then vertices
  // (a long request started early does not run alone at the end).
  Request* take_next() {
    auto pick = queue.begin();
    if (largest_first)
      for (auto it = queue.begin(); it != queue.end(); ++it)
        if ((*it)->qm > (*pick)->qm || ((*it)->qm == (*pick)->qm && (*it)->qn > (*pick)->qn)) pick = it;
    Request* r = *pick;
    queue.erase(pick);
    return r;
  }

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }

  static bool admit_cb(void* ctx, uint64_t bytes) {
    auto* pr = static_cast<std::pair<Server*, Request*>*>(ctx);
    Server* S = pr->first;
    std::unique_lock<std::mutex> lk(S->mu);
    if (bytes > S->budget) bytes = S->budget;  // a request larger than the budget waits for an empty device
    // shutting down still drains the queue, so admission ignores `stopping`
    const bool ok =
        S->cv_mem.wait_for(lk, std::chrono::seconds(600), [&] { return S->in_use + bytes <= S->budget; });
    if (!ok) return false;
    S->in_use += bytes;
    S->peak_in_use = std::max(S->peak_in_use, S->in_use);
    pr->second->admitted_bytes = bytes;
    pr->second->t_admit = S->now_ms();
    return true;
  }
  static void release_cb(void* ctx, uint64_t bytes) {
    auto* pr = static_cast<std::pair<Server*, Request*>*>(ctx);
    Server* S = pr->first;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      const uint64_t b = pr->second->admitted_bytes ? pr->second->admitted_bytes : std::min(bytes, S->budget);
      S->in_use -= std::min(S->in_use, b);
    }
    S->cv_mem.notify_all();
  }

  void slot_loop(uint32_t s) {
    cudaSetDevice(ws[s]->device);
    for (;;) {
      Request* r = nullptr;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_q.wait(lk, [&] { return stopping || !queue.empty(); });
        if (queue.empty()) return;  // stopping and drained
        r = take_next();
        ++active;
        r->t_start = now_ms();
      }
      int rc;
      MatchResult R;
      std::pair<Server*, Request*> ctx(this, r);
      try {
        QueryPlan Q;
        std::string err;
        rc = plan_query(*g, r->qn, r->lab.data(), r->qm, r->edges.empty() ? nullptr : r->edges.data(), Q, err);
        if (rc == GPSM_OK) {
          MatchOptions mo = base;
          mo.admit = &Server::admit_cb;
          mo.release = &Server::release_cb;
          mo.admit_ctx = &ctx;
          mo.collect_rows = collect;
          mo.defer_copies = collect;
          rc = run_query(*ws[s], *g, Q, mo, R);
        } else {
          set_last_error(err);
        }
      } catch (const CudaError& e) {
        rc = e.err == cudaErrorMemoryAllocation ? GPSM_ERR_NOMEM : GPSM_ERR_CUDA;
      } catch (const std::bad_alloc&) {
        set_last_error("server slot: host allocation failed");
        rc = GPSM_ERR_NOMEM;
      } catch (const std::exception& e) {
        set_last_error(std::string("server slot: ") + e.what());
        rc = GPSM_ERR_CUDA;
      }
      if (R.copies_done && rc != GPSM_OK) {  // no request takes the rows: let the copies end here
        cudaEventSynchronize(R.copies_done);
        cudaEventDestroy(R.copies_done);
        R.copies_done = nullptr;
      }
      bool drain = false;
      {
        std::lock_guard<std::mutex> lk(mu);
        if (rc != GPSM_OK) r->err = last_error();
        r->rows = R.rows;
        r->capped = R.capped ? 1 : (R.stats.aborted ? 2 : 0);
        r->device_ms = R.stats.device_ms;
        if (collect && rc == GPSM_OK) {
          r->result = std::move(R.host_rows);
          r->id2pos = R.id2pos;
        }
        --active;
        if (R.copies_done) {
          // the slot takes its next request while the rows finish copying
          // (the next query's joins wait for them on the device)
          draining.emplace_back(r, R.copies_done);
          drain = true;
        } else {
          r->status = rc;
          r->t_end = now_ms();
          finished.push_back(r->id);
        }
      }
      if (drain) cv_drain.notify_one();
      else cv_done.notify_all();
    }
  }

  // Waits for each draining request's copies in turn and publishes it.
  void complete_loop(int device) {
    cudaSetDevice(device);
    for (;;) {
      std::pair<Request*, cudaEvent_t> d;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv_drain.wait(lk, [&] { return slots_done || !draining.empty(); });
        if (draining.empty()) return;  // the slots have stopped and nothing is left
        d = draining.front();
      }
      const cudaError_t e = cudaEventSynchronize(d.second);
      cudaEventDestroy(d.second);
      {
        std::lock_guard<std::mutex> lk(mu);
        draining.pop_front();
        Request* r = d.first;
        if (e != cudaSuccess) {
          r->status = GPSM_ERR_CUDA;
          r->err = std::string("copy of result rows: ") + cudaGetErrorString(e);
          r->result = HostRows();
        } else {
          r->status = GPSM_OK;
        }
        r->t_end = now_ms();
        finished.push_back(r->id);
      }
      cv_done.notify_all();
    }
  }
};

}  // namespace gpsm

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
#include "handles.h"

using namespace gpsm;

struct gpsm_server_s {
  Server* s;
};

extern "C" {

int gpsm_match_batch_parallel(gpsm_graph_t g, uint32_t nq, const uint32_t* q_voff, const uint32_t* q_labels,
                              const uint64_t* q_eoff, const uint32_t* q_edges, const gpsm_match_opts* opts,
                              const int32_t* orders, uint32_t slots, uint64_t slot_arena_bytes_in, uint64_t* counts,
                              int32_t* capped, double* query_ms, gpsm_batch_info* info) {
  if (!g || !q_voff || !q_labels || !q_eoff || slots == 0 || slots > 64) return GPSM_ERR_INVALID;
  try {
    // counts only: final rows are produced on the device and dropped once
    // counted, so the result buffer holds one step's output, not the cap
    MatchOptions base = options_from(opts);
    base.keep_on_device = false;
    base.collect_rows = false;
    SlotPool* pool = slot_pool(g->g->device, slots, slot_arena_bytes_in);
    BatchOut out;
    int rc = run_batch_parallel(*pool, *g->g, nq, q_voff, q_labels, q_eoff, q_edges, base,
                                (opts && opts->order_mode == GPSM_ORDER_GIVEN) ? orders : nullptr, out);
    if (rc != GPSM_OK) set_last_error(out.first_msg);
    for (uint32_t k = 0; k < nq; ++k) {
      if (counts) counts[k] = out.rows[k];
      if (capped) capped[k] = out.capped[k];
      if (query_ms) query_ms[k] = out.query_ms[k];
    }
    if (info) {
      memset(info, 0, sizeof(*info));
      info->device_ms = out.device_ms;
      info->expand_ms = out.expand_ms;
      info->filter_ms = out.filter_ms;
      for (uint32_t k = 0; k < nq; ++k) info->rows += out.rows[k];
      info->launches = out.launches;
      info->expand_launches = out.expand_launches;
      info->join_steps = out.join_steps;
      info->alg_bytes_join = out.alg_bytes;
    }
    return rc;
  } catch (const CudaError& e) {
    return error_from(e);
  }
}

int gpsm_server_create(gpsm_graph_t g, uint32_t slots, uint64_t memory_budget, uint64_t slot_arena,
                       const gpsm_match_opts* opts, int32_t collect_rows, gpsm_server_t* out) {
  if (!g || !out || slots == 0 || slots > 64) return GPSM_ERR_INVALID;
  try {
    Server* S = new Server();
    S->g = g->g;
    S->base = options_from(opts);
    S->collect = collect_rows != 0;
    S->largest_first = opts && (opts->flags & GPSM_F_LARGEST_FIRST) != 0;
    S->base.keep_on_device = !S->collect;
    if (!S->collect && S->base.cap != ~0ULL) S->base.result_rows = std::max<uint64_t>(S->base.result_rows, S->base.cap);
    const uint64_t arena = slot_arena_bytes(slots, slot_arena);
    for (uint32_t i = 0; i < slots; ++i) S->ws.push_back(workspace_create(g->g->device, arena, 1u << 20));
    S->budget = memory_budget ? memory_budget : arena * slots;
    for (uint32_t i = 0; i < slots; ++i) S->threads.emplace_back(&Server::slot_loop, S, i);
    S->completer = std::thread(&Server::complete_loop, S, g->g->device);
    gpsm_server_s* h = new gpsm_server_s();
    h->s = S;
    *out = h;
    return GPSM_OK;
  } catch (const CudaError& e) {
    return error_from(e);
  }
}

// Copies the query and queues it; returns at once with a ticket.
int gpsm_server_submit(gpsm_server_t h, uint32_t qn, const uint32_t* q_labels, uint32_t qm, const uint32_t* q_edges,
                       uint64_t* ticket) {
  if (!h || !q_labels || qn == 0 || (qm && !q_edges)) return GPSM_ERR_INVALID;
  Server* S = h->s;
  Request* r = new Request();
  r->qn = qn;
  r->qm = qm;
  r->lab.assign(q_labels, q_labels + qn);
  if (qm) r->edges.assign(q_edges, q_edges + 2 * (size_t)qm);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stopping) {
      delete r;
      return GPSM_ERR_STATE;
    }
    r->id = S->next_id++;
    r->t_submit = S->now_ms();
    S->all[r->id] = r;
    S->queue.push_back(r);
    if (ticket) *ticket = r->id;
  }
  S->cv_q.notify_one();
  return GPSM_OK;
}

// Waits for a request (timeout_s < 0: forever); fills info and, when the
// server collects rows and rows != NULL, a malloc'd copy of its rows
// (free with gpsm_free) and its id_map (qn entries).
// Hands a finished request to the caller and forgets it (S->mu held).
static int collect_request(Server* S, std::map<uint64_t, Request*>::iterator it, gpsm_request_info* info,
                           uint32_t** rows, int32_t* id_map) {
  Request* r = it->second;
  if (info) {
    memset(info, 0, sizeof(*info));
    info->status = r->status;
    info->rows = r->rows;
    info->capped = r->capped;
    info->submit_ms = r->t_submit;
    info->start_ms = r->t_start;
    info->admit_ms = r->t_admit;
    info->end_ms = r->t_end;
    info->device_ms = r->device_ms;
    info->admitted_bytes = r->admitted_bytes;
  }
  if (rows) *rows = r->result.empty() ? nullptr : r->result.release();  // the caller frees it
  if (id_map)
    for (uint32_t i = 0; i < r->qn; ++i) id_map[i] = i < r->id2pos.size() ? r->id2pos[i] : -1;
  const int st = r->status;
  if (st != GPSM_OK) set_last_error(r->err);  // the failing slot thread's text, on the caller's thread
  S->all.erase(it);
  delete r;
  return st;
}

int gpsm_server_wait(gpsm_server_t h, uint64_t ticket, double timeout_s, gpsm_request_info* info, uint32_t** rows,
                     int32_t* id_map) {
  if (!h) return GPSM_ERR_INVALID;
  Server* S = h->s;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->all.find(ticket);
  if (it == S->all.end()) return GPSM_ERR_INVALID;
  Request* r = it->second;
  auto done = [&] { return r->status != 1; };
  if (timeout_s < 0) S->cv_done.wait(lk, done);
  else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), done)) return GPSM_ERR_TIMEOUT;
  return collect_request(S, it, info, rows, id_map);
}

int gpsm_server_wait_any(gpsm_server_t h, double timeout_s, uint64_t* ticket, gpsm_request_info* info,
                         uint32_t** rows, int32_t* id_map) {
  if (!h || !ticket) return GPSM_ERR_INVALID;
  Server* S = h->s;
  std::unique_lock<std::mutex> lk(S->mu);
  // finished tickets already collected by gpsm_server_wait are skipped
  auto ready = [&] {
    while (!S->finished.empty() && !S->all.count(S->finished.front())) S->finished.pop_front();
    return !S->finished.empty() || S->all.empty();
  };
  if (timeout_s < 0) S->cv_done.wait(lk, ready);
  else if (!S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) return GPSM_ERR_TIMEOUT;
  if (S->finished.empty()) {
    set_last_error("gpsm_server_wait_any: no request outstanding");
    return GPSM_ERR_STATE;
  }
  *ticket = S->finished.front();
  S->finished.pop_front();
  return collect_request(S, S->all.find(*ticket), info, rows, id_map);
}

int gpsm_server_stats(gpsm_server_t h, uint64_t* in_use, uint64_t* peak_in_use, uint64_t* budget, uint32_t* queued,
                      uint32_t* active) {
  if (!h) return GPSM_ERR_INVALID;
  Server* S = h->s;
  std::lock_guard<std::mutex> lk(S->mu);
  if (in_use) *in_use = S->in_use;
  if (peak_in_use) *peak_in_use = S->peak_in_use;
  if (budget) *budget = S->budget;
  if (queued) *queued = (uint32_t)S->queue.size();
  if (active) *active = S->active;
  return GPSM_OK;
}

// Finishes every queued request, then stops the slots and frees them.
int gpsm_server_destroy(gpsm_server_t h) {
  if (!h) return GPSM_ERR_INVALID;
  Server* S = h->s;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stopping = true;
  }
  S->cv_q.notify_all();
  S->cv_mem.notify_all();
  for (auto& t : S->threads) t.join();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->slots_done = true;
  }
  S->cv_drain.notify_all();
  S->completer.join();  // every draining request is published first
  for (Workspace* w : S->ws) workspace_free(w);
  for (auto& kv : S->all) delete kv.second;
  delete S;
  delete h;
  return GPSM_OK;
}

}  // extern "C"
