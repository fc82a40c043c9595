// extern "C" entry points of libgpsm.so (declared in include/gpsm.h).
//
// Each entry point catches every error and returns a status code; the
// reference instead exits the process on any CUDA error
// (match/Match.h:53-65) and on a missing device (match/Match.cu:20-23).
#include <cuda_runtime.h>

#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>

#include "engine.h"
#include "learned.h"

using namespace gpsm;

#include "handles.h"

namespace {

std::mutex g_mu;
int g_device = -1;
gpsm_engine_s* g_default = nullptr;

int map_error(const CudaError& e) {
  if (e.err == cudaErrorMemoryAllocation) return GPSM_ERR_NOMEM;
  if (e.err == cudaErrorInvalidValue) return GPSM_ERR_INVALID;
  return GPSM_ERR_CUDA;
}

template <class F>
int guarded(F f) {
  try {
    return f();
  } catch (const CudaError& e) {
    return map_error(e);
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return GPSM_ERR_NOMEM;
  } catch (...) {
    set_last_error("unexpected exception");
    return GPSM_ERR_STATE;
  }
}

uint64_t default_arena_bytes() {
  const char* e = getenv("GPSM_ARENA_GB");
  if (e) return (uint64_t)(atof(e) * (double)(1ull << 30));
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 4ull << 30;
  uint64_t want = 16ull << 30;
  return std::min<uint64_t>(want, (uint64_t)(free_b * 0.6));
}

gpsm_engine_s* engine_or_default(gpsm_engine_t e) { return e ? e : g_default; }

}  // namespace

MatchOptions gpsm::options_from(const gpsm_match_opts* o) {
  MatchOptions m;
  if (!o) return m;
  m.cap = o->cap ? o->cap : ~0ULL;
  if (o->order_mode == GPSM_ORDER_GIVEN) {
    m.order_mode = ORDER_GIVEN;
  }
  if (o->level_bytes) m.level_bytes = o->level_bytes;
  if (o->result_rows) m.result_rows = o->result_rows;
  m.keep_on_device = (o->flags & GPSM_F_KEEP_ON_DEVICE) != 0;
  m.collect_rows = (o->flags & GPSM_F_COUNT_ONLY) == 0;
  if (o->order_mode == GPSM_ORDER_LEARNED) {
    m.order_mode = ORDER_LEARNED;
    m.model = o->model ? o->model->m : nullptr;
  }
  m.memory_budget = o->memory_budget;
  m.work_cap = o->work_cap;
  m.directed = (o->flags & GPSM_F_DIRECTED) != 0;
  return m;
}

int gpsm::error_from(const CudaError& e) {
  if (e.err == cudaErrorMemoryAllocation) return GPSM_ERR_NOMEM;
  if (e.err == cudaErrorInvalidValue) return GPSM_ERR_INVALID;
  return GPSM_ERR_CUDA;
}

namespace {

MatchOptions to_options(const gpsm_match_opts* o) { return options_from(o); }

void fill_info(const MatchResult& R, gpsm_match_info* info) {
  if (!info) return;
  memset(info, 0, sizeof(*info));
  info->rows = R.rows;
  info->cols = R.cols;
  info->capped = R.capped ? 1 : 0;
  info->empty_filter = R.empty_filter ? 1 : 0;
  info->device_ms = R.stats.device_ms;
  info->filter_ms = R.stats.filter_ms;
  info->join_ms = R.stats.join_ms;
  info->expand_launches = R.stats.expand_launches;
  info->filter_launches = R.stats.filter_launches;
  info->alg_bytes_join = R.stats.alg_bytes_join;
  info->expand_ms = R.stats.expand_ms;
  info->plan_ms = R.stats.plan_ms;
  info->predicted_work = R.stats.predicted_work;
  info->predicted_peak = R.stats.predicted_peak;
  info->order_fallback = R.stats.order_fallback;
  info->aborted = R.stats.aborted ? 1 : 0;
  info->predicted_work_plain = R.stats.predicted_work_plain;
  info->order_attempts = R.stats.order_attempts;
  info->cands_scanned = R.stats.cands_scanned;
  info->cut_steps = R.stats.cut_steps;
}

}  // namespace

extern "C" {

const char* gpsm_last_error(void) { return last_error(); }

int gpsm_init_ex(int dev, uint64_t arena_bytes) {
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(g_mu);
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      set_last_error("no CUDA device");
      return GPSM_ERR_NODEV;
    }
    if (dev < 0 || dev >= count) {
      set_last_error("device index out of range");
      return GPSM_ERR_INVALID;
    }
    if (g_default && g_device == dev) return GPSM_OK;
    if (g_default) {
      workspace_free(g_default->ws);
      delete g_default;
      g_default = nullptr;
    }
    GPSM_CUDA(cudaSetDevice(dev));
    gpsm_engine_s* e = new gpsm_engine_s();
    e->ws = workspace_create(dev, arena_bytes ? arena_bytes : default_arena_bytes(), 1u << 20);
    g_default = e;
    g_device = dev;
    return GPSM_OK;
  });
}

int gpsm_init(int dev) { return gpsm_init_ex(dev, 0); }

int gpsm_shutdown(void) {
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_default) {
      workspace_free(g_default->ws);
      delete g_default;
      g_default = nullptr;
    }
    g_device = -1;
    return GPSM_OK;
  });
}

int gpsm_engine_create(int dev, uint64_t arena_bytes, gpsm_engine_t* out) {
  if (!out) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    GPSM_CUDA(cudaSetDevice(dev));
    gpsm_engine_s* e = new gpsm_engine_s();
    e->ws = workspace_create(dev, arena_bytes ? arena_bytes : default_arena_bytes(), 1u << 20);
    *out = e;
    return GPSM_OK;
  });
}

int gpsm_engine_destroy(gpsm_engine_t e) {
  if (!e) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    workspace_free(e->ws);
    delete e;
    return GPSM_OK;
  });
}

int gpsm_graph_upload(const uint32_t* offsets, const uint32_t* cols, const uint32_t* labels, uint32_t n,
                      gpsm_graph_t* out) {
  if (!out) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    if (g_device < 0) {
      set_last_error("gpsm_init was not called");
      return GPSM_ERR_STATE;
    }
    if (n == 0 || !offsets || !labels) {
      set_last_error("empty data graph");
      return GPSM_ERR_INVALID;
    }
    gpsm_graph_s* h = new gpsm_graph_s();
    h->g = graph_upload(g_device, offsets, cols, labels, n);
    *out = h;
    return GPSM_OK;
  });
}

int gpsm_graph_free(gpsm_graph_t g) {
  if (!g) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    graph_free(g->g);
    delete g;
    return GPSM_OK;
  });
}

int gpsm_graph_build(const uint32_t* edges, uint64_t m, const uint32_t* labels, uint32_t n, gpsm_graph_t* out) {
  if (!out) return GPSM_ERR_INVALID;
  gpsm_engine_s* e = g_default;
  if (!e) {
    set_last_error("gpsm_init was not called");
    return GPSM_ERR_STATE;
  }
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(e->mu);
    gpsm_graph_s* h = new gpsm_graph_s();
    h->g = graph_build(*e->ws, edges, m, labels, n);
    *out = h;
    return GPSM_OK;
  });
}

int gpsm_graph_download(gpsm_graph_t g, uint32_t* offsets, uint32_t* cols) {
  if (!g) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    graph_download(g->g, offsets, cols);
    return GPSM_OK;
  });
}

int gpsm_graph_set_directed(gpsm_graph_t g, uint64_t m, const uint32_t* edges, const uint32_t* labels) {
  if (!g || (m && !edges)) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    graph_set_directed(g->g, m, edges, labels);
    return GPSM_OK;
  });
}

int gpsm_graph_info(gpsm_graph_t g, uint32_t* n, uint64_t* nnz, uint32_t* max_degree) {
  if (!g) return GPSM_ERR_INVALID;
  if (n) *n = g->g->n;
  if (nnz) *nnz = g->g->nnz;
  if (max_degree) *max_degree = g->g->max_degree;
  return GPSM_OK;
}

int gpsm_graph_edge_table(gpsm_graph_t g, uint64_t* slots, uint32_t* max_probe) {
  if (!g) return GPSM_ERR_INVALID;
  if (slots) *slots = g->g->ehash ? (1ull << g->g->ehash_bits) : 0;
  if (max_probe) *max_probe = g->g->ehash ? g->g->ehash_probe : 0;
  return GPSM_OK;
}

int gpsm_engine_match(gpsm_engine_t eng, gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm,
                      const uint32_t* q_edges, const gpsm_match_opts* opts, uint32_t** out_rows, int32_t* id_map,
                      int32_t* pos2id, gpsm_match_info* info) {
  gpsm_engine_s* e = engine_or_default(eng);
  if (!e || !g) {
    set_last_error(!e ? "gpsm_init was not called" : "null graph");
    return !e ? GPSM_ERR_STATE : GPSM_ERR_INVALID;
  }
  if (out_rows) *out_rows = nullptr;
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(e->mu);
    QueryPlan Q;
    std::string err;
    int rc = plan_query(*g->g, qn, q_labels, qm, q_edges, Q, err);
    if (rc != GPSM_OK) {
      set_last_error(err);
      return rc;
    }
    MatchOptions mo = to_options(opts);
    if (mo.order_mode == ORDER_GIVEN) {
      if (!opts->order) {
        set_last_error("order_mode GIVEN without an order");
        return GPSM_ERR_INVALID;
      }
      mo.given_order.assign(opts->order, opts->order + qn);
    }
    if (!out_rows) mo.collect_rows = false;
    if (mo.directed && opts && opts->edge_labels) mo.edge_labels.assign(opts->edge_labels, opts->edge_labels + qm);
    if (mo.keep_on_device) mo.result_rows = std::max<uint64_t>(mo.result_rows, mo.cap == ~0ULL ? 0 : mo.cap);
    MatchResult R;
    rc = run_query(*e->ws, *g->g, Q, mo, R);
    if (rc != GPSM_OK) return rc;
    if (id_map)
      for (uint32_t i = 0; i < qn; ++i) id_map[i] = R.id2pos.empty() ? -1 : R.id2pos[i];
    if (pos2id)
      for (uint32_t i = 0; i < qn; ++i) pos2id[i] = R.pos2id.empty() ? -1 : R.pos2id[i];
    fill_info(R, info);
    if (out_rows && mo.collect_rows) {
      // rows still on the device follow the flushed ones; the caller takes
      // the host block itself
      if (R.d_rows && R.d_rows_count) R.host_rows.append_from_device(*e->ws, R.d_rows, R.d_rows_count * qn);
      R.d_rows = nullptr;
      R.d_rows_count = 0;
      uint32_t* buf = R.host_rows.release();
      if (!buf) buf = (uint32_t*)malloc(sizeof(uint32_t));
      if (!buf) {
        set_last_error("host allocation of the result failed");
        return GPSM_ERR_NOMEM;
      }
      *out_rows = buf;
    }
    e->last = std::move(R);
    return GPSM_OK;
  });
}

int gpsm_match_ex(gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm, const uint32_t* q_edges,
                  const gpsm_match_opts* opts, uint32_t** out_rows, int32_t* id_map, int32_t* pos2id,
                  gpsm_match_info* info) {
  return gpsm_engine_match(nullptr, g, qn, q_labels, qm, q_edges, opts, out_rows, id_map, pos2id, info);
}

int gpsm_match(gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm, const uint32_t* q_edges,
               uint64_t cap, uint32_t** out_rows, uint64_t* out_nrows, uint32_t* out_ncols, int32_t* id_map) {
  gpsm_match_opts o;
  memset(&o, 0, sizeof(o));
  o.cap = cap;
  gpsm_match_info info;
  int rc = gpsm_match_ex(g, qn, q_labels, qm, q_edges, &o, out_rows, id_map, nullptr, &info);
  if (rc == GPSM_OK) {
    if (out_nrows) *out_nrows = info.rows;
    if (out_ncols) *out_ncols = info.cols;
  }
  return rc;
}

void gpsm_free(void* p) { host_free(p); }

void gpsm_host_pool_stats(uint64_t* blocks, uint64_t* pinned_bytes, uint64_t* grown, double* grow_ms) {
  host_pool_stats(blocks, pinned_bytes, grown, grow_ms);
}

int gpsm_last_levels(gpsm_engine_t eng, uint32_t n, uint64_t* level_in, uint64_t* level_cands, uint64_t* level_out) {
  gpsm_engine_s* e = engine_or_default(eng);
  if (!e) return GPSM_ERR_STATE;
  std::lock_guard<std::mutex> lk(e->mu);
  const MatchStats& st = e->last.stats;
  for (uint32_t w = 0; w <= n; ++w) {
    if (level_in) level_in[w] = w < st.level_in.size() ? st.level_in[w] : 0;
    if (level_cands) level_cands[w] = w < st.level_cands.size() ? st.level_cands[w] : 0;
    if (level_out) level_out[w] = w < st.level_rows.size() ? st.level_rows[w] : 0;
  }
  return GPSM_OK;
}

int gpsm_set_tuning(const gpsm_tuning* t) {
  if (!t) return GPSM_ERR_INVALID;
  Tuning& T = tuning();
  if (t->heavy_degree) T.heavy_degree = t->heavy_degree;
  if (t->ext_blocks_per_sm) T.ext_blocks_per_sm = std::min<uint32_t>(t->ext_blocks_per_sm, 8);
  if (t->step_cands) T.step_cands = std::max<uint64_t>(t->step_cands, 1u << 16);
  if (t->level_bytes) T.level_bytes = std::max<uint64_t>(t->level_bytes, 1u << 20);
  if (t->slots) T.slots = std::min<uint32_t>(t->slots, 64);
  if (t->race_share) T.race_share = t->race_share;
  if (t->scan_spin_limit) T.scan_spin_limit = t->scan_spin_limit;
  if (t->ext_items) T.ext_items = t->ext_items >= 8 ? 8u : 4u;
  if (t->filter_team) T.filter_team = t->filter_team >= 32 ? 32u : t->filter_team <= 4 ? 4u : 8u;
  if (t->explore_team) T.explore_team = t->explore_team >= 32 ? 32u : 8u;
  return GPSM_OK;
}

int gpsm_get_tuning(gpsm_tuning* t) {
  if (!t) return GPSM_ERR_INVALID;
  const Tuning& T = tuning();
  t->heavy_degree = T.heavy_degree;
  t->ext_blocks_per_sm = T.ext_blocks_per_sm;
  t->step_cands = T.step_cands;
  t->level_bytes = T.level_bytes;
  t->slots = T.slots;
  t->scan_spin_limit = T.scan_spin_limit;
  t->race_share = T.race_share;
  t->ext_items = T.ext_items;
  t->filter_team = T.filter_team;
  t->explore_team = T.explore_team;
  t->pad = 0;
  return GPSM_OK;
}

int gpsm_model_params(void) { return kParams; }

int gpsm_model_create(int dev, uint64_t seed, gpsm_model_t* out) {
  if (!out) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    gpsm_model_s* h = new gpsm_model_s();
    h->m = model_create(dev, seed);
    *out = h;
    return GPSM_OK;
  });
}

int gpsm_model_destroy(gpsm_model_t m) {
  if (!m) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    model_free(m->m);
    delete m;
    return GPSM_OK;
  });
}

int gpsm_model_set(gpsm_model_t m, const float* params) {
  if (!m || !params) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    model_set(m->m, params);
    return GPSM_OK;
  });
}

int gpsm_model_get(gpsm_model_t m, float* params) {
  if (!m || !params) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    model_get(m->m, params);
    return GPSM_OK;
  });
}

int gpsm_model_train(gpsm_model_t m, const float* x, const float* y, uint32_t n, uint32_t epochs, uint32_t batch,
                     float lr, uint64_t seed, float* loss) {
  if (!m || !x || !y || n == 0) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    float l = model_train(m->m, x, y, n, epochs, batch, lr, seed);
    if (loss) *loss = l;
    return GPSM_OK;
  });
}

int gpsm_model_grad(gpsm_model_t m, const float* x, const float* y, uint32_t n, float* grad, float* loss) {
  if (!m || !x || !y || !grad || n == 0) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    float l = model_grad(m->m, x, y, n, grad);
    if (loss) *loss = l;
    return GPSM_OK;
  });
}

int gpsm_model_predict(gpsm_model_t m, const float* x, uint32_t n, float* y) {
  if (!m || !x || !y) return GPSM_ERR_INVALID;
  if (n == 0) return GPSM_OK;
  return guarded([&]() -> int {
    model_predict(m->m, x, n, y);
    return GPSM_OK;
  });
}

int gpsm_order_features(gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm, const uint32_t* q_edges,
                        const uint32_t* cand_count, const uint64_t* size_fwd, const uint64_t* size_rev,
                        const int32_t* pos2id, float* out) {
  if (!g || !cand_count || !pos2id || !out || (qm && (!size_fwd || !size_rev))) return GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    QueryPlan Q;
    std::string err;
    int rc = plan_query(*g->g, qn, q_labels, qm, q_edges, Q, err);
    if (rc != GPSM_OK) {
      set_last_error(err);
      return rc;
    }
    if (qn > (uint32_t)kMaxPlanQ) {
      set_last_error("query too large for the planner");
      return GPSM_ERR_INVALID;
    }
    std::vector<int32_t> ord(pos2id, pos2id + qn);
    if (!valid_order(Q, ord)) {
      set_last_error("order is not a connected permutation");
      return GPSM_ERR_INVALID;
    }
    std::vector<uint32_t> cand(cand_count, cand_count + qn);
    std::vector<uint64_t> sf(size_fwd, size_fwd + qm), sr(size_rev, size_rev + qm);
    std::unique_ptr<PlanQuery> PQ(new PlanQuery());
    std::unique_ptr<PlanEdges> PE(new PlanEdges());
    build_plan_inputs(*g->g, Q, cand, sf, sr, *PQ, *PE);
    order_features(*PQ, *PE, ord, out);
    return GPSM_OK;
  });
}

// Throughput entry point: matches nq queries back to back on one engine.
// Rows are produced in device memory and overwritten by the next query
// (GPSM_F_KEEP_ON_DEVICE is implied); counts, cap flags and per-query device
// times come back. Device time of the whole batch is taken with events on
// the engine's stream.
int gpsm_match_batch(gpsm_engine_t eng, gpsm_graph_t g, uint32_t nq, const uint32_t* q_voff,
                     const uint32_t* q_labels, const uint64_t* q_eoff, const uint32_t* q_edges,
                     const gpsm_match_opts* opts, const int32_t* orders, uint64_t* counts, int32_t* capped,
                     double* query_ms, gpsm_batch_info* info) {
  gpsm_engine_s* e = engine_or_default(eng);
  if (!e || !g || !q_voff || !q_labels || !q_eoff) return !e ? GPSM_ERR_STATE : GPSM_ERR_INVALID;
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(e->mu);
    Workspace& ws = *e->ws;
    // counts only: final rows are dropped on the device once counted
    MatchOptions base = to_options(opts);
    base.keep_on_device = false;
    base.collect_rows = false;
    gpsm_batch_info bi;
    memset(&bi, 0, sizeof(bi));
    GPSM_CUDA(cudaEventRecord(ws.evb0, ws.stream));
    for (uint32_t k = 0; k < nq; ++k) {
      const uint32_t qn = q_voff[k + 1] - q_voff[k];
      const uint32_t qm = (uint32_t)(q_eoff[k + 1] - q_eoff[k]);
      QueryPlan Q;
      std::string err;
      int rc = plan_query(*g->g, qn, q_labels + q_voff[k], qm, q_edges + 2 * q_eoff[k], Q, err);
      if (rc != GPSM_OK) {
        set_last_error("query " + std::to_string(k) + ": " + err);
        return rc;
      }
      MatchOptions mo = base;
      if (orders && opts && opts->order_mode == GPSM_ORDER_GIVEN) {
        mo.order_mode = ORDER_GIVEN;
        mo.given_order.assign(orders + q_voff[k], orders + q_voff[k + 1]);
      }
      MatchResult R;
      rc = run_query(ws, *g->g, Q, mo, R);
      if (rc != GPSM_OK) return rc;
      if (counts) counts[k] = R.rows;
      if (capped) capped[k] = R.capped ? 1 : (R.stats.aborted ? 2 : 0);
      if (query_ms) query_ms[k] = R.stats.device_ms;
      bi.rows += R.rows;
      bi.launches += R.stats.filter_launches + R.stats.expand_launches;
      bi.expand_launches += R.stats.expand_launches;
      bi.join_steps += R.stats.join_steps;
      bi.alg_bytes_join += R.stats.alg_bytes_join;
      bi.expand_ms += R.stats.expand_ms;
      bi.filter_ms += R.stats.filter_ms;
    }
    GPSM_CUDA(cudaEventRecord(ws.evb1, ws.stream));
    GPSM_CUDA(cudaEventSynchronize(ws.evb1));
    float ms = 0;
    GPSM_CUDA(cudaEventElapsedTime(&ms, ws.evb0, ws.evb1));
    bi.device_ms = ms;
    if (info) *info = bi;
    return GPSM_OK;
  });
}

// Vertices of a device-resident graph with `label` and degree >= min_degree,
// ascending, as the reference's check_kernel + kernel_collect compute them
// (match/Match.cu:431-526). d_labels[n], d_offsets[n+1]: device arrays;
// d_out: device, room for n ids; d_count: device, one u32. Scratch (the
// selection bitmap and the scan state) comes from the engine's workspace.
// Runs on the engine's stream and returns after it finishes.
int gpsm_select_vertices(gpsm_engine_t eng, const uint32_t* d_labels, const uint32_t* d_offsets, uint32_t n,
                         uint32_t label, uint32_t min_degree, uint32_t* d_out, uint32_t* d_count) {
  gpsm_engine_s* e = engine_or_default(eng);
  if (!e) {
    set_last_error("gpsm_init was not called");
    return GPSM_ERR_STATE;
  }
  if (!d_labels || !d_offsets || !d_out || !d_count || n == 0) {
    set_last_error("gpsm_select_vertices: null array or n == 0");
    return GPSM_ERR_INVALID;
  }
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(e->mu);
    Workspace& ws = *e->ws;
    ws.arena.reset();
    uint32_t* bm = (uint32_t*)ws.arena.alloc((size_t)select_words(n) * 4);
    if (!bm) {
      set_last_error("gpsm_select_vertices: workspace too small");
      return GPSM_ERR_NOMEM;
    }
    GPSM_CUDA(cudaMemsetAsync(ws.d_flags, 0, sizeof(uint32_t), ws.stream));
    select_vertices(ws, d_labels, d_offsets, n, label, min_degree, bm, d_out, d_count);
    GPSM_CUDA(cudaMemcpyAsync(ws.h_small, ws.d_flags, sizeof(uint32_t), cudaMemcpyDeviceToHost, ws.stream));
    GPSM_CUDA(cudaStreamSynchronize(ws.stream));
    // a look-back wait that gave up or a ticket out of range leaves the list
    // and count wrong: report it instead of returning them
    if (*reinterpret_cast<const uint32_t*>(ws.h_small) & (DF_SCAN_TIMEOUT | DF_BOUNDS)) {
      set_last_error("gpsm_select_vertices: device wait limit or bounds check tripped");
      ws.dirty = true;
      return GPSM_ERR_TIMEOUT;
    }
    return GPSM_OK;
  });
}

// Writes `bytes` (> L2 size) through the engine's stream so the next timed
// region starts with a cold L2.
int gpsm_flush_l2(gpsm_engine_t eng, uint64_t bytes) {
  gpsm_engine_s* e = engine_or_default(eng);
  if (!e) return GPSM_ERR_STATE;
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(e->mu);
    Workspace& ws = *e->ws;
    bytes = std::min<uint64_t>(bytes, ws.arena.size);
    GPSM_CUDA(cudaMemsetAsync(ws.arena.base, 0x5a, bytes, ws.stream));
    GPSM_CUDA(cudaStreamSynchronize(ws.stream));
    return GPSM_OK;
  });
}

int gpsm_debug_skew_scan_tickets(gpsm_engine_t eng, uint32_t k) {
  gpsm_engine_s* e = engine_or_default(eng);
  if (!e) return GPSM_ERR_STATE;
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(e->mu);
    Workspace& ws = *e->ws;
    unsigned long long c = 0;
    GPSM_CUDA(cudaStreamSynchronize(ws.stream));
    GPSM_CUDA(cudaMemcpy(&c, ws.scan.d_ticket, sizeof(c), cudaMemcpyDeviceToHost));
    c += k;
    GPSM_CUDA(cudaMemcpy(ws.scan.d_ticket, &c, sizeof(c), cudaMemcpyHostToDevice));
    return GPSM_OK;
  });
}

// Candidate statistics of the filter stage for one query, for comparison
// with the reference restatement: final |C(u)| per query vertex, forward and
// reverse candidate-edge totals per edge id, the filter (BFS) order and the
// plain join order. cand_bits (qn*N bytes, 0/1) may be NULL.
int gpsm_debug_filter(gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm, const uint32_t* q_edges,
                      uint32_t* cand_count, uint64_t* size_fwd, uint64_t* size_rev, uint32_t* filter_order,
                      int32_t* plain_pos2id, uint8_t* cand_bits) {
  gpsm_engine_s* e = g_default;
  if (!e || !g) return GPSM_ERR_STATE;
  return guarded([&]() -> int {
    std::lock_guard<std::mutex> lk(e->mu);
    QueryPlan Q;
    std::string err;
    int rc = plan_query(*g->g, qn, q_labels, qm, q_edges, Q, err);
    if (rc != GPSM_OK) {
      set_last_error(err);
      return rc;
    }
    MatchOptions mo;
    mo.filter_only = true;
    mo.collect_rows = false;
    mo.keep_on_device = true;
    MatchResult R;
    rc = run_query(*e->ws, *g->g, Q, mo, R);
    if (rc != GPSM_OK) return rc;
    if (filter_order)
      for (size_t i = 0; i < Q.order.size(); ++i) filter_order[i] = Q.order[i];
    if (cand_count)
      for (uint32_t u = 0; u < qn; ++u) cand_count[u] = R.stats.cand_count.empty() ? 0 : R.stats.cand_count[u];
    for (uint32_t i = 0; i < qm; ++i) {
      if (size_fwd) size_fwd[i] = R.stats.size_fwd.empty() ? 0 : R.stats.size_fwd[i];
      if (size_rev) size_rev[i] = R.stats.size_rev.empty() ? 0 : R.stats.size_rev[i];
    }
    if (plain_pos2id)
      for (uint32_t i = 0; i < qn; ++i) plain_pos2id[i] = R.pos2id.empty() ? -1 : R.pos2id[i];
    if (cand_bits && !R.empty_filter) {
      // the candidate bitmaps are the first allocation of the arena
      const uint32_t W = g->g->words;
      std::vector<uint32_t> bm((size_t)qn * W);
      GPSM_CUDA(cudaMemcpy(bm.data(), e->ws->arena.base, bm.size() * 4, cudaMemcpyDeviceToHost));
      const uint32_t N = g->g->n;
      for (uint32_t u = 0; u < qn; ++u)
        for (uint32_t x = 0; x < N; ++x) cand_bits[(size_t)u * N + x] = (bm[(size_t)u * W + (x >> 5)] >> (x & 31)) & 1;
    } else if (cand_bits) {
      memset(cand_bits, 0, (size_t)qn * g->g->n);
    }
    return R.empty_filter ? 1 : GPSM_OK;
  });
}

}  // extern "C"
