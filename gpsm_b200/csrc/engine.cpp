// Per-query pipeline on one device-resident data graph.
//
// Order of work, as in Match::match (match/Match.cu:1710-1966):
//   plan (host) -> candidate init + explore -> refinement -> final lists
//   -> candidate edges (both directions) -> join order -> joins.
// Differences that are design choices of this engine:
//   - no host round trip per scan: compaction and scans keep their totals on
//     the device; the host waits only twice before the joins (candidate
//     counts, then candidate-edge totals) and once per join chunk;
//   - the join runs depth-first over chunks of rows (a level is expanded only
//     after every deeper level is empty), so intermediate tables are bounded
//     by `level_bytes` per level instead of growing until cudaMalloc fails,
//     while the output keeps the reference's row order;
//   - injectivity is checked while joining, and the embedding cap stops the
//     query after exactly `cap` rows (the first `cap` in row order).
#include "engine.h"

#include "learned.h"

#include <algorithm>
#include <chrono>
#include <memory>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <queue>

namespace gpsm {

bool QueryPlan::adjacent(uint32_t a, uint32_t b) const {
  return std::binary_search(rcol.begin() + roff[a], rcol.begin() + roff[a + 1], b);
}

int QueryPlan::edge_between(uint32_t a, uint32_t b) const {
  uint32_t x = std::min(a, b), y = std::max(a, b);
  for (uint32_t e = 0; e < m; ++e)
    if (efrom[e] == x && eto[e] == y) return (int)e;
  return -1;
}

int plan_query(const DeviceGraph& g, uint32_t qn, const uint32_t* qlab, uint32_t qm, const uint32_t* qe,
               QueryPlan& Q, std::string& err) {
  if (qn == 0 || qlab == nullptr || (qm > 0 && qe == nullptr)) {
    err = "empty query";
    return GPSM_ERR_INVALID;
  }
  if (qn >= kMaxBack) {
    err = "query has too many vertices (limit 127)";
    return GPSM_ERR_INVALID;
  }
  Q = QueryPlan();
  Q.n = qn;
  Q.m = qm;
  Q.lab.assign(qlab, qlab + qn);
  Q.in.assign(qn, {});
  Q.out.assign(qn, {});
  std::vector<uint64_t> seen;
  for (uint32_t i = 0; i < qm; ++i) {
    uint32_t a = qe[2 * i], b = qe[2 * i + 1];
    if (a >= qn || b >= qn) {
      err = "query edge endpoint out of range";
      return GPSM_ERR_INVALID;
    }
    if (a == b) {
      err = "query self loop";
      return GPSM_ERR_INVALID;
    }
    seen.push_back(((uint64_t)std::min(a, b) << 32) | std::max(a, b));
    Q.out[a].push_back(b);
    Q.in[b].push_back(a);
    Q.fe_from.push_back(a);
    Q.fe_to.push_back(b);
  }
  std::sort(seen.begin(), seen.end());
  if (std::adjacent_find(seen.begin(), seen.end()) != seen.end()) {
    err = "parallel query edges";
    return GPSM_ERR_INVALID;
  }
  Q.roff.assign(qn + 1, 0);
  for (uint32_t i = 0; i < qn; ++i) Q.roff[i + 1] = Q.roff[i] + (uint32_t)(Q.in[i].size() + Q.out[i].size());
  Q.rcol.resize(Q.roff[qn]);
  for (uint32_t i = 0; i < qn; ++i) {
    uint32_t p = Q.roff[i];
    for (uint32_t x : Q.in[i]) Q.rcol[p++] = x;
    for (uint32_t x : Q.out[i]) Q.rcol[p++] = x;
    std::sort(Q.rcol.begin() + Q.roff[i], Q.rcol.begin() + Q.roff[i + 1]);
  }
  for (uint32_t i = 0; i < qn; ++i)
    for (uint32_t a : Q.in[i]) {
      Q.efrom.push_back(std::min(a, i));
      Q.eto.push_back(std::max(a, i));
    }
  // connectivity
  {
    std::vector<uint8_t> vis(qn, 0);
    std::vector<uint32_t> st{0};
    vis[0] = 1;
    uint32_t cnt = 1;
    while (!st.empty()) {
      uint32_t t = st.back();
      st.pop_back();
      for (uint32_t k = Q.roff[t]; k < Q.roff[t + 1]; ++k)
        if (!vis[Q.rcol[k]]) {
          vis[Q.rcol[k]] = 1;
          ++cnt;
          st.push_back(Q.rcol[k]);
        }
    }
    if (cnt != qn) {
      err = "query is not connected";
      return GPSM_ERR_INVALID;
    }
  }
  if (qm == 0) {
    Q.order = {0};
    return GPSM_OK;
  }
  // generateSpanningTree (match/Match.cu:339-429): score = degree / label
  // frequency with the reference's float arithmetic; the first edge with the
  // largest score sum (strict >) gives the start; BFS over sorted lists.
  std::vector<float> score(qn);
  for (uint32_t i = 0; i < qn; ++i) {
    float num = (float)g.label_count(Q.lab[i]);
    int degree = (int)(Q.in[i].size() + Q.out[i].size());
    score[i] = (float)(((double)degree + 0.0) / (double)num);
  }
  float maxv = 0.0f;
  int maxi = -1;
  for (uint32_t i = 0; i < qm; ++i) {
    float t = score[Q.efrom[i]] + score[Q.eto[i]];
    if (t > maxv) {
      maxv = t;
      maxi = (int)i;
    }
  }
  if (maxi < 0) maxi = 0;
  uint32_t start = Q.efrom[maxi];
  if (score[Q.eto[maxi]] > score[Q.efrom[maxi]]) start = Q.eto[maxi];
  std::vector<uint8_t> vis(qn, 0);
  std::queue<uint32_t> q;
  Q.order.push_back(start);
  vis[start] = 1;
  q.push(start);
  while (!q.empty()) {
    uint32_t t = q.front();
    q.pop();
    for (uint32_t k = Q.roff[t]; k < Q.roff[t + 1]; ++k) {
      uint32_t a = Q.rcol[k];
      if (vis[a]) continue;
      vis[a] = 1;
      Q.order.push_back(a);
      q.push(a);
    }
  }
  return GPSM_OK;
}

std::vector<int32_t> plain_order(const QueryPlan& Q, const std::vector<uint64_t>& size_fwd, uint64_t nnz) {
  std::vector<int32_t> pos2id;
  if (Q.m == 0) {
    pos2id.push_back(0);
    return pos2id;
  }
  std::vector<uint8_t> vv(Q.n, 0), ve(Q.m, 0);
  uint64_t minv = nnz + 1;
  uint32_t minx = 0;
  for (uint32_t i = 0; i < Q.m; ++i)
    if (size_fwd[i] < minv) {
      minv = size_fwd[i];
      minx = i;
    }
  vv[Q.efrom[minx]] = vv[Q.eto[minx]] = 1;
  ve[minx] = 1;
  pos2id.push_back((int32_t)Q.efrom[minx]);
  pos2id.push_back((int32_t)Q.eto[minx]);
  for (uint32_t c = 1; c < Q.m; ++c) {
    // a closed edge first (both endpoints visited); it adds no column
    uint64_t best = nnz + 1;
    int bx = -1;
    for (uint32_t i = 0; i < Q.m; ++i)
      if (!ve[i] && vv[Q.efrom[i]] && vv[Q.eto[i]] && size_fwd[i] < best) {
        best = size_fwd[i];
        bx = (int)i;
      }
    if (bx < 0) {
      for (uint32_t i = 0; i < Q.m; ++i)
        if (!ve[i] && (vv[Q.efrom[i]] || vv[Q.eto[i]]) && size_fwd[i] < best) {
          best = size_fwd[i];
          bx = (int)i;
        }
      if (bx < 0) break;  // cannot happen for connected queries
      uint32_t u = Q.efrom[bx], v = Q.eto[bx];
      pos2id.push_back((int32_t)(vv[u] ? v : u));
    }
    vv[Q.efrom[bx]] = vv[Q.eto[bx]] = 1;
    ve[bx] = 1;
  }
  return pos2id;
}

void build_plan_inputs(const DeviceGraph& g, const QueryPlan& Q, const std::vector<uint32_t>& cand,
                       const std::vector<uint64_t>& size_fwd, const std::vector<uint64_t>& size_rev, PlanQuery& PQ,
                       PlanEdges& PE) {
  memset(&PQ, 0, sizeof(PQ));
  PQ.n = Q.n;
  for (uint32_t u = 0; u < Q.n; ++u) {
    for (uint32_t k = Q.roff[u]; k < Q.roff[u + 1]; ++k) {
      const uint32_t w = Q.rcol[k];
      PQ.adj[u][w >> 6] |= 1ULL << (w & 63);
    }
    PQ.label[u] = Q.lab[u];
    PQ.qdeg[u] = Q.deg(u);
    PQ.log_cand[u] = std::log2(1.0f + (float)cand[u]);
    uint32_t b, e;
    g.label_range(Q.lab[u], Q.deg(u), &b, &e);
    PQ.log_labdeg[u] = std::log2(1.0f + (float)(e - b));
    PQ.log_label[u] = std::log2(1.0f + (float)g.label_count(Q.lab[u]));
  }
  for (size_t i = 0; i < (size_t)kMaxPlanQ * kMaxPlanQ; ++i) PE.log_size[i] = PE.log_avg[i] = 0.f;
  for (uint32_t e = 0; e < Q.m; ++e) {
    const uint32_t a = Q.efrom[e], b = Q.eto[e];
    const float sf = (float)size_fwd[e], sr = (float)size_rev[e];
    PE.log_size[a * kMaxPlanQ + b] = std::log2(1.f + sf);
    PE.log_size[b * kMaxPlanQ + a] = std::log2(1.f + sr);
    PE.log_avg[a * kMaxPlanQ + b] = std::log2(1.f + sf / std::max(1.f, (float)cand[a]));
    PE.log_avg[b * kMaxPlanQ + a] = std::log2(1.f + sr / std::max(1.f, (float)cand[b]));
  }
}

void order_features(const PlanQuery& PQ, const PlanEdges& PE, const std::vector<int32_t>& pos2id, float* out) {
  uint64_t P[2] = {0, 0};
  P[pos2id[0] >> 6] |= 1ULL << (pos2id[0] & 63);
  for (uint32_t k = 1; k < pos2id.size(); ++k) {
    const uint32_t v = (uint32_t)pos2id[k];
    step_features(PQ, PE, P, k, v, out + (size_t)(k - 1) * kFeat);
    P[v >> 6] |= 1ULL << (v & 63);
  }
}

bool valid_order(const QueryPlan& Q, const std::vector<int32_t>& pos2id) {
  if (pos2id.size() != Q.n) return false;
  std::vector<uint8_t> seen(Q.n, 0);
  for (size_t i = 0; i < pos2id.size(); ++i) {
    int32_t u = pos2id[i];
    if (u < 0 || (uint32_t)u >= Q.n || seen[u]) return false;
    if (i > 0) {
      bool any = false;
      for (uint32_t k = Q.roff[u]; k < Q.roff[u + 1]; ++k) any |= seen[Q.rcol[k]] != 0;
      if (!any) return false;
    }
    seen[u] = 1;
  }
  return true;
}

namespace {

bool trace_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = getenv("GPSM_TRACE");
    on = (e && *e && *e != '0') ? 1 : 0;
  }
  return on == 1;
}

template <class T>
T* arena_alloc(Workspace& ws, uint64_t count) {
  void* p = ws.arena.alloc(std::max<uint64_t>(count, 1) * sizeof(T));
  if (!p) {
    set_last_error("workspace arena exhausted: " + std::to_string(count * sizeof(T)) + " bytes requested, " +
                   std::to_string(ws.arena.used) + " of " + std::to_string(ws.arena.size) + " in use");
    throw CudaError{cudaErrorMemoryAllocation, "arena"};
  }
  return (T*)p;
}

struct Level {
  uint32_t* buf = nullptr;
  uint64_t cap_rows = 0;
  uint64_t nrows = 0;
  uint64_t next = 0;
  double ratio = 4.0;  // observed candidates per input row of the last step from this level
  // share of candidates the last step from this level kept, with headroom
  // (1: a step admits no more candidates than its output holds rows)
  double keep = 1.0;
};

}  // namespace

void launch_plan(cudaStream_t s, const Model* M, const PlanQuery* d_q, const PlanEdges* d_e, const uint32_t* d_starts,
                 uint32_t nstarts, const int32_t* d_fixed, void* d_out);
size_t plan_out_bytes();

// Bytes of one intermediate level buffer: the configured size, shrunk for
// deep queries so that the n - 2 level buffers together take at most half
// of the workspace arena (a 64-vertex query would otherwise ask for 62 full
// buffers).
static uint64_t level_buffer_bytes(const Workspace& ws, const MatchOptions& opt, uint32_t qn) {
  uint64_t lb = opt.level_bytes;
  if (qn > 2) lb = std::min<uint64_t>(lb, (ws.arena.size / 2) / (qn - 2));
  return std::max<uint64_t>(lb, 1ull << 20);
}

// A learned plan replaces the plain order only when the model predicts it
// scans at most this fraction of the plain order's rows: the model's error
// on one step is about 1.2 in log2 (validation MSE 1.49), so small predicted
// gains are noise.
constexpr double kLearnedMargin = 0.5;

// Learned order: greedy MLP plans from up to 8 start vertices on the device,
// scored with the plain order in the same launch; the plan with the smallest
// predicted work wins if it beats the plain order by the margin. Returns {}
// (plain order) otherwise, or when the plan's predicted resident join memory
// exceeds the memory budget.
static std::vector<int32_t> learned_order(Workspace& ws, const DeviceGraph& g, const QueryPlan& Q,
                                          const std::vector<uint32_t>& cnt, const std::vector<uint64_t>& size_fwd,
                                          const std::vector<uint64_t>& size_rev, const std::vector<int32_t>& plain,
                                          const MatchOptions& opt, MatchStats& st) {
  static thread_local std::unique_ptr<PlanQuery> PQ(new PlanQuery());
  static thread_local std::unique_ptr<PlanEdges> PE(new PlanEdges());
  build_plan_inputs(g, Q, cnt, size_fwd, size_rev, *PQ, *PE);
  // starts: endpoints of the two smallest forward candidate-edge sets, then
  // the vertices with the fewest candidates
  std::vector<uint32_t> starts;
  auto add = [&](uint32_t v) {
    if (starts.size() < 8 && std::find(starts.begin(), starts.end(), v) == starts.end()) starts.push_back(v);
  };
  std::vector<uint32_t> eidx(Q.m);
  for (uint32_t e = 0; e < Q.m; ++e) eidx[e] = e;
  std::sort(eidx.begin(), eidx.end(), [&](uint32_t a, uint32_t b) {
    return size_fwd[a] != size_fwd[b] ? size_fwd[a] < size_fwd[b] : a < b;
  });
  for (uint32_t i = 0; i < std::min<uint32_t>(2, Q.m); ++i) {
    add(Q.efrom[eidx[i]]);
    add(Q.eto[eidx[i]]);
  }
  std::vector<uint32_t> vidx(Q.n);
  for (uint32_t u = 0; u < Q.n; ++u) vidx[u] = u;
  std::sort(vidx.begin(), vidx.end(), [&](uint32_t a, uint32_t b) { return cnt[a] != cnt[b] ? cnt[a] < cnt[b] : a < b; });
  for (uint32_t u : vidx) add(u);
  const size_t mark = ws.arena.used;
  PlanQuery* d_q = arena_alloc<PlanQuery>(ws, 1);
  PlanEdges* d_e = arena_alloc<PlanEdges>(ws, 1);
  uint32_t* d_st = arena_alloc<uint32_t>(ws, 8);
  int32_t* d_fixed = arena_alloc<int32_t>(ws, kMaxPlanQ);
  char* d_out = arena_alloc<char>(ws, plan_out_bytes() * 9);
  cudaStream_t s = ws.stream;
  GPSM_CUDA(cudaMemcpyAsync(d_q, PQ.get(), sizeof(PlanQuery), cudaMemcpyHostToDevice, s));
  // only the rows of the n query vertices are read
  GPSM_CUDA(cudaMemcpyAsync(d_e->log_size, PE->log_size, sizeof(float) * kMaxPlanQ * Q.n, cudaMemcpyHostToDevice, s));
  GPSM_CUDA(cudaMemcpyAsync(d_e->log_avg, PE->log_avg, sizeof(float) * kMaxPlanQ * Q.n, cudaMemcpyHostToDevice, s));
  GPSM_CUDA(cudaMemcpyAsync(d_st, starts.data(), starts.size() * 4, cudaMemcpyHostToDevice, s));
  GPSM_CUDA(cudaMemcpyAsync(d_fixed, plain.data(), Q.n * 4, cudaMemcpyHostToDevice, s));
  launch_plan(s, opt.model, d_q, d_e, d_st, (uint32_t)starts.size(), d_fixed, d_out);
  std::vector<char> hout(plan_out_bytes() * (starts.size() + 1));
  char* h_plan = reinterpret_cast<char*>(ws.h_small + 2048);  // the plans, through the pinned mirror
  small_to_host(ws, h_plan, d_out, hout.size());
  stream_wait(ws);
  memcpy(hout.data(), h_plan, hout.size());
  ws.arena.used = mark;  // planner scratch is not needed by the joins
  const size_t ob = plan_out_bytes();
  int best = -1;
  float best_work = 0.f;
  for (size_t i = 0; i < starts.size(); ++i) {
    const int32_t* order = reinterpret_cast<const int32_t*>(hout.data() + i * ob);
    const float work = *reinterpret_cast<const float*>(hout.data() + i * ob + kMaxPlanQ * 4);
    std::vector<int32_t> ord(order, order + Q.n);
    if (!valid_order(Q, ord)) continue;
    if (best < 0 || work < best_work) {
      best = (int)i;
      best_work = work;
    }
  }
  const float plain_work =
      *reinterpret_cast<const float*>(hout.data() + starts.size() * ob + kMaxPlanQ * 4);
  st.predicted_work_plain = plain_work;
  if (best < 0) return {};
  // predicted resident join memory: each width's table is held in chunks of
  // at most one level buffer, the final rows in the result buffer
  const float* logsz = reinterpret_cast<const float*>(hout.data() + (size_t)best * ob + kMaxPlanQ * 4 + 16);
  const uint64_t min_rows = (uint64_t)g.max_degree + 64;
  const uint64_t lb = level_buffer_bytes(ws, opt, Q.n);
  double resident = 0;
  for (uint32_t k = 1; k < Q.n; ++k) {  // position k holds tables of width k + 1
    const uint32_t w = k + 1;
    const double table = std::exp2((double)logsz[k]) * 4.0 * w;
    if (w < Q.n) {
      resident += std::min(table, (double)std::max<uint64_t>(lb, min_rows * 4ull * w));
    } else {
      const double res_rows = std::min<double>((double)std::max<uint64_t>(opt.result_rows, 1), (double)opt.cap);
      resident += std::min(table, res_rows * 4.0 * w);
    }
  }
  st.predicted_work = best_work;
  st.predicted_peak = resident;
  const uint64_t budget = opt.memory_budget ? opt.memory_budget : ws.arena.size;
  if (resident > (double)budget) {
    st.order_fallback = 1;
    return {};
  }
  if ((double)best_work > kLearnedMargin * (double)plain_work) {
    st.order_fallback = 2;
    return {};
  }
  const int32_t* order = reinterpret_cast<const int32_t*>(hout.data() + (size_t)best * ob);
  return std::vector<int32_t>(order, order + Q.n);
}

namespace {
// Products of the filter phase that the joins read.
struct FilterProducts {
  uint32_t* bm = nullptr;              // candidate bitmaps, one per query vertex
  uint32_t* rank = nullptr;            // per-word ranks of the final lists
  std::vector<uint32_t*> list;         // final sorted candidate lists
  std::vector<uint32_t> cnt;           // |C(u)|
  std::vector<CedgeDir> dirs;          // candidate-edge directions (2 per query edge)
  unsigned long long* goff = nullptr;  // candidate-edge list offsets
  uint32_t* nbrs = nullptr;            // candidate-edge lists
  uint64_t nbrs_total = 0;
};
}  // namespace

// Candidate initialisation, exploration, refinement, the final candidate
// lists with ranks and the candidate edges of every query edge in both
// directions (match/Match.cu:661-1139). On return R.empty_filter says the
// query has no embedding (a label is absent or a candidate set ran empty).
static int run_filter(Workspace& ws, const DeviceGraph& g, const QueryPlan& Q, MatchResult& R, FilterProducts& F) {
  const uint32_t qn = Q.n, W = g.words;
  cudaStream_t s = ws.stream;

  // ---- allocations ---------------------------------------------------------
  uint32_t* bm = arena_alloc<uint32_t>(ws, (uint64_t)qn * W);
  uint32_t* rank = arena_alloc<uint32_t>(ws, (uint64_t)qn * W);
  uint32_t* counts = arena_alloc<uint32_t>(ws, qn);
  std::vector<uint32_t*> list(qn);
  std::vector<uint32_t> bound(qn);
  for (uint32_t u = 0; u < qn; ++u) {
    bound[u] = (uint32_t)g.label_count(Q.lab[u]);
    if (bound[u] == 0) {  // a label absent from the data graph: no candidate
      R.empty_filter = true;
      R.id2pos.assign(qn, -1);
      R.pos2id.assign(qn, -1);
      return GPSM_OK;
    }
    list[u] = arena_alloc<uint32_t>(ws, bound[u]);
  }
  GPSM_CUDA(cudaMemsetAsync(bm, 0, sizeof(uint32_t) * (uint64_t)qn * W, s));

  // query structure for the filter kernels: explore targets (v, label,
  // degree) per order position, refinement targets per simple vertex
  std::vector<uint32_t> params;
  std::vector<uint32_t> exp_off(qn + 1, 0), exp_cnt(qn, 0);
  std::vector<uint8_t> initialized(qn, 0);
  {
    std::vector<uint8_t> init_sim(qn, 0);
    for (uint32_t i = 0; i < Q.order.size(); ++i) {
      uint32_t u = Q.order[i];
      init_sim[u] = 1;
      exp_off[i] = (uint32_t)params.size();
      for (uint32_t k = Q.roff[u]; k < Q.roff[u + 1]; ++k) {
        uint32_t v = Q.rcol[k];
        if (!init_sim[v]) {
          params.push_back(v);
          params.push_back(Q.lab[v]);
          params.push_back(Q.deg(v));
          exp_cnt[i]++;
        }
      }
      for (uint32_t k = Q.roff[u]; k < Q.roff[u + 1]; ++k) init_sim[Q.rcol[k]] = 1;
    }
  }
  // generateSimplifiedGraph (match/Match.cu:721-759): degree > 1
  std::vector<uint32_t> simple;
  std::vector<uint8_t> valid(qn, 0);
  for (uint32_t i = 0; i < qn; ++i)
    if (Q.deg(i) > 1) {
      valid[i] = 1;
      simple.push_back(i);
    }
  // refinement targets: (query vertex, its label) pairs
  std::vector<uint32_t> ref_off(simple.size()), ref_cnt(simple.size());
  for (size_t i = 0; i < simple.size(); ++i) {
    ref_off[i] = (uint32_t)params.size();
    for (uint32_t x : Q.in[simple[i]])
      if (valid[x]) params.push_back(x), params.push_back(Q.lab[x]), ref_cnt[i]++;
    for (uint32_t x : Q.out[simple[i]])
      if (valid[x]) params.push_back(x), params.push_back(Q.lab[x]), ref_cnt[i]++;
  }
  uint32_t* d_params = arena_alloc<uint32_t>(ws, params.size() + 1);
  if (!params.empty())
    GPSM_CUDA(cudaMemcpyAsync(d_params, params.data(), params.size() * 4, cudaMemcpyHostToDevice, s));
  uint32_t** d_lists = arena_alloc<uint32_t*>(ws, qn);
  GPSM_CUDA(cudaMemcpyAsync(d_lists, list.data(), qn * sizeof(uint32_t*), cudaMemcpyHostToDevice, s));
  stream_wait(ws);  // params and list are pageable host memory

  auto bm_of = [&](uint32_t u) { return bm + (size_t)u * W; };
  uint64_t launches = 0;

  // ---- candidate initialisation (match/Match.cu:661-719) ---------------------
  // The reference collects C(u) into a list before each explore and refine
  // step (kernel_collect); here those steps read C(u)'s bitmap directly, so
  // only the final lists are compacted. An empty set stays empty (nothing
  // adds candidates to u after its own step) and empties its neighbours' sets
  // in refinement, so the final compaction reports it (DF_EMPTY), as the
  // reference's early return does.
  for (uint32_t i = 0; i < Q.order.size(); ++i) {
    const uint32_t u = Q.order[i];
    if (!initialized[u]) {
      uint32_t b, e;
      g.label_range(Q.lab[u], Q.deg(u), &b, &e);
      launch_mark_range(ws, g, b, e, bm_of(u));
      ++launches;
      initialized[u] = 1;
    }
    if (exp_cnt[i]) {
      launch_explore(ws, g, u, Q.lab[u], Q.deg(u), d_params + exp_off[i], exp_cnt[i], bm);
      ++launches;
    }
    for (uint32_t k = Q.roff[u]; k < Q.roff[u + 1]; ++k) initialized[Q.rcol[k]] = 1;
  }
  // ---- refinement: 4 rounds (match/Match.cu:848-890) -------------------------
  // Launches that would change nothing exit at once (RefineStamp): the
  // rounds and their order are the reference's, so the sets are the same.
  // The reference's fifth round only collects (an emptiness check): the
  // final compaction below does that.
  {
    uint32_t* stamp = arena_alloc<uint32_t>(ws, qn);
    GPSM_CUDA(cudaMemsetAsync(stamp, 0, sizeof(uint32_t) * qn, s));
    std::vector<uint32_t> last_refine(qn, 0);
    uint32_t seq = 0;
    for (int k = 0; k < 4; ++k)
      for (size_t i = 0; i < simple.size(); ++i) {
        const uint32_t u = simple[i];
        if (ref_cnt[i] == 0) continue;
        RefineStamp rs;
        rs.stamp = stamp;
        rs.prev = last_refine[u];
        rs.seq = ++seq;
        launch_refine(ws, g, u, Q.lab[u], Q.deg(u), d_params + ref_off[i], ref_cnt[i], bm, rs);
        last_refine[u] = seq;
        ++launches;
      }
  }
  // ---- final candidate lists with ranks (one launch for every vertex) ------
  launch_compact_multi(ws, bm, W, qn, d_lists, rank, counts);
  ++launches;
  small_to_host(ws, ws.h_small, counts, qn * sizeof(uint32_t));
  small_to_host(ws, ws.h_small + 64, ws.d_flags, sizeof(uint32_t));
  stream_wait(ws);
  std::vector<uint32_t> cnt(qn);
  memcpy(cnt.data(), ws.h_small, qn * sizeof(uint32_t));
  const uint32_t flags = *reinterpret_cast<uint32_t*>(ws.h_small + 64);
  R.stats.cand_count = cnt;
  if (flags & (DF_SCAN_TIMEOUT | DF_BOUNDS)) {
    set_last_error("device wait limit or bounds check tripped in the filter");
    return GPSM_ERR_TIMEOUT;
  }
  if (flags & DF_EMPTY) {
    R.empty_filter = true;
    R.id2pos.assign(qn, -1);
    R.pos2id.assign(qn, -1);
    GPSM_CUDA(cudaEventRecord(ws.ev1, s));
    GPSM_CUDA(cudaEventSynchronize(ws.ev1));
    float ms = 0;
    cudaEventElapsedTime(&ms, ws.ev0, ws.ev1);
    R.stats.device_ms = ms;
    return GPSM_OK;
  }

  // ---- candidate edges, both directions (match/Match.cu:1082-1139) ----------
  const uint32_t m = Q.m;
  const uint32_t ndir = 2 * m;
  std::vector<CedgeDir> dirs(ndir);
  uint64_t items = 0;
  for (uint32_t e = 0; e < m; ++e)
    for (int r = 0; r < 2; ++r) {
      uint32_t u = r ? Q.eto[e] : Q.efrom[e];
      uint32_t v = r ? Q.efrom[e] : Q.eto[e];
      CedgeDir& d = dirs[2 * e + r];
      d.ids = list[u];
      d.n = cnt[u];
      d.v = v;
      d.lab = Q.lab[v];
      d.pad = 0;
      d.item_base = items;
      items += cnt[u];
    }
  unsigned long long* goff = nullptr;
  uint32_t* nbrs = nullptr;
  uint64_t nbrs_total = 0;
  std::vector<uint64_t> dir_total(ndir, 0);
  if (ndir > 0) {
    CedgeDir* d_dirs = arena_alloc<CedgeDir>(ws, ndir);
    uint32_t* ccount = arena_alloc<uint32_t>(ws, items);
    goff = arena_alloc<unsigned long long>(ws, items + 1);
    unsigned long long* d_idx = arena_alloc<unsigned long long>(ws, ndir + 1);
    std::vector<unsigned long long> idx(ndir + 1);
    for (uint32_t d = 0; d < ndir; ++d) idx[d] = dirs[d].item_base;
    idx[ndir] = items;
    GPSM_CUDA(cudaMemcpyAsync(d_dirs, dirs.data(), ndir * sizeof(CedgeDir), cudaMemcpyHostToDevice, s));
    GPSM_CUDA(cudaMemcpyAsync(d_idx, idx.data(), (ndir + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice, s));
    launch_cedge_count(ws, g, d_dirs, ndir, d_idx, items, bm, ccount);
    launch_scan_u32(ws, ccount, items, goff);
    launch_gather_u64(ws, goff, d_idx, ndir + 1, ws.d_small);
    small_to_host(ws, ws.h_small, ws.d_small, (ndir + 1) * sizeof(unsigned long long));
    small_to_host(ws, ws.h_small + 4000, ws.d_flags, sizeof(uint32_t));
    stream_wait(ws);
    if (*reinterpret_cast<uint32_t*>(ws.h_small + 4000) & DF_SCAN_TIMEOUT) {
      set_last_error("device wait limit tripped in candidate-edge scan");
      return GPSM_ERR_TIMEOUT;
    }
    for (uint32_t d = 0; d < ndir; ++d) dir_total[d] = ws.h_small[d + 1] - ws.h_small[d];
    const uint64_t total = ws.h_small[ndir];
    nbrs_total = total;
    nbrs = arena_alloc<uint32_t>(ws, total);
    launch_cedge_write(ws, g, d_dirs, ndir, d_idx, items, bm, goff, nbrs);
    launches += 4;
  }
  R.stats.size_fwd.resize(m);
  R.stats.size_rev.resize(m);
  for (uint32_t e = 0; e < m; ++e) {
    R.stats.size_fwd[e] = dir_total[2 * e];
    R.stats.size_rev[e] = dir_total[2 * e + 1];
  }
  R.stats.filter_launches = launches;
  F.bm = bm;
  F.rank = rank;
  F.list = std::move(list);
  F.cnt = std::move(cnt);
  F.dirs = std::move(dirs);
  F.goff = goff;
  F.nbrs = nbrs;
  F.nbrs_total = nbrs_total;
  return GPSM_OK;
}

// What one join attempt reads and accumulates.
struct JoinContext {
  Workspace& ws;
  const DeviceGraph& g;
  const QueryPlan& Q;
  const MatchOptions& opt;
  MatchResult& R;
  const FilterProducts& F;
  const std::vector<int32_t>& pos2id;
  size_t join_mark;          // arena position where join memory starts
  uint64_t exp_launches = 0;  // over all attempts
  uint64_t alg_bytes = 0;
};

// One attempt joins in the order pos2id until the embeddings are complete,
// the cap is reached or `limit` candidates have been scanned (limit 0: no
// limit); hit_limit reports the last. Every attempt starts from the same
// filter products: it takes join memory from join_mark on and resets the
// result state.
static int join_attempt(JoinContext& C, uint64_t limit, bool& hit_limit) {
  Workspace& ws = C.ws;
  const DeviceGraph& g = C.g;
  const QueryPlan& Q = C.Q;
  const MatchOptions& opt = C.opt;
  MatchResult& R = C.R;
  const std::vector<int32_t>& pos2id = C.pos2id;
  const size_t join_mark = C.join_mark;
  uint64_t& exp_launches = C.exp_launches;
  uint64_t& alg_bytes = C.alg_bytes;
  const uint32_t qn = Q.n, W = g.words;
  cudaStream_t s = ws.stream;
  uint32_t* rank = C.F.rank;
  const std::vector<uint32_t*>& list = C.F.list;
  const std::vector<uint32_t>& cnt = C.F.cnt;
  const std::vector<CedgeDir>& dirs = C.F.dirs;
  unsigned long long* goff = C.F.goff;
  uint32_t* nbrs = C.F.nbrs;
  const uint64_t nbrs_total = C.F.nbrs_total;
  auto bm_of = [&](uint32_t u) { return C.F.bm + (size_t)u * W; };
  // an earlier attempt's copies into the host block end before it is reused
  if (R.copies_pending) {
    GPSM_CUDA(cudaStreamSynchronize(ws.copy_stream));
    R.copies_pending = false;
  }
  // whatever path leaves this attempt, its row copies to the host have
  // ended, unless it returns normally with copies deferred to the caller
  struct CopiesDone {
    Workspace& w;
    bool armed = true;
    ~CopiesDone() {
      if (armed) cudaStreamSynchronize(w.copy_stream);
    }
  } copies_done{ws};
  hit_limit = false;
  ws.arena.used = join_mark;
  R.pos2id = pos2id;
  R.id2pos.assign(qn, -1);
  for (uint32_t p = 0; p < qn; ++p) R.id2pos[pos2id[p]] = (int32_t)p;
  R.host_rows.clear();
  R.d_rows = nullptr;
  R.d_rows_count = 0;
  // a capped query that returns its rows gets a page-locked block for all
  // of them up front: the device copies into it without a bounce buffer
  if (opt.collect_rows && !opt.keep_on_device && opt.cap != ~0ULL)
    R.host_rows.reserve_pinned(opt.cap * (uint64_t)qn);
  // back-neighbour descriptors for each added position p >= 1
  std::vector<BackNbr> hb;
  std::vector<uint32_t> back_off(qn + 1, 0), back_cnt(qn, 0);
  // first estimate of candidates per row when extending to position p: the
  // shortest average candidate-edge list among the placed neighbours (the
  // driver is the shortest list of each row); later steps use what they saw
  std::vector<double> ratio0(qn + 1, 4.0);
  for (uint32_t p = 1; p < qn; ++p) {
    back_off[p] = (uint32_t)hb.size();
    const uint32_t v = (uint32_t)pos2id[p];
    double est = -1.0;
    for (uint32_t k = Q.roff[v]; k < Q.roff[v + 1]; ++k) {
      const uint32_t w = Q.rcol[k];
      if ((uint32_t)R.id2pos[w] >= p) continue;
      const int e = Q.edge_between(w, v);
      const uint32_t d = 2 * (uint32_t)e + (Q.efrom[e] == w ? 0u : 1u);
      const double avg = (double)((d & 1) ? R.stats.size_rev[e] : R.stats.size_fwd[e]) /
                         (double)std::max<uint32_t>(cnt[w], 1);
      if (est < 0 || avg < est) est = avg;
      BackNbr b;
      b.col = (uint32_t)R.id2pos[w];
      b.pad = 0;
      b.bm = bm_of(w);
      b.rank = rank + (size_t)w * W;
      b.off = goff + dirs[d].item_base;
      b.nbrs = nbrs;
      hb.push_back(b);
      back_cnt[p]++;
    }
    if (est >= 0) ratio0[p] = std::max(est, 1.0 / 1024.0);
  }
  BackNbr* d_back = arena_alloc<BackNbr>(ws, hb.size() + 1);
  if (!hb.empty())
    GPSM_CUDA(cudaMemcpyAsync(d_back, hb.data(), hb.size() * sizeof(BackNbr), cudaMemcpyHostToDevice, s));
  // per position: earlier columns holding a query vertex with the same label
  std::vector<uint32_t> inj, inj_off(qn + 1, 0), inj_cnt(qn, 0);
  for (uint32_t p = 1; p < qn; ++p) {
    inj_off[p] = (uint32_t)inj.size();
    for (uint32_t c = 0; c < p; ++c)
      if (Q.lab[pos2id[c]] == Q.lab[pos2id[p]]) {
        inj.push_back(c);
        inj_cnt[p]++;
      }
  }
  uint32_t* d_inj = arena_alloc<uint32_t>(ws, inj.size() + 1);
  if (!inj.empty()) GPSM_CUDA(cudaMemcpyAsync(d_inj, inj.data(), inj.size() * 4, cudaMemcpyHostToDevice, s));
  // two step states used in turn: each step's write pass clears the next
  // step's one (after the host has read it), so no memset per step
  StepState* d_st2 = arena_alloc<StepState>(ws, 2);
  uint32_t st_turn = 0;
  StepState* h_st = reinterpret_cast<StepState*>(ws.h_small + 1024);
  StepState* h_st_dev = reinterpret_cast<StepState*>(ws.h_small_dev + 1024);  // h_st as the device writes it
  JoinScratch js;
  uint32_t max_nb = 1;
  for (uint32_t p = 1; p < qn; ++p) max_nb = std::max(max_nb, back_cnt[p]);
  // per-row scratch: 16 B driver + 8 B offset + 16 B per placed neighbour
  // (at most 1 GiB and a sixteenth of the arena)
  const uint64_t row_scratch = std::min<uint64_t>(1ull << 30, ws.arena.size / 16);
  js.rows = std::max<uint64_t>(std::min<uint64_t>(opt.step_rows, row_scratch / (16ull * max_nb)), 4096);
  js.rng_entries = js.rows * max_nb;
  js.drv = arena_alloc<uint4>(ws, js.rows);
  js.rng = arena_alloc<uint4>(ws, js.rng_entries);
  js.coff = arena_alloc<unsigned long long>(ws, js.rows + 1);
  js.tiles = (opt.step_cands + join_cands_per_extend_tile() - 1) / join_cands_per_extend_tile() + 2;
  js.tile_row = arena_alloc<uint32_t>(ws, js.tiles);
  js.kept_entries = js.tiles * join_cands_per_extend_tile() + join_kept_slack();
  js.kept = arena_alloc<uint2>(ws, js.kept_entries);
  js.tile_cnt = arena_alloc<uint32_t>(ws, js.tiles);
  js.tile_off = arena_alloc<unsigned long long>(ws, js.tiles + 1);
  // zero once: every write pass clears the tile counts it read
  GPSM_CUDA(cudaMemsetAsync(js.tile_cnt, 0, js.tiles * sizeof(uint32_t), s));
  GPSM_CUDA(cudaMemsetAsync(d_st2, 0, 2 * sizeof(StepState), s));
  stream_wait(ws);  // hb is pageable

  R.stats.level_rows.assign(qn + 1, 0);
  R.stats.level_in.assign(qn + 1, 0);
  R.stats.level_cands.assign(qn + 1, 0);
  uint64_t cands_total = 0;
  const uint64_t cap = opt.cap;
  // levels 1..qn; level w holds rows of width w. Level 1 is C(pos2id[0]).
  std::vector<Level> L(qn + 1);
  for (uint32_t w = 1; w < qn; ++w) L[w].ratio = ratio0[w];
  L[1].buf = list[pos2id[0]];
  L[1].nrows = cnt[pos2id[0]];
  L[1].cap_rows = L[1].nrows;
  R.stats.level_rows[1] = L[1].nrows;
  const uint64_t min_rows = (uint64_t)g.max_degree + 64;
  const uint64_t lb = level_buffer_bytes(ws, opt, qn);
  // Levels 2..qn-1 share one stack of the same total size as one buffer per
  // level. A level is extended only when every deeper level is empty, so
  // level w+1 can start right after level w's rows, and a step may use the
  // free top of the stack less a minimum for each deeper level: never less
  // room than its own buffer would give (fixed_rows), and more as the
  // attempt's work grows (stack_ramp), so a long query's deep steps are not
  // held to one level's share while a capped query, which ends early, keeps
  // the small steps that waste little past its cap.
  std::vector<uint64_t> fixed_rows(qn + 1, 0), reserve_words(qn + 2, 0);
  uint64_t stack_words = 0;
  for (uint32_t w = 2; w < qn; ++w) {
    fixed_rows[w] = std::max<uint64_t>(lb / (4ull * w), min_rows);
    stack_words += (fixed_rows[w] * w + 3) & ~3ull;
  }
  for (uint32_t w = qn - 1; w >= 2; --w) reserve_words[w] = reserve_words[w + 1] + ((min_rows * w + 3) & ~3ull);
  uint32_t* stack = qn > 2 ? arena_alloc<uint32_t>(ws, stack_words) : nullptr;
  uint32_t* const stack_end = stack ? stack + stack_words : nullptr;
  if (qn > 2) L[2].buf = stack;
  uint64_t res_cap = std::max<uint64_t>(std::min<uint64_t>(opt.result_rows, cap), 1);
  if (qn > 1) res_cap = std::max<uint64_t>(res_cap, std::min<uint64_t>(cap, min_rows));
  // rows bound for a page-locked block get two result buffers: the joins
  // fill one while the other is copied out on the copy stream. With
  // deferred copies they are the workspace's persistent pair, whose copies
  // from the previous query may still run: the stream waits for them.
  const bool async_rows = opt.collect_rows && !opt.keep_on_device && R.host_rows.pinned();
  const bool ring = async_rows && opt.defer_copies && ws.res_ring_words &&
                    std::min<uint64_t>(res_cap, ws.res_ring_words / qn) >= std::min<uint64_t>(cap, min_rows);
  uint32_t* res_bufs[2] = {nullptr, nullptr};
  if (ring) {
    res_cap = std::min<uint64_t>(res_cap, ws.res_ring_words / qn);
    res_bufs[0] = ws.res_ring[0];
    res_bufs[1] = ws.res_ring[1];
    GPSM_CUDA(cudaStreamWaitEvent(s, ws.ev_copied[0], 0));
    GPSM_CUDA(cudaStreamWaitEvent(s, ws.ev_copied[1], 0));
  } else {
    res_bufs[0] = arena_alloc<uint32_t>(ws, res_cap * qn);
    if (async_rows) res_bufs[1] = (uint32_t*)ws.arena.alloc(std::max<uint64_t>(res_cap * qn, 1) * sizeof(uint32_t));
  }
  uint32_t* res_buf = res_bufs[0];
  int res_cur = 0;
  // directed mode: final rows land in a staging buffer and only those whose
  // query edges are directed, labelled data edges move to the result
  uint32_t* stage = nullptr;
  uint64_t stage_rows = 0;
  uint32_t* d_checks = nullptr;
  unsigned long long* d_kept = nullptr;
  uint32_t nchecks = 0;
  if (opt.directed) {
    if (!g.dir_off) {
      set_last_error("directed mode needs gpsm_graph_set_directed");
      return GPSM_ERR_STATE;
    }
    stage_rows = std::max<uint64_t>(opt.level_bytes / (4ull * qn), min_rows);
    stage = arena_alloc<uint32_t>(ws, stage_rows * qn);
    std::vector<uint32_t> chk;
    for (uint32_t k = 0; k < Q.m; ++k) {  // every query edge a -> b (file order) with its label
      chk.push_back((uint32_t)R.id2pos[Q.fe_from[k]]);
      chk.push_back((uint32_t)R.id2pos[Q.fe_to[k]]);
      chk.push_back(k < opt.edge_labels.size() ? opt.edge_labels[k] : 1u);
    }
    nchecks = (uint32_t)(chk.size() / 3);
    d_checks = arena_alloc<uint32_t>(ws, chk.size() + 1);
    d_kept = arena_alloc<unsigned long long>(ws, 1);
    if (!chk.empty()) GPSM_CUDA(cudaMemcpyAsync(d_checks, chk.data(), chk.size() * 4, cudaMemcpyHostToDevice, s));
    stream_wait(ws);
  }
  uint64_t res_used = 0, emitted = 0;
  bool capped = false;

  auto flush = [&]() {
    if (!opt.collect_rows || res_used == 0) {
      res_used = 0;
      return;
    }
    const uint64_t words = res_used * qn;
    res_used = 0;
    if (res_bufs[1]) {
      GPSM_CUDA(cudaEventRecord(ws.ev_res[res_cur], s));
      if (R.host_rows.append_from_device_async(ws, res_buf, words, ws.ev_res[res_cur], ws.ev_copied[res_cur])) {
        res_cur ^= 1;
        res_buf = res_bufs[res_cur];
        // the other buffer's earlier copy ends before new rows land in it
        GPSM_CUDA(cudaStreamWaitEvent(s, ws.ev_copied[res_cur], 0));
        return;
      }
      GPSM_CUDA(cudaStreamSynchronize(ws.copy_stream));  // no copy may be pending into a block that moves
    }
    R.host_rows.append_from_device(ws, res_buf, words);
  };

  if (qn == 1) {
    // single-vertex query: every candidate is an embedding
    const uint64_t n1 = std::min<uint64_t>(L[1].nrows, cap);
    capped = L[1].nrows >= cap;
    if (n1 > 0)
      GPSM_CUDA(cudaMemcpyAsync(res_buf, L[1].buf, std::min(n1, res_cap) * 4, cudaMemcpyDeviceToDevice, s));
    if (n1 > res_cap) {
      if (opt.keep_on_device) {
        set_last_error("device result buffer full");
        return GPSM_ERR_BUDGET;
      }
      if (opt.collect_rows) {
        R.host_rows.clear();
        R.host_rows.append_from_device(ws, L[1].buf, n1);
      }
    } else {
      res_used = n1;
    }
    emitted = n1;
    R.stats.level_rows[1] = n1;
  }
  bool safe_step = false;  // the next step admits no more candidates than its output holds rows
  // GPSM_DEBUG_WIDE_STEPS=1: every intermediate step admits 16 times the
  // candidates its output holds rows, so every step that keeps more than a
  // sixteenth of them ends at a row boundary (a test of that path: the rows
  // must not change)
  const bool wide_steps = [] {
    const char* e = getenv("GPSM_DEBUG_WIDE_STEPS");
    return e && e[0] == '1';
  }();
  // GPSM_DEBUG_NO_EDGE_HASH=1: search the candidate-edge lists even when the
  // graph has its edge table (the two must give the same rows)
  const bool use_hash = [] {
    const char* e = getenv("GPSM_DEBUG_NO_EDGE_HASH");
    return !(e && e[0] == '1');
  }();
  while (qn > 1 && !capped) {
    // deepest level with rows left
    int lv = -1;
    for (int w = (int)qn - 1; w >= 1; --w)
      if (L[w].next < L[w].nrows) {
        lv = w;
        break;
      }
    if (lv < 0) break;
    Level& A = L[lv];
    const bool final_level = (uint32_t)lv + 1 == qn;
    uint32_t* out;
    uint64_t out_cap, budget;
    bool partial = false;
    bool cut_rows = false;
    if (final_level && opt.directed) {
      uint64_t space = res_cap - res_used;
      if (space == 0) {
        if (opt.keep_on_device) {
          set_last_error("device result buffer full");
          return GPSM_ERR_BUDGET;
        }
        flush();
        space = res_cap;
      }
      out = stage;
      out_cap = std::min<uint64_t>(stage_rows, space);
      budget = std::min<uint64_t>(out_cap, opt.step_cands);
    } else if (final_level) {
      uint64_t space = res_cap - res_used;
      if (!opt.keep_on_device && res_used > 0 && cap - emitted > space &&
          space < std::min<uint64_t>(res_cap, opt.step_cands) / 2) {
        flush();  // a step into the little space left would be a small one
        space = res_cap;
      }
      out = res_buf + res_used * qn;
      if (cap - emitted <= space) {
        // the cap ends the query inside this buffer: rows past it are cut
        out_cap = cap - emitted;
        partial = true;
        budget = std::min<uint64_t>(std::max<uint64_t>(out_cap, min_rows), opt.step_cands);
      } else {
        out_cap = space;
        budget = std::min<uint64_t>(space, opt.step_cands);
      }
    } else {
      Level& B = L[lv + 1];
      const uint32_t wb = (uint32_t)lv + 1;
      B.nrows = 0;
      B.next = 0;
      if (lv >= 2) B.buf = L[lv].buf + ((L[lv].nrows * (uint64_t)lv + 3) & ~3ull);  // after level lv's rows
      const uint64_t room = (uint64_t)(stack_end - B.buf);
      const uint64_t free_rows = room > reserve_words[wb + 1] ? (room - reserve_words[wb + 1]) / wb : 0;
      // the step's room beyond its own buffer grows with the attempt's work:
      // one doubling per doubling of the candidates scanned past 2^26
      uint64_t ramp = fixed_rows[wb];
      for (uint64_t c = cands_total >> 26; c > 0 && ramp < free_rows; c >>= 1) ramp *= 2;
      out = B.buf;
      out_cap = std::min<uint64_t>(free_rows, std::max<uint64_t>(fixed_rows[wb], ramp));
      if (out_cap < min_rows) {
        set_last_error("join level stack exhausted");
        return GPSM_ERR_BUDGET;
      }
      B.cap_rows = out_cap;
      // a level that keeps few of its candidates (dense steps: other placed
      // neighbours' lists reject most) may admit up to out_cap / keep of
      // them; if more rows are kept than out_cap after all, the write pass
      // ends the step at a row boundary and the rest are offered again
      const double keep = wide_steps ? 1.0 / 16.0 : A.keep;
      budget = std::min<uint64_t>(opt.step_cands, safe_step ? out_cap : (uint64_t)((double)out_cap / keep));
      budget = std::max<uint64_t>(budget, std::min<uint64_t>(out_cap, opt.step_cands));
      cut_rows = budget > out_cap;
    }
    // rows offered to this step: enough to fill the budget at the observed
    // candidates per row, within the per-row scratch
    uint64_t want = (uint64_t)(1.25 * (double)budget / std::max(A.ratio, 1.0 / 1024.0)) + 256;
    want = std::min<uint64_t>(want, js.rows);
    const uint64_t rb = A.next, re = std::min<uint64_t>(A.nrows, A.next + want);
    StepState* d_st = d_st2 + st_turn;
    StepState* d_next = d_st2 + (st_turn ^ 1);
    st_turn ^= 1;
    *h_st = StepState{};  // the stream is idle: the step's write pass refills it
    GPSM_CUDA(cudaEventRecord(ws.eve0, s));
    launch_join_step(ws, A.buf, (uint32_t)lv, rb, re, d_back + back_off[lv], back_cnt[lv], nbrs_total, budget, out,
                     out_cap, js, d_st, d_next, d_inj + inj_off[lv], inj_cnt[lv], cut_rows, h_st_dev,
                     use_hash ? g.ehash : nullptr, g.ehash_bits, g.ehash_probe);
    safe_step = false;
    GPSM_CUDA(cudaEventRecord(ws.eve1, s));
    exp_launches += 4;  // locate, check, scan, write
    ++R.stats.join_steps;
    stream_wait(ws);  // the write pass filled h_st
    {
      float ems = 0;
      GPSM_CUDA(cudaEventElapsedTime(&ems, ws.eve0, ws.eve1));
      R.stats.expand_ms += ems;
    }
    const uint64_t admitted = h_st->rows, written = h_st->written, cands = h_st->cands;
    const bool was_cut = h_st->cut != 0;
    const uint64_t cands_done = was_cut ? h_st->cands_done : cands;  // candidates of the rows written whole
    if (trace_enabled()) {
      float ems = 0;
      cudaEventElapsedTime(&ems, ws.eve0, ws.eve1);
      const unsigned long long ab = admitted * 4ull * lv + admitted * 24ull * back_cnt[lv] + cands * 4ull +
                                    written * 4ull * (lv + 1);
      fprintf(stderr,
              "[gpsm] step level=%d nb=%u rows=[%llu,%llu) admitted=%llu cands=%llu written=%llu budget=%llu "
              "alg_bytes=%llu ms=%.3f%s\n",
              lv, back_cnt[lv], (unsigned long long)rb, (unsigned long long)re, (unsigned long long)admitted,
              (unsigned long long)cands, (unsigned long long)written, (unsigned long long)budget, ab, ems,
              was_cut ? " cut" : "");
    }
    if (was_cut) ++R.stats.cut_steps;
    if (was_cut && admitted == 0) {
      // the first row alone keeps more than the output holds at this budget:
      // offer it again with no more candidates than rows fit (the checked
      // candidates still count as work)
      cands_total += cands;
      R.stats.cands_scanned += cands;
      A.keep = 1.0;
      safe_step = true;
      if (limit && cands_total >= limit) {
        hit_limit = true;
        break;
      }
      continue;
    }
    if (admitted == 0) {
      if (final_level && !partial && res_used > 0) {  // make room and retry
        if (opt.keep_on_device) {
          set_last_error("device result buffer full");
          return GPSM_ERR_BUDGET;
        }
        flush();
        continue;
      }
      set_last_error("a single row has more candidates than a join step admits");
      return GPSM_ERR_BUDGET;
    }
    A.ratio = std::max(1.0 / 1024.0, (double)cands_done / (double)admitted);
    if (!final_level && cands_done > 0)  // kept share with 1.5x headroom, at least 1/64
      A.keep = std::min(1.0, std::max(1.0 / 64.0, 1.5 * (double)written / (double)cands_done));
    A.next = rb + admitted;
    alg_bytes += admitted * 4ull * lv + admitted * 24ull * back_cnt[lv] + cands * 4ull + written * 4ull * (lv + 1);
    uint64_t kept = written;
    if (final_level && opt.directed && written) {
      launch_verify_directed(ws, stage, written, qn, d_checks, nchecks, g.dir_off, g.dir_col, g.dir_lab,
                             res_buf + res_used * qn, d_kept);
      small_to_host(ws, &h_st->verified, d_kept, sizeof(unsigned long long));
      stream_wait(ws);
      kept = std::min<uint64_t>(h_st->verified, cap - emitted);  // the cap counts rows that pass
      ++exp_launches;
    }
    R.stats.level_rows[lv + 1] += written;
    R.stats.level_in[lv] += admitted;
    R.stats.level_cands[lv] += cands;
    cands_total += cands;
    R.stats.cands_scanned += cands;
    if (limit && cands_total >= limit) {
      hit_limit = true;
      if (final_level) {
        res_used += kept;
        emitted += kept;
      }
      break;
    }
    if (final_level) {
      res_used += kept;
      emitted += kept;
      if (emitted >= cap) capped = true;
    } else {
      L[lv + 1].nrows = written;
    }
  }
  if (emitted >= cap) capped = true;
  R.rows = emitted;
  R.capped = capped;
  GPSM_CUDA(cudaEventRecord(ws.ev1, s));
  if (opt.collect_rows && !opt.keep_on_device) {
    flush();
  } else {
    R.d_rows = res_buf;
    R.d_rows_count = res_used;
  }
  if (ring) {  // the caller waits for the copies (run_query hands them on)
    copies_done.armed = false;
    R.copies_pending = true;
  }
  return GPSM_OK;
}

// One query: filter (run_filter), join order, admission, then join attempts
// (join_attempt; the learned plan and the plain order take turns when they
// race).
int run_query(Workspace& ws, const DeviceGraph& g, const QueryPlan& Q, const MatchOptions& opt, MatchResult& R) {
  R = MatchResult();
  const uint32_t qn = Q.n;
  cudaStream_t s = ws.stream;
  if (ws.dirty) {
    // an earlier query stopped part-way: re-read the scan ticket counter so
    // the host's per-launch ticket base matches the device again
    stream_wait(ws);
    GPSM_CUDA(cudaMemcpy(&ws.scan.ticket_base, ws.scan.d_ticket, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  }
  ws.dirty = true;
  ws.arena.reset();
  if (opt.defer_copies && opt.collect_rows && !opt.keep_on_device) ws.result_ring();
  // copies still running into R.host_rows end before any path but the
  // successful one leaves (that one hands them to the caller as an event)
  struct PendingCopies {
    Workspace& w;
    MatchResult& r;
    ~PendingCopies() {
      if (r.copies_pending) cudaStreamSynchronize(w.copy_stream);
      r.copies_pending = false;
    }
  } pending_copies{ws, R};
  R.cols = qn;
  GPSM_CUDA(cudaEventRecord(ws.ev0, s));
  GPSM_CUDA(cudaMemsetAsync(ws.d_flags, 0, 64 * sizeof(uint32_t), s));

  FilterProducts F;
  int rc = run_filter(ws, g, Q, R, F);
  if (rc != GPSM_OK || R.empty_filter) return rc;
  const std::vector<uint32_t>& cnt = F.cnt;

  // ---- join order -------------------------------------------------------------
  std::vector<int32_t> pos2id;
  std::vector<int32_t> race;  // the plain order, when a learned plan runs against it
  if (opt.order_mode == ORDER_GIVEN) {
    if (!valid_order(Q, opt.given_order)) {
      set_last_error("given join order is not a connected permutation of the query vertices");
      return GPSM_ERR_INVALID;
    }
    pos2id = opt.given_order;
  } else if (opt.order_mode == ORDER_LEARNED && qn > 2 && qn <= (uint32_t)kMaxPlanQ) {
    if (!opt.model) {
      set_last_error("learned order requested without a model");
      return GPSM_ERR_INVALID;
    }
    const auto tp0 = std::chrono::steady_clock::now();
    const std::vector<int32_t> plain = plain_order(Q, R.stats.size_fwd, g.nnz);
    pos2id = learned_order(ws, g, Q, cnt, R.stats.size_fwd, R.stats.size_rev, plain, opt, R.stats);
    if (pos2id.empty()) pos2id = plain;
    else if (pos2id != plain) race = plain;
    R.stats.plan_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - tp0).count();
  } else {
    pos2id = plain_order(Q, R.stats.size_fwd, g.nnz);
  }
  R.pos2id = pos2id;
  R.id2pos.assign(qn, -1);
  for (uint32_t p = 0; p < qn; ++p) R.id2pos[pos2id[p]] = (int32_t)p;
  GPSM_CUDA(cudaEventRecord(ws.evm, s));
  if (opt.filter_only) {
    stream_wait(ws);
    return GPSM_OK;
  }
  // join memory: level buffers, step scratch and the result buffer are the
  // most the joins can hold; a learned plan predicts how much of it is used
  struct AdmitGuard {
    const MatchOptions& o;
    uint64_t bytes = 0;
    ~AdmitGuard() {
      if (bytes && o.release) o.release(o.admit_ctx, bytes);
    }
  } admit_guard{opt};
  if (opt.admit) {
    const uint64_t min_rows_a = (uint64_t)g.max_degree + 64;
    uint64_t cap_bytes = 0;
    const uint64_t lb = level_buffer_bytes(ws, opt, qn);
    for (uint32_t w = 2; w < qn; ++w)
      cap_bytes += std::max<uint64_t>(lb, min_rows_a * 4ull * w);
    const uint64_t res_rows =
        std::max<uint64_t>(std::min<uint64_t>(std::max<uint64_t>(opt.result_rows, opt.keep_on_device ? opt.cap : 0),
                                              opt.cap),
                           1);
    const uint64_t res_bytes = res_rows * 4ull * qn;
    cap_bytes += res_bytes + (1ull << 30);
    uint64_t want = cap_bytes;
    if (opt.order_mode == ORDER_LEARNED && !R.stats.order_fallback && R.stats.predicted_peak > 0)
      want = std::min<uint64_t>(cap_bytes, (uint64_t)R.stats.predicted_peak + res_bytes + (64ull << 20));
    if (!opt.admit(opt.admit_ctx, want)) {
      set_last_error("admission refused: predicted join memory does not fit the budget");
      return GPSM_ERR_BUDGET;
    }
    admit_guard.bytes = want;
    R.stats.admitted_bytes = want;
  }

  // ---- joins ---------------------------------------------------------------------
  JoinContext ctx{ws, g, Q, opt, R, F, pos2id, ws.arena.used};
  int jrc = GPSM_OK;
  bool hit = false;
  if (race.empty()) {
    jrc = join_attempt(ctx, opt.work_cap, hit);
    R.stats.aborted = hit;
  } else {
    // the learned plan and the plain order take turns with work shares that
    // grow by 4 each round, until one finishes; the total work stays within
    // a small factor of the cheaper order's, so a plan the model got wrong
    // costs a bounded share instead of its whole blowup
    // opt.work_cap bounds the query's candidates over all attempts together
    const std::vector<int32_t> learned_plan = pos2id;
    uint64_t share = tuning().race_share;
    for (uint32_t a = 0;; ++a) {
      const bool learned_turn = (a % 2) == 0;
      pos2id = learned_turn ? learned_plan : race;
      uint64_t limit = share;
      bool last = share >= (1ull << 60);
      if (opt.work_cap) {
        const uint64_t used = R.stats.cands_scanned;
        const uint64_t left = opt.work_cap > used ? opt.work_cap - used : 0;
        if (left <= share) {
          limit = left;
          last = true;
        }
        if (limit == 0) {  // the previous attempt used the whole cap: it stands, stopped
          R.stats.aborted = true;
          break;
        }
      }
      ++R.stats.order_attempts;
      jrc = join_attempt(ctx, limit, hit);
      if (jrc != GPSM_OK || !hit || last) {
        R.stats.aborted = hit;
        if (!learned_turn) R.stats.order_fallback = 3;
        break;
      }
      if (!learned_turn) share *= 4;
    }
  }
  R.stats.expand_launches = ctx.exp_launches;
  R.stats.alg_bytes_join = ctx.alg_bytes;
  if (jrc != GPSM_OK) return jrc;
  small_to_host(ws, ws.h_small + 4001, ws.d_flags, sizeof(uint32_t));
  GPSM_CUDA(cudaEventSynchronize(ws.ev1));
  stream_wait(ws);
  if (*reinterpret_cast<uint32_t*>(ws.h_small + 4001) & (DF_SCAN_TIMEOUT | DF_BOUNDS)) {
    set_last_error("device wait limit or bounds check tripped in the joins");
    return GPSM_ERR_TIMEOUT;
  }
  ws.dirty = false;
  float ms = 0, ms_f = 0;
  GPSM_CUDA(cudaEventElapsedTime(&ms, ws.ev0, ws.ev1));
  GPSM_CUDA(cudaEventElapsedTime(&ms_f, ws.ev0, ws.evm));
  R.stats.device_ms = ms;
  R.stats.filter_ms = ms_f;
  R.stats.join_ms = ms - ms_f;
  if (R.copies_pending) {
    GPSM_CUDA(cudaEventCreateWithFlags(&R.copies_done, cudaEventDisableTiming | cudaEventBlockingSync));
    GPSM_CUDA(cudaEventRecord(R.copies_done, ws.copy_stream));
    R.copies_pending = false;
  }
  return GPSM_OK;
}

}  // namespace gpsm
