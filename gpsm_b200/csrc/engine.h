// Host-side engine: query planning and the per-query device pipeline.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "filter.h"
#include "internal.h"

namespace gpsm {

DeviceGraph* graph_upload(int device, const uint32_t* off, const uint32_t* col, const uint32_t* lab, uint32_t n);
void graph_free(DeviceGraph* g);
// CSR built on the device from m undirected edges (csr_build.cu); ws supplies scratch
DeviceGraph* graph_build(Workspace& ws, const uint32_t* edges, uint64_t m, const uint32_t* lab, uint32_t n);
void graph_download(const DeviceGraph* g, uint32_t* off, uint32_t* col);
// attaches the directed, edge-labelled data edges (m pairs (from, to) + labels or NULL = 1)
void graph_set_directed(DeviceGraph* g, uint64_t m, const uint32_t* edges, const uint32_t* labels);
void launch_verify_directed(Workspace& ws, const uint32_t* in, uint64_t nrows, uint32_t cols, const uint32_t* d_checks,
                            uint32_t nchecks, const uint32_t* off, const uint32_t* col, const uint32_t* lab,
                            uint32_t* out, unsigned long long* d_kept);
Workspace* workspace_create(int device, size_t arena_bytes, uint32_t max_tiles);
void workspace_free(Workspace* ws);

// The query as the reference's Graph/Match classes see it.
struct QueryPlan {
  uint32_t n = 0, m = 0;
  std::vector<uint32_t> lab;
  std::vector<std::vector<uint32_t>> in, out;  // file-order directed lists (graph/Graph.cpp:20-24)
  std::vector<uint32_t> roff, rcol;             // undirected CSR, lists sorted (graph/Graph.cpp:30-65)
  std::vector<uint32_t> efrom, eto;             // edge ids (match/Match.cu:1738-1754), from < to
  std::vector<uint32_t> order;                  // filter order (match/Match.cu:339-429)
  std::vector<uint32_t> fe_from, fe_to;         // edges as given (file order, directed)
  uint32_t deg(uint32_t u) const { return roff[u + 1] - roff[u]; }
  bool adjacent(uint32_t a, uint32_t b) const;
  int edge_between(uint32_t a, uint32_t b) const;  // edge id or -1
};

// Builds the plan; returns GPSM_OK or an error with `err` filled.
int plan_query(const DeviceGraph& g, uint32_t qn, const uint32_t* qlab, uint32_t qm, const uint32_t* qe,
               QueryPlan& Q, std::string& err);

// Reference join order from forward candidate-edge sizes
// (match/Match.cu:1599-1694), restricted to edges with a visited endpoint.
std::vector<int32_t> plain_order(const QueryPlan& Q, const std::vector<uint64_t>& size_fwd, uint64_t nnz);
// true when `pos2id` is a permutation in which every vertex after the first
// has an earlier neighbour.
bool valid_order(const QueryPlan& Q, const std::vector<int32_t>& pos2id);

enum OrderMode : int { ORDER_PLAIN = 0, ORDER_GIVEN = 1, ORDER_LEARNED = 2 };

struct Model;  // learned.cu
Model* model_create(int device, uint64_t seed);
void model_free(Model* M);
void model_set(Model* M, const float* w);
void model_get(Model* M, float* w);
float model_grad(Model* M, const float* x, const float* y, uint32_t n, float* grad);
float model_train(Model* M, const float* x, const float* y, uint32_t n, uint32_t epochs, uint32_t batch, float lr,
                  uint64_t seed);
void model_predict(Model* M, const float* x, uint32_t n, float* y);

struct MatchOptions {
  uint64_t cap = ~0ULL;            // embedding cap (rows after which the query stops)
  int order_mode = ORDER_PLAIN;
  std::vector<int32_t> given_order;  // pos2id when ORDER_GIVEN
  uint64_t level_bytes = tuning().level_bytes;  // per intermediate level buffer
  uint64_t result_rows = 1ull << 22;    // device result buffer rows before flushing to host
  uint64_t step_rows = 1ull << 22;      // input rows one join step may look at
  uint64_t step_cands = tuning().step_cands;  // candidates one join step may admit
  bool keep_on_device = false;          // never flush: fail with GPSM_ERR_BUDGET instead
  bool collect_rows = true;             // false: count only (result rows are discarded)
  bool filter_only = false;             // stop after the join order (debug entry points)
  Model* model = nullptr;               // ORDER_LEARNED
  bool directed = false;                // keep rows whose query edges exist as directed, labelled data edges
  std::vector<uint32_t> edge_labels;    // per query edge in file order (empty = all 1)
  uint64_t memory_budget = 0;           // bytes; predicted peak above it -> plain order (0 = arena size)
  uint64_t work_cap = 0;                // candidates the joins may scan before stopping, all attempts (0 = none)
  // Rows bound for a page-locked block leave through the workspace's two
  // persistent result buffers, and run_query returns while the last copies
  // are still running: R.copies_done is then an event the caller waits on
  // (and destroys) before reading R.host_rows. The next query on the same
  // workspace waits for those copies on the device before writing the
  // buffers, so the slot's next filter overlaps them.
  bool defer_copies = false;
  // Admission hook (serving): called after the order is chosen, before the
  // joins, with the bytes the joins are predicted to use; returns false to
  // refuse (GPSM_ERR_BUDGET). release() gets the same bytes back afterwards.
  bool (*admit)(void* ctx, uint64_t bytes) = nullptr;
  void (*release)(void* ctx, uint64_t bytes) = nullptr;
  void* admit_ctx = nullptr;
};

struct MatchStats {
  std::vector<uint32_t> cand_count;      // final |C(u)|
  std::vector<uint64_t> size_fwd, size_rev;  // candidate-edge totals per edge id
  std::vector<uint64_t> level_rows;      // rows produced at each table width 1..n
  std::vector<uint64_t> level_in;        // rows of width w extended (admitted) by join steps
  std::vector<uint64_t> level_cands;     // candidates scanned when extending width w
  uint64_t expand_launches = 0;
  uint64_t join_steps = 0;      // join steps (each: locate, check, scan, write)
  uint64_t cut_steps = 0;       // steps the write pass ended at a row boundary
  uint64_t filter_launches = 0;
  double device_ms = 0;
  double filter_ms = 0, join_ms = 0;
  uint64_t alg_bytes_join = 0;  // algorithmic bytes of the join phase
  double expand_ms = 0;         // summed device time of the join launches
  double plan_ms = 0;           // learned-order planning (host wall time incl. the planner kernel)
  double predicted_work = 0, predicted_peak = 0;
  double predicted_work_plain = 0;  // the model's work estimate for the plain order
  int order_fallback = 0;  // 1: learned order over the memory budget; 2: not predicted cheaper than plain;
                           // 3: raced the plain order, which finished first
  uint32_t order_attempts = 0;  // join attempts when a learned plan raced the plain order
  uint64_t cands_scanned = 0;   // candidates the joins scanned, over all attempts
  uint64_t admitted_bytes = 0;  // bytes granted by the admission hook
  bool aborted = false;         // work cap reached
  uint64_t alg_bytes_filter = 0;
};

// Result rows on the host: either a page-locked block from the library's
// pool (reserve_pinned; the device copies into it directly) or a malloc'd
// block grown with realloc and never zero-filled. A caller takes the block
// with release() and gives it back with host_free (gpsm_free).
class HostRows {
 public:
  HostRows() = default;
  HostRows(const HostRows&) = delete;
  HostRows& operator=(const HostRows&) = delete;
  HostRows(HostRows&& o) noexcept : p_(o.p_), n_(o.n_), cap_(o.cap_), pinned_(o.pinned_) {
    o.p_ = nullptr, o.n_ = o.cap_ = 0, o.pinned_ = false;
  }
  HostRows& operator=(HostRows&& o) noexcept;
  ~HostRows();
  uint64_t size() const { return n_; }  // words
  bool pinned() const { return pinned_; }
  bool empty() const { return n_ == 0; }
  const uint32_t* data() const { return p_; }
  void clear() { n_ = 0; }
  // take a pool block for `words` words if nothing is held yet (no-op when
  // the pool is at its limit)
  void reserve_pinned(uint64_t words);
  // room for `words` more words at the end; the size grows by that much
  uint32_t* append(uint64_t words);
  // append `words` words copied from device memory on ws's stream
  void append_from_device(Workspace& ws, const uint32_t* d_src, uint64_t words);
  // the same on ws.copy_stream after `ready` (recorded on ws.stream), with
  // `done` recorded when the copy ends; only into a page-locked block that
  // already has room (returns false otherwise, and copies nothing)
  bool append_from_device_async(Workspace& ws, const uint32_t* d_src, uint64_t words, cudaEvent_t ready,
                                cudaEvent_t done);
  uint32_t* release() {
    uint32_t* q = p_;
    p_ = nullptr, n_ = cap_ = 0, pinned_ = false;
    return q;
  }

 private:
  uint32_t* p_ = nullptr;
  uint64_t n_ = 0, cap_ = 0;
  bool pinned_ = false;
};

// Frees a result block: back to the pool if it came from there, else free().
void host_free(void* p);
void host_pool_stats(uint64_t* blocks, uint64_t* pinned_bytes, uint64_t* grown, double* grow_ms);

struct MatchResult {
  uint64_t rows = 0;
  uint32_t cols = 0;
  bool capped = false;
  bool empty_filter = false;        // a candidate set ran empty (no embeddings)
  std::vector<int32_t> id2pos, pos2id;
  HostRows host_rows;               // flushed rows (row-major, table column order)
  uint32_t* d_rows = nullptr;       // rows still on the device (arena memory; valid until the next query)
  uint64_t d_rows_count = 0;        // rows in d_rows (after host_rows)
  MatchStats stats;
  bool copies_pending = false;      // copies into host_rows may still run on the copy stream
  cudaEvent_t copies_done = nullptr;  // defer_copies: recorded after the last copy (the caller destroys it)
};

int run_query(Workspace& ws, const DeviceGraph& g, const QueryPlan& Q, const MatchOptions& opt, MatchResult& R);

struct PlanQuery;
struct PlanEdges;
// Planner inputs from the filter statistics (learned.h).
void build_plan_inputs(const DeviceGraph& g, const QueryPlan& Q, const std::vector<uint32_t>& cand,
                       const std::vector<uint64_t>& size_fwd, const std::vector<uint64_t>& size_rev, PlanQuery& PQ,
                       PlanEdges& PE);
// Features of every step of the order pos2id ((n-1) x kFeat floats).
void order_features(const PlanQuery& PQ, const PlanEdges& PE, const std::vector<int32_t>& pos2id, float* out);

// vertices with `label` and degree >= min_degree, ascending (select.cu)
uint32_t select_words(uint32_t n);
void select_vertices(Workspace& ws, const uint32_t* d_labels, const uint32_t* d_offsets, uint32_t n, uint32_t label,
                     uint32_t min_degree, uint32_t* bm, uint32_t* d_out, uint32_t* d_count);

}  // namespace gpsm
