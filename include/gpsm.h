/* gpsm.h - C ABI of the B200 subgraph-matching engine (libgpsm.so).
 *
 * Plain pointers and sizes only. Every entry point returns an int status
 * (GPSM_OK or a negative GPSM_ERR_*); the reference instead calls exit(1) on
 * any CUDA error (match/Match.h:53-65).
 *
 * Conventions shared with the reference's file format and classes:
 *   - vertex ids are 0-based, labels are 1-based unsigned (README.md);
 *   - a data graph is an undirected CSR: offsets[n+1], cols[offsets[n]] with
 *     every adjacency list sorted ascending (graph/Graph.cpp:30-65);
 *   - a query is (qn labels, qm edges as (from, to) pairs in file order),
 *     exactly what io/IO.cpp:46-128 reads from `v`/`e` lines.
 * Embeddings are non-induced, injective, undirected and edge-unlabelled.
 */
#ifndef GPSM_H
#define GPSM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define GPSM_OK 0
#define GPSM_ERR_INVALID -1   /* bad argument or malformed graph */
#define GPSM_ERR_CUDA -2      /* a CUDA runtime call failed */
#define GPSM_ERR_NOMEM -3     /* device or host allocation failed */
#define GPSM_ERR_NOT_FOUND -4 /* generator could not find a query */
#define GPSM_ERR_BUDGET -5    /* request exceeds the memory budget */
#define GPSM_ERR_TIMEOUT -6   /* a bounded device-side wait gave up */
#define GPSM_ERR_NODEV -7     /* no CUDA device */
#define GPSM_ERR_STATE -8     /* call order violated (e.g. no gpsm_init) */

/* ---- synthetic workloads (host) --------------------------------------- */
/* Erdos-Renyi G(n, m): m unique undirected edges (u < v), no self loops.
 * edges: 2*m uint32. */
int gpsm_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t* edges);
/* R-MAT over 2^scale vertices with quadrant probabilities a, b, c
 * (d = 1-a-b-c): exactly m unique undirected edges, no self loops, vertex ids
 * randomly permuted. edges: 2*m uint32, each pair (min, max). */
int gpsm_gen_rmat(int scale, uint64_t m, double a, double b, double c, uint64_t seed,
                  uint32_t* edges);
/* i.i.d. vertex labels in 1..num_labels with P(k) ~ k^-zipf_s (0 = uniform). */
int gpsm_gen_labels(uint32_t n, uint32_t num_labels, double zipf_s, uint64_t seed,
                    uint32_t* labels);
/* Undirected CSR from m undirected edges; each list sorted ascending.
 * offsets: n+1, cols: 2*m. Replaces Graph::transformToCSR (graph/Graph.cpp:30-65). */
int gpsm_csr_from_edges(uint32_t n, uint64_t m, const uint32_t* edges, uint32_t* offsets,
                        uint32_t* cols);
/* Random-walk query of qn vertices (mode 0 induced, 1 tree, 2 dense with
 * p_extra). q_labels: qn; q_edges: qn*(qn-1) uint32; q_data_ids: qn or NULL.
 * Returns the number of query edges (>= 0) or a negative status. */
int64_t gpsm_gen_query(uint32_t n, const uint32_t* offsets, const uint32_t* cols,
                       const uint32_t* labels, uint32_t qn, int mode, double p_extra,
                       double min_avg_degree, uint64_t seed, uint32_t* q_labels,
                       uint32_t* q_edges, uint32_t* q_data_ids);

/* ---- the reference's graph text format at full speed ------------------- */
/* io/IO.cpp:46-128 reads `t # id`, a counts line, `v id label`, `e from to
 * label`, ending with `t # -1`, one fscanf per token. These parse a whole
 * file from a memory map with one thread per chunk of lines; vertices are
 * numbered in file order (the `v` id is ignored, as Graph::addVertex does).
 */
typedef struct gpsm_text_s* gpsm_text_t;
int gpsm_text_open(const char* path, gpsm_text_t* out);
int gpsm_text_count(gpsm_text_t t, uint32_t* ngraphs);
int gpsm_text_graph_info(gpsm_text_t t, uint32_t k, uint32_t* n, uint64_t* m, int32_t* id);
/* labels[n]; edges[2m] (from, to) in file order; edge_labels[m] or NULL */
int gpsm_text_graph_read(gpsm_text_t t, uint32_t k, uint32_t* labels, uint32_t* edges,
                         uint32_t* edge_labels);
int gpsm_text_close(gpsm_text_t t);
/* Writes one graph (append != 0: after the file's contents); edge_labels
 * NULL writes label 1; terminate != 0 adds the closing `t # -1`. */
int gpsm_text_write(const char* path, int append, int32_t id, uint32_t n, const uint32_t* labels,
                    uint64_t m, const uint32_t* edges, const uint32_t* edge_labels, int terminate);

/* ---- engine: device, data graph, matching ------------------------------ */
typedef struct gpsm_graph_s* gpsm_graph_t;   /* device-resident data graph */
typedef struct gpsm_engine_s* gpsm_engine_t; /* stream + workspace on one device */

/* Text of the last error on the calling thread. */
const char* gpsm_last_error(void);

/* Selects device `dev` and creates the default engine (workspace arena of
 * arena_bytes; 0 = min(16 GiB, 60% of free memory), or GPSM_ARENA_GB).
 * Replaces Match::initGPU (match/Match.cu:15-70), which exits when no device
 * exists and reserves a 4 GB device heap for kernel-side new/delete. */
int gpsm_init(int dev);
int gpsm_init_ex(int dev, uint64_t arena_bytes);
int gpsm_shutdown(void);

/* Additional engines (one stream and arena each) for concurrent callers. */
int gpsm_engine_create(int dev, uint64_t arena_bytes, gpsm_engine_t* out);
int gpsm_engine_destroy(gpsm_engine_t e);

/* Uploads an undirected CSR (offsets[n+1], cols[offsets[n]], labels[n]) once;
 * every later query reuses it. Replaces Match::copyGraphToGPU
 * (match/Match.cu:128-143), which re-uploads the graph for every query. */
int gpsm_graph_upload(const uint32_t* offsets, const uint32_t* cols, const uint32_t* labels,
                      uint32_t n, gpsm_graph_t* out);
int gpsm_graph_free(gpsm_graph_t g);
/* Builds the undirected CSR on the device from m undirected edges (pairs,
 * each edge once) and labels[n]: Graph::transformToCSR's job
 * (graph/Graph.cpp:30-65) done by a device radix sort. Same arrays as
 * gpsm_csr_from_edges + gpsm_graph_upload. Scratch: the default engine. */
int gpsm_graph_build(const uint32_t* edges, uint64_t m, const uint32_t* labels, uint32_t n,
                     gpsm_graph_t* out);
/* Copies a device graph's CSR back (offsets[n+1], cols[offsets[n]]; either may be NULL). */
int gpsm_graph_download(gpsm_graph_t g, uint32_t* offsets, uint32_t* cols);
int gpsm_graph_info(gpsm_graph_t g, uint32_t* n, uint64_t* nnz, uint32_t* max_degree);
/* The edge table built at upload (no counterpart in the reference): slots
 * (0: not built, the joins search the candidate-edge lists) and the longest
 * probe a lookup needs. */
int gpsm_graph_edge_table(gpsm_graph_t g, uint64_t* slots, uint32_t* max_probe);
/* Attaches the data graph's directed, edge-labelled edges (m pairs (from, to)
 * as in the file, labels[m] or NULL = 1) for GPSM_F_DIRECTED. The reference
 * keeps them in Graph::vertices[].out (graph/Graph.cpp:20-24). */
int gpsm_graph_set_directed(gpsm_graph_t g, uint64_t m, const uint32_t* edges, const uint32_t* labels);

#define GPSM_ORDER_PLAIN 0 /* the reference's join order (match/Match.cu:1599-1694) */
#define GPSM_ORDER_GIVEN 1 /* opts.order gives the table columns (pos -> query vertex) */
#define GPSM_ORDER_LEARNED 2 /* opts.model chooses the order (plain order beyond the memory budget) */

typedef struct gpsm_model_s* gpsm_model_t; /* learned join-order model (MLP on one device) */

#define GPSM_F_COUNT_ONLY 1u      /* do not return rows (count and statistics only) */
#define GPSM_F_KEEP_ON_DEVICE 2u  /* rows stay in device memory; never spill to host */
#define GPSM_F_DIRECTED 4u        /* keep rows whose query edges a->b (label) are data edges
                                     row[a]->row[b] with that label: IO::verify on the device
                                     (io/IO.cpp:146-180); needs gpsm_graph_set_directed */
#define GPSM_F_LARGEST_FIRST 8u   /* gpsm_server_create: a free slot takes the queued request
                                     with the most query edges (then vertices) instead of the
                                     oldest; ties in submission order */

typedef struct gpsm_match_opts {
  uint64_t cap;          /* embedding cap: stop after the first `cap` rows; 0 = none */
  int32_t order_mode;    /* GPSM_ORDER_* */
  int32_t pad;
  const int32_t* order;  /* pos2id[qn] for GPSM_ORDER_GIVEN */
  uint64_t level_bytes;  /* bytes per intermediate join level; 0 = 256 MiB */
  uint64_t result_rows;  /* device result buffer rows; 0 = 4 Mi */
  uint32_t flags;        /* GPSM_F_* */
  uint32_t pad2;
  gpsm_model_t model;    /* GPSM_ORDER_LEARNED */
  uint64_t memory_budget; /* bytes: predicted peak table above it -> plain order (0 = workspace size) */
  uint64_t work_cap;     /* candidates the joins may scan before the query stops, over all of its
                            join attempts together (a learned plan racing the plain order); 0 = none */
  const uint32_t* edge_labels; /* GPSM_F_DIRECTED: label per query edge (NULL = 1) */
} gpsm_match_opts;

typedef struct gpsm_match_info {
  uint64_t rows;             /* embeddings returned (== cap when capped) */
  uint32_t cols;             /* query vertices */
  int32_t capped;            /* 1 when the cap stopped the query */
  int32_t empty_filter;      /* 1 when a candidate set ran empty */
  int32_t pad;
  double device_ms;          /* device time of the whole query */
  double filter_ms;          /* filter + candidate edges */
  double join_ms;            /* joins */
  uint64_t expand_launches;
  uint64_t filter_launches;
  uint64_t alg_bytes_join;   /* algorithmic bytes of the joins (roofline numerator) */
  double expand_ms;          /* summed device time of the join launches */
  double plan_ms;            /* learned-order planning */
  double predicted_work;     /* learned order: predicted rows over the intermediate tables (final table excluded) */
  double predicted_peak;     /* learned order: predicted peak table bytes */
  int32_t order_fallback;    /* plain order used instead of the learned plan: 1 its predicted join memory is
                                over the budget; 2 it is not predicted to scan under half the plain order's rows;
                                3 the two orders took turns with growing work shares and the plain order
                                finished first */
  int32_t aborted;           /* 1: work_cap stopped the joins (rows are a prefix) */
  double predicted_work_plain; /* learned order: the model's predicted work of the plain order */
  uint32_t order_attempts;   /* learned order: join attempts of the two orders (0: no race) */
  uint32_t pad2;
  uint64_t cands_scanned;    /* candidates the joins scanned, over all attempts */
  uint64_t cut_steps;        /* join steps that kept more rows than their output held and ended
                                at a row boundary (the rest offered again) */
} gpsm_match_info;

typedef struct gpsm_batch_info {
  double device_ms;          /* engine-stream events: first query start to last query end */
  double expand_ms;          /* summed device time of the join launches */
  double filter_ms;          /* summed filter + candidate-edge time */
  uint64_t rows;             /* embeddings over the batch */
  uint64_t launches;         /* kernels launched by the batch */
  uint64_t expand_launches;
  uint64_t alg_bytes_join;
  uint64_t join_steps;       /* join steps (each: locate, check, scan, write launches) */
} gpsm_batch_info;

/* Matches one query. Replaces Match::match (match/Match.cu:1710-1966).
 * Rows are row-major with qn columns in table-column order; column p holds
 * query vertex pos2id[p], so query vertex j of row r is
 * rows[r*qn + id_map[j]] (the reference's id_map convention, run.cpp:76-84).
 * *out_rows is malloc'd (free with gpsm_free); NULL out_rows = count only.
 * id_map and pos2id (qn entries each) may be NULL. */
int gpsm_match_ex(gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm,
                  const uint32_t* q_edges, const gpsm_match_opts* opts, uint32_t** out_rows,
                  int32_t* id_map, int32_t* pos2id, gpsm_match_info* info);
int gpsm_engine_match(gpsm_engine_t e, gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels,
                      uint32_t qm, const uint32_t* q_edges, const gpsm_match_opts* opts,
                      uint32_t** out_rows, int32_t* id_map, int32_t* pos2id, gpsm_match_info* info);
/* Shorthand: plain order, optional cap (0 = none). */
int gpsm_match(gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm,
               const uint32_t* q_edges, uint64_t cap, uint32_t** out_rows, uint64_t* out_nrows,
               uint32_t* out_ncols, int32_t* id_map);
void gpsm_free(void* p);
/* The process-wide pool of page-locked result blocks: blocks it holds,
 * bytes pinned, blocks added since the process started and the host time
 * spent touching and pinning them (no counterpart in the reference). */
void gpsm_host_pool_stats(uint64_t* blocks, uint64_t* pinned_bytes, uint64_t* grown, double* grow_ms);

/* Matches nq queries back to back (query k: labels q_labels[q_voff[k]..],
 * edges q_edges[2*q_eoff[k]..]); rows are produced in device memory and
 * overwritten by the next query. orders: concatenated pos2id per query when
 * opts->order_mode is GPSM_ORDER_GIVEN. counts, capped, query_ms: nq each or
 * NULL (capped[k]: 1 the cap stopped query k, 2 opts->work_cap did). A
 * throughput entry point with no counterpart in the reference, whose
 * run.cpp loops Match::match per query (main/run.cpp:60-97). */
int gpsm_match_batch(gpsm_engine_t e, gpsm_graph_t g, uint32_t nq, const uint32_t* q_voff,
                     const uint32_t* q_labels, const uint64_t* q_eoff, const uint32_t* q_edges,
                     const gpsm_match_opts* opts, const int32_t* orders, uint64_t* counts,
                     int32_t* capped, double* query_ms, gpsm_batch_info* info);
/* Vertices with `label` and degree >= min_degree, ascending, on device
 * arrays (d_labels[n], d_offsets[n+1]); d_out (device) must hold n ids,
 * d_count (device) gets the count. Replaces check_kernel + kernel_collect
 * (match/Match.cu:431-526). Scratch comes from the engine's workspace
 * (e = NULL: the default engine); returns after the work finishes. */
int gpsm_select_vertices(gpsm_engine_t e, const uint32_t* d_labels, const uint32_t* d_offsets,
                         uint32_t n, uint32_t label, uint32_t min_degree, uint32_t* d_out,
                         uint32_t* d_count);
/* gpsm_select_vertices for callers that cannot allocate device memory (a
 * host that owns every allocation, such as a framework pool or a plugin host,
 * or a caller that cannot pay for cudaMalloc at call time). No counterpart in
 * the reference. It allocates nothing: its scratch is a fixed array of about
 * 513 KiB compiled into the library (held on every GPU that loads it), so n
 * is limited to 4194304 vertices (larger n: GPSM_ERR_BUDGET). Runs on
 * `stream` (a cudaStream_t, NULL = default stream) of the current device;
 * every call copies the error flags back and synchronises `stream` before it
 * returns. The first call on a device looks up the array's device address;
 * make it before any stream capture. All calls share the
 * array: calls that overlap on the GPU race. Needs no gpsm_init. */
int gpsm_select_vertices_static(const uint32_t* d_labels, const uint32_t* d_offsets, uint32_t n,
                                uint32_t label, uint32_t min_degree, uint32_t* d_out,
                                uint32_t* d_count, void* stream);
/* The batch on `slots` engine slots of the graph's device (each its own
 * stream and workspace of slot_arena bytes, 0 = automatic), each slot
 * taking the next query when it finishes one, so queries overlap on the GPU.
 * Same outputs as gpsm_match_batch; device time is the span from the first slot's start to
 * the last slot's end. */
int gpsm_match_batch_parallel(gpsm_graph_t g, uint32_t nq, const uint32_t* q_voff,
                              const uint32_t* q_labels, const uint64_t* q_eoff,
                              const uint32_t* q_edges, const gpsm_match_opts* opts,
                              const int32_t* orders, uint32_t slots, uint64_t slot_arena,
                              uint64_t* counts, int32_t* capped, double* query_ms,
                              gpsm_batch_info* info);

/* ---- serving: a request loop with memory admission ---------------------- */
/* No counterpart in the reference (main/run.cpp matches queries one after
 * another). Requests queue until a slot is free; the slot runs the filter
 * and chooses the order, then the request waits until its predicted join
 * memory fits memory_budget (0 = all slot workspaces) before joining. */
typedef struct gpsm_server_s* gpsm_server_t;
typedef struct gpsm_request_info {
  int32_t status;          /* GPSM_OK or an error */
  int32_t capped;          /* 1 the embedding cap stopped it, 2 opts->work_cap did */
  uint64_t rows;
  double submit_ms, start_ms, admit_ms, end_ms;  /* server clock */
  double device_ms;
  uint64_t admitted_bytes;
} gpsm_request_info;
int gpsm_server_create(gpsm_graph_t g, uint32_t slots, uint64_t memory_budget, uint64_t slot_arena,
                       const gpsm_match_opts* opts, int32_t collect_rows, gpsm_server_t* out);
int gpsm_server_submit(gpsm_server_t s, uint32_t qn, const uint32_t* q_labels, uint32_t qm,
                       const uint32_t* q_edges, uint64_t* ticket);
int gpsm_server_wait(gpsm_server_t s, uint64_t ticket, double timeout_s, gpsm_request_info* info,
                     uint32_t** rows, int32_t* id_map);
/* The first finished request not yet collected (completion order): its
 * ticket, info, rows and id_map (room for 128 entries: query vertices are
 * fewer than 128). A client that takes results as they finish keeps only
 * unfinished requests' rows in host memory. GPSM_ERR_STATE when nothing is
 * outstanding; GPSM_ERR_TIMEOUT after timeout_s (< 0: wait). */
int gpsm_server_wait_any(gpsm_server_t s, double timeout_s, uint64_t* ticket, gpsm_request_info* info,
                         uint32_t** rows, int32_t* id_map);
int gpsm_server_stats(gpsm_server_t s, uint64_t* in_use, uint64_t* peak_in_use, uint64_t* budget,
                      uint32_t* queued, uint32_t* active);
int gpsm_server_destroy(gpsm_server_t s);

/* Writes `bytes` of device memory on the engine's stream (an L2 flush). */
int gpsm_flush_l2(gpsm_engine_t e, uint64_t bytes);
/* Testing aid for the bounded device waits (no counterpart in the
 * reference): takes k stray tickets from the engine's look-back ticket
 * counter without telling the host, so the next query's scans wait on
 * predecessor tiles that never publish. Those waits give up after
 * scan_spin_limit polls (gpsm_set_tuning) and that query returns
 * GPSM_ERR_TIMEOUT; the engine re-reads the counter before its next query,
 * which then runs normally. */
int gpsm_debug_skew_scan_tickets(gpsm_engine_t e, uint32_t k);

/* Per-width join statistics of the engine's last gpsm_match_ex/
 * gpsm_engine_match call (n+1 entries each, index = table width):
 * rows extended, candidates scanned, rows produced. */
int gpsm_last_levels(gpsm_engine_t e, uint32_t n, uint64_t* level_in, uint64_t* level_cands,
                     uint64_t* level_out);

/* ---- launch tuning (no counterpart in the reference) ------------------- */
/* Process-wide launch choices; zero fields are left unchanged. The
 * reference fixes its launch shapes in code (block sizes 32/256/1024,
 * match/Match.cu:455, 649, 1313). */
typedef struct gpsm_tuning {
  uint32_t heavy_degree;       /* candidates with more neighbours: one block each (default 1024) */
  uint32_t ext_blocks_per_sm;  /* persistent join-check blocks per SM (1..8, default 8; at most what an SM holds) */
  uint64_t step_cands;         /* candidates one join step may admit (default 2^25) */
  uint64_t level_bytes;        /* bytes per intermediate join level (default 256 MiB) */
  uint32_t slots;              /* engine slots for batches and serving (default 4) */
  uint32_t scan_spin_limit;    /* polls a look-back scan makes of one predecessor before it gives up,
                                  flags the launch and the call returns GPSM_ERR_TIMEOUT
                                  (default 2^22; ~a second at most) */
  uint64_t race_share;         /* learned order: first work share (candidates) when the learned plan
                                  and the plain order take turns (default 2^28) */
  uint32_t ext_items;          /* candidates per thread of the join check kernel: 4 or 8 (default 4) */
  uint32_t filter_team;        /* lanes per candidate in the refinement steps: 4, 8 or 32 (default 8) */
  uint32_t explore_team;       /* lanes per candidate in the exploration steps: 8 or 32 (default 32) */
  uint32_t pad;
} gpsm_tuning;
int gpsm_set_tuning(const gpsm_tuning* t);
int gpsm_get_tuning(gpsm_tuning* t);

/* ---- learned join order (no counterpart in the reference) -------------- */
/* 16 -> 64 -> 64 -> 1 MLP, BF16 weights, FP32 accumulation and masters.
 * It predicts log2(rows out / rows in) of the join step that adds a query
 * vertex to the placed set, from 16 features of the query and the filter
 * statistics (gpsm_order_features). */
int gpsm_model_params(void);
int gpsm_model_create(int dev, uint64_t seed, gpsm_model_t* out);
int gpsm_model_destroy(gpsm_model_t m);
int gpsm_model_set(gpsm_model_t m, const float* params);
int gpsm_model_get(gpsm_model_t m, float* params);
/* Adam on minibatches of (x[n][16], y[n]) on the GPU; *loss = last epoch. */
int gpsm_model_train(gpsm_model_t m, const float* x, const float* y, uint32_t n, uint32_t epochs,
                     uint32_t batch, float lr, uint64_t seed, float* loss);
/* Gradient of the mean squared error over all n samples, no update. */
int gpsm_model_grad(gpsm_model_t m, const float* x, const float* y, uint32_t n, float* grad,
                    float* loss);
int gpsm_model_predict(gpsm_model_t m, const float* x, uint32_t n, float* y);
/* Features of every step of a vertex order (pos2id) for one query, from the
 * filter statistics gpsm_debug_filter returns: out[(qn-1)*16]. */
int gpsm_order_features(gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm,
                        const uint32_t* q_edges, const uint32_t* cand_count,
                        const uint64_t* size_fwd, const uint64_t* size_rev,
                        const int32_t* pos2id, float* out);

/* Filter-stage results for comparison with the reference restatement:
 * final |C(u)|, candidate-edge totals per edge id (forward = from->to with
 * from < to, reverse = to->from), the filter (BFS) order, the plain join
 * order and optionally every candidate set as qn*N bytes (0/1).
 * Returns 1 (not an error) when a candidate set ran empty. */
int gpsm_debug_filter(gpsm_graph_t g, uint32_t qn, const uint32_t* q_labels, uint32_t qm,
                      const uint32_t* q_edges, uint32_t* cand_count, uint64_t* size_fwd,
                      uint64_t* size_rev, uint32_t* filter_order, int32_t* plain_pos2id,
                      uint8_t* cand_bits);

#ifdef __cplusplus
}
#endif

#endif /* GPSM_H */
