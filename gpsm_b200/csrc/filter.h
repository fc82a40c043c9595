// Kernel launchers shared by the engine (device code in filter.cu / join.cu).
#pragma once
#include "internal.h"

namespace gpsm {

// Plain device pointers of a DeviceGraph, passed by value to kernels.
struct GraphView {
  const uint32_t* __restrict__ off;
  const uint32_t* __restrict__ col;
  const uint2* __restrict__ labdeg;
  const uint32_t* __restrict__ lcol;     // label-sorted lists (null: scan col)
  const uint32_t* __restrict__ run_off;
  const uint2* __restrict__ runs;
  uint32_t n;
};

inline GraphView view(const DeviceGraph& g) {
  return GraphView{g.off, g.col, g.labdeg, g.lcol, g.run_off, g.runs, g.n};
}

// Builds g.lcol / g.run_off / g.runs on the device (leaves them null when
// vertex ids and label ranks do not fit one 32-bit key).
void build_label_runs(DeviceGraph& g, const uint32_t* h_lab);
// Builds g.ehash from the CSR (leaves it null when the table does not fit
// the free memory or a probe sequence grows past its limit).
void build_edge_hash(DeviceGraph& g);

#ifdef __CUDACC__
// Whether data edge (a, b) exists, from g.ehash (a != b).
__device__ __forceinline__ bool edge_in_hash(const unsigned long long* __restrict__ table, uint32_t bits,
                                             uint32_t probe, uint32_t a, uint32_t b) {
  const unsigned long long key = a < b ? ((unsigned long long)a << 32 | b) : ((unsigned long long)b << 32 | a);
  const unsigned long long mask = (1ull << bits) - 1;
  unsigned long long s = (key * 0x9E3779B97F4A7C15ull) >> (64 - bits);
  for (uint32_t p = 0; p <= probe; ++p) {
    const unsigned long long k = __ldg(table + s);
    if (k == key) return true;
    if (k == ~0ull) return false;
    s = (s + 1) & mask;
  }
  return false;
}
#endif

// Candidates deferred by a warp kernel to a block-per-candidate kernel.
struct HeavyList {
  uint32_t* items = nullptr;
  uint32_t* count = nullptr;
  uint32_t cap = 0;
  uint32_t threshold = 1024;  // degree above which a candidate is deferred
};

// One direction u->v of a query edge for candidate-edge collection.
struct CedgeDir {
  const uint32_t* ids;           // final sorted candidate list of u
  uint32_t n;                    // |C(u)|
  uint32_t v;                    // target query vertex (its bitmap is probed)
  uint32_t lab;                  // its label
  uint32_t pad;
  unsigned long long item_base;  // first work item (index into counts/offsets)
};

// Refinement bookkeeping for skipping exact no-ops: every refine launch has
// a sequence number (seq, from 1); a launch that removes a candidate of u
// writes stamp[u] = seq. A refinement of u changes nothing when no target's
// candidate set changed since u's previous refinement (prev): one pass
// leaves every remaining candidate with a neighbour in every target's set.
struct RefineStamp {
  uint32_t* stamp = nullptr;  // [n] device, zero at query start
  uint32_t prev = 0;          // seq of u's previous refinement (0: none, run)
  uint32_t seq = 0;           // this launch
};

// Copies `bytes` (a multiple of 4) of device memory into ws.h_small at h_dst
// with a kernel on ws.stream (no copy engine); read after a stream sync.
void small_to_host(Workspace& ws, void* h_dst, const void* d_src, size_t bytes);
void launch_mark_range(Workspace& ws, const DeviceGraph& g, uint32_t begin, uint32_t end, uint32_t* bm);
// stamp/u/prev (optional): skip when C(u) has not changed since the
// compaction that ran when the last refine seq was `prev` (list and count
// are still current).
void launch_compact(Workspace& ws, const uint32_t* bm, uint32_t words, uint32_t* list, uint32_t* rank,
                    uint32_t* count, bool set_empty_flag, const uint32_t* stamp = nullptr, uint32_t u = 0,
                    uint32_t prev = 0);
// Exploration and refinement of query vertex u (label lab_u, query degree
// deg_u) over the candidates in u's bitmap, hubs included, in one launch.
// tgt: explore (v, label, degree) per target; refine (x, label) per target.
// Final lists, ranks and counts of the bitmaps of vertices 0..nverts-1 in one
// launch (d_lists: device array of nverts list pointers; rank: nverts x words).
void launch_compact_multi(Workspace& ws, const uint32_t* bm, uint32_t words, uint32_t nverts, uint32_t* const* d_lists,
                          uint32_t* rank, uint32_t* counts);
void launch_explore(Workspace& ws, const DeviceGraph& g, uint32_t u, uint32_t lab_u, uint32_t deg_u,
                    const uint32_t* tgt, uint32_t ntgt, uint32_t* bm);
void launch_refine(Workspace& ws, const DeviceGraph& g, uint32_t u, uint32_t lab_u, uint32_t deg_u,
                   const uint32_t* tgt, uint32_t ntgt, uint32_t* bm, RefineStamp rs = RefineStamp());
// d_base[ndir+1]: first work item of each direction, d_base[ndir] = items
void launch_cedge_count(Workspace& ws, const DeviceGraph& g, const CedgeDir* d_dirs, uint32_t ndir,
                        const unsigned long long* d_base, uint64_t items, const uint32_t* bm, uint32_t* cnt);
void launch_cedge_write(Workspace& ws, const DeviceGraph& g, const CedgeDir* d_dirs, uint32_t ndir,
                        const unsigned long long* d_base, uint64_t items, const uint32_t* bm,
                        const unsigned long long* goff, uint32_t* nbrs);
void launch_scan_u32(Workspace& ws, const uint32_t* in, uint64_t n, unsigned long long* out);
void launch_gather_u64(Workspace& ws, const unsigned long long* src, const unsigned long long* idx, uint32_t n,
                       unsigned long long* dst);

// ---- joins ---------------------------------------------------------------
// An already-placed query neighbour w of the vertex being added.
struct BackNbr {
  uint32_t col;                         // column of w in the input table
  uint32_t pad;
  const uint32_t* bm;                   // final C(w) bitmap
  const uint32_t* rank;                 // per-word ranks of C(w)
  const unsigned long long* off;        // candidate-edge offsets of w->v, by rank of mu in C(w)
  const uint32_t* nbrs;                 // candidate-edge neighbour array
};

constexpr uint32_t kMaxBack = 128;  // query vertices are < 128 here; checked on the host

// Device-side bookkeeping of one join step (initialised by the host).
struct StepState {
  unsigned long long rows;         // input rows admitted (a prefix of the step's rows)
  unsigned long long written;      // output rows written (<= out_cap)
  unsigned long long next_tile;    // tile counter of the check pass
  unsigned long long cands;        // candidates of the admitted rows
  unsigned long long verified;     // directed mode: rows that passed the verify filter (host copy)
  unsigned long long cand_end;     // end offset of the last admitted row's candidates
  unsigned long long full;         // a row failed admission: later locate tiles skip their rows
  // the write pass cut the output at a row boundary (more kept rows than
  // out_cap): rows and written were reduced to the rows written whole,
  // cands_done is their candidates (cands stays all that were checked)
  unsigned long long cut;
  unsigned long long cands_done;
};

// Per-row scratch of a join step: driver list (lo, hi32 of lo, length, j)
// and candidate offsets (rows + 1 entries).
struct JoinScratch {
  uint4* drv = nullptr;
  uint4* rng = nullptr;               // rows x nb list ranges (lo, lo>>32, length, 0)
  unsigned long long* coff = nullptr;
  uint32_t* tile_row = nullptr;       // per extend tile: the row holding its first candidate
  uint2* kept = nullptr;              // per tile (256 x items): kept (row, new value) of each tile, in order
  uint32_t* tile_cnt = nullptr;       // kept candidates per tile
  unsigned long long* tile_off = nullptr;  // tiles + 1: output row of each tile's first kept candidate
  uint64_t rows = 0;
  uint64_t rng_entries = 0;
  uint64_t tiles = 0;                 // entries of tile_row
  uint64_t kept_entries = 0;          // entries of kept
};
// Candidates of the smallest check tile (sizes tile counts) and the extra
// kept entries that cover rounding the budget up to the largest tile.
uint64_t join_cands_per_extend_tile();
uint64_t join_kept_slack();

// One join step over input rows [row_begin, row_end) (in_cols columns,
// d_st: this step's state, zero on entry; d_next: the next step's, cleared
// by this step once its last launch no longer reads d_st; js.tile_cnt must
// be zero on entry and is left zero;
// row-major): rows are admitted in order while their candidates fit
// `budget`; admitted rows are extended by the query vertex whose placed
// neighbours are back[0..nb) into `out` (in_cols+1 columns), at most out_cap
// rows (the first out_cap in order). nbrs_total bounds every list range.
// d_inj[0..ninj): the input columns whose query vertex has the new vertex's
// label (the only columns a candidate can repeat). cut_rows: when more rows
// are kept than out_cap, the step ends at a row boundary instead (rows and
// written count only the rows written whole; the rest are offered again).
// host_st: the device address of a page-locked StepState the write pass
// fills with the step's final state. ehash (null: none): the data graph's
// edge table (DeviceGraph::ehash), which replaces the list searches of steps
// with more than one placed neighbour.
void launch_join_step(Workspace& ws, const uint32_t* in, uint32_t in_cols, uint64_t row_begin, uint64_t row_end,
                      const BackNbr* d_back, uint32_t nb, uint64_t nbrs_total, uint64_t budget, uint32_t* out,
                      uint64_t out_cap, const JoinScratch& js, StepState* d_st, StepState* d_next,
                      const uint32_t* d_inj, uint32_t ninj, bool cut_rows, StepState* host_st,
                      const unsigned long long* ehash, uint32_t ehash_bits, uint32_t ehash_probe);

}  // namespace gpsm
