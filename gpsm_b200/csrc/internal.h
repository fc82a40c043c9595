// Internal structures of the engine (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "gpsm.h"

namespace gpsm {

// ---------------------------------------------------------------------------
// error plumbing: every CUDA call is checked; failures become GPSM_ERR_CUDA
// (the reference exits the process instead, match/Match.h:53-65)
// ---------------------------------------------------------------------------
struct CudaError {
  cudaError_t err;
  const char* what;
};

void set_last_error(const std::string& msg);
const char* last_error();

#define GPSM_CUDA(call)                                                                    \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess) {                                                               \
      ::gpsm::set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_) + " at " + \
                             __FILE__ + ":" + std::to_string(__LINE__));                   \
      throw ::gpsm::CudaError{e_, #call};                                                  \
    }                                                                                      \
  } while (0)

#define GPSM_LAUNCHED() GPSM_CUDA(cudaGetLastError())

// device-side error flags (bitwise OR into Workspace::d_flags[0])
enum DeviceFlag : uint32_t {
  DF_EMPTY = 1u << 0,       // a candidate set collected empty (no embedding exists)
  DF_SCAN_TIMEOUT = 1u << 1,  // a decoupled look-back wait hit its iteration limit
  DF_BOUNDS = 1u << 2,      // an index check failed (result invalid)
  DF_OVERFLOW = 1u << 3,    // a 32-bit count overflowed
};

// ---------------------------------------------------------------------------
// device-resident data graph (uploaded once, reused by every query)
// ---------------------------------------------------------------------------
struct DeviceGraph {
  int device = 0;
  uint32_t n = 0;
  uint64_t nnz = 0;           // offsets[n] = 2 * undirected edges
  uint32_t* off = nullptr;    // [n+1]
  uint32_t* col = nullptr;    // [nnz], each list sorted ascending
  uint32_t* lab = nullptr;    // [n]
  uint2* labdeg = nullptr;    // [n] (label, degree): one 8-byte gather per neighbour
  uint32_t* lab_vtx = nullptr;  // [n] vertices grouped by label, degree descending
  // host-side label index (labels sorted ascending)
  std::vector<uint32_t> h_labels;   // distinct labels
  std::vector<uint32_t> h_lab_ptr;  // [L+1] offsets into lab_vtx
  std::vector<uint32_t> h_lab_deg;  // [n] degrees in lab_vtx order (for cut-offs)
  uint32_t words = 0;               // bitmap words per candidate set (padded to 4)
  // directed, edge-labelled data edges (optional): out-CSR sorted by (target, label)
  uint32_t* dir_off = nullptr;
  uint32_t* dir_col = nullptr;
  uint32_t* dir_lab = nullptr;
  uint32_t max_degree = 0;
  // label runs: every adjacency list again, sorted by (neighbour label, id),
  // with a directory of (label, first index) per run; lets the filter scan
  // only a candidate's neighbours that carry one query vertex's label
  uint32_t* lcol = nullptr;     // [nnz] or null (not built)
  uint32_t* run_off = nullptr;  // [n+1] directory offsets per vertex
  uint2* runs = nullptr;        // [run_off[n]] (label, index into lcol), labels ascending per vertex
  // every undirected edge once, as (smaller << 32 | larger), in an open-
  // addressing table of 2^ehash_bits slots (all ones: empty), at most half
  // full, probed linearly; no lookup needs more than ehash_probe + 1 slots.
  // The join checks a candidate against a placed neighbour's list with one
  // lookup here (null: not built, the list is searched)
  unsigned long long* ehash = nullptr;
  uint32_t ehash_bits = 0;
  uint32_t ehash_probe = 0;
  // label frequency as the reference computes it (Graph::inverse_num)
  uint64_t label_count(uint32_t label) const;
  // [begin, end) of lab_vtx for vertices with `label` and degree >= d
  void label_range(uint32_t label, uint32_t d, uint32_t* begin, uint32_t* end) const;
};

// ---------------------------------------------------------------------------
// decoupled look-back scan state: tiles take tickets in launch order from a
// monotone 64-bit counter whose per-launch base the host tracks, and publish
// (epoch, flag, value) words; no memset between scans is needed.
// ---------------------------------------------------------------------------
struct ScanState {
  unsigned long long* d_ticket = nullptr;  // monotone ticket counter
  unsigned long long* d_status = nullptr;  // [max_tiles] status words
  uint32_t max_tiles = 0;
  unsigned long long ticket_base = 0;  // host copy of the counter value before the next launch
  uint32_t epoch = 0;        // 20-bit epoch of the next launch
  // reserve `tiles` tickets for one launch; returns (base, epoch)
  void next_launch(uint32_t tiles, unsigned long long* base, uint32_t* ep) {
    *base = ticket_base;
    ticket_base += tiles;
    epoch = (epoch + 1) & 0xFFFFF;
    if (epoch == 0) epoch = 1;
    *ep = epoch;
  }
};

// Launch choices the autotuner may change (process-wide; read at each launch).
struct Tuning {
  uint32_t heavy_degree = 1024;    // candidates above it go to block-per-candidate kernels
  uint32_t ext_blocks_per_sm = 8;  // persistent extend blocks per SM
  uint64_t step_cands = 1ull << 25;  // candidates one join step may admit
  uint64_t level_bytes = 256ull << 20;  // bytes per intermediate join level
  uint32_t slots = 4;              // engine slots for batches and serving
  // first work share (candidates scanned) of a learned plan racing the plain
  // order: about 20 ms of joins on one B200, enough for a capped query of
  // 10^7 embeddings in a good order
  uint64_t race_share = 1ull << 28;
  // polls of one predecessor's status a look-back makes before giving up
  // (DF_SCAN_TIMEOUT): the bound on every inter-block wait
  uint32_t scan_spin_limit = 1u << 22;
  // candidates per thread of the join check kernel (4 or 8): its tile is
  // 256 x ext_items candidates
  uint32_t ext_items = 4;
  // lanes per candidate in the refinement steps (4, 8 or 32)
  uint32_t filter_team = 8;
  // lanes per candidate in the exploration steps (8 or 32)
  uint32_t explore_team = 32;
};
Tuning& tuning();
int sm_count();

// bump allocator over one device allocation; reset per query
struct Arena {
  char* base = nullptr;
  size_t size = 0;
  size_t used = 0;
  size_t high_water = 0;
  void* alloc(size_t bytes, size_t align = 256) {
    size_t p = (used + align - 1) & ~(align - 1);
    if (p + bytes > size) return nullptr;
    used = p + bytes;
    if (used > high_water) high_water = used;
    return base + p;
  }
  void reset() { used = 0; }
};

struct Workspace {
  int device = 0;
  cudaStream_t stream = nullptr;
  Arena arena;
  ScanState scan;
  uint32_t* d_flags = nullptr;      // [64] device flags and small counters
  unsigned long long* d_small = nullptr;  // [64] device scratch for results of scans
  unsigned long long* h_small = nullptr;  // pinned mirror (4096 words)
  // h_small as the device addresses it: small results are written there by
  // a kernel (small_to_host), not copied by a copy engine, so they never wait
  // behind the large row copies other slots have queued on the engines
  unsigned long long* h_small_dev = nullptr;
  cudaEvent_t ev0 = nullptr, evm = nullptr, ev1 = nullptr;
  cudaEvent_t eve0 = nullptr, eve1 = nullptr;  // around each join launch
  cudaEvent_t evb0 = nullptr, evb1 = nullptr;  // around a batch
  bool dirty = false;  // a query stopped part-way; resynchronise scan tickets
  uint32_t* d_heavy = nullptr;        // high-degree candidates handed to block-per-candidate kernels
  uint32_t* d_heavy_count = nullptr;
  uint32_t heavy_cap = 0;
  // two pinned staging buffers for result rows on their way to the host
  // (allocated at the first copy): the DMA fills one while the host thread
  // moves the other into the caller's buffer
  static constexpr size_t kStageBytes = 32ull << 20;
  void* h_stage[2] = {nullptr, nullptr};
  cudaEvent_t ev_stage[2] = {nullptr, nullptr};
  // result rows copied to page-locked host blocks on their own stream, so a
  // slot's joins fill one device result buffer while the other is copied
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_res[2] = {nullptr, nullptr};     // buffer k written (on stream)
  cudaEvent_t ev_copied[2] = {nullptr, nullptr};  // buffer k copied out (on copy_stream)
  cudaEvent_t ev_block = nullptr;  // stream_wait's sleeping event (created at first use)
  // Two result buffers that outlive a query (carved once from the top of
  // the arena, which shrinks by their size): a query's last copies out of
  // them may still run while the slot's next query starts; its joins wait
  // for those copies on the device (ev_copied) before writing the buffers.
  static constexpr size_t kRingBytes = 512ull << 20;  // per buffer
  uint32_t* res_ring[2] = {nullptr, nullptr};
  uint64_t res_ring_words = 0;  // words per buffer (0: not carved)
  // The pair, carved at the first call; false when the arena is too small
  // to give it up (the caller then uses per-query buffers).
  bool result_ring() {
    if (res_ring_words) return true;
    if (arena.used != 0 || arena.size < 8 * kRingBytes) return false;
    // the pair starts on a 4 KiB boundary whatever the arena's size
    arena.size = (arena.size - 2 * kRingBytes) & ~(size_t)4095;
    res_ring[0] = reinterpret_cast<uint32_t*>(arena.base + arena.size);
    res_ring[1] = reinterpret_cast<uint32_t*>(arena.base + arena.size + kRingBytes);
    res_ring_words = kRingBytes / sizeof(uint32_t);
    return true;
  }
};

// Waits for everything queued on ws.stream. With GPSM_BLOCKING_SYNC=1 the
// thread sleeps on an event created with cudaEventBlockingSync instead of
// spinning: many slot threads in several processes (one per GPU) on a few
// host cores would otherwise spin one another off the cores.
void stream_wait(Workspace& ws);

// Copies `words` 32-bit words from device memory to pageable host memory
// through the workspace's pinned staging buffers, on the workspace stream;
// returns when dst holds them.
void copy_to_host(Workspace& ws, uint32_t* dst, const uint32_t* d_src, uint64_t words);

}  // namespace gpsm
