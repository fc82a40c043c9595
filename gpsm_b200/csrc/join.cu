// Join kernels: one step extends a range of partial embeddings (rows of a
// row-major table) by one query vertex v and checks all of v's edges to
// already-placed vertices at once.
//
// The reference joins one query edge at a time (match/Match.cu:1141-1569):
// table_kernel seeds pairs, expand_kernel + link_kernel add a column for a
// tree edge, join_kernel + filter_kernel drop rows failing a non-tree edge.
// Each of those kernels finds mu in the candidate list by a warp-wide
// LINEAR scan of C(u) per row, runs one warp per row whatever the row's
// list length, and none checks injectivity (io/IO.cpp:146-180 filters on the
// host afterwards).
//
// Here a step is four kernels:
//   k_locate        (one thread per input row) finds, for every placed
//                   neighbour w of v, the candidate-edge list N(row[w]) ∩ C(v)
//                   with an O(1) rank lookup in C(w)'s bitmap, keeps the
//                   shortest one as the row's driver, and turns the driver
//                   lengths into candidate offsets with a single-pass
//                   decoupled look-back scan. Rows are admitted in order while
//                   their candidates fit the step budget.
//   k_extend_check  (persistent blocks, tiles of 256 x ITEMS candidates)
//                   takes candidate t of row r from the driver list and keeps
//                   it if it differs from every value in the row that could
//                   repeat (injectivity) and lies in every other placed
//                   neighbour's list (sorted-list intersection). A thread
//                   takes ITEMS consecutive candidates: ascending values of
//                   one row (mostly), so the row's state is loaded once and
//                   each list is searched from where the previous value was
//                   found (galloping), not from its start. Each tile writes
//                   its kept (row, value) pairs in order and its count.
//   k_scan_u32      turns the tile counts into output offsets.
//   k_extend_write  copies each tile's kept rows (input row + new value) to
//                   its offset: one contiguous, coalesced span per tile.
// No block waits for another: an order-preserving look-back inside the
// check kernel kept ~900 resident blocks waiting on their predecessors for
// 40% of its time.
// Work is spread by candidate, not by row, so a hub row with 60k candidates
// and a row with one candidate cost the same per candidate. The output keeps
// the reference's row order (input rows in order, each row's candidates
// ascending), and the output never overflows: a step admits rows only while
// their candidate count (an upper bound on outputs) fits the buffer.
#include <cuda_runtime.h>

#include "filter.h"
#include "scan.cuh"

namespace gpsm {

constexpr int kLocBlock = 256;  // rows per locate tile
constexpr int kExtBlock = 256;
constexpr uint32_t kMinExtTile = kExtBlock * 4;   // tiles are 256 x {4, 8} candidates
constexpr uint32_t kMaxExtTile = kExtBlock * 8;
constexpr int kInjReg = 8;  // injectivity columns a thread holds in registers per row

// Candidates per check thread of the next step (tuning; 4 or 8).
static uint32_t ext_items() { return tuning().ext_items >= 8 ? 8u : 4u; }

// First index in a[lo, hi) whose value is >= key (hi when none). Indices
// are 32-bit offsets from the list's base pointer (a list is shorter than
// 2^32), which keeps each probe to a few integer instructions.
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi,
                                                    uint32_t key) {
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(a + mid) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// The same, given that every value before lo is < key: probes lo, lo+1,
// lo+3, lo+7, ... until a value >= key, then a binary search inside the last
// gap; O(log d) for an answer d places after lo.
__device__ __forceinline__ uint32_t gallop_u32(const uint32_t* __restrict__ a, uint32_t lo, uint32_t hi,
                                               uint32_t key) {
  uint32_t step = 1, probe = lo;
  while (probe < hi && __ldg(a + probe) < key) {
    lo = probe + 1;
    probe = lo + step;
    step <<= 1;
  }
  return lower_bound_u32(a, lo, min(probe, hi), key);
}

// lower_bound over a whole list a[0, len) whose values spread about evenly
// over their range (vertex ids are permuted at random when a graph is
// generated): up to three probes where the key would sit if the values
// between the known bounds were evenly spread, then a binary search in the
// gap left. The answer is the exact lower bound whatever the values.
__device__ __forceinline__ uint32_t search_interp_u32(const uint32_t* __restrict__ a, uint32_t len, uint32_t key) {
  if (len <= 16) return lower_bound_u32(a, 0, len, key);
  uint32_t L = 0, H = len - 1;  // a[L] < key <= a[H] once the ends are checked
  uint32_t vL = __ldg(a), vH = __ldg(a + H);
  if (key <= vL) return 0;
  if (key > vH) return len;
#pragma unroll 1
  for (int it = 0; it < 3 && H - L > 8; ++it) {
    const float f = (float)(key - vL) / (float)(vH - vL);  // in (0, 1]
    uint32_t p = L + 1 + (uint32_t)(f * (float)(H - L - 1));
    p = min(max(p, L + 1), H - 1);
    const uint32_t v = __ldg(a + p);
    if (v < key) {
      L = p;
      vL = v;
    } else {
      H = p;
      vH = v;
    }
  }
  return lower_bound_u32(a, L + 1, H, key);  // H when nothing in (L, H) is >= key: a[H] >= key
}

// Candidate-edge list of data vertex mu (a candidate of w) towards v.
__device__ __forceinline__ bool locate_list(const BackNbr& b, uint32_t mu, unsigned long long nbrs_total,
                                            unsigned long long* lo, unsigned long long* hi) {
  const uint32_t word = mu >> 5, bit = mu & 31;
  const uint32_t bw = __ldg(b.bm + word);
  if (!((bw >> bit) & 1u)) return false;  // every table value is a candidate of its column's vertex
  const uint32_t idx = __ldg(b.rank + word) + __popc(bw & ((1u << bit) - 1u));
  *lo = __ldg(b.off + idx);
  *hi = __ldg(b.off + idx + 1);
  return *lo <= *hi && *hi <= nbrs_total;
}

__device__ __forceinline__ void stage_back(BackNbr* dst_back, const BackNbr* __restrict__ back, uint32_t nb) {
  const uint32_t* src = reinterpret_cast<const uint32_t*>(back);
  uint32_t* dst = reinterpret_cast<uint32_t*>(dst_back);
  const uint32_t words = nb * (uint32_t)(sizeof(BackNbr) / 4);
  for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
}

struct LocateShared {
  BackNbr back[kMaxBack];
  uint32_t tile;
  unsigned long long prefix;
};

__global__ void __launch_bounds__(kLocBlock) k_locate(const uint32_t* __restrict__ in, uint32_t cols,
                                                     unsigned long long row_begin, unsigned long long nrows,
                                                     const BackNbr* __restrict__ back, uint32_t nb,
                                                     unsigned long long nbrs_total, unsigned long long budget,
                                                     uint4* __restrict__ drv, uint4* __restrict__ rng,
                                                     unsigned long long* __restrict__ coff,
                                                     uint32_t* __restrict__ tile_row, unsigned long long tile_cap,
                                                     uint32_t ext_tile, StepState* __restrict__ st, Lookback lb) {
  __shared__ LocateShared S;
  __shared__ uint32_t s_skip;
  if (threadIdx.x == 0) {
    S.tile = lb_take_ticket(lb);
    // an earlier tile (smaller ticket, so earlier rows) already found a row
    // past the budget: no row of this tile can be admitted
    s_skip = *(volatile unsigned long long*)&st->full != 0;
  }
  stage_back(S.back, back, nb);
  __syncthreads();
  const uint32_t tile = S.tile;
  const unsigned long long ntiles = (nrows + kLocBlock - 1) / kLocBlock;
  if ((unsigned long long)tile >= ntiles) {  // ticket base out of step with the device counter
    if (threadIdx.x == 0) atomicOr(lb.flags, (uint32_t)DF_BOUNDS);
    return;
  }
  if (s_skip) {
    // publish a total past the budget so later tiles that are already
    // working see every following row as not admitted
    if (threadIdx.x < 32) lb_exclusive(lb, tile, budget + 1);
    return;
  }
  const unsigned long long i = (unsigned long long)tile * kLocBlock + threadIdx.x;
  unsigned long long best_lo = 0, best_len = 0;
  uint32_t best_j = 0;
  if (i < nrows && nb > 0) {
    const uint32_t* row = in + (row_begin + i) * cols;
    best_len = ~0ULL;
    for (uint32_t j = 0; j < nb; ++j) {
      unsigned long long lo, hi;
      if (!locate_list(S.back[j], __ldg(row + S.back[j].col), nbrs_total, &lo, &hi)) {
        atomicOr(lb.flags, (uint32_t)DF_BOUNDS);
        lo = hi = 0;
      }
      rng[i * nb + j] = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)(hi - lo), 0u);
      if (hi - lo < best_len) {
        best_len = hi - lo;
        best_lo = lo;
        best_j = j;
      }
    }
  }
  if (i < nrows) drv[i] = make_uint4((uint32_t)best_lo, (uint32_t)(best_lo >> 32), (uint32_t)best_len, best_j);
  unsigned long long total;
  const unsigned long long mine = block_exclusive_scan<kLocBlock>(best_len, &total);
  if (threadIdx.x < 32) {
    const unsigned long long ex = lb_exclusive(lb, tile, total);
    if (threadIdx.x == 0) S.prefix = ex;
  }
  __syncthreads();
  const unsigned long long off = S.prefix + mine;
  // rows are admitted in order while all their candidates fit the budget;
  // offsets grow with the row, so the admitted rows of a tile are a prefix
  const bool fits = i < nrows && off + best_len <= budget;
  const int nfit = __syncthreads_count(fits);
  if (i < nrows) {
    coff[i] = off;
    if (i + 1 == nrows) coff[nrows] = off + best_len;
    // extend tiles whose first candidate lies in this row start at this row
    if (best_len > 0)
      for (unsigned long long T = (off + ext_tile - 1) / ext_tile;
           T * ext_tile < off + best_len && T < tile_cap; ++T)
        tile_row[T] = (uint32_t)i;
  }
  if (nfit > 0 && threadIdx.x == (uint32_t)nfit - 1) {
    atomicMax(&st->rows, i + 1);
    atomicMax(&st->cand_end, off + best_len);
  }
  const unsigned long long in_tile = min((unsigned long long)kLocBlock, nrows - (unsigned long long)tile * kLocBlock);
  if (threadIdx.x == 0 && (unsigned long long)nfit < in_tile) atomicExch(&st->full, 1ULL);
}

constexpr uint32_t kSpan = kMaxExtTile;  // rows of one tile whose offsets are staged in shared memory

struct ExtendShared {
  BackNbr back[kMaxBack];
  uint32_t inj[kMaxBack];  // columns whose query vertex has the new vertex's label
  uint32_t tile;
  unsigned long long r0, r1;  // rows holding the tile's first and (at most) last candidate
  uint32_t warp_sum[kExtBlock / 32];  // kept candidates per warp, then their exclusive prefix
  unsigned long long coff[kSpan + 1];
};

// Row of candidate t: the last row r < nr with coff[r] <= t.
__device__ __forceinline__ unsigned long long row_of(const unsigned long long* __restrict__ coff,
                                                     unsigned long long nr, unsigned long long t) {
  unsigned long long lo = 0, hi = nr;  // coff[lo] <= t < coff[hi]
  while (hi - lo > 1) {
    const unsigned long long mid = (lo + hi) >> 1;
    if (__ldg(coff + mid) <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Persistent blocks take tiles of 256 x ITEMS consecutive candidates from a
// counter. Thread i of a block takes candidates ITEMS*i .. ITEMS*i+ITEMS-1
// of the tile, in two passes:
//   1. per candidate: its row (one search for the first, then the next
//      rows in order), its value y, the parallel-edge repeat check and
//      injectivity against the row's same-label columns, which are loaded
//      into registers once per row;
//   2. per other placed neighbour j: every surviving candidate is looked up
//      in that neighbour's list. Values of one row ascend, so the search
//      for the next candidate starts where the previous one ended.
// The tile's kept candidates go to kept[tile * tile_size ...] in candidate
// order, their number to tile_cnt[tile].
//
// HASH: pass 2 asks the data graph's edge table instead: y is in w's list
// N(row[w]) ∩ C(v) exactly when edge (row[w], y) exists, since y comes from
// the driver list and so is in C(v) already; one lookup of the same cost
// for every candidate, where the list search takes as long as its gap.
template <int ITEMS, bool HASH>
__global__ void __launch_bounds__(kExtBlock, ITEMS == 4 ? (HASH ? 4 : 5) : 3) k_extend_check(const uint32_t* __restrict__ in, uint32_t cols,
                                                           unsigned long long row_begin,
                                                           const BackNbr* __restrict__ back, uint32_t nb,
                                                           const uint4* __restrict__ drv,
                                                           const uint4* __restrict__ rng,
                                                           const unsigned long long* __restrict__ coff,
                                                           const uint32_t* __restrict__ tile_row,
                                                           uint2* __restrict__ kept, uint32_t* __restrict__ tile_cnt,
                                                           StepState* __restrict__ st,
                                                           const uint32_t* __restrict__ inj, uint32_t ninj,
                                                           const unsigned long long* __restrict__ ehash,
                                                           uint32_t ehash_bits, uint32_t ehash_probe) {
  constexpr uint32_t kTile = kExtBlock * ITEMS;
  __shared__ ExtendShared S;
  stage_back(S.back, back, nb);
  for (uint32_t i = threadIdx.x; i < ninj; i += blockDim.x) S.inj[i] = inj[i];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned long long nr = st->rows;     // rows admitted by k_locate
  // coff[nr] may lie in a tile k_locate skipped; the admitted rows' end is exact
  const unsigned long long ncand = nr ? st->cand_end : 0;
  const unsigned long long ntiles = (ncand + kTile - 1) / kTile;
  if (blockIdx.x == 0 && threadIdx.x == 0) st->cands = ncand;
  for (;;) {
    __syncthreads();  // the previous tile's shared state is no longer read
    if (threadIdx.x == 0) {
      const unsigned long long tile = atomicAdd(&st->next_tile, 1ULL);
      S.tile = (uint32_t)min(tile, ntiles);
      if (tile < ntiles) {
        // k_locate recorded the row of every tile's first candidate; the row
        // of the next tile's first candidate bounds this tile's last row
        S.r0 = __ldg(tile_row + tile);
        S.r1 = tile + 1 < ntiles ? min((unsigned long long)__ldg(tile_row + tile + 1), nr - 1) : nr - 1;
      }
    }
    __syncthreads();
    const uint32_t tile = S.tile;
    if ((unsigned long long)tile >= ntiles) break;
    const unsigned long long t_first = (unsigned long long)tile * kTile;
    const unsigned long long t_end = min(t_first + kTile, ncand);
    const unsigned long long r0 = S.r0, span = S.r1 - S.r0 + 1;
    const bool staged = span <= kSpan;
    if (staged)
      for (uint32_t x = threadIdx.x; x <= span; x += blockDim.x)
        S.coff[x] = r0 + x < nr ? __ldg(coff + r0 + x) : ncand;
    __syncthreads();
    uint32_t kr[ITEMS], ky[ITEMS], kd[ITEMS];  // item k's row, value and driver list index
    uint32_t keep = 0;
    const unsigned long long tb = t_first + (unsigned long long)threadIdx.x * ITEMS;
    if (tb < t_end) {
      // pass 1: rows, values, repeats and injectivity
      unsigned long long r, rstart, rend;
      uint32_t li = 0;
      if (staged) {
        uint32_t lo_ = 0, hi_ = (uint32_t)span;  // S.coff[lo_] <= tb < S.coff[hi_]
        while (hi_ - lo_ > 1) {
          const uint32_t mid = (lo_ + hi_) >> 1;
          if (S.coff[mid] <= tb) lo_ = mid;
          else hi_ = mid;
        }
        li = lo_;
        r = r0 + li;
        rstart = S.coff[li];
        rend = S.coff[li + 1];
      } else {
        r = row_of(coff, nr, tb);
        rstart = __ldg(coff + r);
        rend = r + 1 < nr ? __ldg(coff + r + 1) : ncand;
      }
      uint4 d = __ldg(drv + r);
      unsigned long long lo = ((unsigned long long)d.y << 32) | d.x;
      const uint32_t* __restrict__ nbrs = S.back[d.w].nbrs;
      const uint32_t* row = in + (row_begin + r) * cols;
      uint32_t injv[kInjReg];
#pragma unroll
      for (int c = 0; c < kInjReg; ++c) injv[c] = (uint32_t)c < ninj ? __ldg(row + S.inj[c]) : 0u;
      uint32_t prev = 0;
      bool has_prev = tb > rstart;  // parallel data edges: each neighbour once
      if (has_prev) prev = __ldg(nbrs + lo + (tb - rstart) - 1);
#pragma unroll
      for (int k = 0; k < ITEMS; ++k) {
        const unsigned long long t = tb + k;
        kr[k] = (uint32_t)r;
        ky[k] = 0;
        kd[k] = d.w;
        if (t >= t_end) continue;
        while (t >= rend) {  // the next row with candidates
          ++r;
          if (staged) {
            ++li;
            rstart = S.coff[li];
            rend = S.coff[li + 1];
          } else {
            rstart = __ldg(coff + r);
            rend = r + 1 < nr ? __ldg(coff + r + 1) : ncand;
          }
          d = __ldg(drv + r);
          lo = ((unsigned long long)d.y << 32) | d.x;
          nbrs = S.back[d.w].nbrs;
          row = in + (row_begin + r) * cols;
#pragma unroll
          for (int c = 0; c < kInjReg; ++c) injv[c] = (uint32_t)c < ninj ? __ldg(row + S.inj[c]) : 0u;
          has_prev = false;
        }
        const uint32_t y = __ldg(nbrs + lo + (t - rstart));
        bool ok = !(has_prev && prev == y);
        prev = y;
        has_prev = true;
#pragma unroll
        for (int c = 0; c < kInjReg; ++c) ok = ok && !((uint32_t)c < ninj && injv[c] == y);
        for (uint32_t c = kInjReg; ok && c < ninj; ++c) ok = __ldg(row + S.inj[c]) != y;
        kr[k] = (uint32_t)r;
        ky[k] = y;
        kd[k] = d.w;
        keep |= (ok ? 1u : 0u) << k;
      }
      // pass 2: y must lie in every other placed neighbour's list
      if (HASH) {
        for (uint32_t j = 0; keep && j < nb; ++j) {
          uint32_t cur = 0xffffffffu, wv = 0;  // this row's value in w's column
#pragma unroll
          for (int k = 0; k < ITEMS; ++k) {
            if (!((keep >> k) & 1u) || kd[k] == j) continue;
            if (kr[k] != cur) {
              cur = kr[k];
              wv = __ldg(in + (row_begin + cur) * cols + S.back[j].col);
            }
            if (!edge_in_hash(ehash, ehash_bits, ehash_probe, wv, ky[k])) keep &= ~(1u << k);
          }
        }
      }
      for (uint32_t j = 0; !HASH && keep && j < nb; ++j) {
        uint32_t cur = 0xffffffffu;
        const uint32_t* __restrict__ list = nullptr;  // this row's list towards v, from its first entry
        uint32_t pos = 0, len = 0;
#pragma unroll
        for (int k = 0; k < ITEMS; ++k) {
          if (!((keep >> k) & 1u) || kd[k] == j) continue;
          if (kr[k] != cur) {  // first candidate of this row in this list: search the whole list
            cur = kr[k];
            const uint4 g2 = __ldg(rng + (unsigned long long)cur * nb + j);
            list = S.back[j].nbrs + (((unsigned long long)g2.y << 32) | g2.x);
            len = g2.z;
            pos = search_interp_u32(list, len, ky[k]);
          } else {
            pos = gallop_u32(list, pos, len, ky[k]);
          }
          if (!(pos < len && __ldg(list + pos) == ky[k])) keep &= ~(1u << k);
        }
      }
    }
    // in-tile positions: warp inclusive scan of the per-thread counts, then
    // the warps' exclusive prefix
    const uint32_t cnt = __popc(keep);
    uint32_t incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= (uint32_t)o) incl += x;
    }
    if (lane == 31) S.warp_sum[wid] = incl;
    __syncthreads();
    if (threadIdx.x < 32) {
      const uint32_t v = lane < kExtBlock / 32 ? S.warp_sum[lane] : 0;
      uint32_t x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
      }
      if (lane < kExtBlock / 32) S.warp_sum[lane] = x - v;
      if (lane == 31) tile_cnt[tile] = x;
    }
    __syncthreads();
    uint2* dst = kept + (unsigned long long)tile * kTile + S.warp_sum[wid] + incl - cnt;
#pragma unroll
    for (int k = 0; k < ITEMS; ++k)
      if (keep & (1u << k)) *dst++ = make_uint2(kr[k], ky[k]);
  }
}

// Bulk copy shared -> global on the async (TMA) engine, in a bulk group.
// Both addresses and the size must be multiples of 16 bytes: callers check.
// Every thread that wrote the source calls proxy_fence_shared() before the
// barrier that precedes this.
__device__ __forceinline__ void bulk_store(void* gdst, const void* ssrc, uint32_t bytes) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(ssrc);
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(gdst), "r"(s), "r"(bytes)
               : "memory");
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// Makes this thread's shared-memory writes visible to the async proxy.
__device__ __forceinline__ void proxy_fence_shared() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// Waits until at most N bulk groups of this thread still read shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory");
}
// Waits until every bulk group of this thread has completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

constexpr uint32_t kWriteStage = 4096;  // words per staging buffer (two buffers)
constexpr uint32_t kWriteRows = 1024;   // rows per chunk at most (their kept pairs are staged)
constexpr uint32_t kWriteBlock = 256;   // threads of k_extend_write

// Block per tile (grid-stride): the tile's kept rows go to output rows
// tile_off[tile] ...; rows past out_cap are cut. Block 0 reports the rows
// written and clears the next step's state; each tile's count is cleared
// once read, so the next step's check pass starts from zero counts.
// The tile's output is one contiguous span. It is built in chunks of whole
// rows in shared memory: the chunk's kept (row, value) pairs are staged
// first (one coalesced load per row), then the threads fill the chunk in
// row groups: thread t owns column t % w of rows t / w, t / w + g, ... (w
// the output width, g = 256 / w rows per group), so consecutive threads
// write consecutive words, a thread's column (an input column, or the new
// value) never changes, and kU rows' loads are in flight per thread. The
// chunk leaves by one bulk copy on the async engine; it is laid out so that
// every word has the same 16-byte phase in shared memory as in the output,
// so the aligned middle goes in one copy and at most three words at each
// end by plain stores. Two staging buffers alternate: gathering the next
// chunk overlaps the copy of the previous one.
__global__ void __launch_bounds__(kWriteBlock, 4) k_extend_write(const uint32_t* __restrict__ in, uint32_t cols,
                                                                 unsigned long long row_begin,
                                                                 const uint2* __restrict__ kept,
                                                                 uint32_t* __restrict__ tile_cnt,
                                                                 const unsigned long long* __restrict__ tile_off,
                                                                 uint32_t ntiles_max, uint32_t ext_tile,
                                                                 uint32_t* __restrict__ out,
                                                                 unsigned long long out_cap,
                                                                 const unsigned long long* __restrict__ coff,
                                                                 uint32_t cut_rows, StepState* __restrict__ st,
                                                                 StepState* __restrict__ next,
                                                                 StepState* __restrict__ host_st) {
  constexpr int kU = 4;
  __shared__ __align__(128) uint32_t sbuf[2][kWriteStage + 4];
  __shared__ uint2 s_kept[kWriteRows];
  const uint32_t out_cols = cols + 1;  // at most 128
  // >= 31 rows (rows hold at most 128 words), <= kWriteRows
  const uint32_t chunk_rows = min(kWriteStage / out_cols, kWriteRows);
  const uint32_t group = kWriteBlock / out_cols;  // rows per group, >= 2
  const uint32_t trow = threadIdx.x / out_cols, tcol = threadIdx.x - trow * out_cols;
  const bool gathers = trow < group;  // threads past the last whole row of a group idle
  const bool new_col = tcol == cols;  // this thread writes the new value
  const uint32_t* __restrict__ inb = in + row_begin * cols + tcol;  // column tcol of row r: inb + r * cols
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const unsigned long long total = tile_off[ntiles_max];
    if (cut_rows && total > out_cap) {
      // more kept rows than the output holds: keep only the input rows whose
      // outputs all fit. Outputs are in input-row order, so if r is the row
      // of output out_cap, the rows before r are whole and start no later
      // than r's first output. Output p is entry p - tile_off[T] of tile T.
      uint32_t lo = 0, hi = ntiles_max;  // tile_off[lo] <= out_cap < tile_off[hi]
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (tile_off[mid] <= out_cap) lo = mid;
        else hi = mid;
      }
      const uint32_t r = kept[(unsigned long long)lo * ext_tile + (out_cap - tile_off[lo])].x;
      // row r's first candidate lies in tile t0; that tile's kept rows before
      // r are the last outputs of the whole rows
      const unsigned long long cr = coff[r];
      const uint32_t t0 = (uint32_t)(cr / ext_tile);
      const uint2* k0 = kept + (unsigned long long)t0 * ext_tile;
      uint32_t a = 0, b = (uint32_t)(tile_off[t0 + 1] - tile_off[t0]);  // entries of tile t0
      while (a < b) {
        const uint32_t m = (a + b) >> 1;
        if (k0[m].x < r) a = m + 1;
        else b = m;
      }
      st->written = tile_off[t0] + a;
      st->rows = r;
      st->cands_done = cr;
      st->cut = 1;
    } else {
      st->written = min(total, out_cap);
      st->cands_done = st->cands;
    }
    // the step's final state, straight into the host's page-locked mirror
    // (read after the stream is synchronised)
    *host_st = *st;
    __threadfence_system();
    *next = StepState{};  // the next step starts from zero
  }
  uint32_t chunk_no = 0;  // chunks this block has issued (selects the staging buffer)
  for (uint32_t tile = blockIdx.x; tile < ntiles_max; tile += gridDim.x) {
    const uint32_t c = tile_cnt[tile];
    const unsigned long long o = tile_off[tile];
    __syncthreads();  // every thread has read the count: clear it for the next step
    if (threadIdx.x == 0 && c) tile_cnt[tile] = 0;
    if (c == 0 || o >= out_cap) continue;
    const uint32_t rows = (uint32_t)min((unsigned long long)c, out_cap - o);
    const uint2* kt = kept + (unsigned long long)tile * ext_tile;
    for (uint32_t q0 = 0; q0 < rows; q0 += chunk_rows, ++chunk_no) {
      const uint32_t nq = min(chunk_rows, rows - q0);
      const uint32_t words = nq * out_cols;
      uint32_t* dst = out + (o + q0) * out_cols;
      const uint32_t lead = (uint32_t)(((uintptr_t)dst >> 2) & 3);  // dst's word phase within 16 bytes
      uint32_t* sb = sbuf[chunk_no & 1];
      if (threadIdx.x == 0) bulk_wait_read<1>();  // the copy that last read this buffer is done with it
      __syncthreads();  // ... and the previous chunk's gather no longer reads s_kept
      for (uint32_t i = threadIdx.x; i < nq; i += kWriteBlock) s_kept[i] = __ldg(kt + q0 + i);
      __syncthreads();
      if (gathers) {
        uint32_t* sw = sb + lead + threadIdx.x;  // word (trow, tcol) of the chunk; a group is group*w words
        const uint32_t gw = group * out_cols;     // words per group
        uint32_t r0 = trow;
        // whole rounds of kU rows (every row exists: no checks), then the rest
        for (; r0 + (kU - 1) * group < nq; r0 += kU * group, sw += kU * gw) {
          uint32_t val[kU];
#pragma unroll
          for (int u = 0; u < kU; ++u) {
            const uint2 e = s_kept[r0 + u * group];
            val[u] = new_col ? e.y : __ldg(inb + (size_t)e.x * cols);
          }
#pragma unroll
          for (int u = 0; u < kU; ++u) sw[u * gw] = val[u];
        }
        for (; r0 < nq; r0 += group, sw += gw) {
          const uint2 e = s_kept[r0];
          *sw = new_col ? e.y : __ldg(inb + (size_t)e.x * cols);
        }
      }
      proxy_fence_shared();
      __syncthreads();
      // aligned middle [k0, k1) by one bulk copy, the ends by plain stores
      const uint32_t k0 = min((4u - lead) & 3u, words);
      const uint32_t k1 = k0 + ((words - k0) & ~3u);
      bool bulk = false;
      if (k1 > k0) {
        const uintptr_t ga = (uintptr_t)(dst + k0), sa = (uintptr_t)(sb + lead + k0);
        bulk = ((ga | sa) & 15u) == 0 && (((k1 - k0) * 4u) & 15u) == 0;
      }
      if (bulk) {
        if (threadIdx.x == 0) bulk_store(dst + k0, sb + lead + k0, (k1 - k0) * 4u);
        // head: threads 0..k0-1; tail (words - k1 <= 3 words): threads 4..
        const uint32_t t = threadIdx.x;
        if (t < k0) dst[t] = sb[lead + t];
        else if (t >= 4 && t - 4 < words - k1) dst[k1 + t - 4] = sb[lead + k1 + t - 4];
      } else {
        for (uint32_t k = threadIdx.x; k < words; k += kWriteBlock) dst[k] = sb[lead + k];
      }
    }
  }
  if (threadIdx.x == 0) bulk_wait_all();  // the span is in global memory before the block ends
}

// Blocks of k_extend_check<ITEMS> one SM holds at once (registers and shared
// memory decide it); asked once per process.
template <int ITEMS, bool HASH>
static uint32_t ext_resident_per_sm() {
  static const uint32_t n = [] {
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_extend_check<ITEMS, HASH>, kExtBlock, 0) != cudaSuccess ||
        b < 1)
      b = 1;
    return (uint32_t)b;
  }();
  return n;
}

template <int ITEMS, bool HASH>
static uint32_t ext_grid() {  // persistent extend blocks: all resident at once
  const uint32_t per_sm =
      std::min<uint32_t>(std::max<uint32_t>(1, tuning().ext_blocks_per_sm), ext_resident_per_sm<ITEMS, HASH>());
  return (uint32_t)sm_count() * per_sm;
}

__global__ void k_gather_u64(const unsigned long long* __restrict__ src, const unsigned long long* __restrict__ idx,
                             uint32_t n, unsigned long long* __restrict__ dst) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

void launch_gather_u64(Workspace& ws, const unsigned long long* src, const unsigned long long* idx, uint32_t n,
                       unsigned long long* dst) {
  if (n == 0) return;
  k_gather_u64<<<(n + 255) / 256, 256, 0, ws.stream>>>(src, idx, n, dst);
  GPSM_LAUNCHED();
}

static Lookback next_lb(Workspace& ws, uint64_t tiles) {
  if (tiles > ws.scan.max_tiles) {
    set_last_error("join step: too many tiles for the scan state");
    throw CudaError{cudaErrorInvalidValue, "join tiles"};
  }
  Lookback lb;
  lb.ticket = ws.scan.d_ticket;
  lb.status = ws.scan.d_status;
  unsigned long long base;
  uint32_t ep;
  ws.scan.next_launch((uint32_t)tiles, &base, &ep);
  lb.base = base;
  lb.epoch = ep;
  lb.flags = ws.d_flags;
  lb.spin_limit = tuning().scan_spin_limit;
  return lb;
}

uint64_t join_cands_per_extend_tile() { return kMinExtTile; }
uint64_t join_kept_slack() { return 2ull * kMaxExtTile; }

void launch_join_step(Workspace& ws, const uint32_t* in, uint32_t in_cols, uint64_t row_begin, uint64_t row_end,
                      const BackNbr* d_back, uint32_t nb, uint64_t nbrs_total, uint64_t budget, uint32_t* out,
                      uint64_t out_cap, const JoinScratch& js, StepState* d_st, StepState* d_next,
                      const uint32_t* d_inj, uint32_t ninj, bool cut_rows, StepState* host_st,
                      const unsigned long long* ehash, uint32_t ehash_bits, uint32_t ehash_probe) {
  const uint64_t nrows = row_end - row_begin;
  if (nrows == 0) return;
  const uint32_t items = ext_items();
  const uint32_t ext_tile = kExtBlock * items;  // one tile size for the whole step
  const uint64_t ntiles_max = (budget + ext_tile - 1) / ext_tile;
  if (nrows > js.rows || nrows * nb > js.rng_entries || ntiles_max > js.tiles ||
      ntiles_max * ext_tile > js.kept_entries) {
    set_last_error("join step: more rows than the step scratch holds");
    throw CudaError{cudaErrorInvalidValue, "join rows"};
  }
  // word arrays on 4-byte and pair arrays on 8-byte boundaries, or no launch
  if ((((uintptr_t)in | (uintptr_t)out) & 3u) || ((uintptr_t)js.kept & 7u)) {
    set_last_error("join step: misaligned row buffer");
    throw CudaError{cudaErrorInvalidValue, "join alignment"};
  }
  if (in_cols + 1 > 128) {  // the write pass puts at least two rows in a 256-thread group
    set_last_error("join step: rows wider than 128 words");
    throw CudaError{cudaErrorInvalidValue, "join width"};
  }
  const uint64_t ltiles = (nrows + kLocBlock - 1) / kLocBlock;
  Lookback lb1 = next_lb(ws, ltiles);
  k_locate<<<(uint32_t)ltiles, kLocBlock, 0, ws.stream>>>(in, in_cols, row_begin, nrows, d_back, nb, nbrs_total,
                                                          budget, js.drv, js.rng, js.coff, js.tile_row, js.tiles,
                                                          ext_tile, d_st, lb1);
  GPSM_LAUNCHED();
  // check pass: persistent blocks take tiles from a counter until the
  // admitted candidates run out
  if (ehash && nb > 1) {
    if (items == 8)
      k_extend_check<8, true><<<ext_grid<8, true>(), kExtBlock, 0, ws.stream>>>(
          in, in_cols, row_begin, d_back, nb, js.drv, js.rng, js.coff, js.tile_row, js.kept, js.tile_cnt, d_st, d_inj,
          ninj, ehash, ehash_bits, ehash_probe);
    else
      k_extend_check<4, true><<<ext_grid<4, true>(), kExtBlock, 0, ws.stream>>>(
          in, in_cols, row_begin, d_back, nb, js.drv, js.rng, js.coff, js.tile_row, js.kept, js.tile_cnt, d_st, d_inj,
          ninj, ehash, ehash_bits, ehash_probe);
  } else if (items == 8) {
    k_extend_check<8, false><<<ext_grid<8, false>(), kExtBlock, 0, ws.stream>>>(
        in, in_cols, row_begin, d_back, nb, js.drv, js.rng, js.coff, js.tile_row, js.kept, js.tile_cnt, d_st, d_inj,
        ninj, nullptr, 0, 0);
  } else {
    k_extend_check<4, false><<<ext_grid<4, false>(), kExtBlock, 0, ws.stream>>>(
        in, in_cols, row_begin, d_back, nb, js.drv, js.rng, js.coff, js.tile_row, js.kept, js.tile_cnt, d_st, d_inj,
        ninj, nullptr, 0, 0);
  }
  GPSM_LAUNCHED();
  launch_scan_u32(ws, js.tile_cnt, std::max<uint64_t>(ntiles_max, 1), js.tile_off);
  const uint32_t wgrid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(ntiles_max, (uint64_t)sm_count() * 8));
  k_extend_write<<<wgrid, kWriteBlock, 0, ws.stream>>>(in, in_cols, row_begin, js.kept, js.tile_cnt, js.tile_off,
                                               (uint32_t)std::max<uint64_t>(ntiles_max, 1), ext_tile, out, out_cap,
                                               js.coff, cut_rows ? 1u : 0u, d_st, d_next, host_st);
  GPSM_LAUNCHED();
}

}  // namespace gpsm
