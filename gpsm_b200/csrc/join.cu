// Join kernels: one launch extends a range of partial embeddings (rows of a
// row-major table) by one query vertex.
//
// The reference joins one query edge at a time (match/Match.cu:1141-1569):
// table_kernel seeds pairs, expand_kernel + link_kernel add a column for a
// tree edge, join_kernel + filter_kernel drop rows failing a non-tree edge.
// Every one of those kernels finds mu in the candidate list by a warp-wide
// LINEAR scan of C(u) per row, and no kernel checks injectivity (the host
// filters afterwards, io/IO.cpp:187-222).
//
// Here a vertex v and all of its edges to already-placed vertices are joined
// in one pass:
//   - the candidate-edge list of every placed neighbour w is located in O(1)
//     with a rank lookup in C(w)'s bitmap (no scan of C(w));
//   - the shortest of those lists drives the row; every other list is probed
//     by binary search (sorted-adjacency intersection);
//   - a candidate equal to a data vertex already in the row is dropped
//     (injectivity), so no homomorphism rows are ever materialised.
// The rows a vertex order produces are the reference's rows after its
// non-tree checks for that vertex, minus the non-injective ones, in the same
// order: input rows in order, each row's candidates ascending.
//
// Output positions come from a single-pass decoupled look-back over 64-row
// tiles, so the table stays in order without a separate scan launch. When
// the output buffer would overflow, the first row that does not fit and
// every later row are left for a later launch (cut_row); with `partial` set
// (the embedding cap) the crossing row is cut inside instead.
#include <cuda_runtime.h>

#include "filter.h"
#include "scan.cuh"

namespace gpsm {

constexpr int kExpBlock = 256;
constexpr int kExpWarps = kExpBlock / 32;
constexpr int kExpRowsPerWarp = 8;
constexpr int kExpTile = kExpWarps * kExpRowsPerWarp;  // 64 rows per tile

__device__ __forceinline__ bool sorted_contains(const uint32_t* __restrict__ a, unsigned long long lo,
                                                unsigned long long hi, uint32_t key) {
  while (lo < hi) {
    unsigned long long mid = (lo + hi) >> 1;
    uint32_t x = a[mid];
    if (x == key) return true;
    if (x < key) lo = mid + 1;
    else hi = mid;
  }
  return false;
}

struct ExpandShared {
  BackNbr back[kMaxBack];
  uint32_t row[kExpWarps][kMaxBack];
  unsigned long long lo[kExpWarps][kMaxBack];
  unsigned long long hi[kExpWarps][kMaxBack];
  uint32_t cnt[kExpTile];
  unsigned long long off[kExpTile];
  uint32_t tile;
  uint32_t cut;
  unsigned long long prefix;
  unsigned long long driver;
  unsigned long long nbrs_total;
  uint32_t* flags;
};

// Processes one row with the calling warp. write=false: returns the number
// of accepted candidates. write=true: writes them starting at output
// position pos (rows at positions >= out_cap are skipped).
__device__ __forceinline__ uint32_t expand_row(ExpandShared& S, uint32_t w, const uint32_t* __restrict__ in,
                                               uint32_t cols, unsigned long long r, uint32_t nb, bool write,
                                               uint32_t* __restrict__ out, unsigned long long pos,
                                               unsigned long long out_cap, unsigned long long* driver_len) {
  const uint32_t lane = threadIdx.x & 31;
  uint32_t* row = S.row[w];
  const uint32_t* src = in + r * cols;
  for (uint32_t k = lane; k < cols; k += 32) row[k] = src[k];
  __syncwarp();
  // locate every placed neighbour's candidate list for its data vertex
  unsigned long long best_len = ~0ULL;
  uint32_t best_j = 0;
  for (uint32_t j = lane; j < nb; j += 32) {
    const BackNbr& b = S.back[j];
    const uint32_t mu = row[b.col];
    const uint32_t word = mu >> 5, bit = mu & 31;
    const uint32_t bw = b.bm[word];
    const uint32_t idx = b.rank[word] + __popc(bw & ((1u << bit) - 1u));
    unsigned long long lo = 0, hi = 0;
    if ((bw >> bit) & 1u) {  // every table value is a candidate of its column's vertex
      lo = b.off[idx];
      hi = b.off[idx + 1];
    }
    if (hi < lo || hi > S.nbrs_total || !((bw >> bit) & 1u)) {
      atomicOr(S.flags, (uint32_t)DF_BOUNDS);
      lo = hi = 0;
    }
    S.lo[w][j] = lo;
    S.hi[w][j] = hi;
    if (hi - lo < best_len) {
      best_len = hi - lo;
      best_j = j;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    unsigned long long ol = __shfl_xor_sync(0xffffffffu, best_len, o);
    uint32_t oj = __shfl_xor_sync(0xffffffffu, best_j, o);
    if (ol < best_len || (ol == best_len && oj < best_j)) {
      best_len = ol;
      best_j = oj;
    }
  }
  __syncwarp();
  const uint32_t d = best_j;
  const unsigned long long lo = S.lo[w][d], hi = S.hi[w][d];
  *driver_len = hi - lo;
  const uint32_t* __restrict__ nd = S.back[d].nbrs;
  uint32_t count = 0;
  uint32_t prev_last = 0xffffffffu;
  const uint32_t out_cols = cols + 1;
  for (unsigned long long base = lo; base < hi; base += 32) {
    const unsigned long long k = base + lane;
    const bool valid = k < hi;
    uint32_t y = valid ? nd[k] : 0xffffffffu;
    uint32_t p = __shfl_up_sync(0xffffffffu, y, 1);
    if (lane == 0) p = prev_last;
    bool ok = valid && !(k > lo && y == p);  // parallel data edges: one candidate
    const unsigned long long last = (hi - base < 32) ? (hi - base - 1) : 31;
    prev_last = __shfl_sync(0xffffffffu, y, (int)last);
    if (ok) {
      for (uint32_t c = 0; c < cols; ++c)
        if (row[c] == y) {
          ok = false;
          break;
        }
    }
    if (ok) {
      for (uint32_t j = 0; j < nb; ++j) {
        if (j == d) continue;
        if (!sorted_contains(S.back[j].nbrs, S.lo[w][j], S.hi[w][j], y)) {
          ok = false;
          break;
        }
      }
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, ok);
    if (write && ok) {
      const unsigned long long q = pos + count + __popc(bal & ((1u << lane) - 1u));
      if (q < out_cap) {
        uint32_t* dst = out + q * out_cols;
        for (uint32_t c = 0; c < cols; ++c) dst[c] = row[c];
        dst[cols] = y;
      }
    }
    count += __popc(bal);
  }
  __syncwarp();
  return count;
}

__global__ void __launch_bounds__(kExpBlock) k_expand(const uint32_t* __restrict__ in, uint32_t cols,
                                                     unsigned long long row_begin, unsigned long long row_end,
                                                     const BackNbr* __restrict__ back, uint32_t nb,
                                                     uint32_t* __restrict__ out, unsigned long long out_cap,
                                                     uint32_t partial, ExpandResult* __restrict__ res,
                                                     Lookback lb, unsigned long long nbrs_total) {
  __shared__ ExpandShared S;
  const uint32_t wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    S.tile = lb_take_ticket(lb);
    S.cut = kExpTile;
    S.driver = 0;
    S.nbrs_total = nbrs_total;
    S.flags = lb.flags;
  }
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(back);
    uint32_t* dst = reinterpret_cast<uint32_t*>(S.back);
    const uint32_t words = nb * (sizeof(BackNbr) / 4);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const uint32_t tile = S.tile;
  const unsigned long long ntiles = (row_end - row_begin + kExpTile - 1) / kExpTile;
  if ((unsigned long long)tile >= ntiles) {  // ticket base out of step with the device counter
    if (threadIdx.x == 0) atomicOr(lb.flags, (uint32_t)DF_BOUNDS);
    return;
  }
  const unsigned long long first = row_begin + (unsigned long long)tile * kExpTile;
  const uint32_t nrows = (uint32_t)min((unsigned long long)kExpTile, row_end - first);
  // pass 1: count accepted candidates per row
  unsigned long long drv = 0;
  for (uint32_t i = 0; i < kExpRowsPerWarp; ++i) {
    const uint32_t rl = wid * kExpRowsPerWarp + i;
    uint32_t c = 0;
    unsigned long long dl = 0;
    if (rl < nrows) c = expand_row(S, wid, in, cols, first + rl, nb, false, out, 0, 0, &dl);
    drv += dl;
    if (lane == 0) S.cnt[rl] = c;
  }
  if (lane == 0 && drv) atomicAdd(&S.driver, drv);
  __syncthreads();
  if (threadIdx.x == 0 && S.driver) atomicAdd(&res->driver, S.driver);
  unsigned long long total;
  const unsigned long long mine =
      block_exclusive_scan<kExpBlock>(threadIdx.x < kExpTile ? S.cnt[threadIdx.x] : 0, &total);
  if (threadIdx.x < kExpTile) S.off[threadIdx.x] = mine;
  if (wid == 0) {
    unsigned long long ex = lb_exclusive(lb, tile, total);
    if (lane == 0) S.prefix = ex;
  }
  __syncthreads();
  const unsigned long long prefix = S.prefix;
  if (!partial && threadIdx.x < nrows) {
    if (prefix + S.off[threadIdx.x] + S.cnt[threadIdx.x] > out_cap) atomicMin(&S.cut, threadIdx.x);
  }
  __syncthreads();
  const uint32_t cut = S.cut;
  if (threadIdx.x == 0 && cut < nrows) {
    atomicMin(&res->cut_row, first + cut);
    atomicMin(&res->cut_pos, prefix + S.off[cut]);
  }
  // pass 2: write the rows that fit
  for (uint32_t i = 0; i < kExpRowsPerWarp; ++i) {
    const uint32_t rl = wid * kExpRowsPerWarp + i;
    if (rl >= nrows || rl >= cut) break;
    const unsigned long long pos = prefix + S.off[rl];
    if (S.cnt[rl] == 0 || pos >= out_cap) continue;
    unsigned long long dl;
    expand_row(S, wid, in, cols, first + rl, nb, true, out, pos, out_cap, &dl);
  }
  if (threadIdx.x == 0 && tile == ntiles - 1) res->total = prefix + total;
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

void launch_expand(Workspace& ws, const uint32_t* in, uint32_t in_cols, uint64_t row_begin, uint64_t row_end,
                   const BackNbr* d_back, uint32_t nb, uint32_t* out, uint64_t out_cap, bool partial,
                   ExpandResult* d_res, uint64_t nbrs_total) {
  if (row_end <= row_begin) return;
  const uint64_t tiles = (row_end - row_begin + kExpTile - 1) / kExpTile;
  if (tiles > ws.scan.max_tiles) {
    set_last_error("expand: too many tiles for the scan state");
    throw CudaError{cudaErrorInvalidValue, "expand tiles"};
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
  k_expand<<<(uint32_t)tiles, kExpBlock, 0, ws.stream>>>(in, in_cols, row_begin, row_end, d_back, nb, out, out_cap,
                                                         partial ? 1u : 0u, d_res, lb,
                                                         (unsigned long long)nbrs_total);
  GPSM_LAUNCHED();
}

uint64_t expand_tile_rows() { return kExpTile; }

}  // namespace gpsm
