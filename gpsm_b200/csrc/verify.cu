// Directed, edge-labelled verification on the device (the reference's
// IO::verify, io/IO.cpp:146-180, which runs on the host per row after the
// undirected match): a row survives when every query edge (a -> b, label l)
// exists as a data edge row[a] -> row[b] with label l. The engine matches
// undirected, edge-unlabelled (as the reference's GPU part does), then runs
// this filter on each new block of final rows, before the embedding cap, so
// the directed mode returns the first `cap` rows that pass.
//
// The directed data edges are an out-CSR sorted by (target, label). Rows
// are compacted in order into a second buffer with a warp ballot, a block
// scan and a decoupled look-back across 256-row tiles.
#include <cuda_runtime.h>

#include "filter.h"
#include "scan.cuh"

namespace gpsm {

constexpr int kVerBlock = 256;

__device__ __forceinline__ bool has_directed_edge(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col,
                                                  const uint32_t* __restrict__ lab, uint32_t a, uint32_t b,
                                                  uint32_t l) {
  uint32_t lo = off[a], hi = off[a + 1];
  while (lo < hi) {  // first entry with target >= b
    const uint32_t mid = (lo + hi) >> 1;
    if (col[mid] < b) lo = mid + 1;
    else hi = mid;
  }
  for (uint32_t j = lo; j < off[a + 1] && col[j] == b; ++j)
    if (lab[j] == l) return true;
  return false;
}

// checks: triples (column of the source, column of the target, label).
__global__ void __launch_bounds__(kVerBlock) k_verify_directed(const uint32_t* __restrict__ in, uint64_t nrows,
                                                               uint32_t cols, const uint32_t* __restrict__ checks,
                                                               uint32_t nchecks, const uint32_t* __restrict__ off,
                                                               const uint32_t* __restrict__ col,
                                                               const uint32_t* __restrict__ lab,
                                                               uint32_t* __restrict__ out,
                                                               unsigned long long* __restrict__ kept, Lookback lb) {
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = lb_take_ticket(lb);
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t ntiles = (nrows + kVerBlock - 1) / kVerBlock;
  if ((uint64_t)tile >= ntiles) {
    if (threadIdx.x == 0) atomicOr(lb.flags, (uint32_t)DF_BOUNDS);
    return;
  }
  const uint64_t r = (uint64_t)tile * kVerBlock + threadIdx.x;
  bool ok = r < nrows;
  if (ok) {
    const uint32_t* row = in + r * cols;
    for (uint32_t k = 0; k < nchecks && ok; ++k)
      ok = has_directed_edge(off, col, lab, row[checks[3 * k]], row[checks[3 * k + 1]], checks[3 * k + 2]);
  }
  unsigned long long total;
  const unsigned long long mine = block_exclusive_scan<kVerBlock>(ok ? 1ULL : 0ULL, &total);
  if (threadIdx.x < 32) {
    const unsigned long long ex = lb_exclusive(lb, tile, total);
    if (threadIdx.x == 0) s_prefix = ex;
  }
  __syncthreads();
  if (ok) {
    const uint32_t* row = in + r * cols;
    uint32_t* dst = out + (s_prefix + mine) * cols;
    for (uint32_t c = 0; c < cols; ++c) dst[c] = row[c];
  }
  if (threadIdx.x == 0 && (uint64_t)tile == ntiles - 1) *kept = s_prefix + total;
}

void launch_verify_directed(Workspace& ws, const uint32_t* in, uint64_t nrows, uint32_t cols, const uint32_t* d_checks,
                            uint32_t nchecks, const uint32_t* off, const uint32_t* col, const uint32_t* lab,
                            uint32_t* out, unsigned long long* d_kept) {
  if (nrows == 0) return;
  const uint64_t tiles = (nrows + kVerBlock - 1) / kVerBlock;
  if (tiles > ws.scan.max_tiles) {
    set_last_error("verify: too many rows for the scan state");
    throw CudaError{cudaErrorInvalidValue, "verify tiles"};
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
  k_verify_directed<<<(uint32_t)tiles, kVerBlock, 0, ws.stream>>>(in, nrows, cols, d_checks, nchecks, off, col, lab,
                                                                   out, d_kept, lb);
  GPSM_LAUNCHED();
}

}  // namespace gpsm
