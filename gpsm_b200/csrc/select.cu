// Vertex selection by label and degree on caller-provided device arrays:
// the reference's check_kernel + kernel_collect (match/Match.cu:431-526) as
// a standalone primitive. One thread builds one 32-bit word of the
// selection bitmap (no atomics, every word written, so the bitmap needs no
// clearing), then the single-pass compaction (k_compact, decoupled
// look-back) turns it into a sorted id list and a count.
#include <cuda_runtime.h>

#include <cstring>

#include "engine.h"

namespace gpsm {

__global__ void k_check_vertices(const uint32_t* __restrict__ lab, const uint32_t* __restrict__ off, uint32_t n,
                                 uint32_t label, uint32_t min_degree, uint32_t words, uint32_t* __restrict__ bm) {
  for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < words; w += gridDim.x * blockDim.x) {
    uint32_t bits = 0;
    const uint32_t v0 = w * 32;
    for (uint32_t b = 0; b < 32; ++b) {
      const uint32_t v = v0 + b;
      if (v < n && lab[v] == label && off[v + 1] - off[v] >= min_degree) bits |= 1u << b;
    }
    bm[w] = bits;
  }
}

uint32_t select_words(uint32_t n) { return (((n + 31) / 32) + 3) & ~3u; }

// Selection on `ws` (its stream, scan state and flags); bm holds
// select_words(n) words of scratch.
void select_vertices(Workspace& ws, const uint32_t* d_labels, const uint32_t* d_offsets, uint32_t n, uint32_t label,
                     uint32_t min_degree, uint32_t* bm, uint32_t* d_out, uint32_t* d_count) {
  const uint32_t words = select_words(n);
  const uint32_t blocks = std::min<uint32_t>((words + 255) / 256, 148 * 8);
  k_check_vertices<<<blocks, 256, 0, ws.stream>>>(d_labels, d_offsets, n, label, min_degree, words, bm);
  GPSM_LAUNCHED();
  launch_compact(ws, bm, words, d_out, nullptr, d_count, false);
}

}  // namespace gpsm
