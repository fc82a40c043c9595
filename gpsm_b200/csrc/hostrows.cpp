// Result rows on their way to the caller's host memory.
//
// A capped query of 10^7 rows and 12 columns returns 480 MB. Copying it
// with one pageable cudaMemcpy into a freshly zero-filled std::vector spent
// most of its time in 4 KiB page faults and in the driver's own bounce
// copies. Here the rows go through two pinned staging buffers per workspace
// (the DMA of one chunk overlaps the host copy of the previous one) into a
// malloc'd block that grows with realloc (mremap for large blocks: no copy)
// and is advised for transparent huge pages. The block is handed to the
// caller as is (gpsm_free releases it).
#include <sys/mman.h>
#include <unistd.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "engine.h"

namespace gpsm {

uint32_t* HostRows::append(uint64_t words) {
  if (n_ + words > cap_) {
    uint64_t want = std::max<uint64_t>(n_ + words, cap_ + cap_ / 2);
    want = std::max<uint64_t>(want, 1024);
    void* q = realloc(p_, want * sizeof(uint32_t));
    if (!q) {
      set_last_error("host allocation of result rows failed");
      throw CudaError{cudaErrorMemoryAllocation, "host rows"};
    }
    p_ = static_cast<uint32_t*>(q);
    cap_ = want;
    const size_t bytes = want * sizeof(uint32_t);
    if (bytes >= (8u << 20)) {
      // madvise wants a page-aligned start; the advice covers whole pages
      const uintptr_t page = (uintptr_t)sysconf(_SC_PAGESIZE);
      const uintptr_t a = ((uintptr_t)p_ + page - 1) & ~(page - 1);
      const uintptr_t e = ((uintptr_t)p_ + bytes) & ~(page - 1);
      if (e > a) madvise((void*)a, e - a, MADV_HUGEPAGE);
    }
  }
  uint32_t* at = p_ + n_;
  n_ += words;
  return at;
}

void copy_to_host(Workspace& ws, uint32_t* dst, const uint32_t* d_src, uint64_t words) {
  if (words == 0) return;
  cudaStream_t s = ws.stream;
  if (!ws.h_stage[0]) {
    for (int i = 0; i < 2; ++i) {
      GPSM_CUDA(cudaMallocHost(&ws.h_stage[i], Workspace::kStageBytes));
      GPSM_CUDA(cudaEventCreateWithFlags(&ws.ev_stage[i], cudaEventDisableTiming));
    }
  }
  const uint64_t chunk = Workspace::kStageBytes / sizeof(uint32_t);
  const uint64_t nchunks = (words + chunk - 1) / chunk;
  auto issue = [&](uint64_t c) {
    const uint64_t off = c * chunk, len = std::min<uint64_t>(chunk, words - off);
    GPSM_CUDA(cudaMemcpyAsync(ws.h_stage[c & 1], d_src + off, len * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    GPSM_CUDA(cudaEventRecord(ws.ev_stage[c & 1], s));
  };
  issue(0);
  for (uint64_t c = 0; c < nchunks; ++c) {
    // the other buffer is free again: its chunk was moved out last iteration
    if (c + 1 < nchunks) issue(c + 1);
    GPSM_CUDA(cudaEventSynchronize(ws.ev_stage[c & 1]));
    const uint64_t off = c * chunk, len = std::min<uint64_t>(chunk, words - off);
    memcpy(dst + off, ws.h_stage[c & 1], len * sizeof(uint32_t));
  }
}

}  // namespace gpsm
