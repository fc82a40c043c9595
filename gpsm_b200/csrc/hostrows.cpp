// Result rows on their way to the caller's host memory.
//
// A capped query of 10^7 rows and 12 columns returns 480 MB; a serving loop
// returns one such block per request. Two paths:
//
// Pooled (the usual one): a process-wide pool of page-locked blocks (malloc'd
// memory registered with the driver, or cudaHostAlloc memory when
// GPSM_HOST_POOL_ALLOC=hostalloc). A query
// with an embedding cap takes a block large enough for cap rows before its
// joins start; the device copies rows straight into it (one DMA per flush,
// no bounce copy, no page faults: the block was touched and pinned when the
// pool grew). The caller gets the block itself, and gpsm_free gives it back
// to the pool, so the next request reuses it. The pool pins at most
// GPSM_HOST_POOL_GB GiB (default: a quarter of the host's memory, at most
// 64 GiB); at that limit a request takes any free block large enough, or
// the free blocks (all too small for it) are released to make room; only
// when blocks in use hold the whole limit do queries use the other path.
// Result sizes vary from a few hundred MB to a few GB, so without that the
// pool filled with blocks of the wrong sizes. A serving loop needs
// blocks for every finished request its client has not collected yet:
// requests finish out of order, so that can be many more than the slots.
//
// Malloc'd: rows go through two pinned staging buffers per workspace (the
// DMA of one chunk overlaps the host copy of the previous one) into a
// malloc'd block that grows with realloc (mremap for large blocks: no copy)
// and is advised for transparent huge pages; gpsm_free frees it.
#include <sys/mman.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace gpsm {

namespace {

struct HostPool {
  std::mutex mu;
  std::multimap<uint64_t, void*> free_blocks;  // capacity bytes -> block
  std::unordered_map<void*, uint64_t> owned;   // every pool block -> capacity bytes
  uint64_t pinned = 0;
  uint64_t limit = 0;
  uint64_t grown = 0;     // blocks added since the process started
  uint64_t evicted = 0;   // free blocks released to make room for larger ones
  double grow_ms = 0;     // host time spent touching and pinning them
  // blocks from cudaHostAlloc instead of malloc'd memory registered with
  // cudaHostRegister (GPSM_HOST_POOL_ALLOC=hostalloc)
  bool host_alloc = false;
  HostPool() {
    if (const char* a = getenv("GPSM_HOST_POOL_ALLOC")) host_alloc = strcmp(a, "hostalloc") == 0;
    if (const char* e = getenv("GPSM_HOST_POOL_GB")) {
      limit = (uint64_t)(atof(e) * (double)(1ull << 30));
    } else {
      const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGESIZE);
      const uint64_t phys = pages > 0 && page > 0 ? (uint64_t)pages * (uint64_t)page : (32ull << 30);
      limit = std::min<uint64_t>(64ull << 30, phys / 4);
    }
  }
};

HostPool& pool() {
  static HostPool* p = new HostPool();  // lives until exit: blocks may be freed late
  return *p;
}

// Unpins and frees a block taken out of the pool (no lock held).
void pool_release_memory(HostPool& P, void* b) {
  if (P.host_alloc) {
    cudaFreeHost(b);
  } else {
    cudaHostUnregister(b);
    free(b);
  }
  cudaGetLastError();
}

// A pinned block of at least `bytes`, or null when pinning fails (the caller
// then uses malloc'd memory). In order: a free block of about the right size
// (at most twice it), a new block while the pool is under its limit, any
// free block large enough, and at the limit with none large enough a new
// block after the free ones (all too small for this request) are released.
// A new block is touched and pinned outside the pool's lock (its size is
// reserved against the limit first), so other slots keep taking and
// returning blocks.
void* pool_acquire(uint64_t bytes, uint64_t* cap) {
  HostPool& P = pool();
  // size classes: multiples of 64 MiB
  const uint64_t size = (bytes + (64ull << 20) - 1) & ~((64ull << 20) - 1);
  std::vector<void*> evicted;
  bool room = false;
  {
    std::lock_guard<std::mutex> lk(P.mu);
    auto it = P.free_blocks.lower_bound(bytes);
    if (it != P.free_blocks.end() && it->first <= 2 * bytes + (64ull << 20)) {
      void* b = it->second;
      *cap = it->first;
      P.free_blocks.erase(it);
      return b;
    }
    if (P.pinned + size <= P.limit) {
      room = true;
    } else if (it != P.free_blocks.end()) {
      void* b = it->second;  // larger than wanted, but pinned already
      *cap = it->first;
      P.free_blocks.erase(it);
      return b;
    } else {
      for (auto e = P.free_blocks.begin(); e != P.free_blocks.end() && P.pinned + size > P.limit;) {
        evicted.push_back(e->second);
        P.pinned -= e->first;
        P.owned.erase(e->second);
        ++P.evicted;
        e = P.free_blocks.erase(e);
      }
      room = P.pinned + size <= P.limit;
    }
    if (room) P.pinned += size;
  }
  for (void* b : evicted) pool_release_memory(P, b);
  if (!room) return nullptr;
  const auto t0 = std::chrono::steady_clock::now();
  void* b = nullptr;
  bool ok;
  if (P.host_alloc) {
    ok = cudaHostAlloc(&b, size, cudaHostAllocDefault) == cudaSuccess;
    if (!ok) cudaGetLastError();
  } else {
    ok = posix_memalign(&b, 2ull << 20, size) == 0;
    if (ok) {
      madvise(b, size, MADV_HUGEPAGE);
      memset(b, 0, size);  // fault the pages in now, once
      ok = cudaHostRegister(b, size, cudaHostRegisterDefault) == cudaSuccess;
      if (!ok) {
        cudaGetLastError();
        free(b);
      }
    }
  }
  std::lock_guard<std::mutex> lk(P.mu);
  if (!ok) {
    P.pinned -= size;
    return nullptr;
  }
  P.owned[b] = size;
  ++P.grown;
  P.grow_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  *cap = size;
  return b;
}

}  // namespace

void host_pool_stats(uint64_t* blocks, uint64_t* pinned_bytes, uint64_t* grown, double* grow_ms) {
  HostPool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  if (blocks) *blocks = P.owned.size();
  if (pinned_bytes) *pinned_bytes = P.pinned;
  if (grown) *grown = P.grown;
  if (grow_ms) *grow_ms = P.grow_ms;
}

bool host_pool_release(void* p) {
  if (!p) return false;
  HostPool& P = pool();
  std::lock_guard<std::mutex> lk(P.mu);
  auto it = P.owned.find(p);
  if (it == P.owned.end()) return false;
  P.free_blocks.emplace(it->second, p);
  return true;
}

void host_free(void* p) {
  if (!host_pool_release(p)) free(p);
}

HostRows::~HostRows() { host_free(p_); }

HostRows& HostRows::operator=(HostRows&& o) noexcept {
  if (this != &o) {
    host_free(p_);
    p_ = o.p_, n_ = o.n_, cap_ = o.cap_, pinned_ = o.pinned_;
    o.p_ = nullptr, o.n_ = o.cap_ = 0, o.pinned_ = false;
  }
  return *this;
}

void HostRows::reserve_pinned(uint64_t words) {
  if (p_ || words == 0) return;
  uint64_t cap = 0;
  void* b = pool_acquire(words * sizeof(uint32_t), &cap);
  if (!b) return;
  p_ = static_cast<uint32_t*>(b);
  cap_ = cap / sizeof(uint32_t);
  n_ = 0;
  pinned_ = true;
}

uint32_t* HostRows::append(uint64_t words) {
  if (n_ + words > cap_) {
    uint64_t want = std::max<uint64_t>(n_ + words, cap_ + cap_ / 2);
    want = std::max<uint64_t>(want, 1024);
    void* q = nullptr;
    if (pinned_) {
      // a pool block cannot grow in place: move to malloc'd memory
      q = malloc(want * sizeof(uint32_t));
      if (q && n_) memcpy(q, p_, n_ * sizeof(uint32_t));
      if (q) host_pool_release(p_);
    } else {
      q = realloc(p_, want * sizeof(uint32_t));
    }
    if (!q) {
      set_last_error("host allocation of result rows failed");
      throw CudaError{cudaErrorMemoryAllocation, "host rows"};
    }
    p_ = static_cast<uint32_t*>(q);
    pinned_ = false;
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

void HostRows::append_from_device(Workspace& ws, const uint32_t* d_src, uint64_t words) {
  if (words == 0) return;
  uint32_t* dst = append(words);
  if (pinned_) {
    GPSM_CUDA(cudaMemcpyAsync(dst, d_src, words * sizeof(uint32_t), cudaMemcpyDeviceToHost, ws.stream));
    GPSM_CUDA(cudaStreamSynchronize(ws.stream));
  } else {
    copy_to_host(ws, dst, d_src, words);
  }
}

bool HostRows::append_from_device_async(Workspace& ws, const uint32_t* d_src, uint64_t words, cudaEvent_t ready,
                                        cudaEvent_t done) {
  if (!pinned_ || n_ + words > cap_ || !ws.copy_stream) return false;
  if (words == 0) return true;
  uint32_t* dst = append(words);
  GPSM_CUDA(cudaStreamWaitEvent(ws.copy_stream, ready, 0));
  GPSM_CUDA(cudaMemcpyAsync(dst, d_src, words * sizeof(uint32_t), cudaMemcpyDeviceToHost, ws.copy_stream));
  GPSM_CUDA(cudaEventRecord(done, ws.copy_stream));
  return true;
}

void stream_wait(Workspace& ws) {
  static const bool blocking = [] {
    const char* e = getenv("GPSM_BLOCKING_SYNC");
    return e && e[0] == '1';
  }();
  if (!blocking) {
    GPSM_CUDA(cudaStreamSynchronize(ws.stream));
    return;
  }
  if (!ws.ev_block) GPSM_CUDA(cudaEventCreateWithFlags(&ws.ev_block, cudaEventDisableTiming | cudaEventBlockingSync));
  GPSM_CUDA(cudaEventRecord(ws.ev_block, ws.stream));
  GPSM_CUDA(cudaEventSynchronize(ws.ev_block));
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
