// Single-pass decoupled look-back prefix scan (Merrill & Garland, "Single-pass
// Parallel Prefix Scan with Decoupled Look-back", NVIDIA TR 2016), restated
// for this engine. It replaces the reference's thrust::exclusive_scan calls
// (match/Match.cu:506, 1115, 1319, 1533) and the orphaned Blelloch scan and
// compaction files (util/prefix_scan.cu, util/compact_scan.cu): the running
// total stays on the device, there is no host round trip per scan and no
// second kernel for block sums.
//
// Tiles take tickets in the order blocks start, from a monotone 64-bit
// counter; the host knows each launch's base, so no memset is needed between
// scans. A status word is [epoch:20 | flag:2 | value:42]: flag 1 publishes a
// tile aggregate, flag 2 an inclusive prefix. Every wait is bounded; when a
// bound is hit the kernel raises DF_SCAN_TIMEOUT and carries on with a wrong
// (but in-range) value, so the host reports an error instead of hanging.
#pragma once
#include <cstdint>

#include "internal.h"

namespace gpsm {

struct Lookback {
  unsigned long long* ticket;
  unsigned long long* status;
  unsigned long long base;
  uint32_t epoch;
  uint32_t* flags;
  uint32_t spin_limit;  // polls of one predecessor before giving up (tuning().scan_spin_limit)
};

constexpr int kLbValueBits = 42;
constexpr unsigned long long kLbValueMask = (1ULL << kLbValueBits) - 1;

__device__ __forceinline__ unsigned long long lb_word(uint32_t epoch, uint32_t flag,
                                                      unsigned long long v) {
  return ((unsigned long long)epoch << 44) | ((unsigned long long)flag << 42) | (v & kLbValueMask);
}

// Thread 0 of the block calls this; the block broadcasts the result.
__device__ __forceinline__ uint32_t lb_take_ticket(const Lookback& lb) {
  return (uint32_t)(atomicAdd(lb.ticket, 1ULL) - lb.base);
}

// Called by all 32 lanes of ONE warp. Publishes `aggregate` for `tile` and
// returns the exclusive prefix of the earlier tiles of its segment (same
// value in every lane). A segment is a run of tiles scanned on its own:
// tiles seg_first .. tile-1 are summed; the default is one segment.
__device__ __forceinline__ unsigned long long lb_exclusive(const Lookback& lb, uint32_t tile,
                                                           unsigned long long aggregate, uint32_t seg_first = 0) {
  const unsigned lane = threadIdx.x & 31;
  volatile unsigned long long* st = lb.status;
  if (tile == seg_first) {
    if (lane == 0) {
      __threadfence();
      st[tile] = lb_word(lb.epoch, 2, aggregate);
    }
    __syncwarp();
    return 0;
  }
  if (lane == 0) {
    __threadfence();
    st[tile] = lb_word(lb.epoch, 1, aggregate);
  }
  __syncwarp();
  unsigned long long exclusive = 0;
  long long window_end = (long long)tile - 1;  // highest predecessor in the window
  unsigned spins = 0;
  bool timed_out = false;
  while (window_end >= 0) {
    long long idx = window_end - (long long)lane;
    unsigned long long w = 0;
    uint32_t flag = 2, ep = lb.epoch;  // lanes before the segment look like a zero prefix
    unsigned long long val = 0;
    if (idx >= (long long)seg_first) {
      for (;;) {
        w = st[idx];
        ep = (uint32_t)(w >> 44);
        flag = (uint32_t)((w >> 42) & 3);
        if (ep == lb.epoch && flag != 0) break;
        if (++spins > lb.spin_limit) {
          timed_out = true;
          flag = 2;
          break;
        }
        __nanosleep(64);
      }
      val = (ep == lb.epoch) ? (w & kLbValueMask) : 0;
    }
    // nearest predecessor holding an inclusive prefix
    unsigned inc = __ballot_sync(0xffffffffu, flag == 2);
    int stop = inc ? __ffs(inc) - 1 : 32;  // lanes [0, stop] contribute
    unsigned long long part = (lane <= (unsigned)stop) ? val : 0;
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    exclusive += part;
    if (inc) break;
    window_end -= 32;
    if (window_end < (long long)seg_first) break;
  }
  if (__any_sync(0xffffffffu, timed_out) && lane == 0) atomicOr(lb.flags, (uint32_t)DF_SCAN_TIMEOUT);
  if (lane == 0) {
    __threadfence();
    st[tile] = lb_word(lb.epoch, 2, exclusive + aggregate);
  }
  __syncwarp();
  return exclusive;
}

// Block-wide exclusive scan of one 64-bit value per thread (blockDim <= 1024).
// Returns the thread's exclusive prefix; *total gets the block total.
template <int BLOCK>
__device__ __forceinline__ unsigned long long block_exclusive_scan(unsigned long long v,
                                                                   unsigned long long* total) {
  __shared__ unsigned long long warp_sums[BLOCK / 32];
  const unsigned lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  unsigned long long x = v;
  for (int o = 1; o < 32; o <<= 1) {
    unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= (unsigned)o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    unsigned long long s = (lane < BLOCK / 32) ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      unsigned long long y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= (unsigned)o) s += y;
    }
    if (lane < BLOCK / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  unsigned long long warp_prefix = wid ? warp_sums[wid - 1] : 0;
  *total = warp_sums[BLOCK / 32 - 1];
  __syncthreads();
  return warp_prefix + x - v;
}

}  // namespace gpsm
