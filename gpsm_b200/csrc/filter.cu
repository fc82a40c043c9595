// Filter-side kernels: candidate initialisation, exploration, refinement,
// bitmap compaction and candidate-edge collection.
//
// Candidate sets live as one bitmap per query vertex (N bits, padded to a
// multiple of 128 bits) instead of the reference's bool[N] rows: a probe is a
// 4-byte gather that stays in L2, and compaction reads 16 bytes per 128
// vertices. Sorted candidate lists and per-word ranks are produced by one
// single-pass compaction kernel (decoupled look-back, scan.cuh).
//
// Semantics follow the reference kernels exactly, because the reference's
// join order depends on the candidate-edge sizes they produce:
//   k_mark_range   == check_kernel      (match/Match.cu:431-446)
//   k_compact      == kernel_collect    (match/Match.cu:463-526)
//   k_filter_step<true, *>  == kernel_collect + explore_kernel (match/Match.cu:528-601)
//   k_filter_step<false, *> == kernel_collect + refine_kernel  (match/Match.cu:761-808)
//   k_cedge_count  == count_kernel      (match/Match.cu:892-943)
//   k_cedge_write  == examine_kernel    (match/Match.cu:961-1064)
#include <cuda_runtime.h>

#include "filter.h"
#include "scan.cuh"

namespace gpsm {

__global__ void k_mark_range(const uint32_t* __restrict__ ids, uint32_t begin, uint32_t end,
                             uint32_t* __restrict__ bm) {
  for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
    uint32_t x = ids[i];
    atomicOr(&bm[x >> 5], 1u << (x & 31));
  }
}

// One tile = 256 threads x 4 words (uint4) = 1024 words = 32768 vertices.
constexpr int kCompactBlock = 256;
constexpr int kCompactWordsPerTile = kCompactBlock * 4;

__global__ void __launch_bounds__(kCompactBlock) k_compact(const uint32_t* __restrict__ bm, uint32_t words,
                                                          uint32_t* __restrict__ list,
                                                          uint32_t* __restrict__ rank,
                                                          uint32_t* __restrict__ count, Lookback lb,
                                                          uint32_t set_empty_flag, const uint32_t* __restrict__ stamp,
                                                          uint32_t u, uint32_t prev) {
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = lb_take_ticket(lb);
  __syncthreads();
  // C(u) unchanged since the last compaction: list and count are current
  // (every block has taken its ticket, so the host's ticket base stays exact)
  if (stamp && prev && stamp[u] <= prev) return;
  const uint32_t tile = s_tile;
  const uint32_t ntiles_c = (words + kCompactWordsPerTile - 1) / kCompactWordsPerTile;
  if (tile >= ntiles_c) {  // ticket base out of step with the device counter
    if (threadIdx.x == 0) atomicOr(lb.flags, (uint32_t)DF_BOUNDS);
    return;
  }
  const uint32_t w0 = tile * kCompactWordsPerTile + threadIdx.x * 4;
  uint4 v = make_uint4(0, 0, 0, 0);
  if (w0 < words) v = *reinterpret_cast<const uint4*>(bm + w0);  // words is a multiple of 4
  const uint32_t c0 = __popc(v.x), c1 = __popc(v.y), c2 = __popc(v.z), c3 = __popc(v.w);
  unsigned long long total;
  unsigned long long mine = block_exclusive_scan<kCompactBlock>(c0 + c1 + c2 + c3, &total);
  if (threadIdx.x < 32) {
    unsigned long long ex = lb_exclusive(lb, tile, total);
    if (threadIdx.x == 0) s_prefix = ex;
  }
  __syncthreads();
  unsigned long long pos = s_prefix + mine;
  if (w0 < words) {
    if (rank) {
      uint4 r;
      r.x = (uint32_t)pos;
      r.y = (uint32_t)(pos + c0);
      r.z = (uint32_t)(pos + c0 + c1);
      r.w = (uint32_t)(pos + c0 + c1 + c2);
      *reinterpret_cast<uint4*>(rank + w0) = r;
    }
    uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint32_t x = wv[k];
      while (x) {
        int b = __ffs(x) - 1;
        x &= x - 1;
        list[pos++] = (w0 + k) * 32 + b;
      }
    }
  }
  const uint32_t ntiles = (words + kCompactWordsPerTile - 1) / kCompactWordsPerTile;
  if (tile == ntiles - 1 && threadIdx.x == 0) {
    unsigned long long c = s_prefix + total;
    *count = (uint32_t)c;
    if (set_empty_flag && c == 0) atomicOr(lb.flags, (uint32_t)DF_EMPTY);
  }
}

// The final candidate lists of query vertices 0..nverts-1 in one launch:
// the block with ticket t compacts tile t % tiles_u of vertex t / tiles_u's
// bitmap; each vertex's tiles are one look-back segment, so every vertex
// gets its own sorted list, per-word ranks and count (DF_EMPTY when one is
// empty), as nverts separate k_compact launches would.
__global__ void __launch_bounds__(kCompactBlock) k_compact_multi(const uint32_t* __restrict__ bm, uint32_t words,
                                                                uint32_t nverts, uint32_t* const* __restrict__ lists,
                                                                uint32_t* __restrict__ rank,
                                                                uint32_t* __restrict__ counts, Lookback lb) {
  __shared__ uint32_t s_ticket;
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_ticket = lb_take_ticket(lb);
  __syncthreads();
  const uint32_t tiles_u = (words + kCompactWordsPerTile - 1) / kCompactWordsPerTile;
  const uint32_t t = s_ticket;
  if (t >= tiles_u * nverts) {  // ticket base out of step with the device counter
    if (threadIdx.x == 0) atomicOr(lb.flags, (uint32_t)DF_BOUNDS);
    return;
  }
  const uint32_t u = t / tiles_u, tile = t - u * tiles_u;
  const uint32_t* bmu = bm + (size_t)u * words;
  uint32_t* list = lists[u];
  uint32_t* ranku = rank + (size_t)u * words;
  const uint32_t w0 = tile * kCompactWordsPerTile + threadIdx.x * 4;
  uint4 v = make_uint4(0, 0, 0, 0);
  if (w0 < words) v = *reinterpret_cast<const uint4*>(bmu + w0);  // words is a multiple of 4
  const uint32_t c0 = __popc(v.x), c1 = __popc(v.y), c2 = __popc(v.z), c3 = __popc(v.w);
  unsigned long long total;
  const unsigned long long mine = block_exclusive_scan<kCompactBlock>(c0 + c1 + c2 + c3, &total);
  if (threadIdx.x < 32) {
    const unsigned long long ex = lb_exclusive(lb, t, total, u * tiles_u);
    if (threadIdx.x == 0) s_prefix = ex;
  }
  __syncthreads();
  unsigned long long pos = s_prefix + mine;
  if (w0 < words) {
    uint4 r;
    r.x = (uint32_t)pos;
    r.y = (uint32_t)(pos + c0);
    r.z = (uint32_t)(pos + c0 + c1);
    r.w = (uint32_t)(pos + c0 + c1 + c2);
    *reinterpret_cast<uint4*>(ranku + w0) = r;
    const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      uint32_t x = wv[k];
      while (x) {
        const int b = __ffs(x) - 1;
        x &= x - 1;
        list[pos++] = (w0 + k) * 32 + b;
      }
    }
  }
  if (tile == tiles_u - 1 && threadIdx.x == 0) {
    const unsigned long long c = s_prefix + total;
    counts[u] = (uint32_t)c;
    if (c == 0) atomicOr(lb.flags, (uint32_t)DF_EMPTY);
  }
}

// Warp per candidate mu of u. For each target v (label, degree) in order:
// every neighbour mv of mu with that label and degree >= deg(v) enters C(v);
// if none does, mu leaves C(u) and later targets are skipped.
// Candidates with more than kHeavyDegree neighbours are handed to a block
// per candidate (the *_heavy kernels) through a per-launch list, so one hub
// does not hold a warp for thousands of iterations while the grid idles.
constexpr uint32_t kHeavyBlock = 512;

__device__ __forceinline__ bool defer_heavy(uint32_t deg, uint32_t item, HeavyList hl) {
  if (deg <= hl.threshold || hl.items == nullptr) return false;
  uint32_t slot = 0;
  if ((threadIdx.x & 31) == 0) slot = atomicAdd(hl.count, 1u);
  slot = __shfl_sync(0xffffffffu, slot, 0);
  if (slot >= hl.cap) return false;  // list full: the warp does it
  if ((threadIdx.x & 31) == 0) hl.items[slot] = item;
  return true;
}

// Neighbours of a candidate that can matter for one target all carry the
// target's label: above this degree the filter scans only that label's run
// of the label-sorted list (same vertices, same ascending order) instead of
// the whole list.
constexpr uint32_t kRunMinDegree = 32;

// [*rb, *re) of lcol: mu's neighbours with label l (empty when none). All
// lanes of the warp call it and get the same range.
__device__ __forceinline__ void label_run_warp(const GraphView& g, uint32_t mu, uint32_t l, uint32_t end,
                                               uint32_t* rb, uint32_t* re) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t db = g.run_off[mu], de = g.run_off[mu + 1];
  *rb = *re = 0;
  for (uint32_t k0 = db; k0 < de; k0 += 32) {
    const uint32_t k = k0 + lane;
    uint2 r = make_uint2(0u, 0u);
    bool m = false;
    if (k < de) {
      r = g.runs[k];
      m = r.x == l;
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, m);
    if (bal) {
      const uint32_t src = __ffs(bal) - 1;
      const uint32_t kk = k0 + src;
      *rb = __shfl_sync(0xffffffffu, r.y, src);
      *re = kk + 1 < de ? g.runs[kk + 1].y : end;
      return;
    }
  }
}

// The candidate's scan range for a target of label l: its label run when
// the graph has runs and the list is long, else the whole id-sorted list.
__device__ __forceinline__ const uint32_t* scan_range_warp(const GraphView& g, uint32_t mu, uint32_t l, uint32_t b,
                                                           uint32_t e, uint32_t* rb, uint32_t* re) {
  if (g.lcol && e - b > kRunMinDegree) {
    label_run_warp(g, mu, l, e, rb, re);
    return g.lcol;
  }
  *rb = b;
  *re = e;
  return g.col;
}

// Block kernels: every warp looks the run up itself (the directory entries
// come from L1 after the first warp), so no block barrier is needed.
__device__ __forceinline__ const uint32_t* scan_range_block(const GraphView& g, uint32_t mu, uint32_t l, uint32_t b,
                                                            uint32_t e, uint32_t* rb, uint32_t* re) {
  return scan_range_warp(g, mu, l, b, e, rb, re);
}

// ---- exploration and refinement: one launch per query vertex --------------
// Candidates of u are read from C(u)'s bitmap (no compaction before each
// step): warps of the first `light_blocks` blocks take chunks of `cw` words
// (1..32, so that small bitmaps still spread over thousands of warps) and
// handle their candidates four at a time, 8 lanes each over the candidate's
// neighbours; a candidate with more than `hub_degree` neighbours (a hub) is
// left to the remaining blocks of the same launch, which walk the hubs of
// u's label (a prefix of lab_vtx, degree descending) with threads over
// neighbours. Same candidates, same per-candidate steps, so the sets are
// those of the reference's collect + explore / refine sequence.
struct StepTargets {
  const uint32_t* tgt;  // explore: (v, label, degree) per target; refine: (x, label)
  uint32_t ntgt;
};

// Label run of mu for label l found by a team of G lanes of one warp (the
// lanes first .. first+G-1): G directory entries a step; labels ascend in
// the directory, so the search stops at the first larger label.
template <int G>
__device__ __forceinline__ void label_run_team(const GraphView& g, uint32_t mu, uint32_t l, uint32_t end,
                                               uint32_t* rb, uint32_t* re) {
  const uint32_t lane = threadIdx.x & 31, first = lane & ~(uint32_t)(G - 1), tl = lane - first;
  const uint32_t mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << first);
  const uint32_t db = g.run_off[mu], de = g.run_off[mu + 1];
  *rb = *re = 0;
  for (uint32_t k0 = db; k0 < de; k0 += G) {
    const uint32_t k = k0 + tl;
    uint2 r = make_uint2(0u, 0u);
    if (k < de) r = g.runs[k];
    const uint32_t hit = __ballot_sync(mask, k < de && r.x == l) & mask;
    if (hit) {
      const uint32_t src = __ffs(hit) - 1;  // lane holding the run
      const uint32_t kk = k0 + (src - first);
      *rb = __shfl_sync(mask, r.y, src);
      *re = kk + 1 < de ? g.runs[kk + 1].y : end;
      return;
    }
    if (__ballot_sync(mask, k < de && r.x > l) & mask) return;  // l is absent
  }
}

// Scan range of mu for label l for a team of G lanes (G = 0: a whole block,
// each warp looking the run up itself).
template <int G>
__device__ __forceinline__ const uint32_t* scan_range_team(const GraphView& g, uint32_t mu, uint32_t l, uint32_t b,
                                                           uint32_t e, uint32_t* rb, uint32_t* re) {
  if (g.lcol && e - b > kRunMinDegree) {
    label_run_team<G == 0 ? 32 : G>(g, mu, l, e, rb, re);
    return g.lcol;
  }
  *rb = b;
  *re = e;
  return g.col;
}

// The threads that work on one candidate: G lanes of a warp, or (G = 0) the
// whole block; any() is true on every member when it is on one.
template <int G>
struct Team {
  uint32_t rank, size, mask;
  __device__ __forceinline__ Team() {
    if (G == 0) {
      rank = threadIdx.x;
      size = blockDim.x;
      mask = 0;
    } else {
      const uint32_t lane = threadIdx.x & 31, first = lane & ~(uint32_t)(G - 1);
      rank = lane - first;
      size = G;
      mask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << first);
    }
  }
  __device__ __forceinline__ bool any(bool p) const {
    if (G == 0) return __syncthreads_or(p);
    return (__ballot_sync(mask, p) & mask) != 0;
  }
};

// Explore one candidate mu of u with team T: every neighbour mv with the
// target's label and degree >= the target's enters C(v); mu leaves C(u) at
// the first target that gets none (match/Match.cu:594-598) and later
// targets are skipped. Each lane takes kScanU neighbours a round: their
// list entries, then their (label, degree), then their bitmap words are
// loaded together, so a long run costs a quarter of the dependent rounds.
constexpr uint32_t kScanU = 4;

template <int G>
__device__ __forceinline__ void explore_one(const GraphView& g, uint32_t mu, uint32_t b, uint32_t e,
                                            const uint32_t* s_tgt, uint32_t ntgt, uint32_t* __restrict__ bm,
                                            uint32_t words, uint32_t* bmu) {
  const Team<G> T;
  for (uint32_t t = 0; t < ntgt; ++t) {
    const uint32_t v = s_tgt[3 * t], lv = s_tgt[3 * t + 1], dv = s_tgt[3 * t + 2];
    uint32_t* bmv = bm + (size_t)v * words;
    bool any = false;
    uint32_t rb, re;
    const uint32_t* cl = scan_range_team<G>(g, mu, lv, b, e, &rb, &re);
    for (uint32_t j0 = rb + T.rank; j0 < re; j0 += kScanU * T.size) {
      uint32_t mv[kScanU];
      bool in[kScanU];
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k) {
        const uint32_t j = j0 + k * T.size;
        in[k] = j < re;
        mv[k] = in[k] ? cl[j] : 0u;
      }
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k) {
        if (!in[k]) continue;
        const uint2 ld = g.labdeg[mv[k]];
        in[k] = ld.x == lv && ld.y >= dv;
      }
      uint32_t have[kScanU];
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k) have[k] = in[k] ? bmv[mv[k] >> 5] : 0u;
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k) {
        if (!in[k]) continue;
        // popular vertices are set by many candidates: skip the atomic when
        // the bit is already there (a stale read only costs a spare atomic)
        const uint32_t bit = 1u << (mv[k] & 31);
        if (!(have[k] & bit)) atomicOr(&bmv[mv[k] >> 5], bit);
        any = true;
      }
    }
    if (!T.any(any)) {
      if (T.rank == 0) atomicAnd(&bmu[mu >> 5], ~(1u << (mu & 31)));
      return;
    }
  }
}

// Refine one candidate mu of u with team T: mu stays only if every target
// x has a candidate among mu's neighbours (match/Match.cu:761-808). The
// first round looks at one neighbour per lane (most candidates that stay
// hit there); later rounds at kScanU per lane with their loads together.
template <int G>
__device__ __forceinline__ void refine_one(const GraphView& g, uint32_t mu, uint32_t b, uint32_t e,
                                           const uint32_t* s_tgt, uint32_t ntgt, const uint32_t* __restrict__ bm,
                                           uint32_t words, uint32_t* bmu, const RefineStamp& rs, uint32_t u) {
  const Team<G> T;
  for (uint32_t t = 0; t < ntgt; ++t) {
    const uint32_t* bmv = bm + (size_t)s_tgt[2 * t] * words;
    bool found = false;
    uint32_t rb, re;
    const uint32_t* cl = scan_range_team<G>(g, mu, s_tgt[2 * t + 1], b, e, &rb, &re);
    uint32_t per = 1;  // neighbours per lane this round
    for (uint32_t j0 = rb; j0 < re && !found; j0 += per * T.size, per = kScanU) {
      uint32_t mv[kScanU];
      bool in[kScanU];
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k) {
        const uint32_t j = j0 + k * T.size + T.rank;
        in[k] = k < per && j < re;
        mv[k] = in[k] ? cl[j] : 0u;
      }
      bool hit = false;
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k)
        if (in[k]) hit |= ((bmv[mv[k] >> 5] >> (mv[k] & 31)) & 1u) != 0;
      found = T.any(hit);
    }
    if (!found) {
      if (T.rank == 0) {
        atomicAnd(&bmu[mu >> 5], ~(1u << (mu & 31)));
        if (rs.stamp) rs.stamp[u] = rs.seq;
      }
      return;
    }
  }
}

// Refinement targets worth checking, compacted in place in shared memory
// (thread 0; the caller syncs): every candidate left in C(u) had a
// neighbour in each target's set when u was last refined, and a set only
// shrinks, so a target whose set has not changed since u's previous
// refinement (its stamp is older) cannot reject anyone. Skipping it leaves
// the sets exactly those of checking every target. All of them on u's first
// refinement.
__device__ __forceinline__ uint32_t refine_targets(const RefineStamp& rs, uint32_t* tgt, uint32_t ntgt) {
  if (rs.prev == 0) return ntgt;
  uint32_t n = 0;
  for (uint32_t t = 0; t < ntgt; ++t)
    if (rs.stamp[tgt[2 * t]] >= rs.prev) {
      tgt[2 * n] = tgt[2 * t];
      tgt[2 * n + 1] = tgt[2 * t + 1];
      ++n;
    }
  return n;
}

// EXPLORE: explore_one; otherwise refine_one. hubs: [hub_begin, hub_end) of
// lab_vtx, the vertices of u's label with more than hub_degree neighbours.
// TEAM: lanes per candidate in the light part (4 or 8: eight or four
// candidates' chains of loads in flight per warp; 32: one candidate, all
// lanes over its neighbours), a tuning choice for exploration (8 or 32) and
// refinement (4, 8 or 32) each.
template <bool EXPLORE, uint32_t TEAM>
__global__ void __launch_bounds__(256, 4) k_filter_step(GraphView g, const uint32_t* __restrict__ lab_vtx,
                                                     uint32_t hub_begin, uint32_t hub_end, uint32_t hub_degree,
                                                     uint32_t light_blocks, uint32_t cw, uint32_t u,
                                                     const uint32_t* __restrict__ tgt, uint32_t ntgt,
                                                     uint32_t* __restrict__ bm, uint32_t words,
                                                     const uint32_t* __restrict__ flags, RefineStamp rs) {
  constexpr uint32_t kStride = EXPLORE ? 3 : 2;
  constexpr uint32_t kTeam = TEAM;
  extern __shared__ uint32_t s_tgt[];
  __shared__ uint32_t s_chunk[8][32 * 32];  // per warp: the candidates of one chunk (at most 32 words)
  __shared__ uint32_t s_ntgt;
  for (uint32_t i = threadIdx.x; i < kStride * ntgt; i += blockDim.x) s_tgt[i] = tgt[i];
  __syncthreads();
  if (*flags & DF_EMPTY) return;
  if (!EXPLORE) {
    // only targets whose sets changed since u's previous refinement (the
    // stamps do not change during the launch: it stamps u alone)
    if (threadIdx.x == 0) s_ntgt = refine_targets(rs, s_tgt, ntgt);
    __syncthreads();
    ntgt = s_ntgt;
    if (ntgt == 0) return;  // nothing can change
  }
  uint32_t* bmu = bm + (size_t)u * words;
  if (blockIdx.x < light_blocks) {
    // each warp lists its chunk's candidates (ascending) in shared memory,
    // then its four 8-lane teams take them in turn: four candidates' chains
    // of dependent loads in flight per warp instead of one
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nwarps = light_blocks * (blockDim.x >> 5);
    uint32_t* wl = s_chunk[threadIdx.x >> 5];
    for (uint32_t c0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * cw; c0 < words; c0 += nwarps * cw) {
      // each word of the chunk belongs to this warp alone: only its own
      // candidates' bits are cleared while it runs
      const uint32_t wv = (lane < cw && c0 + lane < words) ? bmu[c0 + lane] : 0u;
      const uint32_t c = __popc(wv);
      uint32_t incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += x;
      }
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      if (total == 0) continue;
      uint32_t p = incl - c;
      for (uint32_t x = wv; x; x &= x - 1) wl[p++] = (c0 + lane) * 32 + (__ffs(x) - 1);
      __syncwarp();
      for (uint32_t i = lane / kTeam; i < total; i += 32 / kTeam) {
        const uint32_t mu = wl[i];
        const uint32_t b = g.off[mu], e = g.off[mu + 1];
        if (e - b > hub_degree) continue;  // a hub: the hub blocks take it
        if (EXPLORE) explore_one<kTeam>(g, mu, b, e, s_tgt, ntgt, bm, words, bmu);
        else refine_one<kTeam>(g, mu, b, e, s_tgt, ntgt, bm, words, bmu, rs, u);
      }
      __syncwarp();  // the list is rewritten for the next chunk
    }
    return;
  }
  for (uint32_t i = hub_begin + (blockIdx.x - light_blocks); i < hub_end; i += gridDim.x - light_blocks) {
    const uint32_t mu = lab_vtx[i];
    if (!((bmu[mu >> 5] >> (mu & 31)) & 1u)) continue;  // not (or no longer) a candidate of u
    const uint32_t b = g.off[mu], e = g.off[mu + 1];
    if (EXPLORE) explore_one<0>(g, mu, b, e, s_tgt, ntgt, bm, words, bmu);
    else refine_one<0>(g, mu, b, e, s_tgt, ntgt, bm, words, bmu, rs, u);
    __syncthreads();  // the bitmap word read above is read again for the next hub
  }
}

// Work item i belongs to edge-direction d with item_base[d] <= i < item_base[d+1].
__device__ __forceinline__ uint32_t find_dir(const unsigned long long* __restrict__ s_base, uint32_t ndir,
                                             unsigned long long i) {
  uint32_t lo = 0, hi = ndir;  // invariant: s_base[lo] <= i < s_base[hi]
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) >> 1;
    if (s_base[mid] <= i) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Defers a hub item to the block kernels (team version of defer_heavy).
template <int G>
__device__ __forceinline__ bool defer_heavy_team(const Team<G>& T, uint32_t deg, uint32_t item, HeavyList hl) {
  if (deg <= hl.threshold || hl.items == nullptr) return false;
  const uint32_t lead = __ffs(T.mask) - 1;
  uint32_t slot = 0;
  if (T.rank == 0) slot = atomicAdd(hl.count, 1u);
  slot = __shfl_sync(T.mask, slot, lead);
  if (slot >= hl.cap) return false;  // list full: the team does it
  if (T.rank == 0) hl.items[slot] = item;
  return true;
}

// Candidate-edge work items (edge direction u->v, mu in C(u)) go to teams of
// kCedgeTeam lanes (four items per warp in flight); hubs go to the block
// kernels through the deferred list.
constexpr int kCedgeTeam = 8;

// Per (edge direction u->v, mu in C(u)): |N(mu) ∩ C(v)|.
__global__ void __launch_bounds__(256) k_cedge_count(GraphView g, const CedgeDir* __restrict__ dirs,
                                                     uint32_t ndir, const unsigned long long* __restrict__ s_base,
                                                     const uint32_t* __restrict__ bm, uint32_t words,
                                                     uint32_t* __restrict__ cnt, HeavyList hl) {
  const Team<kCedgeTeam> T;
  const unsigned long long items = s_base[ndir];
  const unsigned long long teams = (gridDim.x * blockDim.x) / kCedgeTeam;
  for (unsigned long long w = (blockIdx.x * blockDim.x + threadIdx.x) / kCedgeTeam; w < items; w += teams) {
    const uint32_t d = find_dir(s_base, ndir, w);
    const CedgeDir cd = dirs[d];
    const uint32_t mu = cd.ids[w - cd.item_base];
    const uint32_t* bmv = bm + (size_t)cd.v * words;
    const uint32_t b = g.off[mu], e = g.off[mu + 1];
    if (defer_heavy_team(T, e - b, (uint32_t)w, hl)) continue;
    uint32_t rb, re;
    const uint32_t* cl = scan_range_team<kCedgeTeam>(g, mu, cd.lab, b, e, &rb, &re);
    uint32_t c = 0;
    for (uint32_t j0 = rb + T.rank; j0 < re; j0 += kScanU * kCedgeTeam) {  // kScanU loads in flight
      uint32_t mv[kScanU];
      bool in[kScanU];
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k) {
        in[k] = j0 + k * kCedgeTeam < re;
        mv[k] = in[k] ? cl[j0 + k * kCedgeTeam] : 0u;
      }
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k)
        if (in[k]) c += (bmv[mv[k] >> 5] >> (mv[k] & 31)) & 1u;
    }
    for (int o = kCedgeTeam / 2; o > 0; o >>= 1) c += __shfl_xor_sync(T.mask, c, o);
    if (T.rank == 0) cnt[w] = c;
  }
}

// Writes N(mu) ∩ C(v) in adjacency (ascending) order at goff[item].
__global__ void __launch_bounds__(256) k_cedge_write(GraphView g, const CedgeDir* __restrict__ dirs,
                                                     uint32_t ndir, const unsigned long long* __restrict__ s_base,
                                                     const uint32_t* __restrict__ bm, uint32_t words,
                                                     const unsigned long long* __restrict__ goff,
                                                     uint32_t* __restrict__ nbrs, HeavyList hl) {
  const Team<kCedgeTeam> T;
  const uint32_t lead = __ffs(T.mask) - 1;
  const unsigned long long items = s_base[ndir];
  const unsigned long long teams = (gridDim.x * blockDim.x) / kCedgeTeam;
  for (unsigned long long w = (blockIdx.x * blockDim.x + threadIdx.x) / kCedgeTeam; w < items; w += teams) {
    const uint32_t d = find_dir(s_base, ndir, w);
    const CedgeDir cd = dirs[d];
    const uint32_t mu = cd.ids[w - cd.item_base];
    const uint32_t* bmv = bm + (size_t)cd.v * words;
    const uint32_t b = g.off[mu], e = g.off[mu + 1];
    if (defer_heavy_team(T, e - b, (uint32_t)w, hl)) continue;
    uint32_t rb, re;
    const uint32_t* cl = scan_range_team<kCedgeTeam>(g, mu, cd.lab, b, e, &rb, &re);
    unsigned long long pos = goff[w];
    // kScanU neighbours per lane a round: their loads go out together, then
    // they are written in adjacency order (round k covers the k-th group of
    // kCedgeTeam neighbours)
    for (uint32_t j0 = rb; j0 < re; j0 += kScanU * kCedgeTeam) {
      uint32_t mv[kScanU];
      bool hit[kScanU];
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k) {
        const uint32_t j = j0 + k * kCedgeTeam + T.rank;
        hit[k] = j < re;
        mv[k] = hit[k] ? cl[j] : 0u;
      }
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k)
        if (hit[k]) hit[k] = (bmv[mv[k] >> 5] >> (mv[k] & 31)) & 1u;
#pragma unroll
      for (uint32_t k = 0; k < kScanU; ++k) {
        const uint32_t bal = (__ballot_sync(T.mask, hit[k]) & T.mask) >> lead;  // bit r: team rank r
        if (hit[k]) nbrs[pos + __popc(bal & ((1u << T.rank) - 1u))] = mv[k];
        pos += __popc(bal);
      }
    }
  }
}

// Block per deferred (direction, candidate) item: the count as a block sum.
__global__ void __launch_bounds__(kHeavyBlock) k_cedge_count_heavy(GraphView g, const CedgeDir* __restrict__ dirs,
                                                                   uint32_t ndir,
                                                                   const unsigned long long* __restrict__ s_base,
                                                                   const uint32_t* __restrict__ bm, uint32_t words,
                                                                   uint32_t* __restrict__ cnt, HeavyList hl) {
  __shared__ uint32_t s_part[kHeavyBlock / 32];
  const uint32_t n = min(*hl.count, hl.cap);
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t w = hl.items[i];
    const uint32_t d = find_dir(s_base, ndir, w);
    const CedgeDir cd = dirs[d];
    const uint32_t mu = cd.ids[w - cd.item_base];
    const uint32_t* bmv = bm + (size_t)cd.v * words;
    const uint32_t b = g.off[mu], e = g.off[mu + 1];
    uint32_t rb, re;
    const uint32_t* cl = scan_range_block(g, mu, cd.lab, b, e, &rb, &re);
    uint32_t c = 0;
    for (uint32_t j = rb + threadIdx.x; j < re; j += blockDim.x) {
      const uint32_t mv = cl[j];
      c += (bmv[mv >> 5] >> (mv & 31)) & 1u;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (uint32_t k = 0; k < blockDim.x / 32; ++k) t += s_part[k];
      cnt[w] = t;
    }
    __syncthreads();
  }
}

// Block per deferred item: N(mu) ∩ C(v) written in adjacency order; each
// chunk of blockDim neighbours is compacted with warp ballots and a scan of
// the warp totals.
__global__ void __launch_bounds__(kHeavyBlock) k_cedge_write_heavy(GraphView g, const CedgeDir* __restrict__ dirs,
                                                                   uint32_t ndir,
                                                                   const unsigned long long* __restrict__ s_base,
                                                                   const uint32_t* __restrict__ bm, uint32_t words,
                                                                   const unsigned long long* __restrict__ goff,
                                                                   uint32_t* __restrict__ nbrs, HeavyList hl) {
  __shared__ uint32_t s_warp[kHeavyBlock / 32];
  __shared__ uint32_t s_total;
  const uint32_t n = min(*hl.count, hl.cap);
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x / 32;
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const uint32_t w = hl.items[i];
    const uint32_t d = find_dir(s_base, ndir, w);
    const CedgeDir cd = dirs[d];
    const uint32_t mu = cd.ids[w - cd.item_base];
    const uint32_t* bmv = bm + (size_t)cd.v * words;
    const uint32_t b = g.off[mu], e = g.off[mu + 1];
    uint32_t rb, re;
    const uint32_t* cl = scan_range_block(g, mu, cd.lab, b, e, &rb, &re);
    unsigned long long pos = goff[w];
    for (uint32_t j0 = rb; j0 < re; j0 += blockDim.x) {
      const uint32_t j = j0 + threadIdx.x;
      uint32_t mv = 0;
      bool hit = false;
      if (j < re) {
        mv = cl[j];
        hit = (bmv[mv >> 5] >> (mv & 31)) & 1u;
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, hit);
      if (lane == 0) s_warp[wid] = __popc(bal);
      __syncthreads();
      if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t k = 0; k < nw; ++k) {
          const uint32_t x = s_warp[k];
          s_warp[k] = run;
          run += x;
        }
        s_total = run;
      }
      __syncthreads();
      if (hit) nbrs[pos + s_warp[wid] + __popc(bal & ((1u << lane) - 1u))] = mv;
      pos += s_total;
      __syncthreads();
    }
  }
}

// Exclusive scan of n uint32 counts into n+1 uint64 offsets (out[n] = total).
constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;

__global__ void __launch_bounds__(kScanBlock) k_scan_u32(const uint32_t* __restrict__ in, unsigned long long n,
                                                        unsigned long long* __restrict__ out, Lookback lb) {
  __shared__ uint32_t s_tile;
  __shared__ unsigned long long s_prefix;
  if (threadIdx.x == 0) s_tile = lb_take_ticket(lb);
  __syncthreads();
  const uint32_t tile = s_tile;
  {
    const unsigned long long per = (unsigned long long)kScanBlock * kScanItems;
    const unsigned long long nt = (n + per - 1) / per;
    if ((unsigned long long)tile >= (nt ? nt : 1)) {
      if (threadIdx.x == 0) atomicOr(lb.flags, (uint32_t)DF_BOUNDS);
      return;
    }
  }
  const unsigned long long i0 = ((unsigned long long)tile * kScanBlock + threadIdx.x) * kScanItems;
  uint32_t v[kScanItems];
  unsigned long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (i0 + k < n) ? in[i0 + k] : 0;
    s += v[k];
  }
  unsigned long long total;
  unsigned long long mine = block_exclusive_scan<kScanBlock>(s, &total);
  if (threadIdx.x < 32) {
    unsigned long long ex = lb_exclusive(lb, tile, total);
    if (threadIdx.x == 0) s_prefix = ex;
  }
  __syncthreads();
  unsigned long long pos = s_prefix + mine;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (i0 + k < n) out[i0 + k] = pos;
    pos += v[k];
  }
  const unsigned long long per_tile = (unsigned long long)kScanBlock * kScanItems;
  const unsigned long long ntiles = (n + per_tile - 1) / per_tile;
  if (threadIdx.x == 0 && (unsigned long long)tile == (ntiles ? ntiles - 1 : 0)) out[n] = s_prefix + total;
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
static Lookback make_lb(Workspace& ws, uint32_t tiles) {
  Lookback lb;
  lb.ticket = ws.scan.d_ticket;
  lb.status = ws.scan.d_status;
  unsigned long long base;
  uint32_t ep;
  if (tiles > ws.scan.max_tiles) {
    set_last_error("scan: too many tiles");
    throw CudaError{cudaErrorInvalidValue, "scan tiles"};
  }
  ws.scan.next_launch(tiles, &base, &ep);
  lb.base = base;
  lb.epoch = ep;
  lb.flags = ws.d_flags;
  lb.spin_limit = tuning().scan_spin_limit;
  return lb;
}

static uint32_t grid_for(uint64_t warps_needed, uint32_t cap_blocks) {
  uint64_t blocks = (warps_needed + 7) / 8;
  if (blocks < 1) blocks = 1;
  if (blocks > cap_blocks) blocks = cap_blocks;
  return (uint32_t)blocks;
}

// Small device results to the workspace's page-locked mirror: one block
// stores the words into the mirror through its device address and fences
// them to the system, so the host reads them after a stream sync.
__global__ void k_words_to_host(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, uint32_t n) {
  for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
  __threadfence_system();
}

void small_to_host(Workspace& ws, void* h_dst, const void* d_src, size_t bytes) {
  const size_t off = (size_t)((const char*)h_dst - (const char*)ws.h_small);
  if (bytes == 0) return;
  if ((const char*)h_dst < (const char*)ws.h_small || off + bytes > 4096 * sizeof(unsigned long long) ||
      (off | bytes | (size_t)(uintptr_t)d_src) & 3) {
    set_last_error("small_to_host: destination outside the mirror or unaligned");
    throw CudaError{cudaErrorInvalidValue, "small_to_host"};
  }
  k_words_to_host<<<1, 256, 0, ws.stream>>>(static_cast<const uint32_t*>(d_src),
                                            reinterpret_cast<uint32_t*>((char*)ws.h_small_dev + off),
                                            (uint32_t)(bytes / 4));
  GPSM_LAUNCHED();
}

void launch_mark_range(Workspace& ws, const DeviceGraph& g, uint32_t begin, uint32_t end, uint32_t* bm) {
  if (end <= begin) return;
  uint32_t blocks = (uint32_t)std::min<uint64_t>((end - begin + 255) / 256, 148 * 8);
  k_mark_range<<<blocks, 256, 0, ws.stream>>>(g.lab_vtx, begin, end, bm);
  GPSM_LAUNCHED();
}

void launch_compact(Workspace& ws, const uint32_t* bm, uint32_t words, uint32_t* list, uint32_t* rank,
                    uint32_t* count, bool set_empty_flag, const uint32_t* stamp, uint32_t u, uint32_t prev) {
  uint32_t tiles = (words + kCompactWordsPerTile - 1) / kCompactWordsPerTile;
  Lookback lb = make_lb(ws, tiles);
  k_compact<<<tiles, kCompactBlock, 0, ws.stream>>>(bm, words, list, rank, count, lb, set_empty_flag ? 1u : 0u,
                                                     stamp, u, prev);
  GPSM_LAUNCHED();
}

void launch_compact_multi(Workspace& ws, const uint32_t* bm, uint32_t words, uint32_t nverts, uint32_t* const* d_lists,
                          uint32_t* rank, uint32_t* counts) {
  const uint32_t tiles = ((words + kCompactWordsPerTile - 1) / kCompactWordsPerTile) * nverts;
  Lookback lb = make_lb(ws, tiles);
  k_compact_multi<<<tiles, kCompactBlock, 0, ws.stream>>>(bm, words, nverts, d_lists, rank, counts, lb);
  GPSM_LAUNCHED();
}

static HeavyList heavy_list(Workspace& ws, const DeviceGraph& g) {
  HeavyList hl;
  hl.threshold = std::max<uint32_t>(tuning().heavy_degree, 32);
  if (g.max_degree <= hl.threshold || ws.d_heavy == nullptr) return hl;
  hl.items = ws.d_heavy;
  hl.count = ws.d_heavy_count;
  hl.cap = ws.heavy_cap;
  GPSM_CUDA(cudaMemsetAsync(ws.d_heavy_count, 0, sizeof(uint32_t), ws.stream));
  return hl;
}

// Words per warp chunk of a bitmap of `words` words: about 8192 warps (a
// full B200 holds 148 x 64), at most 32 words (one per lane) a chunk.
static uint32_t chunk_words(uint32_t words) { return std::max<uint32_t>(1, std::min<uint32_t>(32, (words + 8191) / 8192)); }

// Blocks of 8 warps that cover the bitmap in chunks of chunk_words(words).
static uint32_t light_blocks_for(uint32_t words) {
  const uint32_t cw = chunk_words(words);
  const uint32_t chunks = (words + cw - 1) / cw;
  return std::max<uint32_t>(1, std::min<uint32_t>((chunks + 7) / 8, 148 * 16));
}

template <bool EXPLORE>
static void launch_filter_step(Workspace& ws, const DeviceGraph& g, uint32_t u, uint32_t lab_u, uint32_t deg_u,
                               const uint32_t* tgt, uint32_t ntgt, uint32_t* bm, RefineStamp rs) {
  if (ntgt == 0) return;
  const uint32_t hub = std::max<uint32_t>(tuning().heavy_degree, 32);
  uint32_t hb = 0, he = 0;
  if (g.max_degree > hub) g.label_range(lab_u, std::max(hub + 1, deg_u), &hb, &he);
  const uint32_t light = light_blocks_for(g.words);
  const uint32_t hubs = std::min<uint32_t>(he - hb, (uint32_t)sm_count() * 2);
  const size_t smem = (EXPLORE ? 3 : 2) * ntgt * sizeof(uint32_t);
  // exploration scans every neighbour of the target's label: whole warps;
  // refinement stops at the first hit: the tuned team size
  const uint32_t team = EXPLORE ? tuning().explore_team : tuning().filter_team;
  if (EXPLORE && team < 32)
    k_filter_step<true, 8><<<light + hubs, 256, smem, ws.stream>>>(
        view(g), g.lab_vtx, hb, he, hub, light, chunk_words(g.words), u, tgt, ntgt, bm, g.words, ws.d_flags, rs);
  else if (EXPLORE || team >= 32)
    k_filter_step<EXPLORE, 32><<<light + hubs, 256, smem, ws.stream>>>(
        view(g), g.lab_vtx, hb, he, hub, light, chunk_words(g.words), u, tgt, ntgt, bm, g.words, ws.d_flags, rs);
  else if (team <= 4)
    k_filter_step<false, 4><<<light + hubs, 256, smem, ws.stream>>>(
        view(g), g.lab_vtx, hb, he, hub, light, chunk_words(g.words), u, tgt, ntgt, bm, g.words, ws.d_flags, rs);
  else
    k_filter_step<false, 8><<<light + hubs, 256, smem, ws.stream>>>(
        view(g), g.lab_vtx, hb, he, hub, light, chunk_words(g.words), u, tgt, ntgt, bm, g.words, ws.d_flags, rs);
  GPSM_LAUNCHED();
}

void launch_explore(Workspace& ws, const DeviceGraph& g, uint32_t u, uint32_t lab_u, uint32_t deg_u,
                    const uint32_t* tgt, uint32_t ntgt, uint32_t* bm) {
  launch_filter_step<true>(ws, g, u, lab_u, deg_u, tgt, ntgt, bm, RefineStamp());
}

void launch_refine(Workspace& ws, const DeviceGraph& g, uint32_t u, uint32_t lab_u, uint32_t deg_u,
                   const uint32_t* tgt, uint32_t ntgt, uint32_t* bm, RefineStamp rs) {
  launch_filter_step<false>(ws, g, u, lab_u, deg_u, tgt, ntgt, bm, rs);
}

void launch_cedge_count(Workspace& ws, const DeviceGraph& g, const CedgeDir* d_dirs, uint32_t ndir,
                        const unsigned long long* d_base, uint64_t items, const uint32_t* bm, uint32_t* cnt) {
  if (items == 0) return;
  HeavyList hl = heavy_list(ws, g);
  uint32_t blocks = grid_for((items + 3) / 4, 148 * 16);
  k_cedge_count<<<blocks, 256, 0, ws.stream>>>(view(g), d_dirs, ndir, d_base, bm, g.words, cnt, hl);
  GPSM_LAUNCHED();
  if (hl.items) {
    k_cedge_count_heavy<<<sm_count() * 2, kHeavyBlock, 0, ws.stream>>>(view(g), d_dirs, ndir, d_base, bm, g.words, cnt, hl);
    GPSM_LAUNCHED();
  }
}

void launch_cedge_write(Workspace& ws, const DeviceGraph& g, const CedgeDir* d_dirs, uint32_t ndir,
                        const unsigned long long* d_base, uint64_t items, const uint32_t* bm,
                        const unsigned long long* goff, uint32_t* nbrs) {
  if (items == 0) return;
  HeavyList hl = heavy_list(ws, g);
  uint32_t blocks = grid_for((items + 3) / 4, 148 * 16);
  k_cedge_write<<<blocks, 256, 0, ws.stream>>>(view(g), d_dirs, ndir, d_base, bm, g.words, goff, nbrs, hl);
  GPSM_LAUNCHED();
  if (hl.items) {
    k_cedge_write_heavy<<<sm_count() * 2, kHeavyBlock, 0, ws.stream>>>(view(g), d_dirs, ndir, d_base, bm, g.words, goff,
                                                                nbrs, hl);
    GPSM_LAUNCHED();
  }
}

void launch_scan_u32(Workspace& ws, const uint32_t* in, uint64_t n, unsigned long long* out) {
  const uint64_t per_tile = (uint64_t)kScanBlock * kScanItems;
  uint32_t tiles = (uint32_t)std::max<uint64_t>(1, (n + per_tile - 1) / per_tile);
  Lookback lb = make_lb(ws, tiles);
  k_scan_u32<<<tiles, kScanBlock, 0, ws.stream>>>(in, n, out, lb);
  GPSM_LAUNCHED();
}

}  // namespace gpsm
