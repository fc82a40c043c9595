// Undirected CSR construction on the device, the job Graph::transformToCSR
// does on the host (graph/Graph.cpp:30-65; its comment at :26-27 asks for a
// GPU version): every undirected edge (u, v) becomes the keys u<<32|v and
// v<<32|u, an LSD radix sort orders them by (source, target), and the
// targets in key order are the column array, every list ascending. Offsets
// are an exclusive scan of the degrees counted while the keys are written.
//
// Radix sort: 8-bit digits, only over the bits a vertex id can use (for
// 2^24 vertices, 3 digits of the target and 3 of the source). Each pass is
//   k_radix_hist     per-tile digit counts (4096 keys per tile), bin-major
//   k_scan_u32       exclusive scan of the counts (decoupled look-back)
//   k_radix_scatter  stable scatter: each warp owns a contiguous run of the
//                    tile, warp bases per digit come from per-warp counts,
//                    and lanes holding the same digit rank themselves with
//                    __match_any_sync, so equal digits keep their order.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "engine.h"
#include "filter.h"
#include "internal.h"

namespace gpsm {

constexpr int kSortBlock = 256;
constexpr int kSortWarps = kSortBlock / 32;
constexpr int kSortPerThread = 16;
constexpr int kSortTile = kSortBlock * kSortPerThread;  // 4096 keys
constexpr int kSortPerWarp = kSortTile / kSortWarps;    // 512 keys

__global__ void k_edge_keys(const uint32_t* __restrict__ edges, uint64_t m, unsigned long long* __restrict__ keys,
                            uint32_t* __restrict__ deg) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t u = edges[2 * i], v = edges[2 * i + 1];
    keys[2 * i] = ((unsigned long long)u << 32) | v;
    keys[2 * i + 1] = ((unsigned long long)v << 32) | u;
    atomicAdd(&deg[u], 1u);
    atomicAdd(&deg[v], 1u);
  }
}

__global__ void __launch_bounds__(kSortBlock) k_radix_hist(const unsigned long long* __restrict__ keys, uint64_t n,
                                                           uint32_t shift, uint32_t ntiles,
                                                           uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  for (int k = 0; k < kSortPerThread; ++k) {
    const uint64_t i = base + (uint64_t)k * kSortBlock + threadIdx.x;
    if (i < n) atomicAdd(&h[(uint32_t)(keys[i] >> shift) & 0xff], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(kSortBlock) k_radix_scatter(const unsigned long long* __restrict__ in,
                                                              unsigned long long* __restrict__ out, uint64_t n,
                                                              uint32_t shift, uint32_t ntiles,
                                                              const unsigned long long* __restrict__ off) {
  __shared__ uint32_t wh[kSortWarps][256];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (uint32_t d = threadIdx.x; d < kSortWarps * 256; d += blockDim.x) (&wh[0][0])[d] = 0;
  __syncthreads();
  const uint64_t wbase = (uint64_t)blockIdx.x * kSortTile + (uint64_t)wid * kSortPerWarp;
  // per-warp digit counts of the warp's contiguous run
  for (int k = 0; k < kSortPerWarp / 32; ++k) {
    const uint64_t i = wbase + (uint64_t)k * 32 + lane;
    if (i < n) atomicAdd(&wh[wid][(uint32_t)(in[i] >> shift) & 0xff], 1u);
  }
  __syncthreads();
  // warp bases per digit: earlier warps of the tile come first
  {
    const uint32_t d = threadIdx.x;  // blockDim == 256 == digits
    uint32_t run = 0;
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t t = wh[w][d];
      wh[w][d] = run;
      run += t;
    }
  }
  __syncthreads();
  for (int k = 0; k < kSortPerWarp / 32; ++k) {
    const uint64_t i = wbase + (uint64_t)k * 32 + lane;
    const bool valid = i < n;
    const unsigned long long key = valid ? in[i] : 0ULL;
    const uint32_t d = valid ? ((uint32_t)(key >> shift) & 0xff) : 256u;
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    const uint32_t leader = __ffs(peers) - 1;
    if (valid) out[off[(uint64_t)d * ntiles + blockIdx.x] + wh[wid][d] + rank] = key;
    __syncwarp();
    if (valid && lane == leader) wh[wid][d] += __popc(peers);
    __syncwarp();
  }
}

__global__ void k_keys_to_cols(const unsigned long long* __restrict__ keys, uint64_t n, uint32_t* __restrict__ cols) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    cols[i] = (uint32_t)keys[i];
}

__global__ void k_u64_to_u32(const unsigned long long* __restrict__ a, uint64_t n, uint32_t* __restrict__ b) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

static int bits_of(uint64_t n) {
  int b = 1;
  while ((1ULL << b) < n) ++b;
  return b;
}

// Stable LSD passes (8-bit digits at `shifts`) from a into b and back;
// returns the buffer holding the sorted keys.
static unsigned long long* radix_passes(Workspace& ws, unsigned long long* a, unsigned long long* b, uint64_t nk,
                                        const std::vector<uint32_t>& shifts, uint32_t* hist,
                                        unsigned long long* hoff) {
  const uint32_t ntiles = (uint32_t)((nk + kSortTile - 1) / kSortTile);
  for (uint32_t sh : shifts) {
    if (nk == 0) break;
    k_radix_hist<<<ntiles, kSortBlock, 0, ws.stream>>>(a, nk, sh, ntiles, hist);
    GPSM_LAUNCHED();
    launch_scan_u32(ws, hist, (uint64_t)256 * ntiles, hoff);
    k_radix_scatter<<<ntiles, kSortBlock, 0, ws.stream>>>(a, b, nk, sh, ntiles, hoff);
    GPSM_LAUNCHED();
    std::swap(a, b);
  }
  return a;
}

// Builds offsets[n+1] and cols[2m] on the device from host edges (m pairs).
// Scratch comes from ws.arena (reset first). Returns the device arrays,
// allocated with cudaMalloc (the graph owns them).
void build_csr_device(Workspace& ws, uint32_t n, uint64_t m, const uint32_t* h_edges, uint32_t** d_off,
                      uint32_t** d_cols) {
  const uint64_t nk = 2 * m;
  if (nk >= (1ull << 32)) {
    set_last_error("graph too large for 32-bit offsets");
    throw CudaError{cudaErrorInvalidValue, "csr size"};
  }
  cudaStream_t s = ws.stream;
  ws.arena.reset();
  auto take = [&](size_t bytes) {
    void* p = ws.arena.alloc(std::max<size_t>(bytes, 16));
    if (!p) {
      set_last_error("csr build: workspace too small");
      throw CudaError{cudaErrorMemoryAllocation, "csr arena"};
    }
    return p;
  };
  uint32_t* e = (uint32_t*)take(m * 8);
  unsigned long long* ka = (unsigned long long*)take(nk * 8);
  unsigned long long* kb = (unsigned long long*)take(nk * 8);
  uint32_t* deg = (uint32_t*)take((uint64_t)(n + 1) * 4);
  unsigned long long* off64 = (unsigned long long*)take((uint64_t)(n + 2) * 8);
  const uint32_t ntiles = (uint32_t)((nk + kSortTile - 1) / kSortTile);
  uint32_t* hist = (uint32_t*)take((uint64_t)256 * std::max<uint32_t>(ntiles, 1) * 4);
  unsigned long long* hoff = (unsigned long long*)take(((uint64_t)256 * std::max<uint32_t>(ntiles, 1) + 1) * 8);
  if (m) GPSM_CUDA(cudaMemcpyAsync(e, h_edges, m * 8, cudaMemcpyHostToDevice, s));
  GPSM_CUDA(cudaMemsetAsync(deg, 0, (uint64_t)(n + 1) * 4, s));
  const uint32_t grid = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>((m + 255) / 256, 148 * 16));
  if (m) {
    k_edge_keys<<<grid, 256, 0, s>>>(e, m, ka, deg);
    GPSM_LAUNCHED();
  }
  // key bits: target in [0, b), source in [32, 32 + b)
  const int b = bits_of(n);
  std::vector<uint32_t> shifts;
  for (int sh = 0; sh < b; sh += 8) shifts.push_back(sh);
  for (int sh = 0; sh < b; sh += 8) shifts.push_back(32 + sh);
  unsigned long long* src = radix_passes(ws, ka, kb, nk, shifts, hist, hoff);
  launch_scan_u32(ws, deg, n + 1, off64);  // off64[i] = sum of deg[0..i)
  GPSM_CUDA(cudaMalloc(d_off, (uint64_t)(n + 1) * 4));
  GPSM_CUDA(cudaMalloc(d_cols, std::max<uint64_t>(nk, 1) * 4));
  k_u64_to_u32<<<(n + 256) / 256, 256, 0, s>>>(off64, n + 1, *d_off);
  GPSM_LAUNCHED();
  if (nk) {
    k_keys_to_cols<<<(uint32_t)std::min<uint64_t>((nk + 255) / 256, 148 * 32), 256, 0, s>>>(src, nk, *d_cols);
    GPSM_LAUNCHED();
  }
  GPSM_CUDA(cudaStreamSynchronize(s));
}

// ---------------------------------------------------------------------------
// Label runs: each adjacency list sorted by (neighbour label, id), and a
// directory of its runs. Keys hold (vertex << lbits | label rank) in the
// high word and the neighbour in the low word; the CSR already orders them
// by (vertex, neighbour), so stable passes over the high word alone give
// (vertex, label, neighbour) order.
// ---------------------------------------------------------------------------
__global__ void k_label_keys(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col,
                             const uint32_t* __restrict__ lrank, uint32_t n, uint32_t lbits,
                             unsigned long long* __restrict__ keys) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps)
    for (uint32_t j = off[v] + lane; j < off[v + 1]; j += 32) {
      const uint32_t u = col[j];
      keys[j] = ((unsigned long long)((v << lbits) | lrank[u]) << 32) | u;
    }
}

// Runs per vertex: positions where the high word changes (or the list starts).
__global__ void k_label_runs_count(const uint32_t* __restrict__ off, const unsigned long long* __restrict__ keys,
                                   uint32_t n, uint32_t* __restrict__ cnt) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint32_t b = off[v], e = off[v + 1];
    uint32_t c = 0;
    for (uint32_t j = b + lane; j < e; j += 32) c += (j == b || (keys[j] >> 32) != (keys[j - 1] >> 32)) ? 1u : 0u;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[v] = c;
  }
}

__global__ void k_label_runs_write(const uint32_t* __restrict__ off, const unsigned long long* __restrict__ keys,
                                   uint32_t n, const unsigned long long* __restrict__ run_base,
                                   const uint32_t* __restrict__ label_of_rank, uint32_t lmask,
                                   uint32_t* __restrict__ lcol, uint2* __restrict__ runs) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
    const uint32_t b = off[v], e = off[v + 1];
    unsigned long long pos = run_base[v];
    for (uint32_t j0 = b; j0 < e; j0 += 32) {
      const uint32_t j = j0 + lane;
      bool start = false;
      unsigned long long k = 0;
      if (j < e) {
        k = keys[j];
        lcol[j] = (uint32_t)k;
        start = j == b || (k >> 32) != (keys[j - 1] >> 32);
      }
      const uint32_t bal = __ballot_sync(0xffffffffu, start);
      if (start) runs[pos + __popc(bal & ((1u << lane) - 1u))] = make_uint2(label_of_rank[(k >> 32) & lmask], j);
      pos += __popc(bal);
    }
  }
}

// A warp per vertex u inserts its edges (u, b) with u < b: a slot holds the
// key or, if empty, takes it by compare-and-swap; otherwise the next slot.
// The longest distance from a key's home slot goes to *probe; a key that
// would go farther than kMaxProbe sets DF_OVERFLOW and is dropped (the
// table is then not used).
constexpr uint32_t kMaxProbe = 4096;

__global__ void k_edge_hash_build(const uint32_t* __restrict__ off, const uint32_t* __restrict__ col, uint32_t n,
                                  unsigned long long* __restrict__ table, uint32_t bits, uint32_t* __restrict__ probe,
                                  uint32_t* __restrict__ flags) {
  const uint32_t lane = threadIdx.x & 31;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const unsigned long long mask = (1ull << bits) - 1;
  uint32_t longest = 0;
  for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += nwarps) {
    const uint32_t e = off[u + 1];
    for (uint32_t j = off[u] + lane; j < e; j += 32) {
      const uint32_t b = col[j];
      if (b <= u) continue;
      const unsigned long long key = (unsigned long long)u << 32 | b;
      unsigned long long s = (key * 0x9E3779B97F4A7C15ull) >> (64 - bits);
      uint32_t d = 0;
      for (;; ++d) {
        if (d > kMaxProbe) {
          atomicOr(flags, (uint32_t)DF_OVERFLOW);
          break;
        }
        const unsigned long long prev = atomicCAS(table + s, ~0ull, key);
        if (prev == ~0ull || prev == key) break;
        s = (s + 1) & mask;
      }
      longest = max(longest, d);
    }
  }
  for (int o = 16; o > 0; o >>= 1) longest = max(longest, __shfl_xor_sync(0xffffffffu, longest, o));
  if (lane == 0 && longest) atomicMax(probe, longest);
}

void build_edge_hash(DeviceGraph& g) {
  const uint64_t edges = g.nnz / 2;
  if (edges == 0) return;
  uint32_t bits = 10;
  while ((1ull << bits) < 2 * edges) ++bits;  // at most half full
  const size_t bytes = (size_t)8 << bits;
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess || bytes > free_b / 4) {
    cudaGetLastError();
    return;  // the joins search the lists instead
  }
  unsigned long long* table = nullptr;
  uint32_t* d_aux = nullptr;  // [0] longest probe, [1] flags
  if (cudaMalloc(&table, bytes) != cudaSuccess || cudaMalloc(&d_aux, 8) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(table);
    cudaFree(d_aux);
    return;
  }
  uint32_t aux[2] = {0, 0};
  bool ok = cudaMemset(table, 0xff, bytes) == cudaSuccess && cudaMemset(d_aux, 0, 8) == cudaSuccess;
  if (ok) {
    const uint32_t grid = (uint32_t)std::min<uint64_t>(((uint64_t)g.n * 32 + 255) / 256, 148 * 64);
    k_edge_hash_build<<<grid, 256>>>(g.off, g.col, g.n, table, bits, d_aux, d_aux + 1);
    ok = cudaGetLastError() == cudaSuccess && cudaMemcpy(aux, d_aux, 8, cudaMemcpyDeviceToHost) == cudaSuccess;
  }
  cudaFree(d_aux);
  if (!ok || (aux[1] & DF_OVERFLOW)) {
    cudaGetLastError();
    cudaFree(table);
    return;
  }
  g.ehash = table;
  g.ehash_bits = bits;
  g.ehash_probe = aux[0];
}

void build_label_runs(DeviceGraph& g, const uint32_t* h_lab) {
  const uint32_t n = g.n;
  const uint64_t nnz = g.nnz;
  const uint32_t L = (uint32_t)g.h_labels.size();
  const int vbits = bits_of(n), lbits = bits_of(std::max<uint32_t>(L, 2));
  if (nnz == 0 || vbits + lbits > 32) return;  // the filter scans whole lists
  std::vector<uint32_t> lrank(n);
  for (uint32_t x = 0; x < n; ++x)
    lrank[x] = (uint32_t)(std::lower_bound(g.h_labels.begin(), g.h_labels.end(), h_lab[x]) - g.h_labels.begin());
  const uint32_t ntiles = (uint32_t)((nnz + kSortTile - 1) / kSortTile);
  const uint64_t arena = 2 * nnz * 8 + (uint64_t)256 * ntiles * 4 + ((uint64_t)256 * ntiles + 1) * 8 +
                         (uint64_t)(n + 1) * 16 + (uint64_t)L * 4 + (64ull << 20);
  Workspace* ws = workspace_create(g.device, arena, 1u << 20);
  try {
    auto take = [&](size_t bytes) {
      void* p = ws->arena.alloc(std::max<size_t>(bytes, 16));
      if (!p) throw CudaError{cudaErrorMemoryAllocation, "label runs arena"};
      return p;
    };
    unsigned long long* ka = (unsigned long long*)take(nnz * 8);
    unsigned long long* kb = (unsigned long long*)take(nnz * 8);
    uint32_t* hist = (uint32_t*)take((uint64_t)256 * ntiles * 4);
    unsigned long long* hoff = (unsigned long long*)take(((uint64_t)256 * ntiles + 1) * 8);
    uint32_t* d_lrank = (uint32_t*)take((uint64_t)n * 4);
    uint32_t* d_cnt = (uint32_t*)take((uint64_t)(n + 1) * 4);
    unsigned long long* d_base = (unsigned long long*)take((uint64_t)(n + 2) * 8);
    uint32_t* d_labels = (uint32_t*)take((uint64_t)std::max<uint32_t>(L, 1) * 4);
    cudaStream_t s = ws->stream;
    GPSM_CUDA(cudaMemcpyAsync(d_lrank, lrank.data(), (uint64_t)n * 4, cudaMemcpyHostToDevice, s));
    GPSM_CUDA(cudaMemcpyAsync(d_labels, g.h_labels.data(), (uint64_t)L * 4, cudaMemcpyHostToDevice, s));
    const uint32_t vgrid = (uint32_t)std::min<uint64_t>(((uint64_t)n * 32 + 255) / 256, 148 * 64);
    k_label_keys<<<vgrid, 256, 0, s>>>(g.off, g.col, d_lrank, n, (uint32_t)lbits, ka);
    GPSM_LAUNCHED();
    std::vector<uint32_t> shifts;
    for (int sh = 0; sh < vbits + lbits; sh += 8) shifts.push_back(32 + sh);
    unsigned long long* sorted = radix_passes(*ws, ka, kb, nnz, shifts, hist, hoff);
    k_label_runs_count<<<vgrid, 256, 0, s>>>(g.off, sorted, n, d_cnt);
    GPSM_LAUNCHED();
    launch_scan_u32(*ws, d_cnt, n, d_base);  // d_base[n] = runs in all
    unsigned long long total = 0;
    GPSM_CUDA(cudaMemcpyAsync(&total, d_base + n, 8, cudaMemcpyDeviceToHost, s));
    GPSM_CUDA(cudaStreamSynchronize(s));
    GPSM_CUDA(cudaMalloc(&g.lcol, nnz * 4));
    GPSM_CUDA(cudaMalloc(&g.run_off, (uint64_t)(n + 1) * 4));
    GPSM_CUDA(cudaMalloc(&g.runs, std::max<uint64_t>(total, 1) * sizeof(uint2)));
    k_u64_to_u32<<<(n + 256) / 256, 256, 0, s>>>(d_base, n + 1, g.run_off);
    GPSM_LAUNCHED();
    k_label_runs_write<<<vgrid, 256, 0, s>>>(g.off, sorted, n, d_base, d_labels, (1u << lbits) - 1u, g.lcol,
                                             g.runs);
    GPSM_LAUNCHED();
    GPSM_CUDA(cudaStreamSynchronize(s));
    uint32_t flags = 0;
    GPSM_CUDA(cudaMemcpy(&flags, ws->d_flags, 4, cudaMemcpyDeviceToHost));
    if (flags & (DF_SCAN_TIMEOUT | DF_BOUNDS)) {
      set_last_error("label runs: device wait limit or bounds check tripped");
      throw CudaError{cudaErrorLaunchFailure, "label runs"};
    }
  } catch (...) {
    cudaFree(g.lcol);
    cudaFree(g.run_off);
    cudaFree(g.runs);
    g.lcol = g.run_off = nullptr;
    g.runs = nullptr;
    workspace_free(ws);
    throw;
  }
  workspace_free(ws);
}

}  // namespace gpsm
