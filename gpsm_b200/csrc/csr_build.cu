// Undirected CSR construction on the device, the job Graph::transformToCSR
// does on the host (graph/Graph.cpp:190-226; its comment at :187 asks for a
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
  unsigned long long* src = ka;
  unsigned long long* dst = kb;
  for (uint32_t sh : shifts) {
    if (nk == 0) break;
    k_radix_hist<<<ntiles, kSortBlock, 0, s>>>(src, nk, sh, ntiles, hist);
    GPSM_LAUNCHED();
    launch_scan_u32(ws, hist, (uint64_t)256 * ntiles, hoff);
    k_radix_scatter<<<ntiles, kSortBlock, 0, s>>>(src, dst, nk, sh, ntiles, hoff);
    GPSM_LAUNCHED();
    std::swap(src, dst);
  }
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

}  // namespace gpsm
