// Device-resident data graph and per-stream workspaces.
//
// The reference copies the whole data CSR to the GPU inside every
// Match::match call (copyGraphToGPU, match/Match.cu:128-143, called at
// :1714) and frees only part of it afterwards. Here the graph is uploaded
// once (gpsm_graph_upload) and every query reuses it. Upload also builds two
// derived arrays that the reference does not have:
//   labdeg[x]  = (label, degree): one 8-byte gather per neighbour in the
//                filter kernels instead of three 4-byte gathers;
//   lab_vtx    = vertices grouped by label, degree descending: the root
//                candidates of a query vertex (label l, degree >= d) are a
//                prefix of label l's group, so initialisation touches only
//                those vertices instead of scanning all N (check_kernel,
//                match/Match.cu:431-446);
//   lcol, runs = every adjacency list sorted by (neighbour label, id) with a
//                directory of its label runs (csr_build.cu): the filter
//                scans only the neighbours that carry a target's label.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>

#include "filter.h"
#include "internal.h"

namespace gpsm {

static Tuning g_tuning;
Tuning& tuning() { return g_tuning; }

int sm_count() {
  static int cached = 0;
  if (cached == 0) {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && n > 0)
      cached = n;
    else
      return 148;
  }
  return cached;
}

static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* last_error() { return g_last_error.c_str(); }

__global__ void k_labdeg(const uint32_t* __restrict__ off, const uint32_t* __restrict__ lab, uint32_t n,
                         uint2* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = make_uint2(lab[i], off[i + 1] - off[i]);
}

uint64_t DeviceGraph::label_count(uint32_t label) const {
  auto it = std::lower_bound(h_labels.begin(), h_labels.end(), label);
  if (it == h_labels.end() || *it != label) return 0;
  size_t k = it - h_labels.begin();
  return h_lab_ptr[k + 1] - h_lab_ptr[k];
}

void DeviceGraph::label_range(uint32_t label, uint32_t d, uint32_t* begin, uint32_t* end) const {
  auto it = std::lower_bound(h_labels.begin(), h_labels.end(), label);
  if (it == h_labels.end() || *it != label) {
    *begin = *end = 0;
    return;
  }
  size_t k = it - h_labels.begin();
  uint32_t b = h_lab_ptr[k], e = h_lab_ptr[k + 1];
  // degrees descend within the group: find the first position with degree < d
  const uint32_t* p = h_lab_deg.data();
  uint32_t lo = b, hi = e;
  while (lo < hi) {
    uint32_t mid = lo + (hi - lo) / 2;
    if (p[mid] >= d) lo = mid + 1;
    else hi = mid;
  }
  *begin = b;
  *end = lo;
}

// Label index, derived arrays and bookkeeping for a graph whose offsets are
// known on the host and whose CSR arrays are already on the device.
static DeviceGraph* graph_finish(int device, uint32_t n, const uint32_t* off, const uint32_t* lab, uint32_t* d_off,
                                 uint32_t* d_col) {
  DeviceGraph* g = new DeviceGraph();
  g->device = device;
  g->n = n;
  g->nnz = off[n];
  g->words = (((n + 31) / 32) + 3) & ~3u;
  g->off = d_off;
  g->col = d_col;
  uint32_t maxd = 0;
  for (uint32_t i = 0; i < n; ++i) maxd = std::max(maxd, off[i + 1] - off[i]);
  g->max_degree = maxd;
  std::vector<uint32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0u);
  std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
    if (lab[a] != lab[b]) return lab[a] < lab[b];
    uint32_t da = off[a + 1] - off[a], db = off[b + 1] - off[b];
    if (da != db) return da > db;
    return a < b;
  });
  g->h_lab_deg.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t x = idx[i];
    g->h_lab_deg[i] = off[x + 1] - off[x];
    if (i == 0 || lab[x] != lab[idx[i - 1]]) {
      g->h_labels.push_back(lab[x]);
      g->h_lab_ptr.push_back(i);
    }
  }
  g->h_lab_ptr.push_back(n);
  try {
    GPSM_CUDA(cudaMalloc(&g->lab, sizeof(uint32_t) * n));
    GPSM_CUDA(cudaMalloc(&g->labdeg, sizeof(uint2) * n));
    GPSM_CUDA(cudaMalloc(&g->lab_vtx, sizeof(uint32_t) * n));
    GPSM_CUDA(cudaMemcpy(g->lab, lab, sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    GPSM_CUDA(cudaMemcpy(g->lab_vtx, idx.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    k_labdeg<<<std::min<uint32_t>((n + 255) / 256, 148 * 8), 256>>>(g->off, g->lab, n, g->labdeg);
    GPSM_LAUNCHED();
    GPSM_CUDA(cudaDeviceSynchronize());
    build_label_runs(*g, lab);
    build_edge_hash(*g);
  } catch (...) {
    cudaFree(g->off);
    cudaFree(g->col);
    cudaFree(g->lab);
    cudaFree(g->labdeg);
    cudaFree(g->lab_vtx);
    delete g;
    throw;
  }
  return g;
}

void build_csr_device(Workspace& ws, uint32_t n, uint64_t m, const uint32_t* h_edges, uint32_t** d_off,
                      uint32_t** d_cols);

// CSR built on the device from an edge list (every undirected edge once).
DeviceGraph* graph_build(Workspace& ws, const uint32_t* edges, uint64_t m, const uint32_t* lab, uint32_t n) {
  if (n == 0 || lab == nullptr || (m && edges == nullptr)) throw CudaError{cudaErrorInvalidValue, "graph args"};
  for (uint64_t i = 0; i < 2 * m; ++i)
    if (edges[i] >= n) {
      set_last_error("edge endpoint out of range");
      throw CudaError{cudaErrorInvalidValue, "edges"};
    }
  GPSM_CUDA(cudaSetDevice(ws.device));
  uint32_t *d_off = nullptr, *d_col = nullptr;
  build_csr_device(ws, n, m, edges, &d_off, &d_col);
  std::vector<uint32_t> off(n + 1);
  GPSM_CUDA(cudaMemcpy(off.data(), d_off, (n + 1) * 4ull, cudaMemcpyDeviceToHost));
  return graph_finish(ws.device, n, off.data(), lab, d_off, d_col);
}

void graph_download(const DeviceGraph* g, uint32_t* off, uint32_t* col) {
  GPSM_CUDA(cudaSetDevice(g->device));
  if (off) GPSM_CUDA(cudaMemcpy(off, g->off, (g->n + 1) * 4ull, cudaMemcpyDeviceToHost));
  if (col && g->nnz) GPSM_CUDA(cudaMemcpy(col, g->col, g->nnz * 4ull, cudaMemcpyDeviceToHost));
}

DeviceGraph* graph_upload(int device, const uint32_t* off, const uint32_t* col, const uint32_t* lab, uint32_t n) {
  if (n == 0 || off == nullptr || lab == nullptr) throw CudaError{cudaErrorInvalidValue, "graph args"};
  const uint64_t nnz = off[n];
  if (nnz > 0 && col == nullptr) throw CudaError{cudaErrorInvalidValue, "graph cols"};
  if (off[0] != 0) {
    set_last_error("graph offsets must start at 0");
    throw CudaError{cudaErrorInvalidValue, "offsets"};
  }
  for (uint32_t i = 0; i < n; ++i)
    if (off[i + 1] < off[i]) {
      set_last_error("graph offsets are not monotone");
      throw CudaError{cudaErrorInvalidValue, "offsets"};
    }
  for (uint64_t j = 0; j < nnz; ++j)
    if (col[j] >= n) {
      set_last_error("graph column index out of range");
      throw CudaError{cudaErrorInvalidValue, "cols"};
    }
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = off[i] + 1; j < off[i + 1]; ++j)
      if (col[j] < col[j - 1]) {
        set_last_error("graph adjacency lists must be sorted ascending");
        throw CudaError{cudaErrorInvalidValue, "cols"};
      }
  GPSM_CUDA(cudaSetDevice(device));
  DeviceGraph* g = new DeviceGraph();
  g->device = device;
  g->n = n;
  g->nnz = nnz;
  g->words = (((n + 31) / 32) + 3) & ~3u;
  uint32_t maxd = 0;
  for (uint32_t i = 0; i < n; ++i) maxd = std::max(maxd, off[i + 1] - off[i]);
  g->max_degree = maxd;
  // label index on the host: stable by (label asc, degree desc, id asc)
  std::vector<uint32_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0u);
  std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
    if (lab[a] != lab[b]) return lab[a] < lab[b];
    uint32_t da = off[a + 1] - off[a], db = off[b + 1] - off[b];
    if (da != db) return da > db;
    return a < b;
  });
  g->h_lab_deg.resize(n);
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t x = idx[i];
    g->h_lab_deg[i] = off[x + 1] - off[x];
    if (i == 0 || lab[x] != lab[idx[i - 1]]) {
      g->h_labels.push_back(lab[x]);
      g->h_lab_ptr.push_back(i);
    }
  }
  g->h_lab_ptr.push_back(n);
  try {
    GPSM_CUDA(cudaMalloc(&g->off, sizeof(uint32_t) * (n + 1)));
    GPSM_CUDA(cudaMalloc(&g->col, sizeof(uint32_t) * std::max<uint64_t>(nnz, 1)));
    GPSM_CUDA(cudaMalloc(&g->lab, sizeof(uint32_t) * n));
    GPSM_CUDA(cudaMalloc(&g->labdeg, sizeof(uint2) * n));
    GPSM_CUDA(cudaMalloc(&g->lab_vtx, sizeof(uint32_t) * n));
    GPSM_CUDA(cudaMemcpy(g->off, off, sizeof(uint32_t) * (n + 1), cudaMemcpyHostToDevice));
    if (nnz) GPSM_CUDA(cudaMemcpy(g->col, col, sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice));
    GPSM_CUDA(cudaMemcpy(g->lab, lab, sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    GPSM_CUDA(cudaMemcpy(g->lab_vtx, idx.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    k_labdeg<<<std::min<uint32_t>((n + 255) / 256, 148 * 8), 256>>>(g->off, g->lab, n, g->labdeg);
    GPSM_LAUNCHED();
    GPSM_CUDA(cudaDeviceSynchronize());
    build_label_runs(*g, lab);
    build_edge_hash(*g);
  } catch (...) {
    cudaFree(g->off);
    cudaFree(g->col);
    cudaFree(g->lab);
    cudaFree(g->labdeg);
    cudaFree(g->lab_vtx);
    delete g;
    throw;
  }
  return g;
}

void graph_set_directed(DeviceGraph* g, uint64_t m, const uint32_t* edges, const uint32_t* labels) {
  std::vector<uint32_t> off(g->n + 1, 0);
  for (uint64_t i = 0; i < m; ++i) {
    if (edges[2 * i] >= g->n || edges[2 * i + 1] >= g->n) {
      set_last_error("directed edge endpoint out of range");
      throw CudaError{cudaErrorInvalidValue, "directed edges"};
    }
    off[edges[2 * i] + 1]++;
  }
  for (uint32_t i = 0; i < g->n; ++i) off[i + 1] += off[i];
  std::vector<uint64_t> key(m);  // (source, target, label) sorted: targets ascending per source
  std::vector<uint32_t> pos(off.begin(), off.end() - 1);
  std::vector<uint32_t> col(m), lab(m);
  for (uint64_t i = 0; i < m; ++i) {
    const uint32_t a = edges[2 * i];
    const uint32_t k = pos[a]++;
    col[k] = edges[2 * i + 1];
    lab[k] = labels ? labels[i] : 1u;
  }
  for (uint32_t a = 0; a < g->n; ++a) {
    std::vector<std::pair<uint32_t, uint32_t>> t;
    for (uint32_t k = off[a]; k < off[a + 1]; ++k) t.emplace_back(col[k], lab[k]);
    std::sort(t.begin(), t.end());
    for (uint32_t k = off[a]; k < off[a + 1]; ++k) {
      col[k] = t[k - off[a]].first;
      lab[k] = t[k - off[a]].second;
    }
  }
  GPSM_CUDA(cudaSetDevice(g->device));
  cudaFree(g->dir_off);
  cudaFree(g->dir_col);
  cudaFree(g->dir_lab);
  g->dir_off = g->dir_col = g->dir_lab = nullptr;
  GPSM_CUDA(cudaMalloc(&g->dir_off, (g->n + 1) * 4));
  GPSM_CUDA(cudaMalloc(&g->dir_col, std::max<uint64_t>(m, 1) * 4));
  GPSM_CUDA(cudaMalloc(&g->dir_lab, std::max<uint64_t>(m, 1) * 4));
  GPSM_CUDA(cudaMemcpy(g->dir_off, off.data(), (g->n + 1) * 4, cudaMemcpyHostToDevice));
  if (m) {
    GPSM_CUDA(cudaMemcpy(g->dir_col, col.data(), m * 4, cudaMemcpyHostToDevice));
    GPSM_CUDA(cudaMemcpy(g->dir_lab, lab.data(), m * 4, cudaMemcpyHostToDevice));
  }
}

void graph_free(DeviceGraph* g) {
  if (!g) return;
  cudaSetDevice(g->device);
  cudaFree(g->dir_off);
  cudaFree(g->dir_col);
  cudaFree(g->dir_lab);
  cudaFree(g->off);
  cudaFree(g->col);
  cudaFree(g->lab);
  cudaFree(g->labdeg);
  cudaFree(g->lab_vtx);
  cudaFree(g->lcol);
  cudaFree(g->run_off);
  cudaFree(g->runs);
  cudaFree(g->ehash);
  delete g;
}

Workspace* workspace_create(int device, size_t arena_bytes, uint32_t max_tiles) {
  GPSM_CUDA(cudaSetDevice(device));
  arena_bytes = std::max<size_t>(arena_bytes & ~((size_t(2) << 20) - 1), size_t(2) << 20);  // whole 2 MiB units
  Workspace* ws = new Workspace();
  ws->device = device;
  try {
    GPSM_CUDA(cudaStreamCreateWithFlags(&ws->stream, cudaStreamNonBlocking));
    GPSM_CUDA(cudaStreamCreateWithFlags(&ws->copy_stream, cudaStreamNonBlocking));
    for (int i = 0; i < 2; ++i) {
      GPSM_CUDA(cudaEventCreateWithFlags(&ws->ev_res[i], cudaEventDisableTiming));
      GPSM_CUDA(cudaEventCreateWithFlags(&ws->ev_copied[i], cudaEventDisableTiming));
    }
    GPSM_CUDA(cudaMalloc(&ws->arena.base, arena_bytes));
    ws->arena.size = arena_bytes;
    ws->scan.max_tiles = max_tiles;
    GPSM_CUDA(cudaMalloc(&ws->scan.d_ticket, sizeof(unsigned long long)));
    GPSM_CUDA(cudaMemset(ws->scan.d_ticket, 0, sizeof(unsigned long long)));
    GPSM_CUDA(cudaMalloc(&ws->scan.d_status, sizeof(unsigned long long) * max_tiles));
    GPSM_CUDA(cudaMemset(ws->scan.d_status, 0, sizeof(unsigned long long) * max_tiles));
    GPSM_CUDA(cudaMalloc(&ws->d_flags, 64 * sizeof(uint32_t)));
    GPSM_CUDA(cudaMemset(ws->d_flags, 0, 64 * sizeof(uint32_t)));
    GPSM_CUDA(cudaMalloc(&ws->d_small, 4096 * sizeof(unsigned long long)));
    ws->heavy_cap = 1u << 20;
    GPSM_CUDA(cudaMalloc(&ws->d_heavy, ws->heavy_cap * sizeof(uint32_t)));
    GPSM_CUDA(cudaMalloc(&ws->d_heavy_count, sizeof(uint32_t)));
    GPSM_CUDA(cudaMallocHost(&ws->h_small, 4096 * sizeof(unsigned long long)));
    GPSM_CUDA(cudaHostGetDevicePointer((void**)&ws->h_small_dev, ws->h_small, 0));
    GPSM_CUDA(cudaEventCreate(&ws->ev0));
    GPSM_CUDA(cudaEventCreate(&ws->evm));
    GPSM_CUDA(cudaEventCreate(&ws->eve0));
    GPSM_CUDA(cudaEventCreate(&ws->eve1));
    GPSM_CUDA(cudaEventCreate(&ws->evb0));
    GPSM_CUDA(cudaEventCreate(&ws->evb1));
    GPSM_CUDA(cudaEventCreate(&ws->ev1));
  } catch (...) {
    // partial construction: release what exists
    if (ws->stream) cudaStreamDestroy(ws->stream);
    if (ws->copy_stream) cudaStreamDestroy(ws->copy_stream);
    cudaFree(ws->arena.base);
    cudaFree(ws->scan.d_ticket);
    cudaFree(ws->scan.d_status);
    cudaFree(ws->d_flags);
    cudaFree(ws->d_small);
    cudaFree(ws->d_heavy);
    cudaFree(ws->d_heavy_count);
    if (ws->h_small) cudaFreeHost(ws->h_small);
    delete ws;
    throw;
  }
  return ws;
}

void workspace_free(Workspace* ws) {
  if (!ws) return;
  cudaSetDevice(ws->device);
  cudaStreamSynchronize(ws->stream);
  cudaStreamSynchronize(ws->copy_stream);
  cudaStreamDestroy(ws->stream);
  cudaStreamDestroy(ws->copy_stream);
  for (int i = 0; i < 2; ++i) {
    if (ws->ev_res[i]) cudaEventDestroy(ws->ev_res[i]);
    if (ws->ev_copied[i]) cudaEventDestroy(ws->ev_copied[i]);
  }
  if (ws->ev_block) cudaEventDestroy(ws->ev_block);
  cudaFree(ws->arena.base);
  cudaFree(ws->scan.d_ticket);
  cudaFree(ws->scan.d_status);
  cudaFree(ws->d_flags);
  cudaFree(ws->d_small);
  cudaFree(ws->d_heavy);
  cudaFree(ws->d_heavy_count);
  cudaFreeHost(ws->h_small);
  for (int i = 0; i < 2; ++i) {
    if (ws->h_stage[i]) cudaFreeHost(ws->h_stage[i]);
    if (ws->ev_stage[i]) cudaEventDestroy(ws->ev_stage[i]);
  }
  cudaEventDestroy(ws->ev0);
  cudaEventDestroy(ws->evm);
  cudaEventDestroy(ws->eve0);
  cudaEventDestroy(ws->eve1);
  cudaEventDestroy(ws->evb0);
  cudaEventDestroy(ws->evb1);
  cudaEventDestroy(ws->ev1);
  delete ws;
}

}  // namespace gpsm
