// gpsm_select_vertices_static: the vertex-selection primitive
// (gpsm_select_vertices) for callers that must not allocate device memory.
//
// Who needs it: a host that owns all device memory (a framework's memory
// pool, or a plugin host that forbids its plugins to allocate after start-up)
// and callers that cannot accept cudaMalloc's cost at call time (it can
// synchronise the device). Such a caller passes its own input and output
// buffers; everything else this entry point touches is a fixed array
// compiled into the library.
//
// The scratch (selection bitmap, look-back scan status, ticket counter and
// error flags) is one file-scope __device__ array of kStaticScratchBytes
// (about 513 KiB). Every GPU that loads the library holds it until the
// process exits. The largest graph it serves has kStaticMaxVertices
// (2^22 = 4,194,304) vertices; larger n is rejected with GPSM_ERR_BUDGET
// before any work is queued.
//
// The array's host-side name is only a stand-in for the device copy, so host
// code never passes it to a kernel: the first call on each device looks up
// the device address with cudaGetSymbolAddress (with that device current)
// and caches it; later calls on that device reuse it. Make that first call
// before any stream capture. Every call reads the error flags back and waits
// for `stream` to finish before it returns. Every call shares the one array and it keeps
// the last call's contents, so each call rewrites the whole bitmap and
// clears the scan state and flags it needs zeroed; two calls that overlap on
// the GPU (different streams, or host threads racing) corrupt each other.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "engine.h"

namespace gpsm {
namespace {

constexpr uint32_t kStaticMaxVertices = 1u << 22;
constexpr uint32_t kStaticWords = ((kStaticMaxVertices + 31) / 32 + 3) & ~3u;  // 131072
constexpr uint32_t kStaticTiles = (kStaticWords + 1023) / 1024;                // compaction tiles: 128
constexpr size_t kBitmapOff = 0;
constexpr size_t kStatusOff = kBitmapOff + (size_t)kStaticWords * 4;
constexpr size_t kTicketOff = kStatusOff + (size_t)kStaticTiles * 8;
constexpr size_t kFlagsOff = kTicketOff + 256;
constexpr size_t kStaticScratchBytes = kFlagsOff + 256;

static __device__ __align__(256) unsigned char g_select_scratch[kStaticScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

// Device address of g_select_scratch on the current device (set-up on the
// first call per device).
int scratch_address(int dev, unsigned char** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_select_scratch);
    if (rc != cudaSuccess || p == nullptr) {
      set_last_error(std::string("gpsm_select_vertices_static: cudaGetSymbolAddress failed: ") +
                     cudaGetErrorString(rc));
      return GPSM_ERR_CUDA;
    }
    g_scratch_addr[dev] = (unsigned char*)p;
  }
  *out = g_scratch_addr[dev];
  return GPSM_OK;
}

}  // namespace
}  // namespace gpsm

using namespace gpsm;

extern "C" int gpsm_select_vertices_static(const uint32_t* d_labels, const uint32_t* d_offsets, uint32_t n,
                                           uint32_t label, uint32_t min_degree, uint32_t* d_out,
                                           uint32_t* d_count, void* stream) {
  if (!d_labels || !d_offsets || !d_out || !d_count || n == 0) {
    set_last_error("gpsm_select_vertices_static: null array or n == 0");
    return GPSM_ERR_INVALID;
  }
  if (n > kStaticMaxVertices) {
    set_last_error("gpsm_select_vertices_static: n exceeds the static scratch limit of 4194304 vertices");
    return GPSM_ERR_BUDGET;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    set_last_error("gpsm_select_vertices_static: no current CUDA device");
    return GPSM_ERR_NODEV;
  }
  unsigned char* base = nullptr;
  int rc = scratch_address(dev, &base);
  if (rc != GPSM_OK) return rc;
  try {
    Workspace ws;  // views of the static scratch only; owns nothing
    ws.device = dev;
    ws.stream = (cudaStream_t)stream;
    ws.scan.d_status = (unsigned long long*)(base + kStatusOff);
    ws.scan.d_ticket = (unsigned long long*)(base + kTicketOff);
    ws.scan.max_tiles = kStaticTiles;
    ws.scan.ticket_base = 0;
    ws.scan.epoch = 0;
    ws.d_flags = (uint32_t*)(base + kFlagsOff);
    // the bitmap is rewritten in full by the selection kernel; the scan state
    // and flags must start at zero
    GPSM_CUDA(cudaMemsetAsync(base + kStatusOff, 0, kFlagsOff + 256 - kStatusOff, ws.stream));
    select_vertices(ws, d_labels, d_offsets, n, label, min_degree, (uint32_t*)(base + kBitmapOff), d_out, d_count);
    uint32_t flags = 0;
    GPSM_CUDA(cudaMemcpyAsync(&flags, ws.d_flags, sizeof(flags), cudaMemcpyDeviceToHost, ws.stream));
    GPSM_CUDA(cudaStreamSynchronize(ws.stream));
    if (flags & (DF_SCAN_TIMEOUT | DF_BOUNDS)) {
      set_last_error("gpsm_select_vertices_static: device wait limit or bounds check tripped");
      return GPSM_ERR_TIMEOUT;
    }
  } catch (const CudaError& e) {
    return e.err == cudaErrorInvalidValue ? GPSM_ERR_INVALID : GPSM_ERR_CUDA;
  } catch (const std::bad_alloc&) {  // nothing may cross the C boundary
    set_last_error("gpsm_select_vertices_static: host allocation failed");
    return GPSM_ERR_NOMEM;
  } catch (...) {
    set_last_error("gpsm_select_vertices_static: unexpected exception");
    return GPSM_ERR_STATE;
  }
  return GPSM_OK;
}
