// Opaque handle types of the C ABI (shared by capi.cpp and batch.cpp).
#pragma once
#include <mutex>
#include <vector>

#include "engine.h"

struct gpsm_graph_s {
  gpsm::DeviceGraph* g;
};

struct gpsm_model_s {
  gpsm::Model* m;
};

struct gpsm_engine_s {
  gpsm::Workspace* ws = nullptr;
  std::mutex mu;
  gpsm::QueryPlan last_plan;
  gpsm::MatchResult last;  // statistics of the last match (gpsm_last_levels)
  std::vector<uint32_t*> last_lists;
};

namespace gpsm {
// options shared by every entry point that takes gpsm_match_opts
MatchOptions options_from(const struct gpsm_match_opts* o);
int error_from(const CudaError& e);
}  // namespace gpsm
