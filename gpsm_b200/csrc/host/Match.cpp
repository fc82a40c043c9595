// Match: the reference's entry point (match/Match.h:80-125) over the C ABI.
// Error behaviour follows the reference: no device or a CUDA failure ends
// the process with exit(1) (match/Match.h:58-65, match/Match.cu:20-23); a
// query without embeddings returns final_result = NULL, rows = 0,
// cols = query size (match/Match.cu:1771-1773).
#include "gpsm_host/Match.h"

#include <climits>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <mutex>

#include "gpsm.h"

namespace {
std::mutex g_mu;
// data graphs already on the device, keyed by the Graph object; an entry
// lives exactly as long as its Graph's CSR (Graph::~Graph and
// Graph::transformToCSR drop it), so a new Graph that reuses a deleted one's
// address is uploaded afresh. Never destroyed: a Graph may die after static
// destructors have run.
std::map<const Graph*, gpsm_graph_t>& graphs() {
  static auto* m = new std::map<const Graph*, gpsm_graph_t>();
  return *m;
}
uint64_t g_cap = 0;

void die(const char* what, int rc) {
  std::cerr << "gpsm error in " << what << ": " << rc << " " << gpsm_last_error() << std::endl;
  exit(1);
}

gpsm_graph_t device_graph(Graph* data) {
  if (!data->undirected_row_offset) data->transformToCSR();
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = graphs().find(data);
  if (it != graphs().end()) return it->second;
  gpsm_graph_t h = nullptr;
  int rc = gpsm_graph_upload(data->undirected_row_offset, data->undirected_column_index, data->vertex_value,
                             data->vertex_num, &h);
  if (rc != GPSM_OK) die("gpsm_graph_upload", rc);
  graphs()[data] = h;
  return h;
}
}  // namespace

// Called by Graph::~Graph and Graph::transformToCSR: the device copy (if any)
// belongs to the CSR being dropped.
void gpsm_host_forget_graph(const Graph* g) {
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = graphs().find(g);
  if (it == graphs().end()) return;
  gpsm_graph_free(it->second);
  graphs().erase(it);
}

void Match::initGPU(int dev) {
  int rc = gpsm_init(dev);
  if (rc == GPSM_ERR_NODEV) {
    fprintf(stderr, "error: no devices supporting CUDA.\n");
    exit(EXIT_FAILURE);
  }
  if (rc != GPSM_OK) die("gpsm_init", rc);
}

void Match::setCap(uint64_t cap) { g_cap = cap; }

void Match::releaseGraph(Graph* data) { gpsm_host_forget_graph(data); }

Match::Match(Graph* q, Graph* d) : query(q), data(d), id2pos(nullptr) {}

Match::~Match() { delete[] id2pos; }

void Match::match(IO& io, unsigned*& final_result, unsigned& rows, unsigned& cols, int*& id_map) {
  (void)io;
  gpsm_graph_t g = device_graph(data);
  const unsigned qn = (unsigned)query->vertices.size();
  std::vector<uint32_t> labels(qn);
  std::vector<uint32_t> edges;
  // edges grouped by target vertex in in-list order: the engine derives the
  // reference's edge ids (match/Match.cu:1738-1754) from exactly these lists
  for (unsigned i = 0; i < qn; ++i) {
    labels[i] = (uint32_t)query->vertices[i].label;
    for (const Neighbor& nb : query->vertices[i].in) {
      edges.push_back((uint32_t)nb.vid);
      edges.push_back(i);
    }
  }
  gpsm_match_opts opts;
  memset(&opts, 0, sizeof(opts));
  opts.cap = g_cap;
  uint32_t* out = nullptr;
  delete[] id2pos;
  id2pos = new int[qn > 0 ? qn : 1];
  gpsm_match_info info;
  int rc = gpsm_match_ex(g, qn, labels.data(), (uint32_t)(edges.size() / 2), edges.empty() ? nullptr : edges.data(),
                         &opts, &out, id2pos, nullptr, &info);
  if (rc != GPSM_OK) die("gpsm_match_ex", rc);
  id_map = id2pos;
  cols = qn;
  if (info.rows == 0) {
    gpsm_free(out);
    final_result = nullptr;
    rows = 0;
    return;
  }
  if (info.rows > UINT_MAX || info.rows * qn / qn != info.rows) die("result larger than 2^32 rows", GPSM_ERR_BUDGET);
  rows = (unsigned)info.rows;
  final_result = new unsigned[(size_t)rows * qn];
  memcpy(final_result, out, (size_t)rows * qn * sizeof(unsigned));
  gpsm_free(out);
}
