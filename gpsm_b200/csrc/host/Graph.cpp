// Graph: the reference's in-memory graph model (graph/Graph.cpp), written
// for this library. Semantics kept exactly: addEdge appends to the source's
// out-list and the target's in-list; transformToCSR concatenates in- then
// out-neighbours per vertex and sorts each list ascending (parallel edges
// and A->B plus B->A stay as repeated entries, as in the reference); the
// inverse label list counts vertices per label in ascending label order.
#include "gpsm_host/Graph.h"

#include <algorithm>
#include <cstdio>

// Drops the device copy the drop-in Match uploaded for this graph (host/Match.cpp).
void gpsm_host_forget_graph(const Graph* g);

void Graph::addVertex(LABEL vlb) { vertices.push_back(Vertex(vlb)); }

void Graph::addEdge(VID from, VID to, LABEL elb) {
  vertices[from].out.push_back(Neighbor(to, elb));
  vertices[to].in.push_back(Neighbor(from, elb));
}

Graph::Graph()
    : vertex_num(0), vertex_value(nullptr), undirected_row_offset(nullptr), undirected_column_index(nullptr),
      label_num(0), inverse_label(nullptr), inverse_num(nullptr) {}

Graph::~Graph() {
  // the reference's driver deletes each data graph (main/run.cpp:97) and the
  // next one may be allocated at the same address
  gpsm_host_forget_graph(this);
  delete[] vertex_value;
  delete[] undirected_row_offset;
  delete[] undirected_column_index;
  delete[] inverse_label;
  delete[] inverse_num;
}

void Graph::transformToCSR() {
  gpsm_host_forget_graph(this);  // a device copy of the old CSR is stale
  delete[] vertex_value;
  delete[] undirected_row_offset;
  delete[] undirected_column_index;
  delete[] inverse_label;
  delete[] inverse_num;
  vertex_num = (unsigned)vertices.size();
  vertex_value = new unsigned[vertex_num > 0 ? vertex_num : 1];
  undirected_row_offset = new unsigned[vertex_num + 1];
  undirected_row_offset[0] = 0;
  for (unsigned i = 0; i < vertex_num; ++i) {
    vertex_value[i] = (unsigned)vertices[i].label;
    undirected_row_offset[i + 1] = undirected_row_offset[i] + vertices[i].eSize();
  }
  const unsigned nnz = undirected_row_offset[vertex_num];
  undirected_column_index = new unsigned[nnz > 0 ? nnz : 1];
  for (unsigned i = 0; i < vertex_num; ++i) {
    unsigned p = undirected_row_offset[i];
    for (const Neighbor& nb : vertices[i].in) undirected_column_index[p++] = (unsigned)nb.vid;
    for (const Neighbor& nb : vertices[i].out) undirected_column_index[p++] = (unsigned)nb.vid;
    std::sort(undirected_column_index + undirected_row_offset[i], undirected_column_index + p);
  }
  std::vector<unsigned> labs(vertex_value, vertex_value + vertex_num);
  std::sort(labs.begin(), labs.end());
  std::vector<unsigned> lab, cnt;
  for (unsigned i = 0; i < vertex_num; ++i) {
    if (i == 0 || labs[i] != labs[i - 1]) {
      lab.push_back(labs[i]);
      cnt.push_back(0);
    }
    cnt.back()++;
  }
  label_num = (unsigned)lab.size();
  inverse_label = new unsigned[label_num > 0 ? label_num : 1];
  inverse_num = new unsigned[label_num + 1];
  for (unsigned k = 0; k < label_num; ++k) {
    inverse_label[k] = lab[k];
    inverse_num[k] = cnt[k];
  }
  inverse_num[label_num] = 0;
}

bool Graph::isEdgeContained(VID from, VID to, LABEL label) {
  for (const Neighbor& nb : vertices[from].out)
    if (nb.vid == to && nb.elb == label) return true;
  return false;
}

void Graph::printGraph() {
  printf("vertex value:\n");
  for (unsigned i = 0; i < vertex_num; ++i) printf("%u ", vertex_value[i]);
  printf("\nrow offset:\n");
  for (unsigned i = 0; i <= vertex_num; ++i) printf("%u ", undirected_row_offset[i]);
  printf("\ncolumn index in:\n");
  for (unsigned i = 0; i < eSize(); ++i) printf("%u ", undirected_column_index[i]);
  printf("\n");
}
