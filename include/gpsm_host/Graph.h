// Drop-in for the reference's Graph class (graph/Graph.h:20-158): the same
// public members and methods, so code written against the reference
// compiles unchanged. The CSR it builds is what gpsm_graph_upload takes.
#pragma once
#include <cstdint>
#include <vector>

typedef int LABEL;
typedef int VID;

class Neighbor {
 public:
  VID vid;
  LABEL elb;
  Neighbor() : vid(-1), elb(-1) {}
  Neighbor(int v, int e) : vid(v), elb(e) {}
  bool operator<(const Neighbor& o) const { return elb == o.elb ? vid < o.vid : elb < o.elb; }
};

class Vertex {
 public:
  LABEL label;
  std::vector<Neighbor> in;
  std::vector<Neighbor> out;
  Vertex() : label(-1) {}
  explicit Vertex(LABEL lb) : label(lb) {}
  unsigned eSize() const { return (unsigned)(in.size() + out.size()); }
};

class Graph {
 public:
  std::vector<Vertex> vertices;
  void addVertex(LABEL vlb);
  void addEdge(VID from, VID to, LABEL elb);

  unsigned vertex_num;
  unsigned* vertex_value;
  unsigned* undirected_row_offset;
  unsigned* undirected_column_index;
  unsigned label_num;
  unsigned* inverse_label;
  unsigned* inverse_num;

  Graph();
  ~Graph();
  Graph(const Graph&) = delete;
  Graph& operator=(const Graph&) = delete;

  // in- and out-lists merged into one undirected CSR, every list sorted
  // ascending; label -> count lists (graph/Graph.cpp:30-104)
  void transformToCSR();
  // directed, edge-labelled test used by IO::verify (graph/Graph.cpp:107-118)
  bool isEdgeContained(VID from, VID to, LABEL label);
  void printGraph();

  unsigned eSize() const { return undirected_row_offset[vertex_num]; }
  unsigned vSize() const { return vertex_num; }
  void getNeighbor(unsigned id, unsigned& neighbor_num, unsigned& neighbor_offset) {
    neighbor_offset = undirected_row_offset[id];
    neighbor_num = undirected_row_offset[id + 1] - neighbor_offset;
  }
  int getVertexDegree(unsigned id) { return (int)(undirected_row_offset[id + 1] - undirected_row_offset[id]); }
};
