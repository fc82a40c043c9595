// Drop-in for the reference's Match class (match/Match.h:80-125).
//
//   Match::initGPU(dev);                     // gpsm_init
//   Match m(query, data);
//   m.match(io, final_result, rows, cols, id_map);
//   ... final_result[r*cols + id_map[j]] is query vertex j of row r ...
//   delete[] final_result;                   // caller frees, as in run.cpp
//
// Unlike the reference, the data graph is uploaded once per Graph object
// (first match against it) and reused by later queries until that Graph is
// deleted or its CSR rebuilt (both drop the device copy), rows are injective
// embeddings (no homomorphism rows), and CUDA errors are reported on stderr
// with an empty result instead of exit(1). `id_map` stays owned by Match.
#pragma once
#include <cstdint>

#include "Graph.h"
#include "IO.h"

class Match {
 public:
  Match(Graph* query, Graph* data);
  ~Match();
  void match(IO& io, unsigned*& final_result, unsigned& result_row_num, unsigned& result_col_num, int*& id_map);
  static void initGPU(int dev);
  // embedding cap for later calls (0 = none); not in the reference
  static void setCap(uint64_t cap);
  // drops the device copy of a data graph now (deleting the Graph does too)
  static void releaseGraph(Graph* data);

 private:
  Graph* query;
  Graph* data;
  int* id2pos;
};
