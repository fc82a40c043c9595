// Drop-in for the reference's IO class (io/IO.h:15-39): the `t`/`v`/`e`
// text format (0-based vertex ids, 1-based labels, files end with `t # -1`),
// per-query headers and the `(j, k) ` embedding lines after the host-side
// directed, edge-labelled verification.
#pragma once
#include <cstdio>
#include <string>
#include <vector>

#include "Graph.h"

class IO {
 public:
  IO();
  IO(std::string query, std::string data, std::string file);
  bool input(std::vector<Graph*>& query_list);
  bool input(Graph*& data_graph);
  Graph* input(FILE* fp);
  bool output(int qid);
  bool output();
  bool output(unsigned* final_result, unsigned result_row_num, unsigned result_col_num, int* id_map,
              Graph* query_graph, Graph* data_graph);
  bool output(int* m, int size);
  void flush();
  ~IO();

 private:
  std::string line;
  int data_id;
  FILE* qfp;
  FILE* dfp;
  FILE* ofp;
  bool verify(int* id_map, unsigned* ans, unsigned num, Graph* query_graph, Graph* data_graph);
};
