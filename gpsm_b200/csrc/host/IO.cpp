// IO: the reference's text format and output (io/IO.cpp), written for this
// library. Format: `t # <id>` then a line of four counts (ignored), `v <id>
// <label>` per vertex in id order, `e <from> <to> <label>` per edge; a file
// ends with `t # -1`. Unlike the reference reader, end of file without
// `t # -1` ends the input instead of looping forever.
#include "gpsm_host/IO.h"

#include <chrono>
#include <cstring>
#include <iostream>
#include <set>

IO::IO() : data_id(-1), qfp(nullptr), dfp(nullptr), ofp(nullptr) {}

IO::IO(std::string query, std::string data, std::string file)
    : line("============================================================"), data_id(-1), qfp(nullptr), dfp(nullptr),
      ofp(nullptr) {
  qfp = fopen(query.c_str(), "r");
  if (!qfp) {
    std::cerr << "input open error!" << std::endl;
    return;
  }
  dfp = fopen(data.c_str(), "r");
  if (!dfp) {
    std::cerr << "input open error!" << std::endl;
    return;
  }
  ofp = fopen(file.c_str(), "w+");
  if (!ofp) std::cerr << "output open error!" << std::endl;
}

Graph* IO::input(FILE* fp) {
  if (!fp) return nullptr;
  Graph* g = nullptr;
  for (;;) {
    int c = fgetc(fp);
    if (c == EOF) return g;
    if (c == ' ' || c == '\n' || c == '\r' || c == '\t') continue;
    if (c == 't') {
      if (g) {  // next graph starts: leave its header for the next call
        ungetc(c, fp);
        return g;
      }
      char hash;
      int id;
      if (fscanf(fp, " %c %d", &hash, &id) != 2) return nullptr;
      if (id == -1) return nullptr;
      g = new Graph;
      int nv, ne, nvl, nel;
      if (fscanf(fp, " %d %d %d %d", &nv, &ne, &nvl, &nel) != 4) {
        delete g;
        return nullptr;
      }
    } else if (c == 'v') {
      int id, lb;
      if (!g || fscanf(fp, " %d %d", &id, &lb) != 2) {
        std::cerr << "ERROR in input() -- bad vertex line" << std::endl;
        delete g;
        return nullptr;
      }
      g->addVertex(lb);
    } else if (c == 'e') {
      int a, b, lb;
      if (!g || fscanf(fp, " %d %d %d", &a, &b, &lb) != 3 || a < 0 || b < 0 ||
          a >= (int)g->vertices.size() || b >= (int)g->vertices.size()) {
        std::cerr << "ERROR in input() -- bad edge line" << std::endl;
        delete g;
        return nullptr;
      }
      g->addEdge(a, b, lb);
    } else {
      std::cerr << "ERROR in input() -- invalid char" << std::endl;
      delete g;
      return nullptr;
    }
  }
}

bool IO::input(Graph*& data_graph) {
  data_graph = input(dfp);
  if (!data_graph) return false;
  ++data_id;
  data_graph->transformToCSR();
  return true;
}

bool IO::input(std::vector<Graph*>& query_list) {
  for (;;) {
    Graph* g = input(qfp);
    if (!g) break;
    g->transformToCSR();
    query_list.push_back(g);
  }
  return true;
}

bool IO::output(int qid) {
  fprintf(ofp, "query graph:%d    data graph:%d\n", qid, data_id);
  fprintf(ofp, "%s\n", line.c_str());
  return true;
}

bool IO::output() {
  fprintf(ofp, "\n\n\n");
  return true;
}

// injective, and every query in-edge (src -> i, label) exists as a data
// out-edge ans[src] -> ans[i] with that label (io/IO.cpp:146-180)
bool IO::verify(int* id_map, unsigned* ans, unsigned num, Graph* query, Graph* data) {
  std::set<unsigned> seen;
  for (unsigned i = 0; i < num; ++i)
    if (!seen.insert(ans[i]).second) return false;
  std::vector<Vertex>& qv = query->vertices;
  for (size_t i = 0; i < qv.size(); ++i)
    for (const Neighbor& nb : qv[i].in) {
      int to = (int)ans[id_map[i]];
      int from = (int)ans[id_map[nb.vid]];
      if (!data->isEdgeContained(from, to, nb.elb)) return false;
    }
  return true;
}

bool IO::output(unsigned* final_result, unsigned rows, unsigned cols, int* id_map, Graph* query, Graph* data) {
  auto t0 = std::chrono::steady_clock::now();
  for (unsigned i = 0; i < rows; ++i) {
    unsigned* ans = final_result + (size_t)i * cols;
    if (!verify(id_map, ans, cols, query, data)) continue;
    for (unsigned j = 0; j < cols; ++j) fprintf(ofp, "(%u, %u) ", j, ans[id_map[j]]);
    fprintf(ofp, "\n");
  }
  fprintf(ofp, "\n\n\n");
  auto t1 = std::chrono::steady_clock::now();
  std::cout << "output used " << std::chrono::duration_cast<std::chrono::milliseconds>(t1 - t0).count() << " ms"
            << std::endl;
  return true;
}

bool IO::output(int* m, int size) {
  for (int i = 0; i < size; ++i) fprintf(ofp, "(%d, %d) ", i, m[i]);
  fprintf(ofp, "\n");
  return true;
}

void IO::flush() {
  if (ofp) fflush(ofp);
}

IO::~IO() {
  if (qfp) fclose(qfp);
  if (dfp) fclose(dfp);
  if (ofp) fclose(ofp);
}
