// gpsm_run: the reference's command line driver (main/run.cpp:20-119) over
// the drop-in classes.  gpsm_run DATA QUERY [OUT=ans.txt] [DEV=0]
// For every data graph in DATA, every query of QUERY is matched and written
// to OUT; `match used: X ms` covers all queries of one data graph, like the
// reference. GPSM_CAP=<n> sets an embedding cap per query.
#include <chrono>
#include <cstdlib>
#include <iostream>
#include <vector>

#include "gpsm_host/Graph.h"
#include "gpsm_host/IO.h"
#include "gpsm_host/Match.h"

int main(int argc, const char* argv[]) {
  if (argc > 5 || argc < 3) {
    std::cerr << "invalid arguments!" << std::endl;
    return -1;
  }
  std::string data = argv[1], query = argv[2], output = argc >= 4 ? argv[3] : "ans.txt";
  int dev = argc == 5 ? atoi(argv[4]) : 0;
  Match::initGPU(dev);
  if (const char* c = getenv("GPSM_CAP")) Match::setCap(strtoull(c, nullptr, 10));
  auto t1 = std::chrono::steady_clock::now();
  IO io(query, data, output);
  std::vector<Graph*> query_list;
  io.input(query_list);
  std::cerr << "input ok!" << std::endl;
  auto t2 = std::chrono::steady_clock::now();
  Graph* data_graph = nullptr;
  while (io.input(data_graph)) {
    auto start = std::chrono::steady_clock::now();
    for (size_t i = 0; i < query_list.size(); ++i) {
      Match m(query_list[i], data_graph);
      io.output((int)i);
      unsigned* final_result = nullptr;
      unsigned rows = 0, cols = 0;
      int* id_map = nullptr;
      m.match(io, final_result, rows, cols, id_map);
      io.output(final_result, rows, cols, id_map, query_list[i], data_graph);
      io.flush();
      delete[] final_result;
    }
    auto end = std::chrono::steady_clock::now();
    std::cerr << "match used: " << std::chrono::duration_cast<std::chrono::milliseconds>(end - start).count() << " ms"
              << std::endl;
    Match::releaseGraph(data_graph);
    delete data_graph;
  }
  std::cerr << "match ended!" << std::endl;
  auto t3 = std::chrono::steady_clock::now();
  auto ms = [](auto a, auto b) { return (long long)std::chrono::duration_cast<std::chrono::milliseconds>(b - a).count(); };
  std::cerr << "part 1 used: " << ms(t1, t2) << "ms" << std::endl;
  std::cerr << "part 2 used: " << ms(t2, t3) << "ms" << std::endl;
  std::cerr << "total time used: " << ms(t1, t3) << "ms" << std::endl;
  for (Graph* q : query_list) delete q;
  io.flush();
  return 0;
}
